"""CPU tests of the host-side path control: the per-depth strategy search (nrrs_ubs_*) and the
training schedule (nrrs_train_schedule_*) against the restatement in oracle/schedule.py, frame by
frame, plus known answers: the search finds the strategy string that it is made to prefer."""
from __future__ import annotations

import numpy as np
import pytest

import nrrs_b200 as nb
from schedule import ScheduleRef, UBSRef


def run_search(max_depth: int, score, res=1920 * 1080, frames_cap=5000):
    """Drive the library and the restatement through a whole search as the reference's render
    loop does: next state at the start of a frame, the strategies used in it, the frame's time
    and error at its end. score(state_digits) -> (seconds, error sum) of a frame."""
    lib, ref = nb.UBS(max_depth), UBSRef(max_depth)
    lib.UBSResetAndBeginSearch()
    ref.begin()
    t = 0.0
    frames = 0
    while True:
        a, b = lib.UBSNextState(), ref.next_state()
        assert a == b
        if not a:
            break
        digits = tuple(lib.strategy(d) for d in range(max_depth))
        assert digits == tuple(ref.strategy(d) for d in range(max_depth))
        for d in range(max_depth + 2):
            assert lib.isInferMode(d) == ref.need_infer(d, 1, 0.05, 8.0, 6, 1)
        dt, err = score(digits)
        t += dt
        lib.UBSAnalyseFrame(t, err, res)
        ref.analyse(t, err, res)
        frames += 1
        assert frames < frames_cap
    best, eff = lib.best()
    assert best == ref.array[:max_depth] and np.float32(eff) == ref.best_eff
    return lib, ref, best, frames


@pytest.mark.parametrize("max_depth", [1, 2, 4])
def test_search_finds_the_preferred_strategy(max_depth):
    target = tuple([2, 1, 0, 2][:max_depth])

    def score(digits):   # the target is the fastest with the smallest error
        miss = sum(a != b for a, b in zip(digits, target))
        return 1 / 60 + 1e-3 * miss, 100.0 + 50.0 * miss

    lib, _, best, frames = run_search(max_depth, score)
    assert tuple(best) == target
    assert not lib.searching
    # every state once; the reference restarts the search on its first two frames (the timer,
    # then the first attempt) and plays one frame more to score the last state
    assert frames == 3 ** max_depth + 3
    # the best strategy is not applied until asked for (UBSEndSearch leaves mUseBestStrategy)
    assert lib.strategy(0) == -1
    lib.set_best("".join(map(str, best)))
    assert [lib.strategy(d) for d in range(max_depth)] == list(target)
    for d in range(max_depth):
        infer, src = lib.isInferMode(d)
        assert infer == (target[d] != 0)
        assert src == (nb.FACTOR_RRSNET if target[d] == 2 else nb.FACTOR_ADRRS)


@pytest.mark.parametrize("max_depth", [3, 6, 7])
def test_search_matches_restatement_on_random_frames(max_depth):
    rng = np.random.default_rng(max_depth)
    table = {}

    def score(digits):
        if digits not in table:
            table[digits] = (float(rng.uniform(0.01, 0.03)), float(rng.uniform(10, 1000)))
        return table[digits]

    run_search(max_depth, score, frames_cap=4000)


def test_set_best_digits_and_defaults():
    u, r = nb.UBS(5), UBSRef(5)
    assert u.strategy(0) == -1
    assert u.isInferMode(3, use_net_output_rrs=False) == (True, nb.FACTOR_ADRRS)
    assert u.isInferMode(7, max_rrs_depth=6) == (False, nb.FACTOR_RRSNET)   # beyond the depth cap
    assert u.isInferMode(0, clamp_min=8.0, clamp_max=8.0)[0] is False        # no clamp range
    u.set_best("2x1")       # non-digits and missing depths are fixed RR
    r.set_best("2x1")
    assert [u.strategy(d) for d in range(7)] == [2, 0, 1, 0, 0, 0, 0]
    for d in range(7):
        assert u.isInferMode(d) == r.need_infer(d, 1, 0.05, 8.0, 6, 1)


def test_train_schedule_matches_restatement():
    durations = [2.0, 0.0, 3.0, 1.5]       # a zero-length state passes in the same tick
    lib, ref = nb.TrainSchedule(durations), ScheduleRef(durations)
    t, steps = 0.0, []
    for frame in range(2000):
        t += 1 / 60
        a = lib.tick(t, 1000.0 + t)
        b = ref.tick(t, 1000.0 + t)
        got = {k: getattr(a, k) for k in b}
        assert got == b, (frame, got, b)
        steps.append(a.step)
        if a.request_exit:
            break
    assert a.request_exit and a.state == 4 and a.stop_training
    assert a.seconds_per_frame == pytest.approx(1 / 60)
    # 0 until 2 s, then 1 and at once 2 (state 1 lasts 0 s), then 3 after 5 s
    assert steps[0] == 0 and 2 in steps and 3 in steps and 1 not in steps


def test_bad_arguments():
    with pytest.raises(nb.NRRSError):
        nb.UBS(0)
    with pytest.raises(nb.NRRSError):
        nb.UBS(20)
    with pytest.raises(nb.NRRSError):
        nb.TrainSchedule([1.0, -1.0, 1.0, 1.0])
