"""GPU test of nrrs_decide_emit_noalloc, the decision + emission entry point that allocates no
device memory (for callers that cannot call cudaMalloc: plugins whose host framework owns all
device memory, fixed start-up memory budgets, frame loops that must not synchronise).

Its results must equal those of nrrs_decide_emit on a context whose max_queue is
NRRS_NOALLOC_MAX_N (same exact-sum shift), bit for bit, on calls in a row: a call at the full
NRRS_NOALLOC_MAX_N followed by smaller ones checks that the look-back states and sums left in the
static scratch by an earlier, larger call do not leak into a later result. A too-small next
queue and non-finite factors must give the same clipped queue, required size and status bits
(read with nrrs_noalloc_device_status) as the context path. This file is collected last so a
failure here cannot hide the other tests' results."""
from __future__ import annotations

import numpy as np
import pytest

import nrrs_b200 as nb
from gpu_util import empty, host, make_net, stream, torch_cuda

pytestmark = pytest.mark.gpu


def _inputs(seed, n):
    rng = np.random.default_rng(seed)
    rrs = np.clip(rng.lognormal(-0.2, 1.1, n), 0.05, 8).astype(np.float32)
    rnd = rng.random(n, dtype=np.float32)
    return rrs, rnd


def _outputs(n, cap):
    return dict(norm=empty(n), split=empty(n, "uint8"), q=empty(cap, "int32"), sz=empty(1, "int32"))


def _host(o, n, cap):
    tot = int(host(o["sz"], np.uint32)[0])
    k = min(tot, cap)
    return {"total": tot, "queue": host(o["q"], np.uint32)[:k].copy(),
            "split": host(o["split"])[:n].copy(), "norm": host(o["norm"])[:n].view(np.uint32).copy()}


def _both(net, rrs, rnd, n, budget, nspec, dp, cap, s):
    torch = torch_cuda()
    d_rrs, d_rnd = torch.from_numpy(rrs).cuda(), torch.from_numpy(rnd).cuda()
    ref, got = _outputs(n, cap), _outputs(n, cap)
    net.decideEmit(d_rrs, d_rnd, n, budget, nspec, dp, ref["norm"], ref["split"], ref["q"], cap,
                   ref["sz"], stream=s)
    rc = nb.decide_emit_noalloc(d_rrs, d_rnd, n, budget, nspec, dp, got["norm"], got["split"],
                                got["q"], cap, got["sz"], stream=s)
    assert rc == nb.OK, rc
    torch.cuda.synchronize()
    return _host(ref, n, cap), _host(got, n, cap)


def _same(a, b, what):
    assert a["total"] == b["total"], what
    for k in ("queue", "split", "norm"):
        assert np.array_equal(a[k], b[k]), (what, k)


def test_noalloc_matches_context_entry_point_on_calls_in_a_row():
    net = make_net(max_queue=nb.NOALLOC_MAX_N, max_train=1024)
    s = stream()
    nb.noalloc_device_status(s)  # start from clear status bits
    calls = [(10, nb.NOALLOC_MAX_N, 1), (11, 300_007, 0), (12, 1_000_003, 1)]
    for call, (seed, n, use_ceil) in enumerate(calls):
        rrs, rnd = _inputs(seed, n)
        dp = nb.default_decide(use_ceil=use_ceil)
        a, b = _both(net, rrs, rnd, n, n, n // 40, dp, 9 * n, s)
        assert a["total"] > 0, call
        _same(a, b, call)
    assert nb.noalloc_device_status(s) == (nb.OK, 0)
    assert net.device_status(s) == (nb.OK, 0)
    net.close()


def test_noalloc_small_capacity_and_nan_match_context_status():
    net = make_net(max_queue=nb.NOALLOC_MAX_N, max_train=1024)
    s = stream()
    nb.noalloc_device_status(s)
    net.device_status(s)
    n = 500_001
    rrs, rnd = _inputs(13, n)
    dp = nb.default_decide()
    # next queue far below the total: the same clipped prefix and the same required size
    cap = n // 3
    a, b = _both(net, rrs, rnd, n, n, 0, dp, cap, s)
    assert a["total"] > cap
    _same(a, b, "capacity")
    rc_ctx, f_ctx = net.device_status(s)
    rc_na, f_na = nb.noalloc_device_status(s)
    assert f_ctx == f_na and (f_na & nb.DEV_OVERFLOW), (f_ctx, f_na)
    assert rc_ctx == rc_na == nb.ERR_CAPACITY_OVERFLOW
    # non-finite factors: dropped from the sum, split 0, flagged
    rrs2 = rrs.copy()
    rrs2[[5, 77_777, n - 1]] = np.nan
    a, b = _both(net, rrs2, rnd, n, n, 0, dp, 9 * n, s)
    _same(a, b, "nan")
    assert b["split"][5] == 0 and b["split"][n - 1] == 0
    rc_ctx, f_ctx = net.device_status(s)
    rc_na, f_na = nb.noalloc_device_status(s)
    assert f_ctx == f_na and (f_na & nb.DEV_NAN), (f_ctx, f_na)
    assert rc_ctx == rc_na == nb.ERR_NAN
    assert nb.noalloc_device_status(s) == (nb.OK, 0)
    net.close()


def test_noalloc_rejects_oversize_and_handles_empty():
    torch = torch_cuda()
    dp = nb.default_decide()
    o = _outputs(1, 1)
    rc = nb.decide_emit_noalloc(empty(1), empty(1), nb.NOALLOC_MAX_N + 1, 10, 0, dp, o["norm"],
                                o["split"], o["q"], 1, o["sz"], stream=stream())
    assert rc == nb.ERR_INVALID_ARG
    o["sz"].fill_(7)
    rc = nb.decide_emit_noalloc(empty(1), empty(1), 0, 10, 0, dp, o["norm"], o["split"], o["q"],
                                1, o["sz"], stream=stream())
    torch.cuda.synchronize()
    assert rc == nb.OK and int(host(o["sz"], np.uint32)[0]) == 0
