"""CPU tests of the path-record oracle (oracle/records.c): pinned to the hand-derived trees of
tests/golden/records_cases.json, its fixed-point conversion checked against gcc's correctly
rounded __int128 -> float, and its host logic (node numbering, order independence) checked on
synthetic frames."""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import pytest

import nrrs_b200 as nb
import oracle as O

GOLD = Path(__file__).resolve().parent / "golden"
CASES = json.loads((GOLD / "records_cases.json").read_text())


def bounce_arrays(b: dict) -> dict:
    """A golden bounce as the numpy arrays the oracle and the library take."""
    f = lambda k, dt: np.ascontiguousarray(np.array(b[k], dt))  # noqa: E731
    return {"pos": f("pos", np.float32), "wi": f("wi", np.float32),
            "roughness": f("roughness", np.float32), "thp": f("thp", np.float32),
            "depth": f("depth", np.uint32), "pixel": f("pixel", np.uint32),
            "rrs": f("rrs", np.float32), "record": f("record", np.uint8),
            "parent": f("parent", np.int32), "contrib_node": f("contrib_node", np.int32),
            "contrib": np.array(b["contrib"], np.float32).reshape(-1, 3)}


def check_against_expect(case, node_outs, size, dropped, batch, total, counts, weights):
    e = case["expect"]
    assert size == e["size"] and dropped == e["dropped"]
    for got, want in zip(node_outs, e["node_outs"]):
        assert list(got) == want
    assert total == len(e["batch"])
    for t, row in enumerate(e["batch"]):
        assert batch["target"][t].tolist() == [np.float32(x) for x in row["target"]], (t, row)
        assert batch["thp"][t].tolist() == [np.float32(x) for x in row["thp"]], (t, row)
        assert batch["rrs_target"][t] == np.float32(row["rrs_target"])
        assert batch["pixel"][t] == row["pixel"]
        assert batch["ref_mean"][t] == np.float32(row["ref_mean"])
    assert list(counts) == e["counts"]
    assert [np.float32(x) for x in e["weights"]] == list(weights)


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_matches_golden_trees(case):
    hn = O.HostNodes(case["capacity"])
    outs = []
    for b in case["bounces"]:
        a = bounce_arrays(b)
        outs.append(hn.record_nodes(a))
        hn.record_radiance(a["contrib_node"], a["contrib"])
    image = np.array(case["image"], np.float32)
    counts = np.zeros(len(image), np.uint32)
    prm = nb.TrainDataParams(**case["params"])
    batch, total = hn.generate(prm, 64, image=image, n_pixels=len(image), pixel_samples=counts)
    w = O.sample_weights(batch["pixel"], counts, len(image))
    check_against_expect(case, outs, hn.size, hn.dropped, batch, total, counts, w)
    if case["capacity"] > 5:
        assert hn.status == nb.DEV_NAN      # the NaN contribution is reported
    else:                                   # node 5 was refused: its NaN never lands
        assert hn.status == nb.DEV_OVERFLOW
    # the batch carries the recorded fields of the kept nodes, in node order
    kept = [r["node"] for r in case["expect"]["batch"]]
    assert np.array_equal(batch["pos"], hn.a["pos"][kept])
    assert np.array_equal(batch["depth"], hn.a["depth"][kept])


def test_fixed_point_conversion_matches_gcc_rounding():
    rng = np.random.default_rng(5)
    cases = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, 0, 1), (0, 0, -1),
             (2**32 - 1, 2**32 - 1, 2**40), (2**62, 2**62, 2**61), (-(2**62), 5, -(2**40)),
             # exact ties at bit 24 below the leading bit, both parities
             (0, 0, (1 << 24) + 1), (0, 1 << 31, (1 << 24) + 1), (0, 1 << 31, 1 << 24),
             (1 << 31, (1 << 32) - 1, (1 << 23) - 1)]
    for _ in range(20000):
        l = [int(x) for x in rng.integers(-(2**62), 2**62, size=3)]
        sh = int(rng.integers(0, 62))
        cases.append((l[0] >> sh, l[1] >> int(rng.integers(0, 62)), l[2] >> int(rng.integers(0, 62))))
    for l0, l1, l2 in cases:
        a = O.fixed_to_float(l0, l1, l2)
        g = O.fixed_to_float(l0, l1, l2, gcc=True)
        f = O.fixed_to_float(l0, l1, l2, fast=True)
        assert np.float32(a).tobytes() == np.float32(g).tobytes(), (l0, l1, l2, a, g)
        assert np.float32(a).tobytes() == np.float32(f).tobytes(), (l0, l1, l2, a, f)


def test_fixed_point_round_trip_and_truncation():
    rng = np.random.default_rng(6)
    # mantissa in [1, 2), exponent >= -41: the lowest mantissa bit is worth >= 2^-64
    mant = rng.uniform(1, 2, 4000) * rng.choice([-1.0, 1.0], 4000)
    xs = np.concatenate([mant * np.exp2(rng.integers(-41, 61, 4000)),
                         [0.0, -0.0, 1.0, 0.75, 2.0**61, -(2.0**61), 2.0**-41]]).astype(np.float32)
    for x in xs:   # every bit of x is at or above 2^-64: exact
        assert np.float32(O.fixed_to_float(*O.fixed_limbs(float(x)))) == x
        l0, l1, l2 = O.fixed_limbs(float(x))
        assert 0 <= abs(l0) < 2**32 and 0 <= abs(l1) < 2**32
    tiny = np.float32(3e-20)  # 0.55 of the lowest bit: truncated to 0
    assert O.fixed_limbs(float(tiny)) == (0, 0, 0)
    x = np.float32(1e-15)     # bits below 2^-64 are dropped, toward zero
    v = O.fixed_to_float(*O.fixed_limbs(float(x)))
    assert 0 < x - v < 2.0**-64


def test_oracle_radiance_is_independent_of_contribution_order():
    bounces, image = nb.synth_paths(11, 3000, bounces=6, capacity=12000)
    runs = []
    for perm_seed in (None, 1, 2):
        hn = O.HostNodes(12000)
        for b in bounces:
            hn.record_nodes(b)
        rng = np.random.default_rng(perm_seed)
        node = np.concatenate([b["contrib_node"] for b in bounces])
        contrib = np.concatenate([b["contrib"] for b in bounces])
        if perm_seed is not None:
            p = rng.permutation(len(node))
            node, contrib = node[p], contrib[p]
        hn.record_radiance(node, contrib)
        runs.append(hn.a["radiance"].copy())
    assert np.array_equal(runs[0], runs[1]) and np.array_equal(runs[0], runs[2])


def test_oracle_frame_follows_generator_numbering():
    bounces, image = nb.synth_paths(12, 5000, capacity=20000)
    r = O.frame_training_data(bounces, image, 20000,
                              nb.default_train_data_params(ignore_zero_l=1, dedupe_rrs_target=1))
    for b, no in zip(bounces, r["node_outs"]):
        assert np.array_equal(b["node"], no)
    hn = r["nodes"]
    assert hn.size == sum(int(b["record"].sum()) for b in bounces) and hn.dropped == 0
    assert hn.status == 0
    # every kept sample has a finite, non-negative, non-zero target (zero-L filter)
    t = r["batch"]["target"]
    assert np.isfinite(t).all() and (t >= 0).all() and (t.mean(axis=1) > 0).all()
    # counts add up to the samples that kept their RRSNet target
    assert r["counts"].sum() == (r["batch"]["rrs_target"] >= 0).sum()
    w = r["weights"]
    px = r["batch"]["pixel"]
    assert np.array_equal(w, np.where(r["counts"][px] > 0,
                                      (np.float32(1) / r["counts"][px].astype(np.float32)), 0))


def test_oracle_capacity_overflow_falls_back_to_parent():
    bounces, image = nb.synth_paths(13, 2000, bounces=5, capacity=3000)
    hn = O.HostNodes(3000)
    for b in bounces:
        out = hn.record_nodes(b)
        assert np.array_equal(out, b["node"])
    assert hn.size == 3000
    want = sum(int(b["record"].sum()) for b in bounces) - 3000
    assert hn.dropped == want > 0 and hn.status & nb.DEV_OVERFLOW
    # a batch capacity below the sample count keeps the first samples and flags overflow
    hn.header[4] = 0
    batch, total = hn.generate(nb.default_train_data_params(), 100)
    assert total > 100 and len(batch["target"]) == 100 and hn.status & nb.DEV_OVERFLOW
    full, total2 = hn.generate(nb.default_train_data_params(), total)
    assert total2 == total
    assert np.array_equal(full["target"][:100], batch["target"])


def test_sample_weight_matches_reference_formula():
    px = np.array([0, 1, 2, 2, 5], np.uint32)
    counts = np.array([1, 3, 0, 7], np.uint32)
    w = O.sample_weights(px, counts, 4)
    assert w.tolist() == [1.0, np.float32(1) / np.float32(3), 0.0, 0.0, 0.0]
    assert math.isclose(w[1], 1 / 3, rel_tol=1e-7)


def test_parent_recorded_in_the_same_call_is_cut():
    """Parents must be nodes of earlier record calls; a link to a node of the same call (or to no
    node yet) is stored as -1 and flagged, so node trees stay levelled by call."""
    hn = O.HostNodes(16)
    b = dict(pos=np.zeros((3, 3), np.float32), wi=np.ones((3, 3), np.float32),
             thp=np.ones((3, 3), np.float32), pixel=np.zeros(3, np.uint32),
             parent=np.array([-1, 0, 7], np.int32))
    out = hn.record_nodes(b)
    assert out.tolist() == [0, 1, 2]
    assert hn.a["parent"][:3].tolist() == [-1, -1, -1]
    assert hn.status == nb.DEV_BAD_INDEX
    assert hn.a["children"][:3].tolist() == [0, 0, 0]
    b2 = dict(b, parent=np.array([2, 4, 1], np.int32))   # 2 and 1: earlier call; 4: this call
    out = hn.record_nodes(b2)
    assert out.tolist() == [3, 4, 5]
    assert hn.a["parent"][3:6].tolist() == [2, -1, 1]
    assert hn.a["first_child"][:3].tolist() == [0xffffffff, 5, 3]


def split_calls(bounces, parts: int):
    """Each bounce recorded in `parts` consecutive slices (more record calls, same nodes)."""
    out = []
    for b in bounces:
        n = len(b["pixel"])
        cuts = np.linspace(0, n, parts + 1).astype(int)
        node_keys = ("pos", "wi", "normal", "albedo", "roughness", "thp", "depth", "pixel", "rrs",
                     "record", "parent", "node")
        for k in range(parts):
            s = {key: np.ascontiguousarray(b[key][cuts[k]:cuts[k + 1]]) for key in node_keys}
            s["contrib_node"] = b["contrib_node"] if k == parts - 1 else b["contrib_node"][:0]
            s["contrib"] = b["contrib"] if k == parts - 1 else b["contrib"][:0]
            out.append(s)
    return out


def test_oracle_split_calls_give_the_same_frame():
    bounces, image = nb.synth_paths(14, 3000, capacity=12000)
    prm = nb.default_train_data_params(dedupe_rrs_target=1)
    a = O.frame_training_data(bounces, image, 12000, prm)
    b = O.frame_training_data(split_calls(bounces, 9), image, 12000, prm)
    for k in a["batch"]:
        assert a["batch"][k].tobytes() == b["batch"][k].tobytes()
    assert a["nodes"].status == b["nodes"].status == 0
