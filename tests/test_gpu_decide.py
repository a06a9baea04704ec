"""GPU parity of the decision + emission kernels against the oracle: split counts, the compacted
queue and the normalised factors are compared bit for bit (integrator.cpp:1368-1460)."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

import nrrs_b200 as nb
import oracle as O
from gpu_util import empty, host, make_net, stream, torch_cuda

pytestmark = pytest.mark.gpu
MAXQ = 1 << 21  # max_queue of make_net(): fixes the exact sum's shift
GOLD = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def net():
    n = make_net()
    yield n
    n.close()


def run_decide(net, rrs, rnd, budget, nspec, dp, capacity=None, sidx=None):
    torch = torch_cuda()
    n = rrs.size
    cap = capacity if capacity is not None else int(n * (dp.clamp_max + 2)) + 8
    d_rrs = torch.from_numpy(rrs.astype(np.float32)).cuda() if n else empty(1)
    d_rnd = torch.from_numpy(rnd.astype(np.float32)).cuda() if n else empty(1)
    nst = int(sidx.max()) + 1 if sidx is not None and n else max(n, 1)
    d_sidx = torch.from_numpy(sidx.astype(np.uint32).view(np.int32)).cuda() if sidx is not None else None
    d_norm = empty(nst)
    d_split = empty(n, "uint8")
    d_queue = empty(cap, "int32")
    d_size = empty(1, "int32")
    net.decideEmit(d_rrs, d_rnd, n, budget, nspec, dp, d_norm, d_split, d_queue, cap, d_size,
                   scatter_index=d_sidx, stream=stream())
    rc, flags = net.device_status(stream())
    total = int(host(d_size, np.uint32)[0])
    return {"queue": host(d_queue, np.uint32)[:min(total, cap)], "total": total,
            "split": host(d_split)[:n], "rrs_norm": host(d_norm)[:nst], "flags": flags, "rc": rc}


def compare(g, o):
    assert g["total"] == o["total"]
    assert np.array_equal(g["split"], o["split"])
    assert np.array_equal(g["queue"], o["queue"])
    assert np.array_equal(g["rrs_norm"].view(np.uint32), o["rrs_norm"].view(np.uint32))


@pytest.mark.parametrize("case", json.loads((GOLD / "decide_cases.json").read_text()),
                         ids=lambda c: c["name"])
def test_golden_cases(net, case):
    dp = nb.default_decide(use_ceil=int(case["use_ceil"]), normalize_rate=case["rate"],
                           scale_up=int(case["scale_up"]), clamp_max=8.0)
    sidx = np.array(case["sidx"], np.uint32) if case.get("sidx") else None
    g = run_decide(net, np.array(case["rrs"], np.float32), np.array(case["rnd"], np.float32),
                   case["budget"], case["nspec"], dp, capacity=case.get("capacity"), sidx=sidx)
    assert g["split"].tolist() == case["split"]
    assert g["queue"].tolist() == case["queue"]
    assert g["total"] == case["total"]
    assert bool(g["flags"] & nb.DEV_OVERFLOW) == bool(case["flags"] & nb.DEV_OVERFLOW)
    if case["flags"] & nb.DEV_OVERFLOW:
        assert g["rc"] == nb.ERR_CAPACITY_OVERFLOW


@pytest.mark.parametrize("n", [1, 2047, 2048, 2049, 100003, 2_073_600])
@pytest.mark.parametrize("use_ceil,scale_up", [(1, 0), (0, 0), (0, 1)])
def test_random_bitexact(net, n, use_ceil, scale_up):
    rng = np.random.default_rng(n + 7 * use_ceil + 13 * scale_up)
    rrs = np.clip(rng.lognormal(-0.3, 1.2, n), 0.05, 8).astype(np.float32)
    rnd = rng.random(n, dtype=np.float32)
    dp = nb.default_decide(use_ceil=use_ceil, scale_up=scale_up, normalize_rate=0.85)
    budget, nspec = n, n // 50
    o = O.decide_emit(rrs, rnd, budget, nspec, dp, shift_n=MAXQ)
    g = run_decide(net, rrs, rnd, budget, nspec, dp)
    compare(g, o)
    assert g["rc"] == nb.OK


def test_scatter_index_permutation(net):
    rng = np.random.default_rng(3)
    n = 50000
    rrs = np.clip(rng.lognormal(0, 1, n), 0.05, 8).astype(np.float32)
    rnd = rng.random(n, dtype=np.float32)
    sidx = rng.permutation(n + 100)[:n].astype(np.uint32)
    dp = nb.default_decide()
    o = O.decide_emit(rrs, rnd, n, 0, dp, scatter_index=sidx, shift_n=MAXQ)
    g = run_decide(net, rrs, rnd, n, 0, dp, sidx=sidx)
    compare(g, o)


def test_capacity_overflow_keeps_prefix(net):
    rng = np.random.default_rng(4)
    n = 30000
    rrs = np.clip(rng.lognormal(0, 1, n), 0.05, 8).astype(np.float32)
    rnd = rng.random(n, dtype=np.float32)
    dp = nb.default_decide()
    full = O.decide_emit(rrs, rnd, n, 0, dp, shift_n=MAXQ)
    cap = full["total"] // 2
    g = run_decide(net, rrs, rnd, n, 0, dp, capacity=cap)
    assert g["total"] == full["total"]
    assert np.array_equal(g["queue"], full["queue"][:cap])
    assert g["flags"] & nb.DEV_OVERFLOW and g["rc"] == nb.ERR_CAPACITY_OVERFLOW


def test_empty_queue(net):
    dp = nb.default_decide()
    g = run_decide(net, np.zeros(0, np.float32), np.zeros(0, np.float32), 10, 0, dp)
    assert g["total"] == 0


def test_repeated_launches_reset_scratch(net):
    rng = np.random.default_rng(5)
    n = 123457
    rrs = np.clip(rng.lognormal(0, 1, n), 0.05, 8).astype(np.float32)
    rnd = rng.random(n, dtype=np.float32)
    dp = nb.default_decide()
    o = O.decide_emit(rrs, rnd, n, 0, dp, shift_n=MAXQ)
    for _ in range(3):
        compare(run_decide(net, rrs, rnd, n, 0, dp), o)


def test_device_n_specular(net):
    torch = torch_cuda()
    rng = np.random.default_rng(6)
    n = 9000
    rrs = np.clip(rng.lognormal(0, 1, n), 0.05, 8).astype(np.float32)
    rnd = rng.random(n, dtype=np.float32)
    dp = nb.default_decide(use_ceil=0, normalize_rate=1.0)
    o = O.decide_emit(rrs, rnd, n, 4321, dp, shift_n=MAXQ)
    d_spec = torch.tensor([4321], dtype=torch.int32, device="cuda")
    d_rrs = torch.from_numpy(rrs).cuda()
    d_rnd = torch.from_numpy(rnd).cuda()
    cap = n * 10
    d_norm, d_split, d_q, d_sz = empty(n), empty(n, "uint8"), empty(cap, "int32"), empty(1, "int32")
    net.decideEmit(d_rrs, d_rnd, n, n, 0, dp, d_norm, d_split, d_q, cap, d_sz,
                   n_specular_dev=d_spec, stream=stream())
    assert int(host(d_sz, np.uint32)[0]) == o["total"]
    assert np.array_equal(host(d_split), o["split"])


@pytest.mark.parametrize("n", [2049, 300001])
def test_without_split_and_norm_arrays(net, n):
    """split and rrs_norm are optional outputs: without them the decision keeps the split counts
    in its own scratch, and the queue and its size are still the oracle's"""
    torch = torch_cuda()
    rng = np.random.default_rng(n)
    rrs = np.clip(rng.lognormal(-0.2, 1.1, n), 0.05, 8).astype(np.float32)
    rnd = rng.random(n, dtype=np.float32)
    dp = nb.default_decide()
    o = O.decide_emit(rrs, rnd, n, n // 40, dp, shift_n=MAXQ)
    cap = 9 * n
    d_q, d_sz = empty(cap, "int32"), empty(1, "int32")
    net.decideEmit(torch.from_numpy(rrs).cuda(), torch.from_numpy(rnd).cuda(), n, n, n // 40, dp,
                   None, None, d_q, cap, d_sz, stream=stream())
    tot = int(host(d_sz, np.uint32)[0])
    assert tot == o["total"]
    assert np.array_equal(host(d_q, np.uint32)[:tot], o["queue"])
    assert net.device_status(stream()) == (nb.OK, 0)


def test_chunks_beyond_the_shared_memory_stage(net):
    """scale_up with a few large factors: chunks whose queue entries exceed the emission's
    shared-memory stage (4,096 entries for 2,048 vertices) write them directly"""
    rng = np.random.default_rng(11)
    n = 100_000
    rrs = np.full(n, 0.05, np.float32)
    rrs[:3000] = 8.0
    rrs[50_000:50_500] = rng.uniform(4.0, 8.0, 500).astype(np.float32)
    rnd = rng.random(n, dtype=np.float32)
    dp = nb.default_decide(use_ceil=0, scale_up=1, normalize_rate=1.0)
    o = O.decide_emit(rrs, rnd, n, 0, dp, shift_n=MAXQ)
    assert o["split"][:2048].sum() > 4096
    g = run_decide(net, rrs, rnd, n, 0, dp, capacity=o["total"] + 16)
    compare(g, o)
    assert g["rc"] == nb.OK
