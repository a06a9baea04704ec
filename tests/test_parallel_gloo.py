"""Multi-rank tests of the sharded NRRS step (nrrs_parallel.ShardedNRRS) on CPU with gloo,
world size 2. The GPU library is replaced by an oracle-backed stand-in with the same operations,
so the host logic (sharding, the integer all-reduce of the exact sum, global budget, queue
offsets, data-parallel gradients) is exercised without a GPU. The assertion is the sharding
contract: the per-rank queues, concatenated in rank order, equal the single-process decision on
the whole queue bit for bit, and the averaged shard gradients equal the full-batch gradient."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import nrrs_b200 as nb
import oracle as O
from nrrs_parallel import ShardedNRRS

N_TOTAL = 24_000
MAXQ = 1 << 16


class OracleBackend:
    """CPU stand-in for nrrs_b200.NRRSNetwork (test only): same operations, oracle maths."""

    def __init__(self, cfg, params, shard):
        self.cfg, self.params, self.v = cfg, params, shard
        self.grads = None

    def inferAccumulate(self, soa, n, dp, stats, rrs, sum_acc, stream=0):
        r = O.infer(self.cfg, self.params, self.v, dp, "f32", want=("rrs",))["rrs"]
        rrs[:n] = torch.from_numpy(r)
        shift = O.sum_shift(MAXQ, float(np.ceil(dp.clamp_max)) if dp.use_ceil else dp.clamp_max)
        acc, _ = O.sum_fixed(r, bool(dp.use_ceil), shift)
        sum_acc += acc

    def decideEmitWithSum(self, rrs, rnd, n, budget, n_spec, sum_acc, dp, rrs_norm, split, queue,
                          capacity, next_size, scatter_index=None, stream=0):
        shift = O.sum_shift(MAXQ, float(np.ceil(dp.clamp_max)) if dp.use_ceil else dp.clamp_max)
        d = O.decide_emit_acc(rrs[:n].numpy(), rnd, budget, n_spec, dp, int(sum_acc.item()), shift,
                              capacity=capacity)
        q = d["queue"]
        queue[:q.size] = torch.from_numpy(q.astype(np.int64))
        split[:n] = torch.from_numpy(d["split"].astype(np.int64))
        rrs_norm[:n] = torch.from_numpy(d["rrs_norm"])
        next_size[0] = d["total"]

    def trainGrads(self, soa, target, n, loss=None, stream=0):
        self.grads, _ = O.train_grads(self.cfg, self.params, self.v, self.v["target"], "f64")

    def copyGrads(self, buf, stream=0):
        buf.copy_(torch.from_numpy(self.grads))

    def adamApply(self, buf, scale, stream=0):
        self.applied = buf.numpy() * scale


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, result_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        cfg = nb.default_config(log2_hashmap_size=12, max_queue=MAXQ, step=2)
        npar = O.param_count(cfg)[0]
        params = (np.random.default_rng(0).uniform(-1, 1, npar) * 0.2).astype(np.float32)
        full = nb.synth(1, N_TOTAL)
        lo, hi = rank * N_TOTAL // world, (rank + 1) * N_TOTAL // world
        shard = {k: a[lo:hi].copy() for k, a in full.items()}
        n = hi - lo
        dp = nb.default_decide()
        sh = ShardedNRRS(OracleBackend(cfg, params, shard))
        rrs = torch.zeros(n)
        cap = 10 * n
        queue, split = torch.zeros(cap, dtype=torch.int64), torch.zeros(n, dtype=torch.int64)
        norm, size = torch.zeros(n), torch.zeros(1, dtype=torch.int64)
        acc = torch.zeros(1, dtype=torch.int64)
        sh.step(None, shard["rnd"], n, N_TOTAL, 100, dp, None, rrs, norm, split, queue, cap, size, acc)
        offs = sh.queue_offsets(int(size.item()))
        q = queue[:int(size.item())].numpy() + lo
        grads = torch.zeros(npar, dtype=torch.float64)
        sh.train_step(None, None, n, grads)
        result_q.put((rank, offs, q, split.numpy(), int(acc.item()), sh.backend.applied))
    finally:
        dist.destroy_process_group()


@pytest.fixture(scope="module")
def gloo_results():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in procs:
        r = q.get(timeout=240)
        res[r[0]] = r
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return res


def test_sharded_decision_equals_single_process(gloo_results):
    cfg = nb.default_config(log2_hashmap_size=12, max_queue=MAXQ, step=2)
    npar = O.param_count(cfg)[0]
    params = (np.random.default_rng(0).uniform(-1, 1, npar) * 0.2).astype(np.float32)
    full = nb.synth(1, N_TOTAL)
    dp = nb.default_decide()
    r = O.infer(cfg, params, full, dp, "f32", want=("rrs",))["rrs"]
    ref = O.decide_emit(r, full["rnd"], N_TOTAL, 100, dp, shift_n=MAXQ)
    (r0, offs0, q0, s0, acc0, _), (r1, offs1, q1, s1, acc1, _) = gloo_results[0], gloo_results[1]
    assert acc0 == acc1                                  # every rank holds the global sum
    assert offs0 == offs1 == [0, q0.size]
    assert np.array_equal(np.concatenate([q0, q1]), ref["queue"])
    assert np.array_equal(np.concatenate([s0, s1]), ref["split"])


def test_data_parallel_gradient_is_full_batch_mean(gloo_results):
    cfg = nb.default_config(log2_hashmap_size=12, max_queue=MAXQ, step=2)
    npar = O.param_count(cfg)[0]
    params = (np.random.default_rng(0).uniform(-1, 1, npar) * 0.2).astype(np.float32)
    full = nb.synth(1, N_TOTAL)
    g_full, _ = O.train_grads(cfg, params, full, full["target"], "f64")
    g0, g1 = gloo_results[0][5], gloo_results[1][5]
    assert np.array_equal(g0, g1)
    # StatNet loss is a mean over samples: the mean of equal-size shard gradients is exact
    assert np.allclose(g0, g_full, rtol=1e-9, atol=1e-15)
