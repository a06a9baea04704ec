"""GPU check of the sharded building blocks on one device: two shards of a queue, each adding its
exact-sum terms into one int64 accumulator (what the integer all-reduce produces across GPUs),
then deciding against the global budget, give the same queue as nrrs_step on the whole queue;
the data-parallel training split (grads -> copy -> Adam) equals nrrs_train_step."""
from __future__ import annotations

import numpy as np
import pytest

import nrrs_b200 as nb
from gpu_util import empty, host, make_net, random_params, soa, stream, torch_cuda, upload

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [nb.PREC_FP32, nb.PREC_FP16], ids=["fp32", "fp16"])
def test_two_shards_equal_one_queue(prec):
    torch = torch_cuda()
    net = make_net(precision=prec)
    random_params(net, 40, table_scale=0.5, mlp_scale=0.15)
    n = 300_001
    v = nb.synth(41, n)
    dp = nb.default_decide()
    cap = 9 * n
    d = upload(v)
    full = dict(st=empty(3 * n), rrs=empty(n), norm=empty(n), split=empty(n, "uint8"),
                q=empty(cap, "int32"), sz=empty(1, "int32"))
    net.generateRRSNumber(soa(d), d["rnd"], n, n, 77, dp, full["st"], full["rrs"], full["norm"],
                          full["split"], full["q"], cap, full["sz"], stream())
    cut = 123_457
    acc = torch.zeros(1, dtype=torch.int64, device="cuda")
    shards = []
    for lo, hi in ((0, cut), (cut, n)):
        sub = upload({k: a[lo:hi].copy() for k, a in v.items()})
        o = dict(d=sub, st=empty(3 * (hi - lo)), rrs=empty(hi - lo), norm=empty(hi - lo),
                 split=empty(hi - lo, "uint8"), q=empty(cap, "int32"), sz=empty(1, "int32"))
        net.inferAccumulate(soa(sub), hi - lo, dp, o["st"], o["rrs"], acc, stream())
        shards.append((lo, hi, o))
    for lo, hi, o in shards:
        net.decideEmitWithSum(o["rrs"], o["d"]["rnd"], hi - lo, n, 77, acc, dp, o["norm"],
                              o["split"], o["q"], cap, o["sz"], stream=stream())
    torch.cuda.synchronize()
    tot = int(host(full["sz"], np.uint32)[0])
    qs = [host(o["q"], np.uint32)[:int(host(o["sz"], np.uint32)[0])] + lo for lo, hi, o in shards]
    assert np.array_equal(np.concatenate(qs), host(full["q"], np.uint32)[:tot])
    assert np.array_equal(np.concatenate([host(o["split"])[:hi - lo] for lo, hi, o in shards]),
                          host(full["split"])[:n])
    assert np.array_equal(np.concatenate([host(o["rrs"])[:hi - lo] for lo, hi, o in shards]),
                          host(full["rrs"])[:n])
    net.close()


def test_shard_contexts_with_sum_shards_equal_one_context():
    """two shard contexts of half the capacity created with sum_shards = 2 use the fixed-point
    shift of one context holding the whole queue, so their added sums decide bit-identically to
    it; without sum_shards the shift would leave room for one shard's terms only"""
    torch = torch_cuda()
    n = 2 * 150_000
    full_net = make_net(precision=nb.PREC_FP16, max_queue=n)
    p = random_params(full_net, 44, table_scale=0.5, mlp_scale=0.15)
    shard_net = make_net(precision=nb.PREC_FP16, max_queue=n // 2, sum_shards=2)
    shard_net.set_params(p)
    v = nb.synth(45, n)
    dp = nb.default_decide()
    cap = 9 * n
    d = upload(v)
    full = dict(st=empty(3 * n), rrs=empty(n), norm=empty(n), split=empty(n, "uint8"),
                q=empty(cap, "int32"), sz=empty(1, "int32"))
    full_net.generateRRSNumber(soa(d), d["rnd"], n, n, 0, dp, full["st"], full["rrs"],
                               full["norm"], full["split"], full["q"], cap, full["sz"], stream())
    acc = torch.zeros(1, dtype=torch.int64, device="cuda")
    shards = []
    for lo, hi in ((0, n // 2), (n // 2, n)):
        sub = upload({k: a[lo:hi].copy() for k, a in v.items()})
        o = dict(d=sub, st=empty(3 * (hi - lo)), rrs=empty(hi - lo), norm=empty(hi - lo),
                 split=empty(hi - lo, "uint8"), q=empty(cap, "int32"), sz=empty(1, "int32"))
        shard_net.inferAccumulate(soa(sub), hi - lo, dp, o["st"], o["rrs"], acc, stream())
        shards.append((lo, hi, o))
    for lo, hi, o in shards:
        shard_net.decideEmitWithSum(o["rrs"], o["d"]["rnd"], hi - lo, n, 0, acc, dp, o["norm"],
                                    o["split"], o["q"], cap, o["sz"], stream=stream())
    torch.cuda.synchronize()
    tot = int(host(full["sz"], np.uint32)[0])
    qs = [host(o["q"], np.uint32)[:int(host(o["sz"], np.uint32)[0])] + lo for lo, hi, o in shards]
    assert np.array_equal(np.concatenate(qs), host(full["q"], np.uint32)[:tot])
    assert np.array_equal(np.concatenate([host(o["norm"])[:hi - lo] for lo, hi, o in shards]),
                          host(full["norm"])[:n])
    assert shard_net.device_status(stream()) == (nb.OK, 0)
    full_net.close()
    shard_net.close()


@pytest.mark.parametrize("prec", [nb.PREC_FP32, nb.PREC_FP16], ids=["fp32", "fp16"])
def test_split_training_equals_train_step(prec):
    torch = torch_cuda()
    a = make_net(precision=prec, max_train=1 << 14)
    b = make_net(precision=prec, max_train=1 << 14)
    p = random_params(a, 42, table_scale=0.5, mlp_scale=0.15)
    b.set_params(p)
    n = 9000
    v = nb.synth(43, n)
    d = upload(v)
    la = torch.zeros(2, dtype=torch.float64, device="cuda")
    lb = torch.zeros(2, dtype=torch.float64, device="cuda")
    a.train(soa(d), d["target"], n, la, stream())
    buf = torch.zeros(b.param_count(), dtype=torch.float32, device="cuda")
    b.trainGrads(soa(d), d["target"], n, lb, stream())
    b.copyGrads(buf, stream())
    b.adamApply(buf, 1.0, stream())
    torch.cuda.synchronize()
    assert torch.equal(la, lb)
    pa, pb = a.get_params(), b.get_params()
    # the hash-grid gradient is an atomic scatter-add: its summation order can differ per run
    assert np.allclose(pa, pb, rtol=1e-5, atol=1e-6)
    a.close()
    b.close()
