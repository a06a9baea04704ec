"""GPU parity of the fused inference kernels (encoding, StatNet, glue, RRSNet, activation,
clamp) against the oracle, and of the fused/batched step against separate calls."""
from __future__ import annotations

import numpy as np
import pytest

import nrrs_b200 as nb
import oracle as O
from gpu_util import empty, host, make_net, random_params, soa, stream, torch_cuda, upload

pytestmark = pytest.mark.gpu
MAXQ = 1 << 21  # max_queue of make_net(): fixes the exact sum's shift

# FP32 path: same maths as the FP32 oracle up to FMA contraction and libm ulps
FP32_RTOL, FP32_ATOL = 2e-4, 2e-5
# factor target of the workload: within 1e-2 relative of the FP64 oracle (mixed precision)
MIXED_RTOL = 1e-2


def run_infer(net, v, dp, n):
    d = upload(v)
    stats, rrs = empty(3 * n), empty(n)
    net.inference(soa(d), n, dp, stats, rrs, stream())
    return host(stats)[:3 * n].reshape(n, 3), host(rrs)[:n]


@pytest.fixture(scope="module")
def fp32_net():
    net = make_net()
    yield net
    net.close()


@pytest.mark.parametrize("params", ["init", "random"])
@pytest.mark.parametrize("source", [nb.FACTOR_RRSNET, nb.FACTOR_ADRRS])
def test_fp32_infer_matches_oracle(fp32_net, params, source):
    n = 65536
    v = nb.synth(0, n)
    if params == "random":
        p = random_params(fp32_net, 1)
    else:
        fresh = make_net()
        p = fresh.get_params()
        fresh.close()
        fp32_net.set_params(p)
    dp = nb.default_decide(factor_source=source)
    stats, rrs = run_infer(fp32_net, v, dp, n)
    o32 = O.infer(fp32_net.config, p, v, dp, "f32")
    o64 = O.infer(fp32_net.config, p, v, dp, "f64")
    assert np.allclose(stats, o32["stats"], rtol=FP32_RTOL, atol=FP32_ATOL)
    assert np.allclose(rrs, o32["rrs"], rtol=FP32_RTOL, atol=FP32_ATOL)
    rel = np.abs(rrs - o64["rrs"]) / o64["rrs"]
    assert rel.max() < 1e-4, rel.max()


def test_fp32_ragged_sizes_and_normalized_positions():
    net = make_net(normalize_pos=1, aabb_min=[-2, -1, 0], aabb_max=[3, 2, 5])
    p = random_params(net, 2)
    for n in (1, 127, 129, 1000):
        v = nb.synth(11, n)
        v["pos"] = (v["pos"] * np.array([5, 3, 5], np.float32) + np.array([-2, -1, 0], np.float32)).astype(np.float32)
        dp = nb.default_decide()
        stats, rrs = run_infer(net, v, dp, n)
        o = O.infer(net.config, p, v, dp, "f32")
        assert np.allclose(stats, o["stats"], rtol=FP32_RTOL, atol=FP32_ATOL), n
        assert np.allclose(rrs, o["rrs"], rtol=FP32_RTOL, atol=FP32_ATOL), n
    net.close()


def test_step_equals_infer_then_decide(fp32_net):
    torch = torch_cuda()
    n = 200001
    v = nb.synth(3, n)
    random_params(fp32_net, 3)
    dp = nb.default_decide()
    d = upload(v)
    s = soa(d)
    cap = 9 * n
    a = dict(stats=empty(3 * n), rrs=empty(n), norm=empty(n), split=empty(n, "uint8"),
             q=empty(cap, "int32"), sz=empty(1, "int32"))
    fp32_net.generateRRSNumber(s, d["rnd"], n, n, 0, dp, a["stats"], a["rrs"], a["norm"],
                               a["split"], a["q"], cap, a["sz"], stream())
    b = dict(stats=empty(3 * n), rrs=empty(n), norm=empty(n), split=empty(n, "uint8"),
             q=empty(cap, "int32"), sz=empty(1, "int32"))
    fp32_net.inference(s, n, dp, b["stats"], b["rrs"], stream())
    fp32_net.decideEmit(b["rrs"], d["rnd"], n, n, 0, dp, b["norm"], b["split"], b["q"], cap,
                        b["sz"], stream=stream())
    torch.cuda.synchronize()
    for k in a:
        assert torch.equal(a[k], b[k]), k
    # and the decision equals the oracle's on the GPU factors
    o = O.decide_emit(host(a["rrs"])[:n], v["rnd"], n, 0, dp, shift_n=MAXQ)
    tot = int(host(a["sz"], np.uint32)[0])
    assert tot == o["total"]
    assert np.array_equal(host(a["q"], np.uint32)[:tot], o["queue"])


def test_batched_equals_per_depth(fp32_net):
    torch = torch_cuda()
    random_params(fp32_net, 4)
    counts = [70000, 42000, 25200, 15120, 9072, 0, 3265]
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    N = int(offs[-1])
    v = nb.synth(9, N)
    d = upload(v)
    s = soa(d)
    dp = nb.default_decide()
    caps = [9 * c for c in counts]
    qoffs = np.concatenate([[0], np.cumsum(caps)]).astype(np.int64)
    segs = [nb.Segment(int(offs[k]), counts[k], max(counts[k], 1), k, int(qoffs[k]), caps[k])
            for k in range(len(counts))]
    bat = dict(stats=empty(3 * N), rrs=empty(N), norm=empty(N), split=empty(N, "uint8"),
               q=empty(int(qoffs[-1]), "int32"), sz=empty(len(counts), "int32"))
    fp32_net.generateRRSNumberBatched(s, d["rnd"], segs, dp, bat["stats"], bat["rrs"],
                                      bat["norm"], bat["split"], bat["q"], bat["sz"], stream())
    sz = host(bat["sz"], np.uint32)
    q = host(bat["q"], np.uint32)
    split = host(bat["split"])
    rrs_b = host(bat["rrs"])
    for k, c in enumerate(counts):
        o0, o1 = int(offs[k]), int(offs[k + 1])
        if c == 0:
            assert sz[k] == 0
            continue
        sub = {key: val[o0:o1].copy() for key, val in v.items()}
        ds = upload(sub)
        one = dict(stats=empty(3 * c), rrs=empty(c), norm=empty(c), split=empty(c, "uint8"),
                   q=empty(caps[k], "int32"), sz=empty(1, "int32"))
        fp32_net.generateRRSNumber(soa(ds), ds["rnd"], c, max(c, 1), k, dp, one["stats"],
                                   one["rrs"], one["norm"], one["split"], one["q"], caps[k],
                                   one["sz"], stream())
        tot = int(host(one["sz"], np.uint32)[0])
        assert sz[k] == tot, k
        assert np.array_equal(host(one["rrs"])[:c], rrs_b[o0:o1])
        assert np.array_equal(host(one["split"])[:c], split[o0:o1])
        # the batched queue stores vertex indices of the concatenated SoA
        assert np.array_equal(host(one["q"], np.uint32)[:tot] + o0,
                              q[int(qoffs[k]):int(qoffs[k]) + tot])
    torch.cuda.synchronize()


def test_full_size_queue_properties(fp32_net):
    n = 2_073_600
    v = nb.synth(21, n)
    random_params(fp32_net, 5)
    dp = nb.default_decide()
    d = upload(v)
    cap = 9 * n
    st, rrs, norm = empty(3 * n), empty(n), empty(n)
    split, q, sz = empty(n, "uint8"), empty(cap, "int32"), empty(1, "int32")
    fp32_net.generateRRSNumber(soa(d), d["rnd"], n, n, 0, dp, st, rrs, norm, split, q, cap, sz,
                               stream())
    tot = int(host(sz, np.uint32)[0])
    s = host(split)[:n].astype(np.int64)
    qq = host(q, np.uint32)[:tot]
    assert tot == s.sum()
    assert np.all(np.diff(qq.astype(np.int64)) >= 0)
    assert np.array_equal(np.bincount(qq, minlength=n), s)
    o = O.decide_emit(host(rrs)[:n], v["rnd"], n, 0, dp, shift_n=MAXQ)
    assert tot == o["total"] and np.array_equal(s, o["split"])
    rc, flags = fp32_net.device_status(stream())
    assert rc == nb.OK and flags == 0


def test_save_load_roundtrip(fp32_net, tmp_path):
    p = random_params(fp32_net, 6)
    f = tmp_path / "ckpt.bin"
    fp32_net.saveWeights(f)
    other = make_net()
    other.loadWeights(f)
    assert np.array_equal(other.get_params(), p)
    other.close()


SHAPES = {"w64h2": dict(statnet_width=64, statnet_hidden=2, rrsnet_width=64, rrsnet_hidden=2),
          "w128h3": dict(statnet_width=128, statnet_hidden=3, rrsnet_width=128, rrsnet_hidden=3,
                         log2_hashmap_size=22)}


@pytest.mark.parametrize("prec", [nb.PREC_FP16, nb.PREC_BF16], ids=["fp16", "bf16"])
@pytest.mark.parametrize("shape", list(SHAPES))
def test_mixed_infer_vs_fp64_oracle(prec, shape):
    """tcgen05 path: RRS factors within 1e-2 relative of the FP64 oracle (workload target)."""
    net = make_net(precision=prec, **SHAPES[shape])
    p = random_params(net, 7, table_scale=0.5, mlp_scale=0.15)
    n = 16384 if shape == "w128h3" else 65536
    v = nb.synth(1, n)
    for source in (nb.FACTOR_RRSNET, nb.FACTOR_ADRRS):
        dp = nb.default_decide(factor_source=source)
        stats, rrs = run_infer(net, v, dp, n)
        o = O.infer(net.config, p, v, dp, "f64")
        rel = np.abs(rrs - o["rrs"]) / o["rrs"]
        assert rel.max() < MIXED_RTOL, (source, rel.max())
        err = np.abs(stats - o["stats"])
        assert err.max() < 0.05 * max(1.0, np.abs(o["stats"]).max()), err.max()
    net.close()


@pytest.mark.parametrize("shape", list(SHAPES))
def test_fp32_shapes_vs_oracle(shape):
    net = make_net(**SHAPES[shape])
    p = random_params(net, 8, table_scale=0.5, mlp_scale=0.15)
    n = 8192
    v = nb.synth(2, n)
    dp = nb.default_decide()
    stats, rrs = run_infer(net, v, dp, n)
    o = O.infer(net.config, p, v, dp, "f32")
    assert np.allclose(stats, o["stats"], rtol=FP32_RTOL, atol=FP32_ATOL)
    assert np.allclose(rrs, o["rrs"], rtol=FP32_RTOL, atol=FP32_ATOL)
    net.close()


@pytest.mark.parametrize("prec", [nb.PREC_FP16, nb.PREC_BF16], ids=["fp16", "bf16"])
def test_mixed_step_decisions_match_oracle(prec):
    """decisions are bit-exact given the (mixed-precision) factors the GPU produced"""
    net = make_net(precision=prec)
    random_params(net, 9, table_scale=0.5, mlp_scale=0.15)
    n = 300007
    v = nb.synth(4, n)
    d = upload(v)
    dp = nb.default_decide()
    cap = 9 * n
    st, rrs, norm = empty(3 * n), empty(n), empty(n)
    split, q, sz = empty(n, "uint8"), empty(cap, "int32"), empty(1, "int32")
    net.generateRRSNumber(soa(d), d["rnd"], n, n, 0, dp, st, rrs, norm, split, q, cap, sz, stream())
    tot = int(host(sz, np.uint32)[0])
    o = O.decide_emit(host(rrs)[:n], v["rnd"], n, 0, dp, shift_n=MAXQ)
    assert tot == o["total"]
    assert np.array_equal(host(split)[:n], o["split"])
    assert np.array_equal(host(q, np.uint32)[:tot], o["queue"])
    assert np.array_equal(host(norm)[:n].view(np.uint32), o["rrs_norm"].view(np.uint32))
    net.close()


def test_full_size_4k_bounce():
    """One full 4K bounce (8,294,400 vertices) on the 4K configuration (128 x 3 BF16 networks,
    2^22-entry table): the emitted queue is in vertex order with each vertex as many times as its
    split count; the decision equals the oracle's on the factors the GPU produced, bit for bit;
    and the factors of 4,096 vertices spread over the queue are within the workload's 1e-2 of
    the FP64 oracle."""
    n = 8_294_400
    net = make_net(precision=nb.PREC_BF16, max_queue=n, **SHAPES["w128h3"])
    p = random_params(net, 10, table_scale=0.5, mlp_scale=0.15)
    v = nb.synth(31, n)
    d = upload(v)
    dp = nb.default_decide()
    cap = 9 * n
    st, rrs, norm = empty(3 * n), empty(n), empty(n)
    split, q, sz = empty(n, "uint8"), empty(cap, "int32"), empty(1, "int32")
    net.generateRRSNumber(soa(d), d["rnd"], n, n, 0, dp, st, rrs, norm, split, q, cap, sz,
                          stream())
    tot = int(host(sz, np.uint32)[0])
    s = host(split)[:n].astype(np.int64)
    qq = host(q, np.uint32)[:tot]
    assert tot == s.sum() > 0
    assert np.all(np.diff(qq.astype(np.int64)) >= 0)
    assert np.array_equal(np.bincount(qq, minlength=n), s)
    r = host(rrs)[:n]
    o = O.decide_emit(r, v["rnd"], n, 0, dp, shift_n=n)
    assert tot == o["total"] and np.array_equal(s, o["split"])
    assert np.array_equal(host(norm)[:n].view(np.uint32), o["rrs_norm"].view(np.uint32))
    idx = np.random.default_rng(3).choice(n, 4096, replace=False)
    sub = {k: (a[idx] if isinstance(a, np.ndarray) and len(a) == n else a) for k, a in v.items()}
    o64 = O.infer(net.config, p, sub, dp, "f64")
    rel = np.abs(r[idx] - o64["rrs"]) / o64["rrs"]
    assert rel.max() < MIXED_RTOL, rel.max()
    rc, flags = net.device_status(stream())
    assert rc == nb.OK and flags == 0
    net.close()


def test_batched_gapped_segments_without_split_array(fp32_net):
    """segments at caller-chosen offsets with gaps between them, one empty, and no split
    array: the same sizes, queue and normalised factors as the call that passes one"""
    random_params(fp32_net, 5)
    counts = [5000, 0, 3001, 2048]
    offs = [0, 7000, 7000, 12345]
    N = offs[-1] + counts[-1]
    v = nb.synth(10, N)
    d = upload(v)
    dp = nb.default_decide()
    caps = [9 * c for c in counts]
    qoffs = np.concatenate([[0], np.cumsum(caps)]).astype(np.int64)
    segs = [nb.Segment(offs[k], counts[k], max(counts[k], 1), 0, int(qoffs[k]), caps[k])
            for k in range(len(counts))]
    out = []
    for with_split in (True, False):
        o = dict(stats=empty(3 * N), rrs=empty(N), norm=empty(N),
                 split=empty(N, "uint8") if with_split else None,
                 q=empty(int(qoffs[-1]), "int32"), sz=empty(len(counts), "int32"))
        fp32_net.generateRRSNumberBatched(soa(d), d["rnd"], segs, dp, o["stats"], o["rrs"],
                                          o["norm"], o["split"], o["q"], o["sz"], stream())
        out.append((host(o["sz"], np.uint32).copy(), host(o["q"], np.uint32).copy(),
                    host(o["norm"]).view(np.uint32).copy()))
    (sz_a, q_a, n_a), (sz_b, q_b, n_b) = out
    assert np.array_equal(sz_a, sz_b) and sz_a[1] == 0 and sz_a[0] > 0
    for k, c in enumerate(counts):
        q0 = int(qoffs[k])
        assert np.array_equal(q_a[q0:q0 + sz_a[k]], q_b[q0:q0 + sz_b[k]]), k
        assert np.array_equal(n_a[offs[k]:offs[k] + c], n_b[offs[k]:offs[k] + c]), k
    assert fp32_net.device_status(stream()) == (nb.OK, 0)
