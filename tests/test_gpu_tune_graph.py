"""GPU tests of the launch-shape autotuner and of the CUDA graph of the batched step: every
launch shape gives bit-identical outputs, the tuner's cache is reused, and one graph launch of
the uneven multi-depth step equals the direct batched call."""
from __future__ import annotations

import json

import numpy as np
import pytest

import nrrs_b200 as nb
from gpu_util import empty, host, make_net, random_params, soa, stream, torch_cuda, upload

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [nb.PREC_FP16, nb.PREC_FP32], ids=["fp16", "fp32"])
def test_launch_shapes_give_identical_outputs(prec):
    torch = torch_cuda()
    net = make_net(precision=prec)
    random_params(net, 50, table_scale=0.5, mlp_scale=0.15)
    n = 150_001
    v = nb.synth(51, n)
    d = upload(v)
    dp = nb.default_decide()
    shapes = [(1, 1), (2, 1), (0, 1)] + ([(1, 2), (0, 2)] if prec != nb.PREC_FP32 else [])
    ref = None
    for c, w in shapes:
        net.set_launch_shape(c, w)
        st, rr = empty(3 * n), empty(n)
        net.inference(soa(d), n, dp, st, rr, stream())
        torch.cuda.synchronize()
        out = (host(st)[:3 * n].copy(), host(rr)[:n].copy())
        if ref is None:
            ref = out
        else:
            assert np.array_equal(out[0].view(np.uint32), ref[0].view(np.uint32)), (c, w)
            assert np.array_equal(out[1].view(np.uint32), ref[1].view(np.uint32)), (c, w)
    net.close()


def test_autotune_picks_and_caches(tmp_path):
    net = make_net(precision=nb.PREC_FP16)
    cache = tmp_path / "tune.json"
    rep = json.loads(net.autotune(262144, cache))
    assert rep["trials"] and tuple(rep["best"][:2]) == net.launch_shape()
    assert rep["best"][2] == net.infer_split()
    assert {t["split"] for t in rep["trials"]} == {0, 1, 2, 3}   # every inference mode was timed
    assert min(t["ms"] for t in rep["trials"]) == pytest.approx(rep["best_ms"])
    other = make_net(precision=nb.PREC_FP16)
    rep2 = json.loads(other.autotune(262144, cache))
    assert tuple(rep2["cached"]) == tuple(rep["best"])
    assert tuple(rep2["cached"][:2]) == other.launch_shape() and rep2["cached"][2] == other.infer_split()
    json.loads(cache.read_text())
    net.close()
    other.close()


def test_graph_of_batched_step_equals_direct_call():
    torch = torch_cuda()
    net = make_net(precision=nb.PREC_FP16)
    random_params(net, 52, table_scale=0.5, mlp_scale=0.15)
    counts = [int(round(300_000 * 0.6 ** k)) for k in range(10)]
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    N = int(offs[-1])
    v = nb.synth(53, N)
    d = upload(v)
    dp = nb.default_decide()
    caps = [9 * c for c in counts]
    qoffs = np.concatenate([[0], np.cumsum(caps)]).astype(np.int64)
    segs = [nb.Segment(int(offs[k]), counts[k], counts[k], 0, int(qoffs[k]), caps[k])
            for k in range(len(counts))]

    def bufs():
        return dict(st=empty(3 * N), rrs=empty(N), norm=empty(N), split=empty(N, "uint8"),
                    q=empty(int(qoffs[-1]), "int32"), sz=empty(len(counts), "int32"))

    a, b = bufs(), bufs()
    net.generateRRSNumberBatched(soa(d), d["rnd"], segs, dp, a["st"], a["rrs"], a["norm"],
                                 a["split"], a["q"], a["sz"], stream())
    g = net.captureBatched(soa(d), d["rnd"], segs, dp, b["st"], b["rrs"], b["norm"], b["split"],
                           b["q"], b["sz"])
    for _ in range(2):          # replays reuse the self-resetting scratch
        b["sz"].zero_()
        g.launch(stream())
        torch.cuda.synchronize()
        for k in a:
            assert torch.equal(a[k], b[k]), k
    g.close()
    rc, flags = net.device_status(stream())
    assert rc == nb.OK and flags == 0
    net.close()


SPLIT_SHAPES = {
    "w64h2_fp16": (nb.PREC_FP16, dict()),
    "w64h3_bf16": (nb.PREC_BF16, dict(statnet_width=64, statnet_hidden=3, rrsnet_width=64,
                                      rrsnet_hidden=3)),
    "w128h3_bf16": (nb.PREC_BF16, dict(statnet_width=128, statnet_hidden=3, rrsnet_width=128,
                                       rrsnet_hidden=3, log2_hashmap_size=22)),
}


@pytest.mark.parametrize("factor", [nb.FACTOR_RRSNET, nb.FACTOR_ADRRS], ids=["rrsnet", "adrrs"])
@pytest.mark.parametrize("shape", list(SPLIT_SHAPES))
def test_split_inference_equals_fused(shape, factor):
    """every split mode (encoding kernel + one MLP kernel; encoding + StatNet + RRSNet kernels;
    the same with the hidden activations in TMEM) gives the fused kernel's outputs bit for bit,
    for every warpgroup count that fits, on a ragged multi-segment launch, with RRSNet and
    ADRRS factors"""
    torch = torch_cuda()
    prec, kw = SPLIT_SHAPES[shape]
    net = make_net(precision=prec, **kw)
    random_params(net, 54, table_scale=0.5, mlp_scale=0.1)
    if factor == nb.FACTOR_ADRRS:
        net.setStep(2)
    counts = [70_001, 129, 1, 0, 33_333]
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    N = int(offs[-1])
    v = nb.synth(55, N)
    d = upload(v)
    dp = nb.default_decide(factor_source=factor)
    caps = [9 * c for c in counts]
    qoffs = np.concatenate([[0], np.cumsum(caps)]).astype(np.int64)
    segs = [nb.Segment(int(offs[k]), counts[k], max(counts[k], 1), 0, int(qoffs[k]), caps[k])
            for k in range(len(counts))]

    def run():
        o = dict(st=empty(3 * N), rrs=empty(N), norm=empty(N), split=empty(N, "uint8"),
                 q=empty(int(qoffs[-1]), "int32"), sz=empty(len(counts), "int32"))
        net.generateRRSNumberBatched(soa(d), d["rnd"], segs, dp, o["st"], o["rrs"], o["norm"],
                                     o["split"], o["q"], o["sz"], stream())
        torch.cuda.synchronize()
        return o

    net.set_infer_split(0)
    net.set_launch_shape(0, 1)
    ref = run()
    tried = 0
    for mode in (1, 2, 3):
        net.set_infer_split(mode)
        assert net.infer_split() == mode
        for w in (1, 2, 4):
            try:
                net.set_launch_shape(0, w)
            except nb.NRRSError:
                continue                      # that many warpgroups do not fit in this mode
            tried += 1
            out = run()
            for k in ref:
                assert torch.equal(out[k], ref[k]), (shape, mode, w, k)
    assert tried >= 4
    rc, flags = net.device_status(stream())
    assert rc == nb.OK and flags == 0
    net.close()


def test_split_modes_with_many_tiles_per_warpgroup():
    """one CTA per SM, so every warpgroup walks about 27 tiles and requests each next tile's
    inputs during the current one: no wait runs out (device status clean) and the outputs
    equal the fused kernel's, in every split mode and warpgroup count"""
    torch = torch_cuda()
    prec, kw = SPLIT_SHAPES["w128h3_bf16"]
    net = make_net(precision=prec, **kw)
    random_params(net, 57, table_scale=0.5, mlp_scale=0.1)
    n = 2_000_000
    v = nb.synth(58, n)
    d = upload(v)
    dp = nb.default_decide()

    def run():
        st, rr = empty(3 * n), empty(n)
        net.inference(soa(d), n, dp, st, rr, stream())
        torch.cuda.synchronize()
        return st, rr

    net.set_infer_split(0)
    net.set_launch_shape(0, 1)
    ref = run()
    for mode in (1, 2, 3):
        net.set_infer_split(mode)
        for w in (1, 2, 4):
            try:
                net.set_launch_shape(1, w)
            except nb.NRRSError:
                continue
            out = run()
            assert net.device_status(stream()) == (nb.OK, 0), (mode, w)
            assert torch.equal(out[0], ref[0]) and torch.equal(out[1], ref[1]), (mode, w)
    net.close()


def test_split_mode_graph_equals_fused_direct():
    torch = torch_cuda()
    net = make_net(precision=nb.PREC_FP16)
    random_params(net, 56, table_scale=0.5, mlp_scale=0.15)
    counts = [int(round(200_000 * 0.6 ** k)) for k in range(6)]
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    N = int(offs[-1])
    v = nb.synth(57, N)
    d = upload(v)
    dp = nb.default_decide()
    caps = [9 * c for c in counts]
    qoffs = np.concatenate([[0], np.cumsum(caps)]).astype(np.int64)
    segs = [nb.Segment(int(offs[k]), counts[k], counts[k], 0, int(qoffs[k]), caps[k])
            for k in range(len(counts))]

    def bufs():
        return dict(st=empty(3 * N), rrs=empty(N), norm=empty(N), split=empty(N, "uint8"),
                    q=empty(int(qoffs[-1]), "int32"), sz=empty(len(counts), "int32"))

    a, b = bufs(), bufs()
    net.generateRRSNumberBatched(soa(d), d["rnd"], segs, dp, a["st"], a["rrs"], a["norm"],
                                 a["split"], a["q"], a["sz"], stream())
    net.set_infer_split(True)
    l0 = net.launch_count()
    g = net.captureBatched(soa(d), d["rnd"], segs, dp, b["st"], b["rrs"], b["norm"], b["split"],
                           b["q"], b["sz"])
    assert net.launch_count() - l0 == 4      # encode, MLP, decision count and emit
    g.launch(stream())
    torch.cuda.synchronize()
    for k in a:
        assert torch.equal(a[k], b[k]), k
    g.close()
    net.close()
