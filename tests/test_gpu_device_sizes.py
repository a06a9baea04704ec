"""GPU tests of the device-resident queue sizes (nrrs_infer_dev, nrrs_decide_emit_dev,
nrrs_step_dev, nrrs_step_batched_dev): the reference's inference-queue size lives on the device
(integrator.cpp:1073-1085, 1533-1555), and these forms read it there. Every result equals the
host-size form on the same count, bit for bit; the buffers past the count hold NaN so that a
read beyond it would show. A count above max_n is clamped and flagged. One CUDA graph of the
step replays at two different counts, and a path-traced frame runs every bounce with device
sizes only (no host read between trace and step) and gives the host-size frame's image."""
from __future__ import annotations

import numpy as np
import pytest

import nrrs_b200 as nb
from gpu_util import empty, host, make_net, random_params, soa, stream, torch_cuda, upload

pytestmark = pytest.mark.gpu


def _poisoned(v, n, max_n):
    """vertex arrays of max_n entries: the first n from v, the rest NaN (or ~0 for integers)"""
    out = {}
    for k, a in v.items():
        b = np.empty((max_n,) + a.shape[1:], a.dtype)
        b[:n] = a[:n]
        if a.dtype.kind == "f":
            b[n:] = np.nan
        else:
            b[n:] = np.iinfo(a.dtype).max
        out[k] = b
    return out


def _step_outputs(n, cap):
    return dict(st=empty(3 * n), rrs=empty(n), norm=empty(n), split=empty(n, "uint8"),
                q=empty(cap, "int32"), sz=empty(1, "int32"))


def _host_out(o, n):
    tot = int(host(o["sz"], np.uint32)[0])
    return (tot, host(o["q"], np.uint32)[:tot].copy(), host(o["split"])[:n].copy(),
            host(o["norm"])[:n].view(np.uint32).copy(), host(o["rrs"])[:n].view(np.uint32).copy(),
            host(o["st"])[:3 * n].view(np.uint32).copy())


def _n_dev(n):
    torch = torch_cuda()
    return torch.tensor([n], dtype=torch.int32, device="cuda")


@pytest.mark.parametrize("prec,split", [(nb.PREC_FP16, 0), (nb.PREC_FP16, 2), (nb.PREC_FP32, 0)],
                         ids=["fp16-fused", "fp16-split2", "fp32"])
def test_step_dev_equals_host_size_step(prec, split):
    torch = torch_cuda()
    max_n, n = 300_000, 234_567
    net = make_net(precision=prec, max_queue=max_n)
    if split:
        net.set_infer_split(split)
    random_params(net, 70, table_scale=0.5, mlp_scale=0.15)
    v = _poisoned(nb.synth(71, max_n), n, max_n)
    d = upload(v)
    dp = nb.default_decide()
    cap = 9 * max_n
    a, b = _step_outputs(max_n, cap), _step_outputs(max_n, cap)
    net.generateRRSNumber(soa(d), d["rnd"], n, n, 1000, dp, a["st"], a["rrs"], a["norm"],
                          a["split"], a["q"], cap, a["sz"], stream())
    net.generateRRSNumberDev(soa(d), d["rnd"], _n_dev(n), max_n, n, 1000, dp, b["st"], b["rrs"],
                             b["norm"], b["split"], b["q"], cap, b["sz"], stream=stream())
    torch.cuda.synchronize()
    ha, hb = _host_out(a, n), _host_out(b, n)
    assert ha[0] == hb[0] > 0
    for x, y in zip(ha[1:], hb[1:]):
        assert np.array_equal(x, y)
    assert net.device_status(stream()) == (nb.OK, 0)
    net.close()


def test_infer_and_decide_dev_equal_host_forms_and_read_n_specular_on_device():
    torch = torch_cuda()
    max_n, n = 200_000, 150_001
    net = make_net(precision=nb.PREC_FP16, max_queue=max_n)
    random_params(net, 72, table_scale=0.5, mlp_scale=0.15)
    v = _poisoned(nb.synth(73, max_n), n, max_n)
    d = upload(v)
    dp = nb.default_decide(use_ceil=0)
    st_a, rr_a, st_b, rr_b = empty(3 * max_n), empty(max_n), empty(3 * max_n), empty(max_n)
    net.inference(soa(d), n, dp, st_a, rr_a, stream())
    net.inferDev(soa(d), _n_dev(n), max_n, dp, st_b, rr_b, stream())
    torch.cuda.synchronize()
    assert np.array_equal(host(rr_a)[:n].view(np.uint32), host(rr_b)[:n].view(np.uint32))
    assert np.array_equal(host(st_a)[:3 * n].view(np.uint32), host(st_b)[:3 * n].view(np.uint32))
    nspec = torch.tensor([777], dtype=torch.int32, device="cuda")
    cap = 9 * max_n
    a, b = _step_outputs(max_n, cap), _step_outputs(max_n, cap)
    net.decideEmit(rr_a, d["rnd"], n, n, 777, dp, a["norm"], a["split"], a["q"], cap, a["sz"],
                   stream=stream())
    net.decideEmitDev(rr_a, d["rnd"], _n_dev(n), max_n, n, 0, dp, b["norm"], b["split"], b["q"],
                      cap, b["sz"], n_specular_dev=nspec, stream=stream())
    torch.cuda.synchronize()
    ha, hb = _host_out(a, n), _host_out(b, n)
    for x, y in zip(ha[:4], hb[:4]):
        assert np.array_equal(x, y)
    net.close()


def test_count_above_max_is_clamped_and_flagged_and_zero_is_empty():
    torch = torch_cuda()
    max_n = 70_000
    net = make_net(precision=nb.PREC_FP16, max_queue=max_n)
    v = nb.synth(74, max_n)
    d = upload(v)
    dp = nb.default_decide()
    cap = 9 * max_n
    a, b = _step_outputs(max_n, cap), _step_outputs(max_n, cap)
    net.generateRRSNumber(soa(d), d["rnd"], max_n, max_n, 0, dp, a["st"], a["rrs"], a["norm"],
                          a["split"], a["q"], cap, a["sz"], stream())
    net.generateRRSNumberDev(soa(d), d["rnd"], _n_dev(max_n + 5000), max_n, max_n, 0, dp,
                             b["st"], b["rrs"], b["norm"], b["split"], b["q"], cap, b["sz"],
                             stream=stream())
    torch.cuda.synchronize()
    ha, hb = _host_out(a, max_n), _host_out(b, max_n)
    for x, y in zip(ha, hb):
        assert np.array_equal(x, y)
    rc, flags = net.device_status(stream())
    assert rc == nb.ERR_CAPACITY_OVERFLOW and flags == nb.DEV_OVERFLOW
    b["sz"].fill_(12345)
    net.generateRRSNumberDev(soa(d), d["rnd"], _n_dev(0), max_n, max_n, 0, dp, b["st"], b["rrs"],
                             b["norm"], b["split"], b["q"], cap, b["sz"], stream=stream())
    torch.cuda.synchronize()
    assert int(host(b["sz"], np.uint32)[0]) == 0
    assert net.device_status(stream()) == (nb.OK, 0)
    net.close()


def test_batched_dev_equals_batched_with_host_counts():
    torch = torch_cuda()
    maxc = [int(round(120_000 * 0.6 ** k)) for k in range(8)]
    counts = [c - (17 * k) % max(c, 1) // 3 for k, c in enumerate(maxc)]
    counts[5] = 0
    offs = np.concatenate([[0], np.cumsum(maxc)]).astype(np.int64)
    tot = int(offs[-1])
    net = make_net(precision=nb.PREC_FP16, max_queue=tot)
    random_params(net, 75, table_scale=0.5, mlp_scale=0.15)
    v = nb.synth(76, tot)
    d = upload(v)
    dp = nb.default_decide()
    caps = [9 * c for c in maxc]
    qoffs = np.concatenate([[0], np.cumsum(caps)]).astype(np.int64)
    seg_max = [nb.Segment(int(offs[k]), maxc[k], 100_000, 0, int(qoffs[k]), caps[k])
               for k in range(8)]
    seg_act = [nb.Segment(int(offs[k]), counts[k], 100_000, 0, int(qoffs[k]), caps[k])
               for k in range(8)]
    cnt = torch.tensor(counts, dtype=torch.int32, device="cuda")
    outs = []
    for dev_counts in (False, True):
        o = dict(st=empty(3 * tot), rrs=empty(tot), norm=empty(tot), split=empty(tot, "uint8"),
                 q=empty(int(qoffs[-1]), "int32"), sz=empty(8, "int32"))
        if dev_counts:
            net.generateRRSNumberBatchedDev(soa(d), d["rnd"], seg_max, cnt, dp, o["st"], o["rrs"],
                                            o["norm"], o["split"], o["q"], o["sz"], stream())
        else:
            net.generateRRSNumberBatched(soa(d), d["rnd"], seg_act, dp, o["st"], o["rrs"],
                                         o["norm"], o["split"], o["q"], o["sz"], stream())
        torch.cuda.synchronize()
        outs.append(o)
    a, b = outs
    sa, sb = host(a["sz"], np.uint32)[:8], host(b["sz"], np.uint32)[:8]
    assert np.array_equal(sa, sb) and sa[5] == 0
    for k in range(8):
        a0, a1 = int(offs[k]), int(offs[k]) + counts[k]
        for key in ("split", "rrs", "norm"):
            assert np.array_equal(host(a[key])[a0:a1].view(np.uint8),
                                  host(b[key])[a0:a1].view(np.uint8)), (k, key)
        q0 = int(qoffs[k])
        assert np.array_equal(host(a["q"])[q0:q0 + sa[k]], host(b["q"])[q0:q0 + sb[k]]), k
    assert net.device_status(stream()) == (nb.OK, 0)
    net.close()


def test_one_graph_of_the_device_sized_step_replays_at_two_counts():
    torch = torch_cuda()
    max_n = 180_000
    net = make_net(precision=nb.PREC_FP16, max_queue=max_n)
    random_params(net, 77, table_scale=0.5, mlp_scale=0.15)
    v = nb.synth(78, max_n)
    d = upload(v)
    dp = nb.default_decide()
    cap = 9 * max_n
    n_dev = _n_dev(max_n)
    g_out = _step_outputs(max_n, cap)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):   # warm-up outside the capture (first-launch attributes)
        net.generateRRSNumberDev(soa(d), d["rnd"], n_dev, max_n, max_n, 0, dp, g_out["st"],
                                 g_out["rrs"], g_out["norm"], g_out["split"], g_out["q"], cap,
                                 g_out["sz"], stream=side.cuda_stream)
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, capture_error_mode="thread_local"):
        s = torch.cuda.current_stream().cuda_stream
        net.generateRRSNumberDev(soa(d), d["rnd"], n_dev, max_n, max_n, 0, dp, g_out["st"],
                                 g_out["rrs"], g_out["norm"], g_out["split"], g_out["q"], cap,
                                 g_out["sz"], stream=s)
    for n in (123_457, 179_999):
        n_dev.fill_(n)
        g.replay()
        torch.cuda.synchronize()
        ref = _step_outputs(max_n, cap)
        net.generateRRSNumber(soa(d), d["rnd"], n, max_n, 0, dp, ref["st"], ref["rrs"],
                              ref["norm"], ref["split"], ref["q"], cap, ref["sz"], stream())
        torch.cuda.synchronize()
        ha, hb = _host_out(ref, n), _host_out(g_out, n)
        for x, y in zip(ha, hb):
            assert np.array_equal(x, y), n
    del g
    assert net.device_status(stream()) == (nb.OK, 0)
    net.close()


def test_path_traced_frame_with_device_sizes_only_equals_host_sized_frame():
    """camera rays -> per bounce: trace, shade (device vertex count), the NRRS step on the
    device-sized queue, scatter and shadow rays (device queue size); nothing is read back
    between bounces. The film equals, bit for bit, the frame whose step takes the count read
    back to the host (the reference's pattern)."""
    torch = torch_cuda()
    from test_gpu_render import empty_hits, empty_rays, empty_shadow, empty_vertices
    vtx, tri, mat, mats, env = nb.synth_scene(8, n_boxes=40)
    gs = nb.Scene(vtx, tri, mat, mats, env)
    cam = nb.room_camera(96, 64)
    P = cam.width * cam.height
    cap = 6 * P
    net = make_net(precision=nb.PREC_FP16, max_queue=cap)
    random_params(net, 79, table_scale=0.5, mlp_scale=0.15)
    dp = nb.default_decide()
    rnd = torch.from_numpy(np.random.default_rng(80).random(cap, dtype=np.float32)).cuda()

    def frame(device_sizes: bool):
        s = stream()
        film = torch.zeros((P, 9), dtype=torch.int64, device="cuda")
        rays, hits = empty_rays(cap), empty_hits(cap)
        verts, shadow = empty_vertices(cap), empty_shadow(cap)
        scratch = torch.zeros(nb.shade_scratch_bytes(cap), dtype=torch.uint8, device="cuda")
        n_rays = torch.tensor([P], dtype=torch.int32, device="cuda")
        n_vert, qsize = (torch.zeros(1, dtype=torch.int32, device="cuda") for _ in range(2))
        o = _step_outputs(cap, cap)
        vsoa = nb.vertex_soa(verts["pos"], verts["wi"], verts["normal"], verts["roughness"],
                             verts["albedo"], verts["thp"], verts["depth"])
        R, H = nb.soa(nb.RaySoA, rays), nb.soa(nb.HitSoA, hits)
        V, S = nb.soa(nb.PathVertices, verts), nb.soa(nb.ShadowSoA, shadow)
        nb.camera_rays(cam, 0, 99, R, s)
        reads = 0
        for depth in range(5):
            nb.trace(gs, R, n_rays, cap, H, s)
            nb.shade(gs, R, H, n_rays, cap, depth, film, None, V, n_vert, scratch, s)
            if device_sizes:
                net.generateRRSNumberDev(vsoa, rnd, n_vert, cap, P, 0, dp, o["st"], o["rrs"],
                                         o["norm"], o["split"], o["q"], cap, o["sz"], stream=s)
            else:
                nv = int(host(n_vert)[0])
                reads += 1
                net.generateRRSNumber(vsoa, rnd, nv, P, 0, dp, o["st"], o["rrs"], o["norm"],
                                      o["split"], o["q"], cap, o["sz"], s)
            nb.scatter(gs, V, o["norm"], o["q"], o["sz"], cap, depth, 5, R, S, s)
            nb.trace_shadow(gs, S, o["sz"], cap, film, None, s)
            n_rays.copy_(o["sz"])
        img = torch.zeros((P, 3), device="cuda")
        nb.film_resolve(film, P, 1.0, img, s)
        torch.cuda.synchronize()
        return host(img).copy(), host(film).copy(), reads

    img_h, film_h, reads_h = frame(False)
    img_d, film_d, reads_d = frame(True)
    assert reads_h > 0 and reads_d == 0
    assert np.array_equal(film_h, film_d)
    assert np.array_equal(img_h.view(np.uint32), img_d.view(np.uint32))
    assert float(img_h.mean()) > 0
    assert net.device_status(stream()) == (nb.OK, 0)
    gs.close()
    net.close()
