"""A whole training frame through the library, as the reference's integrator runs one
(renderInternal<true>, integrator.cpp:1485-1644, with trainStep's data side, :2572-2605): camera
rays; per bounce trace, shade, the emitted radiance recorded at the rays' nodes, the decision on
the vertices, the vertices recorded as path nodes (in place on their node indices), scatter,
shadow rays and their radiance recorded; then the training batch from the nodes and the rendered
image, the per-pixel sample counts and the sample weights. The same frame runs in the C
restatement (HostScene + HostNodes), and every node field, the batch, the counts and the weights
must agree bit for bit. The GPU batch then feeds the training step, whose losses must equal the
oracle's on the oracle's batch."""
from __future__ import annotations

import numpy as np
import pytest

import nrrs_b200 as nb
import oracle as O
from gpu_util import host, make_net, random_params, stream, torch_cuda
from test_gpu_records import NODE_FIELDS, GpuNodes, assert_same_batch
from test_gpu_render import (empty_hits, empty_rays, empty_shadow, empty_vertices, same,
                             scene_pair, to_host)

pytestmark = pytest.mark.gpu


def run_training_frame(closed):
    """The frame on the GPU and in the C restatement; returns the GPU node block, the host
    nodes, the rendered image (RGBA per pixel), the pixel count and the node capacity."""
    torch = torch_cuda()
    gs, hs = scene_pair(11, boxes=60, closed=closed)
    cam = nb.room_camera(48, 36, inside=closed)
    n = cam.width * cam.height
    cap = 4 * n
    bounces, seed = 4, 21
    node_cap = 12 * n
    g = GpuNodes(node_cap, cap)
    hn = O.HostNodes(node_cap)

    film = torch.zeros((n, 9), dtype=torch.int64, device="cuda")
    hfilm = np.zeros((n, 9), np.int64)
    rays, hits = empty_rays(cap), empty_hits(cap)
    verts, shadow = empty_vertices(cap), empty_shadow(cap)
    contrib = torch.zeros((cap, 3), device="cuda")
    scontrib = torch.zeros((cap, 3), device="cuda")
    scratch = torch.zeros(nb.shade_scratch_bytes(cap), dtype=torch.uint8, device="cuda")
    n_rays = torch.tensor([n], dtype=torch.int32, device="cuda")
    n_vert = torch.zeros(1, dtype=torch.int32, device="cuda")
    qsize = torch.zeros(1, dtype=torch.int32, device="cuda")
    queue = torch.zeros(cap, dtype=torch.int32, device="cuda")
    rrs_norm = torch.zeros(cap, device="cuda")
    nb.camera_rays(cam, 0, seed, nb.soa(nb.RaySoA, rays), stream())
    hr = hs.camera_rays(cam, 0, seed)
    dp = nb.default_decide(clamp_max=4.0)
    rng = np.random.default_rng(seed)
    recorded = 0
    for depth in range(bounces):
        nr = int(host(n_rays)[0])
        nb.trace(gs, nb.soa(nb.RaySoA, rays), n_rays, cap, nb.soa(nb.HitSoA, hits), stream())
        hh = hs.trace(hr)
        nb.shade(gs, nb.soa(nb.RaySoA, rays), nb.soa(nb.HitSoA, hits), n_rays, cap, depth, film,
                 contrib, nb.soa(nb.PathVertices, verts), n_vert, scratch, stream())
        hv, hc = hs.shade(hr, hh, depth, hfilm)
        # handleEmissiveHit / handleMiss: the radiance reaches the node the ray left
        g.pn.recordRadiance(rays["node"], contrib, nr, stream())
        hn.record_radiance(hr["node"], hc)
        nv = int(host(n_vert)[0])
        assert nv == len(hv["pos"])
        if nv == 0:
            break
        # the decision (the library's, on synthetic factors) between the bounces
        f = rng.uniform(0.3, 2.5, nv).astype(np.float32)
        rnd = rng.uniform(size=nv).astype(np.float32)
        split = torch.zeros(nv, dtype=torch.uint8, device="cuda")
        rc = nb.decide_emit_noalloc(torch.from_numpy(f).cuda(), torch.from_numpy(rnd).cuda(), nv,
                                    nv, 0, dp, rrs_norm, split, queue, cap, qsize, None, stream())
        assert rc == 0
        o = O.decide_emit(f, rnd, nv, 0, dp, capacity=cap, shift_n=nb.NOALLOC_MAX_N)
        # recordNode for the vertices that continue, in place on their node indices
        record = (split > 0).to(torch.uint8)
        vs = nb.vertex_soa(verts["pos"], verts["wi"], verts["normal"], verts["roughness"],
                           verts["albedo"], verts["thp"], verts["depth"])
        g.pn.recordNode(vs, verts["node"], verts["pixel"], rrs_norm, record, nv, verts["node"],
                        stream())
        hb = {k: np.ascontiguousarray(hv[k]) for k in ("pos", "wi", "normal", "albedo",
                                                        "roughness", "thp", "depth", "pixel")}
        hb["parent"] = np.ascontiguousarray(hv["node"], np.int32)
        hb["rrs"] = np.ascontiguousarray(o["rrs_norm"][:nv], np.float32)
        hb["record"] = (o["split"] > 0).astype(np.uint8)
        hv = dict(hv)
        hv["node"] = hn.record_nodes(hb)
        assert host(verts["node"])[:nv].tolist() == hv["node"].tolist()
        recorded += int((hv["node"] >= 0).sum())
        # scatter and shadow rays; the shadow radiance reaches the new nodes
        nb.scatter(gs, nb.soa(nb.PathVertices, verts), rrs_norm, queue, qsize, cap, depth, seed,
                   nb.soa(nb.RaySoA, rays), nb.soa(nb.ShadowSoA, shadow), stream())
        hr, hsh = hs.scatter(hv, o["rrs_norm"], o["queue"], depth, seed)
        nq = int(host(qsize)[0])
        same(to_host(rays, nq), hr, ("origin", "dir", "thp", "pdf", "pixel", "node"))
        nb.trace_shadow(gs, nb.soa(nb.ShadowSoA, shadow), qsize, cap, film, scontrib, stream())
        hco = hs.shadow(hsh, hfilm)
        g.pn.recordRadiance(shadow["node"], scontrib, nq, stream())
        hn.record_radiance(hsh["node"], hco)
        n_rays.copy_(qsize)
    assert recorded > n
    assert host(film).tobytes() == hfilm.tobytes()
    himg = hs.resolve(hfilm, 1.0)
    image = np.concatenate([himg, np.ones((n, 1), np.float32)], axis=1)
    return g, hn, image, n, node_cap


@pytest.mark.parametrize("closed", [False, True], ids=["open", "closed"])
def test_gpu_training_frame_matches_oracle(closed):
    torch = torch_cuda()
    g, hn, image, n, node_cap = run_training_frame(closed)

    # the node buffers
    size, dropped, flags = g.pn.status(stream())
    assert (size, dropped, flags) == (hn.size, hn.dropped, hn.status)
    assert dropped == 0 and flags == 0
    # trainStep's data side: the batch, the per-pixel counts, the weights
    prm = nb.default_train_data_params(copy_rrs_node=1, dedupe_rrs_target=1)
    batch, total, counts, weights = g.generate(prm, node_cap, image=image, n_pixels=n)
    for k in NODE_FIELDS:
        assert g.field(k, hn.size).tobytes() == hn.a[k][:hn.size].tobytes(), k
    hcounts = np.zeros(n, np.uint32)
    hbatch, htotal = hn.generate(prm, node_cap, image=image, n_pixels=n, pixel_samples=hcounts)
    assert total == htotal > 0
    assert_same_batch(batch, hbatch)
    assert counts.tobytes() == hcounts.tobytes()
    assert weights.tobytes() == O.sample_weights(hbatch["pixel"], hcounts, n).tobytes()

    # the batch trains the networks: the library's FP32 losses on the GPU batch equal the
    # oracle's FP64 losses on the oracle's batch
    m = min(total, 8192)
    net = make_net(max_train=1 << 13, step=3, log2_hashmap_size=15, precision=nb.PREC_FP32)
    p0 = random_params(net, 5, table_scale=0.5, mlp_scale=0.15)
    d = {k: torch.from_numpy(np.ascontiguousarray(
        batch[k][:m].view(np.int32) if batch[k].dtype == np.uint32 else batch[k][:m])).cuda()
        for k in ("pos", "wi", "normal", "roughness", "albedo", "thp", "depth", "ref_mean",
                  "target")}
    loss = torch.zeros(2, dtype=torch.float64, device="cuda")
    net.trainGrads(nb.vertex_soa(d["pos"], d["wi"], d["normal"], d["roughness"], d["albedo"],
                                 d["thp"], d["depth"], d["ref_mean"]), d["target"], m, loss,
                   stream())
    ob = {k: np.ascontiguousarray(hbatch[k][:m]) for k in hbatch}
    _, l64 = O.train_grads(net.config, p0, ob, ob["target"], "f64")
    assert host(loss) == pytest.approx(l64, rel=1e-4)
    net.close()


def test_gpu_training_frames_learn():
    """The loop closes: frames rendered through the library (trace, shade, records, the step
    with the network's own factors, scatter, shadow), each one's batch trains the networks, and
    the StatNet loss on fresh frames falls as the frames go by."""
    torch = torch_cuda()
    gs, _ = scene_pair(11, boxes=60, closed=True)
    cam = nb.room_camera(64, 48, inside=True)
    n = cam.width * cam.height
    cap = 4 * n
    node_cap = 12 * n
    net = make_net(precision=nb.PREC_FP16, max_queue=cap, max_train=1 << 14)
    net.setStep(3)
    dp = nb.default_decide(clamp_min=1.0)
    g = GpuNodes(node_cap, cap)
    f = lambda *s: torch.zeros(*s, device="cuda")                       # noqa: E731
    i = lambda *s: torch.zeros(*s, dtype=torch.int32, device="cuda")    # noqa: E731
    rays, hits = empty_rays(cap), empty_hits(cap)
    verts, shadow = empty_vertices(cap), empty_shadow(cap)
    contrib, scontrib, film = f(cap, 3), f(cap, 3), torch.zeros((n, 9), dtype=torch.int64,
                                                                 device="cuda")
    scratch = torch.zeros(nb.shade_scratch_bytes(cap), dtype=torch.uint8, device="cuda")
    n_rays, n_vert, qsize = i(1), i(1), i(1)
    stats, rrs, rrs_norm = f(3 * cap), f(cap), f(cap)
    split = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    queue = i(cap)
    img = f(n, 3)
    widths = {"pos": 3, "wi": 3, "normal": 3, "albedo": 3, "roughness": 1, "thp": 3, "depth": 1,
              "ref_mean": 1, "target": 3, "rrs_target": 1, "pixel": 1}
    batch = {k: (f(node_cap, w) if w > 1 else f(node_cap)) if k not in ("depth", "pixel")
             else i(node_cap) for k, w in widths.items()}
    tb = nb.train_batch(**batch)
    counts, size_d = i(n), i(1)
    prm = nb.default_train_data_params(copy_rrs_node=1, dedupe_rrs_target=1)
    tsoa = nb.vertex_soa(batch["pos"], batch["wi"], batch["normal"], batch["roughness"],
                         batch["albedo"], batch["thp"], batch["depth"], batch["ref_mean"])
    loss = torch.zeros(2, dtype=torch.float64, device="cuda")
    R, Hh, V, S = (nb.soa(nb.RaySoA, rays), nb.soa(nb.HitSoA, hits),
                   nb.soa(nb.PathVertices, verts), nb.soa(nb.ShadowSoA, shadow))
    vsoa = nb.vertex_soa(verts["pos"], verts["wi"], verts["normal"], verts["roughness"],
                         verts["albedo"], verts["thp"], verts["depth"])
    losses = []
    for frame in range(40):
        g.pn.reset(stream())
        film.zero_()
        nb.camera_rays(cam, frame, 77, R, stream())
        n_rays.fill_(n)
        n_cur = n
        for depth in range(4):
            nb.trace(gs, R, n_rays, cap, Hh, stream())
            nb.shade(gs, R, Hh, n_rays, cap, depth, film, contrib, V, n_vert, scratch, stream())
            g.pn.recordRadiance(rays["node"], contrib, n_cur, stream())
            nv = int(host(n_vert)[0])
            if nv == 0:
                break
            rnd = torch.rand(nv, device="cuda", generator=torch.Generator(device="cuda")
                             .manual_seed(1000 * frame + depth))
            net.generateRRSNumber(vsoa, rnd, nv, n, 0, dp, stats, rrs, rrs_norm, split, queue,
                                  cap, qsize, stream())
            g.pn.recordNode(vsoa, verts["node"], verts["pixel"], rrs_norm, split, nv,
                            verts["node"], stream())
            nb.scatter(gs, V, rrs_norm, queue, qsize, cap, depth, 500 + frame, R, S, stream())
            nb.trace_shadow(gs, S, qsize, cap, film, scontrib, stream())
            n_cur = int(host(qsize)[0])
            g.pn.recordRadiance(shadow["node"], scontrib, n_cur, stream())
            n_rays.copy_(qsize)
        nb.film_resolve(film, n, 1.0, img, stream())
        counts.zero_()
        g.pn.generate_training_data(prm, tb, node_cap, size_d, image=img, image_channels=3,
                                    n_pixels=n, pixel_samples=counts, stream=stream())
        m = min(int(host(size_d)[0]), 1 << 14)
        m -= m % 256
        assert m >= 1024
        net.train(tsoa, batch["target"], m, loss, stream())
        losses.append(float(host(loss)[0]))
    first, last = np.mean(losses[:5]), np.mean(losses[-5:])
    assert np.isfinite(losses).all()
    assert last < 0.7 * first, (first, last, losses)
    rc, flags = net.device_status(stream())
    assert rc == nb.OK and flags == 0
    net.close()


def test_gpu_ubs_search_drives_rendered_frames():
    """The per-depth strategy search on real frames: at the start of each frame the search
    moves to its next state. The renderer then runs, depth by depth, the factor source it asks
    for (the RRS step with ADRRS or RRSNet factors, or the fixed-RR scatter when it runs no
    inference). nrrs_ubs_error scores the frame against a reference image, and the frame's
    time and error sum go back to the search. The library's search and the restatement make the
    same choices every frame and end on the same best string, in 3^d + 3 frames."""
    import ctypes as C

    from schedule import UBSRef

    torch = torch_cuda()
    gs, _ = scene_pair(9, boxes=30)
    cam = nb.room_camera(40, 30)
    n = cam.width * cam.height
    cap = 4 * n
    max_depth = 2
    net = make_net(precision=nb.PREC_FP16, max_queue=cap)
    random_params(net, 4, table_scale=0.5, mlp_scale=0.1)
    net.setStep(3)
    f = lambda *s: torch.zeros(*s, device="cuda")                       # noqa: E731
    i = lambda *s: torch.zeros(*s, dtype=torch.int32, device="cuda")    # noqa: E731
    rays, hits = empty_rays(cap), empty_hits(cap)
    verts, shadow = empty_vertices(cap), empty_shadow(cap)
    film = torch.zeros((n, 9), dtype=torch.int64, device="cuda")
    scratch = torch.zeros(nb.shade_scratch_bytes(cap), dtype=torch.uint8, device="cuda")
    n_rays, n_vert, qsize = i(1), i(1), i(1)
    stats, rrs, rrs_norm = f(3 * cap), f(cap), f(cap)
    split = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    queue = i(cap)
    R, Hh, V, S = (nb.soa(nb.RaySoA, rays), nb.soa(nb.HitSoA, hits),
                   nb.soa(nb.PathVertices, verts), nb.soa(nb.ShadowSoA, shadow))
    vsoa = nb.vertex_soa(verts["pos"], verts["wi"], verts["normal"], verts["roughness"],
                         verts["albedo"], verts["thp"], verts["depth"])

    def frame(sample, choose):
        """one frame; choose(depth) -> None (fixed RR) or a factor source"""
        film.zero_()
        nb.camera_rays(cam, sample, 5, R, stream())
        n_rays.fill_(n)
        used = []
        for depth in range(3):
            nb.trace(gs, R, n_rays, cap, Hh, stream())
            nb.shade(gs, R, Hh, n_rays, cap, depth, film, None, V, n_vert, scratch, stream())
            nv = int(host(n_vert)[0])
            if nv == 0:
                break
            src = choose(depth)
            used.append(src)
            if src is None:
                nb.scatter_fixed_rr(gs, V, n_vert, cap, 0.8, depth, 90 + sample, R, S, stream())
                qsize.copy_(n_vert)
            else:
                rnd = torch.rand(nv, device="cuda", generator=torch.Generator(device="cuda")
                                 .manual_seed(sample * 10 + depth))
                dp = nb.default_decide(factor_source=src, clamp_min=0.5)
                net.generateRRSNumber(vsoa, rnd, nv, n, 0, dp, stats, rrs, rrs_norm, split,
                                      queue, cap, qsize, stream())
                nb.scatter(gs, V, rrs_norm, queue, qsize, cap, depth, 90 + sample, R, S, stream())
            nb.trace_shadow(gs, S, qsize, cap, film, None, stream())
            n_rays.copy_(qsize)
        img = f(n, 3)
        nb.film_resolve(film, n, 1.0, img, stream())
        return img, used

    # the reference image: the mean of 16 frames with fixed Russian roulette
    ref = f(n, 3)
    for k in range(16):
        img, _ = frame(1000 + k, lambda d: None)
        ref += img / 16
    pe = nb.default_pixel_error_params(cam.width, cam.height)
    err = f(n)
    esum = torch.zeros(C.sizeof(nb.ErrorSum), dtype=torch.uint8, device="cuda")

    lib, oracle = nb.UBS(max_depth), UBSRef(max_depth)
    lib.UBSResetAndBeginSearch()
    oracle.begin()
    t, frames = 0.0, 0
    while True:
        a, b = lib.UBSNextState(), oracle.next_state()
        assert a == b
        if not a:
            break

        def choose(depth):
            infer, src = lib.isInferMode(depth)
            assert (infer, src) == oracle.need_infer(depth, 1, 0.05, 8.0, 6, 1)
            return src if infer else None

        img, used = frame(frames, choose)
        nb.ubs_error(pe, img, 1, ref, 3, err, esum, stream())
        err_sum = float(host(esum)[28:32].view(np.float32)[0])
        assert np.isfinite(err_sum) and err_sum > 0
        t += 0.02 + 0.001 * len([u for u in used if u is not None])   # the frame's clock
        lib.UBSAnalyseFrame(t, err_sum, n)
        oracle.analyse(t, err_sum, n)
        frames += 1
        assert frames < 50
    assert frames == 3 ** max_depth + 3
    best, eff = lib.best()
    assert best == oracle.array[:max_depth] and np.float32(eff) == oracle.best_eff
    assert not lib.searching
    net.close()


@pytest.mark.parametrize("prec", [nb.PREC_FP32, nb.PREC_FP16], ids=["fp32", "fp16"])
def test_gpu_records_batch_feeds_weighted_training_step(prec):
    """trainStep end to end on the device: the training batch built from this frame's nodes
    (with the per-pixel error arrays and sample counts of the error image gathered into it, the
    -1 RRSNet targets of later siblings, the sample weights and the error sum) goes straight into
    nrrs_train_step_batch with the reference's shipped loss settings (gamma 0.01 / 0.05 / 0 /
    0.01, clamp on at 10). Losses and gradients equal the FP64 oracle's weighted losses on the
    oracle's own batch."""
    torch = torch_cuda()
    g, hn, image, n, node_cap = run_training_frame(False)
    rng = np.random.default_rng(90)
    err = rng.uniform(0.0, 3.0, 2 * n).astype(np.float32)
    err[rng.random(2 * n) < 0.02] = 40.0          # a few pixels far above the clamp
    spp = rng.integers(1, 9, n).astype(np.float32)
    d_err, d_spp = torch.from_numpy(err).cuda(), torch.from_numpy(spp).cuda()
    prm = nb.default_train_data_params(copy_rrs_node=1, dedupe_rrs_target=1,
                                       error_per_pixel=d_err.data_ptr(),
                                       samples_per_patch=d_spp.data_ptr())
    cap = node_cap
    f32 = lambda *s: torch.zeros(*s, dtype=torch.float32, device="cuda")   # noqa: E731
    i32 = lambda *s: torch.zeros(*s, dtype=torch.int32, device="cuda")     # noqa: E731
    out = {"pos": f32(cap, 3), "wi": f32(cap, 3), "normal": f32(cap, 3), "albedo": f32(cap, 3),
           "roughness": f32(cap), "thp": f32(cap, 3), "depth": i32(cap), "ref_mean": f32(cap),
           "target": f32(cap, 3), "rrs_target": f32(cap), "pixel": i32(cap), "error": f32(cap),
           "error_for_avg": f32(cap), "number_samples": f32(cap)}
    counts = i32(n)
    size = i32(1)
    img = torch.from_numpy(image).cuda()
    g.pn.generate_training_data(prm, nb.train_batch(**out), cap, size, image=img,
                                image_channels=4, n_pixels=n, pixel_samples=counts,
                                stream=stream())
    weights = f32(cap)
    nb.calculate_sample_weight(out["pixel"], counts, n, size, cap, weights, stream())
    total = int(host(size)[0])
    m = min(total, 8192)
    assert m > 1000
    esum = float(np.sum(err[n:].astype(np.float64)))
    d_esum = torch.tensor([esum], dtype=torch.float32, device="cuda")
    lp = nb.default_loss_params(gamma1=0.01, gamma2=0.05, gamma3=0.0, gamma4=0.01, clamp_on=1,
                                clamp_max=10.0, n_pixels=n)
    net = make_net(max_train=1 << 13, step=3, log2_hashmap_size=15, precision=prec)
    p0 = random_params(net, 5, table_scale=0.5, mlp_scale=0.15)
    loss = torch.zeros(2, dtype=torch.float64, device="cuda")
    net.trainStepBatch(nb.train_batch(**out), m, weights, d_esum, lp, loss, stream())
    torch.cuda.synchronize()
    gg = net.get_grads().astype(np.float64)
    rc, flags = net.device_status(stream())
    assert rc == nb.OK and flags == 0

    # the oracle's batch, weights and error sum from the C restatement of the same frame
    prm_h = nb.default_train_data_params(copy_rrs_node=1, dedupe_rrs_target=1,
                                         error_per_pixel=err.ctypes.data,
                                         samples_per_patch=spp.ctypes.data)
    hcounts = np.zeros(n, np.uint32)
    hbatch, htotal = hn.generate(prm_h, node_cap, image=image, n_pixels=n, pixel_samples=hcounts)
    assert htotal == total
    hw = O.sample_weights(hbatch["pixel"], hcounts, n)
    ob = {k: np.ascontiguousarray(hbatch[k][:m]) for k in hbatch}
    assert (ob["rrs_target"] < 0).any() and (ob["error"] > 0).any()
    for k in ("error", "error_for_avg", "number_samples", "rrs_target", "thp", "target"):
        assert host(out[k]).reshape(cap, -1)[:m].tobytes() == ob[k].reshape(m, -1).tobytes(), k
    ob["sample_weight"] = hw[:m]
    w, keep = O.loss_weights(ob, gammas=(0.01, 0.05, 0.0, 0.01), clamp_on=1, clamp_max=10.0,
                             error_mean=float(np.float32(esum)) / n)
    g64, l64 = O.train_grads(net.config, p0, ob, ob["target"], "f64", weights=w)
    l = host(loss)
    assert l[0] == pytest.approx(l64[0], rel=1e-4 if prec == nb.PREC_FP32 else 1e-3)
    assert l[1] == pytest.approx(l64[1], rel=1e-4 if prec == nb.PREC_FP32 else 2e-3)
    ntab, nst, nrr = net.param_layout()
    bars = ({"table": 2e-4, "statnet": 2e-4, "rrsnet": 2e-4} if prec == nb.PREC_FP32 else
            {"table": 5e-2, "statnet": 2e-2, "rrsnet": 2e-2})
    for name, sl in (("table", slice(0, ntab)), ("statnet", slice(ntab, ntab + nst)),
                     ("rrsnet", slice(ntab + nst, ntab + nst + nrr))):
        e = np.linalg.norm(gg[sl] - g64[sl]) / max(np.linalg.norm(g64[sl]), 1e-30)
        assert e < bars[name], (name, e)
    net.close()
