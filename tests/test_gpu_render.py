"""GPU parity of the wavefront steps around the NRRS step (nrrs_camera_rays, nrrs_trace,
nrrs_shade, nrrs_scatter, nrrs_scatter_fixed_rr, nrrs_trace_shadow, nrrs_film_resolve) against
the C restatement, bit for bit: BVH closest hits against brute force on camera rays and random
rays, whole frames with the emitted queue of the library's decision (or fixed Russian roulette)
between bounces, and the film. Also checks that splitting and killing by the RRS factors leave
the image unbiased."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import nrrs_b200 as nb
import oracle as O
from gpu_util import host, stream, torch_cuda

pytestmark = pytest.mark.gpu

V3 = ("origin", "dir", "thp", "pos", "wi", "normal", "albedo", "contrib")


def dev_dict(d: dict):
    torch = torch_cuda()
    out = {}
    for k, a in d.items():
        a = np.ascontiguousarray(a)
        if a.dtype == np.uint32:
            a = a.view(np.int32)
        out[k] = torch.from_numpy(a).cuda()
    return out


def empty_rays(n):
    torch = torch_cuda()
    f = lambda *s: torch.zeros(*s, dtype=torch.float32, device="cuda")  # noqa: E731
    i = lambda *s: torch.zeros(*s, dtype=torch.int32, device="cuda")   # noqa: E731
    return {"origin": f(n, 3), "dir": f(n, 3), "thp": f(n, 3), "pdf": f(n), "pixel": i(n),
            "node": i(n)}


def empty_hits(n):
    torch = torch_cuda()
    return {"prim": torch.zeros(n, dtype=torch.int32, device="cuda"),
            "t": torch.zeros(n, device="cuda"), "u": torch.zeros(n, device="cuda"),
            "v": torch.zeros(n, device="cuda")}


def empty_vertices(n):
    torch = torch_cuda()
    f = lambda *s: torch.full(s, -9.0, dtype=torch.float32, device="cuda")  # noqa: E731
    i = lambda *s: torch.zeros(*s, dtype=torch.int32, device="cuda")       # noqa: E731
    return {"pos": f(n, 3), "wi": f(n, 3), "normal": f(n, 3), "albedo": f(n, 3),
            "roughness": f(n), "thp": f(n, 3), "depth": i(n), "pixel": i(n), "node": i(n)}


def empty_shadow(n):
    torch = torch_cuda()
    f = lambda *s: torch.zeros(*s, dtype=torch.float32, device="cuda")  # noqa: E731
    i = lambda *s: torch.zeros(*s, dtype=torch.int32, device="cuda")   # noqa: E731
    return {"origin": f(n, 3), "dir": f(n, 3), "tmax": f(n), "contrib": f(n, 3), "pixel": i(n),
            "node": i(n)}


def to_host(d: dict, n: int):
    out = {}
    for k, t in d.items():
        a = host(t)[:n]
        out[k] = a.view(np.uint32) if k in ("prim", "pixel", "depth") else a
    return out


def same(a, b, keys):
    for k in keys:
        assert np.asarray(a[k]).tobytes() == np.asarray(b[k]).tobytes(), k


def scene_pair(seed=1, boxes=60, closed=False):
    v, t, m, ma, e = nb.synth_scene(seed, n_boxes=boxes, closed=closed)
    return nb.Scene(v, t, m, ma, e), O.HostScene(v, t, m, ma, e)


def test_gpu_trace_matches_brute_force():
    torch = torch_cuda()
    gs, hs = scene_pair(2, boxes=250)
    nn, nl, depth = gs.info()
    assert nl == 2 and nn > 100 and depth < 32
    cam = nb.room_camera(160, 120)
    n = 160 * 120
    rays = empty_rays(2 * n)
    nb.camera_rays(cam, 3, 11, nb.soa(nb.RaySoA, rays), stream())
    r_cam = hs.camera_rays(cam, 3, 11)
    got = to_host(rays, n)
    same(got, r_cam, ("origin", "dir", "thp", "pdf", "pixel", "node"))
    # and random rays from inside the room
    rng = np.random.default_rng(0)
    o = rng.uniform(0.02, 0.98, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r_rand = {"origin": o, "dir": d, "thp": np.ones((n, 3), np.float32),
              "pdf": np.zeros(n, np.float32), "pixel": np.zeros(n, np.uint32),
              "node": np.full(n, -1, np.int32)}
    dr = dev_dict(r_rand)
    for k in r_rand:
        rays[k][n:2 * n].copy_(dr[k])
    r_all = {k: np.concatenate([r_cam[k], r_rand[k]]) for k in r_cam}
    hits = empty_hits(2 * n)
    cnt = torch.tensor([2 * n], dtype=torch.int32, device="cuda")
    nb.trace(gs, nb.soa(nb.RaySoA, rays), cnt, 2 * n, nb.soa(nb.HitSoA, hits), stream())
    want = hs.trace(r_all)
    got = to_host(hits, 2 * n)
    same(got, want, ("prim", "t", "u", "v"))
    assert (want["prim"] != 0xffffffff).mean() > 0.5


def run_frame_pair(gs, hs, cam, seed, bounces, factors, fixed_rr=None, sorted_trace=False):
    """One frame on the GPU and in the oracle, bounce by bounce, with the emitted queue of the
    library's decision (nrrs_decide_emit_noalloc) on the given factor generator between them, or
    at the depths in fixed_rr ({depth: rr}) the fixed Russian-roulette scatter; every array
    compared as it is produced. Returns both films."""
    torch = torch_cuda()
    n = cam.width * cam.height
    cap = 4 * n
    film = torch.zeros((n, 9), dtype=torch.int64, device="cuda")
    hfilm = np.zeros((n, 9), np.int64)
    rays, hits = empty_rays(cap), empty_hits(cap)
    verts, shadow = empty_vertices(cap), empty_shadow(cap)
    contrib = torch.zeros((cap, 3), device="cuda")
    scontrib = torch.zeros((cap, 3), device="cuda")
    scratch = torch.zeros(nb.shade_scratch_bytes(cap), dtype=torch.uint8, device="cuda")
    tscratch = torch.zeros(nb.trace_scratch_bytes(cap), dtype=torch.uint8, device="cuda")
    n_rays = torch.tensor([n], dtype=torch.int32, device="cuda")
    n_vert = torch.zeros(1, dtype=torch.int32, device="cuda")
    qsize = torch.zeros(1, dtype=torch.int32, device="cuda")
    queue = torch.zeros(cap, dtype=torch.int32, device="cuda")
    rrs_norm = torch.zeros(cap, device="cuda")
    nb.camera_rays(cam, 0, seed, nb.soa(nb.RaySoA, rays), stream())
    hr = hs.camera_rays(cam, 0, seed)
    dp = nb.default_decide(clamp_max=4.0)
    rng = np.random.default_rng(seed)
    for depth in range(bounces):
        nr = int(host(n_rays)[0])
        if sorted_trace:
            nb.trace_sorted(gs, nb.soa(nb.RaySoA, rays), n_rays, cap, nb.soa(nb.HitSoA, hits),
                            tscratch, stream())
        else:
            nb.trace(gs, nb.soa(nb.RaySoA, rays), n_rays, cap, nb.soa(nb.HitSoA, hits), stream())
        hh = hs.trace(hr)
        same(to_host(hits, nr), hh, ("prim", "t", "u", "v"))
        nb.shade(gs, nb.soa(nb.RaySoA, rays), nb.soa(nb.HitSoA, hits), n_rays, cap, depth, film,
                 contrib, nb.soa(nb.PathVertices, verts), n_vert, scratch, stream())
        hv, hc = hs.shade(hr, hh, depth, hfilm)
        nv = int(host(n_vert)[0])
        assert nv == len(hv["pos"])
        same(to_host(verts, nv), hv, nb.PATH_VERTEX_FIELDS)
        assert host(contrib)[:nr].tobytes() == hc.tobytes()
        assert host(film).tobytes() == hfilm.tobytes()
        if nv == 0:
            break
        if fixed_rr and depth in fixed_rr:
            rr = fixed_rr[depth]
            nb.scatter_fixed_rr(gs, nb.soa(nb.PathVertices, verts), n_vert, cap, rr, depth, seed,
                                nb.soa(nb.RaySoA, rays), nb.soa(nb.ShadowSoA, shadow), stream())
            hr, hsh = hs.scatter_fixed_rr(hv, rr, depth, seed)
            same(to_host(rays, nv), hr, ("origin", "dir", "thp", "pdf", "pixel", "node"))
            same(to_host(shadow, nv), hsh, ("origin", "dir", "tmax", "contrib", "pixel", "node"))
            kept = (hr["thp"] != 0).any(axis=1).mean()
            assert rr == 1.0 or 0.0 < kept < 1.0
            nb.trace_shadow(gs, nb.soa(nb.ShadowSoA, shadow), n_vert, cap, film, scontrib,
                            stream())
            hco = hs.shadow(hsh, hfilm)
            assert host(scontrib)[:nv].tobytes() == hco.tobytes()
            assert host(film).tobytes() == hfilm.tobytes()
            n_rays.copy_(n_vert)
            continue
        # the emitted queue: the library's decision on synthetic factors (as nrrs_step would)
        f = factors(rng, nv).astype(np.float32)
        rnd = rng.uniform(size=nv).astype(np.float32)
        split = torch.zeros(nv, dtype=torch.uint8, device="cuda")
        rc = nb.decide_emit_noalloc(torch.from_numpy(f).cuda(), torch.from_numpy(rnd).cuda(), nv,
                                    nv, 0, dp, rrs_norm, split, queue, cap, qsize, None, stream())
        assert rc == 0
        o = O.decide_emit(f, rnd, nv, 0, dp, capacity=cap, shift_n=nb.NOALLOC_MAX_N)
        nq = int(host(qsize)[0])
        assert nq == o["total"] and host(queue)[:nq].view(np.uint32).tolist() == o["queue"].tolist()
        nb.scatter(gs, nb.soa(nb.PathVertices, verts), rrs_norm, queue, qsize, cap, depth, seed,
                   nb.soa(nb.RaySoA, rays), nb.soa(nb.ShadowSoA, shadow), stream())
        hr, hsh = hs.scatter(hv, o["rrs_norm"], o["queue"], depth, seed)
        same(to_host(rays, nq), hr, ("origin", "dir", "thp", "pdf", "pixel", "node"))
        same(to_host(shadow, nq), hsh, ("origin", "dir", "tmax", "contrib", "pixel", "node"))
        nb.trace_shadow(gs, nb.soa(nb.ShadowSoA, shadow), qsize, cap, film, scontrib, stream())
        hco = hs.shadow(hsh, hfilm)
        assert host(scontrib)[:nq].tobytes() == hco.tobytes()
        assert host(film).tobytes() == hfilm.tobytes()
        n_rays.copy_(qsize)
    img = torch.zeros((n, 3), device="cuda")
    nb.film_resolve(film, n, 1.0, img, stream())
    himg = hs.resolve(hfilm, 1.0)
    assert host(img).tobytes() == himg.tobytes()
    return host(img), himg


def test_gpu_frame_matches_oracle():
    gs, hs = scene_pair(3, boxes=40)
    cam = nb.room_camera(64, 48)
    img, _ = run_frame_pair(gs, hs, cam, 5, 4,
                            lambda rng, n: rng.uniform(0.3, 2.5, n))
    assert img.mean() > 0


def test_gpu_closed_room_frame_matches_oracle():
    """The render benchmark's kind of scene: a closed room seen from inside, where no ray
    escapes; three bounces with splitting and killing, traced in the sorted order."""
    gs, hs = scene_pair(7, boxes=120, closed=True)
    cam = nb.room_camera(320, 240, inside=True)   # 76,800 rays: the sorted trace sorts
    img, _ = run_frame_pair(gs, hs, cam, 9, 3, lambda rng, n: rng.uniform(0.3, 2.5, n),
                            sorted_trace=True)
    assert img.mean() > 0


def test_gpu_fixed_rr_depths_match_oracle():
    """Depths that run no inference (the strategy search's fixed-RR depths) scatter through the
    fixed Russian-roulette branch; mixed with RRS depths in one frame, bit for bit, including a
    training-style rr = 1 depth that keeps every vertex."""
    gs, hs = scene_pair(5, boxes=50)
    cam = nb.room_camera(56, 40)
    img, _ = run_frame_pair(gs, hs, cam, 13, 5, lambda rng, n: rng.uniform(0.3, 2.5, n),
                            fixed_rr={0: 0.8, 2: 1.0, 3: 0.55})
    assert img.mean() > 0


def test_gpu_scatter_fixed_rr_rejects_bad_rr():
    torch_cuda()
    gs, _ = scene_pair(5, boxes=5)
    n = 16
    verts, rays, shadow = empty_vertices(n), empty_rays(n), empty_shadow(n)
    cnt = torch_cuda().tensor([n], dtype=torch_cuda().int32, device="cuda")
    for rr in (0.0, -0.5, 1.5, float("nan")):
        with pytest.raises(nb.NRRSError):
            nb.scatter_fixed_rr(gs, nb.soa(nb.PathVertices, verts), cnt, n, rr, 0, 1,
                                nb.soa(nb.RaySoA, rays), nb.soa(nb.ShadowSoA, shadow), stream())


def test_gpu_trace_benchmark_scene_matches_brute_force():
    """The render benchmark's own scene (3000 boxes, 36k triangles, a BVH 20+ levels deep):
    closest hits of a sample of its 1920x1080 camera rays and of random rays inside the room,
    against brute force."""
    torch = torch_cuda()
    gs, hs = scene_pair(7, boxes=3000, closed=True)
    nn, nl, depth = gs.info()
    assert nn > 10000 and depth >= 16
    cam = nb.room_camera(1920, 1080, inside=True)
    r_cam = hs.camera_rays(cam, 100, 1234)
    rng = np.random.default_rng(3)
    pick = np.sort(rng.choice(1920 * 1080, 3000, replace=False))
    n = 3000
    o = rng.uniform(0.02, 0.98, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r_all = {k: np.concatenate([np.asarray(r_cam[k])[pick],
                                {"origin": o, "dir": d, "thp": np.ones((n, 3), np.float32),
                                 "pdf": np.zeros(n, np.float32), "pixel": np.zeros(n, np.uint32),
                                 "node": np.full(n, -1, np.int32)}[k]]) for k in r_cam}
    rays = dev_dict(r_all)
    hits = empty_hits(2 * n)
    cnt = torch.tensor([2 * n], dtype=torch.int32, device="cuda")
    nb.trace(gs, nb.soa(nb.RaySoA, rays), cnt, 2 * n, nb.soa(nb.HitSoA, hits), stream())
    want = hs.trace(r_all)
    same(to_host(hits, 2 * n), want, ("prim", "t", "u", "v"))
    assert (want["prim"] != 0xffffffff).mean() > 0.99   # closed: (almost) nothing escapes


def test_gpu_rrs_keeps_the_image_unbiased():
    """The mean image over frames with random kill/split factors matches the mean with factor 1
    (no decision: every vertex continues once) within the frames' standard error."""
    torch = torch_cuda()
    gs, _ = scene_pair(4, boxes=20)
    cam = nb.room_camera(48, 36)
    n = cam.width * cam.height
    cap = 8 * n

    def frame(seed, factor):
        film = torch.zeros((n, 9), dtype=torch.int64, device="cuda")
        rays, hits = empty_rays(cap), empty_hits(cap)
        verts, shadow = empty_vertices(cap), empty_shadow(cap)
        scratch = torch.zeros(nb.shade_scratch_bytes(cap), dtype=torch.uint8, device="cuda")
        n_rays = torch.tensor([n], dtype=torch.int32, device="cuda")
        n_vert, qsize = (torch.zeros(1, dtype=torch.int32, device="cuda") for _ in range(2))
        queue = torch.zeros(cap, dtype=torch.int32, device="cuda")
        rrs_norm = torch.zeros(cap, device="cuda")
        dp = nb.default_decide(clamp_max=4.0, clamp_min=0.0, use_ceil=0, normalize_rate=1.0,
                               scale_up=1)
        nb.camera_rays(cam, seed, 99, nb.soa(nb.RaySoA, rays), stream())
        rng = np.random.default_rng(seed)
        for depth in range(5):
            nb.trace(gs, nb.soa(nb.RaySoA, rays), n_rays, cap, nb.soa(nb.HitSoA, hits), stream())
            nb.shade(gs, nb.soa(nb.RaySoA, rays), nb.soa(nb.HitSoA, hits), n_rays, cap, depth,
                     film, None, nb.soa(nb.PathVertices, verts), n_vert, scratch, stream())
            nv = int(host(n_vert)[0])
            if nv == 0:
                break
            f = factor(rng, nv).astype(np.float32)
            # budget = sum of factors: the normalisation leaves the factors as they are
            budget = max(1, int(round(float(f.sum()))))
            f *= np.float32(budget / max(float(f.sum()), 1e-6))
            rnd = rng.uniform(size=nv).astype(np.float32)
            nb.decide_emit_noalloc(torch.from_numpy(f).cuda(), torch.from_numpy(rnd).cuda(), nv,
                                   budget, 0, dp, rrs_norm, None, queue, cap, qsize, None,
                                   stream())
            nb.scatter(gs, nb.soa(nb.PathVertices, verts), rrs_norm, queue, qsize, cap, depth,
                       seed * 7 + 1, nb.soa(nb.RaySoA, rays), nb.soa(nb.ShadowSoA, shadow),
                       stream())
            nb.trace_shadow(gs, nb.soa(nb.ShadowSoA, shadow), qsize, cap, film, None, stream())
            n_rays.copy_(qsize)
        img = torch.zeros((n, 3), device="cuda")
        nb.film_resolve(film, n, 1.0, img, stream())
        return float(host(img).mean())

    ones = [frame(s, lambda rng, k: np.ones(k)) for s in range(24)]
    rrs = [frame(s, lambda rng, k: rng.choice([0.5, 1.0, 2.0], k)) for s in range(24)]
    a, b = np.mean(ones), np.mean(rrs)
    se = np.sqrt(np.var(ones) / len(ones) + np.var(rrs) / len(rrs))
    assert abs(a - b) < 4 * se + 0.02 * a, (a, b, se)


def test_gpu_scene_without_lights_matches_oracle():
    """No emissive triangle: next-event estimation is skipped (no light to pick) and the only
    light is the environment seen through the open front."""
    v, t, m, ma, _ = nb.synth_scene(6, n_boxes=30)
    ma = ma.copy()
    ma[:, 3:] = 0.0
    env = np.array([0.6, 0.7, 0.8], np.float32)
    gs, hs = nb.Scene(v, t, m, ma, env), O.HostScene(v, t, m, ma, env)
    assert gs.info()[1] == 0
    img, _ = run_frame_pair(gs, hs, nb.room_camera(40, 30), 17, 4,
                            lambda rng, n: rng.uniform(0.5, 2.0, n))
    assert img.mean() > 0


def test_gpu_degenerate_triangles_match_brute_force():
    """Zero-area triangles (collapsed to a point or a line, one of them emissive) are never hit
    and never sampled as lights; the rest of the scene traces as before."""
    torch = torch_cuda()
    v, t, m, ma, e = nb.synth_scene(8, n_boxes=40)
    base = len(v)
    extra_v = np.array([[0.3, 0.3, 0.3], [0.3, 0.3, 0.3], [0.3, 0.3, 0.3],     # a point
                        [0.2, 0.5, 0.5], [0.4, 0.5, 0.5], [0.8, 0.5, 0.5]],    # a line
                       np.float32)
    v2 = np.concatenate([v, extra_v])
    t2 = np.concatenate([t, np.array([[base, base + 1, base + 2], [base + 3, base + 4, base + 5],
                                      [base + 5, base + 3, base + 4]], np.uint32)])
    emissive = int(np.nonzero(ma[:, 3] > 0)[0][0])
    m2 = np.concatenate([m, np.array([emissive, emissive, 0], np.uint32)])
    gs, hs = nb.Scene(v2, t2, m2, ma, e), O.HostScene(v2, t2, m2, ma, e)
    assert gs.info()[1] == nb.Scene(v, t, m, ma, e).info()[1]    # no zero-area light
    n = 20000
    rng = np.random.default_rng(4)
    o = rng.uniform(0.05, 0.95, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    # rays aimed straight at the degenerate triangles too
    o[:200] = np.array([0.3, 0.3, 0.05], np.float32)
    d[:200] = np.array([0.0, 0.0, 1.0], np.float32)
    o[200:400] = np.array([0.5, 0.5, 0.05], np.float32)
    r = {"origin": o, "dir": d, "thp": np.ones((n, 3), np.float32), "pdf": np.zeros(n, np.float32),
         "pixel": np.zeros(n, np.uint32), "node": np.full(n, -1, np.int32)}
    rays, hits = dev_dict(r), empty_hits(n)
    cnt = torch.tensor([n], dtype=torch.int32, device="cuda")
    nb.trace(gs, nb.soa(nb.RaySoA, rays), cnt, n, nb.soa(nb.HitSoA, hits), stream())
    want = hs.trace(r)
    same(to_host(hits, n), want, ("prim", "t", "u", "v"))
    assert not np.isin(want["prim"], np.arange(len(t), len(t2))).any()


def test_gpu_scene_create_rejects_bad_input():
    torch_cuda()
    v, t, m, ma, e = nb.synth_scene(1, n_boxes=2)
    bad_vertex = t.copy()
    bad_vertex[3, 1] = len(v)
    bad_material = m.copy()
    bad_material[0] = len(ma)
    for args in ((v, t[:0], m[:0], ma, e), (v, bad_vertex, m, ma, e), (v, t, bad_material, ma, e),
                 (v, t, m, ma[:0], e)):
        with pytest.raises(nb.NRRSError):
            nb.Scene(*args)


def test_gpu_empty_queues_are_no_ops():
    """A queue size of 0 on the device: every step returns at once and writes nothing."""
    torch = torch_cuda()
    gs, _ = scene_pair(2, boxes=5)
    n = 64
    rays, hits = empty_rays(n), empty_hits(n)
    verts, shadow = empty_vertices(n), empty_shadow(n)
    hits["prim"].fill_(-5)
    zero = torch.zeros(1, dtype=torch.int32, device="cuda")
    n_out = torch.full((1,), 77, dtype=torch.int32, device="cuda")
    film = torch.zeros((n, 9), dtype=torch.int64, device="cuda")
    scratch = torch.zeros(nb.shade_scratch_bytes(n), dtype=torch.uint8, device="cuda")
    before = {k: host(t).copy() for k, t in verts.items()}
    nb.trace(gs, nb.soa(nb.RaySoA, rays), zero, n, nb.soa(nb.HitSoA, hits), stream())
    nb.shade(gs, nb.soa(nb.RaySoA, rays), nb.soa(nb.HitSoA, hits), zero, n, 0, film, None,
             nb.soa(nb.PathVertices, verts), n_out, scratch, stream())
    rrs = torch.ones(n, device="cuda")
    queue = torch.zeros(n, dtype=torch.int32, device="cuda")
    nb.scatter(gs, nb.soa(nb.PathVertices, verts), rrs, queue, zero, n, 0, 1,
               nb.soa(nb.RaySoA, rays), nb.soa(nb.ShadowSoA, shadow), stream())
    nb.scatter_fixed_rr(gs, nb.soa(nb.PathVertices, verts), zero, n, 0.5, 0, 1,
                        nb.soa(nb.RaySoA, rays), nb.soa(nb.ShadowSoA, shadow), stream())
    nb.trace_shadow(gs, nb.soa(nb.ShadowSoA, shadow), zero, n, film, None, stream())
    assert int(host(n_out)[0]) == 0
    assert (host(hits["prim"]) == -5).all()
    assert not host(film).any()
    for k, t in verts.items():
        assert host(t).tobytes() == before[k].tobytes(), k
    assert not host(rays["thp"]).any() and not host(shadow["contrib"]).any()


def test_gpu_nee_off_matches_oracle():
    """mEnableNEE off: no shadow contributions and emitters hit by BSDF rays count in full."""
    gs, hs = scene_pair(3, boxes=40)
    gs.set_nee(False)
    hs.nee = False
    img, _ = run_frame_pair(gs, hs, nb.room_camera(48, 36), 5, 4,
                            lambda rng, n: rng.uniform(0.3, 2.5, n))
    assert img.mean() > 0
    with pytest.raises(nb.NRRSError):
        lib_rc = nb.lib().nrrs_scene_set_nee(gs._h, 2)
        nb._check(lib_rc, "nrrs_scene_set_nee")


def test_gpu_nee_and_bsdf_sampling_agree():
    """Next-event estimation with the power heuristic and pure BSDF sampling estimate the same
    image: the mean over frames agrees within the frames' standard error. Both run D bounces
    of scatter and a final trace and shade, so that each light-sampled path has its BSDF-sampled
    counterpart."""
    torch = torch_cuda()
    gs, _ = scene_pair(4, boxes=20, closed=True)
    cam = nb.room_camera(48, 36, inside=True)
    n = cam.width * cam.height
    cap = 2 * n
    D = 3

    def frame(seed, nee):
        gs.set_nee(nee)
        film = torch.zeros((n, 9), dtype=torch.int64, device="cuda")
        rays, hits = empty_rays(cap), empty_hits(cap)
        verts, shadow = empty_vertices(cap), empty_shadow(cap)
        scratch = torch.zeros(nb.shade_scratch_bytes(cap), dtype=torch.uint8, device="cuda")
        n_rays = torch.tensor([n], dtype=torch.int32, device="cuda")
        n_vert = torch.zeros(1, dtype=torch.int32, device="cuda")
        nb.camera_rays(cam, seed, 99, nb.soa(nb.RaySoA, rays), stream())
        for depth in range(D + 1):
            nb.trace(gs, nb.soa(nb.RaySoA, rays), n_rays, cap, nb.soa(nb.HitSoA, hits), stream())
            nb.shade(gs, nb.soa(nb.RaySoA, rays), nb.soa(nb.HitSoA, hits), n_rays, cap, depth,
                     film, None, nb.soa(nb.PathVertices, verts), n_vert, scratch, stream())
            if depth == D:
                break
            nb.scatter_fixed_rr(gs, nb.soa(nb.PathVertices, verts), n_vert, cap, 1.0, depth,
                                seed * 7 + 1, nb.soa(nb.RaySoA, rays),
                                nb.soa(nb.ShadowSoA, shadow), stream())
            nb.trace_shadow(gs, nb.soa(nb.ShadowSoA, shadow), n_vert, cap, film, None, stream())
            n_rays.copy_(n_vert)
        img = torch.zeros((n, 3), device="cuda")
        nb.film_resolve(film, n, 1.0, img, stream())
        return float(host(img).mean())

    on = [frame(s, True) for s in range(32)]
    off = [frame(s, False) for s in range(32)]
    gs.set_nee(True)
    a, b = np.mean(on), np.mean(off)
    se = np.sqrt(np.var(on) / len(on) + np.var(off) / len(off))
    assert a > 0 and abs(a - b) < 4 * se + 0.01 * a, (a, b, se)
    assert np.std(on) < np.std(off)        # light sampling lowers the variance


def test_gpu_trace_sorted_equals_trace():
    """The sorted trace writes the same hits as the plain one, bit for bit: on the benchmark's
    scene with a queue large enough to sort (camera rays and random rays, with empty slots and a
    device count below the capacity), and below the sorting threshold."""
    torch = torch_cuda()
    v, t, m, ma, e = nb.synth_scene(7, n_boxes=3000, closed=True)
    gs = nb.Scene(v, t, m, ma, e)
    rng = np.random.default_rng(12)
    for n, cap in ((150_000, 160_000), (40_000, 40_000)):
        cam = nb.room_camera(500, n // 500, inside=True)
        rays = empty_rays(cap)
        nb.camera_rays(cam, 2, 5, nb.soa(nb.RaySoA, rays), stream())
        k = n // 2   # the second half: random rays inside the room, some of them empty slots
        o = rng.uniform(0.02, 0.98, (k, 3)).astype(np.float32)
        d = rng.normal(size=(k, 3)).astype(np.float32)
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        thp = np.ones((k, 3), np.float32)
        thp[::7] = 0.0
        rays["origin"][n - k:n] = torch.from_numpy(o).cuda()
        rays["dir"][n - k:n] = torch.from_numpy(d).cuda()
        rays["thp"][n - k:n] = torch.from_numpy(thp).cuda()
        cnt = torch.tensor([n], dtype=torch.int32, device="cuda")
        a, b = empty_hits(cap), empty_hits(cap)
        b["prim"].fill_(-3)
        scratch = torch.zeros(nb.trace_scratch_bytes(cap), dtype=torch.uint8, device="cuda")
        nb.trace(gs, nb.soa(nb.RaySoA, rays), cnt, cap, nb.soa(nb.HitSoA, a), stream())
        nb.trace_sorted(gs, nb.soa(nb.RaySoA, rays), cnt, cap, nb.soa(nb.HitSoA, b), scratch,
                        stream())
        same(to_host(a, n), to_host(b, n), ("prim", "t", "u", "v"))
        assert (host(b["prim"])[n:] == -3).all()      # nothing written past the device count
    gs.close()


@pytest.mark.parametrize("closed,glass", [(False, False), (True, False), (True, True)],
                         ids=["open-mirrors", "closed-mirrors", "closed-mirrors-glass"])
def test_gpu_mirror_frame_matches_oracle(closed, glass):
    """Mirror and thin-glass materials: their hits bypass the inference queue (the closest-hit
    program's specular branch) and count as n_specular against the budget; their vertices bounce
    once, unconditionally, into the ray slots after the RRS-scattered ones (glass reflecting or
    passing through by its Fresnel reflectance). A whole frame, bit for bit, with every array
    compared as it is produced."""
    torch = torch_cuda()
    v, t, m, ma, e = nb.synth_scene(13, n_boxes=60, closed=closed)
    spec = np.zeros(len(ma), np.uint8)
    spec[4::3] = 1                                    # every third box material is a mirror
    if glass:
        spec[5::3] = 2                                # and as many are thin glass
    gs, hs = nb.Scene(v, t, m, ma, e), O.HostScene(v, t, m, ma, e)
    gs.set_specular(spec)
    hs.set_specular(spec)
    cam = nb.room_camera(64, 48, inside=closed)
    n = cam.width * cam.height
    cap = 4 * n
    seed = 31
    film = torch.zeros((n, 9), dtype=torch.int64, device="cuda")
    hfilm = np.zeros((n, 9), np.int64)
    rays, hits = empty_rays(cap), empty_hits(cap)
    verts, verts_s, shadow = empty_vertices(cap), empty_vertices(cap), empty_shadow(cap)
    contrib = torch.zeros((cap, 3), device="cuda")
    scontrib = torch.zeros((cap, 3), device="cuda")
    scratch = torch.zeros(nb.shade_scratch_bytes(cap), dtype=torch.uint8, device="cuda")
    i32 = lambda: torch.zeros(1, dtype=torch.int32, device="cuda")  # noqa: E731
    n_rays, n_vert, n_spec, qsize, n_next = i32(), i32(), i32(), i32(), i32()
    n_rays.fill_(n)
    queue = torch.zeros(cap, dtype=torch.int32, device="cuda")
    rrs_norm = torch.zeros(cap, device="cuda")
    nb.camera_rays(cam, 0, seed, nb.soa(nb.RaySoA, rays), stream())
    hr = hs.camera_rays(cam, 0, seed)
    dp = nb.default_decide(clamp_max=4.0)
    rng = np.random.default_rng(seed)
    mirrored = transmitted = 0
    for depth in range(5):
        nr = int(host(n_rays)[0])
        assert nr == len(hr["pixel"])
        nb.trace(gs, nb.soa(nb.RaySoA, rays), n_rays, cap, nb.soa(nb.HitSoA, hits), stream())
        hh = hs.trace(hr)
        same(to_host(hits, nr), hh, ("prim", "t", "u", "v"))
        nb.shade_split(gs, nb.soa(nb.RaySoA, rays), nb.soa(nb.HitSoA, hits), n_rays, cap, depth,
                       film, contrib, nb.soa(nb.PathVertices, verts), n_vert,
                       nb.soa(nb.PathVertices, verts_s), n_spec, scratch, stream())
        hv, hvs, hc = hs.shade_split(hr, hh, depth, hfilm)
        nv, ns = int(host(n_vert)[0]), int(host(n_spec)[0])
        assert (nv, ns) == (len(hv["pos"]), len(hvs["pos"]))
        same(to_host(verts, nv), hv, nb.PATH_VERTEX_FIELDS)
        same(to_host(verts_s, ns), hvs, nb.PATH_VERTEX_FIELDS)
        assert host(contrib)[:nr].tobytes() == hc.tobytes()
        assert host(film).tobytes() == hfilm.tobytes()
        mirrored += ns
        if nv + ns == 0:
            break
        # the decision on the inference queue; the budget counts the specular vertices too
        f = rng.uniform(0.3, 2.5, nv).astype(np.float32)
        rnd = rng.uniform(size=nv).astype(np.float32)
        nq = 0
        if nv:
            rc = nb.decide_emit_noalloc(torch.from_numpy(f).cuda(), torch.from_numpy(rnd).cuda(),
                                        nv, nv + ns, ns, dp, rrs_norm, None, queue, cap, qsize,
                                        None, stream())
            assert rc == 0
            o = O.decide_emit(f, rnd, nv + ns, ns, dp, capacity=cap, shift_n=nb.NOALLOC_MAX_N)
            nq = int(host(qsize)[0])
            assert nq == o["total"]
        else:
            qsize.zero_()
        nb.scatter(gs, nb.soa(nb.PathVertices, verts), rrs_norm, queue, qsize, cap, depth, seed,
                   nb.soa(nb.RaySoA, rays), nb.soa(nb.ShadowSoA, shadow), stream())
        nb.scatter_specular(gs, nb.soa(nb.PathVertices, verts_s), n_spec, cap, qsize, cap, depth,
                            seed, nb.soa(nb.RaySoA, rays), n_next, stream())
        full = {"origin": np.zeros((cap, 3), np.float32), "dir": np.zeros((cap, 3), np.float32),
                "thp": np.zeros((cap, 3), np.float32), "pdf": np.zeros(cap, np.float32),
                "pixel": np.zeros(cap, np.uint32), "node": np.zeros(cap, np.int32)}
        if nq:
            hr_d, hsh = hs.scatter(hv, o["rrs_norm"], o["queue"], depth, seed)
            for k in full:
                full[k][:nq] = hr_d[k]
        hs.scatter_specular(hvs, full, nq, cap, depth, seed)
        hr = {k: a[:nq + ns] for k, a in full.items()}
        # glass vertices that passed straight through keep the incoming direction
        transmitted += int((np.abs((hr["dir"][nq:] + hvs["wi"]).sum(axis=1)) == 0).sum())
        assert int(host(n_next)[0]) == nq + ns
        same(to_host(rays, nq + ns), hr, ("origin", "dir", "thp", "pdf", "pixel", "node"))
        if nq:
            nb.trace_shadow(gs, nb.soa(nb.ShadowSoA, shadow), qsize, cap, film, scontrib, stream())
            hco = hs.shadow(hsh, hfilm)
            assert host(scontrib)[:nq].tobytes() == hco.tobytes()
        assert host(film).tobytes() == hfilm.tobytes()
        n_rays.copy_(n_next)
    assert mirrored > 100
    if glass:
        assert transmitted > 0
    img = torch.zeros((n, 3), device="cuda")
    nb.film_resolve(film, n, 1.0, img, stream())
    assert host(img).tobytes() == hs.resolve(hfilm, 1.0).tobytes()
