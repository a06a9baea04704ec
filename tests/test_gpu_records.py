"""GPU parity of the path-record entry points (nrrs_record_nodes, nrrs_record_radiance,
nrrs_generate_training_data, nrrs_sample_weights) against the oracle, bit for bit: node
numbering, node fields, radiance integers, training batch, per-pixel counts and weights. Covers the
hand-derived trees, synthetic frames up to 1920x1080, contribution order, radiance recorded after
the batch was built, reuse after reset, both capacities overflowing, empty inputs, non-finite
contributions, and the batch feeding nrrs_train_step."""
from __future__ import annotations

import numpy as np
import pytest

import nrrs_b200 as nb
import oracle as O
from gpu_util import host, make_net, random_params, stream, torch_cuda
from test_records_oracle import CASES, bounce_arrays, check_against_expect, split_calls

pytestmark = pytest.mark.gpu

BOUNCE_KEYS = ("pos", "wi", "normal", "albedo", "roughness", "thp", "depth", "pixel", "rrs",
               "record", "parent")
NODE_FIELDS = {"pos": (np.float32, 3), "wi": (np.float32, 3), "normal": (np.float32, 3),
               "albedo": (np.float32, 3), "roughness": (np.float32, 1), "thp": (np.float32, 3),
               "parent": (np.int32, 1), "pixel": (np.uint32, 1), "rrs": (np.float32, 1),
               "depth": (np.uint32, 1), "radiance": (np.int64, 9),
               "first_child": (np.uint32, 1), "children": (np.uint32, 1),
               "node_flags": (np.uint32, 1)}
BATCH_SHAPES = {"pos": 3, "wi": 3, "normal": 3, "albedo": 3, "roughness": 1, "thp": 3, "depth": 1,
                "ref_mean": 1, "target": 3, "rrs_target": 1, "pixel": 1}


def dev(a):
    torch = torch_cuda()
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint32:
        a = a.view(np.int32)
    return torch.from_numpy(a).cuda()


class GpuNodes:
    """A node block in a CUDA tensor and the library's buffer object over it."""

    def __init__(self, capacity: int, max_record: int):
        torch = torch_cuda()
        self.capacity = capacity
        nbytes = nb.path_nodes_bytes(capacity, max_record)
        self.buf = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
        self.pn = nb.NRRSPathNodesBuffer(self.buf.data_ptr(), nbytes, capacity, max_record,
                                         stream())

    def field(self, name: str, count: int) -> np.ndarray:
        dt, w = NODE_FIELDS[name]
        off = getattr(self.pn.nodes, name) - self.buf.data_ptr()
        nbytes = np.dtype(dt).itemsize * w * count
        raw = host(self.buf[off:off + nbytes])
        a = raw.view(dt)
        return a.reshape(count, w) if w > 1 else a

    def record(self, b: dict) -> "torch.Tensor":
        torch = torch_cuda()
        d = {k: dev(b[k]) for k in BOUNCE_KEYS if b.get(k) is not None}
        n = len(b["pixel"])
        out = torch.full((max(n, 1),), -7, dtype=torch.int32, device="cuda")
        v = nb.vertex_soa(d["pos"], d["wi"], d.get("normal"), d.get("roughness"), d.get("albedo"),
                          d["thp"], d.get("depth"))
        self.pn.recordNode(v, d["parent"], d["pixel"], d.get("rrs"), d.get("record"), n, out,
                           stream())
        return out[:n]

    def radiance(self, node, contrib):
        n = len(node)
        if n == 0:
            self.pn.recordRadiance(None, None, 0, stream())
            return
        self.pn.recordRadiance(dev(np.asarray(node, np.int32)),
                               dev(np.asarray(contrib, np.float32).reshape(-1, 3)), n, stream())

    def generate(self, params, capacity: int, image=None, n_pixels: int = 0):
        torch = torch_cuda()
        cap = max(capacity, 1)
        out = {k: torch.full((cap, w) if w > 1 else (cap,), -3.0 if k != "depth" and k != "pixel"
                             else 0, dtype=torch.int32 if k in ("depth", "pixel") else torch.float32,
                             device="cuda") for k, w in BATCH_SHAPES.items()}
        counts = torch.zeros(max(n_pixels, 1), dtype=torch.int32, device="cuda")
        size = torch.full((1,), 12345, dtype=torch.int32, device="cuda")
        img = dev(image) if image is not None else None
        self.pn.generate_training_data(params, nb.train_batch(**out), capacity, size, image=img,
                                       image_channels=4 if image is not None else 0,
                                       n_pixels=n_pixels,
                                       pixel_samples=counts if image is not None else None,
                                       stream=stream())
        w = torch.full((cap,), -1.0, dtype=torch.float32, device="cuda")
        if image is not None:
            nb.calculate_sample_weight(out["pixel"], counts, n_pixels, size, capacity, w, stream())
        m = int(host(size)[0])
        res = {k: host(t)[:min(m, capacity)] for k, t in out.items()}
        res["pixel"] = res["pixel"].view(np.uint32)
        res["depth"] = res["depth"].view(np.uint32)
        return res, m, host(counts).view(np.uint32)[:n_pixels], host(w)[:min(m, capacity)]


def run_frame(bounces, image, capacity, params, batch_capacity=None, order="bounce"):
    """The library's run of a synthetic frame; order "bounce" records each bounce's
    contributions after its nodes, "shuffled" records all contributions at the end in a random
    order."""
    max_record = max(len(b["pixel"]) for b in bounces)
    g = GpuNodes(capacity, max_record)
    outs = []
    for b in bounces:
        outs.append(host(g.record(b)))
        if order == "bounce":
            g.radiance(b["contrib_node"], b["contrib"])
    if order == "shuffled":
        node = np.concatenate([b["contrib_node"] for b in bounces])
        contrib = np.concatenate([b["contrib"] for b in bounces])
        p = np.random.default_rng(99).permutation(len(node))
        g.radiance(node[p], contrib[p])
    size, dropped, flags = g.pn.status(stream())
    bc = capacity if batch_capacity is None else batch_capacity
    batch, total, counts, weights = g.generate(params, bc, image=image, n_pixels=image.shape[0])
    _, _, flags2 = g.pn.status(stream())
    return dict(g=g, outs=outs, size=size, dropped=dropped, flags=flags | flags2, batch=batch,
                total=total, counts=counts, weights=weights)


def assert_same_batch(a: dict, b: dict):
    for k in BATCH_SHAPES:
        assert a[k].shape == b[k].shape, k
        assert a[k].tobytes() == b[k].tobytes(), k


def assert_frame_matches_oracle(r, o, bounces, batch_capacity, check_radiance=True):
    for got, want, b in zip(r["outs"], o["node_outs"], bounces):
        assert np.array_equal(got, want)
        assert np.array_equal(got, b["node"])
    hn = o["nodes"]
    assert r["size"] == hn.size and r["dropped"] == hn.dropped
    assert r["flags"] == hn.status
    for k in NODE_FIELDS:
        if k == "radiance" and not check_radiance:
            continue
        got = r["g"].field(k, hn.size)
        assert got.tobytes() == hn.a[k][:hn.size].tobytes(), k
    assert r["total"] == min(o["total"], batch_capacity)
    assert_same_batch(r["batch"], o["batch"])
    assert r["counts"].tobytes() == o["counts"].tobytes()
    assert r["weights"].tobytes() == o["weights"].tobytes()


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_gpu_golden_trees(case):
    g = GpuNodes(case["capacity"], 8)
    outs = []
    for b in case["bounces"]:
        a = bounce_arrays(b)
        outs.append(host(g.record(a)))
        g.radiance(a["contrib_node"], a["contrib"])
    size, dropped, flags = g.pn.status(stream())
    image = np.array(case["image"], np.float32)
    batch, total, counts, w = g.generate(nb.TrainDataParams(**case["params"]), 64, image=image,
                                         n_pixels=len(image))
    check_against_expect(case, outs, size, dropped, batch, total, counts, w)
    assert flags == (nb.DEV_NAN if case["capacity"] > 5 else nb.DEV_OVERFLOW)


PARAMS = {
    "reference_defaults": nb.default_train_data_params(),
    "filters": nb.default_train_data_params(ignore_zero_l=1, copy_rrs_node=1,
                                            dedupe_rrs_target=1),
}


@pytest.mark.parametrize("pname", list(PARAMS))
@pytest.mark.parametrize("pixels", [1, 777, 30000])
def test_gpu_frame_matches_oracle(pixels, pname):
    bounces, image = nb.synth_paths(21 + pixels, pixels, capacity=4 * pixels)
    o = O.frame_training_data(bounces, image, 4 * pixels, PARAMS[pname])
    r = run_frame(bounces, image, 4 * pixels, PARAMS[pname])
    assert_frame_matches_oracle(r, o, bounces, 4 * pixels)


def test_gpu_frame_1080p_bit_exact():
    """A whole 1920x1080 frame: 8 bounces, about 10M vertices, 7M nodes, 7.5M contributions."""
    P = 1920 * 1080
    bounces, image = nb.synth_paths(1080, P, capacity=4 * P)
    prm = PARAMS["filters"]
    o = O.frame_training_data(bounces, image, 4 * P, prm)
    r = run_frame(bounces, image, 4 * P, prm)
    assert r["size"] > 6_000_000 and r["total"] > 4_000_000
    assert_frame_matches_oracle(r, o, bounces, 4 * P)


def test_gpu_contribution_order_does_not_change_a_bit():
    bounces, image = nb.synth_paths(31, 20000, capacity=80000)
    prm = PARAMS["filters"]
    a = run_frame(bounces, image, 80000, prm, order="bounce")
    b = run_frame(bounces, image, 80000, prm, order="shuffled")
    assert a["total"] == b["total"]
    assert_same_batch(a["batch"], b["batch"])
    assert a["g"].field("radiance", a["size"]).tobytes() == b["g"].field("radiance", b["size"]).tobytes()
    o = O.frame_training_data(bounces, image, 80000, prm)
    assert_same_batch(b["batch"], o["batch"])


def test_gpu_radiance_recorded_after_the_batch_reaches_ancestors():
    """After nrrs_generate_training_data completed the nodes, new contributions are walked up the
    chain at once; a second batch then equals the oracle's with every contribution."""
    bounces, image = nb.synth_paths(41, 8000, capacity=32000)
    prm = PARAMS["filters"]
    g = GpuNodes(32000, max(len(b["pixel"]) for b in bounces))
    for b in bounces:
        g.record(b)
    node = np.concatenate([b["contrib_node"] for b in bounces])
    contrib = np.concatenate([b["contrib"] for b in bounces])
    half = len(node) // 2
    g.radiance(node[:half], contrib[:half])
    g.generate(prm, 32000, image=image, n_pixels=image.shape[0])
    g.radiance(node[half:], contrib[half:])
    batch, total, counts, w = g.generate(prm, 32000, image=image, n_pixels=image.shape[0])
    o = O.frame_training_data(bounces, image, 32000, prm)
    assert total == o["total"]
    assert_same_batch(batch, o["batch"])
    hn = o["nodes"]
    assert g.field("radiance", hn.size).tobytes() == hn.a["radiance"][:hn.size].tobytes()


def test_gpu_reset_and_reuse():
    prm = PARAMS["filters"]
    b1, img1 = nb.synth_paths(51, 5000, capacity=20000)
    b2, img2 = nb.synth_paths(52, 6000, capacity=20000)
    g = GpuNodes(20000, 6000)
    for frame, (bounces, image) in enumerate(((b1, img1), (b2, img2), (b1, img1))):
        if frame:
            g.pn.reset(stream())
        for b in bounces:
            assert np.array_equal(host(g.record(b)), b["node"])
            g.radiance(b["contrib_node"], b["contrib"])
        batch, total, counts, w = g.generate(prm, 20000, image=image, n_pixels=image.shape[0])
        o = O.frame_training_data(bounces, image, 20000, prm)
        assert total == o["total"]
        assert_same_batch(batch, o["batch"])
        assert w.tobytes() == o["weights"].tobytes()


@pytest.mark.parametrize("node_cap,batch_cap", [(3000, None), (100000, 500), (2500, 700)])
def test_gpu_capacities_overflow_like_the_oracle(node_cap, batch_cap):
    bounces, image = nb.synth_paths(61, 2000, bounces=6, capacity=node_cap)
    prm = PARAMS["filters"]
    o = O.frame_training_data(bounces, image, node_cap, prm, batch_capacity=batch_cap)
    r = run_frame(bounces, image, node_cap, prm, batch_capacity=batch_cap)
    assert_frame_matches_oracle(r, o, bounces, node_cap if batch_cap is None else batch_cap)
    assert r["flags"] & nb.DEV_OVERFLOW
    if batch_cap is not None:
        assert r["total"] == batch_cap and len(r["batch"]["target"]) == batch_cap


def test_gpu_empty_inputs():
    g = GpuNodes(64, 16)
    g.pn.recordNode(nb.VertexSoA(), None, None, None, None, 0, None, stream())
    g.radiance([], [])
    image = np.ones((4, 4), np.float32)
    batch, total, counts, w = g.generate(PARAMS["filters"], 16, image=image, n_pixels=4)
    assert total == 0 and counts.sum() == 0
    assert g.pn.status(stream()) == (0, 0, 0)
    # contributions to no node (-1) or to nodes not yet recorded are skipped
    b = dict(pos=np.zeros((2, 3), np.float32), wi=np.ones((2, 3), np.float32),
             thp=np.ones((2, 3), np.float32), pixel=np.array([0, 1], np.uint32),
             parent=np.array([-1, -1], np.int32))
    assert host(g.record(b)).tolist() == [0, 1]
    g.radiance([-1, 2, 5, 1], [[1, 1, 1]] * 4)
    batch, total, counts, w = g.generate(nb.default_train_data_params(), 16, image=image,
                                         n_pixels=4)
    assert total == 2
    assert batch["target"].tolist() == [[0, 0, 0], [1, 1, 1]]
    assert batch["rrs_target"].tolist() == [1.0, 1.0]       # rrs NULL -> the default 1
    assert batch["normal"].tolist() == [[0, 0, 0], [0, 0, 0]]  # normal NULL -> 0


def test_gpu_nonfinite_contributions_drop_the_chain():
    bounces, image = nb.synth_paths(71, 3000, capacity=12000)
    rng = np.random.default_rng(3)
    for b in bounces[2:5]:
        c = b["contrib"]
        k = rng.choice(len(c), size=max(1, len(c) // 50), replace=False)
        c[k[0::3], 0] = np.nan
        c[k[1::3], 1] = np.inf
        c[k[2::3], 2] = -3e19   # beyond 2^62 in magnitude
    prm = PARAMS["filters"]
    o = O.frame_training_data(bounces, image, 12000, prm)
    r = run_frame(bounces, image, 12000, prm)
    assert_frame_matches_oracle(r, o, bounces, 12000)
    assert r["flags"] & nb.DEV_NAN
    assert (o["nodes"].a["node_flags"][:o["nodes"].size] != 0).sum() > 100


def test_gpu_bad_pixel_is_flagged_and_skipped():
    g = GpuNodes(16, 4)
    b = dict(pos=np.zeros((3, 3), np.float32), wi=np.ones((3, 3), np.float32),
             thp=np.ones((3, 3), np.float32), pixel=np.array([0, 9, 1], np.uint32),
             parent=np.array([-1, -1, -1], np.int32))
    g.record(b)
    g.radiance([0, 1, 2], [[1, 2, 3]] * 3)
    image = np.full((2, 4), 3.0, np.float32)
    batch, total, counts, w = g.generate(nb.default_train_data_params(), 16, image=image,
                                         n_pixels=2)
    assert total == 3
    assert batch["ref_mean"].tolist() == [3.0, 0.0, 3.0]
    assert counts.tolist() == [1, 1] and w.tolist() == [1.0, 0.0, 1.0]
    assert g.pn.status(stream())[2] == nb.DEV_BAD_INDEX


def test_gpu_batch_feeds_the_training_step():
    """The generated batch is nrrs_train_step's input: its FP32 losses equal the oracle's on the
    oracle's batch."""
    torch = torch_cuda()
    bounces, image = nb.synth_paths(81, 3000, capacity=12000)
    prm = PARAMS["filters"]
    r = run_frame(bounces, image, 12000, prm)
    o = O.frame_training_data(bounces, image, 12000, prm)
    n = min(r["total"], 8192)
    net = make_net(max_train=1 << 13, step=3, log2_hashmap_size=15, precision=nb.PREC_FP32)
    p0 = random_params(net, 5, table_scale=0.5, mlp_scale=0.15)
    bt = {k: dev(np.ascontiguousarray(r["batch"][k][:n])) for k in BATCH_SHAPES}
    soa = nb.vertex_soa(bt["pos"], bt["wi"], bt["normal"], bt["roughness"], bt["albedo"],
                        bt["thp"], bt["depth"], bt["ref_mean"])
    loss = torch.zeros(2, dtype=torch.float64, device="cuda")
    net.trainGrads(soa, bt["target"], n, loss, stream())
    ob = {k: np.ascontiguousarray(o["batch"][k][:n]) for k in BATCH_SHAPES}
    _, l64 = O.train_grads(net.config, p0, ob, ob["target"], "f64")
    assert host(loss) == pytest.approx(l64, rel=1e-4)
    net.close()


def test_gpu_parent_in_the_same_call_is_cut():
    g = GpuNodes(16, 4)
    hn = O.HostNodes(16)
    b = dict(pos=np.zeros((3, 3), np.float32), wi=np.ones((3, 3), np.float32),
             thp=np.ones((3, 3), np.float32), pixel=np.zeros(3, np.uint32),
             parent=np.array([-1, 0, 7], np.int32))
    b2 = dict(b, parent=np.array([2, 4, 1], np.int32))
    for x in (b, b2):
        assert host(g.record(x)).tolist() == hn.record_nodes(x).tolist()
    for k in ("parent", "first_child", "children"):
        assert g.field(k, 6).tobytes() == hn.a[k][:6].tobytes(), k
    assert g.pn.status(stream()) == (6, 0, nb.DEV_BAD_INDEX)


@pytest.mark.parametrize("parts", [8, 9])
def test_gpu_many_record_calls(parts):
    """8 bounces in `parts` calls each: 64 calls keep the level table (level-by-level radiance
    pass), 72 overflow it (the chain walk); both must match the oracle bit for bit."""
    bounces, image = nb.synth_paths(91, 6000, capacity=24000)
    calls = split_calls(bounces, parts)
    prm = PARAMS["filters"]
    o = O.frame_training_data(calls, image, 24000, prm)
    r = run_frame(calls, image, 24000, prm)
    assert_frame_matches_oracle(r, o, calls, 24000)
