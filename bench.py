"""Benchmark of the NRRS per-vertex step on B200 (one JSON line on rank 0).

The metric is "RRS vertices/s and train samples/s, mixed precision vs plain FP32 at stated
error". The default run measures it on the largest single-GPU configuration of the workload
definition and puts the other two configurations beside it:

  frame4k (headline, `value`)
            one online train-and-infer frame at 3840x2160: 10 bounces of inference, RRS
            decision and emission on 8,294,400 path vertices each, then 10 training steps of
            262,144 samples; StatNet and RRSNet 128 wide with 3 hidden layers in BF16 on the
            tensor cores (FP32 accumulation, FP32 master weights and Adam state), a 2^22-entry
            FP16 hash table, exact 64-bit normalisation sums
  fp32_per_depth
            the same frame on the plain FP32 path (FP32 table, FP32 SIMT MLPs), one launch
            sequence per bounce, on the same GPU and the same inputs
  errors    stats, factors and training losses of both paths against the FP64 oracle and
            against each other; decisions of the mixed path against the oracle's at equal
            factors
  secondary.frame1080p
            the 1080p frame: 6 bounces x 2,073,600 vertices + 1 training step, 64 wide x 2
            hidden, FP16, 2^19 table; mixed against plain FP32
  secondary.batched
            depths 0..9 with round(2,073,600 x 0.6^d) vertices, 10 % of them split into U{1..4}
            copies (5,925,732 vertices): the mixed path as ONE CUDA-graph launch of the batched
            step, against the plain FP32 path launched depth by depth

Single workloads (--workload frame4k|frame1080p|batched|records1080p|render1080p|
render_train1080p, with --only) run one arm for profiling.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload ...] [--only] [--precision fp16|bf16|fp32] [--no-train]

value    = vertices/s of the whole job (device-timed steps, max over ranks)
e2e      = the same metric through the C-ABI with host (pinned) inputs: the H2D copy of each
           step's vertices and training batch and the D2H read of queue sizes and losses are
           inside the timed region; uploads run on a copy stream, overlapping the compute of
           the previous bounce
roofline = the dominant kernel's algorithmic GB/s against the measured HBM peak
--impl reference times the reference's CPU path (the oracle's FP32 restatement, all host
threads) on a bounded sample of the same workload per step; it loads no product library.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "nrrs-code_b200"))
sys.path.insert(0, str(REPO / "oracle"))

import numpy as np  # noqa: E402

# The product binding is imported by the GPU arms only (load_product()); the reference arm
# never loads the product library.
nb = None

SOA_BYTES = 72            # pos, wi, normal, roughness, albedo, thp, depth, ref_mean
RND_BYTES = 4
TARGET_BYTES = 12
METRIC = "RRS vertices/s and train samples/s, mixed-prec vs FP32 plain at stated error"
FIELDS = ("pos", "wi", "normal", "roughness", "albedo", "thp", "depth", "ref_mean", "rnd")
PREC = {"fp32": 0, "fp16": 1, "bf16": 2}   # nrrs_precision
FACTOR_RRSNET = 3

WORKLOADS = {
    "frame4k": dict(bounces=10, n_vert=8_294_400, train_steps=10, train_batch=262_144,
                    width=128, hidden=3, log2_table=22, steps=5, precision="bf16"),
    "frame1080p": dict(bounces=6, n_vert=2_073_600, train_steps=1, train_batch=262_144,
                       width=64, hidden=2, log2_table=19, steps=50, precision="fp16"),
    "batched": dict(bounces=10, n_vert=2_073_600, train_steps=0, train_batch=262_144,
                    width=64, hidden=2, log2_table=19, steps=50, precision="fp16"),
    # the reference's shipped settings (render/test.json:75-82): node buffer 10 x pixels,
    # throughput scaled by rrs, later siblings without RRSNet target; zero-L samples kept
    # 600 frames: about a second of timed work, so that the clock sampler sees it
    "records1080p": dict(bounces=8, n_vert=2_073_600, node_rate=10, steps=600, precision="fp32"),
    "render1080p": dict(bounces=6, n_vert=2_073_600, width=64, hidden=2, log2_table=19,
                        steps=40, precision="fp16", boxes=3000, train_steps=0,
                        train_batch=0),
    "render_train1080p": dict(bounces=6, n_vert=2_073_600, width=64, hidden=2, log2_table=19,
                              steps=20, precision="fp16", boxes=3000, train_steps=1,
                              train_batch=262_144, node_rate=8),
}


def load_product():
    global nb
    if nb is None:
        import nrrs_b200
        nb = nrrs_b200
    return nb


def env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def measured_peaks():
    """(HBM GB/s, BF16 TFLOP/s burst, source) from MEASURED_PEAKS.json, else the fallback."""
    f = REPO / "MEASURED_PEAKS.json"
    if f.exists():
        j = json.loads(f.read_text())
        return j.get("hbm_gbs", 6650.0), j.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


def traffic_per_vertex(kernel: str, workload: str):
    """DRAM bytes per vertex of the kernel on the workload from the committed ncu summary."""
    f = REPO / "profiles" / "traffic.json"
    if f.exists():
        j = json.loads(f.read_text())
        return j.get(workload, {}).get(kernel)
    return None


def requests_per_vertex(kernel: str, workload: str):
    """L2-to-L1 read sectors per vertex of the kernel on the workload (one L1-to-L2 request
    each: the gathers are random one-sector loads) from the committed ncu summary"""
    f = REPO / "profiles" / "traffic.json"
    if f.exists():
        j = json.loads(f.read_text())
        return j.get("l1_requests", {}).get(workload, {}).get(kernel)
    return None


def request_bound(roof, workload, sm_mhz, sm_count):
    """The gather kernels' real roofline: the L1-to-crossbar interface carries one request per
    cycle per SM, and every random gather sector is one request."""
    if not roof:
        return None
    spv = requests_per_vertex(roof["kernel"], workload)
    if not spv:
        return None
    achieved = spv * roof["vertices_per_launch"] / (roof["launch_ms"] * 1e-3) / 1e9
    peak = sm_count * (sm_mhz or 1965.0) / 1e3
    return {"bound": "l1_to_l2_requests", "achieved": achieved, "peak": peak,
            "unit": "G requests/s", "frac": achieved / peak, "sectors_per_vertex": spv,
            "peak_basis": "1 request per cycle per SM x SMs x median SM clock under load",
            "sectors_source": "ncu l1tex__m_xbar2l1tex_read_sectors_mem_lg_op_ld (profiles/)"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 100 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.p = None
        self.lines = []

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *exc):
        if self.p:
            self.p.terminate()
            try:
                out, _ = self.p.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
                out, _ = self.p.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def config_fields(precision: str, wl: dict, max_queue: int, max_train: int,
                  sum_shards: int = 0) -> dict:
    return dict(precision=PREC[precision], max_queue=max_queue, max_train=max_train,
                statnet_width=wl["width"], statnet_hidden=wl["hidden"],
                rrsnet_width=wl["width"], rrsnet_hidden=wl["hidden"],
                log2_hashmap_size=wl["log2_table"], sum_shards=sum_shards)


def make_config(precision: str, wl: dict, max_queue: int, max_train: int, sum_shards: int = 0):
    return load_product().default_config(**config_fields(precision, wl, max_queue, max_train,
                                                         sum_shards))


def do_train_of(args, wl):
    return not args.no_train and wl["train_steps"] > 0


def workload_name(name: str, wl: dict, train: bool, precision: str) -> str:
    s = (f"{name}_{wl['bounces']}x{wl['n_vert']}_w{wl['width']}h{wl['hidden']}"
         f"_T2^{wl['log2_table']}_infer_decide_emit")
    if train:
        s += f"_train{wl['train_steps']}x{wl['train_batch']}"
    return f"{s}_{precision}"


def frame_config(name: str, wl: dict, train: bool, precision: str, world: int) -> dict:
    """The `config` object of a frame workload; identical in the GPU arm and the reference arm."""
    batched = name == "batched"
    total = batched_total(wl) if batched else wl["bounces"] * wl["n_vert"]
    return {"workload": workload_name(name, wl, train, precision), "bounces": wl["bounces"],
            "vertices_per_bounce": wl["n_vert"], "vertices_per_step": total,
            "train_steps": wl["train_steps"] if train else 0,
            "train_batch": wl["train_batch"] if train else 0,
            "encoding": f"hashgrid L16 F2 T2^{wl['log2_table']} Nmin16 b1.5 (FP16 table) + SH deg4",
            "mlp": f"StatNet 64->{wl['width']}x{wl['hidden']}->3, "
                   f"RRSNet 16->{wl['width']}x{wl['hidden']}->1, {precision} MMA / FP32 accumulate",
            "l2": "inputs larger than L2 (one vertex buffer per bounce)" if not batched else
                  "inputs larger than L2 (one 450 MB SoA of all depths)",
            "parallelism": f"dp{world}"}


# ---- the reference's CPU path: the oracle's FP32 restatement on the host cores ----------------

class CpuFrameSample:
    """Bounded samples of a frame workload on the host cores with the oracle's FP32 path
    (OpenMP, all host threads). One step processes a fraction f of the frame: inference,
    decision and emission on S vertices (f = S / vertices per frame), the gradients of f x the
    frame's training samples, and Adam over f x the frame's training steps x the parameter count
    (a rotating slice of the parameter array: Adam is element-wise). Nothing is extrapolated:
    a step's time is measured whole, and value = S / step time."""

    def __init__(self, wl: dict, train: bool, target_s: float = 0.5):
        import oracle as O
        self.O = O
        O.set_threads(os.cpu_count() or 1)
        self.cores = O.threads()
        self.wl, self.train = wl, train
        self.cfg = O.default_config(**config_fields("fp32", wl, 1 << 21, 1 << 18))
        npar, ntab, _, _ = O.param_count(self.cfg)
        rng = np.random.default_rng(0)
        self.params = np.concatenate([rng.uniform(-0.5, 0.5, ntab),
                                      rng.uniform(-0.1, 0.1, npar - ntab)]).astype(np.float32)
        self.m = np.zeros_like(self.params)
        self.v = np.zeros_like(self.params)
        self.g = np.zeros_like(self.params)   # gradient buffer, reused as a trainer would
        self.t = 0
        self.slice0 = 0
        self.dp = O.default_decide()
        self.frame_vertices = wl["bounces"] * wl["n_vert"]
        self._size(32_768)
        a = time.perf_counter()
        self.step()
        dt = time.perf_counter() - a
        s = int(min(262_144, max(32_768, 32_768 * target_s / max(dt, 1e-3))))
        self._size(s // 1024 * 1024)

    def _size(self, s: int):
        wl, O = self.wl, self.O
        self.S = s
        self.f = s / self.frame_vertices
        self.vx = O.synth(7, s)
        self.nt = max(256, int(round(self.f * wl["train_steps"] * wl["train_batch"]))) \
            if self.train else 0
        self.tv = O.synth(8, self.nt) if self.train else None
        self.n_adam = int(round(self.f * wl["train_steps"] * self.params.size)) if self.train else 0

    def step(self):
        O = self.O
        r = O.infer(self.cfg, self.params, self.vx, self.dp, "f32", want=("stats", "rrs"))
        O.decide_emit(r["rrs"].astype(np.float32), self.vx["rnd"], self.S, 0, self.dp,
                      shift_n=self.S)
        if self.train:
            g, _ = O.train_grads(self.cfg, self.params, self.tv, self.tv["target"], "f32",
                                 out=self.g)
            self.t += 1
            first = self.slice0
            count = min(self.n_adam, self.params.size - first)
            O.adam(self.cfg, self.params, g, self.m, self.v, self.t, first, count)
            self.slice0 = (first + count) % self.params.size

    def describe(self) -> str:
        s = f"per step: infer+decide+emit on {self.S} vertices"
        if self.train:
            s += (f", train gradients on {self.nt} samples and Adam over {self.n_adam} "
                  f"parameters (the same fraction {self.f:.2e} of the frame)")
        return s

    def run(self, steps: int, warmup: int, seconds: float | None = None):
        """(vertices/s, mean step seconds, steps timed)"""
        for _ in range(warmup):
            self.step()
        times = []
        t0 = time.perf_counter()
        while True:
            a = time.perf_counter()
            self.step()
            times.append(time.perf_counter() - a)
            if seconds is None and len(times) >= steps:
                break
            if seconds is not None and time.perf_counter() - t0 > seconds:
                break
        step_s = float(np.mean(times))
        return self.S / step_s, step_s, len(times)


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU path on the host cores, on rank 0 only."""
    if rank != 0:
        return 0
    wl = WORKLOADS[args.workload]
    train = do_train_of(args, wl)
    cpu = CpuFrameSample(wl, train)
    value, step_s, k = cpu.run(args.steps, args.warmup)
    line = {
        "metric": METRIC, "value": value, "unit": "vertices/s", "n_gpus": args.gpus,
        "steps": k, "warmup": args.warmup, "ms_per_step": step_s * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "impl": "reference",
        "config": frame_config(args.workload, wl, train, args.precision, world),
        "cpu_baseline": {"value": value, "unit": "vertices/s", "cores": cpu.cores,
                         "kind": "port", "sample": cpu.describe()},
        "e2e": {"value": value, "unit": "vertices/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "the reference's CPU path: the FP32 C restatement in oracle/ (encoding, MLPs, glue, "
                "factor, decision and emission, losses, gradients, Adam) with OpenMP on all host "
                "threads; the reference itself needs OptiX, KiRaRay and tiny-cuda-nn and cannot be "
                "built here. Each step is a bounded sample of the frame, timed whole",
    }
    print(json.dumps(line), flush=True)
    return 0


# ---- the GPU arms ---------------------------------------------------------------------------

def pinned(torch, v: dict, keys):
    return {k: torch.from_numpy(v[k].view(np.int32) if v[k].dtype == np.uint32 else v[k]).pin_memory()
            for k in keys}


def soa_of(b):
    return nb.vertex_soa(b["pos"], b["wi"], b["normal"], b["roughness"], b["albedo"], b["thp"],
                         b["depth"], b["ref_mean"])


def step_outputs(torch, dev, n, cap, n_sizes=1):
    return dict(stats=torch.empty(3 * n, device=dev), rrs=torch.empty(n, device=dev),
                norm=torch.empty(n, device=dev),
                split=torch.empty(n, dtype=torch.uint8, device=dev),
                q=torch.empty(cap, dtype=torch.int32, device=dev),
                sz=torch.zeros(n_sizes, dtype=torch.int32, device=dev))


def batched_counts(n_top, depths, seed):
    """Depth d holds round(n_top x 0.6^d) path vertices; 10 % of them are split into U{1..4}
    copies. Returns, per depth, the base count and the copy multipliers."""
    rng = np.random.default_rng(seed)
    out = []
    for d in range(depths):
        base = int(round(n_top * 0.6 ** d))
        mult = np.where(rng.random(base) < 0.1, rng.integers(1, 5, base), 1)
        out.append((base, mult))
    return out


def batched_total(wl) -> int:
    return int(sum(int(m.sum()) for _, m in batched_counts(wl["n_vert"], wl["bounces"], 2024)))


def batched_vertices(n_top, depths, seed):
    """The concatenated records of all depths (a split vertex re-enters the next queue several
    times) and the per-depth counts."""
    counts, parts = [], []
    for d, (base, mult) in enumerate(batched_counts(n_top, depths, 2024)):
        v = nb.synth(seed * 131 + d, base)
        idx = np.repeat(np.arange(base), mult)
        sub = {k: np.ascontiguousarray(a[idx]) for k, a in v.items() if k in FIELDS}
        sub["depth"] = np.full(idx.size, d, np.uint32)
        counts.append(int(idx.size))
        parts.append(sub)
    return {k: np.concatenate([p[k] for p in parts]) for k in FIELDS}, counts


class Timer:
    """Device time of K steps on the current stream (CUDA events), max over ranks."""

    def __init__(self, torch, dist, dev):
        self.torch, self.dist, self.dev = torch, dist, dev

    def sync(self):
        self.torch.cuda.synchronize()
        if self.dist:
            self.dist.barrier()
        self.torch.cuda.synchronize()

    def __call__(self, fn, steps, warmup, clocks=None):
        torch = self.torch
        for _ in range(warmup):
            fn()
        self.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ctx = clocks if clocks is not None else _Null()
        with ctx:
            e0.record()
            for _ in range(steps):
                fn()
            e1.record()
            torch.cuda.synchronize()
        self.sync()
        ms = e0.elapsed_time(e1)
        if self.dist:
            t = torch.tensor([ms], device=self.dev)
            self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms / steps


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


class FrameArm:
    """One precision of a per-bounce frame workload on this GPU: the network, its outputs and the
    step (every bounce's nrrs_step, then the frame's training steps)."""

    def __init__(self, torch, dev, stream, wl, precision, dev_b, td, train, world,
                 launch_shape=None, tune=True, sharded=False, cell_image=True):
        self.torch, self.dev, self.stream, self.wl = torch, dev, stream, wl
        self.B, self.N = wl["bounces"], wl["n_vert"]
        self.precision = precision
        self.dev_b, self.td, self.train = dev_b, td, train
        self.net = nb.NRRSNetwork(make_config(precision, wl, self.N, wl["train_batch"],
                                              world if sharded else 0))
        if not cell_image and self.net.cell_image():
            self.net.set_cell_image(False)
        self.tune = None
        if launch_shape:
            shape = [int(x) for x in launch_shape.split(",")]
            if len(shape) > 2 and precision != "fp32":
                self.net.set_infer_split(shape[2])
            self.net.set_launch_shape(shape[0], shape[1])
        elif tune:
            self.tune = json.loads(self.net.autotune(self.N))
        self.cap = 9 * self.N
        self.outs = [step_outputs(torch, dev, self.N, self.cap) for _ in range(self.B)]
        self.soas = [soa_of(b) for b in dev_b]
        self.tsoa = soa_of(td) if train else None
        self.loss = torch.zeros(2, dtype=torch.float64, device=dev)
        self.dp = nb.default_decide()
        self.sharded = None
        self.world = world
        if sharded:
            # each rank holds one shard of an N-times larger queue: one integer all-reduce of the
            # exact sum per bounce, data-parallel gradients per train step
            from nrrs_parallel import ShardedNRRS
            self.sharded = ShardedNRRS(self.net)
            self.acc = torch.zeros(1, dtype=torch.int64, device=dev)
            self.grads_buf = torch.zeros(self.net.param_count(), dtype=torch.float32, device=dev)

    def step(self, pre=None, post=None):
        net, dp, N, s = self.net, self.dp, self.N, self.stream
        for d in range(self.B):
            o = self.outs[d]
            if pre:
                pre(d)
            if self.sharded is None:
                net.generateRRSNumber(self.soas[d], self.dev_b[d]["rnd"], N, N, 0, dp, o["stats"],
                                      o["rrs"], o["norm"], o["split"], o["q"], self.cap, o["sz"], s)
            else:
                self.sharded.step(self.soas[d], self.dev_b[d]["rnd"], N, N * self.world, 0, dp,
                                  o["stats"], o["rrs"], o["norm"], o["split"], o["q"], self.cap,
                                  o["sz"], self.acc, s)
            if post:
                post(d)
        if self.train and pre:
            pre("train")
        for _ in range(self.wl["train_steps"] if self.train else 0):
            if self.sharded is None:
                net.train(self.tsoa, self.td["target"], self.wl["train_batch"], self.loss, s)
            else:
                self.sharded.train_step(self.tsoa, self.td["target"], self.wl["train_batch"],
                                        self.grads_buf, self.loss, s)
        if self.train and post:
            post("train")

    def measure(self, timer, steps, warmup, clocks=None):
        """ms per step, per-kernel profile, our kernel launches in the timed region and the
        device time of the training phase (events around each frame's training steps: its
        kernels overlap across streams, so their summed times would overstate it)"""
        import torch
        net = self.net
        for _ in range(warmup):
            self.step()
        timer.sync()
        spans = []

        def pre(tag):
            if tag == "train":
                e = torch.cuda.Event(enable_timing=True)
                e.record()
                spans.append([e, None])

        def post(tag):
            if tag == "train":
                e = torch.cuda.Event(enable_timing=True)
                e.record()
                spans[-1][1] = e

        l0 = net.launch_count()
        net.profile(True)
        net.profile_read()
        ms = timer(lambda: self.step(pre, post), steps, 0, clocks)
        launches = net.launch_count() - l0
        prof = net.profile_read()
        net.profile(False)
        torch.cuda.synchronize()
        self.train_ms = sum(a.elapsed_time(b) for a, b in spans if b is not None) if spans else None
        return ms, prof, launches

    def close(self):
        self.net.close()


def train_rate(prof, wl, steps, train_ms=None):
    """training samples per second from the device time of the timed frames' training phases
    (or, without it, the summed times of the training kernels)"""
    t_train = train_ms if train_ms else sum(
        t for k, (n, t) in prof.items() if k.startswith("train") or k == "adam"
        or k in ("pack_weights", "table_half"))
    return wl["train_steps"] * wl["train_batch"] * steps / (t_train * 1e-3) if t_train else None


def frame_inputs(torch, dev, wl, seed0, rank, train):
    host_b, dev_b = [], []
    for d in range(wl["bounces"]):
        v = nb.synth(seed0 + 97 * rank + d, wl["n_vert"])
        v["depth"] = np.full(wl["n_vert"], d, np.uint32)
        hb = pinned(torch, v, FIELDS)
        host_b.append(hb)
        dev_b.append({k: t.to(dev) for k, t in hb.items()})
    th = td = None
    if train:
        tv = nb.synth(5000 + rank, wl["train_batch"])
        th = pinned(torch, tv, FIELDS + ("target",))
        td = {k: t.to(dev) for k, t in th.items()}
    return host_b, dev_b, th, td


def roofline_of(prof, precision, mode, wl, inf_vertices, workload):
    """Algorithmic bytes per vertex of each inference kernel (every hash-corner gather at table
    precision) for the HBM line; StatNet + RRSNet FLOPs over the MLP kernels for the tensor line."""
    hbm, bf16, src = measured_peaks()
    feat_bytes = 4 if precision == "fp32" else 2
    gathered = 16 * 8 * 2 * feat_bytes
    attrs = 12 * 5 + 4 * 3                        # wi, normal, albedo, thp, pos; rough, ref, depth
    w_, h_ = wl["width"], wl["hidden"]
    flop_stat = 2 * (64 * w_ + (h_ - 1) * w_ * w_ + w_ * 3)
    flop_rrs = 2 * (16 * w_ + (h_ - 1) * w_ * w_ + w_)
    b_of = {"infer_fp32": SOA_BYTES + gathered + 16,
            "encode": 4 * 12 + gathered + 64,
            "infer_tc": (SOA_BYTES + gathered + 16 if mode == 0 else
                         (64 + attrs - 12 + 16 if mode == 1 else 64 + attrs - 12 + 12 + 32)),
            "infer_rrs": 32 + 4}
    roof = mlp = None
    cands = {k: prof[k] for k in b_of if k in prof and prof[k][0]}
    if cands:
        kind = max(cands, key=lambda k: cands[k][1])
        n_l, ms_l = cands[kind]
        launch_ms = ms_l / n_l
        per_launch = inf_vertices / n_l
        b_vertex = b_of[kind]
        achieved = b_vertex * per_launch / (launch_ms * 1e-3) / 1e9
        tpv = traffic_per_vertex(kind, workload)
        roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_source": src,
                "traffic": (tpv * per_launch) if tpv else None, "kernel": kind,
                "algorithmic_bytes_per_vertex": b_vertex, "vertices_per_launch": per_launch,
                "launch_ms": launch_ms, "inference_mode": mode}
    mlp_kinds = [k for k in ("infer_tc", "infer_rrs") if k in prof and prof[k][0]]
    if precision != "fp32" and mlp_kinds:
        ms_mlp = sum(prof[k][1] for k in mlp_kinds)
        n_launch = prof["infer_tc"][0]
        tflops = (flop_stat + flop_rrs) * inf_vertices / (ms_mlp * 1e-3) / 1e12
        mlp = {"bound": "tensor", "kernels": mlp_kinds, "achieved": tflops, "peak": bf16,
               "unit": "TFLOP/s", "frac": tflops / bf16, "peak_source": src,
               "flop_per_vertex": flop_stat + flop_rrs, "ms_per_launch": ms_mlp / n_launch,
               "note": "StatNet + RRSNet MLP FLOPs (true layer sizes) over the time of the "
                       "kernels that run them; in the fused mode that kernel also gathers"}
    return roof, mlp


def rel_stats(a, b, floor=None):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    d = np.abs(a - b) / (np.maximum(np.abs(b), floor) if floor else np.abs(b))
    return {"max": float(d.max()), "mean": float(d.mean())}


def frame_errors(torch, mixed: FrameArm, fp32: FrameArm, sample_stride: int = 509):
    """Errors of both paths at equal parameters (the mixed network's trained state): stats and
    factors of bounce 0 against the FP64 oracle on a strided sample and against each other on
    every vertex; losses of one training step (gradients only) on a 16,384-sample batch; the
    mixed path's decision against the oracle's on the same factors."""
    import oracle as O
    s = mixed.stream
    p = mixed.net.get_params()
    fp32.net.set_params(p)
    N = mixed.N
    d0 = mixed.dev_b[0]
    res = {}
    outs = {}
    for name, arm in (("mixed", mixed), ("fp32", fp32)):
        st = torch.empty(3 * N, device=mixed.dev)
        rr = torch.empty(N, device=mixed.dev)
        arm.net.inference(mixed.soas[0], N, arm.dp, st, rr, s)
        torch.cuda.synchronize()
        outs[name] = (st.cpu().numpy().reshape(N, 3), rr.cpu().numpy())
    idx = np.arange(0, N, sample_stride)
    host = {k: t.cpu().numpy() for k, t in d0.items()}
    sub = {k: np.ascontiguousarray(host[k][idx]) for k in FIELDS}
    sub["depth"] = sub["depth"].view(np.uint32)
    O.set_threads(os.cpu_count() or 1)
    o64 = O.infer(mixed.net.config, p, sub, mixed.dp, "f64", want=("stats", "rrs"))
    for name in ("mixed", "fp32"):
        st, rr = outs[name]
        res[name + "_vs_fp64_oracle"] = {
            "stats": rel_stats(st[idx], o64["stats"], floor=1.0),
            "factors": rel_stats(rr[idx], o64["rrs"])}
    res["mixed_vs_fp32_path"] = {"stats": rel_stats(outs["mixed"][0], outs["fp32"][0], floor=1.0),
                                 "factors": rel_stats(outs["mixed"][1], outs["fp32"][1])}
    # losses of one training step at p (gradients only, no update) on a 16,384-sample batch
    nt = 16_384
    tv = {k: np.ascontiguousarray(t[:nt].cpu().numpy()) for k, t in mixed.td.items()}
    tv["depth"] = tv["depth"].view(np.uint32)
    tsoa = soa_of({k: t[:nt] for k, t in mixed.td.items()})
    losses = {}
    for name, arm in (("mixed", mixed), ("fp32", fp32)):
        l = torch.zeros(2, dtype=torch.float64, device=mixed.dev)
        arm.net.trainGrads(tsoa, mixed.td["target"][:nt], nt, l, s)
        torch.cuda.synchronize()
        losses[name] = l.cpu().numpy()
    _, l64 = O.train_grads(mixed.net.config, p, tv, tv["target"], "f64")
    for name in ("mixed", "fp32"):
        res[name + "_vs_fp64_oracle"]["loss"] = rel_stats(losses[name], l64)
    res["mixed_vs_fp32_path"]["loss"] = rel_stats(losses["mixed"], losses["fp32"])
    # decisions at equal factors: the mixed factors through the library and through the oracle
    rr_dev = torch.from_numpy(outs["mixed"][1]).to(mixed.dev)
    o = step_outputs(torch, mixed.dev, N, 9 * N)
    mixed.net.decideEmit(rr_dev, d0["rnd"], N, N, 0, mixed.dp, o["norm"], o["split"], o["q"],
                         9 * N, o["sz"], stream=s)
    torch.cuda.synchronize()
    od = O.decide_emit(outs["mixed"][1], host["rnd"], N, 0, mixed.dp, capacity=9 * N,
                       shift_n=mixed.net.config.max_queue)
    tot = int(o["sz"].cpu().numpy().view(np.uint32)[0])
    same = (tot == od["total"] and
            np.array_equal(o["split"].cpu().numpy(), od["split"]) and
            np.array_equal(o["q"][:tot].cpu().numpy().view(np.uint32), od["queue"]))
    res["decisions_bit_exact_at_equal_factors"] = bool(same)
    res["decision_vertices"] = N
    res["sample"] = (f"stats and factors: bounce 0 of the frame, every {sample_stride}th of {N} "
                     f"vertices against the FP64 oracle ({idx.size} vertices), all {N} between "
                     f"the paths; loss: one step's losses on {nt} training samples; relative "
                     f"error |a-b|/|b| (stats: log-statistics, denominator floored at 1); "
                     f"parameters: the mixed network after the timed frames, set on both paths")
    return res


def run_frame_pair(args, torch, dev, stream, timer, name, steps, warmup, fp32_steps, rank, world,
                   headline):
    """The mixed arm and the plain FP32 per-depth arm of one frame workload on the same inputs."""
    wl = WORKLOADS[name]
    train = do_train_of(args, wl)
    host_b, dev_b, th, td = frame_inputs(torch, dev, wl, 1000, rank, train)
    prec = args.precision if headline and args.precision else wl["precision"]
    mixed = FrameArm(torch, dev, stream, wl, prec, dev_b, td, train, world,
                     launch_shape=args.launch_shape, sharded=world > 1,
                     cell_image=args.cell_image)
    out = {"name": name, "wl": wl, "train": train, "precision": prec, "arm": mixed,
           "host_b": host_b, "dev_b": dev_b, "th": th, "td": td}
    clk = ClockSampler(env_int("LOCAL_RANK", 0)) if headline else None
    ms, prof, launches = mixed.measure(timer, steps, warmup, clk)
    out.update(ms=ms, prof=prof, launches=launches, clocks=clk.summary() if clk else None)
    out["value"] = wl["bounces"] * wl["n_vert"] * world / (ms * 1e-3)
    out["train_rate"] = train_rate(prof, wl, steps, mixed.train_ms) if train else None
    out["status"] = mixed.net.device_status(stream)
    if world == 1 and fp32_steps > 0 and prec != "fp32":
        fp = FrameArm(torch, dev, stream, wl, "fp32", dev_b, td, train, 1,
                      tune=True)
        clk32 = ClockSampler(env_int("LOCAL_RANK", 0)) if headline else None
        ms32, prof32, _ = fp.measure(timer, fp32_steps, 1, clk32)
        out["fp32"] = {"value": wl["bounces"] * wl["n_vert"] / (ms32 * 1e-3), "ms_per_step": ms32,
                       "train_samples_per_s": train_rate(prof32, wl, fp32_steps, fp.train_ms)
                       if train else None,
                       "steps": fp32_steps, "warmup": 1,
                       "clocks": clk32.summary() if clk32 else None,
                       "kernels": {k: {"launches": n, "ms_total": t} for k, (n, t) in prof32.items()}}
        if headline and args.errors:
            out["errors"] = frame_errors(torch, mixed, fp)
        fp.close()
    return out


def run_batched(args, torch, dev, stream, timer, steps, warmup, rank):
    """Config 3: the mixed path's batched step as one CUDA-graph launch against the plain FP32
    path launched depth by depth, on the same vertices."""
    wl = WORKLOADS["batched"]
    B, N = wl["bounces"], wl["n_vert"]
    cat, counts = batched_vertices(N, B, 2024 + rank)
    db = {k: t.to(dev) for k, t in pinned(torch, cat, FIELDS).items()}
    total = int(sum(counts))
    dp = nb.default_decide()
    net = nb.NRRSNetwork(make_config(wl["precision"], wl, total, wl["train_batch"]))
    tune = json.loads(net.autotune(N))
    caps = [9 * c for c in counts]
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    qoffs = np.concatenate([[0], np.cumsum(caps)]).astype(np.int64)
    segs = [nb.Segment(int(offs[k]), counts[k], N, 0, int(qoffs[k]), caps[k]) for k in range(B)]
    ob = step_outputs(torch, dev, total, int(qoffs[-1]), B)
    l0 = net.launch_count()
    graph = net.captureBatched(soa_of(db), db["rnd"], segs, dp, ob["stats"], ob["rrs"], ob["norm"],
                               ob["split"], ob["q"], ob["sz"])
    kernels_per_graph = net.launch_count() - l0
    ms_graph = timer(lambda: graph.launch(stream), steps, warmup)
    per = []
    for k in range(B):
        sub = {f: t[int(offs[k]):int(offs[k + 1])] for f, t in db.items()}
        per.append((sub, soa_of(sub), step_outputs(torch, dev, counts[k], caps[k])))

    def per_depth(n_):
        for k, (sub, s, p) in enumerate(per):
            n_.generateRRSNumber(s, sub["rnd"], counts[k], N, 0, dp, p["stats"], p["rrs"],
                                 p["norm"], p["split"], p["q"], caps[k], p["sz"], stream)

    ms_mixed_pd = timer(lambda: per_depth(net), steps, 2)
    same = True
    for k, (sub, s, p) in enumerate(per):
        a0, a1 = int(offs[k]), int(offs[k + 1])
        same &= bool(torch.equal(p["split"], ob["split"][a0:a1]))
        same &= bool(torch.equal(p["rrs"], ob["rrs"][a0:a1]))
        same &= bool(torch.equal(p["q"][:int(p["sz"].item())] + int(offs[k]),
                                 ob["q"][int(qoffs[k]):int(qoffs[k]) + int(ob["sz"][k].item())]))
    fp = nb.NRRSNetwork(make_config("fp32", wl, max(counts), wl["train_batch"]))
    fp.autotune(max(counts))
    ms_fp32_pd = timer(lambda: per_depth(fp), max(3, steps // 5), 1)
    graph.close()
    net.close()
    fp.close()
    return {"workload": workload_name("batched", wl, False, wl["precision"]),
            "vertices_per_step": total, "vertices_per_depth": counts,
            "mixed_graph": {"value": total / (ms_graph * 1e-3), "ms_per_step": ms_graph,
                            "kernels_per_graph": kernels_per_graph, "launches_per_step": 1},
            "mixed_per_depth": {"value": total / (ms_mixed_pd * 1e-3), "ms_per_step": ms_mixed_pd},
            "fp32_per_depth": {"value": total / (ms_fp32_pd * 1e-3), "ms_per_step": ms_fp32_pd},
            "mixed_graph_vs_fp32_per_depth": ms_fp32_pd / ms_graph,
            "graph_decisions_equal_per_depth": same,
            "autotune_best": tune.get("best") or tune.get("cached")}


def e2e_of(torch, dev, timer, arm: FrameArm, host_b, th, steps, warmup):
    """The headline metric end to end through the C-ABI with host-resident inputs."""
    B, wl, train = arm.B, arm.wl, arm.train
    dev_b, td = arm.dev_b, arm.td
    total = B * arm.N
    h2d = total * (SOA_BYTES + RND_BYTES) + (
        wl["train_batch"] * (SOA_BYTES + RND_BYTES + TARGET_BYTES) if train else 0)
    d2h = B * 4 + (16 if train else 0)
    sizes_h = torch.zeros(B, dtype=torch.int32).pin_memory()
    loss_h = torch.zeros(2, dtype=torch.float64).pin_memory()
    # A caller with host-resident inputs overlaps the upload of the next bounce with the compute
    # of the current one: copies run on their own stream, each bounce waits for its inputs, and a
    # buffer is refilled only after the previous step's compute has used it.
    cur = torch.cuda.current_stream()
    copy_stream = torch.cuda.Stream(device=dev)
    keys = list(range(B)) + (["train"] if train else [])
    ev_copied = {k: torch.cuda.Event() for k in keys}
    ev_used = {k: torch.cuda.Event() for k in keys}
    for k in keys:
        ev_used[k].record(cur)

    def step_e2e():
        with torch.cuda.stream(copy_stream):
            for d, (hb, db) in enumerate(zip(host_b, dev_b)):
                copy_stream.wait_event(ev_used[d])
                for k in FIELDS:
                    db[k].copy_(hb[k], non_blocking=True)
                ev_copied[d].record(copy_stream)
            if train:
                copy_stream.wait_event(ev_used["train"])
                for k in FIELDS + ("target",):
                    td[k].copy_(th[k], non_blocking=True)
                ev_copied["train"].record(copy_stream)
        arm.step(pre=lambda k: cur.wait_event(ev_copied[k]), post=lambda k: ev_used[k].record(cur))
        for d in range(B):
            sizes_h[d:d + 1].copy_(arm.outs[d]["sz"], non_blocking=True)
        if train:
            loss_h.copy_(arm.loss, non_blocking=True)

    for _ in range(warmup):
        step_e2e()
    timer.sync()
    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a0.record(cur)
    copy_stream.wait_event(a0)      # no upload starts before the timed region does
    for _ in range(steps):
        step_e2e()
    a1.record(cur)                  # after the last compute, which waited for every upload
    torch.cuda.synchronize()
    ms = a0.elapsed_time(a1) / steps
    if timer.dist:
        t = torch.tensor([ms], device=dev)
        timer.dist.all_reduce(t, op=timer.dist.ReduceOp.MAX)
        ms = float(t.item())
    return {"value": total * arm.world / (ms * 1e-3), "unit": "vertices/s", "ms_per_step": ms,
            "h2d_gbs": h2d / (ms * 1e-3) / 1e9,
            "overlap": "uploads on a copy stream, bounce d+1 during the compute of bounce d",
            "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": steps}


def pair_summary(p):
    s = {"workload": workload_name(p["name"], p["wl"], p["train"], p["precision"]),
         "mixed": {"value": p["value"], "ms_per_step": p["ms"],
                   "train_samples_per_s": p["train_rate"]}}
    if "fp32" in p:
        f = p["fp32"]
        s["fp32_per_depth"] = {k: f[k] for k in ("value", "ms_per_step", "train_samples_per_s",
                                                 "steps")}
        s["mixed_vs_fp32"] = {"vertices_per_s": p["value"] / f["value"],
                              "train_samples_per_s": (p["train_rate"] / f["train_samples_per_s"]
                                                      if p["train_rate"] and f["train_samples_per_s"]
                                                      else None)}
    return s


def run_ours(args, rank, world, local_rank):
    import torch
    load_product()
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream().cuda_stream
    timer = Timer(torch, dist, dev)
    name = args.workload
    if name == "batched":
        b = run_batched(args, torch, dev, stream, timer, args.steps, args.warmup, rank)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": b["mixed_graph"]["value"],
                              "unit": "vertices/s", "n_gpus": world, "steps": args.steps,
                              "warmup": args.warmup, "ms_per_step": b["mixed_graph"]["ms_per_step"],
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                              "dtype": "f16", "data": "synthetic", "batched": b}), flush=True)
        return 0

    # ---- headline: the frame workload, mixed and plain FP32 on the same inputs ----
    wl = WORKLOADS[name]
    fp32_steps = 0 if args.only else max(2, min(args.steps, 3))
    p = run_frame_pair(args, torch, dev, stream, timer, name, args.steps, args.warmup,
                       fp32_steps, rank, world, headline=True)
    arm = p["arm"]
    prof = p["prof"]
    mode = arm.net.infer_split() if p["precision"] != "fp32" else 0
    inf_vertices = wl["bounces"] * wl["n_vert"] * args.steps
    roof, mlp_roof = roofline_of(prof, p["precision"], mode, wl, inf_vertices, name)
    if roof:
        rb = request_bound(roof, name, (p["clocks"] or {}).get("sm_mhz"),
                           torch.cuda.get_device_properties(dev).multi_processor_count)
        if rb:
            roof["request_bound"] = rb
    e2e = e2e_of(torch, dev, timer, arm, p["host_b"], p["th"], max(2, min(args.steps, 10)),
                 min(2, args.warmup))
    line = {
        "metric": METRIC, "value": p["value"], "unit": "vertices/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": p["ms"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {"fp16": "f16", "bf16": "bf16", "fp32": "f32"}[p["precision"]],
        "data": "synthetic (seeded; the distributions of the workload definition)",
        "config": frame_config(name, wl, p["train"], p["precision"], world),
        "clocks": p["clocks"],
        "e2e": e2e,
        "gpu_launches": p["launches"],
        "roofline": roof,
        "mlp_roofline": mlp_roof,
        "train_samples_per_s": p["train_rate"],
    }
    if "fp32" in p:
        f = p["fp32"]
        line["fp32_per_depth"] = f
        line["mixed_vs_fp32"] = pair_summary(p)["mixed_vs_fp32"]
        if "errors" in p:
            line["errors"] = p["errors"]
    line["kernels"] = {k: {"launches": n, "ms_total": t, "ms_per_launch": t / n}
                       for k, (n, t) in prof.items()}
    line["launch_shape"] = list(arm.net.launch_shape()) + (
        [arm.net.infer_split()] if p["precision"] != "fp32" else [])
    if p["precision"] != "fp32":
        line["cell_image"] = arm.net.cell_image()
    if arm.tune:
        line["autotune"] = {"best": arm.tune.get("best") or arm.tune.get("cached"),
                            "trials": arm.tune.get("trials")}
    line["device_status"] = list(p["status"])
    arm.close()
    del p, arm
    torch.cuda.empty_cache()

    # ---- the other configurations of the workload definition, beside the headline ----
    if world == 1 and not args.only:
        sec = {}
        if name != "frame1080p":
            try:
                q = run_frame_pair(args, torch, dev, stream, timer, "frame1080p", 20, 3, 5, rank,
                                   1, headline=False)
                sec["frame1080p"] = pair_summary(q)
                q["arm"].close()
                del q
            except Exception as exc:   # the headline line is printed regardless
                sec["frame1080p"] = {"error": f"{type(exc).__name__}: {exc}"}
            torch.cuda.empty_cache()
        try:
            sec["batched"] = run_batched(args, torch, dev, stream, timer, 20, 3, rank)
        except Exception as exc:
            sec["batched"] = {"error": f"{type(exc).__name__}: {exc}"}
        line["secondary"] = sec
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = CpuFrameSample(wl, do_train_of(args, wl))
        v_c, _, k = cpu.run(0, 1, seconds=12.0)
        line["cpu_baseline"] = {"value": v_c, "unit": "vertices/s", "cores": cpu.cores,
                                "kind": "port", "sample": f"{k} steps; " + cpu.describe()}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


# ---- records1080p: path-node records, radiance and the training batch ------------------------

RECORD_KEYS = ("pos", "wi", "normal", "albedo", "roughness", "thp", "depth", "pixel", "rrs",
               "record", "parent")
CONTRIB_KEYS = ("contrib_node", "contrib")


def records_params(**kw):
    return nb.default_train_data_params(ignore_zero_l=0, copy_rrs_node=1, dedupe_rrs_target=1,
                                        **kw)


def records_frame(seed: int, wl: dict):
    """The synthetic frame: path records, the film (RGBA per pixel) and the frame's radiance per
    pixel (the sum of its samples, spp 1)."""
    P = wl["n_vert"]
    bounces, image = nb.synth_paths(seed, P, bounces=wl["bounces"],
                                    capacity=wl["node_rate"] * P)
    rng = np.random.default_rng(seed + 1)
    pixel_l = (image[:, :3] * rng.lognormal(0.0, 0.5, size=(P, 3))).astype(np.float32)
    return bounces, image, pixel_l


def records_geom(wl):
    """Frame width and height of the workload (a one-row frame for other pixel counts)."""
    P = wl["n_vert"]
    return (1920, 1080) if P == 1920 * 1080 else (P, 1)


def records_name(wl):
    return f"records_{wl['bounces']}bounce_{wl['n_vert']}px_rate{wl['node_rate']}"


def records_cpu(wl, bounces, image, pixel_l, seconds: float):
    """The oracle (sequential C, one core) on whole frames of the workload until `seconds`: the
    patch counts, the per-pixel error and its sum, then the records, the batch and the weights."""
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle as O
    P = wl["n_vert"]
    W, H = records_geom(wl)
    pe = nb.default_pixel_error_params(W, H)
    wl_ = np.zeros((P, 3), np.float32)
    cur = np.zeros((P, 3), np.float32)
    acc = np.zeros(P, np.uint32)
    err = np.zeros(2 * P, np.float32)
    spp = np.zeros(P, np.float32)
    uerr = np.zeros(P, np.float32)
    prm = records_params(frame_width=W, error_image_scale=1, error_per_pixel=err.ctypes.data,
                         samples_per_patch=spp.ctypes.data)
    cap = wl["node_rate"] * P
    hn = O.HostNodes(cap)                 # allocated once, reset per frame, as a renderer would
    out = O.batch_arrays(cap)
    counts = np.zeros(P, np.uint32)
    t, reps, nodes = 0.0, 0, 0
    while True:
        a = time.perf_counter()
        spp[:] = 0
        hn.reset()
        for b in bounces:
            hn.record_nodes(b)
            hn.record_radiance(b["contrib_node"], b["contrib"])
            O.count_patch_samples(pe, b["pixel"], spp)
        O.accumulate_weighted_l(pe, pixel_l, 1, False, wl_, cur, acc)
        O.update_weighted_l(pe, cur, acc, wl_)
        O.calculate_error(pe, image, wl_, spp, err)
        O.ubs_error(pe, pixel_l, 1, image, uerr)
        counts[:] = 0
        batch, total = hn.generate(prm, cap, image=image, n_pixels=P, pixel_samples=counts, out=out)
        O.sample_weights(batch["pixel"], counts, P)
        t += time.perf_counter() - a
        reps += 1
        nodes = hn.size
        if t > seconds:
            break
    return nodes * reps / t, reps, t / reps


def run_records_reference(args, rank, world):
    if rank != 0:
        return 0
    wl = WORKLOADS[args.workload]
    bounces, image, pixel_l = records_frame(4242, wl)
    secs = min(60.0, max(1.0, 0.05 * args.steps))
    value, reps, frame_s = records_cpu(wl, bounces, image, pixel_l, secs)
    line = {
        "metric": "path nodes/s (records + radiance + training batch + weights)",
        "value": value, "unit": "nodes/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": frame_s * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "impl": "reference", "config": {"workload": records_name(wl)},
        "cpu_baseline": {"value": value, "unit": "nodes/s", "cores": 1, "kind": "port",
                         "sample": f"{reps} whole frames"},
        "e2e": {"value": value, "unit": "nodes/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "reference CPU path = sequential C restatement (oracle/records.c) of "
                "recordNode/recordRadiance/nrrs_generate_training_data/"
                "nrrs_calculate_sample_weight and the per-pixel error of trainStep; the "
                "reference runs them on the GPU inside its OptiX integrator, which cannot be "
                "built here",
    }
    print(json.dumps(line), flush=True)
    return 0


def run_records(args, rank, world, local_rank):
    import torch
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local_rank)
    cur = torch.cuda.current_stream()
    stream = cur.cuda_stream
    wl = WORKLOADS[args.workload]
    P = wl["n_vert"]
    cap = wl["node_rate"] * P
    bounces, image, pixel_l = records_frame(4242 + rank, wl)
    W, H = records_geom(wl)
    pe = nb.default_pixel_error_params(W, H)

    def to_t(a):
        a = np.ascontiguousarray(a)
        return torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a)

    host_b = [{k: to_t(b[k]).pin_memory() for k in RECORD_KEYS + CONTRIB_KEYS} for b in bounces]
    dev_b = [{k: t.to(dev) for k, t in hb.items()} for hb in host_b]
    n_of = [len(b["pixel"]) for b in bounces]
    m_of = [len(b["contrib_node"]) for b in bounces]
    outs = [torch.empty(max(n, 1), dtype=torch.int32, device=dev) for n in n_of]
    soas = [nb.vertex_soa(d["pos"], d["wi"], d["normal"], d["roughness"], d["albedo"], d["thp"],
                          d["depth"]) for d in dev_b]
    nbytes = nb.path_nodes_bytes(cap, max(n_of))
    block = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    pn = nb.NRRSPathNodesBuffer(block.data_ptr(), nbytes, cap, max(n_of), stream)
    widths = {"pos": 3, "wi": 3, "normal": 3, "albedo": 3, "roughness": 1, "thp": 3, "depth": 1,
              "ref_mean": 1, "target": 3, "rrs_target": 1, "pixel": 1}
    batch = {k: torch.empty((cap, w) if w > 1 else cap,
                            dtype=torch.int32 if k in ("depth", "pixel") else torch.float32,
                            device=dev) for k, w in widths.items()}
    tb = nb.train_batch(**batch)
    counts = torch.zeros(P, dtype=torch.int32, device=dev)
    weights = torch.empty(cap, dtype=torch.float32, device=dev)
    size_d = torch.zeros(1, dtype=torch.int32, device=dev)
    img_d = torch.from_numpy(image).to(dev)
    img_h = torch.from_numpy(image).pin_memory()
    pl_d = torch.from_numpy(pixel_l).to(dev)
    pl_h = torch.from_numpy(pixel_l).pin_memory()
    size_h = torch.zeros(1, dtype=torch.int32).pin_memory()
    # per-pixel error of the RRSNet loss (trainStep STEP#1-#2), patches of one pixel
    wl_d = torch.zeros((P, 3), dtype=torch.float32, device=dev)
    cur_d = torch.zeros((P, 3), dtype=torch.float32, device=dev)
    acc_d = torch.zeros(P, dtype=torch.int32, device=dev)
    err_d = torch.zeros(2 * P, dtype=torch.float32, device=dev)
    spp_d = torch.zeros(P, dtype=torch.float32, device=dev)
    esum_d = torch.zeros(32, dtype=torch.uint8, device=dev)
    uerr_d = torch.zeros(P, dtype=torch.float32, device=dev)
    usum_d = torch.zeros(32, dtype=torch.uint8, device=dev)
    prm = records_params(frame_width=W, error_image_scale=1, error_per_pixel=err_d.data_ptr(),
                         samples_per_patch=spp_d.data_ptr())

    def step(pre=None, post=None, ev=None):
        pn.reset(stream)
        spp_d.zero_()       # the patch sample counts restart every frame (integrator.cpp:1029)
        for d, db in enumerate(dev_b):
            if pre:
                pre(d)
            if ev:
                ev[("rec", d)][0].record(cur)
            pn.recordNode(soas[d], db["parent"], db["pixel"], db["rrs"], db["record"], n_of[d],
                          outs[d], stream)
            if ev:
                ev[("rec", d)][1].record(cur)
            pn.recordRadiance(db["contrib_node"], db["contrib"], m_of[d], stream)
            if ev:
                ev[("rad", d)][1].record(cur)
            nb.count_patch_samples(pe, db["pixel"], n_of[d], spp_d, stream)
            if ev:
                ev[("cnt", d)][1].record(cur)
            if post:
                post(d)
        counts.zero_()      # mTrainingSamples is zeroed once per frame (integrator.cpp:1041)
        if pre:
            pre("image")
        if ev:
            ev["pe"][0].record(cur)
        nb.accumulate_weighted_l(pe, pl_d, 1, False, wl_d, cur_d, acc_d, stream)
        nb.update_weighted_l(pe, cur_d, acc_d, wl_d, stream)
        nb.calculate_error(pe, img_d, 4, wl_d, spp_d, err_d, esum_d, stream)
        # the frame's error as the per-depth strategy search scores it (UBSAnalyseFrame)
        nb.ubs_error(pe, pl_d, 1, img_d, 4, uerr_d, usum_d, stream)
        if ev:
            ev["pe"][1].record(cur)
        if ev:
            ev["gen"][0].record(cur)
        pn.generate_training_data(prm, tb, cap, size_d, image=img_d, image_channels=4,
                                  n_pixels=P, pixel_samples=counts, stream=stream)
        if ev:
            ev["gen"][1].record(cur)
            # the same call again: the radiance is complete, so it runs the batch kernel alone
            # (and an early-returning radiance launch); the difference times the radiance pass
            counts.zero_()
            ev["batch"][0].record(cur)
            pn.generate_training_data(prm, tb, cap, size_d, image=img_d, image_channels=4,
                                      n_pixels=P, pixel_samples=counts, stream=stream)
            ev["batch"][1].record(cur)
        nb.calculate_sample_weight(batch["pixel"], counts, P, size_d, cap, weights, stream)
        if ev:
            ev["wgt"][1].record(cur)
        if post:
            post("image")

    # per bounce: record count, record writes, radiance, patch counts; then the pixel error
    # (3) and the UBS error, radiance pass, batch, weights (the zero_ fills are torch's)
    launches_per_step = 4 * len(bounces) + 7
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    n_nodes, dropped, flags = pn.status(stream)
    total = int(size_d.item())
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(cur)
        for _ in range(args.steps):
            step()
        e1.record(cur)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    if dist:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    # ---- e2e: host inputs uploaded every frame on a copy stream, the batch size read back ----
    copy_stream = torch.cuda.Stream(device=dev)
    keys = list(range(len(dev_b))) + ["image"]
    ev_copied = {k: torch.cuda.Event() for k in keys}
    ev_used = {k: torch.cuda.Event() for k in keys}
    for k in keys:
        ev_used[k].record(cur)

    def step_e2e():
        with torch.cuda.stream(copy_stream):
            for d, (hb, db) in enumerate(zip(host_b, dev_b)):
                copy_stream.wait_event(ev_used[d])
                for k in hb:
                    db[k].copy_(hb[k], non_blocking=True)
                ev_copied[d].record(copy_stream)
            copy_stream.wait_event(ev_used["image"])
            img_d.copy_(img_h, non_blocking=True)
            pl_d.copy_(pl_h, non_blocking=True)
            ev_copied["image"].record(copy_stream)
        step(pre=lambda k: cur.wait_event(ev_copied[k]), post=lambda k: ev_used[k].record(cur))
        size_h.copy_(size_d, non_blocking=True)

    h2d = (sum(t.numel() * t.element_size() for hb in host_b for t in hb.values()) +
           img_h.numel() * 4 + pl_h.numel() * 4)
    for _ in range(2):
        step_e2e()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2 = max(2, args.steps // 2)
    a0.record(cur)
    copy_stream.wait_event(a0)
    for _ in range(e2):
        step_e2e()
    a1.record(cur)
    torch.cuda.synchronize()
    e2e_ms = a0.elapsed_time(a1) / e2
    if dist:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    assert int(size_h.item()) == total

    # ---- per-call device time (one instrumented frame after the timed ones) ----
    ev = {("rec", d): (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for d in range(len(bounces))}
    ev.update({("rad", d): (ev[("rec", d)][1], torch.cuda.Event(enable_timing=True))
               for d in range(len(bounces))})
    ev.update({("cnt", d): (ev[("rad", d)][1], torch.cuda.Event(enable_timing=True))
               for d in range(len(bounces))})
    ev["pe"] = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    ev["gen"] = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    ev["batch"] = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    ev["wgt"] = (ev["batch"][1], torch.cuda.Event(enable_timing=True))
    step(ev=ev)
    torch.cuda.synchronize()
    t_rec = sum(ev[("rec", d)][0].elapsed_time(ev[("rec", d)][1]) for d in range(len(bounces)))
    t_rad = sum(ev[("rad", d)][0].elapsed_time(ev[("rad", d)][1]) for d in range(len(bounces)))
    t_call = ev["gen"][0].elapsed_time(ev["gen"][1])
    t_gen = ev["batch"][0].elapsed_time(ev["batch"][1])
    t_prop = max(t_call - t_gen, 1e-6)
    t_wgt = ev["wgt"][0].elapsed_time(ev["wgt"][1])
    t_pe = (ev["pe"][0].elapsed_time(ev["pe"][1]) +
            sum(ev[("cnt", d)][0].elapsed_time(ev[("cnt", d)][1]) for d in range(len(bounces))))

    # algorithmic bytes (each array element read or written once; an atomic add counts its
    # 8-byte read and write)
    n_vert, n_contrib = sum(n_of), sum(m_of)
    recorded = n_nodes
    limbs_nz = 6                                    # nonzero limbs of a typical contribution
    # record: per vertex 60 B of three-float fields, 20 B of scalars, the flag and node_out;
    # per node the same 80 B written, 72 B of zeroed radiance, 16 B of tree words and two
    # atomics on the parent
    b_rec = n_vert * (60 + 20 + 1 + 4) + recorded * (60 + 20 + 72 + 16) + recorded * 16
    # radiance: node index and contribution read, the nonzero limbs added
    b_rad = n_contrib * (4 + 12) + n_contrib * limbs_nz * 16
    # radiance pass: per node its parent, flags and 72 B of limbs read, the nonzero limbs added
    b_prop = recorded * (4 + 4 + 72 + limbs_nz * 16)
    # batch: per node limbs, thp, flags, pos, wi, parent and first_child read; per sample
    # normal, albedo, roughness, depth, rrs, pixel and the pixel's image value read, 92 B of
    # sample written and the pixel count incremented
    b_gen = recorded * (72 + 12 + 4 + 12 + 12 + 4 + 4) + total * (24 + 16 + 16 + 92 + 8)
    b_wgt = total * (4 + 4 + 4)
    # pixel error: per ray its pixel read and one atomic on its patch count; per pixel the
    # radiance read, the current sum and count written, blended (read 28 B, write 12 B), the
    # film, estimate and count read and two errors written
    b_pe = n_vert * (4 + 16) + P * (12 + 16 + 28 + 12 + 32 + 8) + P * (12 + 16 + 4)
    # the batch also gathers each sample's two errors and sample count
    b_gen += total * 12
    calls = {"record_nodes": (t_rec, b_rec, 2 * len(bounces)),
             "record_radiance": (t_rad, b_rad, len(bounces)),
             "radiance_pass": (t_prop, b_prop, 1), "batch": (t_gen, b_gen, 1),
             "sample_weights": (t_wgt, b_wgt, 1),
             "pixel_error": (t_pe, b_pe, len(bounces) + 4)}
    peak, _, peak_kind = measured_peaks()
    dom = max(calls, key=lambda k: calls[k][0])
    t_dom, b_dom, n_dom = calls[dom]
    achieved = b_dom / (t_dom * 1e-3) / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind, "traffic": None, "kernel": dom,
            "algorithmic_bytes_per_launch": b_dom / n_dom, "launch_ms": t_dom / n_dom,
            "note": "radiance_pass and batch are the two kernels of nrrs_generate_training_data "
                    "(timed apart by calling it twice: the second call skips the complete "
                    "radiance); record_nodes is a count and a write kernel per call; atomics "
                    "count 16 B (8-byte read and write)"}
    line = {
        "metric": "path nodes/s (records + radiance + training batch + weights)",
        "value": recorded * world / (ms * 1e-3), "unit": "nodes/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": records_name(wl), "pixels": P, "bounces": len(bounces),
                   "vertices_per_frame": n_vert, "nodes_per_frame": recorded,
                   "contributions_per_frame": n_contrib, "samples_per_frame": total,
                   "node_capacity": cap,
                   "switches": "copy_the_rrs_node, ignore_same_training_data_for_rrs_net",
                   "l2": "inputs larger than L2 (about 0.8 GB of vertex and contribution "
                         "arrays per frame, a 3.4 GB node block)",
                   "parallelism": f"replicas{world}"},
        "clocks": clk.summary(),
        "e2e": {"value": recorded * world / (e2e_ms * 1e-3), "unit": "nodes/s",
                "ms_per_step": e2e_ms, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 4,
                "h2d_gbs": h2d / (e2e_ms * 1e-3) / 1e9,
                "overlap": "uploads on a copy stream, bounce d+1 during the records of bounce d"},
        "gpu_launches": launches_per_step * args.steps,
        "roofline": roof,
        "calls": {k: {"ms_per_frame": t, "gbs": b / (t * 1e-3) / 1e9, "launches": n}
                  for k, (t, b, n) in calls.items()},
        "device_status": [dropped, flags],
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        value_c, reps, frame_s = records_cpu(wl, bounces, image, pixel_l, 10.0)
        line["cpu_baseline"] = {"value": value_c, "unit": "nodes/s", "cores": 1, "kind": "port",
                                "sample": f"{reps} whole frames of the workload"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


# ---- render1080p: the path tracer around the NRRS step ---------------------------------------

def run_render(args, rank, world, local_rank):
    import torch
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local_rank)
    cur = torch.cuda.current_stream()
    stream = cur.cuda_stream
    wl = WORKLOADS[args.workload]
    n_pix = wl["n_vert"]               # --vertices gives a smaller 16:9 frame for profiling
    H = 1080 if n_pix == 1920 * 1080 else max(1, int(round((n_pix * 9 / 16) ** 0.5)))
    W = n_pix // H
    P = W * H
    cap = 3 * P
    v, t, m, ma, env = nb.synth_scene(7 + rank, n_boxes=wl["boxes"], closed=True)
    scene = nb.Scene(v, t, m, ma, env)
    n_nodes, n_lights, bvh_depth = scene.info()
    cam = nb.room_camera(W, H, inside=True)
    train = wl.get("train_steps", 0) > 0
    net = nb.NRRSNetwork(make_config(args.precision, wl, cap, max(wl["train_batch"], 1 << 16)))
    net.setStep(3)
    # the library's launch-shape tuner on a queue of one bounce's size, as for the step workloads
    tune = json.loads(net.autotune(P))
    # factors clamped at 1 or above: the normalisation to the pixel budget then keeps about one
    # path per pixel per bounce, as a trained network would; an untrained one kills most paths
    dp = nb.default_decide(clamp_min=1.0)

    f = lambda *sh: torch.zeros(*sh, dtype=torch.float32, device=dev)  # noqa: E731
    i = lambda *sh: torch.zeros(*sh, dtype=torch.int32, device=dev)    # noqa: E731
    rays = {"origin": f(cap, 3), "dir": f(cap, 3), "thp": f(cap, 3), "pdf": f(cap),
            "pixel": i(cap), "node": i(cap)}
    hits = {"prim": i(cap), "t": f(cap), "u": f(cap), "v": f(cap)}
    verts = {"pos": f(cap, 3), "wi": f(cap, 3), "normal": f(cap, 3), "albedo": f(cap, 3),
             "roughness": f(cap), "thp": f(cap, 3), "depth": i(cap), "pixel": i(cap),
             "node": i(cap)}
    shadow = {"origin": f(cap, 3), "dir": f(cap, 3), "tmax": f(cap), "contrib": f(cap, 3),
              "pixel": i(cap), "node": i(cap)}
    film = torch.zeros((P, 9), dtype=torch.int64, device=dev)
    img = f(P, 3)
    scratch = torch.zeros(nb.shade_scratch_bytes(cap), dtype=torch.uint8, device=dev)
    tscratch = torch.zeros(nb.trace_scratch_bytes(cap), dtype=torch.uint8, device=dev)
    n_rays, n_vert, qsize = i(1), i(1), i(1)
    rnd = torch.rand(cap, device=dev, generator=torch.Generator(device=dev).manual_seed(5))
    stats, rrs, rrs_norm = f(3 * cap), f(cap), f(cap)
    split = torch.zeros(cap, dtype=torch.uint8, device=dev)
    queue = i(cap)
    R, Hh, V, S = (nb.soa(nb.RaySoA, rays), nb.soa(nb.HitSoA, hits),
                   nb.soa(nb.PathVertices, verts), nb.soa(nb.ShadowSoA, shadow))
    vsoa = nb.vertex_soa(verts["pos"], verts["wi"], verts["normal"], verts["roughness"],
                         verts["albedo"], verts["thp"], verts["depth"])
    ev = {}

    # ---- a training frame (renderInternal<true> + trainStep): path records, radiance, the
    # per-pixel error, the batch and one training step on it ----
    if train:
        node_cap = wl["node_rate"] * P
        nbytes = nb.path_nodes_bytes(node_cap, cap)
        block = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        pn = nb.NRRSPathNodesBuffer(block.data_ptr(), nbytes, node_cap, cap, stream)
        contrib, scontrib = f(cap, 3), f(cap, 3)
        widths = {"pos": 3, "wi": 3, "normal": 3, "albedo": 3, "roughness": 1, "thp": 3,
                  "depth": 1, "ref_mean": 1, "target": 3, "rrs_target": 1, "pixel": 1,
                  "error": 1, "error_for_avg": 1, "number_samples": 1}
        batch = {k: (f(node_cap, w) if w > 1 else f(node_cap)) if k not in ("depth", "pixel")
                 else i(node_cap) for k, w in widths.items()}
        tb = nb.train_batch(**batch)
        counts, size_d = i(P), i(1)
        pe = nb.default_pixel_error_params(W, H)
        wl_d, cur_d, acc_d = f(P, 3), f(P, 3), i(P)
        err_d, spp_d = f(2 * P), f(P)
        esum_d = torch.zeros(32, dtype=torch.uint8, device=dev)
        tprm = records_params(frame_width=W, error_image_scale=1,
                              error_per_pixel=err_d.data_ptr(), samples_per_patch=spp_d.data_ptr())
        tsoa = nb.vertex_soa(batch["pos"], batch["wi"], batch["normal"], batch["roughness"],
                             batch["albedo"], batch["thp"], batch["depth"], batch["ref_mean"])
        loss = torch.zeros(2, dtype=torch.float64, device=dev)
        trained = [0, 0]   # samples in the batches, samples trained

    bounces_run = [0]
    rays_run = [0, 0]   # closest-hit and shadow rays of the timing frame

    def frame(sample, timing=False):
        vertices = 0
        n_prev = 0
        n_cur = P          # rays of this bounce on the host (training frames read them back)
        film.zero_()
        nb.camera_rays(cam, sample, 1234, R, stream)
        n_rays.fill_(P)
        if train:
            pn.reset(stream)
            spp_d.zero_()
            nb.count_patch_samples(pe, rays["pixel"], P, spp_d, stream)
        for depth in range(wl["bounces"]):
            if timing:
                ev.setdefault(("trace", depth), (torch.cuda.Event(enable_timing=True),
                                                 torch.cuda.Event(enable_timing=True)))
                ev[("trace", depth)][0].record(cur)
            if depth == 0:    # camera rays come in pixel order, already coherent
                nb.trace(scene, R, n_rays, cap, Hh, stream)
            else:
                nb.trace_sorted(scene, R, n_rays, cap, Hh, tscratch, stream)
            if timing:
                ev[("trace", depth)][1].record(cur)
            nb.shade(scene, R, Hh, n_rays, cap, depth, film, contrib if train else None, V,
                     n_vert, scratch, stream)
            if train:   # handleEmissiveHit / handleMiss: radiance to the node the ray left
                pn.recordRadiance(rays["node"], contrib, n_cur, stream)
            nv = int(n_vert.item())          # the reference reads the queue size back too
            if nv == 0:
                break
            vertices += nv
            bounces_run[0] += 1
            if timing:
                ev.setdefault(("nrrs", depth), (torch.cuda.Event(enable_timing=True),
                                                torch.cuda.Event(enable_timing=True)))
                ev[("nrrs", depth)][0].record(cur)
            net.generateRRSNumber(vsoa, rnd, nv, P, 0, dp, stats, rrs, rrs_norm, split, queue,
                                  cap, qsize, stream)
            if timing:
                ev[("nrrs", depth)][1].record(cur)
            if train:   # recordNode for the surviving vertices, in place on their node indices
                pn.recordNode(vsoa, verts["node"], verts["pixel"], rrs_norm, split, nv,
                              verts["node"], stream)
            nb.scatter(scene, V, rrs_norm, queue, qsize, cap, depth, 1234 + sample, R, S, stream)
            if timing:
                ev.setdefault(("shadow", depth), (torch.cuda.Event(enable_timing=True),
                                                  torch.cuda.Event(enable_timing=True)))
                ev[("shadow", depth)][0].record(cur)
            nb.trace_shadow(scene, S, qsize, cap, film, scontrib if train else None, stream)
            if timing:
                ev[("shadow", depth)][1].record(cur)
                rays_run[0] += P if depth == 0 else n_prev
                n_prev = int(qsize.item())
                rays_run[1] += n_prev
            if train:
                n_cur = int(qsize.item())
                nb.count_patch_samples(pe, rays["pixel"], n_cur, spp_d, stream)
                pn.recordRadiance(shadow["node"], scontrib, n_cur, stream)
            n_rays.copy_(qsize)
        nb.film_resolve(film, P, 1.0, img, stream)
        if train:
            if timing:
                ev.setdefault("train_data", (torch.cuda.Event(enable_timing=True),
                                             torch.cuda.Event(enable_timing=True)))
                ev["train_data"][0].record(cur)
            # trainStep STEP#1-#2 (this frame's image stands for both the pixel radiance and
            # the rendered film), then the batch and its per-pixel counts
            nb.accumulate_weighted_l(pe, img, 1, False, wl_d, cur_d, acc_d, stream)
            nb.update_weighted_l(pe, cur_d, acc_d, wl_d, stream)
            nb.calculate_error(pe, img, 3, wl_d, spp_d, err_d, esum_d, stream)
            counts.zero_()
            pn.generate_training_data(tprm, tb, node_cap, size_d, image=img, image_channels=3,
                                      n_pixels=P, pixel_samples=counts, stream=stream)
            m = min(int(size_d.item()), wl["train_batch"])   # the reference reads it back too
            if timing:
                ev["train_data"][1].record(cur)
                ev.setdefault("train", (torch.cuda.Event(enable_timing=True),
                                        torch.cuda.Event(enable_timing=True)))
                ev["train"][0].record(cur)
            m -= m % 256
            if m:
                net.train(tsoa, batch["target"], m, loss, stream)
            if timing:
                ev["train"][1].record(cur)
            trained[0] += int(size_d.item())
            trained[1] += m
        return vertices

    for w in range(args.warmup):
        frame(w)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    total_v = 0
    bounces_run[0] = 0
    if train:
        trained[0] = trained[1] = 0
    launches0 = net.launch_count()
    with ClockSampler(local_rank) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(cur)
        for k in range(args.steps):
            total_v += frame(100 + k)
        e1.record(cur)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    verts_per_frame = total_v / args.steps
    # camera + resolve per frame; ray sort (2, not for the camera rays), trace, shade (2),
    # scatter, shadow per bounce run, and the last trace + shade of a frame whose queue ran out;
    # plus the NRRS step's own launches
    launches = (args.steps * 2 + bounces_run[0] * 7 - args.steps * 2 +
                (net.launch_count() - launches0))
    if train:
        # per bounce: radiance of the shaded rays, record count + writes, patch counts, shadow
        # radiance; per frame: camera patch counts, pixel error (3), radiance pass + batch
        launches += bounces_run[0] * 5 + args.steps * 6
        batch_per_frame = trained[0] / args.steps
        trained_per_frame = trained[1] / args.steps
    if dist:
        tt = torch.tensor([ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    net.profile(True)
    frame(999, timing=True)
    torch.cuda.synchronize()
    kern = net.profile_read()
    net.profile(False)
    t_trace = sum(a.elapsed_time(b) for k, (a, b) in ev.items()
                  if isinstance(k, tuple) and k[0] == "trace")
    t_nrrs = sum(a.elapsed_time(b) for k, (a, b) in ev.items()
                 if isinstance(k, tuple) and k[0] == "nrrs")
    t_shadow = sum(a.elapsed_time(b) for k, (a, b) in ev.items()
                   if isinstance(k, tuple) and k[0] == "shadow")
    line = {
        "metric": "path vertices/s (path-traced frame around the NRRS step)",
        "value": verts_per_frame * world / (ms * 1e-3), "unit": "vertices/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f16", "data": "synthetic",
        "config": {"workload": f"render_{W}x{H}_{wl['bounces']}bounce_{len(t)}tri",
                   "triangles": int(len(t)), "bvh_nodes": n_nodes, "bvh_depth": bvh_depth,
                   "lights": n_lights, "vertices_per_frame": verts_per_frame,
                   "parallelism": f"replicas{world}",
                   "l2": "queues of 2-6M entries per bounce (hundreds of MB) are larger than L2; "
                         "the scene (4 MB of nodes and triangles) is L2-resident"},
        "clocks": clk.summary(),
        "gpu_launches": launches,
        "calls_ms_per_frame": {"trace": t_trace, "nrrs_step": t_nrrs, "shadow": t_shadow},
        "autotune": tune.get("best") or tune.get("cached"),
        "rays_per_frame": {"closest_hit": rays_run[0], "shadow": rays_run[1]},
        "rays_per_s_trace": rays_run[0] / (t_trace * 1e-3) if t_trace else None,
        "rays_per_s_shadow": rays_run[1] / (t_shadow * 1e-3) if t_shadow else None,
        "note": "a step is one frame; per bounce the vertex count is read back (as the "
                "reference reads its queue size) before nrrs_step",
    }
    if train:
        line["metric"] = ("path vertices/s (training frame: path-traced frame around the NRRS "
                          "step, path records, pixel error, training batch, one training step)")
        line["config"]["workload"] = "train_" + line["config"]["workload"]
        line["config"]["train_batch"] = wl["train_batch"]
        line["calls_ms_per_frame"]["train_data"] = ev["train_data"][0].elapsed_time(ev["train_data"][1])
        line["calls_ms_per_frame"]["train_step"] = ev["train"][0].elapsed_time(ev["train"][1])
        line["training"] = {"batch_samples_per_frame": batch_per_frame,
                            "samples_trained_per_frame": trained_per_frame,
                            "loss": [float(x) for x in loss.tolist()]}
        line["note"] += ("; the batch size is read back before the training step, which trains "
                         "on the first train_batch samples of the batch")
    line["kernels_ms_timing_frame"] = {k: round(ms, 4) for k, (n, ms) in kern.items()}
    if rank == 0:
        print(json.dumps(line), flush=True)
    scene.close()
    net.close()
    if dist:
        dist.destroy_process_group()
    return 0



def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", choices=tuple(WORKLOADS), default="frame4k")
    ap.add_argument("--only", action="store_true",
                    help="the workload's own arm only (no FP32 arm, no secondary configurations)")
    ap.add_argument("--no-errors", dest="errors", action="store_false",
                    help="skip the error measurement against the FP64 oracle")
    ap.add_argument("--precision", choices=("fp16", "bf16", "fp32"), default=None)
    ap.add_argument("--no-train", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--launch-shape", default=None,
                    help="CTAS_PER_SM,WARPGROUPS[,SPLIT] of the inference kernels instead of "
                         "autotuning")
    ap.add_argument("--no-cell-image", dest="cell_image", action="store_false",
                    help="gather the dense hash-grid levels from the table rows instead of the "
                         "cell image (bit-identical; for comparisons)")
    ap.add_argument("--bounces", type=int, default=None, help="smaller cases for profiling")
    ap.add_argument("--vertices", type=int, default=None, help="smaller cases for profiling")
    args = ap.parse_args()
    wl = WORKLOADS[args.workload]
    args.warmup = max(3, args.warmup)
    if args.steps is None:
        args.steps = wl["steps"]
    if args.precision is None:
        args.precision = wl["precision"]
    if args.bounces:
        wl["bounces"] = args.bounces
    if args.vertices:
        wl["n_vert"] = args.vertices
    rank, world = env_int("RANK", 0), env_int("WORLD_SIZE", 1)
    local_rank = env_int("LOCAL_RANK", 0)
    if args.workload in ("render1080p", "render_train1080p"):
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference traces with "
                              "OptiX inside its KiRaRay integrator, which cannot be built here"}))
            return 0
        load_product()
        return run_render(args, rank, world, local_rank)
    if args.workload == "records1080p":
        load_product()   # the synthetic path records come from the library's generator
        if args.impl == "reference":
            return run_records_reference(args, rank, world)
        return run_records(args, rank, world, local_rank)
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
