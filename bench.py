"""Benchmark of the NRRS per-vertex step on B200 (one JSON line on rank 0).

Workload (default "frame1080p"): one frame at 1920x1080 with 6 bounces. Each bounce runs
inference, the RRS decision and emission on 2,073,600 synthetic path vertices. The frame then
runs one training step on 262,144 samples. Mixed precision: FP16 table, FP16 tcgen05 MLPs with
FP32 accumulation, exact 64-bit normalisation sums. Inputs are seeded synthetic records with
the workload's distributions; each bounce has its own 158 MB vertex buffer, so inputs are
larger than L2.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--precision fp16|bf16|fp32] [--no-train]

value    = vertices/s of the whole job (device-timed frames, max over ranks)
e2e      = the same metric through the C-ABI with host (pinned) inputs: the H2D copy of each
           bounce's vertices and training batch and the D2H read of queue sizes and losses are
           inside the timed region
roofline = dominant kernel (inference) achieved algorithmic GB/s vs the measured HBM peak
--impl reference times the reference's CPU path (the oracle port of it, all host threads)
on a bounded sample of the same workload.
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

import numpy as np  # noqa: E402

import nrrs_b200 as nb  # noqa: E402

N_VERT = 2_073_600
BOUNCES = 6
TRAIN_BATCH = 262_144
SOA_BYTES = 72            # pos, wi, normal, roughness, albedo, thp, depth, ref_mean
RND_BYTES = 4
TARGET_BYTES = 12
METRIC = "RRS vertices/s and train samples/s, mixed-prec vs FP32 plain at stated error"


def env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def measured_peaks():
    f = REPO / "MEASURED_PEAKS.json"
    if f.exists():
        j = json.loads(f.read_text())
        return j.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def traffic_per_vertex(kernel: str):
    """DRAM bytes per vertex of the kernel from the committed ncu summary, if any."""
    f = REPO / "profiles" / "traffic.json"
    if f.exists():
        j = json.loads(f.read_text())
        if kernel in j:
            return j[kernel]
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.p = None

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
        self.lines = []
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


def make_config(precision: str, max_queue: int, max_train: int):
    prec = {"fp16": nb.PREC_FP16, "bf16": nb.PREC_BF16, "fp32": nb.PREC_FP32}[precision]
    return nb.default_config(precision=prec, max_queue=max_queue, max_train=max_train)


def cpu_sample(precision_cfg, n_sample: int, seconds: float, train_n: int, do_train: bool):
    """Oracle FP32 (OpenMP, all host threads) on a bounded sample of the frame workload;
    returns frame-equivalent vertices/s and the sample description."""
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle as O
    O.set_threads(os.cpu_count() or 1)
    cores = O.threads()
    net_cfg = precision_cfg
    v = nb.synth(7, n_sample)
    params = None
    # parameters: the library's initialisation is reproduced from the seed by the oracle's
    # caller; for throughput only the shapes matter, so use small random weights
    npar = O.param_count(net_cfg)[0]
    params = (np.random.default_rng(0).uniform(-1, 1, npar) * 0.1).astype(np.float32)
    dp = nb.default_decide()
    t_inf, reps = 0.0, 0
    t0 = time.perf_counter()
    while True:
        a = time.perf_counter()
        r = O.infer(net_cfg, params, v, dp, "f32", want=("stats", "rrs"))
        O.decide_emit(r["rrs"].astype(np.float32), v["rnd"], n_sample, 0, dp)
        t_inf += time.perf_counter() - a
        reps += 1
        if time.perf_counter() - t0 > seconds * (0.6 if do_train else 1.0):
            break
    per_vertex = t_inf / (reps * n_sample)
    t_train = 0.0
    if do_train:
        tv = nb.synth(8, train_n)
        treps = 0
        t1 = time.perf_counter()
        while True:
            a = time.perf_counter()
            g, loss = O.train_grads(net_cfg, params, tv, tv["target"], "f32")
            t_train += time.perf_counter() - a
            treps += 1
            if time.perf_counter() - t1 > seconds * 0.4:
                break
        per_sample = t_train / (treps * train_n)
    else:
        per_sample = 0.0
    frame_s = BOUNCES * N_VERT * per_vertex + (TRAIN_BATCH * per_sample if do_train else 0.0)
    sample = (f"{reps} x infer+decide on {n_sample} vertices"
              + (f", {treps} x train grads on {train_n} samples" if do_train else "")
              + "; frame time extrapolated from per-vertex and per-sample costs")
    return BOUNCES * N_VERT / frame_s, cores, sample, frame_s


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    cfg = make_config("fp32", 1 << 21, 1 << 16)
    value, cores, sample, frame_s = cpu_sample(cfg, 131072, 10.0 * max(1, args.steps) / 10, 8192,
                                               not args.no_train)
    line = {
        "metric": METRIC, "value": value, "unit": "vertices/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": frame_s * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "impl": "reference",
        "config": {"workload": workload_name(args), "bounces": BOUNCES,
                   "vertices_per_bounce": N_VERT, "train_batch": TRAIN_BATCH if not args.no_train else 0},
        "cpu_baseline": {"value": value, "unit": "vertices/s", "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "vertices/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "reference CPU path = FP32 C restatement (oracle/) with OpenMP; the reference "
                "itself needs OptiX/KiRaRay/tiny-cuda-nn and cannot be built",
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_name(args):
    return (f"frame1080p_{BOUNCES}bounce_infer_decide_emit"
            + ("" if args.no_train else "_train262144") + f"_{args.precision}")


def run_ours(args, rank, world, local_rank):
    import torch
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream().cuda_stream
    do_train = not args.no_train
    net = nb.NRRSNetwork(make_config(args.precision, N_VERT, TRAIN_BATCH))
    dp = nb.default_decide()
    cap = 9 * N_VERT

    # ---- synthetic inputs: one buffer set per bounce (pinned host + device) ----
    fields = ("pos", "wi", "normal", "roughness", "albedo", "thp", "depth", "ref_mean", "rnd")
    host_b, dev_b = [], []
    for d in range(BOUNCES):
        v = nb.synth(1000 + 97 * rank + d, N_VERT)
        v["depth"] = np.full(N_VERT, d, np.uint32)
        hb = {k: torch.from_numpy(v[k].view(np.int32) if v[k].dtype == np.uint32 else v[k]).pin_memory()
              for k in fields}
        host_b.append(hb)
        dev_b.append({k: t.to(dev) for k, t in hb.items()})
    tv = nb.synth(5000 + rank, TRAIN_BATCH)
    th = {k: torch.from_numpy(tv[k].view(np.int32) if tv[k].dtype == np.uint32 else tv[k]).pin_memory()
          for k in fields + ("target",)}
    td = {k: t.to(dev) for k, t in th.items()}
    outs = [dict(stats=torch.empty(3 * N_VERT, device=dev), rrs=torch.empty(N_VERT, device=dev),
                 norm=torch.empty(N_VERT, device=dev),
                 split=torch.empty(N_VERT, dtype=torch.uint8, device=dev),
                 q=torch.empty(cap, dtype=torch.int32, device=dev),
                 sz=torch.zeros(1, dtype=torch.int32, device=dev)) for _ in range(BOUNCES)]
    loss = torch.zeros(2, dtype=torch.float64, device=dev)

    def soa_of(b):
        return nb.vertex_soa(b["pos"], b["wi"], b["normal"], b["roughness"], b["albedo"],
                             b["thp"], b["depth"], b["ref_mean"])

    soas = [soa_of(b) for b in dev_b]
    tsoa = soa_of(td)

    sharded = None
    if world > 1:
        # each rank holds one 1080p-sized shard of an N-times larger queue: one integer
        # all-reduce of the exact sum per bounce, data-parallel gradients per train step
        from nrrs_parallel import ShardedNRRS
        sharded = ShardedNRRS(net)
        acc = torch.zeros(1, dtype=torch.int64, device=dev)
        grads_buf = torch.zeros(net.param_count(), dtype=torch.float32, device=dev)

    def frame():
        for d in range(BOUNCES):
            o = outs[d]
            if sharded is None:
                net.generateRRSNumber(soas[d], dev_b[d]["rnd"], N_VERT, N_VERT, 0, dp, o["stats"],
                                      o["rrs"], o["norm"], o["split"], o["q"], cap, o["sz"], stream)
            else:
                sharded.step(soas[d], dev_b[d]["rnd"], N_VERT, N_VERT * world, 0, dp, o["stats"],
                             o["rrs"], o["norm"], o["split"], o["q"], cap, o["sz"], acc, stream)
        if do_train:
            if sharded is None:
                net.train(tsoa, td["target"], TRAIN_BATCH, loss, stream)
            else:
                sharded.train_step(tsoa, td["target"], TRAIN_BATCH, grads_buf, loss, stream)

    # ---- device-timed region ----
    for _ in range(args.warmup):
        frame()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = net.launch_count()
    net.profile(True)
    net.profile_read()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        e0.record()
        for _ in range(args.steps):
            frame()
        e1.record()
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = net.launch_count() - launches0
    prof = net.profile_read()
    net.profile(False)
    if dist:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_step = ms / args.steps
    verts = BOUNCES * N_VERT * world
    value = verts / (ms_step * 1e-3)
    rc, flags = net.device_status(stream)

    # ---- end to end through the C-ABI with host buffers ----
    h2d = BOUNCES * N_VERT * (SOA_BYTES + RND_BYTES) + (
        TRAIN_BATCH * (SOA_BYTES + RND_BYTES + TARGET_BYTES) if do_train else 0)
    d2h = BOUNCES * 4 + (16 if do_train else 0)
    sizes_h = torch.zeros(BOUNCES, dtype=torch.int32).pin_memory()
    loss_h = torch.zeros(2, dtype=torch.float64).pin_memory()

    def frame_e2e():
        for d in range(BOUNCES):
            for k in fields:
                dev_b[d][k].copy_(host_b[d][k], non_blocking=True)
        if do_train:
            for k in fields + ("target",):
                td[k].copy_(th[k], non_blocking=True)
        frame()
        for d in range(BOUNCES):
            sizes_h[d:d + 1].copy_(outs[d]["sz"], non_blocking=True)
        if do_train:
            loss_h.copy_(loss, non_blocking=True)

    for _ in range(min(2, args.warmup)):
        frame_e2e()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e2 = max(2, args.steps // 2)
    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a0.record()
    for _ in range(e2):
        frame_e2e()
    a1.record()
    torch.cuda.synchronize()
    e2e_ms = a0.elapsed_time(a1) / e2
    if dist:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())

    # ---- roofline of the dominant kernel ----
    kind = "infer_fp32" if args.precision == "fp32" else "infer_tc"
    feat_bytes = 4 if args.precision == "fp32" else 2
    b_vertex = SOA_BYTES + 16 * 8 * 2 * feat_bytes + 12 + 4
    n_inf, ms_inf = prof.get(kind, (0, 0.0))
    peak, peak_kind = measured_peaks()
    roof = None
    if n_inf:
        launch_ms = ms_inf / n_inf
        achieved = b_vertex * N_VERT / (launch_ms * 1e-3) / 1e9
        tpv = traffic_per_vertex(kind)
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": (tpv * N_VERT) if tpv else None, "kernel": kind,
                "algorithmic_bytes_per_vertex": b_vertex, "launch_ms": launch_ms,
                "note": "algorithmic bytes count 4 B (FP16) per hash-corner gather; the table is "
                        "L2-resident, so the limiter is L2 sector throughput, see profiles/"}
    kernels = {k: {"launches": n, "ms_total": t, "ms_per_launch": t / n} for k, (n, t) in prof.items()}

    line = {
        "metric": METRIC, "value": value, "unit": "vertices/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {"fp16": "f16", "bf16": "bf16", "fp32": "f32"}[args.precision],
        "data": "synthetic",
        "config": {"workload": workload_name(args), "bounces": BOUNCES,
                   "vertices_per_bounce": N_VERT, "train_batch": TRAIN_BATCH if do_train else 0,
                   "encoding": "hashgrid L16 F2 T2^19 Nmin16 b1.5 + SH deg4",
                   "mlp": "StatNet 64->64x2->3, RRSNet 16->64x2->1",
                   "l2": "inputs larger than L2 (one 158 MB vertex buffer per bounce)",
                   "parallelism": f"dp{world}"},
        "clocks": clk.summary(),
        "e2e": {"value": verts / (e2e_ms * 1e-3), "unit": "vertices/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "roofline": roof,
        "kernels": kernels,
        "device_status": [rc, flags],
        "infer_grid": net.last_infer_grid(),
    }
    if do_train and "train_statnet" in prof:
        t_train = sum(t for k, (n, t) in prof.items() if k.startswith("train") or k == "adam"
                      or k in ("pack_weights", "table_half"))
        line["train_samples_per_s"] = TRAIN_BATCH * args.steps / (t_train * 1e-3)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        value_c, cores, sample, _ = cpu_sample(make_config("fp32", 1 << 21, 1 << 16), 131072,
                                               12.0, 8192, do_train)
        line["cpu_baseline"] = {"value": value_c, "unit": "vertices/s", "cores": cores,
                                "kind": "port", "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    net.close()
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--precision", choices=("fp16", "bf16", "fp32"), default="fp16")
    ap.add_argument("--no-train", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--bounces", type=int, default=BOUNCES, help="smaller cases for profiling")
    ap.add_argument("--vertices", type=int, default=N_VERT, help="smaller cases for profiling")
    args = ap.parse_args()
    globals()["BOUNCES"] = args.bounces
    globals()["N_VERT"] = args.vertices
    args.warmup = max(3, args.warmup)
    rank, world = env_int("RANK", 0), env_int("WORLD_SIZE", 1)
    local_rank = env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
