"""ctypes wrapper of the CPU oracle (oracle/_build/libnrrs_oracle.so). TEST INFRASTRUCTURE ONLY:
used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker and the
timed CPU baseline, never by the product library.

PARITY UNPINNED for the encodings, MLPs, losses and optimizer (the reference takes them from its
absent tiny-cuda-nn submodule); the decision, normalisation, glue and activation restatements
are pinned by tests/golden fixtures and, for RRSWeightWindow, by the reference's own header
compiled into oracle/_ref (see oracle/Makefile).
"""
from __future__ import annotations

import ctypes as C
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libnrrs_oracle.so"
REF_LIB = HERE / "_ref" / "libnrrs_ref.so"
REPO = HERE.parent
sys.path.insert(0, str(REPO / "nrrs-code_b200"))
import nrrs_b200 as nb  # noqa: E402  (struct definitions only)

_lib = None
_ref = None


def build(ref: bool = False):
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", str(HERE), "ref"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        vp = C.c_void_p
        L.oracle_level_table.restype = C.c_uint64
        L.oracle_level_table.argtypes = [C.POINTER(nb.Config), vp]
        L.oracle_param_count.restype = C.c_uint64
        L.oracle_param_count.argtypes = [C.POINTER(nb.Config), vp, vp, vp]
        L.oracle_sh16_f64.argtypes = [vp, vp]
        for f in ("oracle_activation_sigma_f32", "oracle_box_cox_f32", "oracle_warp_roughness_f32"):
            getattr(L, f).restype = C.c_float
            getattr(L, f).argtypes = [C.c_float]
        L.oracle_stat_to_l_f32.restype = C.c_float
        L.oracle_stat_to_l_f32.argtypes = [C.c_float, C.c_float]
        L.oracle_weight_window_f32.restype = C.c_float
        L.oracle_weight_window_f32.argtypes = [C.c_float, C.c_float]
        L.oracle_normalize_pos_f32.argtypes = [C.POINTER(nb.Config), vp, vp]
        for f in ("oracle_infer_f64", "oracle_infer_f32"):
            getattr(L, f).argtypes = [C.POINTER(nb.Config), vp, C.c_uint64, C.POINTER(nb.VertexSoA),
                                      C.POINTER(nb.DecideParams), vp, vp, vp, vp, vp]
        L.oracle_sum_shift.restype = C.c_int
        L.oracle_sum_shift.argtypes = [C.c_uint64, C.c_float]
        L.oracle_sum_fixed.restype = C.c_int64
        L.oracle_sum_fixed.argtypes = [vp, C.c_uint64, C.c_int, C.c_int, C.POINTER(C.c_double)]
        L.oracle_decide_emit.restype = C.c_uint64
        L.oracle_decide_emit.argtypes = [vp, vp, vp, C.c_uint64, C.c_uint32, C.c_uint32,
                                         C.POINTER(nb.DecideParams), C.c_uint64, vp, vp, vp,
                                         C.c_uint64, C.POINTER(C.c_uint32)]
        L.oracle_decide_emit_acc.restype = C.c_uint64
        L.oracle_decide_emit_acc.argtypes = [vp, vp, vp, C.c_uint64, C.c_uint32, C.c_uint32,
                                             C.POINTER(nb.DecideParams), C.c_int64, C.c_int, vp,
                                             vp, vp, C.c_uint64, C.POINTER(C.c_uint32)]
        for f in ("oracle_train_grads_f64", "oracle_train_grads_f32"):
            getattr(L, f).argtypes = [C.POINTER(nb.Config), vp, C.c_uint64, C.POINTER(nb.VertexSoA),
                                      vp, vp, vp]
        L.oracle_train_loss_f64.argtypes = [C.POINTER(nb.Config), vp, C.c_uint64,
                                            C.POINTER(nb.VertexSoA), vp, vp]
        for f in ("oracle_train_grads_w_f64", "oracle_train_grads_w_f32"):
            getattr(L, f).argtypes = [C.POINTER(nb.Config), vp, C.c_uint64, C.POINTER(nb.VertexSoA),
                                      vp, C.POINTER(LossW), vp, vp]
        L.oracle_train_loss_w_f64.argtypes = [C.POINTER(nb.Config), vp, C.c_uint64,
                                              C.POINTER(nb.VertexSoA), vp, C.POINTER(LossW), vp]
        L.oracle_adam_f32.argtypes = [C.POINTER(nb.Config), vp, vp, vp, vp, C.c_uint64,
                                      C.c_uint64, C.c_uint64]
        L.oracle_fixed_limbs.argtypes = [C.c_float, vp]
        for f in ("oracle_fixed_to_float", "oracle_fixed_to_float_gcc",
                  "oracle_fixed_to_float_fast"):
            getattr(L, f).restype = C.c_float
            getattr(L, f).argtypes = [C.c_int64, C.c_int64, C.c_int64]
        L.oracle_nodes_reset.argtypes = [C.POINTER(nb.PathNodes)]
        L.oracle_record_nodes.argtypes = [C.POINTER(nb.PathNodes), C.POINTER(nb.VertexSoA), vp,
                                          vp, vp, vp, C.c_uint64, vp]
        L.oracle_record_radiance.argtypes = [C.POINTER(nb.PathNodes), vp, vp, C.c_uint64]
        L.oracle_generate_training_data.restype = C.c_uint64
        L.oracle_generate_training_data.argtypes = [C.POINTER(nb.PathNodes),
                                                    C.POINTER(nb.TrainDataParams), vp, C.c_int,
                                                    C.c_uint32, vp, C.POINTER(nb.TrainBatch),
                                                    C.c_uint64]
        L.oracle_sample_weights.argtypes = [vp, vp, C.c_uint32, C.c_uint64, vp]
        pe = C.POINTER(nb.PixelErrorParams)
        L.oracle_count_patch_samples.argtypes = [pe, vp, C.c_uint64, vp]
        L.oracle_accumulate_weighted_l.argtypes = [pe, vp, C.c_uint32, C.c_int, vp, vp, vp]
        L.oracle_update_weighted_l.argtypes = [pe, vp, vp, vp]
        L.oracle_calculate_error.restype = C.c_float
        L.oracle_calculate_error.argtypes = [pe, vp, C.c_int, vp, vp, vp]
        L.oracle_ubs_error.restype = C.c_float
        L.oracle_ubs_error.argtypes = [pe, vp, C.c_uint32, vp, C.c_int, vp]
        L.oracle_set_threads.argtypes = [C.c_int]
        L.oracle_get_threads.restype = C.c_int
        L.nrrs_synth_vertices.restype = None
        L.nrrs_synth_vertices.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64] + [vp] * 10
        _lib = L
    return _lib


def ref_lib():
    """Reference code compiled from the reference checkout (oracle/ref_harness.cpp): its
    RRSWeightWindow, activationSigma, warp_roughness, box_cox_transform and the "Gen RRS Number"
    and "Gen Tids" lambdas of the integrator; None where it was not built."""
    global _ref
    if _ref is None and REF_LIB.exists():
        L = C.CDLL(str(REF_LIB))
        vp = C.c_void_p
        L.ref_rrs_weight_window.restype = C.c_float
        L.ref_rrs_weight_window.argtypes = [C.c_float, C.c_float]
        for f in ("ref_activation_sigma", "ref_warp_roughness", "ref_box_cox"):
            getattr(L, f).restype = C.c_float
            getattr(L, f).argtypes = [C.c_float]
        L.ref_gen_rrs_number.restype = None
        L.ref_gen_rrs_number.argtypes = [C.c_uint32, C.c_int, vp, vp, vp, C.c_int, C.c_float,
                                         C.c_float, C.c_int, vp, vp]
        L.ref_gen_tids.restype = C.c_uint64
        L.ref_gen_tids.argtypes = [C.c_uint32, vp, vp, C.c_uint32, C.c_uint32, C.c_float, C.c_int,
                                   C.c_float, C.c_int, vp, vp, C.c_uint64]
        _ref = L
    return _ref


def ref_gen_rrs_number(net_out, thp, ref_rgb, dp):
    """The reference's factor lambda (integrator.cpp:1186-1297) on [n][16] network outputs."""
    L = ref_lib()
    n = len(thp)
    net_out = np.ascontiguousarray(net_out, np.float32)
    thp = np.ascontiguousarray(thp, np.float32)
    ref_rgb = np.ascontiguousarray(ref_rgb, np.float32)
    rrs = np.empty(n, np.float32)
    ceil = np.zeros(n, np.float32)
    L.ref_gen_rrs_number(n, 1 if dp.factor_source == nb.FACTOR_RRSNET else 0, net_out.ctypes.data,
                         thp.ctypes.data, ref_rgb.ctypes.data, dp.use_weight_window, dp.clamp_min,
                         dp.clamp_max, dp.use_ceil, rrs.ctypes.data, ceil.ctypes.data)
    return rrs, ceil


def ref_gen_tids(rrs, rnd, budget, n_specular, rcp_sum, dp, capacity=None):
    """The reference's decision and emission lambda (integrator.cpp:1370-1457)."""
    L = ref_lib()
    n = len(rrs)
    rrs = np.ascontiguousarray(rrs, np.float32)
    rnd = np.ascontiguousarray(rnd, np.float32)
    cap = 9 * n if capacity is None else capacity
    norm = np.empty(n, np.float32)
    q = np.zeros(max(cap, 1), np.uint32)
    tot = L.ref_gen_tids(n, rrs.ctypes.data, rnd.ctypes.data, budget, n_specular,
                         np.float32(rcp_sum), dp.use_ceil, dp.normalize_rate, dp.scale_up,
                         norm.ctypes.data, q.ctypes.data, cap)
    return {"total": int(tot), "queue": q[:min(tot, cap)], "rrs_norm": norm}


def synth(seed: int, n: int, first: int = 0) -> dict:
    """Seeded synthetic vertices (host numpy arrays) from the oracle library's copy of the
    generator (the same source as the product library's nrrs_synth_vertices), so that CPU-only
    callers draw identical inputs without loading the product library."""
    out = {
        "pos": np.empty((n, 3), np.float32), "wi": np.empty((n, 3), np.float32),
        "normal": np.empty((n, 3), np.float32), "roughness": np.empty(n, np.float32),
        "albedo": np.empty((n, 3), np.float32), "thp": np.empty((n, 3), np.float32),
        "depth": np.empty(n, np.uint32), "rnd": np.empty(n, np.float32),
        "ref_mean": np.empty(n, np.float32), "target": np.empty((n, 3), np.float32),
    }
    lib().nrrs_synth_vertices(seed, first, n, *(out[k].ctypes.data for k in
                              ("pos", "wi", "normal", "roughness", "albedo", "thp", "depth",
                               "rnd", "ref_mean", "target")))
    return out


# The library's defaults (nrrs_config_default, nrrs_decide_params_default), restated so that
# the CPU baseline can build its configuration without loading the product library;
# tests/test_oracle.py checks that the two agree field by field.
_CONFIG_DEFAULTS = dict(
    n_levels=16, n_features_per_level=2, log2_hashmap_size=19, base_resolution=16,
    per_level_scale=1.5, sh_degree=4, statnet_width=64, statnet_hidden=2, rrsnet_width=64,
    rrsnet_hidden=2, precision=0, seed=0, table_init_scale=1e-4, lr=1e-2, beta1=0.9, beta2=0.99,
    eps=1e-15, l2_reg=0.0, stat_eps=0.01, ref_eps=0.01, loss_clamp_max=10.0, cost_offset=1.0,
    normalize_pos=0, aabb_min=(0.0, 0.0, 0.0), aabb_max=(1.0, 1.0, 1.0), max_queue=1 << 20,
    max_train=1 << 18, step=3, network=0, ema_decay=0.0, lr_rrsnet=0.0, sum_shards=0)
_DECIDE_DEFAULTS = dict(clamp_min=0.05, clamp_max=8.0, normalize_rate=0.85, use_ceil=1,
                        scale_up=0, use_weight_window=0, weight_window_size=5.0,
                        factor_source=nb.FACTOR_RRSNET)


def default_config(**kw) -> nb.Config:
    c = nb.Config()
    for k, v in {**_CONFIG_DEFAULTS, **kw}.items():
        if k in ("aabb_min", "aabb_max"):
            getattr(c, k)[:] = list(v)
        else:
            setattr(c, k, v)
    return c


def reference_config(**kw) -> nb.Config:
    """the reference's shipped network (nrrs_config_reference_network, restated)"""
    base = dict(network=1, n_levels=8, n_features_per_level=2, log2_hashmap_size=19,
                base_resolution=16, per_level_scale=2.0, statnet_width=32, statnet_hidden=3,
                rrsnet_width=32, rrsnet_hidden=3, lr=5e-3, beta1=0.9, beta2=0.99, eps=1e-15,
                l2_reg=3e-6, ema_decay=0.95, lr_rrsnet=5e-4)
    base.update(kw)
    return default_config(**base)


def default_decide(**kw) -> nb.DecideParams:
    p = nb.DecideParams()
    for k, v in {**_DECIDE_DEFAULTS, **kw}.items():
        setattr(p, k, v)
    return p


def _soa(v: dict) -> nb.VertexSoA:
    return nb.VertexSoA(*(v[k].ctypes.data if v.get(k) is not None else None
                          for k in ("pos", "wi", "normal", "roughness", "albedo", "thp", "depth",
                                    "ref_mean", "scatter_index")))


def level_table(cfg):
    out = np.zeros((cfg.n_levels, 4), np.uint32)
    tot = lib().oracle_level_table(C.byref(cfg), out.ctypes.data)
    return out, int(tot)


def param_count(cfg):
    t, s, r = C.c_uint64(), C.c_uint64(), C.c_uint64()
    n = lib().oracle_param_count(C.byref(cfg), C.byref(t), C.byref(s), C.byref(r))
    return int(n), int(t.value), int(s.value), int(r.value)


def infer(cfg, params, v: dict, dp, precision: str = "f64", want=("stats", "rrs")):
    n = v["pos"].shape[0]
    dt = np.float64 if precision == "f64" else np.float32
    outs = {"x0": (n, 64), "stats": (n, 6 if cfg.network else 3), "x1": (n, 16), "raw": (n,),
            "rrs": (n,)}
    res = {k: np.empty(s, dt) for k, s in outs.items() if k in want}
    f = lib().oracle_infer_f64 if precision == "f64" else lib().oracle_infer_f32
    params = np.ascontiguousarray(params, np.float32)
    soa = _soa(v)
    f(C.byref(cfg), params.ctypes.data, n, C.byref(soa), C.byref(dp),
      *(res[k].ctypes.data if k in res else None for k in ("x0", "stats", "x1", "raw", "rrs")))
    return res


def sum_fixed(rrs, use_ceil: bool, shift: int):
    rrs = np.ascontiguousarray(rrs, np.float32)
    s = C.c_double()
    acc = lib().oracle_sum_fixed(rrs.ctypes.data, rrs.size, int(use_ceil), shift, C.byref(s))
    return int(acc), s.value


def sum_shift(n: int, vmax: float) -> int:
    return int(lib().oracle_sum_shift(n, vmax))


def decide_emit(rrs, rnd, budget, n_specular, dp, capacity=None, scatter_index=None, shift_n=0):
    """shift_n: size that fixes the exact sum's shift (pass the library's max_queue)."""
    rrs = np.ascontiguousarray(rrs, np.float32)
    rnd = np.ascontiguousarray(rnd, np.float32)
    n = rrs.size
    cap = capacity if capacity is not None else int(n * (dp.clamp_max + 2)) + 8
    queue = np.zeros(max(cap, 1), np.uint32)
    nstid = int(scatter_index.max()) + 1 if scatter_index is not None and n else n
    rrs_norm = np.zeros(max(nstid, 1), np.float32)
    split = np.zeros(max(n, 1), np.uint8)
    flags = C.c_uint32()
    si = np.ascontiguousarray(scatter_index, np.uint32) if scatter_index is not None else None
    total = lib().oracle_decide_emit(rrs.ctypes.data, rnd.ctypes.data,
                                     si.ctypes.data if si is not None else None, n, budget,
                                     n_specular, C.byref(dp), shift_n, rrs_norm.ctypes.data,
                                     split.ctypes.data, queue.ctypes.data, cap, C.byref(flags))
    return {"queue": queue[:min(int(total), cap)], "total": int(total), "rrs_norm": rrs_norm[:nstid],
            "split": split[:n], "flags": int(flags.value)}


def decide_emit_acc(rrs, rnd, budget, n_specular, dp, acc: int, shift: int, capacity=None):
    """decision of one shard with the exact accumulator summed over all shards"""
    rrs = np.ascontiguousarray(rrs, np.float32)
    rnd = np.ascontiguousarray(rnd, np.float32)
    n = rrs.size
    cap = capacity if capacity is not None else int(n * (dp.clamp_max + 2)) + 8
    queue = np.zeros(max(cap, 1), np.uint32)
    rrs_norm = np.zeros(max(n, 1), np.float32)
    split = np.zeros(max(n, 1), np.uint8)
    flags = C.c_uint32()
    total = lib().oracle_decide_emit_acc(rrs.ctypes.data, rnd.ctypes.data, None, n, budget,
                                         n_specular, C.byref(dp), acc, shift, rrs_norm.ctypes.data,
                                         split.ctypes.data, queue.ctypes.data, cap, C.byref(flags))
    return {"queue": queue[:min(int(total), cap)], "total": int(total), "rrs_norm": rrs_norm[:n],
            "split": split[:n], "flags": int(flags.value)}


class LossW(C.Structure):
    """oracle_loss_w: the per-sample loss weights of nrrs_train_step_batch"""
    _fields_ = [("sample_weight", C.c_void_p), ("rrs_target", C.c_void_p), ("error", C.c_void_p),
                ("error_for_avg", C.c_void_p), ("number_samples", C.c_void_p),
                ("error_mean", C.c_double), ("gamma1", C.c_float), ("gamma2", C.c_float),
                ("gamma3", C.c_float), ("gamma4", C.c_float), ("clamp_on", C.c_int32),
                ("clamp_max", C.c_float)]


def loss_weights(arrays: dict, gammas=(1.0, 0.0, 0.0, 0.0), clamp_on=0, clamp_max=10.0,
                 error_mean=1.0):
    """LossW over host arrays (kept alive by the returned tuple's second element)."""
    keep = {k: np.ascontiguousarray(arrays[k], np.float32) for k in
            ("sample_weight", "rrs_target", "error", "error_for_avg", "number_samples")
            if arrays.get(k) is not None}
    w = LossW(*(keep[k].ctypes.data if k in keep else None for k in
                ("sample_weight", "rrs_target", "error", "error_for_avg", "number_samples")),
              float(error_mean), *map(float, gammas), int(clamp_on), float(clamp_max))
    return w, keep


def train_grads(cfg, params, v: dict, target, precision: str = "f64", out=None, weights=None):
    """(gradients, losses); out, when given, is a reused gradient array of the right size and
    precision (the oracle clears it itself); weights: a LossW (loss_weights()) for the weighted
    losses of nrrs_train_step_batch."""
    n = v["pos"].shape[0]
    npar = param_count(cfg)[0]
    dt = np.float64 if precision == "f64" else np.float32
    g = out if out is not None else np.empty(npar, dt)
    assert g.dtype == dt and g.size == npar
    loss = np.zeros(2, np.float64)
    params = np.ascontiguousarray(params, np.float32)
    target = np.ascontiguousarray(target, np.float32)
    soa = _soa(v)
    if weights is None:
        f = lib().oracle_train_grads_f64 if precision == "f64" else lib().oracle_train_grads_f32
        f(C.byref(cfg), params.ctypes.data, n, C.byref(soa), target.ctypes.data, g.ctypes.data,
          loss.ctypes.data)
    else:
        f = lib().oracle_train_grads_w_f64 if precision == "f64" else lib().oracle_train_grads_w_f32
        f(C.byref(cfg), params.ctypes.data, n, C.byref(soa), target.ctypes.data,
          C.byref(weights), g.ctypes.data, loss.ctypes.data)
    return g, loss


def train_loss(cfg, params64, v: dict, target, weights=None):
    n = v["pos"].shape[0]
    loss = np.zeros(2, np.float64)
    params64 = np.ascontiguousarray(params64, np.float64)
    target = np.ascontiguousarray(target, np.float32)
    soa = _soa(v)
    if weights is None:
        lib().oracle_train_loss_f64(C.byref(cfg), params64.ctypes.data, n, C.byref(soa),
                                    target.ctypes.data, loss.ctypes.data)
    else:
        lib().oracle_train_loss_w_f64(C.byref(cfg), params64.ctypes.data, n, C.byref(soa),
                                      target.ctypes.data, C.byref(weights), loss.ctypes.data)
    return loss


def adam(cfg, params, grads, m, v, t, first=0, count=None):
    count = params.size - first if count is None else count
    lib().oracle_adam_f32(C.byref(cfg), params.ctypes.data, grads.ctypes.data, m.ctypes.data,
                          v.ctypes.data, first, count, t)


def set_threads(n: int):
    lib().oracle_set_threads(n)


def threads() -> int:
    return int(lib().oracle_get_threads())


# ---- path-node records and the training batch (records.c) ----------------------------------

def fixed_limbs(x: float) -> tuple[int, int, int]:
    out = np.zeros(3, np.int64)
    lib().oracle_fixed_limbs(C.c_float(x), out.ctypes.data)
    return int(out[0]), int(out[1]), int(out[2])


def fixed_to_float(l0: int, l1: int, l2: int, gcc: bool = False, fast: bool = False) -> float:
    f = (lib().oracle_fixed_to_float_gcc if gcc else
         lib().oracle_fixed_to_float_fast if fast else lib().oracle_fixed_to_float)
    return float(f(l0, l1, l2))


NODE_ARRAYS = {"pos": (np.float32, 3), "wi": (np.float32, 3), "normal": (np.float32, 3),
               "albedo": (np.float32, 3), "roughness": (np.float32, 1),
               "thp": (np.float32, 3), "parent": (np.int32, 1), "pixel": (np.uint32, 1),
               "rrs": (np.float32, 1), "depth": (np.uint32, 1), "radiance": (np.int64, 9),
               "first_child": (np.uint32, 1), "children": (np.uint32, 1),
               "arrived": (np.uint32, 1),
               "node_flags": (np.uint32, 1)}


class HostNodes:
    """A node block in host memory, for the oracle: the library's nrrs_path_nodes struct
    pointing at numpy arrays."""

    def __init__(self, capacity: int):
        self.capacity = capacity
        self.a = {k: np.zeros((capacity, w) if w > 1 else capacity, dt)
                  for k, (dt, w) in NODE_ARRAYS.items()}
        self.header = np.zeros(16, np.uint32)
        self.nodes = nb.PathNodes(capacity, 0, *(self.a[k].ctypes.data for k in NODE_ARRAYS),
                                  self.header.ctypes.data, None)

    @property
    def size(self) -> int:
        return int(self.header[0])

    @property
    def dropped(self) -> int:
        return int(self.header[1])

    @property
    def status(self) -> int:
        return int(self.header[4])

    def reset(self):
        lib().oracle_nodes_reset(C.byref(self.nodes))

    def record_nodes(self, b: dict) -> np.ndarray:
        n = len(b["pixel"])
        opt = lambda k: b[k].ctypes.data if b.get(k) is not None else None  # noqa: E731
        v = nb.VertexSoA(b["pos"].ctypes.data, b["wi"].ctypes.data, opt("normal"),
                         opt("roughness"), opt("albedo"), b["thp"].ctypes.data,
                         b["depth"].ctypes.data if b.get("depth") is not None else None,
                         None, None)
        out = np.zeros(n, np.int32)
        rrs = b.get("rrs")
        rec = b.get("record")
        lib().oracle_record_nodes(C.byref(self.nodes), C.byref(v), b["parent"].ctypes.data,
                                  b["pixel"].ctypes.data,
                                  rrs.ctypes.data if rrs is not None else None,
                                  rec.ctypes.data if rec is not None else None, n,
                                  out.ctypes.data)
        return out

    def record_radiance(self, node, contrib):
        node = np.ascontiguousarray(node, np.int32)
        contrib = np.ascontiguousarray(contrib, np.float32)
        lib().oracle_record_radiance(C.byref(self.nodes), node.ctypes.data, contrib.ctypes.data,
                                     len(node))

    def generate(self, params, capacity: int, image=None, n_pixels: int = 0,
                 pixel_samples=None, out=None) -> tuple[dict, int]:
        """The training batch as numpy arrays (the first min(total, capacity) rows) and the
        total sample count. out (optional) is a dict of preallocated batch arrays to reuse."""
        cap = max(capacity, 1)
        out = out if out is not None else {"pos": np.zeros((cap, 3), np.float32), "wi": np.zeros((cap, 3), np.float32),
               "normal": np.zeros((cap, 3), np.float32), "albedo": np.zeros((cap, 3), np.float32),
               "roughness": np.zeros(cap, np.float32), "thp": np.zeros((cap, 3), np.float32),
               "depth": np.zeros(cap, np.uint32), "ref_mean": np.zeros(cap, np.float32),
               "target": np.zeros((cap, 3), np.float32), "rrs_target": np.zeros(cap, np.float32),
               "pixel": np.zeros(cap, np.uint32), "error": np.zeros(cap, np.float32),
               "error_for_avg": np.zeros(cap, np.float32),
               "number_samples": np.zeros(cap, np.float32)}
        batch = nb.TrainBatch(*(out[k].ctypes.data for k in nb.TRAIN_BATCH_FIELDS))
        if image is not None:
            image = np.ascontiguousarray(image, np.float32)
        ch = image.shape[1] if image is not None else 0
        total = lib().oracle_generate_training_data(
            C.byref(self.nodes), C.byref(params),
            image.ctypes.data if image is not None else None, ch, n_pixels,
            pixel_samples.ctypes.data if pixel_samples is not None else None, C.byref(batch),
            capacity)
        m = min(int(total), capacity)
        return {k: v[:m] for k, v in out.items()}, int(total)


def sample_weights(pixel, pixel_samples, n_pixels: int) -> np.ndarray:
    pixel = np.ascontiguousarray(pixel, np.uint32)
    pixel_samples = np.ascontiguousarray(pixel_samples, np.uint32)
    w = np.zeros(max(len(pixel), 1), np.float32)
    lib().oracle_sample_weights(pixel.ctypes.data, pixel_samples.ctypes.data, n_pixels,
                                len(pixel), w.ctypes.data)
    return w[:len(pixel)]


def frame_training_data(bounces, image, capacity: int, params, batch_capacity=None,
                        n_pixels=None):
    """The oracle's run of a whole synthetic frame: per bounce record the nodes, then the
    contributions; then the batch, the per-pixel counts and the weights."""
    hn = HostNodes(capacity)
    node_outs = []
    for b in bounces:
        node_outs.append(hn.record_nodes(b))
        hn.record_radiance(b["contrib_node"], b["contrib"])
    n_pixels = image.shape[0] if n_pixels is None else n_pixels
    counts = np.zeros(n_pixels, np.uint32)
    bc = capacity if batch_capacity is None else batch_capacity
    batch, total = hn.generate(params, bc, image=image, n_pixels=n_pixels, pixel_samples=counts)
    weights = sample_weights(batch["pixel"], counts, n_pixels)
    return {"nodes": hn, "node_outs": node_outs, "batch": batch, "total": total,
            "counts": counts, "weights": weights}


# ---- per-pixel error of the RRSNet loss (records.c) -------------------------------------------

def count_patch_samples(params, pixel, spp):
    pixel = np.ascontiguousarray(pixel, np.uint32)
    lib().oracle_count_patch_samples(C.byref(params), pixel.ctypes.data, len(pixel), spp.ctypes.data)


def accumulate_weighted_l(params, pixel_l, spp: int, first: bool, wl, cur, acc):
    pixel_l = np.ascontiguousarray(pixel_l, np.float32)
    lib().oracle_accumulate_weighted_l(C.byref(params), pixel_l.ctypes.data, spp, int(first),
                                       wl.ctypes.data, cur.ctypes.data, acc.ctypes.data)


def update_weighted_l(params, cur, acc, wl):
    lib().oracle_update_weighted_l(C.byref(params), cur.ctypes.data, acc.ctypes.data,
                                   wl.ctypes.data)


def calculate_error(params, ref, wl, spp, err) -> float:
    ref = np.ascontiguousarray(ref, np.float32)
    return float(lib().oracle_calculate_error(C.byref(params), ref.ctypes.data, ref.shape[1],
                                              wl.ctypes.data,
                                              spp.ctypes.data if spp is not None else None,
                                              err.ctypes.data))


def batch_arrays(capacity: int) -> dict:
    """Preallocated batch arrays for HostNodes.generate(out=...)."""
    cap = max(capacity, 1)
    v3 = ("pos", "wi", "normal", "albedo", "thp", "target")
    return {k: np.zeros((cap, 3) if k in v3 else cap,
                        np.uint32 if k in ("depth", "pixel") else np.float32)
            for k in nb.TRAIN_BATCH_FIELDS}


def ubs_error(params, pixel_l, spp: int, ref, err) -> float:
    pixel_l = np.ascontiguousarray(pixel_l, np.float32)
    ref = np.ascontiguousarray(ref, np.float32)
    return float(lib().oracle_ubs_error(C.byref(params), pixel_l.ctypes.data, spp,
                                        ref.ctypes.data, ref.shape[1], err.ctypes.data))


# ---- the wavefront steps around the path (render.c) -------------------------------------------

class HostScene:
    """A scene for the oracle: triangles as v0, e1, e2 in input order and the light list, built
    as the library builds them."""

    def __init__(self, vertices, triangles, tri_material, materials, environment=None):
        self.tm = np.ascontiguousarray(tri_material, np.uint32)
        self.mats = np.ascontiguousarray(materials, np.float32)
        self.env = (np.ascontiguousarray(environment, np.float32) if environment is not None
                    else np.zeros(3, np.float32))
        nt = len(triangles)
        self.nt = nt
        self.tri = np.zeros((nt, 9), np.float32)
        self.lights = np.zeros(nt, np.uint32)
        self.area = np.zeros(nt, np.float32)
        v = np.ascontiguousarray(vertices, np.float32)
        t = np.ascontiguousarray(triangles, np.uint32)
        vp = C.c_void_p
        L = lib()
        L.oracle_scene_tris.restype = C.c_uint32
        L.oracle_scene_tris.argtypes = [vp, vp, C.c_uint32, vp, vp, vp, vp, vp]
        self.nl = int(L.oracle_scene_tris(v.ctypes.data, t.ctypes.data, nt, self.tm.ctypes.data,
                                          self.mats.ctypes.data, self.tri.ctypes.data,
                                          self.lights.ctypes.data, self.area.ctypes.data))
        self.nee = True
        self.spec = None          # [materials] uint8 mirror flags (set_specular)

    def set_specular(self, specular):
        self.spec = np.ascontiguousarray(np.asarray(specular), np.uint8)

    @property
    def nl_sampled(self) -> int:
        """The lights next-event estimation samples (and MIS weighs against): none when off."""
        return self.nl if self.nee else 0

    def camera_rays(self, cam, sample: int, seed: int):
        n = cam.width * cam.height
        o, d = np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32)
        lib().oracle_camera_rays.argtypes = [C.POINTER(nb.Camera), C.c_uint32, C.c_uint32,
                                             C.c_void_p, C.c_void_p]
        lib().oracle_camera_rays(C.byref(cam), sample, seed, o.ctypes.data, d.ctypes.data)
        return {"origin": o, "dir": d, "thp": np.ones((n, 3), np.float32),
                "pdf": np.zeros(n, np.float32), "pixel": np.arange(n, dtype=np.uint32),
                "node": np.full(n, -1, np.int32)}

    def trace(self, rays: dict):
        n = len(rays["pixel"])
        h = {"prim": np.zeros(n, np.uint32), "t": np.zeros(n, np.float32),
             "u": np.zeros(n, np.float32), "v": np.zeros(n, np.float32)}
        f = lib().oracle_trace
        f.argtypes = [C.c_void_p] * 3 + [C.c_uint32] + [C.c_void_p] * 3 + [C.c_uint32] + \
            [C.c_void_p] * 4
        f(self.tri.ctypes.data, self.tm.ctypes.data, self.mats.ctypes.data, self.nt,
          *(np.ascontiguousarray(rays[k]).ctypes.data for k in ("origin", "dir", "thp")), n,
          *(h[k].ctypes.data for k in ("prim", "t", "u", "v")))
        return h

    def shade_split(self, rays: dict, hits: dict, depth: int, film):
        """(inference-queue vertices, specular-queue vertices, contributions)"""
        n = len(rays["pixel"])
        keys = ("pos", "wi", "normal", "albedo", "roughness", "thp", "depth", "pixel", "node")

        def arrays():
            return {"pos": np.zeros((n, 3), np.float32), "wi": np.zeros((n, 3), np.float32),
                    "normal": np.zeros((n, 3), np.float32), "albedo": np.zeros((n, 3), np.float32),
                    "roughness": np.zeros(n, np.float32), "thp": np.zeros((n, 3), np.float32),
                    "depth": np.zeros(n, np.uint32), "pixel": np.zeros(n, np.uint32),
                    "node": np.zeros(n, np.int32)}
        out, outs = arrays(), arrays()
        contrib = np.zeros((n, 3), np.float32)
        ns = np.zeros(1, np.uint32)
        spec = self.spec if self.spec is not None else np.zeros(len(self.mats), np.uint8)
        f = lib().oracle_shade_split
        f.restype = C.c_uint32
        f.argtypes = [C.c_void_p] * 3 + [C.c_uint32, C.c_uint32] + [C.c_void_p] * 10 + \
            [C.c_uint32, C.c_uint32] + [C.c_void_p] * 21
        m = f(self.tri.ctypes.data, self.tm.ctypes.data, self.mats.ctypes.data, self.nt,
              self.nl_sampled, self.env.ctypes.data, spec.ctypes.data,
              *(np.ascontiguousarray(rays[k]).ctypes.data for k in
                ("origin", "dir", "thp", "pdf", "pixel", "node")),
              hits["prim"].ctypes.data, hits["t"].ctypes.data, n, depth, film.ctypes.data,
              contrib.ctypes.data, *(out[k].ctypes.data for k in keys),
              *(outs[k].ctypes.data for k in keys), ns.ctypes.data)
        return ({k: v[:m] for k, v in out.items()}, {k: v[:int(ns[0])] for k, v in outs.items()},
                contrib)

    def scatter_specular(self, vs: dict, rays: dict, off: int, max_rays: int, depth: int,
                         seed: int):
        """writes the specular bounces into rays (a dict of [max_rays] arrays) from slot off"""
        n = len(vs["pixel"])
        f = lib().oracle_scatter_specular
        f.argtypes = [C.c_void_p] * 8 + [C.c_uint32] * 5 + [C.c_void_p] * 6
        f(*(np.ascontiguousarray(vs[k]).ctypes.data for k in
            ("pos", "wi", "normal", "albedo", "thp", "roughness", "pixel", "node")), n, off,
          max_rays, depth, seed,
          *(rays[k].ctypes.data for k in ("origin", "dir", "thp", "pdf", "pixel", "node")))

    def shade(self, rays: dict, hits: dict, depth: int, film):
        n = len(rays["pixel"])
        out = {"pos": np.zeros((n, 3), np.float32), "wi": np.zeros((n, 3), np.float32),
               "normal": np.zeros((n, 3), np.float32), "albedo": np.zeros((n, 3), np.float32),
               "roughness": np.zeros(n, np.float32), "thp": np.zeros((n, 3), np.float32),
               "depth": np.zeros(n, np.uint32), "pixel": np.zeros(n, np.uint32),
               "node": np.zeros(n, np.int32)}
        contrib = np.zeros((n, 3), np.float32)
        f = lib().oracle_shade
        f.restype = C.c_uint32
        f.argtypes = [C.c_void_p] * 3 + [C.c_uint32, C.c_uint32] + [C.c_void_p] * 9 + \
            [C.c_uint32, C.c_uint32] + [C.c_void_p] * 11
        m = f(self.tri.ctypes.data, self.tm.ctypes.data, self.mats.ctypes.data, self.nt,
              self.nl_sampled,
              self.env.ctypes.data,
              *(np.ascontiguousarray(rays[k]).ctypes.data for k in
                ("origin", "dir", "thp", "pdf", "pixel", "node")),
              hits["prim"].ctypes.data, hits["t"].ctypes.data, n, depth, film.ctypes.data,
              contrib.ctypes.data,
              *(out[k].ctypes.data for k in ("pos", "wi", "normal", "albedo", "roughness", "thp",
                                             "depth", "pixel", "node")))
        return {k: v[:m] for k, v in out.items()}, contrib

    def scatter(self, v: dict, rrs_norm, queue, depth: int, seed: int):
        nq = len(queue)
        r = {"origin": np.zeros((nq, 3), np.float32), "dir": np.zeros((nq, 3), np.float32),
             "thp": np.zeros((nq, 3), np.float32), "pdf": np.zeros(nq, np.float32),
             "pixel": np.zeros(nq, np.uint32), "node": np.zeros(nq, np.int32)}
        sh = {"origin": np.zeros((nq, 3), np.float32), "dir": np.zeros((nq, 3), np.float32),
              "tmax": np.zeros(nq, np.float32), "contrib": np.zeros((nq, 3), np.float32),
              "pixel": np.zeros(nq, np.uint32), "node": np.zeros(nq, np.int32)}
        rrs_norm = np.ascontiguousarray(rrs_norm, np.float32)
        queue = np.ascontiguousarray(queue, np.uint32)
        f = lib().oracle_scatter
        f.argtypes = [C.c_void_p] * 3 + [C.c_uint32] + [C.c_void_p] * 2 + [C.c_uint32] + \
            [C.c_void_p] * 8 + [C.c_uint32, C.c_uint32, C.c_uint32] + [C.c_void_p] * 12
        f(self.tri.ctypes.data, self.tm.ctypes.data, self.mats.ctypes.data, self.nt,
          self.lights.ctypes.data, self.area.ctypes.data, self.nl_sampled,
          *(np.ascontiguousarray(v[k]).ctypes.data for k in ("pos", "normal", "albedo", "thp",
                                                             "pixel", "node")),
          rrs_norm.ctypes.data, queue.ctypes.data, nq, depth, seed,
          *(r[k].ctypes.data for k in ("origin", "dir", "thp", "pdf", "pixel", "node")),
          *(sh[k].ctypes.data for k in ("origin", "dir", "tmax", "contrib", "pixel", "node")))
        return r, sh

    def scatter_fixed_rr(self, v: dict, rr: float, depth: int, seed: int):
        n = len(v["pixel"])
        r = {"origin": np.zeros((n, 3), np.float32), "dir": np.zeros((n, 3), np.float32),
             "thp": np.zeros((n, 3), np.float32), "pdf": np.zeros(n, np.float32),
             "pixel": np.zeros(n, np.uint32), "node": np.zeros(n, np.int32)}
        sh = {"origin": np.zeros((n, 3), np.float32), "dir": np.zeros((n, 3), np.float32),
              "tmax": np.zeros(n, np.float32), "contrib": np.zeros((n, 3), np.float32),
              "pixel": np.zeros(n, np.uint32), "node": np.zeros(n, np.int32)}
        f = lib().oracle_scatter_fixed_rr
        f.argtypes = [C.c_void_p] * 5 + [C.c_uint32] + [C.c_void_p] * 6 + \
            [C.c_uint32, C.c_float, C.c_uint32, C.c_uint32] + [C.c_void_p] * 12
        f(self.tri.ctypes.data, self.tm.ctypes.data, self.mats.ctypes.data,
          self.lights.ctypes.data, self.area.ctypes.data, self.nl_sampled,
          *(np.ascontiguousarray(v[k]).ctypes.data for k in ("pos", "normal", "albedo", "thp",
                                                             "pixel", "node")),
          n, rr, depth, seed,
          *(r[k].ctypes.data for k in ("origin", "dir", "thp", "pdf", "pixel", "node")),
          *(sh[k].ctypes.data for k in ("origin", "dir", "tmax", "contrib", "pixel", "node")))
        return r, sh

    def shadow(self, sh: dict, film):
        n = len(sh["pixel"])
        cout = np.zeros((n, 3), np.float32)
        f = lib().oracle_shadow
        f.argtypes = [C.c_void_p, C.c_uint32] + [C.c_void_p] * 5 + [C.c_uint32] + [C.c_void_p] * 2
        f(self.tri.ctypes.data, self.nt,
          *(np.ascontiguousarray(sh[k]).ctypes.data for k in ("origin", "dir", "tmax", "contrib",
                                                             "pixel")),
          n, film.ctypes.data, cout.ctypes.data)
        return cout

    @staticmethod
    def resolve(film, scale: float):
        n = film.shape[0]
        img = np.zeros((n, 3), np.float32)
        f = lib().oracle_film_resolve
        f.argtypes = [C.c_void_p, C.c_uint32, C.c_float, C.c_void_p]
        f(film.ctypes.data, n, scale, img.ctypes.data)
        return img
