"""ctypes binding of libnrrs_b200 (include/nrrs.h) and a host-side mirror of the reference's
NRRSNetwork interface (src/render/nrrs/net/network.h:22-214).

The library is the product; this module only binds it. Device buffers are passed as raw
pointers (`int` addresses, e.g. ``tensor.data_ptr()``), streams as raw ``cudaStream_t`` values.
There is no CPU fallback: if the shared library is missing this module raises on first use,
and on a machine without an sm_100 GPU ``NRRSNetwork`` raises ``NRRSError`` (NO_DEVICE).
"""
from __future__ import annotations

import ctypes as C
import os
import re
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "lib" / "libnrrs_b200.so"
HEADER = HERE.parent / "include" / "nrrs.h"

OK = 0
ERR_INVALID_ARG = -1
ERR_CAPACITY_OVERFLOW = -2
ERR_NAN = -3
ERR_TIMEOUT = -4
ERR_CUDA = -5
ERR_NO_DEVICE = -6
ERR_UNSUPPORTED = -7
ERR_IO = -8

DEV_OVERFLOW = 0x1
DEV_NAN = 0x2
DEV_TIMEOUT = 0x4
DEV_SATURATED = 0x8
DEV_BAD_INDEX = 0x10

PREC_FP32, PREC_FP16, PREC_BF16 = 0, 1, 2
FACTOR_ADRRS, FACTOR_RRSNET = 2, 3
NET_WORKLOAD, NET_REFERENCE = 0, 1


class Config(C.Structure):
    _fields_ = [
        ("n_levels", C.c_int32), ("n_features_per_level", C.c_int32),
        ("log2_hashmap_size", C.c_int32), ("base_resolution", C.c_int32),
        ("per_level_scale", C.c_float), ("sh_degree", C.c_int32),
        ("statnet_width", C.c_int32), ("statnet_hidden", C.c_int32),
        ("rrsnet_width", C.c_int32), ("rrsnet_hidden", C.c_int32),
        ("precision", C.c_int32), ("seed", C.c_uint64), ("table_init_scale", C.c_float),
        ("lr", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float),
        ("l2_reg", C.c_float), ("stat_eps", C.c_float), ("ref_eps", C.c_float),
        ("loss_clamp_max", C.c_float), ("cost_offset", C.c_float),
        ("normalize_pos", C.c_int32), ("aabb_min", C.c_float * 3), ("aabb_max", C.c_float * 3),
        ("max_queue", C.c_uint32), ("max_train", C.c_uint32), ("step", C.c_int32),
        ("network", C.c_int32), ("ema_decay", C.c_float), ("lr_rrsnet", C.c_float),
        ("sum_shards", C.c_uint32),
    ]


class VertexSoA(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in
                ("pos", "wi", "normal", "roughness", "albedo", "thp", "depth", "ref_mean",
                 "scatter_index")]


class DecideParams(C.Structure):
    _fields_ = [
        ("clamp_min", C.c_float), ("clamp_max", C.c_float), ("normalize_rate", C.c_float),
        ("use_ceil", C.c_int32), ("scale_up", C.c_int32), ("use_weight_window", C.c_int32),
        ("weight_window_size", C.c_float), ("factor_source", C.c_int32),
    ]


class Segment(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in
                ("offset", "count", "budget", "n_specular", "queue_offset", "queue_capacity")]


class PathNodes(C.Structure):
    """nrrs_path_nodes: the node block's capacity and device arrays."""
    _fields_ = [("capacity", C.c_uint32), ("max_record", C.c_uint32)] + [
        (n, C.c_void_p) for n in ("pos", "wi", "normal", "albedo", "roughness", "thp", "parent",
                                  "pixel", "rrs",
                                  "depth", "radiance", "first_child", "children", "arrived",
                                  "node_flags",
                                  "header", "scan_states")]


class TrainDataParams(C.Structure):
    _fields_ = [("ignore_zero_l", C.c_int32), ("copy_rrs_node", C.c_int32),
                ("dedupe_rrs_target", C.c_int32), ("thp_eps", C.c_float),
                ("frame_width", C.c_uint32), ("error_image_scale", C.c_uint32),
                ("error_per_pixel", C.c_void_p), ("samples_per_patch", C.c_void_p)]


TRAIN_BATCH_FIELDS = ("pos", "wi", "normal", "albedo", "roughness", "thp", "depth", "ref_mean",
                      "target", "rrs_target", "pixel", "error", "error_for_avg",
                      "number_samples")


class PixelErrorParams(C.Structure):
    """nrrs_pixel_error_params: the frame, its patches and the error switches."""
    _fields_ = [("frame_width", C.c_uint32), ("frame_height", C.c_uint32), ("scale", C.c_uint32),
                ("blend_weight", C.c_float), ("clamp", C.c_int32),
                ("multiply_samples", C.c_int32)]


class ErrorSum(C.Structure):
    """nrrs_error_sum: exact sum of the errors (device struct, zeroed once)."""
    _fields_ = [("acc", C.c_int64 * 3), ("done", C.c_uint32), ("value", C.c_float)]


class TrainBatch(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in TRAIN_BATCH_FIELDS]


class LossParams(C.Structure):
    """nrrs_loss_params: the RRSNet loss settings of nrrs_train_step_batch"""
    _fields_ = [("gamma1", C.c_float), ("gamma2", C.c_float), ("gamma3", C.c_float),
                ("gamma4", C.c_float), ("clamp_on", C.c_int32), ("clamp_max", C.c_float),
                ("n_pixels", C.c_uint32)]


class RaySoA(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("origin", "dir", "thp", "pdf", "pixel", "node")]


class HitSoA(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("prim", "t", "u", "v")]


class ShadowSoA(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("origin", "dir", "tmax", "contrib", "pixel", "node")]


PATH_VERTEX_FIELDS = ("pos", "wi", "normal", "albedo", "roughness", "thp", "depth", "pixel",
                      "node")


class PathVertices(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in PATH_VERTEX_FIELDS]


class Camera(C.Structure):
    _fields_ = [("pos", C.c_float * 3), ("forward", C.c_float * 3), ("up", C.c_float * 3),
                ("tan_half_fov_y", C.c_float), ("width", C.c_uint32), ("height", C.c_uint32)]


class NRRSError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} (status {code})")
        self.code = code


_lib = None

_SIGS = {
    "nrrs_config_default": (None, [C.POINTER(Config)]),
    "nrrs_config_reference_network": (None, [C.POINTER(Config)]),
    "nrrs_decide_params_default": (None, [C.POINTER(DecideParams)]),
    "nrrs_create": (C.c_int, [C.POINTER(Config), C.POINTER(C.c_void_p)]),
    "nrrs_destroy": (None, [C.c_void_p]),
    "nrrs_set_step": (C.c_int, [C.c_void_p, C.c_int32]),
    "nrrs_last_error": (C.c_char_p, [C.c_void_p]),
    "nrrs_status_string": (C.c_char_p, [C.c_int]),
    "nrrs_device_available": (C.c_int, []),
    "nrrs_infer": (C.c_int, [C.c_void_p, C.POINTER(VertexSoA), C.c_uint32,
                             C.POINTER(DecideParams), C.c_void_p, C.c_void_p, C.c_void_p]),
    "nrrs_decide_emit": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                   C.c_uint32, C.c_uint32, C.c_void_p, C.POINTER(DecideParams),
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                   C.c_void_p]),
    "nrrs_step": (C.c_int, [C.c_void_p, C.POINTER(VertexSoA), C.c_void_p, C.c_uint32, C.c_uint32,
                            C.c_uint32, C.POINTER(DecideParams), C.c_void_p, C.c_void_p,
                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                            C.c_void_p]),
    "nrrs_step_batched": (C.c_int, [C.c_void_p, C.POINTER(VertexSoA), C.c_void_p,
                                    C.POINTER(Segment), C.c_int32, C.POINTER(DecideParams),
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p]),
    "nrrs_train_step": (C.c_int, [C.c_void_p, C.POINTER(VertexSoA), C.c_void_p, C.c_uint32,
                                  C.c_void_p, C.c_void_p]),
    "nrrs_param_count": (C.c_uint64, [C.c_void_p]),
    "nrrs_param_layout": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                    C.POINTER(C.c_uint64)]),
    "nrrs_get_params": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "nrrs_set_params": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "nrrs_get_inference_params": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "nrrs_get_grads": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "nrrs_get_adam_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                                      C.POINTER(C.c_uint64)]),
    "nrrs_level_table": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "nrrs_save": (C.c_int, [C.c_void_p, C.c_char_p]),
    "nrrs_load": (C.c_int, [C.c_void_p, C.c_char_p]),
    "nrrs_get_device_status": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.c_void_p]),
    "nrrs_synth_vertices": (None, [C.c_uint64, C.c_uint64, C.c_uint64] + [C.c_void_p] * 10),
    "nrrs_decide_emit_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                           C.c_uint32, C.c_uint32, C.POINTER(DecideParams),
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                           C.c_void_p, C.c_void_p]),
    "nrrs_noalloc_device_status": (C.c_int, [C.POINTER(C.c_uint32), C.c_void_p]),
    "nrrs_loss_params_default": (None, [C.POINTER(LossParams)]),
    "nrrs_train_step_batch": (C.c_int, [C.c_void_p, C.POINTER(TrainBatch), C.c_uint32,
                                        C.c_void_p, C.c_void_p, C.POINTER(LossParams),
                                        C.c_void_p, C.c_void_p]),
    "nrrs_infer_dev": (C.c_int, [C.c_void_p, C.POINTER(VertexSoA), C.c_void_p, C.c_uint32,
                                 C.POINTER(DecideParams), C.c_void_p, C.c_void_p, C.c_void_p]),
    "nrrs_decide_emit_dev": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p,
                                       C.POINTER(DecideParams), C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    "nrrs_step_dev": (C.c_int, [C.c_void_p, C.POINTER(VertexSoA), C.c_void_p, C.c_void_p,
                                C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p,
                                C.POINTER(DecideParams), C.c_void_p, C.c_void_p, C.c_void_p,
                                C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    "nrrs_step_batched_dev": (C.c_int, [C.c_void_p, C.POINTER(VertexSoA), C.c_void_p,
                                        C.POINTER(Segment), C.c_void_p, C.c_int32,
                                        C.POINTER(DecideParams), C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p]),
    "nrrs_infer_accumulate": (C.c_int, [C.c_void_p, C.POINTER(VertexSoA), C.c_uint32,
                                        C.POINTER(DecideParams), C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p]),
    "nrrs_decide_emit_with_sum": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p,
                                            C.POINTER(DecideParams), C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    "nrrs_sum_from_accumulator": (C.c_double, [C.c_void_p, C.POINTER(DecideParams), C.c_int64]),
    "nrrs_train_grads": (C.c_int, [C.c_void_p, C.POINTER(VertexSoA), C.c_void_p, C.c_uint32,
                                   C.c_void_p, C.c_void_p]),
    "nrrs_copy_grads": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "nrrs_adam_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.c_float, C.c_void_p]),
    "nrrs_launch_count": (C.c_uint64, [C.c_void_p]),
    "nrrs_autotune": (C.c_int, [C.c_void_p, C.c_uint32, C.c_char_p, C.c_char_p, C.c_size_t]),
    "nrrs_set_launch_shape": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    "nrrs_get_launch_shape": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "nrrs_set_infer_split": (C.c_int, [C.c_void_p, C.c_int32]),
    "nrrs_get_infer_split": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "nrrs_set_cell_image": (C.c_int, [C.c_void_p, C.c_int32]),
    "nrrs_get_cell_image": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "nrrs_set_train_split": (C.c_int, [C.c_void_p, C.c_int32]),
    "nrrs_get_train_split": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "nrrs_graph_capture_batched": (C.c_int, [C.c_void_p, C.POINTER(VertexSoA), C.c_void_p,
                                             C.POINTER(Segment), C.c_int32,
                                             C.POINTER(DecideParams), C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.POINTER(C.c_void_p)]),
    "nrrs_graph_launch": (C.c_int, [C.c_void_p, C.c_void_p]),
    "nrrs_graph_destroy": (None, [C.c_void_p]),
    "nrrs_path_nodes_bytes": (C.c_uint64, [C.c_uint32, C.c_uint32]),
    "nrrs_path_nodes_init": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32,
                                       C.POINTER(PathNodes), C.c_void_p]),
    "nrrs_path_nodes_reset": (C.c_int, [C.POINTER(PathNodes), C.c_void_p]),
    "nrrs_path_nodes_status": (C.c_int, [C.POINTER(PathNodes), C.POINTER(C.c_uint32),
                                         C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                         C.c_void_p]),
    "nrrs_record_nodes": (C.c_int, [C.POINTER(PathNodes), C.POINTER(VertexSoA), C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                    C.c_void_p]),
    "nrrs_record_radiance": (C.c_int, [C.POINTER(PathNodes), C.c_void_p, C.c_void_p, C.c_uint32,
                                       C.c_void_p]),
    "nrrs_generate_training_data": (C.c_int, [C.POINTER(PathNodes), C.POINTER(TrainDataParams),
                                              C.c_void_p, C.c_int32, C.c_uint32, C.c_void_p,
                                              C.POINTER(TrainBatch), C.c_uint32, C.c_void_p,
                                              C.c_void_p]),
    "nrrs_sample_weights": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32,
                                      C.c_void_p, C.c_void_p]),
    "nrrs_count_patch_samples": (C.c_int, [C.POINTER(PixelErrorParams), C.c_void_p, C.c_uint32,
                                           C.c_void_p, C.c_void_p]),
    "nrrs_accumulate_weighted_l": (C.c_int, [C.POINTER(PixelErrorParams), C.c_void_p, C.c_uint32,
                                             C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_void_p]),
    "nrrs_update_weighted_l": (C.c_int, [C.POINTER(PixelErrorParams), C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_void_p]),
    "nrrs_calculate_error": (C.c_int, [C.POINTER(PixelErrorParams), C.c_void_p, C.c_int32,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p]),
    "nrrs_ubs_error": (C.c_int, [C.POINTER(PixelErrorParams), C.c_void_p, C.c_uint32, C.c_void_p,
                                 C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "nrrs_ubs_create": (C.c_int, [C.c_int32, C.c_double, C.POINTER(C.c_void_p)]),
    "nrrs_ubs_destroy": (None, [C.c_void_p]),
    "nrrs_ubs_begin_search": (C.c_int, [C.c_void_p]),
    "nrrs_ubs_next_state": (C.c_int, [C.c_void_p]),
    "nrrs_ubs_analyse_frame": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_uint32]),
    "nrrs_ubs_get_strategy": (C.c_int, [C.c_void_p, C.c_int32]),
    "nrrs_ubs_need_infer": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_float, C.c_float,
                                      C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
    "nrrs_ubs_best": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_float)]),
    "nrrs_ubs_set_best": (C.c_int, [C.c_void_p, C.c_char_p]),
    "nrrs_ubs_searching": (C.c_int, [C.c_void_p]),
    "nrrs_train_schedule_create": (C.c_int, [C.POINTER(C.c_double), C.POINTER(C.c_void_p)]),
    "nrrs_train_schedule_destroy": (None, [C.c_void_p]),
    "nrrs_train_schedule_tick": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_void_p]),
    "nrrs_scene_create": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p,
                                    C.c_void_p, C.c_uint32, C.c_void_p, C.POINTER(C.c_void_p)]),
    "nrrs_scene_destroy": (None, [C.c_void_p]),
    "nrrs_scene_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                  C.POINTER(C.c_uint32)]),
    "nrrs_camera_rays": (C.c_int, [C.POINTER(Camera), C.c_uint32, C.c_uint32, C.POINTER(RaySoA),
                                   C.c_void_p]),
    "nrrs_trace": (C.c_int, [C.c_void_p, C.POINTER(RaySoA), C.c_void_p, C.c_uint32,
                             C.POINTER(HitSoA), C.c_void_p]),
    "nrrs_shade_scratch_bytes": (C.c_uint64, [C.c_uint32]),
    "nrrs_shade": (C.c_int, [C.c_void_p, C.POINTER(RaySoA), C.POINTER(HitSoA), C.c_void_p,
                             C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p,
                             C.POINTER(PathVertices), C.c_void_p, C.c_void_p, C.c_void_p]),
    "nrrs_scatter": (C.c_int, [C.c_void_p, C.POINTER(PathVertices), C.c_void_p, C.c_void_p,
                               C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(RaySoA),
                               C.POINTER(ShadowSoA), C.c_void_p]),
    "nrrs_scene_set_nee": (C.c_int, [C.c_void_p, C.c_int32]),
    "nrrs_trace_scratch_bytes": (C.c_uint64, [C.c_uint32]),
    "nrrs_shade_split": (C.c_int, [C.c_void_p, C.POINTER(RaySoA), C.POINTER(HitSoA), C.c_void_p,
                                   C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p,
                                   C.POINTER(PathVertices), C.c_void_p, C.POINTER(PathVertices),
                                   C.c_void_p, C.c_void_p, C.c_void_p]),
    "nrrs_scene_set_specular": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32]),
    "nrrs_scatter_specular": (C.c_int, [C.c_void_p, C.POINTER(PathVertices), C.c_void_p,
                                        C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint32,
                                        C.c_uint32, C.POINTER(RaySoA), C.c_void_p, C.c_void_p]),
    "nrrs_trace_sorted": (C.c_int, [C.c_void_p, C.POINTER(RaySoA), C.c_void_p, C.c_uint32,
                                    C.POINTER(HitSoA), C.c_void_p, C.c_void_p]),
    "nrrs_scatter_fixed_rr": (C.c_int, [C.c_void_p, C.POINTER(PathVertices), C.c_void_p,
                                        C.c_uint32, C.c_float, C.c_uint32, C.c_uint32,
                                        C.POINTER(RaySoA), C.POINTER(ShadowSoA), C.c_void_p]),
    "nrrs_trace_shadow": (C.c_int, [C.c_void_p, C.POINTER(ShadowSoA), C.c_void_p, C.c_uint32,
                                    C.c_void_p, C.c_void_p, C.c_void_p]),
    "nrrs_film_resolve": (C.c_int, [C.c_void_p, C.c_uint32, C.c_float, C.c_void_p, C.c_void_p]),
    "nrrs_last_infer_grid": (C.c_int32, [C.c_void_p]),
    "nrrs_kernel_name": (C.c_char_p, [C.c_int32]),
    "nrrs_profile_enable": (C.c_int, [C.c_void_p, C.c_int32]),
    "nrrs_profile_read": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_uint64),
                                    C.POINTER(C.c_double)]),
}

KERNEL_KINDS = ("infer_fp32", "infer_tc", "sum", "decide", "pack_weights", "table_half",
                "train_statnet", "train_rrsnet", "train_wgrad", "train_reduce", "adam", "encode",
                "train_scatter", "train_encode", "infer_rrs", "cell_image")


def lib():
    """Load libnrrs_b200.so (built by nrrs-code_b200/build.py); raise if it is missing."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"{LIB_PATH} is missing: run nrrs-code_b200/build.py")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def header_functions() -> list[str]:
    """Names of every function declared in include/nrrs.h."""
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nrrs_[a-z_0-9]+)\s*\(", text)))


def default_config(**kw) -> Config:
    c = Config()
    lib().nrrs_config_default(C.byref(c))
    for k, v in kw.items():
        if k in ("aabb_min", "aabb_max"):
            getattr(c, k)[:] = list(v)
        else:
            setattr(c, k, v)
    return c


def reference_config(**kw) -> Config:
    """nrrs_config_reference_network (the reference's shipped network), then kw"""
    c = Config()
    lib().nrrs_config_default(C.byref(c))
    lib().nrrs_config_reference_network(C.byref(c))
    for k, v in kw.items():
        if k in ("aabb_min", "aabb_max"):
            getattr(c, k)[:] = list(v)
        else:
            setattr(c, k, v)
    return c


def default_decide(**kw) -> DecideParams:
    p = DecideParams()
    lib().nrrs_decide_params_default(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _ptr(x):
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if hasattr(x, "ctypes"):
        return x.ctypes.data
    raise TypeError(type(x))


def vertex_soa(pos, wi, normal, roughness, albedo, thp, depth=None, ref_mean=None,
               scatter_index=None) -> VertexSoA:
    return VertexSoA(*(_ptr(a) for a in (pos, wi, normal, roughness, albedo, thp, depth, ref_mean,
                                         scatter_index)))


def synth(seed: int, n: int, first: int = 0):
    """Synthetic vertices as a dict of numpy arrays (host), from the library's generator."""
    import numpy as np
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


def synth_paths(seed: int, n_pixels: int, bounces: int = 8, capacity: int | None = None,
                record_prob: float = 0.7, split_probs=(0.35, 0.5, 0.1, 0.05),
                contrib_probs=(0.4, 0.45, 0.15), zero_contrib: float = 0.1):
    """A synthetic training frame for the path-record entry points, as numpy arrays (host).

    Bounce 0 has one vertex per pixel with no parent node. Each vertex records a node with
    probability record_prob, emits 0, 1 or 2 radiance contributions (contrib_probs; a fraction
    zero_contrib of them are zero) to its node, and spawns 0..3 vertices of the next bounce
    (split_probs, mean 0.85) that inherit its pixel and take its node as their parent, as the
    reference's ray payload carries mNodeIdx (integrator.cpp:824-831). Node numbers follow the
    library's rule (recorded vertices in vertex order, until capacity), so each bounce's parent
    array and the expected node_out are known in advance.

    Returns (bounces, image): a list of dicts with pos, wi, normal, albedo, roughness, thp,
    depth, pixel, rrs,
    record, parent, node (expected node_out), contrib_node, contrib; and an RGBA image
    [n_pixels][4] standing in for the rendered frame."""
    import numpy as np
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    n_nodes = 0
    pixel = np.arange(n_pixels, dtype=np.uint32)
    parent = np.full(n_pixels, -1, np.int32)
    thp_prev = np.ones((n_pixels, 3), np.float32)
    for d in range(bounces):
        n = len(pixel)
        if n == 0:
            break
        wi = rng.normal(size=(n, 3)).astype(np.float32)
        wi /= np.linalg.norm(wi, axis=1, keepdims=True)
        thp = (thp_prev * rng.uniform(0.3, 1.0, size=(n, 3))).astype(np.float32)
        nrm = rng.normal(size=(n, 3)).astype(np.float32)
        nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
        b = {
            "pos": rng.uniform(0.0, 1.0, size=(n, 3)).astype(np.float32),
            "wi": wi.astype(np.float32),
            "normal": nrm.astype(np.float32),
            "albedo": rng.uniform(0.0, 1.0, size=(n, 3)).astype(np.float32),
            "roughness": rng.uniform(0.0, 1.0, size=n).astype(np.float32),
            "thp": thp,
            "depth": np.full(n, d, np.uint32),
            "pixel": pixel,
            "rrs": rng.uniform(0.2, 3.0, size=n).astype(np.float32),
            "record": (rng.uniform(size=n) < record_prob).astype(np.uint8),
            "parent": parent,
        }
        rec = b["record"].astype(bool)
        idx = n_nodes + np.cumsum(rec) - 1
        ok = rec & (idx < (capacity if capacity is not None else np.iinfo(np.int64).max))
        node = np.where(ok, idx, parent).astype(np.int32)
        n_nodes = min(n_nodes + int(rec.sum()), capacity) if capacity is not None else n_nodes + int(rec.sum())
        b["node"] = node
        k = rng.choice(3, size=n, p=contrib_probs)
        src = np.repeat(np.arange(n), k)
        le = rng.lognormal(0.0, 1.5, size=(len(src), 3)).astype(np.float32)
        le[rng.uniform(size=len(src)) < zero_contrib] = 0.0
        b["contrib_node"] = node[src]
        b["contrib"] = (thp[src] * le).astype(np.float32)
        out.append(b)
        s = rng.choice(4, size=n, p=split_probs)
        nxt = np.repeat(np.arange(n), s)
        pixel = pixel[nxt]
        parent = node[nxt]
        thp_prev = thp[nxt]
    image = rng.uniform(0.0, 2.0, size=(n_pixels, 4)).astype(np.float32)
    return out, image


NOALLOC_MAX_N = 1 << 24


def decide_emit_noalloc(rrs, rnd, n, budget, n_specular, params, rrs_norm, split, queue,
                        capacity, next_size, scatter_index=None, stream=0) -> int:
    """nrrs_decide_emit_noalloc: the decision + emission without a context or any device
    allocation (scratch lives in a static device array). Returns the status code."""
    return lib().nrrs_decide_emit_noalloc(_ptr(rrs), _ptr(rnd), _ptr(scatter_index), n, budget,
                                          n_specular, C.byref(params), _ptr(rrs_norm),
                                          _ptr(split), _ptr(queue), capacity, _ptr(next_size),
                                          stream)


def noalloc_device_status(stream=0) -> tuple[int, int]:
    """nrrs_noalloc_device_status: (status code, NRRS_DEV_* bits) raised by
    nrrs_decide_emit_noalloc calls since the last read; synchronises the stream and clears them."""
    f = C.c_uint32(0)
    rc = lib().nrrs_noalloc_device_status(C.byref(f), stream)
    return rc, int(f.value)


def _check(rc: int, what: str):
    if rc != OK:
        raise NRRSError(rc, f"{what}: {lib().nrrs_status_string(rc).decode()}")


def path_nodes_bytes(capacity: int, max_record: int) -> int:
    """Bytes of the device block of a node buffer (nrrs_path_nodes_bytes)."""
    return lib().nrrs_path_nodes_bytes(capacity, max_record)


def default_loss_params(**kw) -> LossParams:
    """nrrs_loss_params_default (gamma 1, 0, 0, 0, no clamp: nrrs_train_step's loss), then kw."""
    p = LossParams()
    lib().nrrs_loss_params_default(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def default_train_data_params(**kw) -> TrainDataParams:
    """The reference's defaults: zero-L samples kept, thp not scaled by rrs, no deduplication,
    thp threshold 1e-5."""
    p = TrainDataParams(0, 0, 0, 1e-5, 0, 0, None, None)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def train_batch(**arrays) -> TrainBatch:
    """A TrainBatch from device arrays (any field may be omitted)."""
    bad = set(arrays) - set(TRAIN_BATCH_FIELDS)
    if bad:
        raise KeyError(sorted(bad))
    return TrainBatch(*(_ptr(arrays.get(k)) for k in TRAIN_BATCH_FIELDS))


class NRRSPathNodesBuffer:
    """Mirror of the reference's NRRSPathNodesBuffer (src/render/nrrs/workqueue.h:108-188) over
    a caller-owned device block (e.g. a uint8 CUDA tensor of path_nodes_bytes bytes)."""

    def __init__(self, dev_ptr: int, nbytes: int, capacity: int, max_record: int, stream=0):
        self.nodes = PathNodes()
        _check(lib().nrrs_path_nodes_init(dev_ptr, nbytes, capacity, max_record,
                                          C.byref(self.nodes), stream), "nrrs_path_nodes_init")

    def reset(self, stream=0):
        _check(lib().nrrs_path_nodes_reset(C.byref(self.nodes), stream), "nrrs_path_nodes_reset")

    def status(self, stream=0) -> tuple[int, int, int]:
        """(size, dropped, device flags); synchronises the stream and clears the flags."""
        size, dropped, flags = C.c_uint32(), C.c_uint32(), C.c_uint32()
        _check(lib().nrrs_path_nodes_status(C.byref(self.nodes), C.byref(size),
                                            C.byref(dropped), C.byref(flags), stream),
               "nrrs_path_nodes_status")
        return size.value, dropped.value, flags.value

    def size(self, stream=0) -> int:
        return self.status(stream)[0]

    def recordNode(self, v: VertexSoA, parent, pixel, rrs, record, n: int, node_out, stream=0):
        """recordNode for a wavefront (nrrs_record_nodes)."""
        _check(lib().nrrs_record_nodes(C.byref(self.nodes), C.byref(v), _ptr(parent),
                                       _ptr(pixel), _ptr(rrs), _ptr(record), n, _ptr(node_out),
                                       stream), "nrrs_record_nodes")

    def recordRadiance(self, node, contrib, n: int, stream=0):
        """recordRadiance for a queue of contributions (nrrs_record_radiance)."""
        _check(lib().nrrs_record_radiance(C.byref(self.nodes), _ptr(node), _ptr(contrib), n,
                                          stream), "nrrs_record_radiance")

    def generate_training_data(self, params: TrainDataParams, batch: TrainBatch, capacity: int,
                               size_dev, image=None, image_channels: int = 4, n_pixels: int = 0,
                               pixel_samples=None, stream=0):
        """nrrs_generate_training_data (train.cu:432-570)."""
        _check(lib().nrrs_generate_training_data(C.byref(self.nodes), C.byref(params),
                                                 _ptr(image), image_channels, n_pixels,
                                                 _ptr(pixel_samples), C.byref(batch), capacity,
                                                 _ptr(size_dev), stream),
               "nrrs_generate_training_data")


def default_pixel_error_params(frame_width: int, frame_height: int, **kw) -> PixelErrorParams:
    """The reference's defaults: patches of one pixel (the shipped error_image_scale), blend
    weight 0.5, error clamped at 100, error_for_avg not scaled by the sample count."""
    p = PixelErrorParams(frame_width, frame_height, 1, 0.5, 1, 0)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def count_patch_samples(params: PixelErrorParams, pixel, n: int, samples_per_patch, stream=0):
    """nrrs_count_patch_samples: +1 per ray in its pixel's patch."""
    _check(lib().nrrs_count_patch_samples(C.byref(params), _ptr(pixel), n,
                                          _ptr(samples_per_patch), stream),
           "nrrs_count_patch_samples")


def accumulate_weighted_l(params: PixelErrorParams, pixel_l, spp: int, first_frame: bool,
                          weighted_l, weighted_l_current, weighted_l_current_acc, stream=0):
    """nrrs_accumulate_weighted_l: this frame's radiance per patch (trainStep STEP#1.1)."""
    _check(lib().nrrs_accumulate_weighted_l(C.byref(params), _ptr(pixel_l), spp,
                                            1 if first_frame else 0, _ptr(weighted_l),
                                            _ptr(weighted_l_current),
                                            _ptr(weighted_l_current_acc), stream),
           "nrrs_accumulate_weighted_l")


def update_weighted_l(params: PixelErrorParams, weighted_l_current, weighted_l_current_acc,
                      weighted_l, stream=0):
    """nrrs_update_weighted_l (nrrs_update_weighted_L, train.cu:344-363)."""
    _check(lib().nrrs_update_weighted_l(C.byref(params), _ptr(weighted_l_current),
                                        _ptr(weighted_l_current_acc), _ptr(weighted_l), stream),
           "nrrs_update_weighted_l")


def calculate_error(params: PixelErrorParams, ref, ref_channels: int, weighted_l,
                    samples_per_patch, error, error_sum=None, stream=0):
    """nrrs_calculate_error (train.cu:365-430) and the exact error sum into error_sum, a device
    buffer of at least sizeof(ErrorSum) bytes zeroed once."""
    _check(lib().nrrs_calculate_error(C.byref(params), _ptr(ref), ref_channels, _ptr(weighted_l),
                                      _ptr(samples_per_patch), _ptr(error), _ptr(error_sum),
                                      stream),
           "nrrs_calculate_error")


def ubs_error(params: PixelErrorParams, pixel_l, spp: int, ref, ref_channels: int, error,
              error_sum=None, stream=0):
    """nrrs_ubs_error (nrrs_UBS_calc_error, train.cu:594-608) and its exact sum."""
    _check(lib().nrrs_ubs_error(C.byref(params), _ptr(pixel_l), spp, _ptr(ref), ref_channels,
                                _ptr(error), _ptr(error_sum), stream), "nrrs_ubs_error")


UBS_FIXED_RR, UBS_ADRRS, UBS_NRRS = 0, 1, 2


class UBS:
    """The per-depth strategy search of the reference's NRRSPathTracer (integrator.h:324-439,
    integrator.cpp:2787-2891) over nrrs_ubs_*."""

    def __init__(self, max_depth: int = 6, error_eval_seconds: float = 0.17e-3):
        self._h = None
        h = C.c_void_p()
        _check(lib().nrrs_ubs_create(max_depth, error_eval_seconds, C.byref(h)), "nrrs_ubs_create")
        self._h = h
        self.max_depth = max_depth

    def close(self):
        if self._h:
            lib().nrrs_ubs_destroy(self._h)
            self._h = None

    __del__ = close

    def UBSResetAndBeginSearch(self):
        _check(lib().nrrs_ubs_begin_search(self._h), "nrrs_ubs_begin_search")

    def UBSNextState(self) -> bool:
        return lib().nrrs_ubs_next_state(self._h) == 1

    def UBSAnalyseFrame(self, now_seconds: float, frame_error_sum: float, resolution: int):
        _check(lib().nrrs_ubs_analyse_frame(self._h, now_seconds, frame_error_sum, resolution),
               "nrrs_ubs_analyse_frame")

    def strategy(self, depth: int) -> int:
        return lib().nrrs_ubs_get_strategy(self._h, depth)

    def isInferMode(self, depth: int, enable_rrs=True, clamp_min=0.05, clamp_max=8.0,
                    max_rrs_depth=6, use_net_output_rrs=True) -> tuple[bool, int]:
        """(infer at this depth, factor source) -- isInferMode and the factor choice."""
        src = C.c_int32()
        r = lib().nrrs_ubs_need_infer(self._h, depth, int(enable_rrs), clamp_min, clamp_max,
                                      max_rrs_depth, int(use_net_output_rrs), C.byref(src))
        return r == 1, src.value

    def best(self) -> tuple[list, float]:
        arr = (C.c_int32 * self.max_depth)()
        eff = C.c_float()
        _check(lib().nrrs_ubs_best(self._h, arr, C.byref(eff)), "nrrs_ubs_best")
        return list(arr), eff.value

    def set_best(self, digits: str):
        _check(lib().nrrs_ubs_set_best(self._h, digits.encode()), "nrrs_ubs_set_best")

    @property
    def searching(self) -> bool:
        return lib().nrrs_ubs_searching(self._h) == 1


class TrainScheduleState(C.Structure):
    _fields_ = [("state", C.c_int32), ("step", C.c_int32), ("enable_rrs", C.c_int32),
                ("use_net_output_rrs", C.c_int32), ("stop_training", C.c_int32),
                ("request_exit", C.c_int32), ("seconds_per_frame", C.c_double)]


class TrainSchedule:
    """autoTrainControl (integrator.cpp:2659-2736) over nrrs_train_schedule_*."""

    def __init__(self, durations):
        self._h = None
        h = C.c_void_p()
        d = (C.c_double * 4)(*durations)
        _check(lib().nrrs_train_schedule_create(d, C.byref(h)), "nrrs_train_schedule_create")
        self._h = h

    def close(self):
        if self._h:
            lib().nrrs_train_schedule_destroy(self._h)
            self._h = None

    __del__ = close

    def tick(self, elapsed: float, now_seconds: float) -> TrainScheduleState:
        st = TrainScheduleState()
        _check(lib().nrrs_train_schedule_tick(self._h, elapsed, now_seconds, C.byref(st)),
               "nrrs_train_schedule_tick")
        return st


class Scene:
    """A triangle scene on the device with its BVH (nrrs_scene_*); arrays are host numpy."""

    def __init__(self, vertices, triangles, tri_material, materials, environment=None):
        import numpy as np
        self._h = None
        self.vertices = np.ascontiguousarray(vertices, np.float32)
        self.triangles = np.ascontiguousarray(triangles, np.uint32)
        self.tri_material = np.ascontiguousarray(tri_material, np.uint32)
        self.materials = np.ascontiguousarray(materials, np.float32)
        self.environment = (np.ascontiguousarray(environment, np.float32)
                            if environment is not None else None)
        h = C.c_void_p()
        _check(lib().nrrs_scene_create(
            self.vertices.ctypes.data, len(self.vertices), self.triangles.ctypes.data,
            len(self.triangles), self.tri_material.ctypes.data, self.materials.ctypes.data,
            len(self.materials),
            self.environment.ctypes.data if self.environment is not None else None,
            C.byref(h)), "nrrs_scene_create")
        self._h = h

    def close(self):
        if self._h:
            lib().nrrs_scene_destroy(self._h)
            self._h = None

    __del__ = close

    def set_specular(self, specular):
        """Specular materials: specular[m] = 1 makes material m a perfect mirror, 2 thin glass."""
        import numpy as np
        a = np.ascontiguousarray(np.asarray(specular), np.uint8)
        _check(lib().nrrs_scene_set_specular(self._h, a.ctypes.data, len(a)),
               "nrrs_scene_set_specular")

    def set_nee(self, enable: bool):
        """Next-event estimation on or off (the reference's mEnableNEE)."""
        _check(lib().nrrs_scene_set_nee(self._h, int(bool(enable))), "nrrs_scene_set_nee")

    def info(self) -> tuple[int, int, int]:
        a, b, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
        _check(lib().nrrs_scene_info(self._h, C.byref(a), C.byref(b), C.byref(c)),
               "nrrs_scene_info")
        return a.value, b.value, c.value


def soa(cls, arrays: dict):
    """A ctypes SoA struct (RaySoA, HitSoA, ShadowSoA, PathVertices) from a dict of arrays."""
    return cls(*(_ptr(arrays.get(n)) for n, _ in cls._fields_))


def camera_rays(cam: Camera, sample: int, seed: int, rays: RaySoA, stream=0):
    _check(lib().nrrs_camera_rays(C.byref(cam), sample, seed, C.byref(rays), stream),
           "nrrs_camera_rays")


def trace(scene: Scene, rays: RaySoA, n_dev, max_n: int, hits: HitSoA, stream=0):
    _check(lib().nrrs_trace(scene._h, C.byref(rays), _ptr(n_dev), max_n, C.byref(hits), stream),
           "nrrs_trace")


def shade_scratch_bytes(max_n: int) -> int:
    return lib().nrrs_shade_scratch_bytes(max_n)


def shade(scene: Scene, rays: RaySoA, hits: HitSoA, n_dev, max_n: int, depth: int, film,
          contrib, out: PathVertices, n_out_dev, scratch, stream=0):
    _check(lib().nrrs_shade(scene._h, C.byref(rays), C.byref(hits), _ptr(n_dev), max_n, depth,
                            _ptr(film), _ptr(contrib), C.byref(out), _ptr(n_out_dev),
                            _ptr(scratch), stream), "nrrs_shade")


def scatter(scene: Scene, v: PathVertices, rrs_norm, queue, queue_size_dev, max_queue: int,
            depth: int, seed: int, rays: RaySoA, shadow: ShadowSoA, stream=0):
    _check(lib().nrrs_scatter(scene._h, C.byref(v), _ptr(rrs_norm), _ptr(queue),
                              _ptr(queue_size_dev), max_queue, depth, seed, C.byref(rays),
                              C.byref(shadow), stream), "nrrs_scatter")


def shade_split(scene: Scene, rays: RaySoA, hits: HitSoA, n_dev, max_n: int, depth: int, film,
                contrib, out: PathVertices, n_out_dev, out_specular: PathVertices,
                n_specular_dev, scratch, stream=0):
    """nrrs_shade with mirror hits in their own queue (the closest-hit specular branch)."""
    _check(lib().nrrs_shade_split(scene._h, C.byref(rays), C.byref(hits), _ptr(n_dev), max_n,
                                  depth, _ptr(film), _ptr(contrib), C.byref(out), _ptr(n_out_dev),
                                  C.byref(out_specular), _ptr(n_specular_dev), _ptr(scratch),
                                  stream), "nrrs_shade_split")


def scatter_specular(scene: Scene, v: PathVertices, n_dev, max_n: int, ray_offset_dev,
                     max_rays: int, depth: int, seed: int, rays: RaySoA, n_rays_out_dev,
                     stream=0):
    """The specular bounce (mirror or thin glass) of the specular vertices into ray slots after
    the RRS-scattered ones."""
    _check(lib().nrrs_scatter_specular(scene._h, C.byref(v), _ptr(n_dev), max_n,
                                       _ptr(ray_offset_dev), max_rays, depth, seed,
                                       C.byref(rays), _ptr(n_rays_out_dev), stream),
           "nrrs_scatter_specular")


def trace_scratch_bytes(max_n: int) -> int:
    return int(lib().nrrs_trace_scratch_bytes(max_n))


def trace_sorted(scene: Scene, rays: RaySoA, n_dev, max_n: int, hits: HitSoA, scratch, stream=0):
    """nrrs_trace with the rays walked in (direction octant, origin Morton) order; same hits."""
    _check(lib().nrrs_trace_sorted(scene._h, C.byref(rays), _ptr(n_dev), max_n, C.byref(hits),
                                   _ptr(scratch), stream), "nrrs_trace_sorted")


def scatter_fixed_rr(scene: Scene, v: PathVertices, n_dev, max_n: int, rr: float, depth: int,
                     seed: int, rays: RaySoA, shadow: ShadowSoA, stream=0):
    """The fixed Russian-roulette branch of handleIntersections (depths without inference):
    slot j keeps vertex j with probability rr, thp / rr; a killed vertex leaves an empty slot."""
    _check(lib().nrrs_scatter_fixed_rr(scene._h, C.byref(v), _ptr(n_dev), max_n, rr, depth, seed,
                                       C.byref(rays), C.byref(shadow), stream),
           "nrrs_scatter_fixed_rr")


def trace_shadow(scene: Scene, shadow: ShadowSoA, n_dev, max_n: int, film, contrib_out,
                 stream=0):
    _check(lib().nrrs_trace_shadow(scene._h, C.byref(shadow), _ptr(n_dev), max_n, _ptr(film),
                                   _ptr(contrib_out), stream), "nrrs_trace_shadow")


def film_resolve(film, n_pixels: int, scale: float, image, stream=0):
    _check(lib().nrrs_film_resolve(_ptr(film), n_pixels, scale, _ptr(image), stream),
           "nrrs_film_resolve")


def synth_scene(seed: int, n_boxes: int = 40, size: float = 1.0, closed: bool = False):
    """A room (white walls, a red and a green wall, an emissive ceiling quad; open at the front
    unless closed) filled with n_boxes random axis-aligned boxes of random albedo, as numpy
    arrays: vertices, triangles, tri_material, materials, environment. Deterministic in seed."""
    import numpy as np
    rng = np.random.default_rng(seed)
    verts, tris, mat = [], [], []
    mats = [[0.75, 0.75, 0.75, 0, 0, 0], [0.7, 0.1, 0.1, 0, 0, 0], [0.1, 0.7, 0.1, 0, 0, 0],
            [0.0, 0.0, 0.0, 12.0, 11.0, 9.0]]

    def quad(a, b, c, d, m):
        i = len(verts)
        verts.extend([a, b, c, d])
        tris.extend([[i, i + 1, i + 2], [i, i + 2, i + 3]])
        mat.extend([m, m])

    S = size
    quad([0, 0, 0], [S, 0, 0], [S, 0, S], [0, 0, S], 0)          # floor
    quad([0, S, 0], [0, S, S], [S, S, S], [S, S, 0], 0)          # ceiling
    quad([0, 0, S], [S, 0, S], [S, S, S], [0, S, S], 0)          # back
    quad([0, 0, 0], [0, 0, S], [0, S, S], [0, S, 0], 1)          # left, red
    quad([S, 0, 0], [S, S, 0], [S, S, S], [S, 0, S], 2)          # right, green
    if closed:
        quad([0, 0, 0], [0, S, 0], [S, S, 0], [S, 0, 0], 0)      # front
    c, h = 0.5 * S, 0.12 * S
    quad([c - h, S * 0.999, c - h], [c + h, S * 0.999, c - h], [c + h, S * 0.999, c + h],
         [c - h, S * 0.999, c + h], 3)                           # the light
    for _ in range(n_boxes):
        mats.append(list(rng.uniform(0.2, 0.9, 3)) + [0, 0, 0])
        m = len(mats) - 1
        lo = rng.uniform(0.05, 0.8, 3) * S
        hi = lo + rng.uniform(0.03, 0.15, 3) * S
        x0, y0, z0 = lo
        x1, y1, z1 = hi
        quad([x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0], m)
        quad([x0, y0, z1], [x0, y1, z1], [x1, y1, z1], [x1, y0, z1], m)
        quad([x0, y0, z0], [x0, y1, z0], [x0, y1, z1], [x0, y0, z1], m)
        quad([x1, y0, z0], [x1, y0, z1], [x1, y1, z1], [x1, y1, z0], m)
        quad([x0, y0, z0], [x0, y0, z1], [x1, y0, z1], [x1, y0, z0], m)
        quad([x0, y1, z0], [x1, y1, z0], [x1, y1, z1], [x0, y1, z1], m)
    return (np.asarray(verts, np.float32), np.asarray(tris, np.uint32),
            np.asarray(mat, np.uint32), np.asarray(mats, np.float32),
            np.asarray([0.05, 0.05, 0.08], np.float32))


def room_camera(width: int, height: int, size: float = 1.0, inside: bool = False) -> Camera:
    """A camera looking into synth_scene's room through its open front, or from just inside
    its front wall."""
    z, tan = (0.02 * size, 0.75) if inside else (-1.3 * size, 0.42)
    return Camera((C.c_float * 3)(0.5 * size, 0.5 * size, z),
                  (C.c_float * 3)(0.0, 0.0, 1.0), (C.c_float * 3)(0.0, 1.0, 0.0),
                  tan, width, height)


def calculate_sample_weight(pixel, pixel_samples, n_pixels: int, size_dev, max_n: int, weight,
                            stream=0):
    """nrrs_sample_weights (nrrs_calculate_sample_weight, train.cu:572-592)."""
    _check(lib().nrrs_sample_weights(_ptr(pixel), _ptr(pixel_samples), n_pixels, _ptr(size_dev),
                                     max_n, _ptr(weight), stream), "nrrs_sample_weights")


VERTEX_FIELDS = ("pos", "wi", "normal", "roughness", "albedo", "thp", "depth", "ref_mean")


class BatchedGraph:
    """An instantiated CUDA graph of nrrs_step_batched (nrrs_graph_*)."""

    def __init__(self, handle):
        self._g = handle

    def launch(self, stream=0):
        rc = lib().nrrs_graph_launch(self._g, stream)
        if rc != OK:
            raise NRRSError(rc, "graph launch failed")

    def close(self):
        if getattr(self, "_g", None):
            lib().nrrs_graph_destroy(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class NRRSNetwork:
    """Mirror of the reference NRRSNetwork over the C-ABI.

    reference                                  here
    NRRSNetwork(json) + reset/resize           NRRSNetwork(Config)         (nrrs_create)
    setStep(int)                               setStep                     (nrrs_set_step)
    prepareInferenceData + inference           inference                   (nrrs_infer)
    generateRRSNumber (integrator)             generateRRSNumber           (nrrs_step)
    calcSum2PassAsync + "Gen Tids"             decideEmit                  (nrrs_decide_emit)
    train(input, output, offset, onlyLL2)      train                       (nrrs_train_step)
    saveWeights / loadWeights (stubs there)    saveWeights / loadWeights   (nrrs_save/load)
    """

    def __init__(self, config: Config | None = None):
        self.config = config if config is not None else default_config()
        h = C.c_void_p()
        rc = lib().nrrs_create(C.byref(self.config), C.byref(h))
        if rc != OK:
            raise NRRSError(rc, lib().nrrs_last_error(None).decode())
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().nrrs_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        if rc != OK:
            raise NRRSError(rc, lib().nrrs_last_error(self._h).decode())
        return rc

    @property
    def handle(self):
        return self._h

    # ---- reference-named operations ----
    def setStep(self, step: int):
        self._check(lib().nrrs_set_step(self._h, step))

    def inference(self, soa: VertexSoA, n: int, params: DecideParams, stats, rrs, stream=0):
        return self._check(lib().nrrs_infer(self._h, C.byref(soa), n, C.byref(params),
                                            _ptr(stats), _ptr(rrs), stream))

    def decideEmit(self, rrs, rnd, n, budget, n_specular, params, rrs_norm, split, queue,
                   capacity, next_size, scatter_index=None, n_specular_dev=None, stream=0):
        return self._check(lib().nrrs_decide_emit(
            self._h, _ptr(rrs), _ptr(rnd), _ptr(scatter_index), n, budget, n_specular,
            _ptr(n_specular_dev), C.byref(params), _ptr(rrs_norm), _ptr(split), _ptr(queue),
            capacity, _ptr(next_size), stream))

    def generateRRSNumber(self, soa, rnd, n, budget, n_specular, params, stats, rrs, rrs_norm,
                          split, queue, capacity, next_size, stream=0):
        return self._check(lib().nrrs_step(
            self._h, C.byref(soa), _ptr(rnd), n, budget, n_specular, C.byref(params), _ptr(stats),
            _ptr(rrs), _ptr(rrs_norm), _ptr(split), _ptr(queue), capacity, _ptr(next_size),
            stream))

    def generateRRSNumberBatched(self, soa, rnd, segments, params, stats, rrs, rrs_norm, split,
                                 queue, next_size, stream=0):
        arr = (Segment * len(segments))(*segments)
        return self._check(lib().nrrs_step_batched(
            self._h, C.byref(soa), _ptr(rnd), arr, len(segments), C.byref(params), _ptr(stats),
            _ptr(rrs), _ptr(rrs_norm), _ptr(split), _ptr(queue), _ptr(next_size), stream))

    # ---- device-resident queue sizes (n_dev: a device uint32 word; max_n: host bound) ----
    def inferDev(self, soa: VertexSoA, n_dev, max_n: int, params: DecideParams, stats, rrs,
                 stream=0):
        return self._check(lib().nrrs_infer_dev(self._h, C.byref(soa), _ptr(n_dev), max_n,
                                                C.byref(params), _ptr(stats), _ptr(rrs), stream))

    def decideEmitDev(self, rrs, rnd, n_dev, max_n, budget, n_specular, params, rrs_norm, split,
                      queue, capacity, next_size, scatter_index=None, n_specular_dev=None,
                      stream=0):
        return self._check(lib().nrrs_decide_emit_dev(
            self._h, _ptr(rrs), _ptr(rnd), _ptr(scatter_index), _ptr(n_dev), max_n, budget,
            n_specular, _ptr(n_specular_dev), C.byref(params), _ptr(rrs_norm), _ptr(split),
            _ptr(queue), capacity, _ptr(next_size), stream))

    def generateRRSNumberDev(self, soa, rnd, n_dev, max_n, budget, n_specular, params, stats,
                             rrs, rrs_norm, split, queue, capacity, next_size,
                             n_specular_dev=None, stream=0):
        return self._check(lib().nrrs_step_dev(
            self._h, C.byref(soa), _ptr(rnd), _ptr(n_dev), max_n, budget, n_specular,
            _ptr(n_specular_dev), C.byref(params), _ptr(stats), _ptr(rrs), _ptr(rrs_norm),
            _ptr(split), _ptr(queue), capacity, _ptr(next_size), stream))

    def generateRRSNumberBatchedDev(self, soa, rnd, segments, counts_dev, params, stats, rrs,
                                    rrs_norm, split, queue, next_size, stream=0):
        arr = (Segment * len(segments))(*segments)
        return self._check(lib().nrrs_step_batched_dev(
            self._h, C.byref(soa), _ptr(rnd), arr, _ptr(counts_dev), len(segments),
            C.byref(params), _ptr(stats), _ptr(rrs), _ptr(rrs_norm), _ptr(split), _ptr(queue),
            _ptr(next_size), stream))

    def trainStepBatch(self, batch: TrainBatch, n: int, sample_weight, error_sum_dev,
                       params: LossParams, loss_dev=None, stream=0):
        """nrrs_train_step_batch: NRRSNetwork::train on a training batch with the reference's
        per-sample loss inputs"""
        return self._check(lib().nrrs_train_step_batch(
            self._h, C.byref(batch), n, _ptr(sample_weight), _ptr(error_sum_dev),
            C.byref(params), _ptr(loss_dev), stream))

    def train(self, soa: VertexSoA, target, n: int, loss_dev=None, stream=0):
        return self._check(lib().nrrs_train_step(self._h, C.byref(soa), _ptr(target), n,
                                                 _ptr(loss_dev), stream))

    # ---- sharded (multi-GPU) building blocks ----
    def inferAccumulate(self, soa: VertexSoA, n: int, params: DecideParams, stats, rrs, sum_acc,
                        stream=0):
        return self._check(lib().nrrs_infer_accumulate(self._h, C.byref(soa), n, C.byref(params),
                                                       _ptr(stats), _ptr(rrs), _ptr(sum_acc),
                                                       stream))

    def decideEmitWithSum(self, rrs, rnd, n, budget, n_specular, sum_acc, params, rrs_norm, split,
                          queue, capacity, next_size, scatter_index=None, stream=0):
        return self._check(lib().nrrs_decide_emit_with_sum(
            self._h, _ptr(rrs), _ptr(rnd), _ptr(scatter_index), n, budget, n_specular,
            _ptr(sum_acc), C.byref(params), _ptr(rrs_norm), _ptr(split), _ptr(queue), capacity,
            _ptr(next_size), stream))

    def trainGrads(self, soa: VertexSoA, target, n: int, loss_dev=None, stream=0):
        return self._check(lib().nrrs_train_grads(self._h, C.byref(soa), _ptr(target), n,
                                                  _ptr(loss_dev), stream))

    def copyGrads(self, grads_dev, stream=0):
        return self._check(lib().nrrs_copy_grads(self._h, _ptr(grads_dev), stream))

    def adamApply(self, grads_dev, scale: float, stream=0):
        return self._check(lib().nrrs_adam_apply(self._h, _ptr(grads_dev), scale, stream))

    def saveWeights(self, path: str | os.PathLike):
        self._check(lib().nrrs_save(self._h, str(path).encode()))

    def loadWeights(self, path: str | os.PathLike):
        self._check(lib().nrrs_load(self._h, str(path).encode()))

    # ---- parameters ----
    def param_count(self) -> int:
        return int(lib().nrrs_param_count(self._h))

    def param_layout(self):
        t, s, r = C.c_uint64(), C.c_uint64(), C.c_uint64()
        self._check(lib().nrrs_param_layout(self._h, C.byref(t), C.byref(s), C.byref(r)))
        return int(t.value), int(s.value), int(r.value)

    def get_params(self):
        import numpy as np
        a = np.empty(self.param_count(), np.float32)
        self._check(lib().nrrs_get_params(self._h, a.ctypes.data, a.size))
        return a

    def get_inference_params(self):
        """the weights inference uses (the debiased moving average when ema_decay > 0)"""
        import numpy as np
        a = np.empty(self.param_count(), np.float32)
        self._check(lib().nrrs_get_inference_params(self._h, a.ctypes.data, a.size))
        return a

    def set_params(self, a):
        import numpy as np
        a = np.ascontiguousarray(a, dtype=np.float32)
        self._check(lib().nrrs_set_params(self._h, a.ctypes.data, a.size))

    def get_grads(self):
        import numpy as np
        a = np.empty(self.param_count(), np.float32)
        self._check(lib().nrrs_get_grads(self._h, a.ctypes.data, a.size))
        return a

    def get_adam_state(self):
        import numpy as np
        m = np.empty(self.param_count(), np.float32)
        v = np.empty_like(m)
        t = C.c_uint64()
        self._check(lib().nrrs_get_adam_state(self._h, m.ctypes.data, v.ctypes.data, m.size,
                                              C.byref(t)))
        return m, v, int(t.value)

    def level_table(self):
        import numpy as np
        a = np.zeros((self.config.n_levels, 4), np.uint32)
        self._check(lib().nrrs_level_table(self._h, a.ctypes.data, self.config.n_levels))
        return a

    # ---- launch shape, autotuning and graphs ----
    def autotune(self, n: int, cache_path=None) -> str:
        buf = C.create_string_buffer(8192)
        self._check(lib().nrrs_autotune(self._h, n, str(cache_path).encode() if cache_path else None,
                                        buf, len(buf)))
        return buf.value.decode()

    def set_launch_shape(self, ctas_per_sm: int, warpgroups: int = 1):
        self._check(lib().nrrs_set_launch_shape(self._h, ctas_per_sm, warpgroups))

    def set_infer_split(self, split: int):
        """0 = fused inference, 1 = level-major encoding kernel + MLP kernel (large tables),
        2 = encoding kernel + StatNet kernel + RRSNet kernel, 3 = as 2 with the hidden
        activations in TMEM."""
        self._check(lib().nrrs_set_infer_split(self._h, int(split)))

    def set_train_split(self, split: bool):
        """1 = level-major encoding, StatNet kernel, level-major scatter; 0 = one fused kernel."""
        self._check(lib().nrrs_set_train_split(self._h, int(bool(split))))

    def train_split(self) -> int:
        v = C.c_int32()
        self._check(lib().nrrs_get_train_split(self._h, C.byref(v)))
        return int(v.value)

    def infer_split(self) -> int:
        v = C.c_int32()
        self._check(lib().nrrs_get_infer_split(self._h, C.byref(v)))
        return int(v.value)

    def set_cell_image(self, enable: bool):
        """gathers of the dense levels from the cell image (one 32-byte load per cell) or from
        the table rows; bit-identical results"""
        self._check(lib().nrrs_set_cell_image(self._h, int(bool(enable))))

    def cell_image(self) -> bool:
        v = C.c_int32()
        self._check(lib().nrrs_get_cell_image(self._h, C.byref(v)))
        return bool(v.value)

    def launch_shape(self) -> tuple[int, int]:
        c, w = C.c_int32(), C.c_int32()
        self._check(lib().nrrs_get_launch_shape(self._h, C.byref(c), C.byref(w)))
        return int(c.value), int(w.value)

    def captureBatched(self, soa, rnd, segments, params, stats, rrs, rrs_norm, split, queue,
                       next_size) -> "BatchedGraph":
        arr = (Segment * len(segments))(*segments)
        g = C.c_void_p()
        self._check(lib().nrrs_graph_capture_batched(
            self._h, C.byref(soa), _ptr(rnd), arr, len(segments), C.byref(params), _ptr(stats),
            _ptr(rrs), _ptr(rrs_norm), _ptr(split), _ptr(queue), _ptr(next_size), C.byref(g)))
        return BatchedGraph(g)

    def last_infer_grid(self) -> int:
        return int(lib().nrrs_last_infer_grid(self._h))

    def launch_count(self) -> int:
        return int(lib().nrrs_launch_count(self._h))

    def profile(self, enable: bool = True):
        self._check(lib().nrrs_profile_enable(self._h, int(enable)))

    def profile_read(self) -> dict:
        """{kernel name: (launches, total ms)} of the launches timed since the last read"""
        out = {}
        for k, name in enumerate(KERNEL_KINDS):
            n, ms = C.c_uint64(), C.c_double()
            self._check(lib().nrrs_profile_read(self._h, k, C.byref(n), C.byref(ms)))
            if n.value:
                out[name] = (int(n.value), float(ms.value))
        return out

    def device_status(self, stream=0) -> tuple[int, int]:
        f = C.c_uint32()
        rc = lib().nrrs_get_device_status(self._h, C.byref(f), stream)
        return rc, int(f.value)
