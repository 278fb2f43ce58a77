"""ctypes binding of librgsplat_b200.so (the C ABI declared in include/rgsplat.h).

The library is built in-tree (``python -m rgsplat_b200.build``). There is no
fallback: if the shared library is missing or cannot be loaded, importing the
product API raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librgsplat_b200.so")

RGS_OK = 0
RGS_ERR_INVALID_ARG = -1
RGS_ERR_OOM = -2
RGS_ERR_CUDA = -3
RGS_ERR_NONFINITE = -4
RGS_ERR_SINGULAR_CAMERA = -5
RGS_ERR_CAPACITY = -6
RGS_ERR_NO_DEVICE = -7
RGS_ERR_IO = -8
RGS_ERR_FORMAT = -9

RGS_STEP_PLAIN = 0
RGS_STEP_BATCHED = 1
RGS_NUM_STAGES = 9
STAGE_NAMES = ("project", "depth_sort", "emit", "supertile_sort", "tile_lists", "forward", "loss", "backward", "geometry_adam")
RGS_PROJECT_WGSL = 0
RGS_PROJECT_CPU_MATH = 1
RGS_FB_RGBA_F32 = 0
RGS_FB_RGBA8_SRGB = 1

ERROR_NAMES = {
    RGS_ERR_INVALID_ARG: "invalid argument",
    RGS_ERR_OOM: "out of device memory",
    RGS_ERR_CUDA: "CUDA error",
    RGS_ERR_NONFINITE: "non-finite parameter",
    RGS_ERR_SINGULAR_CAMERA: "singular camera",
    RGS_ERR_CAPACITY: "capacity exceeded",
    RGS_ERR_NO_DEVICE: "no CUDA device",
    RGS_ERR_IO: "file error",
    RGS_ERR_FORMAT: "unsupported model file",
}


class rgs_camera(C.Structure):
    _fields_ = [
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("fx", C.c_float),
        ("fy", C.c_float),
        ("cx", C.c_float),
        ("cy", C.c_float),
        ("c2w", C.c_float * 16),
        ("distortion", C.c_float * 3),
    ]


class rgs_loss_config(C.Structure):
    _fields_ = [("lambda_dssim", C.c_float)]


class rgs_train_config(C.Structure):
    _fields_ = [
        ("num_iterations", C.c_uint64),
        ("lr_position", C.c_float),
        ("lr_rotation", C.c_float),
        ("lr_scale", C.c_float),
        ("lr_opacity", C.c_float),
        ("lr_sh_dc", C.c_float),
        ("lr_sh_rest", C.c_float),
        ("beta1", C.c_float),
        ("beta2", C.c_float),
        ("eps", C.c_float),
        ("densify_from_iter", C.c_uint64),
        ("densify_until_iter", C.c_uint64),
        ("densify_grad_threshold", C.c_float),
        ("opacity_reset_iter", C.c_uint64),
        ("prune_opacity_thresh", C.c_float),
        ("max_gaussians", C.c_uint64),
    ]


class rgs_splat_info_2d(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("sx", "sy", "conic_a", "conic_b", "conic_c", "color_r", "color_g", "color_b", "alpha", "depth")]


class rgs_adam_state(C.Structure):
    _fields_ = [
        ("m1", C.POINTER(C.c_float)),
        ("m2", C.POINTER(C.c_float)),
        ("grad_accum", C.POINTER(C.c_float)),
        ("grad_denom", C.POINTER(C.c_uint32)),
        ("len", C.c_size_t),
        ("t", C.c_uint64),
    ]


class rgs_options(C.Structure):
    _fields_ = [
        ("device", C.c_int),
        ("tile_w", C.c_int),
        ("tile_h", C.c_int),
        ("batch", C.c_int),
        ("reference_compat", C.c_int),
        ("pixels_per_thread", C.c_int),
        ("batch_pair_limit", C.c_uint64),
        ("exact_loss", C.c_int),
    ]


class rgs_stats(C.Structure):
    _fields_ = [
        ("pairs", C.c_uint64),
        ("visible", C.c_uint64),
        ("pair_capacity", C.c_uint64),
        ("graph_captures", C.c_uint32),
        ("overflow_retries", C.c_uint32),
        ("view_groups", C.c_uint32),
        ("reserved", C.c_uint32),
        ("supertile_entries", C.c_uint64),
    ]


class rgs_tune_entry(C.Structure):
    _fields_ = [
        ("tile_w", C.c_int),
        ("tile_h", C.c_int),
        ("batch", C.c_int),
        ("pixels_per_thread", C.c_int),
        ("ms", C.c_float),
    ]


RGS_TUNE_CANDIDATES = 18
RGS_BACKWARD_RECOMPUTE = 0
RGS_BACKWARD_STORE_ALL = 1


class rgs_backward_report(C.Structure):
    _fields_ = [
        ("forward_ms", C.c_float),
        ("backward_ms", C.c_float),
        ("state_bytes", C.c_uint64),
        ("pairs", C.c_uint64),
    ]


_lib = None

FP = C.POINTER(C.c_float)
U32P = C.POINTER(C.c_uint32)
CTX = C.c_void_p

# name -> (restype, argtypes); mirrors include/rgsplat.h
SIGNATURES = {
    "rgs_options_default": (None, [C.POINTER(rgs_options)]),
    "rgs_train_config_default": (None, [C.POINTER(rgs_train_config)]),
    "rgs_create": (C.c_int, [C.POINTER(rgs_options), C.POINTER(C.c_void_p)]),
    "rgs_destroy": (None, [CTX]),
    "rgs_last_error": (C.c_char_p, [CTX]),
    "rgs_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "rgs_synchronize": (C.c_int, [CTX]),
    "rgs_render_and_backward": (C.c_int, [CTX, FP, C.c_size_t, C.POINTER(rgs_camera), FP, FP, C.POINTER(rgs_loss_config), FP, FP]),
    "rgs_render_and_backward_variant": (C.c_int, [CTX, FP, C.c_size_t, C.POINTER(rgs_camera), FP, FP, C.POINTER(rgs_loss_config),
                                                  C.c_int, FP, FP, C.POINTER(rgs_backward_report)]),
    "rgs_trainer_rasterize": (C.c_int, [CTX, C.c_uint32, FP, C.c_int, C.c_void_p]),
    "rgs_rasterize": (C.c_int, [CTX, FP, C.c_size_t, C.POINTER(rgs_camera), FP, C.c_int, C.c_void_p]),
    "rgs_render_color": (C.c_int, [CTX, FP, C.c_size_t, C.POINTER(rgs_camera), FP, FP]),
    "rgs_photometric_loss_grad": (C.c_int, [CTX, FP, FP, C.c_uint32, C.c_uint32, C.c_float, FP, FP]),
    "rgs_photometric_loss_grad_noalloc": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_float,
                                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_size_t]),
    "rgs_adam_step": (C.c_int, [CTX, FP, C.c_size_t, FP, C.POINTER(rgs_adam_state), C.POINTER(rgs_train_config)]),
    "rgs_densify_and_prune": (C.c_int, [CTX, FP, C.c_size_t, FP, U32P, C.POINTER(rgs_train_config), C.c_float, FP, C.c_size_t, C.POINTER(C.c_size_t)]),
    "rgs_reset_opacities": (C.c_int, [CTX, FP, C.c_size_t]),
    "rgs_project": (C.c_int, [CTX, FP, C.c_size_t, C.POINTER(rgs_camera), C.c_int, C.POINTER(rgs_splat_info_2d), U32P]),
    "rgs_gpu_render": (C.c_int, [CTX, FP, C.c_size_t, C.POINTER(rgs_camera), C.c_int, FP, FP]),
    "rgs_save_ply": (C.c_int, [CTX, FP, C.c_size_t, C.c_char_p]),
    "rgs_save_splat": (C.c_int, [CTX, FP, C.c_size_t, C.c_char_p]),
    "rgs_load_ply": (C.c_int, [CTX, C.c_char_p, FP, C.c_size_t, C.POINTER(C.c_size_t)]),
    "rgs_gaussians_from_sfm": (C.c_int, [CTX, C.c_void_p, C.c_void_p, C.c_size_t, FP]),
    "rgs_trainer_init_from_sfm": (C.c_int, [CTX, C.c_void_p, C.c_void_p, C.c_size_t]),
    "rgs_read_points3d_bin": (C.c_int, [CTX, C.c_char_p, C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "rgs_srgb8_to_linear": (C.c_int, [CTX, C.c_void_p, C.c_size_t, FP]),
    "rgs_trainer_set_target_rgba8": (C.c_int, [CTX, C.c_size_t, C.c_void_p]),
    "rgs_trainer_save_ply": (C.c_int, [CTX, C.c_char_p]),
    "rgs_trainer_save_splat": (C.c_int, [CTX, C.c_char_p]),
    "rgs_trainer_load_ply": (C.c_int, [CTX, C.c_char_p, C.POINTER(C.c_size_t)]),
    "rgs_trainer_set_gaussians": (C.c_int, [CTX, FP, C.c_size_t]),
    "rgs_trainer_count": (C.c_int, [CTX, C.POINTER(C.c_size_t)]),
    "rgs_trainer_get_gaussians": (C.c_int, [CTX, FP, C.c_size_t, C.POINTER(C.c_size_t)]),
    "rgs_trainer_set_cameras": (C.c_int, [CTX, C.POINTER(rgs_camera), C.c_size_t]),
    "rgs_trainer_set_target": (C.c_int, [CTX, C.c_size_t, FP]),
    "rgs_trainer_step": (C.c_int, [CTX, U32P, C.c_size_t, FP, C.POINTER(rgs_loss_config), C.POINTER(rgs_train_config), C.c_int, FP]),
    "rgs_trainer_step_host_targets": (C.c_int, [CTX, U32P, C.c_size_t, C.POINTER(C.c_void_p), FP, C.POINTER(rgs_loss_config),
                                                C.POINTER(rgs_train_config), FP]),
    "rgs_trainer_backward": (C.c_int, [CTX, U32P, C.c_size_t, FP, C.POINTER(rgs_loss_config), C.c_int, FP]),
    "rgs_trainer_get_grads": (C.c_int, [CTX, FP]),
    "rgs_trainer_grad_buffer": (C.c_int, [CTX, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "rgs_trainer_apply_adam": (C.c_int, [CTX, C.POINTER(rgs_train_config), C.c_uint32]),
    "rgs_trainer_render": (C.c_int, [CTX, C.c_uint32, FP, FP]),
    "rgs_trainer_densify_and_prune": (C.c_int, [CTX, C.POINTER(rgs_train_config), C.c_float, C.POINTER(C.c_size_t)]),
    "rgs_trainer_reset_opacities": (C.c_int, [CTX]),
    "rgs_trainer_get_adam_state": (C.c_int, [CTX, C.POINTER(rgs_adam_state)]),
    "rgs_trainer_set_adam_state": (C.c_int, [CTX, C.POINTER(rgs_adam_state)]),
    "rgs_get_memory": (C.c_int, [CTX, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.c_int]),
    "rgs_trainer_evaluated_pairs": (C.c_int, [CTX, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "rgs_get_stats": (C.c_int, [CTX, C.POINTER(rgs_stats)]),
    "rgs_get_options": (C.c_int, [CTX, C.POINTER(rgs_options)]),
    "rgs_set_tiling": (C.c_int, [CTX, C.c_int, C.c_int, C.c_int, C.c_int]),
    "rgs_trainer_autotune": (C.c_int, [CTX, U32P, C.c_size_t, FP, C.POINTER(rgs_loss_config), C.c_int,
                                       C.POINTER(rgs_tune_entry), C.POINTER(rgs_options)]),
    "rgs_set_stream": (C.c_int, [CTX, C.c_void_p]),
    "rgs_set_profiling": (C.c_int, [CTX, C.c_int]),
    "rgs_get_stage_times": (C.c_int, [CTX, FP, C.c_int]),
    # include/rgsplat_debug.h
    "rgs_debug_project": (C.c_int, [CTX, FP, C.c_size_t, C.POINTER(rgs_camera), C.POINTER(C.c_int32), FP, C.POINTER(C.c_int32)]),
    "rgs_debug_tile_lists": (C.c_int, [CTX, FP, C.c_size_t, C.POINTER(rgs_camera), C.POINTER(C.c_uint64), C.POINTER(C.c_int32),
                                       C.POINTER(C.c_int32), C.c_size_t]),
    "rgs_debug_pruned_tile_lists": (C.c_int, [CTX, FP, C.c_size_t, C.POINTER(rgs_camera), C.POINTER(C.c_uint64),
                                              C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_size_t]),
    "rgs_debug_forward": (C.c_int, [CTX, FP, C.c_size_t, C.POINTER(rgs_camera), FP, FP, FP, C.POINTER(C.c_int32)]),
    "rgs_debug_backward": (C.c_int, [CTX, FP, C.c_size_t, C.POINTER(rgs_camera), FP, FP, C.c_float, FP, FP]),
    "rgs_debug_trainer_batch_pixels": (C.c_int, [CTX, C.c_size_t, FP, FP, FP]),
    "rgs_debug_exp_sfu_error": (C.c_int, [CTX, C.c_float, C.c_float, C.c_uint32, FP]),
}


def load() -> C.CDLL:
    """Load the in-tree library; raises if it is missing (no fallback path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m rgsplat_b200.build`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
