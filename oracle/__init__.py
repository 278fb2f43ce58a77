"""CPU oracle for rgsplat's differentiable training path (TEST INFRASTRUCTURE ONLY).

This package is the checker for the CUDA library in ``rgsplat_b200``: only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may
import it. It wraps ``oracle/_build/liboracle.so`` (a C++ restatement of the
reference's ``src/math``, ``src/cpu/backward.rs`` and
``src/pipeline/optimizer.rs``; see ``oracle/oracle.hpp`` for the per-function
citations) with numpy-friendly helpers.

Array conventions follow the reference crate:
  * Gaussians: ``(N, 59)`` float32, the ``Gaussian3D`` record
    (position[3], opacity_logit, rotation[4] wxyz, log_scale[3], sh[48]);
  * gradients: ``(N, 60)`` float32, the ``GaussianGrad`` record
    (d_position[3], d_rotation[4], d_log_scale[3], d_opacity_logit, d_sh[48],
    screen_grad_norm);
  * images: interleaved RGB ``(H, W, 3)``; targets interleaved RGBA ``(H, W, 4)``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_SOURCES = ("capi.cpp", "oracle.hpp", "fmath.hpp", "Makefile")


def build(force: bool = False) -> str:
    """Compile the oracle with make if it is missing or older than its sources."""
    newest = max(os.path.getmtime(os.path.join(_HERE, s)) for s in _SOURCES)
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < newest:
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class CameraStruct(C.Structure):
    """Mirror of ``Camera`` (src/math/mod.rs:131-145); ``c2w`` row-major."""

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


class TrainConfigStruct(C.Structure):
    """Mirror of ``TrainConfig`` (src/pipeline/optimizer.rs:22-40)."""

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


@dataclass
class Camera:
    """Pinhole camera (src/math/mod.rs:131-145)."""

    width: int
    height: int
    fx: float
    fy: float
    cx: float
    cy: float
    c2w: np.ndarray  # (4, 4) row-major camera-to-world

    def struct(self) -> CameraStruct:
        s = CameraStruct()
        s.width, s.height = int(self.width), int(self.height)
        s.fx, s.fy, s.cx, s.cy = float(self.fx), float(self.fy), float(self.cx), float(self.cy)
        flat = np.ascontiguousarray(self.c2w, dtype=np.float32).reshape(16)
        for i in range(16):
            s.c2w[i] = float(flat[i])
        return s


def identity_camera(w: int, h: int) -> Camera:
    """The reference tests' camera: origin, looking down +z (backward.rs:828-846)."""
    return Camera(w, h, float(w), float(w), w / 2.0, h / 2.0, np.eye(4, dtype=np.float32))


@dataclass
class TrainConfig:
    """``TrainConfig::default()`` (src/pipeline/optimizer.rs:42-62)."""

    num_iterations: int = 30_000
    lr_position: float = 0.00016
    lr_rotation: float = 0.001
    lr_scale: float = 0.005
    lr_opacity: float = 0.05
    lr_sh_dc: float = 0.0025
    lr_sh_rest: float = 0.000125
    beta1: float = 0.9
    beta2: float = 0.999
    eps: float = 1e-8
    densify_from_iter: int = 500
    densify_until_iter: int = 15_000
    densify_grad_threshold: float = 0.0002
    opacity_reset_iter: int = 3000
    prune_opacity_thresh: float = 0.005
    max_gaussians: int = 3_000_000

    def struct(self) -> TrainConfigStruct:
        s = TrainConfigStruct()
        for name, _ in TrainConfigStruct._fields_:
            setattr(s, name, getattr(self, name))
        return s


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        _declare(_lib)
    return _lib


def _declare(L: C.CDLL) -> None:
    fp = C.POINTER(C.c_float)
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int32)
    up = C.POINTER(C.c_uint32)
    cam = C.POINTER(CameraStruct)
    sz = C.c_size_t
    L.orc_set_threads.argtypes = [C.c_int]
    L.orc_set_threads.restype = C.c_int
    L.orc_set_libm_math.argtypes = [C.c_int]
    L.orc_expf.argtypes = [C.c_float]
    L.orc_expf.restype = C.c_float
    L.orc_logf.argtypes = [C.c_float]
    L.orc_logf.restype = C.c_float
    L.orc_expf_array.argtypes = [fp, fp, sz]
    L.orc_expf_fast_array.argtypes = [fp, fp, sz]
    L.orc_logf_array.argtypes = [fp, fp, sz]
    L.orc_sigmoid_f.argtypes = [C.c_float]
    L.orc_sigmoid_f.restype = C.c_float
    L.orc_logit_f.argtypes = [C.c_float]
    L.orc_logit_f.restype = C.c_float
    L.orc_render_and_backward_f.argtypes = [fp, sz, cam, fp, fp, C.c_float, fp, fp, fp, fp, ip, fp, fp]
    L.orc_render_and_backward_d.argtypes = [dp, sz, cam, dp, dp, C.c_double, dp, dp, dp, dp, ip, dp, dp]
    L.orc_render_color_f.argtypes = [fp, sz, cam, fp, fp, fp, ip]
    L.orc_rasterize_f.argtypes = [fp, sz, cam, fp, fp]
    L.orc_to_u8_srgb.argtypes = [fp, sz, C.POINTER(C.c_uint8)]
    L.orc_linear_to_srgb.argtypes = [fp, sz, fp]
    L.orc_srgb8_to_linear.argtypes = [C.POINTER(C.c_uint8), sz, fp]
    dp = C.POINTER(C.c_double)
    L.orc_gaussians_from_sfm.argtypes = [dp, C.POINTER(C.c_uint8), sz, fp]
    L.orc_sfm_scales.argtypes = [dp, sz, fp]
    L.orc_rust_binary_search.argtypes = [dp, sz, C.c_double, C.POINTER(C.c_int)]
    L.orc_rust_binary_search.restype = C.c_long
    L.orc_parse_points3d_bin.argtypes = [C.POINTER(C.c_uint8), sz, dp, C.POINTER(C.c_uint8), sz, C.POINTER(C.c_size_t)]
    u8p = C.POINTER(C.c_uint8)
    L.orc_save_ply.argtypes = [fp, sz, u8p, sz]
    L.orc_save_ply.restype = C.c_long
    L.orc_save_splat.argtypes = [fp, sz, u8p, sz]
    L.orc_save_splat.restype = C.c_long
    L.orc_load_ply.argtypes = [u8p, sz, fp, sz, C.POINTER(C.c_size_t)]
    L.orc_photometric_loss_grad_f.argtypes = [fp, fp, C.c_int, C.c_int, C.c_float, fp, fp]
    L.orc_photometric_loss_grad_d.argtypes = [dp, dp, C.c_int, C.c_int, C.c_double, dp, dp]
    L.orc_project_f.argtypes = [fp, sz, cam, ip, fp, ip]
    L.orc_bin_f.argtypes = [fp, sz, cam, C.POINTER(C.c_int64), ip, ip, C.c_int64]
    L.orc_adam_step_f.argtypes = [fp, sz, fp, fp, fp, fp, up, C.POINTER(C.c_uint64), C.POINTER(TrainConfigStruct)]
    L.orc_densify_and_prune_f.argtypes = [fp, sz, fp, fp, up, C.POINTER(TrainConfigStruct), C.c_float]
    L.orc_densify_and_prune_f.restype = C.c_int64
    L.orc_reset_opacities_f.argtypes = [fp, sz]
    L.orc_estimate_scene_extent_f.argtypes = [fp, sz]
    L.orc_estimate_scene_extent_f.restype = C.c_float
    L.orc_project_wgsl_f.argtypes = [fp, sz, cam, fp, up]
    L.orc_composite_f.argtypes = [fp, sz, C.c_int, C.c_int, fp, fp]
    L.orc_mat_from_quat_f.argtypes = [fp, fp]
    L.orc_to_rotation_matrix_f.argtypes = [fp, fp]
    L.orc_quat_normalize_f.argtypes = [fp, fp]
    L.orc_rotation_jacobian_f.argtypes = [fp, fp]
    L.orc_build_cov3d_f.argtypes = [fp, fp, fp]
    L.orc_backprop_cov3d_f.argtypes = [fp, fp, fp, fp, fp]
    L.orc_sh_basis_f.argtypes = [fp, fp]
    L.orc_sh_basis_grad_f.argtypes = [fp, fp]
    L.orc_eval_sh_deg3_f.argtypes = [fp, fp, fp]
    L.orc_ssim_channel_f.argtypes = [fp, fp, C.c_int, C.c_int, fp]
    L.orc_ssim_channel_f.restype = C.c_float
    L.orc_gaussian_kernel_1d_f.argtypes = [C.c_int, C.c_float, fp]


def _f(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _d(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _i(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _u(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def camera_struct(c) -> CameraStruct:
    """CameraStruct from any object with width, height, fx, fy, cx, cy, c2w."""
    s = CameraStruct()
    s.width, s.height = int(c.width), int(c.height)
    s.fx, s.fy, s.cx, s.cy = float(c.fx), float(c.fy), float(c.cx), float(c.cy)
    flat = np.ascontiguousarray(c.c2w, dtype=np.float32).reshape(16)
    for i in range(16):
        s.c2w[i] = float(flat[i])
    return s


def set_threads(n: int) -> int:
    return lib().orc_set_threads(int(n))


def set_libm_math(on: bool) -> None:
    lib().orc_set_libm_math(1 if on else 0)


class OracleError(RuntimeError):
    pass


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise OracleError(f"{what} failed with status {rc}")


@dataclass
class RenderOut:
    loss: float
    grads: np.ndarray       # (N, 60)
    rendered: np.ndarray    # (H, W, 3)
    final_t: np.ndarray     # (H, W)
    last_contrib: np.ndarray  # (H, W) int32
    dl_dpix: np.ndarray     # (H, W, 3)
    acc: np.ndarray         # (N, 9) per-Gaussian blend accumulators


def render_and_backward(gaussians, camera: Camera, target_rgba, bg=(0.0, 0.0, 0.0), lambda_dssim=0.2, double=False) -> RenderOut:
    """``render_and_backward`` (src/cpu/backward.rs:107-149) plus its cached intermediates."""
    dt = np.float64 if double else np.float32
    g = np.ascontiguousarray(gaussians, dtype=dt).reshape(-1, 59)
    n = g.shape[0]
    w, h = camera.width, camera.height
    tgt = np.ascontiguousarray(target_rgba, dtype=dt).reshape(h, w, 4)
    bgv = np.asarray(bg, dtype=dt)
    loss = np.zeros(1, dt)
    grads = np.zeros((n, 60), dt)
    rendered = np.zeros((h, w, 3), dt)
    final_t = np.zeros((h, w), dt)
    last = np.zeros((h, w), np.int32)
    dl = np.zeros((h, w, 3), dt)
    acc = np.zeros((n, 9), dt)
    cs = camera_struct(camera)
    if double:
        rc = lib().orc_render_and_backward_d(_d(g), n, C.byref(cs), _d(tgt), _d(bgv), float(lambda_dssim), _d(loss), _d(grads), _d(rendered), _d(final_t), _i(last), _d(dl), _d(acc))
    else:
        rc = lib().orc_render_and_backward_f(_f(g), n, C.byref(cs), _f(tgt), _f(bgv), float(lambda_dssim), _f(loss), _f(grads), _f(rendered), _f(final_t), _i(last), _f(dl), _f(acc))
    _check(rc, "render_and_backward")
    return RenderOut(float(loss[0]), grads, rendered, final_t, last, dl, acc)


def render_color(gaussians, camera: Camera, bg=(0.0, 0.0, 0.0)):
    """``render_color`` (src/cpu/backward.rs:152-166) -> (rgb, final_t, last_contrib)."""
    g = f32(gaussians).reshape(-1, 59)
    w, h = camera.width, camera.height
    rgb = np.zeros((h, w, 3), np.float32)
    ft = np.zeros((h, w), np.float32)
    lc = np.zeros((h, w), np.int32)
    bgv = f32(bg)
    cs = camera_struct(camera)
    _check(lib().orc_render_color_f(_f(g), g.shape[0], C.byref(cs), _f(bgv), _f(rgb), _f(ft), _i(lc)), "render_color")
    return rgb, ft, lc


def rasterize(gaussians, camera: Camera, bg=(0.0, 0.0, 0.0)) -> np.ndarray:
    """``cpu::rasterize`` (src/cpu/rasterizer.rs:72-192) -> Framebuffer RGBA (H, W, 4)."""
    g = f32(gaussians).reshape(-1, 59)
    rgba = np.zeros((camera.height, camera.width, 4), np.float32)
    cs = camera_struct(camera)
    _check(lib().orc_rasterize_f(_f(g), g.shape[0], C.byref(cs), _f(f32(bg)), _f(rgba)), "rasterize")
    return rgba


def linear_to_srgb(x) -> np.ndarray:
    """``linear_to_srgb`` (src/cpu/rasterizer.rs:262-269)."""
    a = f32(np.atleast_1d(x))
    out = np.zeros_like(a)
    _check(lib().orc_linear_to_srgb(_f(a), a.size, _f(out)), "linear_to_srgb")
    return out


def _encode(fn, gaussians) -> bytes:
    g = f32(gaussians).reshape(-1, 59)
    size = fn(_f(g), g.shape[0], None, 0)
    buf = np.zeros(size, np.uint8)
    fn(_f(g), g.shape[0], buf.ctypes.data_as(C.POINTER(C.c_uint8)), size)
    return buf.tobytes()


def save_ply_bytes(gaussians) -> bytes:
    """``io::ply::save_ply`` (src/io/ply.rs:35-104) as the file's bytes."""
    return _encode(lib().orc_save_ply, gaussians)


def save_splat_bytes(gaussians) -> bytes:
    """``io::ply::save_splat`` (src/io/ply.rs:253-285) as the file's bytes."""
    return _encode(lib().orc_save_splat, gaussians)


def load_ply_bytes(data: bytes) -> np.ndarray:
    """``io::ply::load_ply`` (src/io/ply.rs:116-193) of a file's bytes -> (N, 59)."""
    buf = np.frombuffer(data, np.uint8)
    n = C.c_size_t(0)
    p = buf.ctypes.data_as(C.POINTER(C.c_uint8))
    _check(lib().orc_load_ply(p, buf.size, None, 0, C.byref(n)), "load_ply")
    out = np.zeros((n.value, 59), np.float32)
    _check(lib().orc_load_ply(p, buf.size, _f(out), n.value, C.byref(n)), "load_ply")
    return out


def srgb8_to_linear(rgba8) -> np.ndarray:
    """``load_target``'s conversion (src/io/images.rs:67-72): RGBA8 -> linear RGBA f32."""
    a = np.ascontiguousarray(rgba8, np.uint8)
    out = np.zeros(a.shape, np.float32)
    _check(lib().orc_srgb8_to_linear(a.ctypes.data_as(C.POINTER(C.c_uint8)), a.size // 4, _f(out)), "srgb8_to_linear")
    return out


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def gaussians_from_sfm(xyz, rgb) -> np.ndarray:
    """``gaussians_from_sfm`` (src/pipeline/sfm.rs:365-404): (N, 3) f64 points and
    (N, 3) u8 colours -> (N, 59) Gaussians."""
    x = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
    c = np.ascontiguousarray(rgb, np.uint8).reshape(-1, 3)
    if x.shape[0] != c.shape[0]:
        raise ValueError("xyz and rgb hold different point counts")
    out = np.zeros((x.shape[0], 59), np.float32)
    _check(lib().orc_gaussians_from_sfm(_dp(x), c.ctypes.data_as(C.POINTER(C.c_uint8)), x.shape[0], _f(out)),
           "gaussians_from_sfm")
    return out


def sfm_scales(xyz) -> np.ndarray:
    """``estimate_initial_scales`` (src/pipeline/sfm.rs:408-450) -> (N,) f32."""
    x = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
    out = np.zeros(x.shape[0], np.float32)
    _check(lib().orc_sfm_scales(_dp(x), x.shape[0], _f(out)), "sfm_scales")
    return out


def rust_binary_search(xs, t: float):
    """Rust's slice::binary_search_by on sorted f64 keys -> ("ok" | "err", index)."""
    a = np.ascontiguousarray(xs, np.float64)
    ok = C.c_int(0)
    r = lib().orc_rust_binary_search(_dp(a), a.size, float(t), C.byref(ok))
    return ("ok" if ok.value else "err", int(r))


def parse_points3d_bin(data: bytes):
    """``parse_points3d_bin`` (src/pipeline/sfm.rs:147-183) -> (xyz (N, 3) f64, rgb (N, 3) u8)."""
    buf = np.frombuffer(data, np.uint8)
    p = buf.ctypes.data_as(C.POINTER(C.c_uint8))
    n = C.c_size_t(0)
    _check(lib().orc_parse_points3d_bin(p, buf.size, None, None, 0, C.byref(n)), "parse_points3d_bin")
    xyz = np.zeros((n.value, 3), np.float64)
    rgb = np.zeros((n.value, 3), np.uint8)
    _check(lib().orc_parse_points3d_bin(p, buf.size, _dp(xyz), rgb.ctypes.data_as(C.POINTER(C.c_uint8)), n.value,
                                        C.byref(n)), "parse_points3d_bin")
    return xyz, rgb


def to_u8_srgb(rgba) -> np.ndarray:
    """``Framebuffer::to_u8_srgb`` (src/cpu/rasterizer.rs:38-48)."""
    a = f32(rgba)
    out = np.zeros(a.shape, np.uint8)
    _check(lib().orc_to_u8_srgb(_f(a), a.size, out.ctypes.data_as(C.POINTER(C.c_uint8))), "to_u8_srgb")
    return out


def photometric_loss_grad(rendered, target_rgba, w: int, h: int, lam: float, double=False):
    """``photometric_loss_grad`` (src/cpu/backward.rs:646-693)."""
    dt = np.float64 if double else np.float32
    r = np.ascontiguousarray(rendered, dtype=dt).reshape(-1)
    t = np.ascontiguousarray(target_rgba, dtype=dt).reshape(-1)
    loss = np.zeros(1, dt)
    dl = np.zeros(w * h * 3, dt)
    if double:
        rc = lib().orc_photometric_loss_grad_d(_d(r), _d(t), w, h, float(lam), _d(loss), _d(dl))
    else:
        rc = lib().orc_photometric_loss_grad_f(_f(r), _f(t), w, h, float(lam), _f(loss), _f(dl))
    _check(rc, "photometric_loss_grad")
    return float(loss[0]), dl


def project(gaussians, camera: Camera):
    """Per-Gaussian ``project`` (backward.rs:210-280): (visible, rec(N,16), tile_rect(N,4))."""
    g = f32(gaussians).reshape(-1, 59)
    n = g.shape[0]
    vis = np.zeros(n, np.int32)
    rec = np.zeros((n, 16), np.float32)
    rect = np.zeros((n, 4), np.int32)
    cs = camera_struct(camera)
    _check(lib().orc_project_f(_f(g), n, C.byref(cs), _i(vis), _f(rec), _i(rect)), "project")
    return vis, rec, rect


def tile_lists(gaussians, camera: Camera):
    """Tile lists of ``project_and_bin`` (backward.rs:172-208) as CSR of Gaussian indices."""
    g = f32(gaussians).reshape(-1, 59)
    n = g.shape[0]
    cs = camera_struct(camera)
    total = C.c_int64(0)
    L = lib()
    _check(L.orc_bin_f(_f(g), n, C.byref(cs), C.byref(total), None, None, 0), "bin")
    ntiles = ((camera.width + 15) // 16) * ((camera.height + 15) // 16)
    offs = np.zeros(ntiles + 1, np.int32)
    ent = np.zeros(max(total.value, 1), np.int32)
    _check(L.orc_bin_f(_f(g), n, C.byref(cs), C.byref(total), _i(offs), _i(ent), ent.shape[0]), "bin")
    return offs, ent[: total.value]


class AdamState:
    """``AdamState`` (src/pipeline/optimizer.rs:74-106); arrays grow, never shrink."""

    def __init__(self, n: int):
        self.m1 = np.zeros(n * 59, np.float32)
        self.m2 = np.zeros(n * 59, np.float32)
        self.grad_accum = np.zeros(n, np.float32)
        self.grad_denom = np.zeros(n, np.uint32)
        self.t = 0

    def resize(self, new_n: int) -> None:
        old_n = self.m1.shape[0] // 59
        if new_n > old_n:
            self.m1 = np.concatenate([self.m1, np.zeros((new_n - old_n) * 59, np.float32)])
            self.m2 = np.concatenate([self.m2, np.zeros((new_n - old_n) * 59, np.float32)])
            self.grad_accum = np.concatenate([self.grad_accum, np.zeros(new_n - old_n, np.float32)])
            self.grad_denom = np.concatenate([self.grad_denom, np.zeros(new_n - old_n, np.uint32)])


def adam_step(gaussians: np.ndarray, grads, state: AdamState, cfg: TrainConfig) -> None:
    """``adam_step`` (src/pipeline/optimizer.rs:116-163), in place on ``gaussians``."""
    assert gaussians.dtype == np.float32 and gaussians.flags.c_contiguous
    n = gaussians.reshape(-1, 59).shape[0]
    gr = f32(grads).reshape(-1, 60)
    t = C.c_uint64(state.t)
    cs = cfg.struct()
    _check(lib().orc_adam_step_f(_f(gaussians), n, _f(gr), _f(state.m1), _f(state.m2), _f(state.grad_accum), _u(state.grad_denom), C.byref(t), C.byref(cs)), "adam_step")
    state.t = t.value


def densify_and_prune(gaussians: np.ndarray, state: AdamState, cfg: TrainConfig, scene_extent: float) -> np.ndarray:
    """``densify_and_prune`` (src/pipeline/optimizer.rs:206-272); returns the new array."""
    g = f32(gaussians).reshape(-1, 59)
    n = g.shape[0]
    out = np.zeros((3 * n + 1, 59), np.float32)
    cs = cfg.struct()
    k = lib().orc_densify_and_prune_f(_f(g), n, _f(out), _f(state.grad_accum), _u(state.grad_denom), C.byref(cs), float(scene_extent))
    out = np.ascontiguousarray(out[:k])
    state.resize(k)
    state.grad_accum[:] = 0
    state.grad_denom[:] = 0
    return out


def reset_opacities(gaussians: np.ndarray) -> None:
    """``reset_opacities`` (src/pipeline/optimizer.rs:314-319), in place."""
    assert gaussians.dtype == np.float32 and gaussians.flags.c_contiguous
    lib().orc_reset_opacities_f(_f(gaussians), gaussians.reshape(-1, 59).shape[0])


def estimate_scene_extent(gaussians) -> float:
    g = f32(gaussians).reshape(-1, 59)
    return float(lib().orc_estimate_scene_extent_f(_f(g), g.shape[0]))


def project_wgsl(gaussians, camera: Camera):
    """The WGSL ``project`` pass (src/gpu/splat.wgsl:119-191): (SplatInfo2D (N,10), keys (N,))."""
    g = f32(gaussians).reshape(-1, 59)
    n = g.shape[0]
    sp = np.zeros((n, 10), np.float32)
    keys = np.zeros(n, np.uint32)
    cs = camera_struct(camera)
    _check(lib().orc_project_wgsl_f(_f(g), n, C.byref(cs), _f(sp), _u(keys)), "project_wgsl")
    return sp, keys


def composite(splats10, w: int, h: int, bg=(0.0, 0.0, 0.0)) -> np.ndarray:
    """CPU compositor of ``GpuRenderer::render`` (src/gpu/compute.rs:243-296)."""
    sp = f32(splats10).reshape(-1, 10)
    out = np.zeros((h, w, 3), np.float32)
    lib().orc_composite_f(_f(sp), sp.shape[0], w, h, _f(f32(bg)), _f(out))
    return out


# --- small math helpers used by the ported unit tests -----------------------

def expf(x: float) -> float:
    return float(lib().orc_expf(float(x)))


def logf(x: float) -> float:
    return float(lib().orc_logf(float(x)))


def expf_array(x) -> np.ndarray:
    a = f32(x).reshape(-1)
    y = np.empty_like(a)
    lib().orc_expf_array(_f(a), _f(y), a.shape[0])
    return y


def expf_fast_array(x) -> np.ndarray:
    a = f32(x).reshape(-1)
    y = np.empty_like(a)
    lib().orc_expf_fast_array(_f(a), _f(y), a.shape[0])
    return y


def logf_array(x) -> np.ndarray:
    a = f32(x).reshape(-1)
    y = np.empty_like(a)
    lib().orc_logf_array(_f(a), _f(y), a.shape[0])
    return y


def sigmoid(x: float) -> float:
    return float(lib().orc_sigmoid_f(float(x)))


def logit(p: float) -> float:
    return float(lib().orc_logit_f(float(p)))


def _mat(fn, *vecs, out_shape=(3, 3)):
    args = [f32(v) for v in vecs]
    out = np.zeros(int(np.prod(out_shape)), np.float32)
    fn(*[_f(a) for a in args], _f(out))
    return out.reshape(out_shape)


def mat_from_quat_components(q) -> np.ndarray:
    return _mat(lib().orc_mat_from_quat_f, q)


def to_rotation_matrix(q) -> np.ndarray:
    return _mat(lib().orc_to_rotation_matrix_f, q)


def quat_normalize(q) -> np.ndarray:
    return _mat(lib().orc_quat_normalize_f, q, out_shape=(4,))


def rotation_jacobian(q) -> np.ndarray:
    return _mat(lib().orc_rotation_jacobian_f, q, out_shape=(4, 3, 3))


def build_cov3d(scale, q) -> np.ndarray:
    return _mat(lib().orc_build_cov3d_f, scale, q)


def backprop_cov3d(scale, q, dl_dsigma):
    s, qq, g = f32(scale), f32(q), f32(dl_dsigma).reshape(9)
    dls = np.zeros(3, np.float32)
    dq = np.zeros(4, np.float32)
    lib().orc_backprop_cov3d_f(_f(s), _f(qq), _f(g), _f(dls), _f(dq))
    return dls, dq


def sh_basis(d) -> np.ndarray:
    return _mat(lib().orc_sh_basis_f, d, out_shape=(16,))


def sh_basis_grad(d) -> np.ndarray:
    return _mat(lib().orc_sh_basis_grad_f, d, out_shape=(16, 3))


def eval_sh_deg3(coeffs, d) -> np.ndarray:
    return _mat(lib().orc_eval_sh_deg3_f, coeffs, d, out_shape=(3,))


def ssim_channel(x, y, w: int, h: int):
    a, b = f32(x).reshape(-1), f32(y).reshape(-1)
    g = np.zeros(w * h, np.float32)
    s = lib().orc_ssim_channel_f(_f(a), _f(b), w, h, _f(g))
    return float(s), g


def gaussian_kernel_1d(radius: int, sigma: float) -> np.ndarray:
    out = np.zeros(2 * radius + 1, np.float32)
    lib().orc_gaussian_kernel_1d_f(radius, float(sigma), _f(out))
    return out
