"""Host-side mirror of rgsplat's training-path API over the C ABI.

Names, argument meanings and array layouts follow the reference crate:
  * ``render_and_backward`` / ``render_color`` / ``photometric_loss_grad``
    (src/cpu/backward.rs:107-166, 646-693),
  * ``adam_step`` / ``densify_and_prune`` / ``reset_opacities`` with
    ``AdamState`` and ``TrainConfig`` (src/pipeline/optimizer.rs),
  * ``GpuRenderer.project`` / ``GpuRenderer.render`` (src/gpu/compute.rs:88-218),
plus a device-resident ``Trainer`` for the training loop of
src/pipeline/mod.rs:203-265 (plain and batched multi-view steps).

Gaussians are ``(N, 59)`` float32 arrays in the ``Gaussian3D`` record order;
gradients ``(N, 60)`` in the ``GaussianGrad`` order. Where the reference
panics (NaN depth, singular camera) these functions raise ``RgsError``.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

from . import _lib as L

GAUSSIAN_FLOATS = 59
GRAD_FLOATS = 60


class RgsError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{L.ERROR_NAMES.get(code, 'error')} ({code}): {message}")
        self.code = code


# ---------------------------------------------------------------------------
# value types
# ---------------------------------------------------------------------------
@dataclass
class Camera:
    """``Camera`` (src/math/mod.rs:131-145): pinhole, row-major c2w, OpenCV axes."""

    width: int
    height: int
    fx: float
    fy: float
    cx: float
    cy: float
    c2w: np.ndarray = field(default_factory=lambda: np.eye(4, dtype=np.float32))

    def to_c(self) -> L.rgs_camera:
        s = L.rgs_camera()
        s.width, s.height = int(self.width), int(self.height)
        s.fx, s.fy, s.cx, s.cy = float(self.fx), float(self.fy), float(self.cx), float(self.cy)
        flat = np.ascontiguousarray(self.c2w, dtype=np.float32).reshape(16)
        for i in range(16):
            s.c2w[i] = float(flat[i])
        return s

    def position(self) -> np.ndarray:
        """``Camera::position`` (mod.rs:163-165)."""
        m = np.asarray(self.c2w, np.float32)
        return np.array([m[0, 3], m[1, 3], m[2, 3]], np.float32)


@dataclass
class LossConfig:
    """``LossConfig`` (src/cpu/backward.rs:57-67)."""

    lambda_dssim: float = 0.2

    def to_c(self) -> L.rgs_loss_config:
        return L.rgs_loss_config(float(self.lambda_dssim))


@dataclass
class TrainConfig:
    """``TrainConfig`` with ``Default`` (src/pipeline/optimizer.rs:22-62)."""

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

    def to_c(self) -> L.rgs_train_config:
        s = L.rgs_train_config()
        for name, _ in L.rgs_train_config._fields_:
            setattr(s, name, getattr(self, name))
        return s


class AdamState:
    """``AdamState`` (src/pipeline/optimizer.rs:74-106). Arrays only ever grow."""

    def __init__(self, n: int):
        self.m1 = np.zeros(n * GAUSSIAN_FLOATS, np.float32)
        self.m2 = np.zeros(n * GAUSSIAN_FLOATS, np.float32)
        self.grad_accum = np.zeros(n, np.float32)
        self.grad_denom = np.zeros(n, np.uint32)
        self.t = 0

    def __len__(self) -> int:
        return self.grad_accum.shape[0]

    def resize(self, new_n: int) -> None:
        old = len(self)
        if new_n > old:
            extra = new_n - old
            self.m1 = np.concatenate([self.m1, np.zeros(extra * GAUSSIAN_FLOATS, np.float32)])
            self.m2 = np.concatenate([self.m2, np.zeros(extra * GAUSSIAN_FLOATS, np.float32)])
            self.grad_accum = np.concatenate([self.grad_accum, np.zeros(extra, np.float32)])
            self.grad_denom = np.concatenate([self.grad_denom, np.zeros(extra, np.uint32)])

    def to_c(self) -> L.rgs_adam_state:
        s = L.rgs_adam_state()
        s.m1 = self.m1.ctypes.data_as(L.FP)
        s.m2 = self.m2.ctypes.data_as(L.FP)
        s.grad_accum = self.grad_accum.ctypes.data_as(L.FP)
        s.grad_denom = self.grad_denom.ctypes.data_as(L.U32P)
        s.len = len(self)
        s.t = self.t
        return s


# ---------------------------------------------------------------------------
# context
# ---------------------------------------------------------------------------
class Context:
    """One CUDA stream plus the library's device buffers (``rgs_ctx``).

    exact_loss: the SSIM blurs use the reference's separate multiply and add
    (dL/dpixel bit-identical to the reference's) instead of fused
    multiply-adds (the default; within float rounding)."""

    def __init__(self, device: int = 0, tile: tuple[int, int] = (16, 16), batch: int = 256, reference_compat: bool = True,
                 pixels_per_thread: int = 2, batch_pair_limit: int = 0, exact_loss: bool = False):
        self.lib = L.load()
        o = L.rgs_options()
        self.lib.rgs_options_default(C.byref(o))
        o.device = int(device)
        o.tile_w, o.tile_h = int(tile[0]), int(tile[1])
        o.batch = int(batch)
        o.reference_compat = 1 if reference_compat else 0
        o.pixels_per_thread = int(pixels_per_thread)
        o.batch_pair_limit = int(batch_pair_limit)
        o.exact_loss = 1 if exact_loss else 0
        h = C.c_void_p()
        rc = self.lib.rgs_create(C.byref(o), C.byref(h))
        if rc != L.RGS_OK:
            raise RgsError(rc, "rgs_create failed")
        self.handle = h
        self.create_options = o
        self.stream = None  # cudaStream_t the context issues on; None: its own

    def check(self, rc: int) -> None:
        if rc != L.RGS_OK:
            msg = self.lib.rgs_last_error(self.handle)
            raise RgsError(rc, msg.decode() if msg else "")

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.rgs_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, cuda_stream: int | None) -> None:
        """Issue work on an external cudaStream_t (not the legacy default stream)."""
        self.check(self.lib.rgs_set_stream(self.handle, C.c_void_p(cuda_stream or None)))
        self.stream = int(cuda_stream) if cuda_stream else None

    def set_profiling(self, on: bool) -> None:
        self.check(self.lib.rgs_set_profiling(self.handle, 1 if on else 0))

    def stage_times(self, reset: bool = False) -> dict:
        """Milliseconds per training-step stage accumulated since the last reset."""
        ms = (C.c_float * L.RGS_NUM_STAGES)()
        self.check(self.lib.rgs_get_stage_times(self.handle, ms, 1 if reset else 0))
        return {n: float(ms[i]) for i, n in enumerate(L.STAGE_NAMES)}

    def stats(self) -> dict:
        s = L.rgs_stats()
        self.check(self.lib.rgs_get_stats(self.handle, C.byref(s)))
        return {name: getattr(s, name) for name, _ in L.rgs_stats._fields_}

    def memory(self, reset_peak: bool = False) -> dict:
        """Device bytes this context holds through its own buffers and the most
        it has held since creation or the last reset_peak (which restarts the
        high-water mark at the bytes held)."""
        held, peak = C.c_uint64(0), C.c_uint64(0)
        self.check(self.lib.rgs_get_memory(self.handle, C.byref(held), C.byref(peak), 1 if reset_peak else 0))
        return {"held_bytes": int(held.value), "peak_bytes": int(peak.value)}

    def options(self) -> dict:
        o = L.rgs_options()
        self.check(self.lib.rgs_get_options(self.handle, C.byref(o)))
        return {name: getattr(o, name) for name, _ in L.rgs_options._fields_}

    def set_tiling(self, tile: tuple[int, int], batch: int, pixels_per_thread: int) -> None:
        """Blend-kernel layout (results are identical for every layout)."""
        self.check(self.lib.rgs_set_tiling(self.handle, int(tile[0]), int(tile[1]), int(batch), int(pixels_per_thread)))


_tls = threading.local()


def default_context() -> Context:
    """The calling thread's context (the reference is called from one thread per pipeline)."""
    ctx = getattr(_tls, "ctx", None)
    if ctx is None:
        ctx = Context()
        _tls.ctx = ctx
    return ctx


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def _fp(a: np.ndarray):
    return a.ctypes.data_as(L.FP)


def _gauss(g) -> np.ndarray:
    g = _f32(g)
    if g.size % GAUSSIAN_FLOATS:
        raise ValueError("gaussians must be (N, 59) float32")
    return g.reshape(-1, GAUSSIAN_FLOATS)


def camera_c(c) -> L.rgs_camera:
    """``rgs_camera`` from any object with width, height, fx, fy, cx, cy and a 4x4 c2w."""
    return Camera.to_c(c)


# ---------------------------------------------------------------------------
# drop-ins for the reference's free functions
# ---------------------------------------------------------------------------
def render_and_backward(gaussians, camera: Camera, target_rgba, bg=(0.0, 0.0, 0.0), cfg: LossConfig | None = None,
                        ctx: Context | None = None):
    """``render_and_backward`` (src/cpu/backward.rs:107-149) -> (loss, grads (N, 60))."""
    ctx = ctx or default_context()
    g = _gauss(gaussians)
    n = g.shape[0]
    tgt = _f32(target_rgba).reshape(-1)
    if tgt.size != camera.width * camera.height * 4:
        raise ValueError("target must be w*h*4 RGBA floats")
    grads = np.zeros((n, GRAD_FLOATS), np.float32)
    loss = C.c_float(0.0)
    bgv = _f32(bg)
    cam = camera_c(camera)
    lc = (cfg or LossConfig()).to_c()
    ctx.check(ctx.lib.rgs_render_and_backward(ctx.handle, _fp(g), n, C.byref(cam), _fp(tgt), _fp(bgv), C.byref(lc), C.byref(loss), _fp(grads)))
    return float(loss.value), grads


def render_and_backward_variant(gaussians, camera: Camera, target_rgba, store_all: bool, bg=(0.0, 0.0, 0.0),
                                cfg: LossConfig | None = None, ctx: Context | None = None):
    """render_and_backward with the recompute-from-final-T backward (the
    library's path) or the store-all-T variant -> (loss, grads, report) where
    report holds the blend kernel times (ms) and the blend-state bytes."""
    ctx = ctx or default_context()
    g = _gauss(gaussians)
    n = g.shape[0]
    tgt = _f32(target_rgba).reshape(-1)
    if tgt.size != camera.width * camera.height * 4:
        raise ValueError("target must be w*h*4 RGBA floats")
    grads = np.zeros((n, GRAD_FLOATS), np.float32)
    loss = C.c_float(0.0)
    cam = camera_c(camera)
    lc = (cfg or LossConfig()).to_c()
    rep = L.rgs_backward_report()
    variant = L.RGS_BACKWARD_STORE_ALL if store_all else L.RGS_BACKWARD_RECOMPUTE
    ctx.check(ctx.lib.rgs_render_and_backward_variant(ctx.handle, _fp(g), n, C.byref(cam), _fp(tgt), _fp(_f32(bg)), C.byref(lc),
                                                      variant, C.byref(loss), _fp(grads), C.byref(rep)))
    report = {name: getattr(rep, name) for name, _ in L.rgs_backward_report._fields_}
    return float(loss.value), grads, report


def render_color(gaussians, camera: Camera, bg=(0.0, 0.0, 0.0), ctx: Context | None = None) -> np.ndarray:
    """``render_color`` (src/cpu/backward.rs:152-166) -> interleaved RGB (H, W, 3)."""
    ctx = ctx or default_context()
    g = _gauss(gaussians)
    out = np.zeros((camera.height, camera.width, 3), np.float32)
    cam = camera_c(camera)
    ctx.check(ctx.lib.rgs_render_color(ctx.handle, _fp(g), g.shape[0], C.byref(cam), _fp(_f32(bg)), _fp(out)))
    return out


def rasterize(gaussians, camera: Camera, bg=(0.0, 0.0, 0.0), srgb8: bool = False, ctx: Context | None = None) -> np.ndarray:
    """``cpu::rasterize`` (src/cpu/rasterizer.rs:72-192) -> the Framebuffer's RGBA
    (H, W, 4) float32, or with srgb8 its ``to_u8_srgb`` bytes (uint8)."""
    ctx = ctx or default_context()
    g = _gauss(gaussians)
    cam = camera_c(camera)
    if srgb8:
        out = np.zeros((camera.height, camera.width, 4), np.uint8)
        fmt = L.RGS_FB_RGBA8_SRGB
    else:
        out = np.zeros((camera.height, camera.width, 4), np.float32)
        fmt = L.RGS_FB_RGBA_F32
    ctx.check(ctx.lib.rgs_rasterize(ctx.handle, _fp(g), g.shape[0], C.byref(cam), _fp(_f32(bg)), fmt, out.ctypes.data))
    return out


def srgb8_to_linear(rgba8, ctx: Context | None = None) -> np.ndarray:
    """``load_target``'s conversion (src/io/images.rs:67-72): an 8-bit sRGB RGBA
    image (..., 4) uint8 -> linear RGBA float32 of the same shape."""
    ctx = ctx or default_context()
    a = np.ascontiguousarray(rgba8, np.uint8)
    if a.size % 4:
        raise ValueError("RGBA8 input must hold 4 bytes per pixel")
    out = np.zeros(a.shape, np.float32)
    ctx.check(ctx.lib.rgs_srgb8_to_linear(ctx.handle, a.ctypes.data, a.size // 4, _fp(out)))
    return out


def black_target(width: int, height: int) -> np.ndarray:
    """``TargetImage::black`` (src/io/images.rs:26-33): opaque black RGBA (h, w, 4)."""
    t = np.zeros((height, width, 4), np.float32)
    t[..., 3] = 1.0
    return t


def save_ply(gaussians, path, ctx: Context | None = None) -> None:
    """``io::ply::save_ply`` (src/io/ply.rs:35-104): binary little-endian 3DGS .ply."""
    ctx = ctx or default_context()
    g = _gauss(gaussians)
    ctx.check(ctx.lib.rgs_save_ply(ctx.handle, _fp(g), g.shape[0], os.fsencode(path)))


def save_splat(gaussians, path, ctx: Context | None = None) -> None:
    """``io::ply::save_splat`` (src/io/ply.rs:253-285): 32-byte .splat records."""
    ctx = ctx or default_context()
    g = _gauss(gaussians)
    ctx.check(ctx.lib.rgs_save_splat(ctx.handle, _fp(g), g.shape[0], os.fsencode(path)))


def load_ply(path, ctx: Context | None = None) -> np.ndarray:
    """``io::ply::load_ply`` (src/io/ply.rs:116-193) -> (N, 59) Gaussians."""
    ctx = ctx or default_context()
    n = C.c_size_t(0)
    p = os.fsencode(path)
    rc = ctx.lib.rgs_load_ply(ctx.handle, p, None, 0, C.byref(n))
    if rc not in (L.RGS_OK, L.RGS_ERR_CAPACITY):
        ctx.check(rc)
    out = np.zeros((max(n.value, 1), GAUSSIAN_FLOATS), np.float32)
    ctx.check(ctx.lib.rgs_load_ply(ctx.handle, p, _fp(out), out.shape[0], C.byref(n)))
    return out[: n.value]


def _sfm_points(xyz, rgb):
    x = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
    c = np.ascontiguousarray(rgb, np.uint8).reshape(-1, 3)
    if x.shape[0] != c.shape[0]:
        raise ValueError("xyz and rgb hold different point counts")
    return x, c


def gaussians_from_sfm(xyz, rgb, ctx: Context | None = None) -> np.ndarray:
    """``gaussians_from_sfm`` (src/pipeline/sfm.rs:365-404) on the device: (N, 3)
    f64 points and (N, 3) u8 colours -> (N, 59) Gaussians, scales from
    ``estimate_initial_scales`` (:408-450)."""
    ctx = ctx or default_context()
    x, c = _sfm_points(xyz, rgb)
    out = np.zeros((x.shape[0], GAUSSIAN_FLOATS), np.float32)
    ctx.check(ctx.lib.rgs_gaussians_from_sfm(ctx.handle, x.ctypes.data, c.ctypes.data, x.shape[0], _fp(out)))
    return out


def read_points3d_bin(path, ctx: Context | None = None):
    """``parse_points3d_bin`` (src/pipeline/sfm.rs:147-183) of a COLMAP
    points3D.bin -> (xyz (N, 3) f64, rgb (N, 3) u8)."""
    ctx = ctx or default_context()
    n = C.c_size_t(0)
    p = os.fsencode(path)
    rc = ctx.lib.rgs_read_points3d_bin(ctx.handle, p, None, None, 0, C.byref(n))
    if rc not in (L.RGS_OK, L.RGS_ERR_CAPACITY):
        ctx.check(rc)
    xyz = np.zeros((max(n.value, 1), 3), np.float64)
    rgb = np.zeros((max(n.value, 1), 3), np.uint8)
    ctx.check(ctx.lib.rgs_read_points3d_bin(ctx.handle, p, xyz.ctypes.data, rgb.ctypes.data, xyz.shape[0], C.byref(n)))
    return xyz[: n.value], rgb[: n.value]


def photometric_loss_grad(rendered, target_rgba, w: int, h: int, lam: float, ctx: Context | None = None):
    """``photometric_loss_grad`` (src/cpu/backward.rs:646-693) -> (loss, dL/dpixel (w*h*3,))."""
    ctx = ctx or default_context()
    r = _f32(rendered).reshape(-1)
    t = _f32(target_rgba).reshape(-1)
    if r.size != w * h * 3 or t.size != w * h * 4:
        raise ValueError("rendered must be w*h*3 and target w*h*4 floats")
    dl = np.zeros(w * h * 3, np.float32)
    loss = C.c_float(0.0)
    ctx.check(ctx.lib.rgs_photometric_loss_grad(ctx.handle, _fp(r), _fp(t), w, h, float(lam), C.byref(loss), _fp(dl)))
    return float(loss.value), dl


def adam_step(gaussians: np.ndarray, grads, state: AdamState, cfg: TrainConfig, ctx: Context | None = None) -> None:
    """``adam_step`` (src/pipeline/optimizer.rs:116-163): updates ``gaussians`` and ``state`` in place."""
    ctx = ctx or default_context()
    if gaussians.dtype != np.float32 or not gaussians.flags.c_contiguous:
        raise ValueError("gaussians must be a C-contiguous float32 array (updated in place)")
    n = gaussians.size // GAUSSIAN_FLOATS
    gr = _f32(grads).reshape(-1, GRAD_FLOATS)
    st = state.to_c()
    tc = cfg.to_c()
    ctx.check(ctx.lib.rgs_adam_step(ctx.handle, _fp(gaussians), n, _fp(gr), C.byref(st), C.byref(tc)))
    state.t = int(st.t)


def densify_and_prune(gaussians, state: AdamState, cfg: TrainConfig, scene_extent: float, ctx: Context | None = None) -> np.ndarray:
    """``densify_and_prune`` (src/pipeline/optimizer.rs:206-272): returns the new Gaussians;
    ``state`` is resized (grow only) and its densification statistics zeroed, as in the reference."""
    ctx = ctx or default_context()
    g = _gauss(gaussians)
    n = g.shape[0]
    out = np.zeros((2 * n + 1, GAUSSIAN_FLOATS), np.float32)  # kept + cloned, or split in two
    n_out = C.c_size_t(0)
    tc = cfg.to_c()
    ctx.check(ctx.lib.rgs_densify_and_prune(ctx.handle, _fp(g), n, _fp(state.grad_accum), state.grad_denom.ctypes.data_as(L.U32P),
                                            C.byref(tc), float(scene_extent), _fp(out), out.shape[0], C.byref(n_out)))
    k = int(n_out.value)
    state.resize(k)
    state.grad_accum[:] = 0
    state.grad_denom[:] = 0
    return np.ascontiguousarray(out[:k])


def reset_opacities(gaussians: np.ndarray, ctx: Context | None = None) -> None:
    """``reset_opacities`` (src/pipeline/optimizer.rs:314-319), in place."""
    ctx = ctx or default_context()
    if gaussians.dtype != np.float32 or not gaussians.flags.c_contiguous:
        raise ValueError("gaussians must be a C-contiguous float32 array (updated in place)")
    ctx.check(ctx.lib.rgs_reset_opacities(ctx.handle, _fp(gaussians), gaussians.size // GAUSSIAN_FLOATS))


def estimate_scene_extent(gaussians) -> float:
    """``estimate_scene_extent`` (src/pipeline/mod.rs:299-313): bbox diagonal."""
    g = _gauss(gaussians)
    if g.shape[0] == 0:
        return 1.0
    d = (g[:, :3].max(axis=0) - g[:, :3].min(axis=0)).astype(np.float32)
    return float(np.float32(np.sqrt(np.float32(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]))))


class GpuRenderer:
    """``gpu::GpuRenderer`` (src/gpu/compute.rs:80-219) on CUDA.

    ``cpu_math=False`` reproduces the shader's arithmetic (DC-only colour, its
    column-major Jacobian); ``cpu_math=True`` returns the CPU path's splats.
    """

    def __init__(self, ctx: Context | None = None, cpu_math: bool = False):
        self.ctx = ctx or Context()
        self.mode = L.RGS_PROJECT_CPU_MATH if cpu_math else L.RGS_PROJECT_WGSL

    def adapter_name(self) -> str:
        return "CUDA sm_100a"

    def project(self, gaussians, camera: Camera):
        """-> (SplatInfo2D as (N, 10) float32, depth keys (N,) uint32)."""
        g = _gauss(gaussians)
        n = g.shape[0]
        out = np.zeros((max(n, 1), 10), np.float32)
        keys = np.zeros(max(n, 1), np.uint32)
        cam = camera_c(camera)
        self.ctx.check(self.ctx.lib.rgs_project(self.ctx.handle, _fp(g), n, C.byref(cam), self.mode,
                                                out.ctypes.data_as(C.POINTER(L.rgs_splat_info_2d)), keys.ctypes.data_as(L.U32P)))
        return out[:n], keys[:n]

    def render(self, gaussians, camera: Camera, bg=(0.0, 0.0, 0.0)) -> np.ndarray:
        g = _gauss(gaussians)
        out = np.zeros((camera.height, camera.width, 3), np.float32)
        cam = camera_c(camera)
        self.ctx.check(self.ctx.lib.rgs_gpu_render(self.ctx.handle, _fp(g), g.shape[0], C.byref(cam), self.mode, _fp(_f32(bg)), _fp(out)))
        return out


# ---------------------------------------------------------------------------
# device-resident trainer
# ---------------------------------------------------------------------------
class Trainer:
    """Device-resident training state: Gaussians, Adam moments, cameras, targets."""

    PLAIN = L.RGS_STEP_PLAIN
    BATCHED = L.RGS_STEP_BATCHED

    def __init__(self, gaussians, cameras: Sequence[Camera], targets=None, ctx: Context | None = None, **ctx_kwargs):
        self.ctx = ctx or Context(**ctx_kwargs)
        self.lib = self.ctx.lib
        self.cameras = list(cameras)
        self.set_gaussians(gaussians)
        arr = (L.rgs_camera * max(len(self.cameras), 1))()
        for i, c in enumerate(self.cameras):
            arr[i] = camera_c(c)
        self.ctx.check(self.lib.rgs_trainer_set_cameras(self.ctx.handle, arr, len(self.cameras)))
        if targets is not None:
            for i, t in enumerate(targets):
                self.set_target(i, t)

    def set_gaussians(self, gaussians) -> None:
        g = _gauss(gaussians)
        self.ctx.check(self.lib.rgs_trainer_set_gaussians(self.ctx.handle, _fp(g), g.shape[0]))

    def set_target(self, index: int, target_rgba) -> None:
        t = _f32(target_rgba).reshape(-1)
        c = self.cameras[index]
        if t.size != c.width * c.height * 4:
            raise ValueError("target must be w*h*4 RGBA floats")
        self.ctx.check(self.lib.rgs_trainer_set_target(self.ctx.handle, index, _fp(t)))

    def set_target_ptr(self, index: int, host_ptr: int) -> None:
        """Upload camera ``index``'s RGBA target from a raw host pointer (e.g. pinned memory)."""
        self.ctx.check(self.lib.rgs_trainer_set_target(self.ctx.handle, index, C.cast(C.c_void_p(host_ptr), L.FP)))

    def __len__(self) -> int:
        n = C.c_size_t(0)
        self.ctx.check(self.lib.rgs_trainer_count(self.ctx.handle, C.byref(n)))
        return int(n.value)

    def gaussians(self) -> np.ndarray:
        n = len(self)
        out = np.zeros((max(n, 1), GAUSSIAN_FLOATS), np.float32)
        got = C.c_size_t(0)
        self.ctx.check(self.lib.rgs_trainer_get_gaussians(self.ctx.handle, _fp(out), out.shape[0], C.byref(got)))
        return out[: got.value]

    def step(self, views: Sequence[int], bg=(0.0, 0.0, 0.0), loss_cfg: LossConfig | None = None,
             train_cfg: TrainConfig | None = None, mode: int = L.RGS_STEP_BATCHED) -> np.ndarray:
        v = np.ascontiguousarray(views, dtype=np.uint32)
        losses = np.zeros(max(v.size, 1), np.float32)
        lc = (loss_cfg or LossConfig()).to_c()
        tc = (train_cfg or TrainConfig()).to_c()
        self.ctx.check(self.lib.rgs_trainer_step(self.ctx.handle, v.ctypes.data_as(L.U32P), v.size, _fp(_f32(bg)), C.byref(lc),
                                                 C.byref(tc), int(mode), _fp(losses)))
        return losses[: v.size]

    def init_from_sfm(self, xyz, rgb) -> int:
        """The trainer's Gaussians from SfM points (``gaussians_from_sfm``,
        src/pipeline/sfm.rs:365-450) built on the device; the optimiser restarts."""
        x, c = _sfm_points(xyz, rgb)
        self.ctx.check(self.lib.rgs_trainer_init_from_sfm(self.ctx.handle, x.ctypes.data, c.ctypes.data, x.shape[0]))
        return x.shape[0]

    def set_target_rgba8(self, index: int, rgba8) -> None:
        """Camera ``index``'s target from an 8-bit sRGB RGBA image at the camera's
        resolution, converted to linear on the device (images.rs:67-72)."""
        a = np.ascontiguousarray(rgba8, np.uint8)
        c = self.cameras[index]
        if a.size != c.width * c.height * 4:
            raise ValueError("target must be h*w*4 bytes")
        self.ctx.check(self.lib.rgs_trainer_set_target_rgba8(self.ctx.handle, int(index), a.ctypes.data))

    def save_ply(self, path) -> None:
        """The device-resident Gaussians as a 3DGS .ply (io::ply::save_ply)."""
        self.ctx.check(self.lib.rgs_trainer_save_ply(self.ctx.handle, os.fsencode(path)))

    def save_splat(self, path) -> None:
        """The device-resident Gaussians as .splat records (io::ply::save_splat)."""
        self.ctx.check(self.lib.rgs_trainer_save_splat(self.ctx.handle, os.fsencode(path)))

    def load_ply(self, path) -> int:
        """Replace the Gaussians with a .ply file's (decoded on the device); the
        Adam state starts afresh. Returns the count."""
        n = C.c_size_t(0)
        self.ctx.check(self.lib.rgs_trainer_load_ply(self.ctx.handle, os.fsencode(path), C.byref(n)))
        return int(n.value)

    def step_host_targets(self, views: Sequence[int], target_ptrs: Sequence[int], bg=(0.0, 0.0, 0.0),
                          loss_cfg: LossConfig | None = None, train_cfg: TrainConfig | None = None) -> np.ndarray:
        """Batched step whose RGBA targets come from host memory (raw pointers,
        one w*h*4 float32 image per view, page-locked for overlap); the copies
        overlap the step's projection, sort and forward."""
        v = np.ascontiguousarray(views, dtype=np.uint32)
        if len(target_ptrs) != v.size:
            raise ValueError("one target pointer per view")
        ptrs = (C.c_void_p * max(v.size, 1))(*[int(p) for p in target_ptrs])
        losses = np.zeros(max(v.size, 1), np.float32)
        lc = (loss_cfg or LossConfig()).to_c()
        tc = (train_cfg or TrainConfig()).to_c()
        self.ctx.check(self.lib.rgs_trainer_step_host_targets(self.ctx.handle, v.ctypes.data_as(L.U32P), v.size, ptrs,
                                                              _fp(_f32(bg)), C.byref(lc), C.byref(tc), _fp(losses)))
        return losses[: v.size]

    def backward(self, views: Sequence[int], bg=(0.0, 0.0, 0.0), loss_cfg: LossConfig | None = None,
                 mode: int = L.RGS_STEP_PLAIN) -> np.ndarray:
        v = np.ascontiguousarray(views, dtype=np.uint32)
        losses = np.zeros(max(v.size, 1), np.float32)
        lc = (loss_cfg or LossConfig()).to_c()
        self.ctx.check(self.lib.rgs_trainer_backward(self.ctx.handle, v.ctypes.data_as(L.U32P), v.size, _fp(_f32(bg)), C.byref(lc),
                                                     int(mode), _fp(losses)))
        return losses[: v.size]

    def autotune(self, views: Sequence[int], bg=(0.0, 0.0, 0.0), loss_cfg: LossConfig | None = None,
                 reps: int = 3) -> tuple[dict, list[dict]]:
        """Times every blend layout (tile 16x16 / 8x32 / 32x8 x batch 128 / 256 /
        512 x 1 or 2 pixels per thread) on a batched render + backward of
        ``views`` and keeps the fastest. Returns (chosen, all measurements).
        Parameters and the Adam state are not modified."""
        v = np.ascontiguousarray(views, dtype=np.uint32)
        lc = (loss_cfg or LossConfig()).to_c()
        res = (L.rgs_tune_entry * L.RGS_TUNE_CANDIDATES)()
        chosen = L.rgs_options()
        self.ctx.check(self.lib.rgs_trainer_autotune(self.ctx.handle, v.ctypes.data_as(L.U32P), v.size, _fp(_f32(bg)),
                                                     C.byref(lc), int(reps), res, C.byref(chosen)))
        table = [{"tile": f"{e.tile_w}x{e.tile_h}", "batch": e.batch, "pixels_per_thread": e.pixels_per_thread,
                  "ms": round(float(e.ms), 4)} for e in res]
        pick = {"tile": f"{chosen.tile_w}x{chosen.tile_h}", "batch": chosen.batch,
                "pixels_per_thread": chosen.pixels_per_thread}
        return pick, table

    def evaluated_pairs(self) -> tuple[int, int]:
        """(forward, backward) (pixel, splat) pairs the blend kernels evaluated
        in the last batched pass (the FP32 roofline's work count)."""
        f, b = C.c_uint64(0), C.c_uint64(0)
        self.ctx.check(self.lib.rgs_trainer_evaluated_pairs(self.ctx.handle, C.byref(f), C.byref(b)))
        return int(f.value), int(b.value)

    def grads(self) -> np.ndarray:
        out = np.zeros((max(len(self), 1), GRAD_FLOATS), np.float32)
        self.ctx.check(self.lib.rgs_trainer_get_grads(self.ctx.handle, _fp(out)))
        return out[: len(self)]

    def grad_buffer(self):
        """(device pointer, bytes, plane stride) of the gradient planes."""
        p, b, s = C.c_void_p(), C.c_size_t(0), C.c_size_t(0)
        self.ctx.check(self.lib.rgs_trainer_grad_buffer(self.ctx.handle, C.byref(p), C.byref(b), C.byref(s)))
        return int(p.value or 0), int(b.value), int(s.value)

    def apply_adam(self, train_cfg: TrainConfig | None = None, denom_increment: int = 1) -> None:
        tc = (train_cfg or TrainConfig()).to_c()
        self.ctx.check(self.lib.rgs_trainer_apply_adam(self.ctx.handle, C.byref(tc), int(denom_increment)))

    def render(self, view: int, bg=(0.0, 0.0, 0.0)) -> np.ndarray:
        c = self.cameras[view]
        out = np.zeros((c.height, c.width, 3), np.float32)
        self.ctx.check(self.lib.rgs_trainer_render(self.ctx.handle, int(view), _fp(_f32(bg)), _fp(out)))
        return out

    def rasterize(self, view: int, bg=(0.0, 0.0, 0.0), srgb8: bool = False) -> np.ndarray:
        """``cpu::rasterize`` of the device-resident Gaussians for camera ``view``:
        RGBA float32 (H, W, 4), or with srgb8 the ``to_u8_srgb`` bytes."""
        c = self.cameras[view]
        out = np.zeros((c.height, c.width, 4), np.uint8 if srgb8 else np.float32)
        fmt = L.RGS_FB_RGBA8_SRGB if srgb8 else L.RGS_FB_RGBA_F32
        self.ctx.check(self.lib.rgs_trainer_rasterize(self.ctx.handle, int(view), _fp(_f32(bg)), int(fmt), out.ctypes.data))
        return out

    def densify_and_prune(self, train_cfg: TrainConfig, scene_extent: float) -> int:
        n = C.c_size_t(0)
        tc = train_cfg.to_c()
        self.ctx.check(self.lib.rgs_trainer_densify_and_prune(self.ctx.handle, C.byref(tc), float(scene_extent), C.byref(n)))
        return int(n.value)

    def reset_opacities(self) -> None:
        self.ctx.check(self.lib.rgs_trainer_reset_opacities(self.ctx.handle))

    def adam_state(self) -> AdamState:
        st = AdamState(len(self))
        c = st.to_c()
        self.ctx.check(self.lib.rgs_trainer_get_adam_state(self.ctx.handle, C.byref(c)))
        st.t = int(c.t)
        return st

    def set_adam_state(self, state: AdamState) -> None:
        c = state.to_c()
        self.ctx.check(self.lib.rgs_trainer_set_adam_state(self.ctx.handle, C.byref(c)))


# ---------------------------------------------------------------------------
# the training loop
# ---------------------------------------------------------------------------
CAMERA_SEED = 0x9E3779B97F4A7C15


def camera_schedule(n_cams: int, seed: int = CAMERA_SEED):
    """``train_blocking``'s camera picker (src/pipeline/mod.rs:223-230): xorshift64
    (x ^= x << 13; x ^= x >> 7; x ^= x << 17), then ``x % n_cams``."""
    x = seed
    m = (1 << 64) - 1
    while True:
        x ^= (x << 13) & m
        x ^= x >> 7
        x ^= (x << 17) & m
        yield x % n_cams


def train_blocking(trainer: Trainer, cfg: TrainConfig | None = None, bg=(0.0, 0.0, 0.0), loss_cfg: LossConfig | None = None,
                   views_per_step: int = 1, mode: int | None = None, save_interval: int = 0, out_dir=None,
                   before_densify=None, after_densify=None) -> np.ndarray:
    """``train_blocking`` (src/pipeline/mod.rs:203-265) on a device-resident trainer.

    Iterations ``0 .. cfg.num_iterations``: the next ``views_per_step`` cameras of
    the xorshift schedule, one render + backward + Adam step (per-view launches
    for one view unless ``mode`` says otherwise, the captured batched step for
    several, gradients summed over the step's views); ``densify_and_prune``
    when ``densify_from_iter <= iter <= densify_until_iter``, ``iter % 100 == 0``
    and ``iter > 0`` with the extent of the initial Gaussians; ``reset_opacities``
    when ``iter % opacity_reset_iter == 0``; a ``ckpt_{iter:06}.ply`` every
    ``save_interval`` iterations into ``out_dir``. ``before_densify(iter,
    trainer)`` / ``after_densify(iter, trainer, n)`` are called around each
    densification. Returns each iteration's loss summed over its views."""
    cfg = cfg or TrainConfig()
    if mode is None:
        mode = Trainer.PLAIN if views_per_step == 1 else Trainer.BATCHED
    extent = estimate_scene_extent(trainer.gaussians())
    cams = camera_schedule(len(trainer.cameras))
    losses = np.zeros(cfg.num_iterations, np.float32)
    if save_interval and out_dir is not None:
        os.makedirs(out_dir, exist_ok=True)
    for it in range(cfg.num_iterations):
        views = [next(cams) for _ in range(views_per_step)]
        losses[it] = np.float32(trainer.step(views, bg=bg, loss_cfg=loss_cfg, train_cfg=cfg, mode=mode).sum())
        if cfg.densify_from_iter <= it <= cfg.densify_until_iter and it % 100 == 0 and it > 0:
            if before_densify:
                before_densify(it, trainer)
            n = trainer.densify_and_prune(cfg, extent)
            if after_densify:
                after_densify(it, trainer, n)
        if cfg.opacity_reset_iter and it % cfg.opacity_reset_iter == 0 and it > 0:
            trainer.reset_opacities()
        if save_interval and out_dir is not None and it % save_interval == 0 and it > 0:
            trainer.save_ply(os.path.join(out_dir, f"ckpt_{it:06d}.ply"))
    return losses
