"""Introspection of one view's intermediate state (include/rgsplat_debug.h).

Exposes the caches the reference keeps private inside `render_and_backward`
(src/cpu/backward.rs:172-512) so tests can compare them element by element.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .api import Camera, Context, _f32, _fp, _gauss, camera_c, default_context


def project(gaussians, camera: Camera, ctx: Context | None = None):
    """-> (visible (N,) int32, rec (N, 10), tile rect (N, 4) int32)."""
    ctx = ctx or default_context()
    g = _gauss(gaussians)
    n = g.shape[0]
    vis = np.zeros(max(n, 1), np.int32)
    rec = np.zeros((max(n, 1), 10), np.float32)
    rect = np.zeros((max(n, 1), 4), np.int32)
    cam = camera_c(camera)
    ctx.check(ctx.lib.rgs_debug_project(ctx.handle, _fp(g), n, C.byref(cam), vis.ctypes.data_as(C.POINTER(C.c_int32)), _fp(rec),
                                        rect.ctypes.data_as(C.POINTER(C.c_int32))))
    return vis[:n], rec[:n], rect[:n]


def tile_lists(gaussians, camera: Camera, ctx: Context | None = None, pruned: bool = False):
    """-> (offsets (tiles+1,), entries (pairs,)) over the context's CTA tiles;
    pruned: the lists the zero-background paths bin (rgs_debug_pruned_tile_lists)."""
    ctx = ctx or default_context()
    fn = ctx.lib.rgs_debug_pruned_tile_lists if pruned else ctx.lib.rgs_debug_tile_lists
    g = _gauss(gaussians)
    n = g.shape[0]
    cam = camera_c(camera)
    o = ctx.options()
    tw, th = o["tile_w"], o["tile_h"]
    tiles = ((camera.width + tw - 1) // tw) * ((camera.height + th - 1) // th)
    npairs = C.c_uint64(0)
    ip = C.POINTER(C.c_int32)
    ctx.check(fn(ctx.handle, _fp(g), n, C.byref(cam), C.byref(npairs), None, None, 0))
    offs = np.zeros(tiles + 1, np.int32)
    ent = np.zeros(max(int(npairs.value), 1), np.int32)
    ctx.check(fn(ctx.handle, _fp(g), n, C.byref(cam), C.byref(npairs), offs.ctypes.data_as(ip), ent.ctypes.data_as(ip),
                 ent.shape[0]))
    return offs, ent[: int(npairs.value)]


def forward(gaussians, camera: Camera, bg=(0.0, 0.0, 0.0), ctx: Context | None = None):
    """-> (rgb (H, W, 3), final_t (H, W), last_contrib (H, W) int32)."""
    ctx = ctx or default_context()
    g = _gauss(gaussians)
    h, w = camera.height, camera.width
    rgb = np.zeros((h, w, 3), np.float32)
    ft = np.zeros((h, w), np.float32)
    last = np.zeros((h, w), np.int32)
    cam = camera_c(camera)
    ctx.check(ctx.lib.rgs_debug_forward(ctx.handle, _fp(g), g.shape[0], C.byref(cam), _fp(_f32(bg)), _fp(rgb), _fp(ft),
                                        last.ctypes.data_as(C.POINTER(C.c_int32))))
    return rgb, ft, last


def backward(gaussians, camera: Camera, target_rgba, bg=(0.0, 0.0, 0.0), lam: float = 0.2, ctx: Context | None = None):
    """-> (per-Gaussian blend accumulators (N, 9), dL/dpixel (H, W, 3))."""
    ctx = ctx or default_context()
    g = _gauss(gaussians)
    n = g.shape[0]
    acc = np.zeros((max(n, 1), 9), np.float32)
    dl = np.zeros((camera.height, camera.width, 3), np.float32)
    cam = camera_c(camera)
    tgt = _f32(target_rgba).reshape(-1)
    ctx.check(ctx.lib.rgs_debug_backward(ctx.handle, _fp(g), n, C.byref(cam), _fp(tgt), _fp(_f32(bg)), float(lam), _fp(acc), _fp(dl)))
    return acc[:n], dl


def trainer_batch_pixels(trainer, views, k: int):
    """View at position k of the trainer's last batched pass over ``views``, read
    from the batch's own buffers -> (rgb (H, W, 3), final_t (H, W),
    dL/dpixel (H, W, 3))."""
    ctx = trainer.ctx
    c = trainer.cameras[views[k]]
    rgb = np.zeros((c.height, c.width, 3), np.float32)
    ft = np.zeros((c.height, c.width), np.float32)
    dl = np.zeros((c.height, c.width, 3), np.float32)
    ctx.check(ctx.lib.rgs_debug_trainer_batch_pixels(ctx.handle, int(k), _fp(rgb), _fp(ft), _fp(dl)))
    return rgb, ft, dl


def exp_sfu_error(lo: float = -8.0, hi: float = 0.0, n: int = 1 << 24, ctx: Context | None = None) -> float:
    """Largest relative difference of the backward's SFU exponential from the
    forward's exp over n points on [lo, hi]."""
    ctx = ctx or default_context()
    out = np.zeros(1, np.float32)
    ctx.check(ctx.lib.rgs_debug_exp_sfu_error(ctx.handle, float(lo), float(hi), int(n), _fp(out)))
    return float(out[0])
