"""Seeded synthetic scenes standing in for the reference's SfM-initialised data.

The reference initialises Gaussians from COLMAP points and trains on photos;
neither is available here, so these generators produce the workloads the
benchmark and tests use, with the shapes and distributions stated per config:
  means uniform in [-r, r]^3, log-scales N(mu, sigma), quaternions = normalised
  N(0, 1) 4-vectors, opacity logits N(mu, sigma), SH degree 3 with the three DC
  terms (sh[0], sh[16], sh[32]) ~ N(0, 0.3) and the rest ~ N(0, 0.05).
Cameras follow the reference's OpenCV convention (+z forward, +y down; c2w
columns = right, down, forward; src/cpu/backward.rs:225-234), principal point at
the image centre. Targets are rendered from a copy of the scene with means
perturbed by N(0, 0.02).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .api import Camera

DC_INDICES = (11, 11 + 16, 11 + 32)  # record offsets of sh[0], sh[16], sh[32]


def random_gaussians(n: int, seed: int, mean_range: float = 1.0, log_scale=(-4.0, 0.5), opacity=(0.0, 1.0),
                     sh_dc_sigma: float = 0.3, sh_rest_sigma: float = 0.05) -> np.ndarray:
    rng = np.random.default_rng(seed)
    g = np.zeros((n, 59), np.float32)
    g[:, 0:3] = rng.uniform(-mean_range, mean_range, (n, 3))
    g[:, 3] = rng.normal(opacity[0], opacity[1], n)
    q = rng.normal(0.0, 1.0, (n, 4))
    q /= np.maximum(np.linalg.norm(q, axis=1, keepdims=True), 1e-12)
    g[:, 4:8] = q
    g[:, 8:11] = rng.normal(log_scale[0], log_scale[1], (n, 3))
    sh = rng.normal(0.0, sh_rest_sigma, (n, 48))
    for k in (0, 16, 32):
        sh[:, k] = rng.normal(0.0, sh_dc_sigma, n)
    g[:, 11:59] = sh
    return g


def perturbed(g: np.ndarray, seed: int, sigma: float = 0.02) -> np.ndarray:
    rng = np.random.default_rng(seed)
    out = g.copy()
    out[:, 0:3] += rng.normal(0.0, sigma, (g.shape[0], 3)).astype(np.float32)
    return out


def look_at(eye, target, width: int, height: int, fx: float, fy: float | None = None) -> Camera:
    eye = np.asarray(eye, np.float64)
    fwd = np.asarray(target, np.float64) - eye
    fwd /= np.linalg.norm(fwd)
    up = np.array([0.0, 0.0, 1.0])
    if abs(np.dot(up, fwd)) > 0.999:
        up = np.array([0.0, 1.0, 0.0])
    right = np.cross(fwd, up)
    right /= np.linalg.norm(right)
    down = np.cross(fwd, right)
    c2w = np.eye(4)
    c2w[:3, 0], c2w[:3, 1], c2w[:3, 2], c2w[:3, 3] = right, down, fwd, eye
    return Camera(width, height, float(fx), float(fy if fy is not None else fx), width / 2.0, height / 2.0, c2w.astype(np.float32))


def sphere_cameras(count: int, radius: float, sizes, focal_per_width: float) -> list[Camera]:
    """Fibonacci-sphere cameras looking at the origin; sizes cycle through ``sizes``."""
    cams = []
    golden = np.pi * (3.0 - np.sqrt(5.0))
    for i in range(count):
        y = 1.0 - 2.0 * (i + 0.5) / count
        r = np.sqrt(max(0.0, 1.0 - y * y))
        th = golden * i
        eye = radius * np.array([np.cos(th) * r, np.sin(th) * r, y])
        w, h = sizes[i % len(sizes)]
        cams.append(look_at(eye, (0.0, 0.0, 0.0), w, h, focal_per_width * w))
    return cams


@dataclass
class SceneConfig:
    name: str
    n: int
    mean_range: float
    log_scale: tuple
    opacity: tuple
    cameras: list = field(default_factory=list)
    views_per_step: int = 1
    iterations: int = 100
    seed: int = 0


def config(index: int, n: int | None = None, seed: int = 0) -> SceneConfig:
    """The five benchmark workloads (scene generation only; n may be reduced for tests)."""
    if index == 0:
        cams = [look_at((0.0, 0.0, -4.0), (0.0, 0.0, 0.0), 256, 256, 300.0)]
        return SceneConfig("10k Gaussians, 1 view 256x256", n or 10_000, 1.0, (-4.0, 0.5), (0.0, 1.0), cams, 1, 100, seed)
    if index == 1:
        cams = sphere_cameras(64, 5.0, [(800, 800)], 1000.0 / 800.0)
        return SceneConfig("200k Gaussians, 64 cams 800x800", n or 200_000, 2.0, (-4.0, 0.5), (0.0, 1.0), cams, 1, 2000, seed)
    if index == 2:
        cams = [look_at((0.0, 0.0, -4.0), (0.0, 0.0, 0.0), 512, 512, 600.0)]
        return SceneConfig("50k Gaussians, 1 view 512x512", n or 50_000, 1.0, (-4.0, 0.5), (0.0, 1.0), cams, 1, 1, seed)
    if index == 3:
        cams = sphere_cameras(128, 5.0, [(1600, 1064), (1280, 720), (960, 540)], 1.25)
        return SceneConfig("1M Gaussians, 8 views/step, mixed 1600x1064/1280x720/960x540", n or 1_000_000, 2.0, (-4.0, 0.5),
                           (0.0, 1.0), cams, 8, 3000, seed)
    if index == 4:
        cams = sphere_cameras(256, 5.0, [(1920, 1080)], 1.0)
        return SceneConfig("3M Gaussians anisotropic, 16 views/step 1920x1080", n or 3_000_000, 2.0, (-3.5, 1.0), (1.0, 1.0), cams,
                           16, 10_000, seed)
    raise ValueError(index)


def make_gaussians(cfg: SceneConfig) -> np.ndarray:
    return random_gaussians(cfg.n, cfg.seed, cfg.mean_range, cfg.log_scale, cfg.opacity)
