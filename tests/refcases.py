"""Scenes and helpers restated from the reference's own tests.

Record layout (``Gaussian3D``, src/math/mod.rs:27-46): position 0..2,
opacity_logit 3, rotation 4..7 (w, x, y, z), log_scale 8..10, sh 11..58
(channel-major: R0..R15, G0..G15, B0..B15).
"""
import math

import numpy as np

POS, OPA, ROT, SCL, SH = slice(0, 3), 3, slice(4, 8), slice(8, 11), slice(11, 59)


def gaussian_new(position):
    """``Gaussian3D::new`` (src/math/mod.rs:52-62)."""
    g = np.zeros(59, np.float32)
    g[POS] = position
    g[ROT] = [1.0, 0.0, 0.0, 0.0]
    g[SCL] = [-3.0, -3.0, -3.0]
    g[OPA] = -2.0
    return g


def logit(p):
    return math.log(p / (1.0 - p))


def solid_target(w, h, color):
    t = np.zeros((h, w, 4), np.float32)
    t[..., :3] = color
    t[..., 3] = 1.0
    return t


def fd_scene():
    """The single Gaussian of ``parameter_gradients_match_finite_difference``
    (src/cpu/backward.rs:906-927)."""
    g = gaussian_new([0.1, -0.05, 2.0])
    g[OPA] = np.float32(logit(0.6))
    g[SCL] = [-2.2, -2.0, -2.1]
    q = np.array([0.9, 0.1, -0.2, 0.15], np.float32)
    g[ROT] = q / np.float32(np.sqrt(np.float32((q * q).sum())))
    for ch in range(3):
        g[11 + ch * 16] = 0.4
        for k in range(1, 16):
            g[11 + ch * 16 + k] = np.float32(math.sin((ch * 16 + k) * 0.05) * 0.04)
    return g[None, :].copy()


def training_scene():
    """Five Gaussians of ``training_reduces_photometric_loss``
    (tests/training_reduces_loss.rs:99-110)."""
    gs = []
    for (x, y) in [(-0.3, -0.3), (0.3, -0.3), (-0.3, 0.3), (0.3, 0.3), (0.0, 0.0)]:
        g = gaussian_new([x, y, 2.0])
        g[OPA] = np.float32(logit(0.5))
        g[SCL] = [-1.3, -1.3, -1.3]
        for ch in range(3):
            g[11 + ch * 16] = 0.0
        gs.append(g)
    return np.stack(gs).astype(np.float32)


def loss_grad_images(w=12, h=12):
    """Deterministic buffers of ``image_loss_gradient_matches_finite_difference``
    (src/cpu/backward.rs:858-870)."""
    rendered = np.zeros(w * h * 3, np.float32)
    target = np.zeros(w * h * 4, np.float32)
    for p in range(w * h):
        for ch in range(3):
            rendered[p * 3 + ch] = np.float32(math.sin(np.float32(p * 3 + ch) * np.float32(0.123))) * np.float32(0.4) + np.float32(0.5)
            target[p * 4 + ch] = np.float32(math.cos(np.float32(p * 5 + ch) * np.float32(0.077))) * np.float32(0.4) + np.float32(0.5)
        target[p * 4 + 3] = 1.0
    return rendered, target


# Gradient record (GaussianGrad, src/cpu/backward.rs:33-41)
G_POS, G_ROT, G_SCL, G_OPA, G_SH, G_SCREEN = slice(0, 3), slice(3, 7), slice(7, 10), 10, slice(11, 59), 59


# ---------------------------------------------------------------------------
# estimate_initial_scales (src/pipeline/sfm.rs:408-450) in plain Python, a
# second restatement for pinning the C oracle on small clouds.
# ---------------------------------------------------------------------------
def rust_binary_search_py(xs, t):
    """Rust's slice::binary_search_by, size-halving form (last of equal keys)."""
    n = len(xs)
    if n == 0:
        return ("err", 0)
    base, size = 0, n
    while size > 1:
        half = size // 2
        mid = base + half
        if not xs[mid] > t:
            base = mid
        size -= half
    if xs[base] == t:
        return ("ok", base)
    return ("err", base + (1 if xs[base] < t else 0))


def sfm_scales_py(xyz):
    import math

    pts = [tuple(float(v) for v in p) for p in xyz]
    n = len(pts)
    order = sorted(range(n), key=lambda i: pts[i][0])  # stable
    sx = [pts[i][0] for i in order]
    out = []
    window = min(50, n)
    for i, q in enumerate(pts):
        kind, found = rust_binary_search_py(sx, q[0])
        if kind != "ok":
            found = 0
        start = found - min(found, window // 2)
        end = min(start + window, n)
        d = []
        for p in range(start, end):
            j = order[p]
            if j == i:
                continue
            o = pts[j]
            dx, dy, dz = o[0] - q[0], o[1] - q[1], o[2] - q[2]
            d.append(math.sqrt(dx * dx + dy * dy + dz * dz))
        d.sort()
        if not d:
            out.append(0.01)
        else:
            k = min(3, len(d))
            s = -0.0
            for v in d[:k]:
                s += v
            out.append(s / k)
    import numpy as np

    return np.array(out, dtype=np.float64).astype(np.float32)


def sfm_cloud(n, seed, dup_x=0):
    """A seeded SfM-like cloud: clustered points, some exactly repeated, some
    sharing x, a -0.0 / +0.0 pair, colours over the full byte range."""
    import numpy as np

    rng = np.random.default_rng(seed)
    c = rng.normal(size=(max(n // 40, 1), 3)) * 3.0
    xyz = c[rng.integers(0, c.shape[0], n)] + rng.normal(size=(n, 3)) * 0.05
    if n >= 8:
        xyz[1] = xyz[0]                      # an exact duplicate point
        xyz[3, 0] = xyz[2, 0]                # same x, different y / z
        xyz[4, 0], xyz[5, 0] = -0.0, 0.0     # signed zeros compare equal
    if dup_x:
        xyz[-dup_x:, 0] = xyz[-1, 0]         # a long run of equal x
    rgb = rng.integers(0, 256, size=(n, 3), dtype=np.uint8)
    if n >= 2:
        rgb[0] = (0, 255, 128)
    return xyz, rgb
