"""Generates tests/golden/fd_config2.npz: FP64 central finite differences of the
photometric loss on the differentiation-check workload (50k Gaussians, one
512x512 view), at 256 sampled parameters.

The loss is evaluated by the oracle in double precision (the C++ restatement
of src/cpu/backward.rs:107-149, templated on double), with eps = 1e-4 in the
parameter's own units, as the reference's finite-difference tests do
(src/cpu/backward.rs:906-982), and again with eps = 1e-6: with 50k Gaussians
a 1e-4 step of a position often moves some pixel's alpha across the 1/255 or
0.99 cut-off, and the jump, not the derivative, dominates that difference. The scene is regenerated from its seed by
rgsplat_b200.scenes; a hash of the float32 parameters and of the target image
is stored so a test can detect generator drift.

Sampled parameters: 28 visible Gaussians x 8 fields (position x, y, z; one
log-scale axis; opacity logit; the DC SH coefficient of one channel; one
higher-order SH coefficient of that channel and one of another) and 8 further
Gaussians with all four rotation components (the analytic rotation gradient
has no radial term, so rotation is compared after projecting out q itself).

Run from the repository root:  python tests/golden/make_fd_config2.py
"""
import hashlib
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from rgsplat_b200 import scenes  # noqa: E402

EPS = 1e-4
EPS_FINE = 1e-6  # a second difference: a step that crosses an alpha cut-off is not a derivative
LAMBDA = 0.2
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fd_config2.npz")


def workload():
    cfg = scenes.config(2)
    g = scenes.make_gaussians(cfg)
    cam = cfg.cameras[0]
    tg = scenes.perturbed(g, cfg.seed + 1)
    rgb, _, _ = O.render_color(tg, cam)
    target = np.concatenate([rgb, np.ones((cam.height, cam.width, 1), np.float32)], axis=2)
    return g, cam, target


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def main():
    O.set_threads(os.cpu_count() or 1)
    g, cam, target = workload()
    gd = g.astype(np.float64)
    base = O.render_and_backward(gd, cam, target, double=True)
    rng = np.random.default_rng(2024)
    # visible Gaussians with a clearly non-zero opacity gradient
    mag = np.abs(base.grads[:, 10])
    cand = np.nonzero(mag > np.quantile(mag[mag > 0], 0.5))[0]
    pick = rng.choice(cand, 36, replace=False)
    gauss, field = [], []
    for i in pick[:28]:
        ch = int(rng.integers(3))
        gauss += [i] * 8
        ch2 = (ch + 1 + int(rng.integers(2))) % 3
        field += [0, 1, 2, 8 + int(rng.integers(3)), 3, 11 + 16 * ch, 11 + 16 * ch + 1 + int(rng.integers(15)),
                  11 + 16 * ch2 + 1 + int(rng.integers(15))]
    for i in pick[28:]:
        gauss += [i] * 4
        field += [4, 5, 6, 7]
    gauss = np.array(gauss, np.int64)
    field = np.array(field, np.int64)
    assert gauss.size == 256
    fd = np.zeros(256)
    fd_fine = np.zeros(256)
    t0 = time.time()
    for k in range(256):
        for eps, out in ((EPS, fd), (EPS_FINE, fd_fine)):
            gp, gm = gd.copy(), gd.copy()
            gp[gauss[k], field[k]] += eps
            gm[gauss[k], field[k]] -= eps
            lp = O.render_and_backward(gp, cam, target, double=True).loss
            lm = O.render_and_backward(gm, cam, target, double=True).loss
            out[k] = (lp - lm) / (2 * eps)
        if k % 32 == 31:
            print(f"{k + 1}/256 ({time.time() - t0:.0f} s)", flush=True)
    np.savez_compressed(OUT, gauss=gauss, field=field, fd=fd, fd_fine=fd_fine, eps=EPS, eps_fine=EPS_FINE, lam=LAMBDA,
                        analytic_fp64=base.grads[gauss], loss_fp64=base.loss,
                        scene_sha256=digest(g, target))
    print("wrote", OUT)


if __name__ == "__main__":
    main()
