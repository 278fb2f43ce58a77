"""The CUDA path against the reference's own transcendentals.

The reference evaluates every exp / ln with the platform libm (Rust's f32::exp
and f32::ln call glibc's expf / logf on Linux): alpha = opacity * exp(power)
per (pixel, splat) (src/cpu/backward.rs:344, :444), the SSIM window
(backward.rs:764), sigmoid / logit and the scale decode
(src/math/mod.rs:72-78, :183-192). The kernels evaluate them with the
library's own deterministic routines, and the oracle by default with the same
routines, which is what makes the other parity tests bit-exact. Here the
oracle switches to glibc (``set_libm_math(True)``), i.e. to the reference's
arithmetic, and the CUDA results are held to the stated tolerances against it:

* tile lists bit-exact except for entries whose 3-sigma rectangle flipped at a
  truncation boundary (counted, at most 1 per million pairs plus 2);
* rendered image and final transmittance within 1e-4 max abs at every pixel
  whose last contributor agrees; pixels where an alpha >= 1/255 or T < 1e-4
  decision flipped (counted by the last contributor) at most 1 per 100k
  pixels plus 2;
* loss within 1e-4 relative of the reference image's loss summed in double
  (the reference's own serial f32 sum drifts by percents on a 1600x1064
  image, so its value is no bar there), every gradient group within 1e-3
  relative.

Workloads: the 10k-Gaussian 256x256 view, the 50k-Gaussian 512x512 view and
one 1600x1064 view of the 1M-Gaussian scene. The flip counts are printed
(``pytest -s``).
"""
import os

import numpy as np
import pytest

import oracle as O
import rgsplat_b200 as R
from rgsplat_b200 import debug as D
from rgsplat_b200 import scenes

pytestmark = pytest.mark.gpu

GROUPS = {"position": slice(0, 3), "rotation": slice(3, 7), "log_scale": slice(7, 10), "opacity": slice(10, 11),
          "sh": slice(11, 59), "screen_grad_norm": slice(59, 60)}


@pytest.fixture
def libm():
    O.set_threads(os.cpu_count() or 1)
    O.set_libm_math(True)
    try:
        yield
    finally:
        O.set_libm_math(False)


def tile_list_flips(a_off, a_ent, b_off, b_ent) -> int:
    """Entries present in one set of tile lists and not the other (order kept
    within a tile, so a reordering counts too)."""
    if np.array_equal(a_off, b_off) and np.array_equal(a_ent, b_ent):
        return 0
    flips = 0
    for t in range(a_off.shape[0] - 1):
        x = a_ent[a_off[t]:a_off[t + 1]]
        y = b_ent[b_off[t]:b_off[t + 1]]
        if x.shape == y.shape and np.array_equal(x, y):
            continue
        flips += len(set(x.tolist()) ^ set(y.tolist())) or max(len(x), 1)
    return flips


@pytest.mark.parametrize("case", ["10k_256", "50k_512", "1M_1600x1064"])
def test_cuda_path_against_libm_reference_math(case, libm):
    if case == "10k_256":
        cfg = scenes.config(0)
        cam = cfg.cameras[0]
    elif case == "50k_512":
        cfg = scenes.config(2)
        cam = cfg.cameras[0]
    else:
        cfg = scenes.config(3)
        cam = cfg.cameras[0]
    g = scenes.make_gaussians(cfg)
    rgb_t, _, _ = O.render_color(scenes.perturbed(g, cfg.seed + 1), cam)
    target = np.concatenate([rgb_t, np.ones((cam.height, cam.width, 1), np.float32)], axis=2)
    ctx = R.Context()

    ref = O.render_and_backward(g, cam, target)
    r_off, r_ent = O.tile_lists(g, cam)
    loss, grads = R.render_and_backward(g, cam, target, ctx=ctx)
    rgb, ft, last = D.forward(g, cam, ctx=ctx)
    g_off, g_ent = D.tile_lists(g, cam, ctx=ctx)

    pairs = int(r_ent.shape[0])
    tflips = tile_list_flips(g_off, g_ent, r_off, r_ent)
    px = cam.width * cam.height
    pflip = last != ref.last_contrib
    npf = int(pflip.sum())
    keep = ~pflip
    img_err = float(np.abs(rgb - ref.rendered)[keep].max()) if keep.any() else 0.0
    t_err = float(np.abs(ft - ref.final_t)[keep].max()) if keep.any() else 0.0
    rel = {k: float(np.linalg.norm(grads[:, s] - ref.grads[:, s]) / max(np.linalg.norm(ref.grads[:, s]), 1e-30))
           for k, s in GROUPS.items()}
    exact, _ = O.photometric_loss_grad(ref.rendered, target, cam.width, cam.height, 0.2, double=True)
    print(f"\n[{case}] pairs {pairs}, tile-list flips {tflips}; pixels {px}, last-contributor flips {npf}; "
          f"image max abs {img_err:.3e}, final T max abs {t_err:.3e}; loss rel to the double sum "
          f"{abs(loss - exact) / exact:.3e} (reference's f32 sum {abs(ref.loss - exact) / exact:.3e}); gradient rel " + ", ".join(f"{k} {v:.2e}" for k, v in rel.items()))

    assert tflips <= pairs // 1_000_000 + 2
    assert npf <= px // 100_000 + 2
    assert img_err <= 1e-4 and t_err <= 1e-4
    assert abs(loss - exact) <= 1e-4 * exact
    for k, e in rel.items():
        assert e < 1e-3, f"{k}: {e:.2e}"
