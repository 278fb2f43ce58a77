"""The benchmarked workload at full size, against the oracle.

1M Gaussians (means U[-2, 2]^3, log-scales N(-4, 0.5), SH degree 3), 8 views
per step drawn by the reference's xorshift camera schedule from 128
Fibonacci-sphere cameras of 1600x1064, 1280x720 and 960x540 pixels: the step
the benchmark times, in the blend layout it tunes to (16x16 tiles, 128-splat
batches, 2 pixels per thread). At this size the batched pipeline runs paths no
smaller test reaches: ~50k CTA tiles over the batch (16-bit global tile ids),
~3.4k supertiles (two 8-bit passes of the supertile sort) over ~16M (supertile,
splat) entries, ~66M (tile, splat) pairs after pruning, ~8.5M pixels at
per-view offsets in one buffer.

Multi-view semantics (the reference trains one view per step,
src/pipeline/mod.rs:235-246): the batch's loss is the per-view losses and its
gradient the sum of the per-view GaussianGrads of ``render_and_backward``
(src/cpu/backward.rs:107-149), then one Adam step with grad_denom += 8. Bars:
every view's rendered image and final transmittance bit-exact against the
oracle's forward_pass (the stated image tolerance is 1e-4), dL/dpixel of the
benchmarked (fused-tap) loss within float rounding of the reference's and
bit-exact with exact_loss on the same images,
per-view losses within 1e-4 of the same image's loss summed in double (the
reference's serial f32 sum drifts by percents at this size), every gradient
group within 1e-3 relative, Gaussians the oracle leaves untouched have zero gradients, and the
parameters after the Adam step within the trainer tests' step tolerance.

The oracle runs each view on all host threads (~2 s per view on 16 threads).
"""
import itertools
import os

import numpy as np
import pytest

import oracle as O
import rgsplat_b200 as R
from rgsplat_b200 import debug as D
from rgsplat_b200 import scenes
from tests.test_gpu_parity import assert_dl_close
from tests.test_gpu_trainer import assert_steps_close

pytestmark = pytest.mark.gpu

GROUPS = {"position": slice(0, 3), "rotation": slice(3, 7), "log_scale": slice(7, 10), "opacity": slice(10, 11),
          "sh": slice(11, 59), "screen_grad_norm": slice(59, 60)}


@pytest.fixture(scope="module")
def headline():
    O.set_threads(os.cpu_count() or 1)
    cfg = scenes.config(3)
    g = scenes.make_gaussians(cfg)
    views = list(itertools.islice(R.camera_schedule(len(cfg.cameras)), cfg.views_per_step))
    ctx = R.Context(tile=(16, 16), batch=128, pixels_per_thread=2)
    painter = R.Trainer(scenes.perturbed(g, cfg.seed + 1), cfg.cameras, ctx=ctx)
    targets = {}
    for v in sorted(set(views)):
        rgb = painter.render(v)
        targets[v] = np.concatenate([rgb, np.ones(rgb.shape[:2] + (1,), np.float32)], axis=2)
    del painter
    tr = R.Trainer(g, cfg.cameras, ctx=ctx)
    for v, t in targets.items():
        tr.set_target(v, t)
    losses = tr.backward(views, mode=R.Trainer.BATCHED)
    stats = ctx.stats()
    pixels = [D.trainer_batch_pixels(tr, views, k) for k in range(len(views))]
    grads = tr.grads()
    ref = []
    total = np.zeros((g.shape[0], 60), np.float64)
    for v in views:
        out = O.render_and_backward(g, cfg.cameras[v], targets[v])
        total += out.grads
        ref.append((out.loss, out.rendered, out.final_t, out.dl_dpix))
    return dict(cfg=cfg, g=g, views=views, targets=targets, ctx=ctx, losses=losses, stats=stats, pixels=pixels,
                grads=grads, ref=ref, total=total)


def test_headline_batch_shape(headline):
    """The batch ran as one view group over the large-batch paths."""
    st, cfg, views = headline["stats"], headline["cfg"], headline["views"]
    assert st["view_groups"] == 1
    assert st["pairs"] > 1 << 25
    tiles = sum(((cfg.cameras[v].width + 15) // 16) * ((cfg.cameras[v].height + 15) // 16) for v in views)
    assert tiles > 1 << 15  # 16-bit global tile ids
    # more supertiles than one 8-bit sort pass orders, each splat binned once per
    # supertile it meets (fewer entries than pairs)
    supertiles = sum(((cfg.cameras[v].width + 63) // 64) * ((cfg.cameras[v].height + 63) // 64) for v in views)
    assert supertiles > 1 << 8
    assert st["visible"] < st["supertile_entries"] < st["pairs"]


def test_headline_images_bit_exact_and_pixel_gradients(headline):
    """Images and final T bit-exact; the batched step's dL/dpixel (fused blur
    taps) within float rounding of the reference's; the same images through
    an exact_loss context give the reference's dL/dpixel bit for bit."""
    cfg, targets = headline["cfg"], headline["targets"]
    exact_ctx = R.Context(exact_loss=True)
    for k, v in enumerate(headline["views"]):
        rgb, ft, dl = headline["pixels"][k]
        _, ref_rgb, ref_ft, ref_dl = headline["ref"][k]
        assert np.array_equal(rgb.view(np.uint32), ref_rgb.view(np.uint32)), f"view {v}: rgb"
        assert np.array_equal(ft.view(np.uint32), ref_ft.view(np.uint32)), f"view {v}: final T"
        c = cfg.cameras[v]
        _, xdl = O.photometric_loss_grad(ref_rgb, targets[v], c.width, c.height, 0.2, double=True)
        assert_dl_close(dl, ref_dl, xdl)
        _, dl_e = R.photometric_loss_grad(rgb, targets[v], c.width, c.height, 0.2, ctx=exact_ctx)
        assert np.array_equal(dl_e.reshape(-1).view(np.uint32), ref_dl.reshape(-1).view(np.uint32)), f"view {v}"


def test_headline_losses(headline):
    """Per-view losses against the same image's loss summed in double: within
    1e-4 relative (the library sums each 32x32 block in f32 and the blocks in
    double). The reference sums the loss serially in f32 (backward.rs:646-693,
    restated by the float oracle); over the 1.5M-5.1M terms of these views that
    sum drifts by several percent (4.2 % low at 1600x1064), so the float
    oracle's value is no bar here: the library's value is closer to the exact
    one. The loss is reported, never differentiated."""
    cfg, views, targets = headline["cfg"], headline["views"], headline["targets"]
    got = headline["losses"].astype(np.float64)
    serial_f32 = np.array([r[0] for r in headline["ref"]])
    for k, v in enumerate(views):
        c = cfg.cameras[v]
        exact, _ = O.photometric_loss_grad(headline["ref"][k][1], targets[v], c.width, c.height, 0.2, double=True)
        assert abs(got[k] - exact) <= 1e-4 * exact, (v, got[k], exact)
        assert abs(got[k] - exact) <= abs(serial_f32[k] - exact), (v, got[k], serial_f32[k], exact)


def test_headline_gradients_match_oracle_sum(headline):
    grads, total = headline["grads"].astype(np.float64), headline["total"]
    for name, sl in GROUPS.items():
        e = np.linalg.norm(grads[:, sl] - total[:, sl]) / np.linalg.norm(total[:, sl])
        assert e < 1e-3, f"{name}: relative error {e:.2e}"
    untouched = ~np.any(total != 0.0, axis=1)
    assert untouched.sum() > 0
    assert not np.any(grads[untouched] != 0.0)


def test_headline_step_matches_oracle_adam(headline):
    cfg, g, views, targets = headline["cfg"], headline["g"], headline["views"], headline["targets"]
    tr = R.Trainer(g, cfg.cameras, ctx=headline["ctx"])
    for v, t in targets.items():
        tr.set_target(v, t)
    losses = tr.step(views, mode=R.Trainer.BATCHED)
    assert np.array_equal(losses, headline["losses"])
    go = g.copy()
    so = O.AdamState(g.shape[0])
    O.adam_step(go, headline["total"].astype(np.float32), so, O.TrainConfig())
    so.grad_denom += np.uint32(len(views) - 1)
    assert_steps_close(tr.gaussians(), go, 1)
    st = tr.adam_state()
    assert st.t == 1
    assert np.array_equal(st.grad_denom[: g.shape[0]], so.grad_denom)
    assert np.allclose(st.grad_accum[: g.shape[0]], so.grad_accum, rtol=1e-3, atol=1e-9)
