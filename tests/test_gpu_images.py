"""Target upload (load_target, src/io/images.rs:55-82) through the C ABI: the
device converts 8-bit sRGB RGBA to the loss's linear RGBA f32, bit-identical
to the oracle, and a trainer given the bytes trains exactly as one given the
oracle's converted floats."""
import numpy as np
import pytest

import oracle as O
import rgsplat_b200 as R
from rgsplat_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return R.Context()


def test_every_byte_value_bit_exact(ctx):
    u = np.arange(256, dtype=np.uint8)
    img = np.stack([u, np.roll(u, 1), np.roll(u, 2), u[::-1]], 1)
    got = R.srgb8_to_linear(img, ctx=ctx)
    assert np.array_equal(got.view(np.uint32), O.srgb8_to_linear(img).view(np.uint32))


@pytest.mark.parametrize("w,h", [(1600, 1064), (1, 1), (33, 7)])
def test_image_bit_exact(ctx, w, h):
    rng = np.random.default_rng(w * 7 + h)
    img = rng.integers(0, 256, size=(h, w, 4), dtype=np.uint8)
    got = R.srgb8_to_linear(img, ctx=ctx)
    assert got.shape == (h, w, 4)
    assert np.array_equal(got.view(np.uint32), O.srgb8_to_linear(img.reshape(-1, 4)).reshape(h, w, 4).view(np.uint32))


def test_empty_and_bad_input(ctx):
    assert R.srgb8_to_linear(np.zeros((0, 4), np.uint8), ctx=ctx).shape == (0, 4)
    with pytest.raises(ValueError):
        R.srgb8_to_linear(np.zeros(6, np.uint8), ctx=ctx)


def test_trainer_target_from_bytes_matches_float_target():
    g = scenes.random_gaussians(3000, 5, 1.5, (-3.5, 0.7), (0.0, 1.5))
    cams = scenes.sphere_cameras(3, 4.0, [(96, 64), (80, 48)], 1.2)
    rng = np.random.default_rng(11)
    imgs = [rng.integers(0, 256, size=(c.height, c.width, 4), dtype=np.uint8) for c in cams]
    a = R.Trainer(g, cams)
    b = R.Trainer(g, cams)
    for i, im in enumerate(imgs):
        a.set_target_rgba8(i, im)
        b.set_target(i, O.srgb8_to_linear(im.reshape(-1, 4)))
    la = a.step([0, 1, 2])
    lb = b.step([0, 1, 2])
    assert np.array_equal(la.view(np.uint32), lb.view(np.uint32))
    with pytest.raises(ValueError):
        a.set_target_rgba8(0, imgs[1])
