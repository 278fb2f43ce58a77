"""SfM initialisation (gaussians_from_sfm + estimate_initial_scales,
src/pipeline/sfm.rs:365-450) through the C ABI: the device sort, window search
and KNN scales must give the oracle's Gaussians bit for bit, edge cases
(ties in x, signed zeros, coincident points, tiny clouds) included."""
import numpy as np
import pytest

import oracle as O
import rgsplat_b200 as R
from rgsplat_b200 import scenes
from tests import refcases as RC
from tests.test_oracle_pins import points3d_bin

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return R.Context()


def same(a, b):
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("n,seed,dup", [(1, 1, 0), (2, 2, 0), (3, 3, 0), (49, 4, 0), (50, 5, 0), (51, 6, 0),
                                        (400, 8, 60), (5000, 9, 300), (100_000, 10, 0)])
def test_gaussians_from_sfm_bit_exact(ctx, n, seed, dup):
    xyz, rgb = RC.sfm_cloud(n, seed, dup)
    assert same(R.gaussians_from_sfm(xyz, rgb, ctx=ctx), O.gaussians_from_sfm(xyz, rgb))


def test_full_size_cloud_bit_exact(ctx):
    """One million points, the size of the training workload's cloud."""
    rng = np.random.default_rng(17)
    xyz = rng.normal(size=(1_000_000, 3)) * np.array([4.0, 2.0, 3.0])
    xyz[::1000, 0] = np.round(xyz[::1000, 0], 1)  # many exact ties in x
    rgb = rng.integers(0, 256, size=(1_000_000, 3), dtype=np.uint8)
    assert same(R.gaussians_from_sfm(xyz, rgb, ctx=ctx), O.gaussians_from_sfm(xyz, rgb))


def test_every_x_equal_and_signed_zero_keys(ctx):
    rng = np.random.default_rng(3)
    xyz = rng.normal(size=(300, 3))
    xyz[:, 0] = 0.0
    xyz[::2, 0] = -0.0
    rgb = rng.integers(0, 256, size=(300, 3), dtype=np.uint8)
    assert same(R.gaussians_from_sfm(xyz, rgb, ctx=ctx), O.gaussians_from_sfm(xyz, rgb))
    xyz[:, 0] = -1e300  # negative keys, all tied
    assert same(R.gaussians_from_sfm(xyz, rgb, ctx=ctx), O.gaussians_from_sfm(xyz, rgb))


def test_empty_and_invalid(ctx):
    assert R.gaussians_from_sfm(np.zeros((0, 3)), np.zeros((0, 3), np.uint8), ctx=ctx).shape == (0, 59)
    bad = np.zeros((10, 3))
    bad[7, 2] = np.inf
    with pytest.raises(R.RgsError):
        R.gaussians_from_sfm(bad, np.zeros((10, 3), np.uint8), ctx=ctx)
    with pytest.raises(ValueError):
        R.gaussians_from_sfm(np.zeros((4, 3)), np.zeros((3, 3), np.uint8), ctx=ctx)
    # the context stays usable after the rejected cloud
    xyz, rgb = RC.sfm_cloud(64, 2)
    assert same(R.gaussians_from_sfm(xyz, rgb, ctx=ctx), O.gaussians_from_sfm(xyz, rgb))


def test_points3d_bin_and_trainer_init(tmp_path):
    xyz, rgb = RC.sfm_cloud(3000, 21, 40)
    p = tmp_path / "points3D.bin"
    data = points3d_bin(xyz, rgb, [k % 7 for k in range(3000)])
    p.write_bytes(data)
    cams = scenes.sphere_cameras(2, 8.0, [(64, 48)], 1.2)
    tr = R.Trainer(np.zeros((1, 59), np.float32), cams)
    px, pc = R.read_points3d_bin(p, ctx=tr.ctx)
    assert np.array_equal(px, xyz) and np.array_equal(pc, rgb)
    assert tr.init_from_sfm(px, pc) == 3000
    assert same(tr.gaussians(), O.gaussians_from_sfm(xyz, rgb))
    assert tr.adam_state().t == 0
    p.write_bytes(data[:-5])
    with pytest.raises(R.RgsError):
        R.read_points3d_bin(p, ctx=tr.ctx)
