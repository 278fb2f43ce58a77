"""train_blocking's schedule (src/pipeline/mod.rs:203-265) on the host, with a
stand-in trainer that records what the loop asks of it (no GPU)."""
import itertools
import os

import numpy as np

import rgsplat_b200 as R
from rgsplat_b200 import api


class FakeTrainer:
    def __init__(self, n_cams=7):
        self.cameras = [None] * n_cams
        self.calls = []

    def gaussians(self):
        g = np.zeros((2, 59), np.float32)
        g[1, :3] = (3.0, 4.0, 0.0)  # extent 5
        return g

    def step(self, views, bg, loss_cfg, train_cfg, mode):
        self.calls.append(("step", tuple(views), mode))
        return np.full(len(views), 0.5, np.float32)

    def densify_and_prune(self, cfg, extent):
        self.calls.append(("densify", extent))
        return 2

    def reset_opacities(self):
        self.calls.append(("reset",))

    def save_ply(self, path):
        self.calls.append(("save", os.path.basename(path)))


def test_camera_schedule_is_xorshift64():
    x = R.api.CAMERA_SEED
    m = (1 << 64) - 1
    want = []
    for _ in range(20):
        x ^= (x << 13) & m
        x ^= x >> 7
        x ^= (x << 17) & m
        want.append(x % 64)
    assert list(itertools.islice(R.camera_schedule(64), 20)) == want


def test_schedule_of_densify_reset_and_checkpoints(tmp_path):
    tr = FakeTrainer()
    cfg = R.TrainConfig(num_iterations=3101, densify_from_iter=500, densify_until_iter=1000, opacity_reset_iter=3000)
    seen = []
    losses = R.train_blocking(tr, cfg, save_interval=1000, out_dir=str(tmp_path),
                              before_densify=lambda it, t: seen.append(it),
                              after_densify=lambda it, t, n: seen.append(-n))
    assert losses.shape == (3101,) and np.all(losses == 0.5)
    steps = [c for c in tr.calls if c[0] == "step"]
    assert len(steps) == 3101 and all(len(c[1]) == 1 and c[2] == R.Trainer.PLAIN for c in steps)
    assert [c[1][0] for c in steps[:20]] == list(itertools.islice(R.camera_schedule(7), 20))
    dens = [it for it in seen if it > 0]
    assert dens == [500, 600, 700, 800, 900, 1000]
    assert all(c[1] == 5.0 for c in tr.calls if c[0] == "densify")
    assert sum(1 for c in tr.calls if c[0] == "reset") == 1
    assert [c[1] for c in tr.calls if c[0] == "save"] == ["ckpt_001000.ply", "ckpt_002000.ply", "ckpt_003000.ply"]
    # the reset at 3000 follows that iteration's step
    i = tr.calls.index(("reset",))
    assert tr.calls[i - 1][0] == "step" and sum(1 for c in tr.calls[:i] if c[0] == "step") == 3001


def test_batched_steps_take_consecutive_cameras():
    tr = FakeTrainer(n_cams=128)
    R.train_blocking(tr, R.TrainConfig(num_iterations=3), views_per_step=8)
    steps = [c for c in tr.calls if c[0] == "step"]
    flat = [v for c in steps for v in c[1]]
    assert flat == list(itertools.islice(R.camera_schedule(128), 24))
    assert all(c[2] == R.Trainer.BATCHED for c in steps)
    assert api.Trainer.BATCHED != api.Trainer.PLAIN
