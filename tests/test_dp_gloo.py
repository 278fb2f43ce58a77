"""Multi-process view-parallel training step (rgsplat_b200.dp) on CPU ranks.

Two gloo ranks split one batch of 8 views, each back-propagates its 4 views,
the gradient planes are all-reduced and both apply the same Adam update. The
result must equal one process stepping all 8 views (gradients summed over
views, denom += 8), and the ranks must stay bit-identical. The "trainer" here
is the CPU oracle behind the same backward / apply_adam interface as the
library's Trainer, so the host logic runs without a GPU.
"""
import os
import socket
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


class OracleTrainer:
    def __init__(self, g, cams, targets):
        import oracle as O
        import torch

        self.O = O
        self.g = g.copy()
        self.cams, self.targets = cams, targets
        self.state = O.AdamState(g.shape[0])
        self.grad = np.zeros((g.shape[0], 60), np.float32)
        self._t = torch.from_numpy(self.grad.reshape(-1))

    def backward(self, views, loss_cfg=None, mode=None):
        self.grad[:] = 0.0
        losses = []
        for v in views:
            out = self.O.render_and_backward(self.g, self.cams[v], self.targets[v])
            self.grad += out.grads
            losses.append(out.loss)
        return np.array(losses, np.float32)

    def grad_tensor(self):
        return self._t

    def apply_adam(self, train_cfg, denom_increment=1):
        self.O.adam_step(self.g, self.grad, self.state, self.O.TrainConfig())
        self.state.grad_denom += np.uint32(denom_increment - 1)


def scene():
    import oracle as O
    from rgsplat_b200 import scenes

    g = scenes.random_gaussians(300, 5, 1.0, (-3.0, 0.5), (0.0, 1.0))
    cams = scenes.sphere_cameras(8, 4.0, [(64, 48), (48, 40)], 1.2)
    tg = scenes.perturbed(g, 6)
    targets = []
    for c in cams:
        rgb, _, _ = O.render_color(tg, c)
        targets.append(np.concatenate([rgb, np.ones((c.height, c.width, 1), np.float32)], axis=2))
    return g, cams, targets


STEPS = ([0, 1, 2, 3, 4, 5, 6, 7], [7, 5, 3, 1, 6, 4, 2, 0])


def _rank(rank, world, port, out_dir):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    from rgsplat_b200 import dp

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        g, cams, targets = scene()
        tr = OracleTrainer(g, cams, targets)
        step = dp.ViewParallelStep(tr)
        assert step.world == world
        for views in STEPS:
            step(dp.split_views(views, rank, world))
        np.save(os.path.join(out_dir, f"params_{rank}.npy"), tr.g)
        np.save(os.path.join(out_dir, f"denom_{rank}.npy"), tr.state.grad_denom)
        np.save(os.path.join(out_dir, f"accum_{rank}.npy"), tr.state.grad_accum)
        # densification needs no exchange either: every rank holds the same
        # all-reduced statistics and parameters, so each densifies identically
        avg = tr.state.grad_accum / np.maximum(tr.state.grad_denom, 1)
        cfg = tr.O.TrainConfig(densify_grad_threshold=float(np.quantile(avg, 0.5)))
        dens = tr.O.densify_and_prune(tr.g, tr.state, cfg, tr.O.estimate_scene_extent(g))
        np.save(os.path.join(out_dir, f"densified_{rank}.npy"), dens)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_view_parallel_step_matches_single_process(tmp_path):
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp

    world = 2
    mp.start_processes(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn", join=True)
    p = [np.load(tmp_path / f"params_{r}.npy") for r in range(world)]
    # the ranks hold bit-identical parameters without any broadcast
    assert np.array_equal(p[0].view(np.uint32), p[1].view(np.uint32))
    assert np.array_equal(np.load(tmp_path / "denom_0.npy"), np.load(tmp_path / "denom_1.npy"))
    d = [np.load(tmp_path / f"densified_{r}.npy") for r in range(world)]
    assert d[0].shape[0] > p[0].shape[0] and np.array_equal(d[0].view(np.uint32), d[1].view(np.uint32))

    # one process, all 8 views per step
    g, cams, targets = scene()
    ref = OracleTrainer(g, cams, targets)
    for views in STEPS:
        ref.backward(views)
        ref.apply_adam(None, denom_increment=len(views))
    assert np.array_equal(np.load(tmp_path / "denom_0.npy"), ref.state.grad_denom)
    assert np.all(ref.state.grad_denom == 8 * len(STEPS))
    # gradients summed in a different order (per rank, then across ranks):
    # Adam moves each parameter by about lr per step, so compare at 1e-3 of lr
    lr = np.full(59, 0.000125, np.float32)
    lr[0:3], lr[3], lr[4:8], lr[8:11], lr[11:14] = 0.00016, 0.05, 0.001, 0.005, 0.0025
    assert (np.abs(p[0] - ref.g) <= len(STEPS) * 1e-3 * lr[None, :]).all()
    assert np.allclose(np.load(tmp_path / "accum_0.npy"), ref.state.grad_accum, rtol=1e-5, atol=1e-12)


def test_split_views_and_seeds():
    sys.path.insert(0, ROOT)
    from rgsplat_b200 import dp

    views = list(range(10))
    parts = [dp.split_views(views, r, 3) for r in range(3)]
    assert sorted(sum(parts, [])) == views and parts[0] == [0, 3, 6, 9]
    seeds = {dp.rank_seed(0x9E3779B97F4A7C15, r) for r in range(8)}
    assert len(seeds) == 8 and dp.rank_seed(0x9E3779B97F4A7C15, 0) == 0x9E3779B97F4A7C15


def _rank_with_dead_peer(rank, world, port, out_dir):
    import datetime

    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    from rgsplat_b200 import dp

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=5))
    if rank == 1:
        # this rank leaves between steps, with nothing in flight
        os._exit(0)
    g, cams, targets = scene()
    tr = OracleTrainer(g, cams, targets)
    step = dp.ViewParallelStep(tr)
    outcome = "completed"
    try:
        step(dp.split_views(STEPS[0], rank, world))
    except Exception as e:  # the survivor's collective fails instead of waiting for good
        outcome = "error: " + type(e).__name__
    with open(os.path.join(out_dir, "outcome.txt"), "w") as f:
        f.write(outcome)
    os._exit(0)


def test_dead_rank_fails_the_step_on_the_survivor(tmp_path):
    pytest.importorskip("torch")
    import time

    import torch.multiprocessing as mp

    t0 = time.time()
    ctx = mp.start_processes(_rank_with_dead_peer, args=(2, _free_port(), str(tmp_path)), nprocs=2, start_method="spawn",
                             join=False)
    while not ctx.join(timeout=60):
        assert time.time() - t0 < 120, "survivor did not finish"
    outcome = (tmp_path / "outcome.txt").read_text()
    assert outcome.startswith("error"), outcome
