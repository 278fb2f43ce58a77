"""The device side of the view-parallel multi-GPU step, on one GPU.

A rank of ``rgsplat_b200.dp.ViewParallelStep`` runs the gradient-only pass
(``rgs_trainer_backward``: the batched pipeline with the geometry kernel
writing gradient planes instead of applying Adam), hands the library's
gradient planes to NCCL as a zero-copy torch tensor
(``rgs_trainer_grad_buffer``), and applies Adam separately
(``rgs_trainer_apply_adam`` with grad_denom += views x ranks). With one rank
that sum is the identity, so the split step must equal the single-process
fused step (``rgs_trainer_step``: geometry backward and Adam in one kernel
pass, src/pipeline/mod.rs:235-246 per view) bit for bit: parameters, both
moments, grad_accum and grad_denom. The two-rank exchange itself runs on CPU
in tests/test_dp_gloo.py (gloo, oracle trainer); this file checks the kernels
and buffers that exchange reads and writes on a GPU.
"""
import numpy as np
import pytest

import rgsplat_b200 as R
from rgsplat_b200 import dp
from tests.test_gpu_trainer import multi_view_scene

pytestmark = pytest.mark.gpu

STEPS = [[0, 2, 3, 5], [1, 4, 4, 0], [5, 3, 2, 1]]


def assert_same_state(a, b):
    ga, gb = a.gaussians(), b.gaussians()
    assert np.array_equal(ga.view(np.uint32), gb.view(np.uint32))
    sa, sb = a.adam_state(), b.adam_state()
    assert sa.t == sb.t
    for name in ("m1", "m2", "grad_accum"):
        x, y = getattr(sa, name), getattr(sb, name)
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), name
    assert np.array_equal(sa.grad_denom, sb.grad_denom)


@pytest.mark.parametrize("mode", [R.Trainer.BATCHED, R.Trainer.PLAIN])
def test_gradient_pass_then_adam_equals_fused_step(mode):
    g, cams, targets = multi_view_scene(n=4000, seed=31)
    split = R.Trainer(g, cams, targets)
    fused = R.Trainer(g, cams, targets)
    for views in STEPS:
        ls = split.backward(views, mode=mode)
        split.apply_adam(R.TrainConfig(), denom_increment=len(views))
        lf = fused.step(views, mode=mode)
        assert np.array_equal(ls, lf)
    assert_same_state(split, fused)


def test_grad_buffer_tensor_is_the_gradient_planes():
    """The zero-copy torch view of rgs_trainer_grad_buffer holds exactly the
    gradients rgs_trainer_get_grads returns (plane layout: 15 float4 planes of
    `plane_stride` floats, record order per optimizer.rs:165-173)."""
    torch = pytest.importorskip("torch")
    g, cams, targets = multi_view_scene(n=3000, seed=32)
    tr = R.Trainer(g, cams, targets)
    tr.backward([1, 3, 4], mode=R.Trainer.BATCHED)
    ptr, nbytes, stride = tr.grad_buffer()
    t = dp.trainer_grad_tensor(tr, "cuda:0")
    assert t.numel() * 4 == nbytes and t.data_ptr() == ptr
    planes = t.cpu().numpy()[: 15 * stride * 4].reshape(15, stride, 4)[:, : g.shape[0]]
    grads = tr.grads()
    # GaussianGrad: d_position[3], d_rotation[4], d_log_scale[3], d_opacity_logit, d_sh[48], screen_grad_norm
    assert np.array_equal(planes[0, :, :3], grads[:, 0:3])
    assert np.array_equal(planes[0, :, 3], grads[:, 10])
    assert np.array_equal(planes[1], grads[:, 3:7])
    assert np.array_equal(planes[2, :, :3], grads[:, 7:10])
    assert np.array_equal(planes[2, :, 3], grads[:, 59])
    assert np.array_equal(planes[3:].transpose(1, 0, 2).reshape(-1, 48), grads[:, 11:59])


def test_view_parallel_step_under_a_one_rank_nccl_group():
    """ViewParallelStep and an explicit NCCL all-reduce of the library's
    gradient planes, in a one-rank process group, against the fused step."""
    torch = pytest.importorskip("torch")
    import datetime
    import socket

    import torch.distributed as dist

    if not dist.is_nccl_available():
        pytest.skip("no NCCL")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60), device_id=torch.device("cuda", 0))
    try:
        g, cams, targets = multi_view_scene(n=4000, seed=33)
        stepper = R.Trainer(g, cams, targets)
        reduced = R.Trainer(g, cams, targets)
        fused = R.Trainer(g, cams, targets)
        step = dp.ViewParallelStep(stepper, device="cuda:0", mode=R.Trainer.BATCHED)
        grads = dp.trainer_grad_tensor(reduced, "cuda:0")
        for views in STEPS:
            l0 = step(views)
            l1 = reduced.backward(views, mode=R.Trainer.BATCHED)
            dist.all_reduce(grads)  # one rank: the sum is the planes themselves
            torch.cuda.current_stream(0).synchronize()
            reduced.apply_adam(R.TrainConfig(), denom_increment=len(views))
            l2 = fused.step(views, mode=R.Trainer.BATCHED)
            assert np.array_equal(l0, l2) and np.array_equal(l1, l2)
        assert_same_state(stepper, fused)
        assert_same_state(reduced, fused)
    finally:
        dist.destroy_process_group()
