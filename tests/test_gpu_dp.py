"""The device side of the view-parallel multi-GPU step, on one GPU.

A rank of ``rgsplat_b200.dp.ViewParallelStep`` runs the gradient-only pass
(``rgs_trainer_backward``: the render + backward pipeline with the geometry
kernel writing gradient planes instead of applying Adam), hands the library's
gradient planes to NCCL as a zero-copy torch tensor
(``rgs_trainer_grad_buffer``), and applies Adam separately
(``rgs_trainer_apply_adam`` with grad_denom += views x ranks). The reference
step being sharded is src/pipeline/mod.rs:235-246.

The blend backward adds each splat's per-tile partial gradients with global
float atomics, so two runs of a pass agree to rounding, not bit for bit.
What is exact is checked exactly:
* given the gradients a pass produced, the separate Adam update equals the
  oracle's adam_step (src/pipeline/optimizer.rs:116-163) on those gradients
  bit for bit, with grad_denom += views;
* a one-rank NCCL all-reduce of the zero-copy tensor leaves the planes
  bit-identical;
and the split step tracks the fused single-process step
(``rgs_trainer_step``) within the trainer tests' step tolerance.
The two-rank exchange itself runs on CPU in tests/test_dp_gloo.py (gloo,
oracle trainer).
"""
import numpy as np
import pytest

import oracle as O
import rgsplat_b200 as R
from rgsplat_b200 import dp
from tests.test_gpu_trainer import assert_steps_close, multi_view_scene

pytestmark = pytest.mark.gpu

STEPS = [[0, 2, 3, 5], [1, 4, 4, 0], [5, 3, 2, 1]]


def oracle_state(st: R.AdamState, n: int) -> O.AdamState:
    so = O.AdamState(n)
    so.m1[:] = st.m1[: n * 59]
    so.m2[:] = st.m2[: n * 59]
    so.grad_accum[:] = st.grad_accum[:n]
    so.grad_denom[:] = st.grad_denom[:n]
    so.t = st.t
    return so


def check_adam_against_oracle(tr, before_g, before_st, grads, nviews):
    """tr has just applied Adam to `grads`: compare with the oracle's update."""
    n = before_g.shape[0]
    go = before_g.copy()
    so = oracle_state(before_st, n)
    O.adam_step(go, grads, so, O.TrainConfig())
    so.grad_denom += np.uint32(nviews - 1)
    after = tr.adam_state()
    assert np.array_equal(tr.gaussians().view(np.uint32), go.view(np.uint32))
    assert np.array_equal(after.m1[: n * 59].view(np.uint32), so.m1.view(np.uint32))
    assert np.array_equal(after.m2[: n * 59].view(np.uint32), so.m2.view(np.uint32))
    assert np.array_equal(after.grad_accum[:n].view(np.uint32), so.grad_accum.view(np.uint32))
    assert np.array_equal(after.grad_denom[:n], so.grad_denom)
    assert after.t == so.t


@pytest.mark.parametrize("mode", [R.Trainer.BATCHED, R.Trainer.PLAIN])
def test_gradient_pass_then_adam(mode):
    g, cams, targets = multi_view_scene(n=4000, seed=31)
    split = R.Trainer(g, cams, targets)
    fused = R.Trainer(g, cams, targets)
    for views in STEPS:
        before_g, before_st = split.gaussians(), split.adam_state()
        ls = split.backward(views, mode=mode)
        grads = split.grads()
        split.apply_adam(R.TrainConfig(), denom_increment=len(views))
        check_adam_against_oracle(split, before_g, before_st, grads, len(views))
        lf = fused.step(views, mode=mode)
        assert np.allclose(ls, lf, rtol=1e-5, atol=1e-8)
    assert_steps_close(split.gaussians(), fused.gaussians(), len(STEPS))
    a, b = split.adam_state(), fused.adam_state()
    assert a.t == b.t == len(STEPS)
    assert np.array_equal(a.grad_denom, b.grad_denom)


def test_grad_buffer_tensor_is_the_gradient_planes():
    """The zero-copy torch view of rgs_trainer_grad_buffer holds exactly the
    gradients rgs_trainer_get_grads returns (15 float4 planes of
    `plane_stride` Gaussians; record order per optimizer.rs:165-173)."""
    pytest.importorskip("torch")
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
    """In a one-rank NCCL process group: an all-reduce of the library's
    gradient planes through the zero-copy tensor leaves them bit-identical and
    the update that follows equals the oracle's; ViewParallelStep tracks the
    fused step."""
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
        planes = dp.trainer_grad_tensor(reduced, "cuda:0")
        for views in STEPS:
            before_g, before_st = reduced.gaussians(), reduced.adam_state()
            reduced.backward(views, mode=R.Trainer.BATCHED)
            g0 = reduced.grads()
            dist.all_reduce(planes)  # one rank: the sum is the planes themselves
            torch.cuda.current_stream(0).synchronize()
            assert np.array_equal(reduced.grads().view(np.uint32), g0.view(np.uint32))
            reduced.apply_adam(R.TrainConfig(), denom_increment=len(views))
            check_adam_against_oracle(reduced, before_g, before_st, g0, len(views))
            l0 = step(views)
            l2 = fused.step(views, mode=R.Trainer.BATCHED)
            assert np.allclose(l0, l2, rtol=1e-5, atol=1e-8)
        assert_steps_close(stepper.gaussians(), fused.gaussians(), len(STEPS))
        assert np.array_equal(stepper.adam_state().grad_denom, fused.adam_state().grad_denom)
    finally:
        dist.destroy_process_group()
