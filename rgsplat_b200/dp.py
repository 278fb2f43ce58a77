"""View-parallel data parallelism for the training step (one process per GPU).

Every rank holds all N Gaussians and the same Adam state. A step renders and
back-propagates the rank's own views (gradients only, no optimiser update),
sums the dense gradient planes over ranks with one all-reduce (NCCL between
GPUs), and applies the same Adam update everywhere with
grad_denom += (views per rank) x (ranks), which is what the single-process
multi-view step does with all views at once (gradients summed over views,
one Adam step, denom += views). Parameters therefore stay bit-identical
across ranks without any broadcast.

The reference trains one view per step on one device
(src/pipeline/mod.rs:203-265); this module is the multi-device extension of
its step. It is plain host logic over torch.distributed: the trainer object
supplies ``backward``, ``grad_tensor`` and ``apply_adam``.
"""
from __future__ import annotations

from typing import Sequence


class CudaArray:
    """Zero-copy torch view of a device buffer owned by the library
    (``torch.as_tensor(CudaArray(ptr, nbytes), device=...)``)."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (nbytes // 4,), "typestr": "<f4", "data": (ptr, False), "version": 3,
                                         "strides": None}


def rank_seed(base: int, rank: int) -> int:
    """Per-rank xorshift64 seed for the camera schedule (src/pipeline/mod.rs:224-230
    uses 0x9E3779B97F4A7C15 on one device; rank r offsets it)."""
    return (base ^ (rank * 0x5851F42D4C957F2D)) & ((1 << 64) - 1) or base


def split_views(views: Sequence[int], rank: int, world: int) -> list[int]:
    """Rank `rank`'s share of one global batch of views (round robin)."""
    return list(views[rank::world])


def trainer_grad_tensor(trainer, device):
    """The trainer's device gradient planes as a flat float32 torch tensor."""
    import torch

    ptr, nbytes, _ = trainer.grad_buffer()
    return torch.as_tensor(CudaArray(ptr, nbytes), device=device)


class ViewParallelStep:
    """One training step per call over this rank's views.

    trainer: object with ``backward(views, loss_cfg=..., mode=...) -> losses``,
    ``apply_adam(train_cfg, denom_increment=...)`` and a gradient tensor
    (``grad_tensor()`` or, for the library's Trainer, its device buffer).
    """

    def __init__(self, trainer, group=None, device=None, mode=None):
        import torch.distributed as dist

        self.trainer = trainer
        self.group = group
        self.dist = dist
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.device = device
        self.mode = mode

    def _grad(self):
        if hasattr(self.trainer, "grad_tensor"):
            return self.trainer.grad_tensor()
        return trainer_grad_tensor(self.trainer, self.device)

    def _order_after_collective(self) -> None:
        """The all-reduce is enqueued on torch's current stream; the update runs
        on the library context's stream. Unless they are the same stream, the
        host waits for the collective before the update is issued, so Adam
        never reads gradient planes the collective is still writing."""
        ctx = getattr(self.trainer, "ctx", None)
        if ctx is None or self.device is None:
            return
        import torch

        cur = torch.cuda.current_stream(self.device)
        if getattr(ctx, "stream", None) != cur.cuda_stream:
            cur.synchronize()

    def __call__(self, views: Sequence[int], loss_cfg=None, train_cfg=None):
        kw = {"loss_cfg": loss_cfg}
        if self.mode is not None:
            kw["mode"] = self.mode
        # the backward returns with its work finished (it reads the losses back)
        losses = self.trainer.backward(list(views), **kw)
        if self.world > 1:
            self.dist.all_reduce(self._grad(), group=self.group)
            self._order_after_collective()
        self.trainer.apply_adam(train_cfg, denom_increment=len(views) * self.world)
        return losses
