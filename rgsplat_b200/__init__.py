"""rgsplat_b200: rgsplat's differentiable Gaussian-splatting training step on B200.

The compute lives in ``librgsplat_b200.so`` (hand-written sm_100a CUDA behind
the C ABI of ``include/rgsplat.h``); this package is its host-side mirror of
the reference crate's API. See ``rgsplat_b200.api``.
"""
from .api import (  # noqa: F401
    AdamState,
    Camera,
    Context,
    GpuRenderer,
    LossConfig,
    RgsError,
    TrainConfig,
    Trainer,
    adam_step,
    default_context,
    densify_and_prune,
    estimate_scene_extent,
    photometric_loss_grad,
    rasterize,
    black_target,
    srgb8_to_linear,
    gaussians_from_sfm,
    read_points3d_bin,
    load_ply,
    save_ply,
    save_splat,
    render_and_backward,
    render_and_backward_variant,
    render_color,
    reset_opacities,
    camera_schedule,
    train_blocking,
)

__version__ = "0.1.0"
