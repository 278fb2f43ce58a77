"""rgs_photometric_loss_grad_noalloc against rgs_photometric_loss_grad.

The no-allocation variant exists for callers that must not allocate device
memory (an application whose own pool owns the GPU, or a latency-critical
path that cannot take cudaMalloc's implicit synchronisation). It runs the
same loss kernels on the caller's device buffers with its scratch in a static
device array that every call reuses, so its loss and dL/dpixel must equal the
context entry point's bit for bit on two calls in a row. This file is
collected last so a run that stops at its first failure has run everything
else first; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _images(seed, w, h):
    rng = np.random.default_rng(seed)
    rendered = rng.random(w * h * 3, dtype=np.float32)
    target = rng.random(w * h * 4, dtype=np.float32)
    return rendered, target


def _noalloc(lib, torch, rendered, target, w, h, lam, device=0):
    dev = torch.device(f"cuda:{device}")
    r = torch.from_numpy(rendered).to(dev)
    t = torch.from_numpy(target).to(dev)
    dl = torch.full((w * h * 3,), float("nan"), device=dev)
    loss = torch.full((1,), float("nan"), device=dev)
    err = C.create_string_buffer(256)
    stream = torch.cuda.current_stream(dev)
    rc = lib.rgs_photometric_loss_grad_noalloc(device, r.data_ptr(), t.data_ptr(), w, h, lam, loss.data_ptr(),
                                               dl.data_ptr(), stream.cuda_stream, err, len(err))
    assert rc == 0, err.value.decode()
    stream.synchronize()
    return float(loss.cpu()[0]), dl.cpu().numpy()


def test_noalloc_matches_context_entry_point_twice():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from rgsplat_b200 import _lib, api

    lib = _lib.load()
    ctx = api.Context(device=0)
    # two calls in a row, different sizes (ragged 32x32 loss blocks) and weights
    for seed, (w, h), lam in ((11, (200, 150), 0.2), (12, (333, 97), 0.35)):
        rendered, target = _images(seed, w, h)
        want_loss, want_dl = api.photometric_loss_grad(rendered, target, w, h, lam, ctx=ctx)
        got_loss, got_dl = _noalloc(lib, torch, rendered, target, w, h, lam)
        assert np.isfinite(got_loss) and np.all(np.isfinite(got_dl))
        assert np.float32(got_loss) == np.float32(want_loss)
        assert np.array_equal(got_dl, want_dl)


def test_noalloc_on_a_second_device():
    """The first call on each device sets that device up (scratch address and
    the loss kernel's shared-memory limit): a call on device 1 after device 0,
    before any context exists on device 1, must match the context entry point
    there. Needs two GPUs; skipped otherwise."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available() or torch.cuda.device_count() < 2:
        pytest.skip("needs two GPUs")
    from rgsplat_b200 import _lib, api

    lib = _lib.load()
    w, h, lam = 257, 130, 0.2
    rendered, target = _images(13, w, h)
    got = [_noalloc(lib, torch, rendered, target, w, h, lam, device=d) for d in (0, 1)]
    for d in (0, 1):
        want_loss, want_dl = api.photometric_loss_grad(rendered, target, w, h, lam, ctx=api.Context(device=d))
        assert np.float32(got[d][0]) == np.float32(want_loss)
        assert np.array_equal(got[d][1], want_dl)


def test_noalloc_rejects_images_beyond_scratch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from rgsplat_b200 import _lib

    lib = _lib.load()
    dummy = torch.zeros(4, device="cuda:0")
    p = dummy.data_ptr()
    err = C.create_string_buffer(256)
    # 4097 x 4096 needs 129 x 128 loss blocks > 16384: rejected before any launch
    rc = lib.rgs_photometric_loss_grad_noalloc(0, p, p, 4097, 4096, 0.2, p, p, None, err, len(err))
    assert rc == -6 and b"static scratch holds 16384" in err.value
    rc = lib.rgs_photometric_loss_grad_noalloc(0, None, p, 64, 64, 0.2, p, p, None, err, len(err))
    assert rc == -1 and err.value == b"null argument"
