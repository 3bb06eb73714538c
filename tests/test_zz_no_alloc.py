"""lpaici_backward_noalloc (adjoint with its workspace in a static device array, no allocation) against
lpaici_backward, called through the C ABI.  Collected last, so it runs both alone and after every other
test has used the library on the same device.

Tolerance: the same as the adjoint tests, |got - ref| <= 2e-5 * max|ref| + 1e-6 (both entry points run
the same FP32 kernels)."""
import ctypes as C

import numpy as np
import pytest

import lpaici
import oracle_bind as ob
from conftest import GAUSS_M2, SYM, kernel_file

SIGMA_20 = float(np.float32(20.0) / np.float32(255.0))
SIGMA_25 = float(np.float32(25.0) / np.float32(255.0))
RTOL = 2e-5
SCRATCH_BYTES = 64 << 20  # LPAICI_NOALLOC_SCRATCH_BYTES


def _call(name, ks, x, g, out, sigma, gamma):
    import torch

    fn = getattr(lpaici.lib(), name)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = fn(ks.handle, C.c_void_p(x.data_ptr()), x.stride(0), C.c_void_p(g.data_ptr()), g.stride(0),
            C.c_void_p(out.data_ptr()), out.stride(0), x.shape[1], x.shape[0], sigma, gamma, stream)
    assert rc == lpaici.OK, lpaici.lib().lpaici_last_error().decode()
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _inputs(W, H, sigma, seed):
    import torch

    noisy = lpaici.add_noise(lpaici.synth_image(W, H, seed), sigma, 20250910 + seed)
    g = np.random.default_rng(seed).standard_normal((H, W)).astype(np.float32)
    return noisy, g, torch.from_numpy(noisy).cuda(), torch.from_numpy(g).cuda()


def _close(got, ref):
    err = np.abs(got - ref).max()
    assert err <= RTOL * np.abs(ref).max() + 1e-6, (err, np.abs(ref).max())


@pytest.mark.gpu
def test_noalloc_matches_backward_two_calls_in_a_row():
    """Two consecutive calls with different kernel sets and sizes (the second near the scratch limit)
    share the scratch; each equals lpaici_backward, the first also the FP64 oracle's adjoint."""
    import torch

    cases = [(SYM, 257, 131, SIGMA_20, 2.0, 21), (GAUSS_M2, 1920, 1080, SIGMA_25, 1.5, 22)]
    results = []
    for name, W, H, sigma, gamma, seed in cases:
        ks = lpaici.KernelSet.load(kernel_file(name))
        noisy, g, xt, gt = _inputs(W, H, sigma, seed)
        out = torch.full((H, W), float("nan"), device="cuda")
        got = _call("lpaici_backward_noalloc", ks, xt, gt, out, sigma, gamma)
        results.append((name, ks, noisy, g, sigma, gamma, got, xt, gt))
    for name, ks, noisy, g, sigma, gamma, got, xt, gt in results:
        ref = _call("lpaici_backward", ks, xt, gt, torch.empty_like(xt), sigma, gamma)
        assert np.isfinite(got).all()
        _close(got, ref)
    name, ks, noisy, g, sigma, gamma, got = results[0][:7]
    ko = ob.oracle_load_kernels(kernel_file(name))
    var = ks.variances(sigma)
    _, smap, _ = ob.oracle_forward_f32(noisy, ko, var, gamma, want_map=True)
    _close(got, ob.oracle_adjoint_f64(ko, var, smap, g.astype(np.float64)))


@pytest.mark.gpu
def test_noalloc_pitched_buffers_and_repeat():
    """Pitched input, cotangent and gradient views; the same call twice gives the same gradient."""
    import torch

    ks = lpaici.KernelSet.load(kernel_file(SYM))
    W, H = 300, 201
    noisy, g, xt, gt = _inputs(W, H, SIGMA_20, 23)
    xp = torch.zeros((H, W + 13), device="cuda")
    xp[:, :W] = xt
    gp = torch.zeros((H, W + 7), device="cuda")
    gp[:, :W] = gt
    op = torch.full((H, W + 5), float("nan"), device="cuda")
    a = _call("lpaici_backward_noalloc", ks, xp[:, :W], gp[:, :W], op[:, :W], SIGMA_20, 2.0)
    b = _call("lpaici_backward_noalloc", ks, xp[:, :W], gp[:, :W], op[:, :W], SIGMA_20, 2.0)
    ref = _call("lpaici_backward", ks, xt, gt, torch.empty_like(xt), SIGMA_20, 2.0)
    _close(a, ref)
    _close(b, ref)
    assert np.isnan(op[:, W:].cpu().numpy()).all()  # nothing written outside the gradient's columns


def _r256(n: int) -> int:
    return (n + 255) & ~255


def _scratch_need(ks, W: int, H: int) -> int:
    """Bytes lpaici_backward_noalloc needs: the two device kernel blobs (sizes from the kernel set's
    info), each 256-rounded, then D*W*H selection bytes (256-rounded) and W*H floats of 1/den."""
    info = ks.info
    return _r256(info.blob_bytes) + _r256(info.adjoint_blob_bytes) + _r256(ks.D * W * H) + 4 * W * H


def _largest_rows(ks, W: int) -> int:
    H = SCRATCH_BYTES // (ks.D + 4) // W
    while _scratch_need(ks, W, H + 1) <= SCRATCH_BYTES:
        H += 1
    while _scratch_need(ks, W, H) > SCRATCH_BYTES:
        H -= 1
    return H


def test_noalloc_size_limit_is_exact():
    """The largest image the scratch holds is accepted and one more row is rejected, both before any
    device work.  The rejected call never touches its (fake) pointers; the accepted one is made only
    where no CUDA device is visible, so it stops at the first CUDA call."""
    import torch

    ks = lpaici.KernelSet.load(kernel_file(SYM))
    lib = lpaici.lib()
    fake = C.c_void_p(256)
    W = 1920
    H = _largest_rows(ks, W)
    assert _scratch_need(ks, W, H) <= SCRATCH_BYTES < _scratch_need(ks, W, H + 1)
    rc = lib.lpaici_backward_noalloc(ks.handle, fake, W, fake, W, fake, W, W, H + 1, SIGMA_20, 2.0, None)
    assert rc == lpaici.ERR_UNSUPPORTED
    assert f"needs {_scratch_need(ks, W, H + 1)} bytes" in lib.lpaici_last_error().decode()
    if not torch.cuda.is_available():
        rc = lib.lpaici_backward_noalloc(ks.handle, fake, W, fake, W, fake, W, W, H, SIGMA_20, 2.0, None)
        assert rc != lpaici.OK and "needs" not in lib.lpaici_last_error().decode()


def test_noalloc_rejects_bad_parameters_before_any_copy():
    """Non-finite sigma or gamma and more scales than the selection sweep keeps are refused up front."""
    ks = lpaici.KernelSet.load(kernel_file(SYM))
    lib = lpaici.lib()
    fake = C.c_void_p(256)
    for sigma, gamma in ((float("inf"), 2.0), (SIGMA_20, float("inf")), (float("nan"), 2.0), (SIGMA_20, 0.0)):
        rc = lib.lpaici_backward_noalloc(ks.handle, fake, 8, fake, 8, fake, 8, 8, 8, sigma, gamma, None)
        assert rc == lpaici.ERR_INVALID_ARG, (sigma, gamma)
        assert "finite positive" in lib.lpaici_last_error().decode()


@pytest.mark.gpu
def test_noalloc_at_the_size_limit():
    """The largest accepted image (1920 columns): the blob offsets and the 1/den tail at the end of the
    scratch are right, so the gradient equals lpaici_backward's."""
    import torch

    ks = lpaici.KernelSet.load(kernel_file(SYM))
    W = 1920
    H = _largest_rows(ks, W)
    noisy, g, xt, gt = _inputs(W, H, SIGMA_20, 24)
    out = torch.full((H, W), float("nan"), device="cuda")
    got = _call("lpaici_backward_noalloc", ks, xt, gt, out, SIGMA_20, 2.0)
    ref = _call("lpaici_backward", ks, xt, gt, torch.empty_like(xt), SIGMA_20, 2.0)
    assert np.isfinite(got).all()
    _close(got, ref)


def test_noalloc_rejects_images_beyond_the_scratch():
    """Sizes are checked before any CUDA call, so this runs without a GPU: the pointers are never used."""
    ks = lpaici.KernelSet.load(kernel_file(SYM))
    lib = lpaici.lib()
    fake = C.c_void_p(256)
    W = H = 2048  # 16 directions: 16 * 4 Mpx selection bytes alone exceed 64 MiB
    assert 20 * W * H > SCRATCH_BYTES
    rc = lib.lpaici_backward_noalloc(ks.handle, fake, W, fake, W, fake, W, W, H, SIGMA_20, 2.0, None)
    assert rc == lpaici.ERR_UNSUPPORTED
    msg = lib.lpaici_last_error().decode()
    assert "lpaici_backward_noalloc" in msg and str(SCRATCH_BYTES) in msg
    assert lib.lpaici_backward_noalloc(None, fake, 1, fake, 1, fake, 1, 1, 1, SIGMA_20, 2.0, None) == \
        lpaici.ERR_INVALID_ARG
