"""Every kernel set of the reference (its 15 kernel files: D = 4, 8, 16; S = 4, 5, 7; square, wedge,
gaussian and tapered windows), committed as binary tap-list files made by the reference's own loader
(tests/golden/make_kernel_taps.py).  CPU: each file reloads to the reference loader's dense output.
GPU: the forward on every set equals the FP32 oracle bit for bit, estimates and selected scales, and the
adjoint matches the FP64 oracle's."""
import glob
import os

import numpy as np
import pytest

import lpaici
import oracle_bind as ob
from conftest import GOLDEN, REFERENCE_KERNELS

TAPS = sorted(glob.glob(os.path.join(GOLDEN, "kernels", "taps", "*.taps")))


def _dense(ks):
    w, off, rows, cols = ks.dense()
    return ob.DenseKernels(ks.D, ks.S, np.ascontiguousarray(w, np.float32), np.ascontiguousarray(off, np.int32),
                           np.ascontiguousarray(rows, np.int32), np.ascontiguousarray(cols, np.int32))


def test_fixture_count():
    assert len(TAPS) == 15


@pytest.mark.parametrize("path", TAPS, ids=[os.path.basename(p) for p in TAPS])
def test_taps_equal_reference_loader(path):
    text = os.path.join(REFERENCE_KERNELS, os.path.basename(path)[:-5] + ".txt")
    if not (os.path.exists(text) and ob.ref_available("v1_0")):
        pytest.skip("reference tree or in-process reference not available")
    ref = ob.ref_load_kernels(text)
    got = _dense(lpaici.KernelSet.load(path))
    assert (got.D, got.S) == (ref.D, ref.S)
    for f in ("off", "rows", "cols"):
        assert np.array_equal(getattr(got, f), getattr(ref, f)), f
    assert np.array_equal(got.w, ref.w)  # signed zeros outside the runs compare equal


@pytest.mark.gpu
@pytest.mark.parametrize("path", TAPS, ids=[os.path.basename(p) for p in TAPS])
def test_forward_bit_exact_on_every_kernel_set(path):
    import torch

    ks = lpaici.KernelSet.load(path)
    ko = _dense(ks)
    sigma = float(np.float32(25.0) / np.float32(255.0))
    noisy = lpaici.add_noise(lpaici.synth_image(83, 61, 9), sigma, 10)
    var = ks.variances(sigma)
    ref, rmap, _ = ob.oracle_forward_f32(noisy, ko, var, 1.5, want_map=True)
    out, smap = lpaici.forward(ks, torch.from_numpy(noisy).cuda(), sigma, 1.5, scale_map=True)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(smap.cpu().numpy(), rmap)


@pytest.mark.gpu
@pytest.mark.parametrize("path", TAPS, ids=[os.path.basename(p) for p in TAPS])
def test_adjoint_on_every_kernel_set(path):
    """The adjoint on every set against the FP64 oracle's frozen-selection adjoint (tolerance as in the
    adjoint tests: 2e-5 * max|ref| + 1e-6)."""
    import torch

    ks = lpaici.KernelSet.load(path)
    ko = _dense(ks)
    sigma = float(np.float32(20.0) / np.float32(255.0))
    noisy = lpaici.add_noise(lpaici.synth_image(77, 58, 12), sigma, 13)
    g = np.random.default_rng(14).standard_normal(noisy.shape).astype(np.float32)
    var = ks.variances(sigma)
    _, smap, _ = ob.oracle_forward_f32(noisy, ko, var, 2.0, want_map=True)
    ref = ob.oracle_adjoint_f64(ko, var, smap, g.astype(np.float64))
    got = lpaici.backward(ks, torch.from_numpy(noisy).cuda(), torch.from_numpy(g).cuda(), sigma, 2.0).cpu().numpy()
    err = np.abs(got - ref).max()
    assert err <= 2e-5 * np.abs(ref).max() + 1e-6, (err, np.abs(ref).max())
