"""Pins the oracle (oracle/lpaici_oracle.c) to the reference.

1. Against the committed golden fixtures, which the reference's own functions produced
   (tests/golden/make_golden.py): runs everywhere.
2. Against the reference compiled in-process from its sources (oracle/_ref/): runs where the
   reference tree and oracle/_ref/ exist (this container), on fresh seeded inputs and every kernel file.
"""
import glob
import json
import os

import numpy as np
import pytest

import oracle_bind as ob
from conftest import GOLDEN, REFERENCE_KERNELS, SMALL, SYM, kernel_file
from lpaici.synth import synth_image

CASES = json.load(open(os.path.join(GOLDEN, "forward_cases.json")))
ARR = np.load(os.path.join(GOLDEN, "forward_cases.npz"))
SIGMA_20 = np.float32(20.0) / np.float32(255.0)


def bits_equal(a, b):
    return a.shape == b.shape and np.array_equal(np.asarray(a, np.float32).view(np.uint32),
                                                 np.asarray(b, np.float32).view(np.uint32))


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_golden_forward(name):
    c = CASES[name]
    k = ob.oracle_load_kernels(kernel_file(c["kernels"]))
    sigma, gamma = ARR[f"{name}/params"]
    var = ob.oracle_variances(k, sigma)
    assert bits_equal(var, ARR[f"{name}/var"])
    out, _, _ = ob.oracle_forward_f32(ARR[f"{name}/noisy"], k, var, float(gamma))
    assert bits_equal(out, ARR[f"{name}/out"])
    psnr = ARR[f"{name}/psnr"]
    assert ob.oracle_psnr(ARR[f"{name}/clean"], ARR[f"{name}/noisy"]) == psnr[0]
    assert ob.oracle_psnr(ARR[f"{name}/clean"], out) == psnr[1]


def test_oracle_barbara_published_psnr():
    """readme.md:7 -- noisy 22.1056 dB, denoised 25.0736 dB on data/barbara.png with the defaults."""
    import hashlib

    meta = json.load(open(os.path.join(GOLDEN, "barbara.json")))
    u8 = np.load(os.path.join(GOLDEN, "barbara_gray_u8.npy"))
    lut = (np.power((np.arange(256, dtype=np.float32) / np.float32(255.0)).astype(np.float64),
                    np.float64(np.float32(2.2))) * 1.0).astype(np.float32)
    clean = lut[u8]
    assert hashlib.sha256(clean.tobytes()).hexdigest() == meta["clean_sha256"]
    import lpaici

    noisy = lpaici.add_noise(clean, SIGMA_20, 20250910)
    assert hashlib.sha256(noisy.tobytes()).hexdigest() == meta["noisy_sha256"]
    k = ob.oracle_load_kernels(kernel_file(SYM))
    var = ob.oracle_variances(k, SIGMA_20)
    out, _, _ = ob.oracle_forward_f32(noisy, k, var, 2.0)
    assert hashlib.sha256(out.tobytes()).hexdigest() == meta["denoised_sha256"]
    assert round(ob.oracle_psnr(clean, noisy), 4) == meta["published_psnr_noisy"]
    assert round(ob.oracle_psnr(clean, out), 4) == meta["published_psnr_denoised"]


def test_oracle_scale_map_consistent():
    """The scale map the oracle emits reproduces its own output (est of s*, var of s*)."""
    name = "sym_64x48"
    k = ob.oracle_load_kernels(kernel_file(SYM))
    var = ARR[f"{name}/var"]
    out, smap, taps = ob.oracle_forward_f32(ARR[f"{name}/noisy"], k, var, 2.0, want_map=True)
    assert smap.shape == (16, 48, 64) and smap.max() < 7
    assert taps == ob.oracle_count_taps(smap, k)
    assert 0 < taps <= 6008 * 64 * 48


# ---- against the reference itself (in-process) --------------------------------------------------
needs_ref = pytest.mark.skipif(not (ob.ref_available("v1_0") and os.path.isdir(REFERENCE_KERNELS)),
                               reason="reference tree / oracle/_ref not available")


@needs_ref
@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(REFERENCE_KERNELS, "*.txt"))),
                         ids=lambda p: os.path.basename(p))
def test_oracle_loader_variances_packer_vs_reference(path):
    ko = ob.oracle_load_kernels(path)
    kr = ob.ref_load_kernels(path)
    for a in ("w", "off", "rows", "cols"):
        assert np.array_equal(getattr(ko, a), getattr(kr, a)), a
    assert (ko.D, ko.S) == (kr.D, kr.S)
    assert bits_equal(ob.oracle_variances(ko, SIGMA_20), ob.ref_variances(kr, SIGMA_20))
    if ob.ref_available("v4_1"):
        po, pr = ob.oracle_pack_runs(ko), ob.ref_pack_runs(kr)
        for key in po:
            assert np.array_equal(po[key], pr[key]), key


@needs_ref
@pytest.mark.parametrize("kname,W,H,sigma,gamma,seed", [
    (SYM, 48, 40, 20.0, 2.0, 101), (SYM, 31, 70, 35.0, 1.5, 102), (SMALL, 57, 33, 15.0, 2.5, 103),
    ("lpa_kernels_m_0_0_d_4_square.txt", 40, 40, 20.0, 2.0, 104),
    ("lpa_kernels_m_1_0_d_8_h12_1_15_15_30.txt", 45, 38, 20.0, 2.0, 105),
])
def test_oracle_forward_vs_reference(kname, W, H, sigma, gamma, seed):
    path = os.path.join(REFERENCE_KERNELS, kname)
    k = ob.ref_load_kernels(path)
    s = np.float32(sigma) / np.float32(255.0)
    var = ob.ref_variances(k, s)
    clean = synth_image(W, H, seed)
    noisy = ob.ref_noise(clean, s, 20250910 + seed)
    ref = ob.ref_forward(noisy, k, var, gamma)
    out, _, _ = ob.oracle_forward_f32(noisy, k, var, gamma)
    assert bits_equal(out, ref)
    assert ob.oracle_psnr(clean, out) == ob.ref_psnr(clean, ref)


@needs_ref
def test_reference_naive_equals_fused():
    """v0_0 (full sweep) and v1_0 (early exit) agree bit for bit, so one oracle serves both."""
    if not ob.ref_available("v0_0"):
        pytest.skip("v0_0 not built")
    k = ob.ref_load_kernels(os.path.join(REFERENCE_KERNELS, SMALL))
    var = ob.ref_variances(k, SIGMA_20)
    noisy = ob.ref_noise(synth_image(40, 36, 7), SIGMA_20, 20250910)
    assert bits_equal(ob.ref_forward(noisy, k, var, 2.0, name="v0_0"), ob.ref_forward(noisy, k, var, 2.0))


@needs_ref
def test_rgbe_quantizer_matches_stb(tmp_path):
    from lpaici.synth import rgbe_quantize

    raw = synth_image(97, 61, 3, rgbe=False)
    p = str(tmp_path / "x.hdr")
    ob.ref_stbi_write_hdr(p, raw)
    assert bits_equal(ob.ref_stbi_loadf(p), rgbe_quantize(raw))
    q = synth_image(97, 61, 3)
    ob.ref_stbi_write_hdr(p, q)
    assert bits_equal(ob.ref_stbi_loadf(p), q)  # idempotent: the benchmark image survives .hdr


@needs_ref
def test_noise_and_psnr_vs_reference():
    import lpaici

    clean = synth_image(70, 50, 12)
    for sigma, seed in ((SIGMA_20, 20250910), (np.float32(0.3), 1), (np.float32(1e-3), 4294967295)):
        a = lpaici.add_noise(clean, sigma, seed)
        b = ob.ref_noise(clean, sigma, seed)
        assert bits_equal(a, b)
        assert lpaici.psnr(clean, a) == ob.ref_psnr(clean, b)
