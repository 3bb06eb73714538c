"""lpaici_forward_ffma (each tap one fused multiply-add) against the bit-exact forward.

The contracted mode is not bit-exact with the reference, so it is held to the accuracy criteria of the
project's goal instead, image by image, on all 15 reference kernel sets (256x256 synthetic images),
barbara (the reference's own image and settings) and a 1024x1024 benchmark-style image:
  * selected scales agree with the exact forward's on >= 99.99 % of (direction, pixel);
  * PSNR against the clean image within 0.01 dB of the exact forward's;
  * on pixels whose scales all agree, |ffma - exact| <= 1e-4 (a few ULP in practice).
Where a scale flips (an FP32 tie in the interval test, as between the reference's FP32 and an FP64
evaluation) the pixel's output moves by up to about 1e-2, which is above the 1e-4 bound: that count and
size are reported, not asserted.  Against the FP64 oracle both modes are at rounding level (median
error <= 1e-6) except at the few tie pixels (at most 0.1 % above 1e-4).
"""
import glob
import json
import os

import numpy as np
import pytest

import lpaici
import oracle_bind as ob
from conftest import GOLDEN, SYM, kernel_file

pytestmark = pytest.mark.gpu
SIGMA_20 = float(np.float32(20.0) / np.float32(255.0))
TAPS = sorted(glob.glob(os.path.join(GOLDEN, "kernels", "taps", "*.taps")))


def _compare(ks, noisy, clean, sigma, gamma):
    import torch

    x = torch.from_numpy(noisy).cuda()
    ex, emap = lpaici.forward(ks, x, sigma, gamma, scale_map=True)
    fx, fmap = lpaici.forward(ks, x, sigma, gamma, scale_map=True, ffma=True)
    torch.cuda.synchronize()
    ex, emap, fx, fmap = ex.cpu().numpy(), emap.cpu().numpy(), fx.cpu().numpy(), fmap.cpu().numpy()
    agree = emap == fmap
    px_agree = agree.all(axis=0)
    diff = np.abs(fx.astype(np.float64) - ex.astype(np.float64))
    return dict(map_agreement=float(agree.mean()), flipped_pixels=int((~px_agree).sum()),
                max_err_all=float(diff.max()), max_err_agreeing=float(diff[px_agree].max()) if px_agree.any() else 0.0,
                psnr_delta=float(lpaici.psnr(clean, fx) - lpaici.psnr(clean, ex)), out=fx, exact=ex)


def _check(r, what):
    assert r["map_agreement"] >= 0.9999, (what, r["map_agreement"])
    assert abs(r["psnr_delta"]) <= 0.01, (what, r["psnr_delta"])
    assert r["max_err_agreeing"] <= 1e-4, (what, r["max_err_agreeing"])
    assert np.isfinite(r["out"]).all()


@pytest.mark.parametrize("path", TAPS, ids=[os.path.basename(p) for p in TAPS])
def test_ffma_every_kernel_set(path):
    ks = lpaici.KernelSet.load(path)
    clean = lpaici.synth_image(256, 256, 31)
    noisy = lpaici.add_noise(clean, SIGMA_20, 20250910)
    _check(_compare(ks, noisy, clean, SIGMA_20, 2.0), os.path.basename(path))


def test_ffma_barbara():
    meta = json.load(open(os.path.join(GOLDEN, "barbara.json")))
    u8 = np.load(os.path.join(GOLDEN, "barbara_gray_u8.npy"))
    lut = (np.power((np.arange(256, dtype=np.float32) / np.float32(255.0)).astype(np.float64),
                    np.float64(np.float32(2.2))) * 1.0).astype(np.float32)
    clean = lut[u8]
    noisy = lpaici.add_noise(clean, SIGMA_20, 20250910)
    r = _compare(lpaici.KernelSet.load(kernel_file(SYM)), noisy, clean, SIGMA_20, 2.0)
    _check(r, "barbara")
    assert abs(lpaici.psnr(clean, r["out"]) - meta["psnr_denoised"]) <= 0.01


def test_ffma_1024_and_error_against_fp64():
    ks = lpaici.KernelSet.load(kernel_file(SYM))
    clean = lpaici.synth_image(1024, 1024, 20250910)
    noisy = lpaici.add_noise(clean, SIGMA_20, 20250910)
    r = _compare(ks, noisy, clean, SIGMA_20, 2.0)
    _check(r, "1024")
    # error against an FP64 evaluation of the same algorithm, on a 256^2 crop (whole-image semantics)
    ko = ob.oracle_load_kernels(kernel_file(SYM))
    crop_n, crop_c = noisy[:256, :256].copy(), clean[:256, :256].copy()
    ref64, _ = ob.oracle_forward_f64(crop_n, ko, SIGMA_20, 2.0)
    rc = _compare(ks, crop_n, crop_c, SIGMA_20, 2.0)
    err_ffma = np.abs(rc["out"].astype(np.float64) - ref64)
    err_exact = np.abs(rc["exact"].astype(np.float64) - ref64)
    # both FP32 evaluations sit at rounding level from FP64 except where a tie flips a scale
    assert np.median(err_ffma) <= 1e-6 and np.median(err_exact) <= 1e-6
    assert np.mean(err_ffma > 1e-4) <= 1e-3 and np.mean(err_exact > 1e-4) <= 1e-3
