"""Generates the committed fixtures of tests/golden/ from the reference itself.

Run where the reference tree exists (--reference, default $LPAICI_REFERENCE) and oracle/_ref/ is built
(`make -C oracle`).  Everything here comes out of the reference's own code, called in-process:
  kernels/*.txt.gz         copies of four of the reference's kernel files (inputs of the path)
  barbara_gray_u8.npy      data/barbara.png as stbi_load(.., 1) returns it (8-bit gray, before the
                           gamma-2.2 float conversion)
  barbara.json             the reference's PSNRs on it (noisy and denoised, defaults of Config.hpp)
                           and a hash of its denoised float image
  forward_cases.npz        small seeded cases: clean, noisy (create_noisy_image), variances
                           (compute_kernel_variances) and the denoised image of
                           anisotropic_lpa_ici_cpu_fused (src/v1_0_lpa_ici_2D_fused.cpp:851-930)

    python tests/golden/make_golden.py [--reference <reference root>]   (default: $LPAICI_REFERENCE)
"""
import argparse
import gzip
import hashlib
import json
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "lpa-ici-cuda_b200"))
import oracle_bind as ob  # noqa: E402
from lpaici.synth import synth_image  # noqa: E402  (pure numpy: needs no GPU)

KERNELS = {
    "sym": "lpa_kernels_m_1_0_d_16_h12_1_2_4_8_16_24_32_symmetric.txt",
    "gauss_m2": "lpa_kernels_m_2_0_d_16_h12_1_2_4_8_16_24_32_gaussian.txt",
    "small": "lpa_kernels_m_1_0_d_8_h12_1_2_4_8.txt",
    "tapered": "lpa_kernels_python_16_tapered.txt",
}
SIGMA_20 = np.float32(20.0) / np.float32(255.0)
SIGMA_25 = np.float32(25.0) / np.float32(255.0)
SEED = 20250910

# name: (kernel key, width, height, sigma, gamma, image seed)
CASES = {
    "sym_64x48": ("sym", 64, 48, SIGMA_20, 2.0, 1),
    "sym_1x1": ("sym", 1, 1, SIGMA_20, 2.0, 2),
    "sym_17x1": ("sym", 17, 1, SIGMA_20, 2.0, 3),
    "sym_1x23": ("sym", 1, 23, SIGMA_20, 2.0, 4),
    "sym_63x63": ("sym", 63, 63, SIGMA_20, 2.0, 5),
    "sym_64x65": ("sym", 64, 65, SIGMA_20, 2.0, 6),
    "sym_130x37": ("sym", 130, 37, SIGMA_20, 2.0, 7),
    "small_96x80": ("small", 96, 80, SIGMA_20, 2.0, 8),
    "gauss_m2_80x72": ("gauss_m2", 80, 72, SIGMA_25, 1.5, 9),
    "tapered_72x40": ("tapered", 72, 40, SIGMA_20, 2.0, 10),
    "sym_gamma1_40x40": ("sym", 40, 40, np.float32(10.0) / np.float32(255.0), 1.0, 11),
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("LPAICI_REFERENCE"), required="LPAICI_REFERENCE" not in os.environ)
    args = ap.parse_args()
    kdir = os.path.join(HERE, "kernels")
    os.makedirs(kdir, exist_ok=True)
    paths = {}
    for key, name in KERNELS.items():
        src = os.path.join(args.reference, "kernels", name)
        with open(src, "rb") as f, gzip.GzipFile(os.path.join(kdir, name + ".gz"), "wb", mtime=0) as g:
            shutil.copyfileobj(f, g)
        paths[key] = src

    # barbara: the published golden values (readme.md:7) reproduced by the reference in-process
    png = os.path.join(args.reference, "data", "barbara.png")
    gray_u8 = ob.ref_stbi_load_u8(png)
    np.save(os.path.join(HERE, "barbara_gray_u8.npy"), gray_u8)
    clean = ob.ref_stbi_loadf(png)
    k = ob.ref_load_kernels(paths["sym"])
    var = ob.ref_variances(k, SIGMA_20)
    noisy = ob.ref_noise(clean, SIGMA_20, SEED)
    out = ob.ref_forward(noisy, k, var, 2.0)
    meta = {
        "source": "data/barbara.png, Config.hpp defaults (sigma 20/255, gamma 2, seed 20250910, symmetric 16x7)",
        "published_psnr_noisy": 22.1056,
        "published_psnr_denoised": 25.0736,
        "psnr_noisy": ob.ref_psnr(clean, noisy),
        "psnr_denoised": ob.ref_psnr(clean, out),
        "clean_sha256": hashlib.sha256(clean.tobytes()).hexdigest(),
        "noisy_sha256": hashlib.sha256(noisy.tobytes()).hexdigest(),
        "denoised_sha256": hashlib.sha256(out.tobytes()).hexdigest(),
    }
    with open(os.path.join(HERE, "barbara.json"), "w") as f:
        json.dump(meta, f, indent=1)

    arrays = {}
    for name, (kk, W, H, sigma, gamma, seed) in CASES.items():
        k = ob.ref_load_kernels(paths[kk])
        clean = synth_image(W, H, seed)
        noisy = ob.ref_noise(clean, sigma, SEED)
        var = ob.ref_variances(k, sigma)
        out = ob.ref_forward(noisy, k, var, gamma)
        arrays[f"{name}/clean"] = clean
        arrays[f"{name}/noisy"] = noisy
        arrays[f"{name}/var"] = var
        arrays[f"{name}/out"] = out
        arrays[f"{name}/params"] = np.array([sigma, gamma], np.float32)
        arrays[f"{name}/psnr"] = np.array([ob.ref_psnr(clean, noisy), ob.ref_psnr(clean, out)], np.float64)
    np.savez_compressed(os.path.join(HERE, "forward_cases.npz"), **arrays)
    with open(os.path.join(HERE, "forward_cases.json"), "w") as f:
        json.dump({n: {"kernels": KERNELS[c[0]], "width": c[1], "height": c[2], "sigma": float(c[3]),
                       "gamma": c[4], "image_seed": c[5], "noise_seed": SEED} for n, c in CASES.items()}, f, indent=1)
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main()
