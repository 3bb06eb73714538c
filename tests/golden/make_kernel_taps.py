"""Generates tests/golden/kernels/taps/*.taps: every kernel file of the reference (kernels/*.txt), read
by the reference's own loader (load_LPA_kernels_standardized, compiled in-process from its sources into
oracle/_ref/) and stored as this library's binary tap-list file (lpaici_kernelset_save), so that the GPU
tests can run every kernel set without the reference tree.

    python tests/golden/make_kernel_taps.py [--reference <reference root>]   (default: $LPAICI_REFERENCE)
"""
import argparse
import glob
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "lpa-ici-cuda_b200"))
import oracle_bind as ob  # noqa: E402
import lpaici  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("LPAICI_REFERENCE"), required="LPAICI_REFERENCE" not in os.environ)
    args = ap.parse_args()
    out_dir = os.path.join(HERE, "kernels", "taps")
    os.makedirs(out_dir, exist_ok=True)
    for path in sorted(glob.glob(os.path.join(args.reference, "kernels", "*.txt"))):
        k = ob.ref_load_kernels(path)
        ks = lpaici.KernelSet.from_dense(k.w, k.off, k.rows, k.cols, k.D, k.S)
        name = os.path.basename(path)[:-4] + ".taps"
        ks.save(os.path.join(out_dir, name))
        print(name, k.D, k.S, os.path.getsize(os.path.join(out_dir, name)))


if __name__ == "__main__":
    main()
