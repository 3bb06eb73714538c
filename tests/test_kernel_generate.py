"""Kernel generation (lpaici_kernelset_generate) against the reference's shipped kernel files.

The reference's kernels come from a MATLAB script that is not in its tree; the uniform-window families
are regenerated here from their definition (a wedge or quadrant support, a least-squares polynomial
along the direction).  Written as text with 6 decimals (as the shipped files are) and read back, the
generated sets equal the shipped ones after the loader's crop, bit for bit up to the sign of weights that
are zero in exact arithmetic (which changes no result): the default 16x7 symmetric
set, and the two 4-direction square sets (polynomial orders 0 and 1).  Full precision, every weight is
within 5e-7 of the file's (the files' 6-decimal rounding).  The fixtures are the committed text file
of the default set and the tap-list files the reference's own loader produced (tests/golden)."""
import os

import numpy as np
import pytest

import lpaici
from conftest import GOLDEN, SYM, kernel_file

TAPS = os.path.join(GOLDEN, "kernels", "taps")
CASES = [
    (kernel_file(SYM), 16, [1, 2, 4, 8, 16, 24, 32], 0, "sector"),
    (os.path.join(TAPS, "lpa_kernels_m_0_0_d_4_square.taps"), 4, [1, 2, 4, 8, 16], 0, "quadrant"),
    (os.path.join(TAPS, "lpa_kernels_m_1_0_d_4_square.taps"), 4, [1, 2, 4, 8, 16], 1, "quadrant"),
]


def _dense(ks):
    w, o, r, c = ks.dense()
    return [w[o[k]:o[k] + r[k] * c[k]].reshape(r[k], c[k]) for k in range(ks.D * ks.S)]


@pytest.mark.parametrize("path,D,scales,order,shape", CASES, ids=[os.path.basename(c[0]) for c in CASES])
def test_generated_sets_equal_the_shipped_files(tmp_path, path, D, scales, order, shape):
    want = lpaici.KernelSet.load(path)
    gen = lpaici.KernelSet.generate(D, scales, order, shape)
    # full precision: within the files' 6-decimal rounding
    for a, b in zip(_dense(gen), _dense(want)):
        assert a.shape == b.shape
        assert np.abs(a.astype(np.float64) - b).max() <= 5e-7
    # written as text and read back: the same kernels, the same run-length packing
    txt = str(tmp_path / "k.txt")
    gen.save_text(txt)
    back = lpaici.KernelSet.load(txt)
    for a, b in zip(_dense(back), _dense(want)):
        assert np.array_equal(a, b)
    ra, rb = back.runs(), want.runs()
    for f in ("run_row", "run_col", "run_len", "kernel_first_run", "kernel_num_runs"):
        assert np.array_equal(getattr(ra, f), getattr(rb, f)), f
    # every nonzero weight bit for bit; a weight that is zero in exact arithmetic may carry either sign
    # (the files' own zeros do), which changes no sum: a running sum started at +0 never becomes -0
    assert np.array_equal(ra.weights, rb.weights)
    nz = rb.weights != 0
    assert np.array_equal(ra.weights[nz].view(np.uint32), rb.weights[nz].view(np.uint32))


def test_text_format_matches_the_reference_layout(tmp_path):
    gen = lpaici.KernelSet.generate(16, [1, 2], 0, "sector")
    txt = str(tmp_path / "k.txt")
    gen.save_text(txt)
    lines = open(txt).read().split("\n")
    assert lines[0] == "16 2" and lines[1] == "1 1" and lines[2] == "1.000000 "
    assert lines[3] == "3 3" and lines[4] == "0.000000 0.000000 0.000000 0.000000 0.500000 0.500000 " \
                                          "0.000000 0.000000 0.000000 "


def test_generate_rejects_bad_arguments():
    with pytest.raises(lpaici.LpaIciError):
        lpaici.KernelSet.generate(16, [1, 0], 0, "sector")
    with pytest.raises(lpaici.LpaIciError):
        lpaici.KernelSet.generate(16, [1, 2], 7, "sector")
