"""Binary tap-list files (lpaici_kernelset_save / lpaici_kernelset_load): a saved kernel set loads back
to the same kernel set -- runs, weights, variances and dense arrays (zeros outside the runs) -- and a
damaged file is refused."""
import os

import numpy as np
import pytest

import lpaici
from conftest import GAUSS_M2, SYM, kernel_file

NAMES = [SYM, GAUSS_M2, "lpa_kernels_m_1_0_d_8_h12_1_2_4_8.txt", "lpa_kernels_python_16_tapered.txt"]


def _same(a: lpaici.KernelSet, b: lpaici.KernelSet):
    assert (a.D, a.S) == (b.D, b.S)
    ra, rb = a.runs(), b.runs()
    for f in ("run_row", "run_col", "run_len", "kernel_first_run", "kernel_num_runs", "kernel_first_weight"):
        assert np.array_equal(getattr(ra, f), getattr(rb, f)), f
    assert np.array_equal(ra.weights.view(np.uint32), rb.weights.view(np.uint32))
    da, db = a.dense(), b.dense()
    for x, y in zip(da, db):
        assert np.array_equal(np.asarray(x), np.asarray(y))  # +0 and -0 compare equal outside the runs
    sig = float(np.float32(20.0) / np.float32(255.0))
    assert np.array_equal(a.variances(sig).view(np.uint32), b.variances(sig).view(np.uint32))


@pytest.mark.parametrize("name", NAMES)
def test_round_trip(tmp_path, name):
    path = kernel_file(name)
    ks = lpaici.KernelSet.load(path)
    out = str(tmp_path / "k.taps")
    ks.save(out)
    assert open(out, "rb").read(8) == b"LPAICIT1"
    assert os.path.getsize(out) < os.path.getsize(path)
    _same(ks, lpaici.KernelSet.load(out))


def test_damaged_files_refused(tmp_path):
    ks = lpaici.KernelSet.load(kernel_file(SYM))
    good = tmp_path / "k.taps"
    ks.save(str(good))
    data = good.read_bytes()
    cases = {"flip": data[:100] + bytes([data[100] ^ 1]) + data[101:], "truncated": data[:-9],
             "short": data[:12], "extended": data + b"\0"}
    for tag, blob in cases.items():
        p = tmp_path / f"{tag}.taps"
        p.write_bytes(blob)
        with pytest.raises(lpaici.LpaIciError) as e:
            lpaici.KernelSet.load(str(p))
        assert e.value.code == lpaici.ERR_KERNEL_FORMAT, tag
