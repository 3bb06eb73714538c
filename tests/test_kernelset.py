"""The product's kernel-set loader, run packer and variances (through the C ABI; no GPU needed), checked
against the oracle, plus the loader's error behaviour on malformed files."""
import glob
import os

import numpy as np
import pytest

import lpaici
import oracle_bind as ob
from conftest import GAUSS_M2, REFERENCE_KERNELS, SMALL, SYM, TAPERED, kernel_file

SIGMA_20 = np.float32(20.0) / np.float32(255.0)


def _all_kernel_files():
    files = [kernel_file(n) for n in (SYM, GAUSS_M2, SMALL, TAPERED)]
    files += sorted(glob.glob(os.path.join(REFERENCE_KERNELS, "*.txt")))
    return files


@pytest.mark.parametrize("path", _all_kernel_files(), ids=lambda p: os.path.basename(p))
def test_loader_and_packer_match_oracle(path):
    ks = lpaici.KernelSet.load(path)
    ko = ob.oracle_load_kernels(path)
    w, o, r, c = ks.dense()
    assert (ks.D, ks.S) == (ko.D, ko.S)
    assert np.array_equal(w.view(np.uint32), ko.w.view(np.uint32))
    assert np.array_equal(o, ko.off) and np.array_equal(r, ko.rows) and np.array_equal(c, ko.cols)
    runs = ks.runs()
    po = ob.oracle_pack_runs(ko)
    assert np.array_equal(runs.weights.view(np.uint32), po["weights"].view(np.uint32))
    for key in ("run_row", "run_col", "run_len", "k_first_run", "k_num_runs", "k_first_weight"):
        name = key.replace("k_", "kernel_")
        assert np.array_equal(getattr(runs, name), po[key]), key
    for sigma in (SIGMA_20, np.float32(25.0) / np.float32(255.0), np.float32(0.5)):
        assert np.array_equal(ks.variances(sigma).view(np.uint32), ob.oracle_variances(ko, sigma).view(np.uint32))
    assert np.array_equal(ks.nnz(), ko.nnz())
    assert ks.radius == max(max(abs(a), abs(b), abs(b + l - 1))
                            for a, b, l in zip(po["run_row"], po["run_col"], po["run_len"]))


def test_symmetric_set_sizes(sym_path):
    """The default set: 16 x 7 kernels of 1, 3, 7, 15, 31, 47, 63 px; 6,008 weights in 1,052 runs
    (38,000 B in the reference's constant memory), radius 31."""
    ks = lpaici.KernelSet.load(sym_path)
    assert (ks.D, ks.S, ks.info.n_taps, ks.info.n_runs, ks.radius) == (16, 7, 6008, 1052, 31)
    assert ks.info.dense_size == 16 * sum(n * n for n in (1, 3, 7, 15, 31, 47, 63))


def test_tapered_set_exceeds_reference_constant_memory(tapered_path):
    """python_16_tapered has 12,320 weights: the reference's v3/v4 stop on it (8,192-weight cap,
    src/v4_1_lpa_ici_2D_sparse_shared.cu:43,1180-1186); here the tables live in global memory."""
    ks = lpaici.KernelSet.load(tapered_path)
    assert ks.info.n_taps > 8192


def test_from_dense_equals_load(small_path):
    a = lpaici.KernelSet.load(small_path)
    b = lpaici.KernelSet.from_dense(*a.dense(), a.D, a.S)
    ra, rb = a.runs(), b.runs()
    assert all(np.array_equal(getattr(ra, f), getattr(rb, f)) for f in ra.__dataclass_fields__)


def _write(tmp_path, text, name="k.txt"):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


MALFORMED = [
    "", "0 3\n", "2 -1\n", "x 1\n", "1 1\n3 3\n1 2 3 4 5\n", "1 1\n0 3\n", "1 2\n1 1\n1\n",
    "2 1\n3 3\n0 0 0 0 1 0 0 0 0\n1 1\n1\n",  # direction 1 smaller than direction 0
    "1 1\n1 1\nnan\n", "1 1\n1 1\n1e999\n", "1 1\n1 1\ninf\n", "1 1\n3.0 1\n1 2 3\n", "1 1\n1 1\n1e\n",
    "1 1\n1 1\n.\n", "1 1\n1 2\n0x10 1\n",
]
ODD_BUT_VALID = [  # operator>> reads a numeric prefix and leaves the rest
    "1 1\n1 1\n1e-50\n", "1 1\n1 1\n+.5\n", "1 1\n1 1\n0x10\n", "1 1\n1 1\n1.5abc\n", "1 1\n1 1\n-0\n",
    "1 1\n1 3\n1. 2.5e+1 -3E-2\n", "1 1\n 3 3\n" + "0 " * 4 + "1e-45 " + "0 " * 4 + "\n",
]


def _result_product(p):
    try:
        ks = lpaici.KernelSet.load(p)
    except lpaici.LpaIciError as e:
        return ("error", e.code)
    w, o, r, c = ks.dense()
    return ("ok", w.view(np.uint32).tolist(), r.tolist(), c.tolist())


def _result_oracle(p):
    try:
        k = ob.oracle_load_kernels(p)
    except ValueError:
        return ("error", lpaici.ERR_KERNEL_FORMAT)
    return ("ok", k.w.view(np.uint32).tolist(), k.rows.tolist(), k.cols.tolist())


@pytest.mark.parametrize("text", MALFORMED + ODD_BUT_VALID)
def test_loader_edge_inputs(tmp_path, text):
    p = _write(tmp_path, text)
    prod, orac = _result_product(p), _result_oracle(p)
    assert prod == orac
    if text in MALFORMED:
        assert prod == ("error", lpaici.ERR_KERNEL_FORMAT)
    if ob.ref_available("v1_0"):
        try:
            k = ob.ref_load_kernels(p)
            ref = ("ok", k.w.view(np.uint32).tolist(), k.rows.tolist(), k.cols.tolist())
        except ValueError:
            ref = ("error", lpaici.ERR_KERNEL_FORMAT)
        assert prod == ref


def test_radius_limit(tmp_path):
    """A 255x255 kernel whose only tap sits at a corner has radius 127, the supported maximum."""
    ks = lpaici.KernelSet.load(_write(tmp_path, "1 1\n255 255\n" + "0 " * (255 * 255 - 1) + "1\n"))
    assert ks.radius == 127
    with pytest.raises(lpaici.LpaIciError) as e:
        lpaici.KernelSet.load(_write(tmp_path, "1 1\n257 257\n" + "0 " * (257 * 257 - 1) + "1\n", "k2.txt"))
    assert e.value.code == lpaici.ERR_UNSUPPORTED


def test_loader_missing_file(tmp_path):
    with pytest.raises(lpaici.LpaIciError) as e:
        lpaici.KernelSet.load(str(tmp_path / "nope.txt"))
    assert e.value.code == lpaici.ERR_FILE


def test_crop_to_direction_zero(tmp_path):
    """Direction 1's 5x5 kernel is centre-cropped to direction 0's 3x3 (offset (5-3)/2 = 1)."""
    d1 = np.arange(25, dtype=np.float32).reshape(5, 5) + 1
    text = "2 1\n3 3\n" + " ".join(["1"] * 9) + "\n5 5\n" + " ".join(f"{v:g}" for v in d1.ravel()) + "\n"
    ks = lpaici.KernelSet.load(_write(tmp_path, text))
    w, o, r, c = ks.dense()
    assert list(r) == [3, 3] and list(c) == [3, 3]
    assert np.array_equal(w[9:18].reshape(3, 3), d1[1:4, 1:4])


def test_too_many_kernels(tmp_path):
    with pytest.raises(lpaici.LpaIciError) as e:
        lpaici.KernelSet.load(_write(tmp_path, "20 20\n"))
    assert e.value.code == lpaici.ERR_UNSUPPORTED
