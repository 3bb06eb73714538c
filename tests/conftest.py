import gzip
import os
import shutil
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "lpa-ici-cuda_b200")
TESTS = os.path.join(ROOT, "tests")
for p in (PKG, TESTS):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(TESTS, "golden")


def _reference_root():
    """Root of the reference project: LPAICI_REFERENCE, else the tree oracle/_ref/ was built from
    (recorded by oracle/Makefile); None when neither names an existing directory."""
    root = os.environ.get("LPAICI_REFERENCE")
    if not root:
        rec = os.path.join(ROOT, "oracle", "_ref", "reference_root")
        if os.path.exists(rec):
            with open(rec) as f:
                root = f.read().strip()
    return root if root and os.path.isdir(root) else None


REFERENCE_ROOT = _reference_root()
# the reference's kernel files (kernels/*.txt); a path that does not exist when the tree is absent
REFERENCE_KERNELS = os.path.join(REFERENCE_ROOT, "kernels") if REFERENCE_ROOT else os.path.join(ROOT, "_no_reference")
SYM = "lpa_kernels_m_1_0_d_16_h12_1_2_4_8_16_24_32_symmetric.txt"
GAUSS_M2 = "lpa_kernels_m_2_0_d_16_h12_1_2_4_8_16_24_32_gaussian.txt"
SMALL = "lpa_kernels_m_1_0_d_8_h12_1_2_4_8.txt"
TAPERED = "lpa_kernels_python_16_tapered.txt"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def pytest_collection_modifyitems(config, items):
    import torch

    if torch.cuda.is_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


_kernel_cache = os.path.join(GOLDEN, "kernels", "_unpacked")


def kernel_file(name: str) -> str:
    """Path of a kernel file: the committed gzip fixture (unpacked once), else the reference tree."""
    gz = os.path.join(GOLDEN, "kernels", name + ".gz")
    if os.path.exists(gz):
        out = os.path.join(_kernel_cache, name)
        if not os.path.exists(out):
            os.makedirs(_kernel_cache, exist_ok=True)
            tmp = out + f".{os.getpid()}.tmp"
            with gzip.open(gz, "rb") as f, open(tmp, "wb") as g:
                shutil.copyfileobj(f, g)
            os.replace(tmp, out)
        return out
    ref = os.path.join(REFERENCE_KERNELS, name)
    if os.path.exists(ref):
        return ref
    pytest.skip(f"kernel file {name} not available")


@pytest.fixture(scope="session")
def sym_path():
    return kernel_file(SYM)


@pytest.fixture(scope="session")
def small_path():
    return kernel_file(SMALL)


@pytest.fixture(scope="session")
def gauss_path():
    return kernel_file(GAUSS_M2)


@pytest.fixture(scope="session")
def tapered_path():
    return kernel_file(TAPERED)
