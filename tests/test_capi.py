"""The C ABI library loads without a GPU and exports every function include/lpaici.h declares; host-only
entry points return the documented status codes."""
import ctypes as C
import os
import re

import numpy as np

import lpaici
from conftest import PKG, ROOT

HEADER = os.path.join(ROOT, "include", "lpaici.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lpaici_\w+)\s*\(", text)))


def test_header_functions_exported():
    lib = C.CDLL(os.path.join(PKG, "lib", "liblpaici.so"))
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert set(declared_functions()) <= set(lpaici.EXPORTED)


def test_status_strings():
    lib = lpaici.lib()
    for code, name in ((0, "LPAICI_OK"), (1, "LPAICI_ERR_INVALID_ARG"), (2, "LPAICI_ERR_FILE"),
                       (3, "LPAICI_ERR_KERNEL_FORMAT"), (4, "LPAICI_ERR_UNSUPPORTED"), (5, "LPAICI_ERR_CUDA"),
                       (6, "LPAICI_ERR_NO_MEMORY")):
        assert lib.lpaici_status_string(code).decode() == name


def test_null_arguments_rejected():
    lib = lpaici.lib()
    assert lib.lpaici_kernelset_load(None, None) == lpaici.ERR_INVALID_ARG
    assert lib.lpaici_kernelset_get_info(None, None) == lpaici.ERR_INVALID_ARG
    assert lib.lpaici_forward(None, None, 1, None, 1, 1, 1, 0.1, 2.0, None, None) == lpaici.ERR_INVALID_ARG
    assert lib.lpaici_backward(None, None, 1, None, 1, None, 1, 1, 1, 0.1, 2.0, None) == lpaici.ERR_INVALID_ARG
    assert lib.lpaici_batch_create(None, None, 0, None, None, None) == lpaici.ERR_INVALID_ARG
    assert lib.lpaici_set_tile_config(None, 0) == lpaici.ERR_INVALID_ARG
    assert lib.lpaici_tile_config_desc(99, None, None, None, None) == lpaici.ERR_INVALID_ARG
    assert "tile config 99" in lib.lpaici_last_error().decode()
    assert lib.lpaici_kernelset_destroy(None) == lpaici.OK
    assert lib.lpaici_batch_destroy(None) == lpaici.OK


def test_reference_engine_argument_checks():
    """A channel count outside 1..64 and kernels outside the weight array are refused before any device
    work."""
    w = np.ones(9, np.float32)
    off, rows, cols = (np.array([v], np.int32) for v in (0, 3, 3))
    x = np.zeros((4, 4), np.float32)
    var = np.ones(1, np.float32)
    lib = lpaici.lib()
    fp = C.POINTER(C.c_float)
    ip = C.POINTER(C.c_int)
    args = lambda ch, size: (x.ctypes.data_as(fp), x.copy().ctypes.data_as(fp), 4, 4, ch, None, 1, 1,
                             w.ctypes.data_as(fp), size, off.ctypes.data_as(ip), rows.ctypes.data_as(ip),
                             cols.ctypes.data_as(ip), var.ctypes.data_as(fp), 2.0, None)
    assert lib.lpaici_anisotropic_gpu_fused(*args(0, 9)) == lpaici.ERR_INVALID_ARG
    assert lib.lpaici_anisotropic_gpu_fused(*args(65, 9)) == lpaici.ERR_INVALID_ARG
    assert lib.lpaici_anisotropic_gpu_fused(*args(1, 8)) == lpaici.ERR_KERNEL_FORMAT


def test_tile_configs_describe_all():
    cfgs = lpaici.tile_configs()
    assert len(cfgs) == lpaici.lib().lpaici_num_tile_configs() >= 3
    for tw, th, threads, ppt in cfgs:
        assert tw * th == threads * ppt  # every thread owns ppt pixels of the tile


def test_backward_batch_arguments_checked_on_host():
    """A null pointer or a bad size in any image is refused before any device work."""
    lib = lpaici.lib()
    arr = (lpaici.GradImage * 2)()
    arr[0] = lpaici.GradImage(16, 16, 16, 4, 4, 4, 4, 4, 0.1, 2.0)
    arr[1] = lpaici.GradImage(16, None, 16, 4, 4, 4, 4, 4, 0.1, 2.0)
    ks = lpaici.KernelSet.load(__import__("conftest").kernel_file(__import__("conftest").SYM))
    h = C.c_void_p()
    assert lib.lpaici_backward_batch_create(ks.handle, arr, 2, None, None, C.byref(h)) == lpaici.ERR_INVALID_ARG
    assert "image 1" in lib.lpaici_last_error().decode()
    arr[1] = lpaici.GradImage(16, 16, 16, 4, 4, 3, 4, 4, 0.1, 2.0)  # noisy pitch < width
    assert lib.lpaici_backward_batch_create(ks.handle, arr, 2, None, None, C.byref(h)) == lpaici.ERR_INVALID_ARG
    arr[1] = lpaici.GradImage(16, 16, 16, 4, 4, 4, 4, 4, 0.0, 2.0)  # sigma 0
    assert lib.lpaici_backward_batch_create(ks.handle, arr, 2, None, None, C.byref(h)) == lpaici.ERR_INVALID_ARG
    assert lib.lpaici_backward_batch_destroy(None) == lpaici.OK
