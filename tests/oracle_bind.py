"""ctypes bindings for the oracle (oracle/liboracle.so) and the in-process reference (oracle/_ref/).

Test infrastructure: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import this
module, and only to check or time against the reference.  The product never does.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
REF_DIR = os.path.join(ORACLE_DIR, "_ref")
KERNELS_DIR = os.path.join(ROOT, "tests", "golden", "kernels")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


@dataclass
class DenseKernels:
    """The loader's output: dense cropped weights + per-kernel offset/rows/cols (D*S each)."""

    D: int
    S: int
    w: np.ndarray
    off: np.ndarray
    rows: np.ndarray
    cols: np.ndarray

    @property
    def nk(self) -> int:
        return self.D * self.S

    def kernel(self, d: int, s: int) -> np.ndarray:
        k = d * self.S + s
        r, c = int(self.rows[k]), int(self.cols[k])
        return self.w[self.off[k] : self.off[k] + r * c].reshape(r, c)

    def nnz(self) -> np.ndarray:
        return np.array([np.count_nonzero(self.kernel(k // self.S, k % self.S)) for k in range(self.nk)], np.int32)


_oracle = None


def oracle_lib() -> C.CDLL:
    global _oracle
    if _oracle is None:
        path = os.path.join(ORACLE_DIR, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: run `make -C oracle` (or __graft_entry__.build())")
        lib = C.CDLL(path)
        lib.oracle_load_kernels.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                            C.POINTER(C.POINTER(C.c_float)), C.POINTER(C.POINTER(C.c_int)),
                                            C.POINTER(C.POINTER(C.c_int)), C.POINTER(C.POINTER(C.c_int))]
        lib.oracle_load_kernels.restype = C.c_int
        lib.oracle_free.argtypes = [C.c_void_p]
        lib.oracle_variances.argtypes = [_f32p, _i32p, _i32p, _i32p, C.c_int, C.c_float, _f32p]
        lib.oracle_pack_runs.argtypes = [_f32p, _i32p, _i32p, _i32p, C.c_int, _f32p, _i32p, _i32p, _i32p, _i32p,
                                         _i32p, _i32p, C.POINTER(C.c_int)]
        lib.oracle_pack_runs.restype = C.c_int
        lib.oracle_forward_f32.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, _f32p, _i32p, _i32p, _i32p,
                                           _f32p, C.c_float, _f32p, C.c_void_p, C.POINTER(C.c_double)]
        lib.oracle_forward_f64.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, _f32p, _i32p, _i32p, _i32p,
                                           C.c_double, C.c_double, _f64p, C.c_void_p]
        lib.oracle_psnr.argtypes = [_f32p, _f32p, C.c_long]
        lib.oracle_psnr.restype = C.c_double
        lib.oracle_count_taps.argtypes = [_u8p, C.c_long, C.c_int, C.c_int, _i32p]
        lib.oracle_count_taps.restype = C.c_double
        lib.oracle_adjoint_f64.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _f32p, _i32p, _i32p, _i32p, _f32p,
                                           _u8p, _f64p, _f64p]
        lib.oracle_fd_grad_f64.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, _f32p, _i32p, _i32p, _i32p,
                                           _f32p, _u8p, _f64p, _i64p, C.c_int, C.c_double, _f64p]
        _oracle = lib
    return _oracle


def _take(ptr, n, dtype, free):
    arr = np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)
    free(ptr)
    return arr


def oracle_load_kernels(path: str) -> DenseKernels:
    lib = oracle_lib()
    D, S = C.c_int(), C.c_int()
    w, off, rows, cols = C.POINTER(C.c_float)(), C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_int)()
    rc = lib.oracle_load_kernels(path.encode(), C.byref(D), C.byref(S), C.byref(w), C.byref(off), C.byref(rows),
                                 C.byref(cols))
    if rc != 0:
        raise ValueError(f"oracle_load_kernels({path}) failed with {rc}")
    nk = D.value * S.value
    off_a = _take(off, nk, np.int32, lib.oracle_free)
    rows_a = _take(rows, nk, np.int32, lib.oracle_free)
    cols_a = _take(cols, nk, np.int32, lib.oracle_free)
    nw = int(off_a[-1] + rows_a[-1] * cols_a[-1])
    w_a = _take(w, nw, np.float32, lib.oracle_free)
    return DenseKernels(D.value, S.value, w_a, off_a, rows_a, cols_a)


def oracle_variances(k: DenseKernels, sigma: float) -> np.ndarray:
    var = np.zeros(k.nk, np.float32)
    oracle_lib().oracle_variances(k.w, k.off, k.rows, k.cols, k.nk, sigma, var)
    return var


def oracle_pack_runs(k: DenseKernels):
    nr_max = int(k.rows.sum())
    weights = np.zeros(k.w.size, np.float32)
    rr, rc, rl = (np.zeros(nr_max, np.int32) for _ in range(3))
    kfr, knr, kfw = (np.zeros(k.nk, np.int32) for _ in range(3))
    nw = C.c_int()
    nr = oracle_lib().oracle_pack_runs(k.w, k.off, k.rows, k.cols, k.nk, weights, rr, rc, rl, kfr, knr, kfw,
                                       C.byref(nw))
    return dict(weights=weights[: nw.value], run_row=rr[:nr], run_col=rc[:nr], run_len=rl[:nr],
                k_first_run=kfr, k_num_runs=knr, k_first_weight=kfw)


def oracle_forward_f32(x: np.ndarray, k: DenseKernels, var: np.ndarray, gamma: float, want_map: bool = False):
    """Returns (out, scale_map or None, algorithmic taps)."""
    H, W = x.shape
    x = np.ascontiguousarray(x, np.float32)
    out = np.zeros((H, W), np.float32)
    smap = np.zeros((k.D, H, W), np.uint8) if want_map else None
    taps = C.c_double()
    oracle_lib().oracle_forward_f32(x, W, H, k.D, k.S, k.w, k.off, k.rows, k.cols,
                                    np.ascontiguousarray(var, np.float32), gamma, out,
                                    smap.ctypes.data if smap is not None else None, C.byref(taps))
    return out, smap, taps.value


def oracle_forward_f64(x: np.ndarray, k: DenseKernels, sigma: float, gamma: float, want_map: bool = False):
    H, W = x.shape
    out = np.zeros((H, W), np.float64)
    smap = np.zeros((k.D, H, W), np.uint8) if want_map else None
    oracle_lib().oracle_forward_f64(np.ascontiguousarray(x, np.float32), W, H, k.D, k.S, k.w, k.off, k.rows,
                                    k.cols, sigma, gamma, out, smap.ctypes.data if smap is not None else None)
    return out, smap


def oracle_psnr(a: np.ndarray, b: np.ndarray) -> float:
    a = np.ascontiguousarray(a, np.float32).ravel()
    b = np.ascontiguousarray(b, np.float32).ravel()
    return oracle_lib().oracle_psnr(a, b, a.size)


def oracle_count_taps(smap: np.ndarray, k: DenseKernels) -> float:
    D = smap.shape[0]
    return oracle_lib().oracle_count_taps(np.ascontiguousarray(smap), smap[0].size, D, k.S, k.nnz())


def oracle_adjoint_f64(k: DenseKernels, var: np.ndarray, smap: np.ndarray, g: np.ndarray) -> np.ndarray:
    H, W = g.shape
    grad = np.zeros((H, W), np.float64)
    oracle_lib().oracle_adjoint_f64(W, H, k.D, k.S, k.w, k.off, k.rows, k.cols, np.ascontiguousarray(var, np.float32),
                                    np.ascontiguousarray(smap), np.ascontiguousarray(g, np.float64), grad)
    return grad


def oracle_fd_grad_f64(x, k: DenseKernels, var, smap, g, q: np.ndarray, eps: float = 1e-3) -> np.ndarray:
    H, W = x.shape
    fd = np.zeros(q.size, np.float64)
    oracle_lib().oracle_fd_grad_f64(np.ascontiguousarray(x, np.float32), W, H, k.D, k.S, k.w, k.off, k.rows,
                                    k.cols, np.ascontiguousarray(var, np.float32), np.ascontiguousarray(smap),
                                    np.ascontiguousarray(g, np.float64), np.ascontiguousarray(q, np.int64),
                                    q.size, eps, fd)
    return fd


# ---------------------------------------------------------------------------------------------
# The reference itself, compiled in-process from its sources (oracle/_ref/).
# ---------------------------------------------------------------------------------------------
_refs: dict[str, C.CDLL] = {}


def ref_available(name: str = "v1_0") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libref_{name}.so"))


def ref_lib(name: str = "v1_0") -> C.CDLL:
    if name not in _refs:
        lib = C.CDLL(os.path.join(REF_DIR, f"libref_{name}.so"))
        if name in ("v1_0", "v0_0"):
            lib.ref_load_kernels.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                             C.POINTER(C.POINTER(C.c_float)), C.POINTER(C.c_int),
                                             C.POINTER(C.POINTER(C.c_int)), C.POINTER(C.POINTER(C.c_int)),
                                             C.POINTER(C.POINTER(C.c_int))]
            lib.ref_free.argtypes = [C.c_void_p]
            lib.ref_variances.argtypes = [_f32p, C.c_int, _i32p, _i32p, _i32p, C.c_int, C.c_float, _f32p]
            lib.ref_noise.argtypes = [_f32p, _f32p, C.c_int, C.c_float, C.c_uint]
            lib.ref_psnr.argtypes = [_f32p, _f32p, C.c_int]
            lib.ref_psnr.restype = C.c_double
            lib.ref_forward.argtypes = [_f32p, _f32p, C.c_int, C.c_int, _f32p, C.c_int, _i32p, _i32p, _i32p,
                                        C.c_int, C.c_int, _f32p, C.c_float]
            lib.ref_stbi_loadf.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
            lib.ref_stbi_loadf.restype = C.POINTER(C.c_float)
            lib.ref_stbi_free.argtypes = [C.c_void_p]
            lib.ref_stbi_load_u8.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
            lib.ref_stbi_load_u8.restype = C.POINTER(C.c_ubyte)
            lib.ref_stbi_write_hdr.argtypes = [C.c_char_p, C.c_int, C.c_int, _f32p]
            lib.ref_stbi_write_hdr.restype = C.c_int
            lib.ref_stbi_loadf_rgb.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
            lib.ref_stbi_loadf_rgb.restype = C.POINTER(C.c_float)
            lib.ref_stbi_write_hdr_rgb.argtypes = [C.c_char_p, C.c_int, C.c_int, _f32p]
            lib.ref_stbi_write_hdr_rgb.restype = C.c_int
        else:
            lib.ref_pack_runs.argtypes = [_f32p, _i32p, _i32p, _i32p, C.c_int, _f32p, _i32p, _i32p, _i32p, _i32p,
                                          _i32p, _i32p, C.POINTER(C.c_int)]
            lib.ref_pack_runs.restype = C.c_int
            lib.ref_gpu_fused.argtypes = [_f32p, _f32p, C.c_int, C.c_int, _f32p, C.c_int, _i32p, _i32p, _i32p,
                                          C.c_int, C.c_int, _f32p, C.c_float]
        _refs[name] = lib
    return _refs[name]


def ref_load_kernels(path: str, name: str = "v1_0") -> DenseKernels:
    lib = ref_lib(name)
    D, S, nw = C.c_int(), C.c_int(), C.c_int()
    w, off, rows, cols = C.POINTER(C.c_float)(), C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_int)()
    if not lib.ref_load_kernels(path.encode(), C.byref(D), C.byref(S), C.byref(w), C.byref(nw), C.byref(off),
                                C.byref(rows), C.byref(cols)):
        raise ValueError(f"reference loader rejected {path}")
    nk = D.value * S.value
    return DenseKernels(D.value, S.value, _take(w, nw.value, np.float32, lib.ref_free),
                        _take(off, nk, np.int32, lib.ref_free), _take(rows, nk, np.int32, lib.ref_free),
                        _take(cols, nk, np.int32, lib.ref_free))


def ref_variances(k: DenseKernels, sigma: float, name: str = "v1_0") -> np.ndarray:
    var = np.zeros(k.nk, np.float32)
    ref_lib(name).ref_variances(k.w, k.w.size, k.off, k.rows, k.cols, k.nk, sigma, var)
    return var


def ref_noise(clean: np.ndarray, sigma: float, seed: int, name: str = "v1_0") -> np.ndarray:
    c = np.ascontiguousarray(clean, np.float32)
    out = np.zeros_like(c)
    ref_lib(name).ref_noise(c.ravel(), out.ravel(), c.size, sigma, seed)
    return out


def ref_psnr(a: np.ndarray, b: np.ndarray, name: str = "v1_0") -> float:
    a = np.ascontiguousarray(a, np.float32).ravel()
    b = np.ascontiguousarray(b, np.float32).ravel()
    return ref_lib(name).ref_psnr(a, b, a.size)


def ref_forward(x: np.ndarray, k: DenseKernels, var: np.ndarray, gamma: float, name: str = "v1_0") -> np.ndarray:
    H, W = x.shape
    out = np.zeros((H, W), np.float32)
    ref_lib(name).ref_forward(np.ascontiguousarray(x, np.float32), out, W, H, k.w, k.w.size, k.off, k.rows, k.cols,
                              k.D, k.S, np.ascontiguousarray(var, np.float32), gamma)
    return out


def ref_stbi_loadf(path: str) -> np.ndarray:
    lib = ref_lib("v1_0")
    W, H = C.c_int(), C.c_int()
    p = lib.ref_stbi_loadf(path.encode(), C.byref(W), C.byref(H))
    if not p:
        raise ValueError(f"stbi_loadf failed on {path}")
    arr = np.ctypeslib.as_array(p, shape=(H.value * W.value,)).astype(np.float32, copy=True).reshape(H.value, W.value)
    lib.ref_stbi_free(C.cast(p, C.c_void_p))
    return arr


def ref_stbi_load_u8(path: str) -> np.ndarray:
    lib = ref_lib("v1_0")
    W, H = C.c_int(), C.c_int()
    p = lib.ref_stbi_load_u8(path.encode(), C.byref(W), C.byref(H))
    if not p:
        raise ValueError(f"stbi_load failed on {path}")
    arr = np.ctypeslib.as_array(p, shape=(H.value * W.value,)).astype(np.uint8, copy=True).reshape(H.value, W.value)
    lib.ref_stbi_free(C.cast(p, C.c_void_p))
    return arr


def ref_stbi_write_hdr(path: str, img: np.ndarray) -> None:
    H, W = img.shape
    if not ref_lib("v1_0").ref_stbi_write_hdr(path.encode(), W, H, np.ascontiguousarray(img, np.float32).ravel()):
        raise IOError(f"stbi_write_hdr failed on {path}")


def ref_pack_runs(k: DenseKernels):
    lib = ref_lib("v4_1")
    nr_max = int(k.rows.sum())
    weights = np.zeros(k.w.size, np.float32)
    rr, rc, rl = (np.zeros(nr_max, np.int32) for _ in range(3))
    kfr, knr, kfw = (np.zeros(k.nk, np.int32) for _ in range(3))
    nw = C.c_int()
    nr = lib.ref_pack_runs(k.w, k.off, k.rows, k.cols, k.nk, weights, rr, rc, rl, kfr, knr, kfw, C.byref(nw))
    return dict(weights=weights[: nw.value], run_row=rr[:nr], run_col=rc[:nr], run_len=rl[:nr],
                k_first_run=kfr, k_num_runs=knr, k_first_weight=kfw)


def ref_stbi_loadf_rgb(path: str) -> np.ndarray:
    """stbi_loadf(path, .., 3) of the reference's vendored stb_image: H x W x 3."""
    lib = ref_lib("v1_0")
    W, H = C.c_int(), C.c_int()
    p = lib.ref_stbi_loadf_rgb(path.encode(), C.byref(W), C.byref(H))
    if not p:
        raise IOError(path)
    img = np.ctypeslib.as_array(p, shape=(H.value, W.value, 3)).copy()
    lib.ref_stbi_free(C.cast(p, C.c_void_p))
    return img


def ref_stbi_write_hdr_rgb(path: str, img: np.ndarray) -> None:
    H, W, _ = img.shape
    if not ref_lib("v1_0").ref_stbi_write_hdr_rgb(path.encode(), W, H, np.ascontiguousarray(img, np.float32).ravel()):
        raise IOError(path)
