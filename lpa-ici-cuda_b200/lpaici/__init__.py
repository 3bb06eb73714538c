"""Python bindings of the B200 LPA-ICI denoiser (ctypes over lib/liblpaici.so, C ABI in include/lpaici.h).

Device buffers are torch CUDA tensors (float32, 2-D, row-major); their data pointers and the current
torch stream are handed to the C ABI.  There is no CPU fallback: if the shared library is missing,
importing this module raises ImportError.

Names follow the reference (titocapovilla/lpa-ici-cuda):
  KernelSet.load        <- load_LPA_kernels_standardized  src/v1_0_lpa_ici_2D_fused.cpp:466-551
  KernelSet.variances   <- compute_kernel_variances       src/v1_0_lpa_ici_2D_fused.cpp:691-717
  KernelSet.runs        <- build_sparse_kernels           src/v4_1_lpa_ici_2D_sparse_shared.cu:826-877
  forward               <- the directional loop of anisotropic_lpa_ici_gpu_fused
                           src/v4_1_lpa_ici_2D_sparse_shared.cu:1216-1235
  anisotropic_gpu_fused <- anisotropic_lpa_ici_gpu_fused  src/v4_1_lpa_ici_2D_sparse_shared.cu:1122-1244
  add_noise / psnr      <- create_noisy_image / calculate_PSNR  src/v1_0_lpa_ici_2D_fused.cpp:759-799
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "liblpaici.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is missing: build it with `make -C lpa-ici-cuda_b200` "
                      "(or __graft_entry__.build()); there is no CPU fallback")

_lib = C.CDLL(LIB_PATH)

OK = 0
ERR_INVALID_ARG = 1
ERR_FILE = 2
ERR_KERNEL_FORMAT = 3
ERR_UNSUPPORTED = 4
ERR_CUDA = 5
ERR_NO_MEMORY = 6


class LpaIciError(RuntimeError):
    """A nonzero status of the C ABI; .code is the LPAICI_ERR_* value."""

    def __init__(self, code: int, where: str):
        self.code = code
        msg = _lib.lpaici_last_error().decode(errors="replace")
        name = _lib.lpaici_status_string(code).decode()
        super().__init__(f"{where}: {name}: {msg}")


class KernelSetInfo(C.Structure):
    _fields_ = [("num_dirs", C.c_int), ("num_scales", C.c_int), ("dense_size", C.c_int), ("n_taps", C.c_int),
                ("n_runs", C.c_int), ("radius", C.c_int), ("blob_bytes", C.c_int), ("adjoint_blob_bytes", C.c_int)]


class Image(C.Structure):
    """lpaici_image: one image of a batch (device pointers)."""

    _fields_ = [("noisy", C.c_void_p), ("denoised", C.c_void_p), ("width", C.c_int), ("height", C.c_int),
                ("noisy_pitch", C.c_int), ("out_pitch", C.c_int), ("sigma", C.c_float), ("gamma", C.c_float),
                ("scale_map", C.c_void_p)]


class BatchOptions(C.Structure):
    _fields_ = [("use_graph", C.c_int), ("tile_config", C.c_int)]


class GradImage(C.Structure):
    """lpaici_grad_image"""

    _fields_ = [("noisy", C.c_void_p), ("grad_out", C.c_void_p), ("grad_in", C.c_void_p), ("width", C.c_int),
                ("height", C.c_int), ("noisy_pitch", C.c_int), ("gout_pitch", C.c_int), ("gin_pitch", C.c_int),
                ("sigma", C.c_float), ("gamma", C.c_float)]


_vp, _i, _f, _fp, _ip = C.c_void_p, C.c_int, C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_int)
_SIGS = {
    "lpaici_last_error": ([], C.c_char_p),
    "lpaici_status_string": ([_i], C.c_char_p),
    "lpaici_kernelset_load": ([C.c_char_p, C.POINTER(_vp)], _i),
    "lpaici_kernelset_create": ([_fp, _ip, _ip, _ip, _i, _i, C.POINTER(_vp)], _i),
    "lpaici_kernelset_save": ([_vp, C.c_char_p], _i),
    "lpaici_kernelset_destroy": ([_vp], _i),
    "lpaici_kernelset_get_info": ([_vp, C.POINTER(KernelSetInfo)], _i),
    "lpaici_kernelset_get_dense": ([_vp, _fp, _ip, _ip, _ip], _i),
    "lpaici_kernelset_get_runs": ([_vp, _fp, _ip, _ip, _ip, _ip, _ip, _ip], _i),
    "lpaici_kernel_variances": ([_vp, _f, _fp], _i),
    "lpaici_forward": ([_vp, _vp, _i, _vp, _i, _i, _i, _f, _f, _vp, _vp], _i),
    "lpaici_forward_var": ([_vp, _vp, _i, _vp, _i, _i, _i, _fp, _f, _vp, _vp], _i),
    "lpaici_forward_rows": ([_vp, _vp, _i, _i, _i, _i, _i, _vp, _i, _f, _f, _vp, _vp], _i),
    "lpaici_batch_create": ([_vp, C.POINTER(Image), _i, C.POINTER(BatchOptions), _vp, C.POINTER(_vp)], _i),
    "lpaici_batch_run": ([_vp, _vp], _i),
    "lpaici_batch_destroy": ([_vp], _i),
    "lpaici_forward_batched": ([_vp, C.POINTER(Image), _i, _vp], _i),
    "lpaici_num_tile_configs": ([], _i),
    "lpaici_tile_config_desc": ([_i, _ip, _ip, _ip, _ip], _i),
    "lpaici_autotune": ([_vp, _vp, _i, _i, _i, _f, _f, _i, _ip, _fp, _vp], _i),
    "lpaici_set_tile_config": ([_vp, _i], _i),
    "lpaici_backward": ([_vp, _vp, _i, _vp, _i, _vp, _i, _i, _i, _f, _f, _vp], _i),
    "lpaici_backward_noalloc": ([_vp, _vp, _i, _vp, _i, _vp, _i, _i, _i, _f, _f, _vp], _i),
    "lpaici_forward_ffma": ([_vp, _vp, _i, _vp, _i, _i, _i, _f, _f, _vp, _vp], _i),
    "lpaici_kernelset_generate": ([_i, _i, _ip, _i, _i, C.POINTER(_vp)], _i),
    "lpaici_kernelset_write_text": ([_vp, C.c_char_p], _i),
    "lpaici_trim_workspace": ([], _i),
    "lpaici_forward_channels": ([_vp, _vp, _i, _vp, _i, _i, _i, _i, _f, _f, _vp], _i),
    "lpaici_adjoint_state_bytes": ([_vp, _i, _i], C.c_size_t),
    "lpaici_forward_state": ([_vp, _vp, _i, _vp, _i, _i, _i, _f, _f, _vp, _vp], _i),
    "lpaici_backward_state": ([_vp, _vp, _vp, _i, _vp, _i, _i, _i, _f, _vp], _i),
    "lpaici_backward_batch_create": ([_vp, C.POINTER(GradImage), _i, C.POINTER(BatchOptions), _vp, C.POINTER(_vp)],
                                     _i),
    "lpaici_backward_batch_run": ([_vp, _vp], _i),
    "lpaici_backward_batch_destroy": ([_vp], _i),
    "lpaici_anisotropic_gpu_fused": ([_fp, _fp, _i, _i, _i, _fp, _i, _i, _fp, _i, _ip, _ip, _ip, _fp, _f,
                                      C.POINTER(C.c_double)], _i),
    "lpaici_denoise_host": ([_vp, _fp, _fp, _i, _i, _f, _f, _vp], _i),
    "lpaici_release_host_buffers": ([], _i),
    "lpaici_add_noise": ([_fp, _fp, C.c_long, _f, C.c_uint], _i),
    "lpaici_psnr": ([_fp, _fp, C.c_long], C.c_double),
}
for _name, (_args, _res) in _SIGS.items():
    _fn = getattr(_lib, _name)
    _fn.argtypes = _args
    _fn.restype = _res

EXPORTED = tuple(_SIGS)


def lib() -> C.CDLL:
    return _lib


def _check(code: int, where: str) -> None:
    if code != OK:
        raise LpaIciError(code, where)


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(_fp)


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(_ip)


@dataclass
class Runs:
    """The run-length packing in the reference's layout (build_sparse_kernels)."""

    weights: np.ndarray
    run_row: np.ndarray
    run_col: np.ndarray
    run_len: np.ndarray
    kernel_first_run: np.ndarray
    kernel_num_runs: np.ndarray
    kernel_first_weight: np.ndarray


class KernelSet:
    """An immutable LPA kernel set (D directions x S scales), packed into row runs in device memory."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)
        info = KernelSetInfo()
        _check(_lib.lpaici_kernelset_get_info(self._h, C.byref(info)), "lpaici_kernelset_get_info")
        self.info = info

    @classmethod
    def load(cls, path: str) -> "KernelSet":
        h = C.c_void_p()
        _check(_lib.lpaici_kernelset_load(os.fsencode(path), C.byref(h)), f"lpaici_kernelset_load({path})")
        return cls(h.value)

    @classmethod
    def from_dense(cls, weights, offsets, rows, cols, num_dirs: int, num_scales: int) -> "KernelSet":
        w = np.ascontiguousarray(weights, np.float32)
        o, r, c = (np.ascontiguousarray(a, np.int32) for a in (offsets, rows, cols))
        h = C.c_void_p()
        _check(_lib.lpaici_kernelset_create(_fptr(w), _iptr(o), _iptr(r), _iptr(c), num_dirs, num_scales,
                                            C.byref(h)), "lpaici_kernelset_create")
        return cls(h.value)

    @classmethod
    def generate(cls, num_dirs: int, scales, order: int = 0, shape: str = "sector") -> "KernelSet":
        """Directional LPA kernels from their definition (lpaici_kernelset_generate): `shape` "sector"
        or "quadrant", polynomial `order` along the direction, one kernel per scale in `scales`."""
        sc = np.ascontiguousarray(scales, np.int32)
        code = {"sector": 0, "quadrant": 1}[shape]
        h = C.c_void_p()
        _check(_lib.lpaici_kernelset_generate(num_dirs, sc.size, _iptr(sc), order, code, C.byref(h)),
               "lpaici_kernelset_generate")
        return cls(h.value)

    def save_text(self, path: str) -> None:
        """The reference's text kernel format (lpaici_kernelset_write_text)."""
        _check(_lib.lpaici_kernelset_write_text(self._h, path.encode()), "lpaici_kernelset_write_text")

    def save(self, path: str) -> None:
        """Writes the binary tap-list file that load() reads back (lpaici_kernelset_save)."""
        _check(_lib.lpaici_kernelset_save(self.handle, os.fsencode(path)), f"lpaici_kernelset_save({path})")

    def close(self) -> None:
        if self._h and self._h.value:
            _lib.lpaici_kernelset_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    @property
    def D(self) -> int:
        return self.info.num_dirs

    @property
    def S(self) -> int:
        return self.info.num_scales

    @property
    def radius(self) -> int:
        return self.info.radius

    def dense(self):
        """(weights, offsets, rows, cols) exactly as the reference's loader returns them."""
        nk = self.D * self.S
        w = np.zeros(self.info.dense_size, np.float32)
        o, r, c = (np.zeros(nk, np.int32) for _ in range(3))
        _check(_lib.lpaici_kernelset_get_dense(self._h, _fptr(w), _iptr(o), _iptr(r), _iptr(c)),
               "lpaici_kernelset_get_dense")
        return w, o, r, c

    def runs(self) -> Runs:
        nk = self.D * self.S
        w = np.zeros(self.info.n_taps, np.float32)
        rr, rc, rl = (np.zeros(self.info.n_runs, np.int32) for _ in range(3))
        kfr, knr, kfw = (np.zeros(nk, np.int32) for _ in range(3))
        _check(_lib.lpaici_kernelset_get_runs(self._h, _fptr(w), _iptr(rr), _iptr(rc), _iptr(rl), _iptr(kfr),
                                              _iptr(knr), _iptr(kfw)), "lpaici_kernelset_get_runs")
        return Runs(w, rr, rc, rl, kfr, knr, kfw)

    def variances(self, sigma: float) -> np.ndarray:
        var = np.zeros(self.D * self.S, np.float32)
        _check(_lib.lpaici_kernel_variances(self._h, sigma, _fptr(var)), "lpaici_kernel_variances")
        return var

    def nnz(self) -> np.ndarray:
        """Nonzero taps per kernel (k = d*S + s)."""
        w, o, r, c = self.dense()
        return np.array([np.count_nonzero(w[o[k]:o[k] + r[k] * c[k]]) for k in range(self.D * self.S)], np.int64)

    def autotune(self, width: int, height: int, sigma: float, gamma: float, sample=None, reps: int = 3):
        """Times every tile configuration; makes the fastest this kernel set's default on this device.
        Returns (best_config, per-config milliseconds)."""
        import torch

        n = _lib.lpaici_num_tile_configs()
        ms = np.zeros(n, np.float32)
        best = C.c_int(-1)
        ptr, pitch = (None, width) if sample is None else (C.c_void_p(sample.data_ptr()), sample.stride(0))
        _check(_lib.lpaici_autotune(self._h, ptr, width, height, pitch, sigma, gamma, reps, C.byref(best),
                                    _fptr(ms), _stream(torch)), "lpaici_autotune")
        return best.value, ms

    def set_tile_config(self, config: int) -> None:
        _check(_lib.lpaici_set_tile_config(self._h, config), "lpaici_set_tile_config")


def tile_configs():
    """[(tile_w, tile_h, threads, pixels_per_thread)] of every tile configuration."""
    out = []
    for i in range(_lib.lpaici_num_tile_configs()):
        v = [C.c_int() for _ in range(4)]
        _check(_lib.lpaici_tile_config_desc(i, *[C.byref(x) for x in v]), "lpaici_tile_config_desc")
        out.append(tuple(x.value for x in v))
    return out


# ---- device entry points (torch tensors) --------------------------------------------------------

def _stream(torch):
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _check_image(t, name: str):
    import torch

    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.dim() == 2
            and t.stride(1) == 1):
        raise ValueError(f"{name} must be a 2-D float32 CUDA tensor with unit column stride")


def forward(ks: KernelSet, noisy, sigma: float, gamma: float, out=None, scale_map: bool | object = False,
            variances: Optional[np.ndarray] = None, ffma: bool = False):
    """Denoises one image on its device.  Returns out, or (out, scale_map uint8 [D, H, W]) when scale_map
    is True (or a preallocated tensor).  With `variances` (D*S floats) the reference's caller-supplied
    variances are used instead of sigma.  ffma=True: lpaici_forward_ffma (fused multiply-adds, not
    bit-exact with the reference)."""
    import torch

    _check_image(noisy, "noisy")
    H, W = noisy.shape
    if out is None:
        out = torch.empty((H, W), dtype=torch.float32, device=noisy.device)
    _check_image(out, "out")
    smap = None
    if scale_map is True:
        smap = torch.empty((ks.D, H, W), dtype=torch.uint8, device=noisy.device)
    elif scale_map is not False and scale_map is not None:
        smap = scale_map
    sp = C.c_void_p(smap.data_ptr()) if smap is not None else None
    with torch.cuda.device(noisy.device):
        if ffma:
            if variances is not None:
                raise ValueError("ffma=True takes sigma, not variances")
            rc = _lib.lpaici_forward_ffma(ks.handle, C.c_void_p(noisy.data_ptr()), noisy.stride(0),
                                          C.c_void_p(out.data_ptr()), out.stride(0), W, H, sigma, gamma, sp,
                                          _stream(torch))
            _check(rc, "lpaici_forward_ffma")
        elif variances is None:
            rc = _lib.lpaici_forward(ks.handle, C.c_void_p(noisy.data_ptr()), noisy.stride(0),
                                     C.c_void_p(out.data_ptr()), out.stride(0), W, H, sigma, gamma, sp, _stream(torch))
            _check(rc, "lpaici_forward")
        else:
            v = np.ascontiguousarray(variances, np.float32)
            rc = _lib.lpaici_forward_var(ks.handle, C.c_void_p(noisy.data_ptr()), noisy.stride(0),
                                         C.c_void_p(out.data_ptr()), out.stride(0), W, H, _fptr(v), gamma, sp,
                                         _stream(torch))
            _check(rc, "lpaici_forward_var")
    return (out, smap) if smap is not None else out


def forward_rows(ks: KernelSet, band, row_begin: int, row_count: int, sigma: float, gamma: float, out=None,
                 scale_map=None):
    """Output rows [row_begin, row_begin + row_count) of the band `band` (rows outside it are zero)."""
    import torch

    _check_image(band, "band")
    H_in, W = band.shape
    if out is None:
        out = torch.empty((row_count, W), dtype=torch.float32, device=band.device)
    sp = C.c_void_p(scale_map.data_ptr()) if scale_map is not None else None
    with torch.cuda.device(band.device):
        rc = _lib.lpaici_forward_rows(ks.handle, C.c_void_p(band.data_ptr()), band.stride(0), W, H_in, row_begin,
                                      row_count, C.c_void_p(out.data_ptr()), out.stride(0), sigma, gamma, sp,
                                      _stream(torch))
    _check(rc, "lpaici_forward_rows")
    return out


def forward_channels(ks: KernelSet, noisy, sigma: float, gamma: float, out=None):
    """Denoises every channel of an interleaved H x W x C image (CUDA float32, rows contiguous within
    themselves) on its own: lpaici_forward_channels."""
    import torch

    if noisy.dim() != 3 or noisy.dtype != torch.float32 or not noisy.is_cuda or noisy.stride(2) != 1 or \
            noisy.stride(1) != noisy.shape[2]:
        raise ValueError("noisy: a CUDA float32 H x W x C tensor with interleaved channels")
    H, W, Cn = noisy.shape
    if out is None:
        out = torch.empty_like(noisy)
    with torch.cuda.device(noisy.device):
        rc = _lib.lpaici_forward_channels(ks.handle, C.c_void_p(noisy.data_ptr()), noisy.stride(0),
                                          C.c_void_p(out.data_ptr()), out.stride(0), W, H, Cn, sigma, gamma,
                                          _stream(torch))
    _check(rc, "lpaici_forward_channels")
    return out


def forward_state(ks: KernelSet, noisy, sigma: float, gamma: float, out=None, state=None):
    """lpaici_forward_state: (denoised, state), the state (uint8 CUDA tensor, reused when given) holding
    what backward_state needs."""
    import torch

    _check_image(noisy, "noisy")
    H, W = noisy.shape
    if out is None:
        out = torch.empty((H, W), dtype=torch.float32, device=noisy.device)
    _check_image(out, "out")
    nbytes = int(_lib.lpaici_adjoint_state_bytes(ks.handle, W, H))
    if state is None:
        state = torch.empty(nbytes, dtype=torch.uint8, device=noisy.device)
    elif state.numel() < nbytes or state.dtype != torch.uint8:
        raise ValueError(f"state: a uint8 tensor of at least {nbytes} bytes")
    with torch.cuda.device(noisy.device):
        rc = _lib.lpaici_forward_state(ks.handle, C.c_void_p(noisy.data_ptr()), noisy.stride(0),
                                       C.c_void_p(out.data_ptr()), out.stride(0), W, H, sigma, gamma,
                                       C.c_void_p(state.data_ptr()), _stream(torch))
    _check(rc, "lpaici_forward_state")
    return out, state


def backward_state(ks: KernelSet, state, grad_out, sigma: float, grad_in=None):
    """lpaici_backward_state: the adjoint from a forward_state state (gather pass only)."""
    import torch

    _check_image(grad_out, "grad_out")
    H, W = grad_out.shape
    if grad_in is None:
        grad_in = torch.empty((H, W), dtype=torch.float32, device=grad_out.device)
    with torch.cuda.device(grad_out.device):
        rc = _lib.lpaici_backward_state(ks.handle, C.c_void_p(state.data_ptr()), C.c_void_p(grad_out.data_ptr()),
                                        grad_out.stride(0), C.c_void_p(grad_in.data_ptr()), grad_in.stride(0), W, H,
                                        sigma, _stream(torch))
    _check(rc, "lpaici_backward_state")
    return grad_in


def backward(ks: KernelSet, noisy, grad_out, sigma: float, gamma: float, grad_in=None):
    """d(sum(grad_out * forward(noisy)))/d(noisy) with the ICI selection held fixed."""
    import torch

    _check_image(noisy, "noisy")
    _check_image(grad_out, "grad_out")
    H, W = noisy.shape
    if grad_in is None:
        grad_in = torch.empty((H, W), dtype=torch.float32, device=noisy.device)
    with torch.cuda.device(noisy.device):
        rc = _lib.lpaici_backward(ks.handle, C.c_void_p(noisy.data_ptr()), noisy.stride(0),
                                  C.c_void_p(grad_out.data_ptr()), grad_out.stride(0), C.c_void_p(grad_in.data_ptr()),
                                  grad_in.stride(0), W, H, sigma, gamma, _stream(torch))
    _check(rc, "lpaici_backward")
    return grad_in


class Batch:
    """A planned batch of images (lpaici_batch): one persistent launch over a shared tile queue,
    optionally replayed from a CUDA graph."""

    def __init__(self, ks: KernelSet, noisy: Sequence, outs: Sequence, sigmas: Sequence[float],
                 gammas: Sequence[float], use_graph: bool = True, tile_config: int = -1, scale_maps=None):
        import torch

        n = len(noisy)
        self._keep = (list(noisy), list(outs), scale_maps)
        arr = (Image * n)()
        for i in range(n):
            _check_image(noisy[i], f"noisy[{i}]")
            _check_image(outs[i], f"outs[{i}]")
            H, W = noisy[i].shape
            arr[i] = Image(noisy[i].data_ptr(), outs[i].data_ptr(), W, H, noisy[i].stride(0), outs[i].stride(0),
                           float(sigmas[i]), float(gammas[i]),
                           scale_maps[i].data_ptr() if scale_maps is not None else None)
        opts = BatchOptions(1 if use_graph else 0, tile_config)
        h = C.c_void_p()
        self.device = noisy[0].device
        with torch.cuda.device(self.device):
            _check(_lib.lpaici_batch_create(ks.handle, arr, n, C.byref(opts), _stream(torch), C.byref(h)),
                   "lpaici_batch_create")
        self._h = h

    def run(self) -> None:
        import torch

        with torch.cuda.device(self.device):
            _check(_lib.lpaici_batch_run(self._h, _stream(torch)), "lpaici_batch_run")

    def close(self) -> None:
        if self._h and self._h.value:
            _lib.lpaici_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BackwardBatch:
    """A planned batched adjoint (lpaici_backward_batch): selection of all images in one persistent
    launch, gather of all images' tiles in one launch, optionally replayed from a CUDA graph."""

    def __init__(self, ks: KernelSet, noisy: Sequence, grad_out: Sequence, grad_in: Sequence,
                 sigmas: Sequence[float], gammas: Sequence[float], use_graph: bool = True, tile_config: int = -1):
        import torch

        n = len(noisy)
        self._keep = (list(noisy), list(grad_out), list(grad_in))
        arr = (GradImage * n)()
        for i in range(n):
            for t, name in ((noisy[i], "noisy"), (grad_out[i], "grad_out"), (grad_in[i], "grad_in")):
                _check_image(t, f"{name}[{i}]")
            H, W = noisy[i].shape
            arr[i] = GradImage(noisy[i].data_ptr(), grad_out[i].data_ptr(), grad_in[i].data_ptr(), W, H,
                               noisy[i].stride(0), grad_out[i].stride(0), grad_in[i].stride(0), float(sigmas[i]),
                               float(gammas[i]))
        opts = BatchOptions(1 if use_graph else 0, tile_config)
        h = C.c_void_p()
        self.device = noisy[0].device
        with torch.cuda.device(self.device):
            _check(_lib.lpaici_backward_batch_create(ks.handle, arr, n, C.byref(opts), _stream(torch), C.byref(h)),
                   "lpaici_backward_batch_create")
        self._h = h

    def run(self) -> None:
        import torch

        with torch.cuda.device(self.device):
            _check(_lib.lpaici_backward_batch_run(self._h, _stream(torch)), "lpaici_backward_batch_run")

    def close(self) -> None:
        if self._h and self._h.value:
            _lib.lpaici_backward_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def forward_batched(ks: KernelSet, noisy: Sequence, sigmas: Sequence[float], gammas: Sequence[float], outs=None):
    """One-shot batched forward (plans, runs, synchronises, frees)."""
    import torch

    if outs is None:
        outs = [torch.empty_like(x) for x in noisy]
    n = len(noisy)
    arr = (Image * n)()
    for i in range(n):
        H, W = noisy[i].shape
        arr[i] = Image(noisy[i].data_ptr(), outs[i].data_ptr(), W, H, noisy[i].stride(0), outs[i].stride(0),
                       float(sigmas[i]), float(gammas[i]), None)
    with torch.cuda.device(noisy[0].device):
        _check(_lib.lpaici_forward_batched(ks.handle, arr, n, _stream(torch)), "lpaici_forward_batched")
    return outs


# ---- host-pointer entry points ------------------------------------------------------------------

def anisotropic_gpu_fused(noisy: np.ndarray, weights, offsets, rows, cols, num_dirs: int, num_scales: int,
                          variances, gamma: float):
    """The reference engine's signature: host in, host out, caller's variances.  Returns (out, seconds)."""
    x = np.ascontiguousarray(noisy, np.float32)
    H, W = x.shape
    out = np.zeros_like(x)
    w = np.ascontiguousarray(weights, np.float32)
    o, r, c = (np.ascontiguousarray(a, np.int32) for a in (offsets, rows, cols))
    v = np.ascontiguousarray(variances, np.float32)
    secs = C.c_double()
    _check(_lib.lpaici_anisotropic_gpu_fused(_fptr(x), _fptr(out), W, H, 1, None, num_dirs, num_scales, _fptr(w),
                                             w.size, _iptr(o), _iptr(r), _iptr(c), _fptr(v), gamma, C.byref(secs)),
           "lpaici_anisotropic_gpu_fused")
    return out, secs.value


def denoise_host(ks: KernelSet, noisy: np.ndarray, sigma: float, gamma: float, out: Optional[np.ndarray] = None,
                 stream=None):
    """Host array in, host array out (H2D, forward, D2H, synchronise).  Pinned `noisy`/`out` copy fastest."""
    x = np.ascontiguousarray(noisy, np.float32)
    H, W = x.shape
    if out is None:
        out = np.empty_like(x)
    _check(_lib.lpaici_denoise_host(ks.handle, _fptr(x), _fptr(out), W, H, sigma, gamma, stream),
           "lpaici_denoise_host")
    return out


def add_noise(clean: np.ndarray, sigma: float, seed: int) -> np.ndarray:
    """clean + N(0, sigma) from std::mt19937{seed} / std::normal_distribution<float> (create_noisy_image)."""
    c = np.ascontiguousarray(clean, np.float32)
    out = np.empty_like(c)
    _check(_lib.lpaici_add_noise(_fptr(c), _fptr(out), c.size, sigma, seed), "lpaici_add_noise")
    return out


def psnr(a: np.ndarray, b: np.ndarray) -> float:
    """calculate_PSNR: 10*log10(1/MSE), float differences squared in float, summed in double."""
    x = np.ascontiguousarray(a, np.float32)
    y = np.ascontiguousarray(b, np.float32)
    return _lib.lpaici_psnr(_fptr(x), _fptr(y), x.size)


from .synth import synth_image  # noqa: E402  (benchmark input generator)
