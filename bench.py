#!/usr/bin/env python
"""Benchmark of the B200 LPA-ICI denoiser; prints ONE JSON line (rank 0).

Workload (one step): the plain single-image forward on a 4096x4096 FP32 synthetic image (polygons,
linear ramp, 4-16 px stripes; RGBE-quantised; noise sigma = 20/255 from seed 20250910), 16 directions
x 7 scales of the symmetric m=(1,0) kernel set, gamma = 2.  With --gpus N every rank denoises its own
4096^2 image (weak scaling, no collective on the data path); `value` = all ranks' pixels / the slowest
rank's time.

  value     Mpix/s with the input resident in HBM, device time of the forward launch (CUDA events on
            the launching stream), L2 flushed (256 MB write) between timed steps
  e2e       the same metric through the C ABI's host-pointer entry (lpaici_denoise_host): pinned host
            input -> H2D -> forward -> D2H -> host (row bands, copies overlapped with the kernels on
            separate streams), returns when the output is in host memory, wall clock per step
  roofline  FP32 bound: every tap is one multiply and one separately rounded add (bit-exact with the
            reference), so the peak is the FP32 pipe's measured rate for exactly that (probe in
            lib/liblpaici_bench.so, the faster of scalar FMUL+FADD and packed fma(w,x,-0)+add);
            achieved = 2 x algorithmic taps / kernel time
  cpu_baseline  the reference's own CPU engine (anisotropic_lpa_ici_cpu_fused of
            src/v1_0_lpa_ici_2D_fused.cpp, compiled in-process into oracle/_ref/) on all host cores,
            one 256x256 crop of the benchmark image per thread; its naive engine (v0_0) beside it
  parity    the GPU image against those reference outputs, bit for bit, on every crop pixel whose
            neighbourhood lies inside its crop
  extra     batched forward (one launch) over 64 images (sides U[256,2048], sigma U[10,40]/255, gamma
            U[1.5,2.5]) in a CUDA graph, four 4096^2 images as one plan, and the adjoint on 8 x 1024^2
            (with the gather's FFMA rate), each against the plain forward on the same images; forward
            and adjoint on one 8192^2 image with the gaussian m=(2,0) kernels (sigma 25/255, gamma 1.5);
            adjoint checked by sum(g*out) = sum(grad*x)

--impl reference runs only the reference's CPU engine (bounded sample per step, all host threads).
"""
from __future__ import annotations

import argparse
import datetime
import gzip
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "lpa-ici-cuda_b200")
sys.path.insert(0, PKG)

METRIC = "Mpix/s at 4096^2 16x7: batched+adjoint vs plain on same GPU, max err<=1e-4"
UNIT = "Mpix/s"
SYM = "lpa_kernels_m_1_0_d_16_h12_1_2_4_8_16_24_32_symmetric.txt"
GAUSS_M2 = "lpa_kernels_m_2_0_d_16_h12_1_2_4_8_16_24_32_gaussian.txt"
SIGMA = float(np.float32(20.0) / np.float32(255.0))
GAMMA = 2.0
SEED = 20250910
SIZE = 4096
# DRAM bytes of one forward launch on the 4096^2 workload, read + written, from the ncu capture in
# profiles/forward_4096_sym.md (dram__bytes_read.sum + dram__bytes_write.sum; the halo re-reads are
# served by L2), valid for the tile configurations listed (the two 768-thread shapes, which stage the
# same halo'd tiles): reported only when the run uses one of them at that size.
FORWARD_DRAM_BYTES = 95.0e6
FORWARD_DRAM_CONFIGS = (9, 10)


def kernel_path(name: str, tmp: str) -> str:
    gz = os.path.join(ROOT, "tests", "golden", "kernels", name + ".gz")
    out = os.path.join(tmp, name)
    with gzip.open(gz, "rb") as f, open(out, "wb") as g:
        shutil.copyfileobj(f, g)
    return out


def bench_image(size: int, seed: int, sigma: float):
    import lpaici

    clean = lpaici.synth_image(size, size, seed)
    return clean, lpaici.add_noise(clean, sigma, SEED)


def synth_module():
    """lpaici/synth.py loaded on its own (numpy only): the reference arm builds the same image without
    importing the package, whose import loads this project's library."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("lpaici_synth", os.path.join(PKG, "lpaici", "synth.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def reference_bench_image(size: int, seed: int, sigma: float):
    """The benchmark image of bench_image, noise drawn by the reference's own create_noisy_image
    (src/v1_0_lpa_ici_2D_fused.cpp:759-776, compiled into oracle/_ref/): bit-identical to lpaici.add_noise
    (same std::mt19937 and std::normal_distribution<float>)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_bind as ob

    clean = synth_module().synth_image(size, size, seed)
    return clean, ob.ref_noise(clean, sigma, SEED)


class Clocks:
    """nvidia-smi samples during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "10"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def wait_samples(self, n: int, keep_busy, timeout_s: float = 5.0) -> None:
        """Runs keep_busy() (untimed GPU work) until the sampler has delivered n lines, so the
        timed region starts with the sampler already running under load."""
        t_end = time.perf_counter() + timeout_s
        while self.proc is not None and len(self.lines) < n and time.perf_counter() < t_end:
            keep_busy()

    def mark(self, start: bool) -> None:
        if start:
            self.t0 = time.perf_counter()
        else:
            self.t1 = time.perf_counter()

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        # samples taken while the timed steps ran; nvidia-smi delivers one every ~10-100 ms, so a short
        # region is widened by 150 ms on each side, where the GPU runs the warm-up steps and the flush
        t0, t1 = getattr(self, "t0", 0.0) - 0.15, getattr(self, "t1", float("inf")) + 0.15
        for t, ln in self.lines:
            if not t0 <= t <= t1:
                continue
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                smax.append(float(f[1]))
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm), "window": "timed region +- 150 ms"}


def fp32_peak() -> dict:
    import ctypes as C

    lib = C.CDLL(os.path.join(PKG, "lib", "liblpaici_bench.so"))
    lib.lpaici_bench_fp32_peak.argtypes = [C.POINTER(C.c_double)]
    r = (C.c_double * 3)()
    if lib.lpaici_bench_fp32_peak(r) != 0:
        raise RuntimeError("FP32 peak probe failed")
    return {"ffma_ops_per_s": r[0], "muladd_ops_per_s": r[1], "prodadd2_ops_per_s": r[2]}


def algorithmic_taps(torch, ks, smap) -> float:
    """Taps the reference's fused loop convolves: for every (direction, pixel), all nonzero taps of
    scales 0 .. min(s*+1, S-1) (the first rejected scale is convolved, then dropped)."""
    nnz = torch.tensor(ks.nnz().reshape(ks.D, ks.S), dtype=torch.float64, device=smap.device)
    prefix = torch.cumsum(nnz, dim=1)  # prefix[d, s] = taps of scales 0..s
    stop = torch.clamp(smap.long() + 1, max=ks.S - 1)
    total = 0.0
    for d in range(ks.D):
        total += float(prefix[d][stop[d]].sum())
    return total


def time_launches(torch, fn, steps: int, warmup: int, flush) -> list[float]:
    """Per-step device milliseconds of fn() (events on the current stream), L2 flushed in between."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ms = []
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    return ms


def cpu_reference_sample(noisy: np.ndarray, crop: int, threads: int, sigma: float, gamma: float, seed: int = 0,
                         engine: str = "v1_0", keep: bool = False):
    """The reference's CPU engine (`engine`: v1_0 fused or v0_0 naive) on `threads` distinct crop x crop
    pieces of `noisy`, one per thread, each denoised as a whole image (as the reference's executables
    do).  Returns (Mpix/s, seconds, [(y, x, output)] if keep else None)."""
    import concurrent.futures as cf

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_bind as ob  # the reference compiled from its sources (oracle/_ref): timed, not shipped

    H, W = noisy.shape
    rng = np.random.default_rng(seed)
    corners, crops = [], []
    for _ in range(threads):
        y, x = (int(v) for v in rng.integers(0, [H - crop + 1, W - crop + 1]))
        corners.append((y, x))
        crops.append(np.ascontiguousarray(noisy[y:y + crop, x:x + crop]))
    tmp = tempfile.mkdtemp()
    with quiet_stdout():  # the reference prints progress lines on stdout: keep them off the JSON line
        try:
            k = ob.ref_load_kernels(kernel_path(SYM, tmp), name=engine)
        finally:
            shutil.rmtree(tmp, ignore_errors=True)
        var = ob.ref_variances(k, np.float32(sigma), name=engine)
        t0 = time.perf_counter()
        with cf.ThreadPoolExecutor(max_workers=threads) as ex:
            outs = list(ex.map(lambda c: ob.ref_forward(c, k, var, gamma, name=engine), crops))
        secs = time.perf_counter() - t0
    kept = [(y, x, o) for (y, x), o in zip(corners, outs)] if keep else None
    return threads * crop * crop / secs / 1e6, secs, kept


def crop_parity(got: np.ndarray, kept, R: int) -> dict:
    """The GPU result against the reference's own CPU results on the crops: every crop pixel whose
    R-neighbourhood lies inside the crop sees the same input as in the full image, so it must match
    bit for bit."""
    n = mism = 0
    err = 0.0
    for y, x, ref in kept:
        h, w = ref.shape
        a = got[y + R:y + h - R, x + R:x + w - R]
        b = ref[R:h - R, R:w - R]
        n += a.size
        mism += int(np.count_nonzero(a.view(np.uint32) != b.view(np.uint32)))
        err = max(err, float(np.abs(a.astype(np.float64) - b.astype(np.float64)).max()))
    return {"against": "reference CPU engine (v1_0) on the cpu_baseline crops, interior pixels",
            "pixels": n, "bit_mismatches": mism, "max_abs_err": err, "bit_exact": mism == 0}


class quiet_stdout:
    """Sends file descriptor 1 to /dev/null (C and C++ writers included, buffers flushed both ways)."""

    def __enter__(self):
        import ctypes

        self.libc = ctypes.CDLL(None)
        sys.stdout.flush()
        self.libc.fflush(None)
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)

    def __exit__(self, *exc):
        self.libc.fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)
        return False


class capture_stdout(quiet_stdout):
    """Like quiet_stdout, into a temporary file whose text is .text after the block."""

    def __enter__(self):
        import ctypes

        self.libc = ctypes.CDLL(None)
        sys.stdout.flush()
        self.libc.fflush(None)
        self.saved = os.dup(1)
        self.file = tempfile.TemporaryFile(mode="w+b")
        self.null = os.dup(self.file.fileno())
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *exc):
        super().__exit__(*exc)
        self.file.seek(0)
        self.text = self.file.read().decode(errors="replace")
        self.file.close()
        return False


def reference_gpu_v4_1(clean: np.ndarray, noisy: np.ndarray, ours: np.ndarray, steps: int) -> dict:
    """The reference's own fastest GPU engine, anisotropic_lpa_ici_gpu_fused of
    src/v4_1_lpa_ici_2D_sparse_shared.cu (:1122-1244: 16 launches of process_direction_fused_kernel +
    aggregation, kernels in constant memory), compiled from its sources for sm_100a into
    oracle/_ref/libref_v4_1.so and called as its main() does, on this run's image and GPU.  Timed by its
    own window (after the uploads to after the download of the result, :1216-1240), read from the line it
    prints, and by the wall clock of the whole call.  Its output is compared with this project's, which
    is bit-exact with the reference's CPU engine: the v4_1 build lets nvcc contract its multiply-adds
    into FFMA (default -fmad=true), so it differs where rounding moves an ICI decision."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_bind as ob

    if not (ob.ref_available("v4_1") and ob.ref_available("v1_0")):
        return {"unavailable": "oracle/_ref/libref_v4_1.so or libref_v1_0.so not built"}
    tmp = tempfile.mkdtemp()
    try:
        with quiet_stdout():
            k = ob.ref_load_kernels(kernel_path(SYM, tmp))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    var = ob.ref_variances(k, np.float32(SIGMA))
    H, W = noisy.shape
    x = np.ascontiguousarray(noisy, np.float32)
    out = np.zeros_like(x)
    lib = ob.ref_lib("v4_1")
    windows, walls = [], []
    for i in range(1 + steps):  # the first call (module load, constant uploads) is not kept
        with capture_stdout() as cap:
            t0 = time.perf_counter()
            lib.ref_gpu_fused(x, out, W, H, k.w, k.w.size, k.off, k.rows, k.cols, k.D, k.S, var, np.float32(GAMMA))
            wall = time.perf_counter() - t0
        t = [float(ln.rsplit(":", 1)[1].split()[0]) for ln in cap.text.splitlines()
             if ln.startswith("Time taken for directional loops + aggregation")]
        if i > 0 and t:
            windows.append(t[-1])
            walls.append(wall)
    if not windows:
        return {"unavailable": "the reference engine printed no timing line"}
    px = W * H
    a64, b64 = ours.astype(np.float64), out.astype(np.float64)
    with quiet_stdout():
        psnr_ours = ob.ref_psnr(clean, ours)
        psnr_ref = ob.ref_psnr(clean, out)
    return {"engine": "anisotropic_lpa_ici_gpu_fused, src/v4_1_lpa_ici_2D_sparse_shared.cu (built -O3 for sm_100a)",
            "size": W, "steps": len(windows), "unit": UNIT,
            "value": px / float(np.mean(windows)) / 1e6,
            "window": "the reference's own: after the uploads to after the download of the result",
            "value_wall": px / float(np.mean(walls)) / 1e6,
            "ms_window": float(np.mean(windows)) * 1e3, "ms_wall": float(np.mean(walls)) * 1e3,
            "ours_e2e_over_reference": None,
            "output_vs_ours": {"max_abs_err": float(np.abs(a64 - b64).max()),
                               "pixels_differing": int(np.count_nonzero(ours.view(np.uint32) != out.view(np.uint32))),
                               "pixels_over_1e-4": int(np.count_nonzero(np.abs(a64 - b64) > 1e-4)),
                               "psnr_ours_db": psnr_ours, "psnr_reference_gpu_db": psnr_ref,
                               "psnr_delta_db": psnr_ref - psnr_ours}}


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference(args, rank: int, world: int) -> None:
    if rank != 0:
        return
    threads = host_threads()
    _, noisy = reference_bench_image(SIZE, SEED, SIGMA)
    for _ in range(args.warmup):
        cpu_reference_sample(noisy, 64, threads, SIGMA, GAMMA, seed=1)
    vals, secs = [], []
    for i in range(args.steps):
        v, s, _ = cpu_reference_sample(noisy, args.ref_crop, threads, SIGMA, GAMMA, seed=100 + i)
        vals.append(v)
        secs.append(s)
    value = float(np.mean(vals))
    sample = (f"{threads} crops of {args.ref_crop}x{args.ref_crop} px of the 4096^2 benchmark image per step, "
              f"one per host thread, each denoised as a whole image by anisotropic_lpa_ici_cpu_fused")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(secs)) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"plain LPA-ICI forward, sym 16x7, sigma 20/255, gamma 2: a sample of {threads} crops "
                               f"of {args.ref_crop}x{args.ref_crop} px of the 4096x4096 synthetic benchmark image per "
                               "step, each denoised as a whole image",
                   "reference": "titocapovilla/lpa-ici-cuda src/v1_0_lpa_ici_2D_fused.cpp (CPU, built -O3)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank: int, world: int, local_rank: int) -> None:
    import torch

    import lpaici

    dist = world > 1
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    tmp = tempfile.mkdtemp()
    ks = lpaici.KernelSet.load(kernel_path(SYM, tmp))
    size = args.size
    clean, noisy_h = bench_image(size, SEED + rank, SIGMA)
    x = torch.from_numpy(noisy_h).to(dev)
    out = torch.empty_like(x)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2

    # untimed: tile autotune on this image, scale maps for the algorithmic tap count
    if args.tile_config >= 0:
        best, tune_ms = args.tile_config, []
        ks.set_tile_config(best)
    else:
        best, tune_ms = ks.autotune(size, size, SIGMA, GAMMA, sample=x, reps=2)
    _, smap = lpaici.forward(ks, x, SIGMA, GAMMA, out=out, scale_map=True)
    torch.cuda.synchronize()
    taps = algorithmic_taps(torch, ks, smap)
    del smap

    fwd = lambda: lpaici.forward(ks, x, SIGMA, GAMMA, out=out)  # noqa: E731
    clocks = Clocks(local_rank)
    clocks.start()
    for _ in range(args.warmup):
        fwd()
    torch.cuda.synchronize()
    clocks.wait_samples(2, lambda: (fwd(), torch.cuda.synchronize()))  # more untimed warm-up steps
    if dist:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks.mark(True)
    ms = time_launches(torch, fwd, args.steps, 0, flush)
    torch.cuda.synchronize()
    clocks.mark(False)
    if dist:
        torch.distributed.barrier()
    clk = clocks.stop()
    ms_step = float(np.mean(ms))
    if dist:
        t = torch.tensor([ms_step], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms_step = float(t.item())
    px = size * size
    value = world * px / (ms_step * 1e-3) / 1e6


    # e2e through the C ABI with pinned host buffers
    pin_in = torch.from_numpy(noisy_h).pin_memory()
    pin_out = torch.empty_like(pin_in).pin_memory()
    host_in, host_out = pin_in.numpy(), pin_out.numpy()
    for _ in range(max(1, args.warmup)):
        lpaici.denoise_host(ks, host_in, SIGMA, GAMMA, out=host_out)
    if dist:
        torch.distributed.barrier()
    e2e_s = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lpaici.denoise_host(ks, host_in, SIGMA, GAMMA, out=host_out)
        e2e_s.append(time.perf_counter() - t0)
    e2e_step = float(np.mean(e2e_s))
    if dist:
        t = torch.tensor([e2e_step], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_step = float(t.item())
    if not np.array_equal(host_out.view(np.uint32), out.cpu().numpy().view(np.uint32)):
        raise RuntimeError("host-pointer path differs from the device path")

    extra = None
    peak = None
    if rank == 0:
        peak = fp32_peak()
    if rank == 0 and world == 1 and not args.no_extras:
        extra = run_extras(torch, lpaici, ks, args, flush, peak)
        # the batched plan on the benchmark image itself, beside the plain launch
        outb = torch.empty_like(x)
        plan = lpaici.Batch(ks, [x], [outb], [SIGMA], [GAMMA], use_graph=True)
        b_ms = time_launches(torch, plan.run, args.steps, 1, flush)
        same = torch.equal(outb.view(torch.int32), out.view(torch.int32))
        plan.close()
        extra["batched_one_image"] = {"size": size, "value": px / (np.mean(b_ms) * 1e-3) / 1e6,
                                      "plain": value, "unit": UNIT, "graph": True, "bit_equal_to_plain": bool(same)}
        # four images of the benchmark's size, sigma and gamma as one plan (one launch, a grid layer per
        # image) beside the same four as plain calls
        xs4 = [x] + [torch.from_numpy(bench_image(size, SEED + k, SIGMA)[1]).cuda() for k in (1, 2, 3)]
        outs4 = [torch.empty_like(v) for v in xs4]
        plain4 = [torch.empty_like(v) for v in xs4]
        plan4 = lpaici.Batch(ks, xs4, outs4, [SIGMA] * 4, [GAMMA] * 4, use_graph=True)
        b4_ms = time_launches(torch, plan4.run, args.steps, 1, flush)

        def plain_four():
            for v, o in zip(xs4, plain4):
                lpaici.forward(ks, v, SIGMA, GAMMA, out=o)

        p4_ms = time_launches(torch, plain_four, args.steps, 1, flush)
        same4 = all(torch.equal(a.view(torch.int32), b.view(torch.int32)) for a, b in zip(outs4, plain4))
        plan4.close()
        extra["batched_four_images"] = {"size": size, "images": 4, "value": 4 * px / (np.mean(b4_ms) * 1e-3) / 1e6,
                                        "plain_same_images": 4 * px / (np.mean(p4_ms) * 1e-3) / 1e6, "unit": UNIT,
                                        "graph": True, "bit_equal_to_plain": bool(same4),
                                        "how": "one launch of the single-image kernel with a grid layer per image"}
        del xs4, outs4, plain4
        # work rate (algorithmic taps per second) of the 64-image batch against the plain 4096^2 launch:
        # its images carry other sigmas, gammas and sizes, hence other taps per pixel
        extra["batched"]["work_rate_over_plain"] = extra["batched"]["taps_per_s"] / (taps / (ms_step * 1e-3))
        extra["ffma"] = run_ffma(torch, lpaici, ks, x, out, clean, taps, peak, args, flush)
        ref_gpu = reference_gpu_v4_1(clean, noisy_h, out.cpu().numpy(), min(args.steps, 3))
        if "value" in ref_gpu:
            ref_gpu["ours_e2e_over_reference"] = (px / e2e_step / 1e6) / ref_gpu["value"]
            ref_gpu["ours_device_over_reference"] = value / ref_gpu["value"]
        extra["reference_gpu_v4_1"] = ref_gpu

    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = host_threads()
        v, s, kept = cpu_reference_sample(noisy_h, 256, threads, SIGMA, GAMMA, keep=True)
        parity = crop_parity(out.cpu().numpy(), kept, ks.radius)
        v0, s0, _ = cpu_reference_sample(noisy_h, 128, threads, SIGMA, GAMMA, seed=1, engine="v0_0")
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "reference",
               "sample": f"{threads} crops of 256x256 px of the benchmark image, one per host thread, each "
                         f"denoised whole by the reference's anisotropic_lpa_ici_cpu_fused ({s:.1f} s)",
               "v0_0": {"value": v0, "unit": UNIT, "cores": threads,
                        "sample": f"{threads} crops of 128x128 px, the reference's naive engine "
                                  f"(src/v0_0_lpa_ici_2D_naive.cpp) ({s0:.1f} s)"}}

    if rank != 0:
        if dist:
            torch.distributed.barrier()
        return
    kernel_s = ms_step * 1e-3
    exact_ops = max(peak["muladd_ops_per_s"], peak["prodadd2_ops_per_s"])  # the exact forms only
    ffma_flops = peak["ffma_ops_per_s"]  # the FP32 FMA pipe: 2 FLOP per FFMA
    achieved = 2.0 * taps / kernel_s  # one multiply + one add per tap
    tw, th, thr, ppt = lpaici.tile_configs()[best]
    traffic = FORWARD_DRAM_BYTES if (size == SIZE and best in FORWARD_DRAM_CONFIGS) else None
    traffic_note = ("bytes per launch, dram__bytes_read.sum + dram__bytes_write.sum: a constant from the ncu capture "
                    "in profiles/forward_4096_sym.md (67.8 MB read + 27.2 MB written; algorithmic 134.2 MB: 4 B in "
                    "+ 4 B out per pixel), not measured by this run")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"plain LPA-ICI forward, one {size}x{size} synthetic image per GPU, sym 16x7 kernels, "
                               "sigma 20/255, gamma 2",
                   "image": "polygons + linear ramp + 4-16 px stripes, RGBE-quantised, seed 20250910 (+rank)",
                   "l2": "flushed between timed steps (256 MB write)",
                   "tile": {"config": best, "tile_w": tw, "tile_h": th, "threads": thr, "pixels_per_thread": ppt},
                   "parallelism": f"dp{world} (independent images, no collective)"},
        "roofline": {"bound": "fp32", "achieved": achieved / 1e12, "peak": ffma_flops / 1e12, "unit": "TFLOP/s",
                     "frac": achieved / ffma_flops,
                     "frac_exact_form": achieved / exact_ops, "peak_exact_form": exact_ops / 1e12,
                     "traffic": traffic,
                     "traffic_note": (traffic_note if traffic is not None else
                                      f"null: the ncu figure is for tile configurations {FORWARD_DRAM_CONFIGS} at "
                                      f"{SIZE}^2, this run used configuration {best} at {size}^2"),
                     "note": "FLOP = 2 per algorithmic tap (one multiply and one add); peak = the FP32 FMA pipe "
                             "(scalar FFMA chains, measured live on this GPU, 2 FLOP per FFMA).  The kernel keeps "
                             "every product and sum separately rounded (bit-exact with the reference), so it cannot "
                             "use FFMA: frac_exact_form divides by the exact forms' measured peak (the faster of "
                             "scalar FMUL+FADD and packed fma(w,x,-0)+add), which is half the FFMA peak",
                     "algorithmic_taps_per_px": taps / px,
                     "fp32_probe_tops": {k: v / 1e12 for k, v in peak.items()}},
        "cpu_baseline": cpu,
        "e2e": {"value": world * px / e2e_step / 1e6, "unit": UNIT, "h2d_bytes_per_step": px * 4,
                "d2h_bytes_per_step": px * 4},
        "gpu_launches": args.steps,
        "clocks": clk,
        "parity": parity,
        "extra": extra,
        "autotune_ms": [float(v) for v in tune_ms],
    }
    print(json.dumps(line), flush=True)
    if dist:
        torch.distributed.barrier()
    shutil.rmtree(tmp, ignore_errors=True)


def gather_taps_per_px(ks) -> int:
    """Multiply-adds per output pixel of the adjoint's gather: the taps of the runs of its telescoped
    kernels D_0 = h_0, D_s = h_s - h_{s-1} (each difference formed in double over the union of the two
    kernels' boxes and rounded to float, as the library builds them; a run spans a row from its first to
    its last nonzero)."""
    w, off, rows, cols = ks.dense()
    taps = 0
    for d in range(ks.D):
        prev = None
        for s in range(ks.S):
            k = d * ks.S + s
            h = w[off[k]:off[k] + rows[k] * cols[k]].reshape(rows[k], cols[k]).astype(np.float64)
            if prev is not None:
                hy, hx = max(h.shape[0], prev.shape[0]) // 2, max(h.shape[1], prev.shape[1]) // 2
                box = np.zeros((2 * hy + 1, 2 * hx + 1))
                box[hy - h.shape[0] // 2:hy - h.shape[0] // 2 + h.shape[0], hx - h.shape[1] // 2:hx - h.shape[1] // 2 + h.shape[1]] += h
                box[hy - prev.shape[0] // 2:hy - prev.shape[0] // 2 + prev.shape[0],
                    hx - prev.shape[1] // 2:hx - prev.shape[1] // 2 + prev.shape[1]] -= prev
            else:
                box = h
            for row in box.astype(np.float32):
                nz = np.nonzero(row)[0]
                if len(nz):
                    taps += int(nz[-1] - nz[0] + 1)
            prev = h
    return taps


def run_extras(torch, lpaici, ks, args, flush, peak) -> dict:
    import concurrent.futures as cf

    from lpaici.synth import mixed_batch

    spec = mixed_batch(64, SEED)
    n = len(spec)
    sig = [s[2] for s in spec]
    gam = [s[3] for s in spec]

    def make(i):
        w, h, s, _, img_seed, noise_seed = spec[i]
        return lpaici.add_noise(lpaici.synth_image(w, h, img_seed), s, noise_seed)

    with cf.ThreadPoolExecutor(max_workers=min(16, host_threads())) as ex:
        hosts = list(ex.map(make, range(n)))
    xs = [torch.from_numpy(h).cuda() for h in hosts]
    outs = [torch.empty_like(x) for x in xs]
    total_px = float(sum(h.size for h in hosts))
    batch = lpaici.Batch(ks, xs, outs, [float(s) for s in sig], [float(g) for g in gam], use_graph=True)
    steps = max(2, min(args.steps, 5))
    b_ms = time_launches(torch, batch.run, steps, 1, flush)
    singles = [torch.empty_like(x) for x in xs]

    def plain():
        for x, o, s, g in zip(xs, singles, sig, gam):
            lpaici.forward(ks, x, float(s), float(g), out=o)

    p_ms = time_launches(torch, plain, steps, 1, flush)
    same = all(torch.equal(a.view(torch.int32), b.view(torch.int32)) for a, b in zip(outs, singles))
    batch.close()
    # the batch's algorithmic taps (its sigmas and gammas differ from the benchmark image's), so that its
    # work rate can be set beside the plain launch's
    batch_taps = 0.0
    for x, s, g in zip(xs, sig, gam):
        _, sm = lpaici.forward(ks, x, float(s), float(g), scale_map=True)
        batch_taps += algorithmic_taps(torch, ks, sm)
        del sm
    del xs, outs, singles

    # adjoint: 8 x 1024^2, sigma 20/255, gamma 2, g ~ N(0, 1)
    m = 8
    xa = [torch.from_numpy(lpaici.add_noise(lpaici.synth_image(1024, 1024, SEED + 100 + i), SIGMA, SEED + i)).cuda()
          for i in range(m)]
    ga = [torch.randn(1024, 1024, generator=torch.Generator().manual_seed(i)).cuda() for i in range(m)]
    gi = [torch.empty_like(x) for x in xa]
    fo = [torch.empty_like(x) for x in xa]

    def adj():
        for x, g, o in zip(xa, ga, gi):
            lpaici.backward(ks, x, g, SIGMA, GAMMA, grad_in=o)

    def fwd8():
        for x, o in zip(xa, fo):
            lpaici.forward(ks, x, SIGMA, GAMMA, out=o)

    a_ms = time_launches(torch, adj, steps, 1, flush)
    f_ms = time_launches(torch, fwd8, steps, 1, flush)
    ident8 = max(adjoint_identity(torch, x, g, o, gr) for x, g, o, gr in zip(xa, ga, fo, gi))
    # the same 8 images as one batched adjoint plan and one batched forward plan (CUDA graphs)
    gb = [torch.empty_like(x) for x in xa]
    fb = [torch.empty_like(x) for x in xa]
    bplan = lpaici.BackwardBatch(ks, xa, ga, gb, [SIGMA] * m, [GAMMA] * m, use_graph=True)
    fplan = lpaici.Batch(ks, xa, fb, [SIGMA] * m, [GAMMA] * m, use_graph=True)
    ab_ms = time_launches(torch, bplan.run, steps, 1, flush)
    fb_ms = time_launches(torch, fplan.run, steps, 1, flush)
    batched_same = all(torch.equal(a.view(torch.int32), b.view(torch.int32)) for a, b in zip(gb, gi))
    bplan.close()
    fplan.close()
    # kept state: the forward keeps s* and 1/den (D+4 B/px), the adjoint is the gather alone
    states = [lpaici.forward_state(ks, x, SIGMA, GAMMA, out=o)[1] for x, o in zip(xa, fo)]
    gk = [torch.empty_like(x) for x in xa]

    def fwd_keep():
        for x, o, st in zip(xa, fo, states):
            lpaici.forward_state(ks, x, SIGMA, GAMMA, out=o, state=st)

    def adj_keep():
        for st, g, o in zip(states, ga, gk):
            lpaici.backward_state(ks, st, g, SIGMA, grad_in=o)

    gtaps = gather_taps_per_px(ks)
    fk_ms = time_launches(torch, fwd_keep, steps, 1, flush)
    ak_ms = time_launches(torch, adj_keep, steps, 1, flush)
    kept_same = all(torch.equal(a.view(torch.int32), b.view(torch.int32)) for a, b in zip(gk, gi))
    del states, gk
    del xa, ga, gi, fo, gb, fb
    large = run_large(torch, lpaici, steps, flush)
    return {
        "batched": {"images": n, "mpix": total_px / 1e6, "value": total_px / (np.mean(b_ms) * 1e-3) / 1e6,
                    "plain_same_images": total_px / (np.mean(p_ms) * 1e-3) / 1e6, "unit": UNIT,
                    "graph": True, "bit_equal_to_plain": bool(same),
                    "algorithmic_taps_per_px": batch_taps / total_px,
                    "taps_per_s": batch_taps / (np.mean(b_ms) * 1e-3)},
        "adjoint": {"images": m, "size": 1024, "unit": UNIT,
                    "value": m * 1024 * 1024 / (np.mean(ab_ms) * 1e-3) / 1e6,
                    "forward_same_images": m * 1024 * 1024 / (np.mean(fb_ms) * 1e-3) / 1e6,
                    "adjoint_over_forward_time": float(np.mean(ab_ms) / np.mean(fb_ms)),
                    "how": "batched plans (selection, u = g/den and gather: one launch each; one forward "
                           "launch), CUDA graphs",
                    "bit_equal_to_single": bool(batched_same),
                    "single_image_calls": {"value": m * 1024 * 1024 / (np.mean(a_ms) * 1e-3) / 1e6,
                                           "forward_same_images": m * 1024 * 1024 / (np.mean(f_ms) * 1e-3) / 1e6,
                                           "adjoint_over_forward_time": float(np.mean(a_ms) / np.mean(f_ms))},
                    "identity_rel_err": ident8,
                    "gather_roofline": {
                        "taps_per_px": gtaps, "achieved_tflops": 2.0 * gtaps * m * 1024 * 1024 / (np.mean(ak_ms) * 1e-3) / 1e12,
                        "frac_of_ffma": 2.0 * gtaps * m * 1024 * 1024 / (np.mean(ak_ms) * 1e-3) / peak["ffma_ops_per_s"],
                        "how": "the gather alone (from kept state, one call per image), 2 FLOP per tap of its "
                               "telescoped kernels, against the measured FFMA rate; a 1024^2 launch is 128 tiles "
                               "of 128x64 outputs (0.86 of a wave on 148 SMs)"},
                    "kept_state": {"forward_state_over_forward": float(np.mean(fk_ms) / np.mean(f_ms)),
                                   "backward_state_over_forward": float(np.mean(ak_ms) / np.mean(f_ms)),
                                   "bit_equal_to_recomputed": bool(kept_same),
                                   "how": "single-image calls; the forward keeps D+4 bytes per pixel"}},
        "large": large,
    }


def run_ffma(torch, lpaici, ks, x, exact_out, clean, taps, peak, args, flush) -> dict:
    """The contracted mode (lpaici_forward_ffma: one fused multiply-add per tap) on the benchmark image:
    its speed, its FP32 FMA fraction (same algorithmic taps), and its agreement with the exact forward
    against the accuracy criteria of the goal (scale maps >= 99.99 %, max abs error <= 1e-4, PSNR within
    0.01 dB)."""
    H, W = x.shape
    fo = torch.empty_like(x)
    ms = time_launches(torch, lambda: lpaici.forward(ks, x, SIGMA, GAMMA, out=fo, ffma=True), args.steps, 1, flush)
    _, emap = lpaici.forward(ks, x, SIGMA, GAMMA, out=exact_out, scale_map=True)
    _, fmap = lpaici.forward(ks, x, SIGMA, GAMMA, out=fo, scale_map=True, ffma=True)
    torch.cuda.synchronize()
    agree = (emap == fmap)
    px_agree = agree.all(dim=0)
    diff = (fo.double() - exact_out.double()).abs()
    a, b = fo.cpu().numpy(), exact_out.cpu().numpy()
    t = float(np.mean(ms)) * 1e-3
    return {"value": W * H / t / 1e6, "unit": UNIT, "ms": t * 1e3,
            "roofline_frac": 2.0 * taps / t / peak["ffma_ops_per_s"],
            "vs_exact": {"map_agreement": float(agree.double().mean()),
                         "pixels_with_a_flipped_scale": int((~px_agree).sum()),
                         "max_abs_err": float(diff.max()),
                         "max_abs_err_agreeing_pixels": float(diff[px_agree].max()),
                         "pixels_over_1e-4": int((diff > 1e-4).sum()),
                         "psnr_delta_db": float(lpaici.psnr(clean, a) - lpaici.psnr(clean, b))}}


def adjoint_identity(torch, x, g, out, grad) -> float:
    """With the selection frozen the forward is linear in its input, out = J x, so
    sum(g * out) = sum(g * J x) = sum(J^T g * x) = sum(grad * x): the relative gap of the two sums
    (FP64 reductions of the FP32 results) checks the adjoint at any size."""
    a = float((g.double() * out.double()).sum())
    b = float((grad.double() * x.double()).sum())
    scale = float((g.double().abs() * out.double().abs()).sum())
    return abs(a - b) / scale


def run_large(torch, lpaici, steps, flush) -> dict:
    """Forward and adjoint (scale maps recomputed in the backward) on one 8192^2 image, gaussian
    m=(2,0) 16x7 kernels, sigma 25/255, gamma 1.5."""
    tmp = tempfile.mkdtemp()
    try:
        kg = lpaici.KernelSet.load(kernel_path(GAUSS_M2, tmp))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    n = 8192
    sigma = float(np.float32(25.0) / np.float32(255.0))
    gamma = 1.5
    _, noisy = bench_image(n, SEED, sigma)
    x = torch.from_numpy(noisy).cuda()
    g = torch.randn(n, n, generator=torch.Generator().manual_seed(5)).cuda()
    out = torch.empty_like(x)
    grad = torch.empty_like(x)
    f_ms = time_launches(torch, lambda: lpaici.forward(kg, x, sigma, gamma, out=out), steps, 1, flush)
    a_ms = time_launches(torch, lambda: lpaici.backward(kg, x, g, sigma, gamma, grad_in=grad), steps, 1, flush)
    ident = adjoint_identity(torch, x, g, out, grad)
    return {"size": n, "kernels": "gaussian m=(2,0) 16x7", "sigma": sigma, "gamma": gamma,
            "forward": n * n / (np.mean(f_ms) * 1e-3) / 1e6, "adjoint": n * n / (np.mean(a_ms) * 1e-3) / 1e6,
            "unit": UNIT, "forward_ms": float(np.mean(f_ms)), "adjoint_ms": float(np.mean(a_ms)),
            "adjoint_over_forward_time": float(np.mean(a_ms) / np.mean(f_ms)), "identity_rel_err": ident}


def run_profile(args) -> None:
    """One operation on one synthetic size x size image, warmup + steps times, for profiler captures
    (no bench line)."""
    import torch

    import lpaici

    tmp = tempfile.mkdtemp()
    gauss = args.kernels == "gauss_m2"
    ks = lpaici.KernelSet.load(kernel_path(GAUSS_M2 if gauss else SYM, tmp))
    shutil.rmtree(tmp, ignore_errors=True)
    sigma = float(np.float32(25.0) / np.float32(255.0)) if gauss else SIGMA
    gamma = 1.5 if gauss else GAMMA
    if args.tile_config >= 0:
        ks.set_tile_config(args.tile_config)
    if args.profile == "batched_one":  # a batched plan over the one --size image, one launch per step
        _, noisy_h = bench_image(args.size, SEED, sigma)
        xs = [torch.from_numpy(noisy_h).cuda()]
        outs = [torch.empty_like(xs[0])]
        plan = lpaici.Batch(ks, xs, outs, [sigma], [gamma], use_graph=True)
        op = plan.run
    elif args.profile == "batched":  # the 64-image plan of the batched benchmark, one launch per step
        from lpaici.synth import mixed_batch

        spec = mixed_batch(64, SEED)
        xs = [torch.from_numpy(lpaici.add_noise(lpaici.synth_image(w, h, i_s), s, n_s)).cuda()
              for w, h, s, _, i_s, n_s in spec]
        outs = [torch.empty_like(t) for t in xs]
        plan = lpaici.Batch(ks, xs, outs, [v[2] for v in spec], [v[3] for v in spec], use_graph=True)
        op = plan.run
    else:
        _, noisy_h = bench_image(args.size, SEED, sigma)
        x = torch.from_numpy(noisy_h).cuda()
        out = torch.empty_like(x)
        g = torch.randn(args.size, args.size, generator=torch.Generator().manual_seed(0)).cuda()
        ops = {"forward": lambda: lpaici.forward(ks, x, sigma, gamma, out=out),
               "ffma": lambda: lpaici.forward(ks, x, sigma, gamma, out=out, ffma=True),
               "adjoint": lambda: lpaici.backward(ks, x, g, sigma, gamma, grad_in=out)}
        op = ops[args.profile]
    for _ in range(args.warmup):
        op()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        op()
    torch.cuda.synchronize()
    print(json.dumps({"profile": args.profile, "size": args.size, "steps": args.steps,
                      "ms_per_step_wall": (time.perf_counter() - t0) * 1e3 / max(1, args.steps)}))


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--ref-crop", type=int, default=256, help="crop side per thread for --impl reference")
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--size", type=int, default=SIZE, help="image side (profiling runs use a smaller case)")
    ap.add_argument("--tile-config", type=int, default=-1, help="fixed tile configuration instead of autotuning")
    ap.add_argument("--profile", choices=["forward", "ffma", "adjoint", "batched", "batched_one"], default=None,
                    help="run only this operation on one --size image, or the 64-image batched plan (for "
                         "profiler captures; no bench line)")
    ap.add_argument("--kernels", choices=["sym", "gauss_m2"], default="sym",
                    help="kernel set of a --profile run: the 16x7 symmetric set (sigma 20/255, gamma 2) or the "
                         "gaussian m=(2,0) set (sigma 25/255, gamma 1.5)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.profile:
        run_profile(args)
        return
    if world > 1:
        import torch

        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch

            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
