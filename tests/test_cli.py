"""The drop-in command line (lpa-ici-cuda_b200/bin/lpaici) and its image I/O (lib/liblpaici_io.so).

CPU: option parsing and messages of src/Config.hpp; PNG (every color type, bit depth, row filter,
Adam7), PGM and Radiance HDR decoding against stb_image (the reference's loader, in-process), HDR
writing against stbi_write_hdr.  GPU: a full run on barbara prints the reference's PSNR lines and writes
the reference's files."""
import ctypes as C
import hashlib
import json
import os
import struct
import subprocess
import zlib

import numpy as np
import pytest

import lpaici
import oracle_bind as ob
from conftest import GOLDEN, PKG, SYM, kernel_file
from lpaici.synth import rgbe_quantize

CLI = os.path.join(PKG, "bin", "lpaici")
IO = C.CDLL(os.path.join(PKG, "lib", "liblpaici_io.so"))
IO.lpaici_io_load_gray.argtypes = [C.c_char_p, C.POINTER(C.POINTER(C.c_float)), C.POINTER(C.c_int),
                                   C.POINTER(C.c_int)]
IO.lpaici_io_free.argtypes = [C.c_void_p]
IO.lpaici_io_write_hdr.argtypes = [C.c_char_p, np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS"), C.c_int,
                                   C.c_int]
IO.lpaici_io_load_rgb.argtypes = [C.c_char_p, C.POINTER(C.POINTER(C.c_float)), C.POINTER(C.c_int),
                                  C.POINTER(C.c_int)]
IO.lpaici_io_write_hdr_rgb.argtypes = [C.c_char_p, np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS"), C.c_int,
                                       C.c_int]
needs_ref = pytest.mark.skipif(not ob.ref_available("v1_0"), reason="reference not built in-process")


def io_load(path):
    p, w, h = C.POINTER(C.c_float)(), C.c_int(), C.c_int()
    if IO.lpaici_io_load_gray(path.encode(), C.byref(p), C.byref(w), C.byref(h)) != 0:
        raise ValueError(path)
    a = np.ctypeslib.as_array(p, shape=(h.value * w.value,)).copy().reshape(h.value, w.value)
    IO.lpaici_io_free(C.cast(p, C.c_void_p))
    return a


def io_load_rgb(path):
    p, w, h = C.POINTER(C.c_float)(), C.c_int(), C.c_int()
    if IO.lpaici_io_load_rgb(path.encode(), C.byref(p), C.byref(w), C.byref(h)) != 0:
        raise ValueError(path)
    a = np.ctypeslib.as_array(p, shape=(h.value * w.value * 3,)).copy().reshape(h.value, w.value, 3)
    IO.lpaici_io_free(C.cast(p, C.c_void_p))
    return a


def run_cli(*args, cwd=None):
    return subprocess.run([CLI, *args], capture_output=True, text=True, cwd=cwd, timeout=600)


# ---- options (src/Config.hpp:39-92) ------------------------------------------------------------

def test_help():
    r = run_cli("-h")
    assert r.returncode == 0
    assert r.stdout.startswith(f"Usage: {CLI} [options]\n")
    assert "  -s, --sigma <value>    noise standard deviation on the 0-255 scale (default 20)\n" in r.stdout


@pytest.mark.parametrize("args,msg", [
    (["-s", "-3"], "Error: -s needs a positive number, got '-3'"),
    (["--gamma", "0"], "Error: --gamma needs a positive number, got '0'"),
    (["-g", "2x"], "Error: -g needs a positive number, got '2x'"),
    (["--seed", "12a"], "Error: --seed needs an unsigned integer, got '12a'"),
    (["-i"], "Error: unknown option or missing value for '-i'"),
    (["--bogus", "1"], "Error: unknown option '--bogus'"),
])
def test_option_errors(args, msg):
    r = run_cli(*args)
    assert r.returncode == 1
    assert r.stderr.startswith(msg + "\n\n")
    assert "Usage:" in r.stdout


def test_config_echo_and_default_output(tmp_path):
    img = tmp_path / "pics" / "tiny.pgm"
    img.parent.mkdir()
    img.write_bytes(b"P5\n4 3\n255\n" + bytes(range(12)))
    r = run_cli("-i", str(img), "-k", str(tmp_path / "missing.txt"), "-s", "25", "-g", "1.5", "--seed", "7")
    lines = r.stdout.splitlines()
    assert lines[:4] == [f"Image: {img}", f"Kernels: {tmp_path / 'missing.txt'}",
                         f"Output: {img.parent}/tiny_lpaici_b200_gpu.hdr", "Sigma: 25/255, gamma: 1.5, seed: 7"]
    assert "Loaded image with a width of 4 px, a height of 3 px and (imported) 1 channels" in lines
    assert f"Saving gray image as {img.parent}/gray_image.hdr" in lines
    assert r.returncode == 1 and "Failed to open" in r.stderr  # the kernel file is missing


def test_image_load_error(tmp_path):
    r = run_cli("-i", str(tmp_path / "none.png"))
    assert r.returncode == 1
    assert f"Error in loading the image {tmp_path / 'none.png'}" in r.stderr


# ---- image I/O against stb ------------------------------------------------------------------------

def _paeth(a, b, c):
    p = a + b - c
    pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
    return a if pa <= pb and pa <= pc else (b if pb <= pc else c)


def _filter_rows(rows, bpp):
    out = bytearray()
    prev = bytes(len(rows[0])) if rows else b""
    for y, row in enumerate(rows):
        ft = y % 5
        out.append(ft)
        for i, x in enumerate(row):
            a = row[i - bpp] if i >= bpp else 0
            b = prev[i]
            c = prev[i - bpp] if i >= bpp else 0
            pred = [0, a, b, (a + b) >> 1, _paeth(a, b, c)][ft]
            out.append((x - pred) & 0xFF)
        prev = row
    return bytes(out)


def _pack(samples, depth):
    """One row of samples (ints) at bit depth `depth`."""
    if depth == 8:
        return bytes(int(v) for v in samples)
    if depth == 16:
        return b"".join(struct.pack(">H", int(v)) for v in samples)
    per = 8 // depth
    out = bytearray((len(samples) + per - 1) // per)
    for i, v in enumerate(samples):
        out[i // per] |= int(v) << (8 - depth * (i % per + 1))
    return bytes(out)


def make_png(path, arr, ctype, depth, palette=None, interlace=False):
    """arr: H x W x channels ints (palette indices for ctype 3)."""
    H, W = arr.shape[:2]
    ch = arr.shape[2]
    bpp = max(1, ch * depth // 8)

    def encode(sub):
        rows = [_pack(sub[y].reshape(-1), depth) for y in range(sub.shape[0])]
        return _filter_rows(rows, bpp) if rows and sub.shape[1] else b""

    if not interlace:
        raw = encode(arr)
    else:
        raw = b""
        for xo, yo, xs, ys in ((0, 0, 8, 8), (4, 0, 8, 8), (0, 4, 4, 8), (2, 0, 4, 4), (0, 2, 2, 4), (1, 0, 2, 2),
                               (0, 1, 1, 2)):
            sub = arr[yo::ys, xo::xs]
            if sub.shape[0] and sub.shape[1]:
                raw += encode(sub)

    def chunk(t, d):
        return struct.pack(">I", len(d)) + t + d + struct.pack(">I", zlib.crc32(t + d) & 0xFFFFFFFF)

    data = b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", W, H, depth, ctype, 0, 0, int(interlace)))
    if palette is not None:
        data += chunk(b"PLTE", bytes(palette.reshape(-1)))
    data += chunk(b"IDAT", zlib.compress(raw)) + chunk(b"IEND", b"")
    open(path, "wb").write(data)


PNG_CASES = [(0, 1), (0, 2), (0, 4), (0, 8), (0, 16), (2, 8), (2, 16), (3, 1), (3, 4), (3, 8), (4, 8), (4, 16),
             (6, 8), (6, 16)]


@needs_ref
@pytest.mark.parametrize("interlace", [False, True])
@pytest.mark.parametrize("ctype,depth", PNG_CASES)
def test_png_decoding_matches_stb(tmp_path, ctype, depth, interlace):
    rng = np.random.default_rng(ctype * 100 + depth)
    H, W = 13, 21
    ch = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}[ctype]
    top = (1 << depth) - 1
    pal = None
    if ctype == 3:
        n = min(256, 1 << depth)
        pal = rng.integers(0, 256, (n, 3)).astype(np.uint8)
        arr = rng.integers(0, n, (H, W, 1))
    else:
        arr = rng.integers(0, top + 1, (H, W, ch))
    p = str(tmp_path / "x.png")
    make_png(p, arr, ctype, depth, pal, interlace)
    ref = ob.ref_stbi_loadf(p)
    got = io_load(p)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


@needs_ref
@pytest.mark.parametrize("ctype,depth", PNG_CASES)
def test_png_rgb_decoding_matches_stb(tmp_path, ctype, depth):
    """The colour mode's loader against stbi_loadf(path, .., 3) on every PNG type."""
    rng = np.random.default_rng(ctype * 101 + depth)
    H, W = 11, 19
    ch = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}[ctype]
    pal = None
    if ctype == 3:
        n = min(256, 1 << depth)
        pal = rng.integers(0, 256, (n, 3)).astype(np.uint8)
        arr = rng.integers(0, n, (H, W, 1))
    else:
        arr = rng.integers(0, (1 << depth), (H, W, ch))
    p = str(tmp_path / "c.png")
    make_png(p, arr, ctype, depth, pal, False)
    ref = ob.ref_stbi_loadf_rgb(p)
    got = io_load_rgb(p)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


@needs_ref
@pytest.mark.parametrize("W,H", [(64, 40), (5, 7), (300, 2)])
def test_hdr_rgb_roundtrip_with_stb(tmp_path, W, H):
    """RGB .hdr writing and reading: same pixel bytes as stbi_write_hdr(.., 3), both loaders agree."""
    rng = np.random.default_rng(W + H)
    img = rng.uniform(0.0, 2.0, (H, W, 3)).astype(np.float32)
    img[0, 0] = 0.0
    img[-1, -1, 1] = 1e-35
    ours, theirs = str(tmp_path / "ours.hdr"), str(tmp_path / "stb.hdr")
    assert IO.lpaici_io_write_hdr_rgb(ours.encode(), np.ascontiguousarray(img), W, H) == 0
    ob.ref_stbi_write_hdr_rgb(theirs, img)
    a, b = open(ours, "rb").read(), open(theirs, "rb").read()
    assert a[a.index(b"-Y"):] == b[b.index(b"-Y"):]
    assert np.array_equal(io_load_rgb(theirs).view(np.uint32), ob.ref_stbi_loadf_rgb(theirs).view(np.uint32))
    # the gray loader of an RGB file averages the channels as stbi_loadf(.., 1) does
    assert np.array_equal(io_load(theirs).view(np.uint32), ob.ref_stbi_loadf(theirs).view(np.uint32))


def test_barbara_png_to_float():
    """data/barbara.png decoded and converted like stb (hash of the reference's float image)."""
    meta = json.load(open(os.path.join(GOLDEN, "barbara.json")))
    u8 = np.load(os.path.join(GOLDEN, "barbara_gray_u8.npy"))
    import tempfile

    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "b.png")
        make_png(p, u8[:, :, None], 0, 8)
        img = io_load(p)
        assert hashlib.sha256(img.tobytes()).hexdigest() == meta["clean_sha256"]
        q = os.path.join(d, "b.pgm")
        open(q, "wb").write(b"P5\n512 512\n255\n" + u8.tobytes())
        assert hashlib.sha256(io_load(q).tobytes()).hexdigest() == meta["clean_sha256"]


@needs_ref
@pytest.mark.parametrize("W,H", [(64, 40), (5, 7), (1, 1), (300, 2), (33000, 1)])
def test_hdr_roundtrip_with_stb(tmp_path, W, H):
    img = (lpaici.synth_image(W, H, 3, rgbe=False) * np.float32(1.7)).astype(np.float32)
    img[0, 0] = 0.0
    ours, theirs = str(tmp_path / "ours.hdr"), str(tmp_path / "stb.hdr")
    assert IO.lpaici_io_write_hdr(ours.encode(), img, W, H) == 0
    ob.ref_stbi_write_hdr(theirs, img)
    want = rgbe_quantize(img)
    assert np.array_equal(ob.ref_stbi_loadf(ours).view(np.uint32), want.view(np.uint32))
    assert np.array_equal(io_load(theirs).view(np.uint32), want.view(np.uint32))
    a, b = open(ours, "rb").read(), open(theirs, "rb").read()
    assert a[a.index(b"-Y"):] == b[b.index(b"-Y"):]  # same pixel bytes as stbi_write_hdr


# ---- full run -----------------------------------------------------------------------------------

@pytest.mark.gpu
def test_cli_barbara_end_to_end(tmp_path):
    """The default run of the reference on data/barbara.png: PSNR lines 22.1056 / 25.0736 and the
    three .hdr files, the denoised one holding the reference's denoised image (RGBE-encoded)."""
    u8 = np.load(os.path.join(GOLDEN, "barbara_gray_u8.npy"))
    img = tmp_path / "data" / "barbara.png"
    img.parent.mkdir()
    make_png(str(img), u8[:, :, None], 0, 8)
    out = tmp_path / "out" / "den.hdr"
    out.parent.mkdir()
    r = run_cli("-i", str(img), "-k", kernel_file(SYM), "-o", str(out))
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    assert "Calculated PSNR of host_img_gray_noisy: 22.1056" in lines
    assert "Calculated PSNR of img_denoised: 25.0736" in lines
    assert any(ln.startswith("Time taken for directional loops + aggregation: ") for ln in lines)
    assert any(ln.startswith("Time taken for lpa function execution: ") for ln in lines)
    for f in ("gray_image.hdr", "gray_image_noisy.hdr", "den.hdr"):
        assert (out.parent / f).exists()
    meta = json.load(open(os.path.join(GOLDEN, "barbara.json")))
    clean = io_load(str(img))
    noisy = lpaici.add_noise(clean, np.float32(20.0) / np.float32(255.0), 20250910)
    ks = lpaici.KernelSet.load(kernel_file(SYM))
    den = lpaici.denoise_host(ks, noisy, float(np.float32(20.0) / np.float32(255.0)), 2.0)
    assert hashlib.sha256(den.tobytes()).hexdigest() == meta["denoised_sha256"]
    assert np.array_equal(io_load(str(out)).view(np.uint32), rgbe_quantize(den).view(np.uint32))


@pytest.mark.gpu
def test_cli_color_end_to_end(tmp_path):
    """--color: R, G, B loaded as stb does, noise over all channels, every channel denoised on its own;
    the RGB output file holds exactly the library's interleaved-channel result."""
    import torch

    rng = np.random.default_rng(5)
    H, W = 72, 96
    rgb = np.stack([np.round(lpaici.synth_image(W, H, 60 + c, rgbe=False) * 255) for c in range(3)], axis=2)
    rgb = np.clip(rgb + rng.integers(-3, 4, rgb.shape), 0, 255).astype(np.int64)
    img = tmp_path / "c.png"
    make_png(str(img), rgb, 2, 8)
    out = tmp_path / "den.hdr"
    r = run_cli("-i", str(img), "-k", kernel_file(SYM), "-o", str(out), "-s", "25", "--color")
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    assert any("and (imported) 3 channels" in ln for ln in lines)
    for f in ("color_image.hdr", "color_image_noisy.hdr", "den.hdr"):
        assert (tmp_path / f).exists()
    sigma = float(np.float32(25.0) / np.float32(255.0))
    clean = io_load_rgb(str(img))
    noisy = lpaici.add_noise(clean.reshape(-1), sigma, 20250910).reshape(H, W, 3)
    ks = lpaici.KernelSet.load(kernel_file(SYM))
    den = lpaici.forward_channels(ks, torch.from_numpy(noisy).cuda(), sigma, 2.0).cpu().numpy()
    mine = tmp_path / "mine.hdr"
    assert IO.lpaici_io_write_hdr_rgb(str(mine).encode(), np.ascontiguousarray(den), W, H) == 0
    a, b = open(out, "rb").read(), open(mine, "rb").read()
    assert a[a.index(b"-Y"):] == b[b.index(b"-Y"):]
    want = f"Calculated PSNR of img_denoised: {lpaici.psnr(clean, den):.6g}"
    assert want in lines, (want, [ln for ln in lines if "PSNR" in ln])
