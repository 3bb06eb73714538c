"""The command line's BMP and TGA readers against stb_image, the reference's loader (stbi_loadf(path, .., 1)
and (.., 3), src/v4_1_lpa_ici_2D_sparse_shared.cu:375), called in-process from the reference build.

The files are written here by small writers of the two formats: BMP with 1/4/8-bit palettes, 16-bit
5-5-5 and 5-6-5 (bit fields), 24 and 32 bits, bottom-up and top-down, and a V5 header; TGA truecolor
(15/16/24/32 bits), gray (8 and 16 bits), color-mapped, raw and run-length, both row orders.  Every
float of the result must be bit-equal to stb's.
"""
import struct

import numpy as np
import pytest

import oracle_bind as ob
from test_cli import io_load, io_load_rgb, needs_ref

H, W = 13, 23


def write_bmp(path, rgb=None, bpp=24, idx=None, palette=None, top_down=False, masks=None, hsz=40):
    """rgb: H x W x 3 uint8 (bpp 24/32), or H x W uint16/uint32 raw pixels (bpp 16/32 with masks);
    idx + palette for bpp <= 8."""
    h, w = (idx.shape if idx is not None else rgb.shape[:2])
    stride = ((w * bpp + 31) // 32) * 4
    rows = []
    for y in range(h):
        if bpp <= 8:
            row = bytearray()
            acc, n = 0, 0
            for x in range(w):
                acc = (acc << bpp) | int(idx[y, x])
                n += bpp
                if n == 8:
                    row.append(acc)
                    acc, n = 0, 0
            if n:
                row.append(acc << (8 - n))
        elif bpp == 24:
            row = bytearray(rgb[y, :, ::-1].tobytes())
        elif bpp == 16:
            row = bytearray(rgb[y].astype("<u2").tobytes())
        else:
            row = bytearray(rgb[y].astype("<u4").tobytes()) if rgb.ndim == 2 else bytearray(
                np.concatenate([rgb[y, :, ::-1], np.full((w, 1), 255, np.uint8)], axis=1).tobytes())
        rows.append(bytes(row) + b"\0" * (stride - len(row)))
    data = b"".join(rows if top_down else rows[::-1])
    pal = b""
    if bpp <= 8:
        pal = b"".join(bytes([b, g, r, 0]) for r, g, b in palette)
    compress = 3 if masks is not None else 0
    header = struct.pack("<iiHHIIiiII", w, -h if top_down else h, 1, bpp, compress, len(data), 2835, 2835,
                         len(palette) if bpp <= 8 else 0, 0)
    extra = b""
    if hsz == 40 and masks is not None:
        extra = struct.pack("<III", *masks)
    elif hsz == 124:
        m = masks if masks is not None else (0, 0, 0)
        header += struct.pack("<IIII", m[0], m[1], m[2], 0) + b"\0" * (124 - 40 - 16)
    info = struct.pack("<I", hsz) + header
    off = 14 + len(info) + len(extra) + len(pal)
    open(path, "wb").write(b"BM" + struct.pack("<IHHI", off + len(data), 0, 0, off) + info + extra + pal + data)


def write_tga(path, pixels, kind, bpp, rle=False, top_left=False, palette=None, pal_bits=24):
    """pixels: H x W x 3 uint8 (truecolor 24/32), H x W uint16 (truecolor 15/16 raw 5-5-5), H x W uint8
    (gray 8, or indexes), H x W x 2 (gray + alpha)."""
    h, w = pixels.shape[:2]
    cmap_type = 1 if kind == 1 else 0
    typ = kind + (8 if rle else 0)
    pal_bytes = b""
    cmap_len = 0
    if kind == 1:
        cmap_len = len(palette)
        pal_bytes = b"".join(bytes([b, g, r]) for r, g, b in palette)
    header = struct.pack("<BBBHHBHHHHBB", 0, cmap_type, typ, 0, cmap_len, pal_bits if kind == 1 else 0, 0, 0, w, h,
                         bpp, 32 if top_left else 0)
    rows = range(h) if top_left else range(h - 1, -1, -1)

    def pix(y, x):
        p = pixels[y, x]
        if kind == 3:
            return bytes([int(p)]) if bpp == 8 else bytes([int(p[0]), int(p[1])])
        if kind == 1:
            return bytes([int(p)])
        if bpp in (15, 16):
            return struct.pack("<H", int(p))
        return bytes([p[2], p[1], p[0]]) + (b"\xff" if bpp == 32 else b"")

    seq = [pix(y, x) for y in rows for x in range(w)]
    body = b""
    if not rle:
        body = b"".join(seq)
    else:
        i = 0
        while i < len(seq):
            j = i
            while j + 1 < len(seq) and seq[j + 1] == seq[i] and j - i < 127:
                j += 1
            if j > i:
                body += bytes([128 | (j - i)]) + seq[i]
                i = j + 1
            else:
                k = i
                while k + 1 < len(seq) and seq[k + 1] != seq[k] and k - i < 127:
                    k += 1
                body += bytes([k - i]) + b"".join(seq[i:k + 1])
                i = k + 1
    open(path, "wb").write(header + pal_bytes + body)


def _same(path):
    assert np.array_equal(io_load(path).view(np.uint32), ob.ref_stbi_loadf(path).view(np.uint32))
    assert np.array_equal(io_load_rgb(path).view(np.uint32), ob.ref_stbi_loadf_rgb(path).view(np.uint32))


def _rgb(seed, runs=False):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, 256, (H, W, 3)).astype(np.uint8)
    if runs:  # long runs, so run-length packets are exercised
        a[:, : W // 2] = a[:, :1]
    return a


@needs_ref
@pytest.mark.parametrize("bpp", [1, 4, 8])
def test_bmp_palette(tmp_path, bpp):
    rng = np.random.default_rng(bpp)
    n = 1 << bpp
    pal = rng.integers(0, 256, (n, 3)).astype(np.uint8)
    p = str(tmp_path / "x.bmp")
    write_bmp(p, bpp=bpp, idx=rng.integers(0, n, (H, W)), palette=pal)
    _same(p)


@needs_ref
@pytest.mark.parametrize("bpp,top_down,hsz", [(24, False, 40), (24, True, 40), (32, False, 40), (24, False, 124),
                                              (32, True, 124)])
def test_bmp_truecolor(tmp_path, bpp, top_down, hsz):
    p = str(tmp_path / "x.bmp")
    write_bmp(p, _rgb(bpp + hsz), bpp=bpp, top_down=top_down, hsz=hsz)
    _same(p)


@needs_ref
@pytest.mark.parametrize("masks", [None, (0xF800, 0x07E0, 0x001F), (0x7C00, 0x03E0, 0x001F)])
def test_bmp_16bit(tmp_path, masks):
    raw = np.random.default_rng(16).integers(0, 1 << 16, (H, W)).astype(np.uint16)
    if masks is None or masks[0] == 0x7C00:
        raw &= 0x7FFF
    p = str(tmp_path / "x.bmp")
    write_bmp(p, raw, bpp=16, masks=masks)
    _same(p)


@needs_ref
def test_bmp_32bit_bitfields(tmp_path):
    raw = np.random.default_rng(32).integers(0, 1 << 31, (H, W)).astype(np.uint32)
    p = str(tmp_path / "x.bmp")
    write_bmp(p, raw, bpp=32, masks=(0x0000FF00, 0x7F000000, 0x003F0000))  # 8, 7 and 6 bits, any order
    _same(p)
    q = str(tmp_path / "y.bmp")
    write_bmp(q, raw, bpp=32, masks=(0x3FF00000, 0x000FFC00, 0x000003FF))  # 10-bit fields: refused by both
    with pytest.raises(ValueError):
        ob.ref_stbi_loadf(q)
    with pytest.raises(ValueError):
        io_load(q)


@needs_ref
@pytest.mark.parametrize("bpp", [24, 32])
@pytest.mark.parametrize("rle", [False, True])
@pytest.mark.parametrize("top_left", [False, True])
def test_tga_truecolor(tmp_path, bpp, rle, top_left):
    p = str(tmp_path / "x.tga")
    write_tga(p, _rgb(bpp + rle, runs=rle), 2, bpp, rle=rle, top_left=top_left)
    _same(p)


@needs_ref
@pytest.mark.parametrize("bpp", [15, 16])
def test_tga_rgb16(tmp_path, bpp):
    raw = (np.random.default_rng(bpp).integers(0, 1 << 15, (H, W))).astype(np.uint16)
    p = str(tmp_path / "x.tga")
    write_tga(p, raw, 2, bpp)
    _same(p)


@needs_ref
@pytest.mark.parametrize("rle", [False, True])
def test_tga_gray(tmp_path, rle):
    g = np.random.default_rng(8).integers(0, 256, (H, W)).astype(np.uint8)
    g[:, :9] = 77
    p = str(tmp_path / "x.tga")
    write_tga(p, g, 3, 8, rle=rle)
    _same(p)
    ga = np.stack([g, 255 - g], axis=2)
    p2 = str(tmp_path / "y.tga")
    write_tga(p2, ga, 3, 16)
    _same(p2)


@needs_ref
@pytest.mark.parametrize("rle", [False, True])
def test_tga_colormapped(tmp_path, rle):
    rng = np.random.default_rng(9)
    pal = rng.integers(0, 256, (40, 3)).astype(np.uint8)
    idx = rng.integers(0, 40, (H, W)).astype(np.uint8)
    p = str(tmp_path / "x.tga")
    write_tga(p, idx, 1, 8, rle=rle, palette=pal)
    _same(p)


def test_bmp_rle_refused(tmp_path):
    p = str(tmp_path / "x.bmp")
    write_bmp(p, _rgb(1), bpp=24)
    data = bytearray(open(p, "rb").read())
    data[30:34] = struct.pack("<I", 1)  # BI_RLE8
    open(p, "wb").write(bytes(data))
    with pytest.raises(ValueError):
        io_load(p)
