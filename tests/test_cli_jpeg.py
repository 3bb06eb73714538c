"""The command line's JPEG reader against stb_image, the reference's loader (stbi_loadf(path, .., 1) and
(.., 3), src/v4_1_lpa_ici_2D_sparse_shared.cu:375), called in-process from the reference build.

The files come from a small baseline encoder written here (float DCT, per-image Huffman codes of equal
length, optional restart intervals, 8- or 16-bit quantisation tables): gray, YCbCr 4:4:4, 4:2:2, 4:2:0
and 1x2 sampling, RGB-coded (Adobe transform 0), odd sizes, one interleaved scan or one scan per
component.  Every float of the result must be bit-equal to stb's.
"""
import struct

import numpy as np
import pytest

import oracle_bind as ob
from test_cli import io_load, io_load_rgb, needs_ref

ZIGZAG = np.array([0, 1, 8, 16, 9, 2, 3, 10, 17, 24, 32, 25, 18, 11, 4, 5, 12, 19, 26, 33, 40, 48, 41, 34, 27, 20,
                   13, 6, 7, 14, 21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51, 58, 59, 52,
                   45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63])
_k = np.arange(8)
DCT = np.sqrt(2.0 / 8) * np.cos((2 * _k[None, :] + 1) * _k[:, None] * np.pi / 16)
DCT[0] /= np.sqrt(2.0)


class Bits:
    def __init__(self):
        self.out = bytearray()
        self.acc = 0
        self.n = 0

    def put(self, code, length):
        for i in range(length - 1, -1, -1):
            self.acc = (self.acc << 1) | ((code >> i) & 1)
            self.n += 1
            if self.n == 8:
                self.out.append(self.acc)
                if self.acc == 0xFF:
                    self.out.append(0)
                self.acc = self.n = 0

    def flush(self):
        while self.n:
            self.put(1, 1)


def _category(v):
    return 0 if v == 0 else int(abs(v)).bit_length()


def _bits_of(v, s):
    return v if v >= 0 else v + (1 << s) - 1


def _table(symbols):
    """Canonical code with every used symbol at one length (the all-ones code left unused)."""
    syms = sorted(set(symbols))
    L = max(1, (len(syms) + 1 - 1).bit_length())
    while (1 << L) - 1 < len(syms):
        L += 1
    counts = [0] * 16
    counts[L - 1] = len(syms)
    codes = {s: (i, L) for i, s in enumerate(syms)}
    return counts, syms, codes


def encode_jpeg(path, img, sampling, quality_q=None, restart=0, rgb_coded=False, per_component_scans=False,
                q16=False, seed=0):
    """img: H x W (gray) or H x W x 3 uint8.  sampling: [(h, v)] per component."""
    rng = np.random.default_rng(seed)
    H, W = img.shape[:2]
    if img.ndim == 2:
        planes = [img.astype(np.float64)]
    elif rgb_coded:
        planes = [img[..., c].astype(np.float64) for c in range(3)]
    else:
        r, g, b = (img[..., c].astype(np.float64) for c in range(3))
        y = 0.299 * r + 0.587 * g + 0.114 * b
        cb = -0.168736 * r - 0.331264 * g + 0.5 * b + 128
        cr = 0.5 * r - 0.418688 * g - 0.081312 * b + 128
        planes = [np.clip(np.round(p), 0, 255) for p in (y, cb, cr)]
    n = len(planes)
    hmax = max(s[0] for s in sampling)
    vmax = max(s[1] for s in sampling)
    mcux, mcuy = -(-W // (8 * hmax)), -(-H // (8 * vmax))
    qt = [rng.integers(1, 40 if not q16 else 300, 64) for _ in range(n)]
    if quality_q is not None:
        qt = [np.full(64, quality_q) for _ in range(n)]
    blocks = []  # per component: [by][bx] -> 64 zigzag ints
    for c in range(n):
        h, v = sampling[c]
        # full-resolution plane padded to whole MCUs by edge replication, then box-filtered down
        P = np.pad(planes[c], ((0, mcuy * 8 * vmax - H), (0, mcux * 8 * hmax - W)), mode="edge")
        fy, fx = vmax // v, hmax // h
        P = P.reshape(P.shape[0] // fy, fy, P.shape[1] // fx, fx).mean(axis=(1, 3))
        nby, nbx = P.shape[0] // 8, P.shape[1] // 8
        B = {}
        for by in range(nby):
            for bx in range(nbx):
                blk = P[by * 8:by * 8 + 8, bx * 8:bx * 8 + 8] - 128
                coef = DCT @ blk @ DCT.T
                qz = np.round(coef.reshape(64) / qt[c]).astype(int)
                B[by, bx] = qz[ZIGZAG]
        blocks.append((nby, nbx, B))
    # symbol streams, then codes
    def units():
        if per_component_scans and n > 1:
            for c in range(n):
                h, v = sampling[c]
                cw, ch = -(-W * h // hmax), -(-H * v // vmax)
                yield [[(c, by, bx)] for by in range(-(-ch // 8)) for bx in range(-(-cw // 8))]
        else:
            mcus = []
            for my in range(mcuy):
                for mx in range(mcux):
                    u = []
                    for c in range(n):
                        h, v = sampling[c]
                        u += [(c, my * v + y, mx * h + x) for y in range(v) for x in range(h)]
                    mcus.append(u)
            yield mcus

    scans = list(units())
    dc_syms, ac_syms = [[] for _ in range(n)], [[] for _ in range(n)]
    for scan in scans:
        pred = [0] * n
        for i, u in enumerate(scan):
            if restart and i % restart == 0:
                pred = [0] * n
            for c, by, bx in u:
                z = blocks[c][2][by, bx]
                d = int(z[0]) - pred[c]
                pred[c] = int(z[0])
                dc_syms[c].append(_category(d))
                run = 0
                last = max([k for k in range(1, 64) if z[k] != 0], default=0)
                for k in range(1, last + 1):
                    if z[k] == 0:
                        run += 1
                        continue
                    while run > 15:
                        ac_syms[c].append(0xF0)
                        run -= 16
                    ac_syms[c].append((run << 4) | _category(int(z[k])))
                    run = 0
                if last < 63:
                    ac_syms[c].append(0)
    tabs = [(_table(dc_syms[c] or [0]), _table(ac_syms[c] or [0])) for c in range(n)]
    out = bytearray(b"\xff\xd8")
    if rgb_coded:
        out += b"\xff\xee" + struct.pack(">H", 14) + b"Adobe" + bytes([0, 100, 0, 0, 0, 0, 0])
    else:
        out += b"\xff\xe0" + struct.pack(">H", 16) + b"JFIF\0" + bytes([1, 1, 0, 0, 1, 0, 1, 0, 0])
    for c in range(n):
        pq = 1 if q16 else 0
        body = bytes([(pq << 4) | c]) + b"".join(struct.pack(">H" if pq else ">B", int(v)) for v in qt[c][ZIGZAG])
        out += b"\xff\xdb" + struct.pack(">H", 2 + len(body)) + body
    sof = bytes([8]) + struct.pack(">HH", H, W) + bytes([n])
    for c in range(n):
        sof += bytes([c + 1, (sampling[c][0] << 4) | sampling[c][1], c])
    out += b"\xff\xc0" + struct.pack(">H", 2 + len(sof)) + sof
    for c in range(n):
        for cls, (counts, syms, _) in ((0, tabs[c][0]), (1, tabs[c][1])):
            body = bytes([(cls << 4) | c]) + bytes(counts) + bytes(syms)
            out += b"\xff\xc4" + struct.pack(">H", 2 + len(body)) + body
    if restart:
        out += b"\xff\xdd" + struct.pack(">HH", 4, restart)
    for scan in scans:
        comps = sorted({c for u in scan for c, _, _ in u})
        sos = bytes([len(comps)]) + b"".join(bytes([c + 1, (c << 4) | c]) for c in comps) + bytes([0, 63, 0])
        out += b"\xff\xda" + struct.pack(">H", 2 + len(sos)) + sos
        bw = Bits()
        pred = [0] * n
        for i, u in enumerate(scan):
            if restart and i % restart == 0 and i:
                bw.flush()
                out += bw.out + bytes([0xFF, 0xD0 + ((i // restart - 1) % 8)])
                bw = Bits()
                pred = [0] * n
            for c, by, bx in u:
                z = blocks[c][2][by, bx]
                d = int(z[0]) - pred[c]
                pred[c] = int(z[0])
                s = _category(d)
                bw.put(*tabs[c][0][2][s])
                bw.put(_bits_of(d, s), s)
                run = 0
                last = max([k for k in range(1, 64) if z[k] != 0], default=0)
                for k in range(1, last + 1):
                    v = int(z[k])
                    if v == 0:
                        run += 1
                        continue
                    while run > 15:
                        bw.put(*tabs[c][1][2][0xF0])
                        run -= 16
                    s = _category(v)
                    bw.put(*tabs[c][1][2][(run << 4) | s])
                    bw.put(_bits_of(v, s), s)
                    run = 0
                if last < 63:
                    bw.put(*tabs[c][1][2][0])
        bw.flush()
        out += bw.out
    out += b"\xff\xd9"
    open(path, "wb").write(bytes(out))


def _image(H, W, seed):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:H, 0:W]
    base = np.stack([128 + 100 * np.sin(xx / 5.0 + c) * np.cos(yy / 7.0 - c) for c in range(3)], axis=2)
    return np.clip(base + rng.normal(0, 25, (H, W, 3)), 0, 255).astype(np.uint8)


def _same(path, rgb=True):
    assert np.array_equal(io_load(path).view(np.uint32), ob.ref_stbi_loadf(path).view(np.uint32))
    if rgb:
        assert np.array_equal(io_load_rgb(path).view(np.uint32), ob.ref_stbi_loadf_rgb(path).view(np.uint32))


@needs_ref
@pytest.mark.parametrize("sampling", [[(1, 1), (1, 1), (1, 1)], [(2, 1), (1, 1), (1, 1)], [(2, 2), (1, 1), (1, 1)],
                                      [(1, 2), (1, 1), (1, 1)]], ids=["444", "422", "420", "440"])
@pytest.mark.parametrize("H,W", [(37, 45), (64, 48), (9, 1), (1, 23)])
def test_jpeg_ycbcr(tmp_path, sampling, H, W):
    p = str(tmp_path / "x.jpg")
    encode_jpeg(p, _image(H, W, H * W), sampling, seed=H + W)
    _same(p)


@needs_ref
@pytest.mark.parametrize("restart", [1, 3])
@pytest.mark.parametrize("per_component_scans", [False, True])
def test_jpeg_restart_and_scans(tmp_path, restart, per_component_scans):
    p = str(tmp_path / "x.jpg")
    encode_jpeg(p, _image(50, 70, 5), [(2, 2), (1, 1), (1, 1)], restart=restart,
                per_component_scans=per_component_scans, seed=restart)
    _same(p)


@needs_ref
def test_jpeg_gray_16bit_tables_and_rgb_coded(tmp_path):
    g = _image(40, 33, 7)[..., 0]
    p = str(tmp_path / "g.jpg")
    encode_jpeg(p, g, [(1, 1)], q16=True)
    _same(p)
    q = str(tmp_path / "rgb.jpg")
    encode_jpeg(q, _image(24, 30, 8), [(1, 1), (1, 1), (1, 1)], rgb_coded=True)
    _same(q)
    fine = str(tmp_path / "fine.jpg")  # quantisation 1: large coefficients, the IDCT's clamping at 0 and 255
    encode_jpeg(fine, _image(16, 16, 9), [(1, 1), (1, 1), (1, 1)], quality_q=1)
    _same(fine)


def test_progressive_jpeg_refused(tmp_path):
    p = str(tmp_path / "x.jpg")
    encode_jpeg(p, _image(16, 16, 1)[..., 0], [(1, 1)])
    data = open(p, "rb").read().replace(b"\xff\xc0", b"\xff\xc2", 1)
    open(p, "wb").write(data)
    with pytest.raises(ValueError):
        io_load(p)
