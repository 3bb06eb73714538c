"""Seeded synthetic grayscale test images: piecewise-constant polygons, a smooth linear ramp and
sinusoidal stripe textures (period 4-16 px, random orientation), clamped to [0, 1].

The reference benchmarks one natural photograph; there is no public benchmark set for this path, so
these images stand in for it.  Sizes are in pixels, not relative to the image, so the density of
edges and textures -- which decides where the ICI rule stops -- is the same at 512^2 and 8192^2.

With rgbe=True (default) every value is quantised through the Radiance RGBE encoding a .hdr file
stores (8-bit mantissa, shared exponent, gray as R=G=B), so the image written as .hdr and read back
by stb_image (the reference's loader) is bit-identical to the array.
"""
from __future__ import annotations

import numpy as np


def rgbe_quantize(v: np.ndarray) -> np.ndarray:
    """Gray float32 -> RGBE (R=G=B) -> gray float32, with the float arithmetic of the usual
    encoder (mantissa*256/max, truncated to 8 bits) and of a 1-channel decoder ((R+G+B)*2^(e-136)/3)."""
    v = np.ascontiguousarray(v, np.float32)
    out = np.zeros_like(v)
    nz = v >= np.float32(1e-32)
    x = v[nz]
    m, e = np.frexp(x)
    normalize = (m.astype(np.float32) * np.float32(256.0)) / x
    byte = np.trunc(x * normalize).astype(np.int32)
    f1 = np.ldexp(np.float32(1.0), (e + 128) - 136).astype(np.float32)
    out[nz] = (np.float32(3) * byte.astype(np.float32)) * f1 / np.float32(3.0)
    return out


def _polygon_mask(h, w, cy, cx, angles, radii, y0, x0):
    """Inside test of a star-shaped polygon (vertices at `angles`/`radii` around (cy, cx)) over the
    box [y0, y0+h) x [x0, x0+w)."""
    yy, xx = np.mgrid[y0:y0 + h, x0:x0 + w].astype(np.float32)
    dy, dx = yy - cy, xx - cx
    phi = np.mod(np.arctan2(dy, dx), 2 * np.pi)
    k = np.searchsorted(angles, phi, side="right") - 1  # segment (k, k+1), wrapping
    k = np.mod(k, len(angles))
    k1 = np.mod(k + 1, len(angles))
    vy = radii * np.sin(angles)
    vx = radii * np.cos(angles)
    ay, ax, by, bx = vy[k], vx[k], vy[k1], vx[k1]
    # same side of edge (a, b) as the centre (origin): cross(b - a, p - a) has the sign of cross(b - a, -a)
    c_p = (bx - ax) * (dy - ay) - (by - ay) * (dx - ax)
    c_o = (bx - ax) * (-ay) - (by - ay) * (-ax)
    return c_p * c_o >= 0


def synth_image(width: int, height: int, seed: int, rgbe: bool = True) -> np.ndarray:
    """The benchmark image: float32 [height, width] in [0, 1]."""
    rng = np.random.default_rng(seed)
    H, W = height, width
    yy, xx = np.mgrid[0:H, 0:W].astype(np.float32)
    # smooth linear ramp
    a, b = rng.uniform(-0.35, 0.35, size=2)
    img = (np.float32(0.5) + np.float32(a) * (xx / max(W, 1) - 0.5) + np.float32(b) * (yy / max(H, 1) - 0.5))
    img = img.astype(np.float32)
    del yy, xx
    # piecewise-constant polygons, some carrying a stripe texture
    n_poly = max(8, int(round(W * H / (96.0 * 96.0))))
    for _ in range(n_poly):
        r_max = rng.uniform(12.0, 128.0)
        cy, cx = rng.uniform(0, H), rng.uniform(0, W)
        nv = int(rng.integers(3, 10))
        angles = np.sort(rng.uniform(0, 2 * np.pi, nv)).astype(np.float32)
        radii = (r_max * rng.uniform(0.45, 1.0, nv)).astype(np.float32)
        level = np.float32(rng.uniform(0.0, 1.0))
        striped = rng.uniform() < 0.5
        period = rng.uniform(4.0, 16.0)
        theta = rng.uniform(0.0, np.pi)
        amp = np.float32(rng.uniform(0.05, 0.2))
        y0, y1 = int(max(0, np.floor(cy - r_max))), int(min(H, np.ceil(cy + r_max) + 1))
        x0, x1 = int(max(0, np.floor(cx - r_max))), int(min(W, np.ceil(cx + r_max) + 1))
        if y1 <= y0 or x1 <= x0:
            continue
        m = _polygon_mask(y1 - y0, x1 - x0, np.float32(cy), np.float32(cx), angles, radii, y0, x0)
        patch = img[y0:y1, x0:x1]
        if striped:
            py, px = np.mgrid[y0:y1, x0:x1].astype(np.float32)
            tex = amp * np.sin(np.float32(2 * np.pi / period) *
                               (px * np.float32(np.cos(theta)) + py * np.float32(np.sin(theta))))
            patch[m] = (level + tex[m]).astype(np.float32)
        else:
            patch[m] = level
    np.clip(img, 0.0, 1.0, out=img)
    return rgbe_quantize(img) if rgbe else img


def mixed_batch(n: int = 64, seed: int = 20250910):
    """The mixed batch of the batched benchmark: n images with width and height drawn uniformly from
    256..2048, sigma uniform in 10/255..40/255 and gamma uniform in 1.5..2.5 (FP32), all from one
    generator seeded with `seed`.  Returns (width, height, sigma, gamma, image_seed, noise_seed) per
    image: image i is synth_image(width, height, seed + 1 + i) with noise seed seed + i."""
    rng = np.random.default_rng(seed)
    dims = rng.integers(256, 2049, size=(n, 2))
    sig = (rng.uniform(10, 40, n).astype(np.float32) / np.float32(255.0)).astype(np.float32)
    gam = rng.uniform(1.5, 2.5, n).astype(np.float32)
    return [(int(dims[i, 0]), int(dims[i, 1]), float(sig[i]), float(gam[i]), seed + 1 + i, seed + i)
            for i in range(n)]
