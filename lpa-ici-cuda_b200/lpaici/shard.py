"""Multi-GPU decomposition (one process per GPU, torch.distributed for the plumbing).

The path has no exchange step: images are independent, and inside one image every output pixel only
reads input pixels within the kernel radius R.  So
  * a batch is split by whole images, largest first onto the least loaded rank (no collective);
  * one large image is split into row bands; a forward band carries R real rows above and below
    (2R for the adjoint: a gradient row depends on pixels within R whose selection depends on pixels
    within R of them); the outputs are disjoint bands, gathered to rank 0.
Every rank reads its own band (with halo) from the host copy it has and uploads it into its own
memory; no kernel reads another GPU's memory.

The band computation is a callable, so the decomposition runs the same way with the CUDA kernels
(forward_band / backward_band below) or, in CPU tests over gloo, with any other implementation.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, List, Sequence

import numpy as np


def assign_images(pixel_counts: Sequence[int], world: int) -> List[List[int]]:
    """Longest-processing-time-first: images by decreasing size, each onto the rank with the least
    work so far (ties to the lowest rank).  Returns the image indices of every rank, in order."""
    loads = [0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(pixel_counts)), key=lambda j: (-pixel_counts[j], j)):
        r = min(range(world), key=lambda q: (loads[q], q))
        out[r].append(i)
        loads[r] += pixel_counts[i]
    return out


@dataclass(frozen=True)
class Band:
    """Output rows [row0, row1) computed from input rows [in0, in1); output row r of the band is input
    row (row0 - in0) + r of the input band."""

    row0: int
    row1: int
    in0: int
    in1: int

    @property
    def row_begin(self) -> int:
        return self.row0 - self.in0

    @property
    def rows(self) -> int:
        return self.row1 - self.row0


def row_bands(height: int, world: int, halo: int) -> List[Band]:
    """Near-equal row bands (the first height % world bands one row taller), with `halo` rows of
    input on each side where the image has them."""
    base, extra = divmod(height, world)
    bands, y = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        bands.append(Band(y, y + n, max(0, y - halo), min(height, y + n + halo)))
        y += n
    return bands


BandFn = Callable[[np.ndarray, Band], np.ndarray]


def split_image(image: np.ndarray, band_fn: BandFn, halo: int, rank: int, world: int, group=None) -> np.ndarray | None:
    """Every rank computes its band of `image` (each rank holds the full host image) with band_fn and
    rank 0 gathers the bands (torch.distributed.gather of CPU tensors; works over gloo and NCCL
    groups with a CPU-capable backend).  Returns the full result on rank 0, None elsewhere."""
    import torch
    import torch.distributed as dist

    H, W = image.shape
    bands = row_bands(H, world, halo)
    b = bands[rank]
    mine = np.ascontiguousarray(band_fn(np.ascontiguousarray(image[b.in0:b.in1]), b), dtype=np.float32)
    if mine.shape != (b.rows, W):
        raise ValueError(f"band function returned {mine.shape}, expected {(b.rows, W)}")
    if world == 1:
        return mine
    # gather needs equal shapes: pad every band to the tallest
    tall = max(x.rows for x in bands)
    buf = torch.zeros((tall, W), dtype=torch.float32)
    buf[: b.rows] = torch.from_numpy(mine)
    gathered = [torch.zeros((tall, W), dtype=torch.float32) for _ in range(world)] if rank == 0 else None
    dist.gather(buf, gathered, dst=0, group=group)
    if rank != 0:
        return None
    return np.concatenate([g[: x.rows].numpy() for g, x in zip(gathered, bands)], axis=0)


# ---- the CUDA band functions ------------------------------------------------------------------

def forward_band(ks, sigma: float, gamma: float, device=None) -> BandFn:
    """Band function of the forward on the current (or given) CUDA device: uploads the band with its
    halo, runs lpaici_forward_rows on exactly the band's output rows, downloads them."""
    import torch

    import lpaici

    def fn(band_in: np.ndarray, b: Band) -> np.ndarray:
        x = torch.from_numpy(band_in).to(device or torch.device("cuda", torch.cuda.current_device()))
        out = lpaici.forward_rows(ks, x, b.row_begin, b.rows, sigma, gamma)
        return out.cpu().numpy()

    return fn


def backward_band(ks, grad_out: np.ndarray, sigma: float, gamma: float, device=None) -> BandFn:
    """Band function of the adjoint (halo 2R): runs lpaici_backward on the band with its halo
    (cotangent zero outside [row0, row1) would be wrong -- the halo rows keep their cotangent) and
    keeps the band's own rows."""
    import torch

    import lpaici

    def fn(band_in: np.ndarray, b: Band) -> np.ndarray:
        dev = device or torch.device("cuda", torch.cuda.current_device())
        x = torch.from_numpy(band_in).to(dev)
        g = torch.from_numpy(np.ascontiguousarray(grad_out[b.in0:b.in1], np.float32)).to(dev)
        gi = lpaici.backward(ks, x, g, sigma, gamma)
        return gi[b.row_begin:b.row_begin + b.rows].cpu().numpy()

    return fn
