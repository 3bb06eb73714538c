"""Multi-GPU decomposition logic over torch.distributed with gloo (world_size 2 and 3, on CPU).

The band computation is the oracle here (the CUDA band functions are the same calls as the
single-GPU tests); stitching the bands must give exactly the full-image result."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from lpaici.shard import Band, assign_images, row_bands

SIGMA = float(np.float32(20.0) / np.float32(255.0))


def test_assign_images_lpt():
    sizes = [100, 5, 60, 60, 7, 40]
    a = assign_images(sizes, 2)
    assert sorted(sum(a, [])) == list(range(len(sizes)))
    loads = [sum(sizes[i] for i in r) for r in a]
    assert max(loads) - min(loads) <= max(sizes)
    assert a[0][0] == 0  # largest first, onto rank 0
    assert assign_images(sizes, 1) == [sorted(range(6), key=lambda i: -sizes[i])]
    assert assign_images([3], 4) == [[0], [], [], []]


def test_row_bands_cover_and_halo():
    for H, world, halo in ((100, 3, 31), (7, 4, 31), (4096, 8, 62), (1, 2, 5)):
        bands = row_bands(H, world, halo)
        assert bands[0].row0 == 0 and bands[-1].row1 == H
        for a, b in zip(bands, bands[1:]):
            assert a.row1 == b.row0
        for b in bands:
            assert b.in0 == max(0, b.row0 - halo) and b.in1 == min(H, b.row1 + halo)
            assert b.row_begin == b.row0 - b.in0


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, mode, image, gout, result_path):
    import torch.distributed as dist

    import oracle_bind as ob
    from conftest import SYM, kernel_file
    from lpaici.shard import split_image

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ko = ob.oracle_load_kernels(kernel_file(SYM))
        var = ob.oracle_variances(ko, np.float32(SIGMA))
        R = 31
        if mode == "forward":
            def fn(x, b: Band):
                out, _, _ = ob.oracle_forward_f32(x, ko, var, 2.0)
                return out[b.row_begin:b.row_begin + b.rows]
            res = split_image(image, fn, R, rank, world)
        else:
            def fn(x, b: Band):
                _, smap, _ = ob.oracle_forward_f32(x, ko, var, 2.0, want_map=True)
                g = gout[b.in0:b.in1].astype(np.float64)
                gr = ob.oracle_adjoint_f64(ko, var, smap, g)
                return gr[b.row_begin:b.row_begin + b.rows].astype(np.float32)
            res = split_image(image, fn, 2 * R, rank, world)
        if rank == 0:
            np.save(result_path, res)
        else:
            assert res is None
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,mode", [(2, "forward"), (3, "forward"), (2, "adjoint")])
def test_split_image_gloo(tmp_path, world, mode):
    import lpaici
    import oracle_bind as ob
    from conftest import SYM, kernel_file

    H, W = 150, 48
    image = lpaici.add_noise(lpaici.synth_image(W, H, 21), SIGMA, 5)
    gout = np.random.default_rng(1).standard_normal((H, W)).astype(np.float32)
    out = str(tmp_path / "res.npy")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, mode, image, gout, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    got = np.load(out)
    ko = ob.oracle_load_kernels(kernel_file(SYM))
    var = ob.oracle_variances(ko, np.float32(SIGMA))
    if mode == "forward":
        full, _, _ = ob.oracle_forward_f32(image, ko, var, 2.0)
        assert np.array_equal(got.view(np.uint32), full.view(np.uint32))
    else:
        _, smap, _ = ob.oracle_forward_f32(image, ko, var, 2.0, want_map=True)
        full = ob.oracle_adjoint_f64(ko, var, smap, gout.astype(np.float64)).astype(np.float32)
        assert np.array_equal(got.view(np.uint32), full.view(np.uint32))


@pytest.mark.gpu
def test_cuda_band_functions_stitch_exactly():
    """forward_band / backward_band on one GPU, bands computed one after the other."""
    import torch

    import lpaici
    from conftest import SYM, kernel_file
    from lpaici.shard import backward_band, forward_band

    ks = lpaici.KernelSet.load(kernel_file(SYM))
    H, W = 203, 96
    image = lpaici.add_noise(lpaici.synth_image(W, H, 31), SIGMA, 9)
    g = np.random.default_rng(2).standard_normal((H, W)).astype(np.float32)
    x = torch.from_numpy(image).cuda()
    full = lpaici.forward(ks, x, SIGMA, 2.0).cpu().numpy()
    fb = forward_band(ks, SIGMA, 2.0)
    parts = [fb(np.ascontiguousarray(image[b.in0:b.in1]), b) for b in row_bands(H, 3, ks.radius)]
    assert np.array_equal(np.concatenate(parts).view(np.uint32), full.view(np.uint32))
    gfull = lpaici.backward(ks, x, torch.from_numpy(g).cuda(), SIGMA, 2.0).cpu().numpy()
    bb = backward_band(ks, g, SIGMA, 2.0)
    parts = [bb(np.ascontiguousarray(image[b.in0:b.in1]), b) for b in row_bands(H, 3, 2 * ks.radius)]
    err = np.abs(np.concatenate(parts) - gfull).max()
    assert err <= 2e-5 * np.abs(gfull).max() + 1e-6
