"""Parity at the shapes of two benchmark configurations, through the batched plans a user runs.

Mixed batch (64 images, sides 256-2048, sigma U[10,40]/255, gamma U[1.5,2.5], 16x7 symmetric kernels,
CUDA graph): every image's output and selected scales are bit-equal to the FP32 oracle (the reference's
anisotropic_lpa_ici_cpu_fused, src/v1_0_lpa_ici_2D_fused.cpp:851-930, restated) on four windows per
image -- two opposite corners, a point on the top edge and one in the interior -- each evaluated by the
oracle on the window plus its R-pixel halo, which is exactly the input those pixels see.

Adjoint batch (8 images of 1024x1024, sigma 20/255, gamma 2, cotangent g ~ N(0, 1), through the batched
adjoint plan): the selected scales of every image equal the oracle's on the whole image, and at 256
seeded random pixels (32 per image) the gradient of sum(g * out) matches central finite differences
(eps = 1e-3) of the frozen-selection map in the FP64 oracle, within |grad - fd| <= 2e-5 * max|fd| + 1e-6.

The oracle calls run in threads (ctypes releases the GIL), so the CPU side takes seconds, not minutes.
"""
import concurrent.futures as cf

import numpy as np
import pytest

import lpaici
import oracle_bind as ob
from conftest import SYM, kernel_file
from lpaici.synth import mixed_batch

pytestmark = [pytest.mark.gpu, pytest.mark.slow]
SEED = 20250910
SIGMA_20 = float(np.float32(20.0) / np.float32(255.0))
RTOL = 2e-5
WIN = 32
THREADS = 16


def _windows(W, H, n):
    return [(0, 0), (H - n, W - n), (0, (W - n) // 2), (H // 2 - n // 2, W // 3)]


def test_mixed_batch_64_images_windows_bit_exact():
    import torch

    ks = lpaici.KernelSet.load(kernel_file(SYM))
    ko = ob.oracle_load_kernels(kernel_file(SYM))
    R = ks.radius
    spec = mixed_batch(64, SEED)
    hosts = [lpaici.add_noise(lpaici.synth_image(w, h, img_seed), s, noise_seed)
             for w, h, s, _, img_seed, noise_seed in spec]
    xs = [torch.from_numpy(h).cuda() for h in hosts]
    outs = [torch.full_like(x, float("nan")) for x in xs]
    maps = [torch.empty((ks.D,) + tuple(x.shape), dtype=torch.uint8, device="cuda") for x in xs]
    plan = lpaici.Batch(ks, xs, outs, [s[2] for s in spec], [s[3] for s in spec], use_graph=True, scale_maps=maps)
    plan.run()
    torch.cuda.synchronize()
    got = [o.cpu().numpy() for o in outs]
    got_maps = [m.cpu().numpy() for m in maps]
    plan.close()

    def check(i):
        w, h, s, gm, _, _ = spec[i]
        var = ks.variances(s)
        bad = []
        for y, x in _windows(w, h, WIN):
            y0, x0, y1, x1 = max(0, y - R), max(0, x - R), min(h, y + WIN + R), min(w, x + WIN + R)
            ref, ref_map, _ = ob.oracle_forward_f32(hosts[i][y0:y1, x0:x1], ko, var, gm, want_map=True)
            a = got[i][y:y + WIN, x:x + WIN]
            b = ref[y - y0:y - y0 + WIN, x - x0:x - x0 + WIN]
            if not np.array_equal(a.view(np.uint32), b.view(np.uint32)):
                bad.append((i, y, x, "out", float(np.abs(a - b).max())))
            if not np.array_equal(got_maps[i][:, y:y + WIN, x:x + WIN], ref_map[:, y - y0:y - y0 + WIN,
                                                                               x - x0:x - x0 + WIN]):
                bad.append((i, y, x, "scale map"))
        return bad

    with cf.ThreadPoolExecutor(max_workers=THREADS) as ex:
        bad = [b for r in ex.map(check, range(len(spec))) for b in r]
    assert not bad, bad[:8]
    assert all(np.isfinite(g).all() for g in got)


def test_adjoint_batch_8x1024_vs_central_differences():
    import torch

    ks = lpaici.KernelSet.load(kernel_file(SYM))
    ko = ob.oracle_load_kernels(kernel_file(SYM))
    m, n = 8, 1024
    var = ks.variances(SIGMA_20)
    hosts = [lpaici.add_noise(lpaici.synth_image(n, n, SEED + 100 + i), SIGMA_20, SEED + i) for i in range(m)]
    gs = [torch.randn(n, n, generator=torch.Generator().manual_seed(i)) for i in range(m)]
    xs = [torch.from_numpy(h).cuda() for h in hosts]
    gd = [g.cuda() for g in gs]
    grads = [torch.full_like(x, float("nan")) for x in xs]
    plan = lpaici.BackwardBatch(ks, xs, gd, grads, [SIGMA_20] * m, [2.0] * m, use_graph=True)
    plan.run()
    torch.cuda.synchronize()
    got = [g.cpu().numpy() for g in grads]
    plan.close()
    gpu_maps = [lpaici.forward(ks, x, SIGMA_20, 2.0, scale_map=True)[1].cpu().numpy() for x in xs]
    rng = np.random.default_rng(SEED)
    qs = [rng.choice(n * n, size=32, replace=False).astype(np.int64) for _ in range(m)]

    def check(i):
        _, smap, _ = ob.oracle_forward_f32(hosts[i], ko, var, 2.0, want_map=True)
        same_maps = np.array_equal(smap, gpu_maps[i])
        fd = ob.oracle_fd_grad_f64(hosts[i], ko, var, smap, gs[i].numpy().astype(np.float64), qs[i], 1e-3)
        return same_maps, fd, got[i].ravel()[qs[i]]

    with cf.ThreadPoolExecutor(max_workers=THREADS) as ex:
        res = list(ex.map(check, range(m)))
    assert all(r[0] for r in res), "selected scales differ from the oracle's"
    fd = np.concatenate([r[1] for r in res])
    g = np.concatenate([r[2] for r in res]).astype(np.float64)
    assert fd.size == 256
    err = np.abs(g - fd).max()
    assert err <= RTOL * np.abs(fd).max() + 1e-6, (err, np.abs(fd).max())
    assert all(np.isfinite(x).all() for x in got)
