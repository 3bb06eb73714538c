"""Batched adjoint plan (lpaici_backward_batch_*): images of uneven sizes, sigmas and gammas in one
selection launch and one gather launch (optionally one CUDA graph).  Every gradient equals the
single-image lpaici_backward's bit for bit -- the same kernels run on the same tiles with the same
tables -- with and without the graph, and on a second run of the plan."""
import numpy as np
import pytest

import lpaici
from conftest import GAUSS_M2, SYM, kernel_file

pytestmark = pytest.mark.gpu
SHAPES = [(300, 200), (1024, 77), (129, 513), (64, 64), (1, 1)]


def _images(seed):
    import torch

    rng = np.random.default_rng(seed)
    xs, gs, sig, gam = [], [], [], []
    for i, (W, H) in enumerate(SHAPES):
        s = float(np.float32(rng.uniform(10, 40)) / np.float32(255.0))
        xs.append(torch.from_numpy(lpaici.add_noise(lpaici.synth_image(W, H, seed + i), s, seed + i)).cuda())
        gs.append(torch.from_numpy(rng.standard_normal((H, W)).astype(np.float32)).cuda())
        sig.append(s)
        gam.append(float(rng.uniform(1.5, 2.5)))
    return xs, gs, sig, gam


@pytest.mark.parametrize("name,use_graph", [(SYM, True), (SYM, False), (GAUSS_M2, True)])
def test_batched_equals_single(name, use_graph):
    import torch

    ks = lpaici.KernelSet.load(kernel_file(name))
    xs, gs, sig, gam = _images(31)
    outs = [torch.full_like(x, float("nan")) for x in xs]
    plan = lpaici.BackwardBatch(ks, xs, gs, outs, sig, gam, use_graph=use_graph)
    for rep in range(2):
        plan.run()
        torch.cuda.synchronize()
        for x, g, o, s, a in zip(xs, gs, outs, sig, gam):
            ref = lpaici.backward(ks, x, g, s, a)
            assert torch.equal(o.view(torch.int32), ref.view(torch.int32)), (rep, tuple(x.shape))
        for o in outs:
            o.fill_(float("nan"))
    plan.close()


def test_batched_pitched_views():
    import torch

    ks = lpaici.KernelSet.load(kernel_file(SYM))
    xs, gs, sig, gam = _images(37)
    big = [torch.zeros((x.shape[0], x.shape[1] + 5), device="cuda") for x in xs]
    views = [b[:, : x.shape[1]] for b, x in zip(big, xs)]
    plan = lpaici.BackwardBatch(ks, xs, gs, views, sig, gam)
    plan.run()
    torch.cuda.synchronize()
    for x, g, v, b, s, a in zip(xs, gs, views, big, sig, gam):
        assert torch.equal(v, lpaici.backward(ks, x, g, s, a))
        assert torch.count_nonzero(b[:, x.shape[1]:]) == 0  # nothing written beside the gradient
    plan.close()
