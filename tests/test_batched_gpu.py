"""Batched forward: images of uneven sizes, sigmas and gammas in one launch must give, image
by image, exactly the single-image result (which is bit-exact with the reference)."""
import numpy as np
import pytest

import lpaici
import oracle_bind as ob
from conftest import SYM, kernel_file

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    import torch

    ks = lpaici.KernelSet.load(kernel_file(SYM))
    ko = ob.oracle_load_kernels(kernel_file(SYM))
    rng = np.random.default_rng(123)
    sizes = [(1, 1), (1, 40), (37, 1), (64, 64), (130, 37), (257, 129), (300, 211), (72, 32), (5, 300)]
    imgs, sig, gam = [], [], []
    for i, (W, H) in enumerate(sizes):
        s = float(np.float32(rng.uniform(10, 40)) / np.float32(255.0))
        g = float(np.float32(rng.uniform(1.5, 2.5)))
        x = lpaici.add_noise(lpaici.synth_image(W, H, 1000 + i), s, 20250910 + i)
        imgs.append(torch.from_numpy(x).cuda())
        sig.append(s)
        gam.append(g)
    singles = [lpaici.forward(ks, x, s, g) for x, s, g in zip(imgs, sig, gam)]
    torch.cuda.synchronize()
    return torch, ks, ko, imgs, sig, gam, singles


@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_equals_single(setup, use_graph):
    torch, ks, ko, imgs, sig, gam, singles = setup
    outs = [torch.full_like(x, float("nan")) for x in imgs]
    b = lpaici.Batch(ks, imgs, outs, sig, gam, use_graph=use_graph)
    for rep in range(3):  # reruns reuse the plan
        for o in outs:
            o.fill_(float("nan"))
        b.run()
        torch.cuda.synchronize()
        for o, s in zip(outs, singles):
            assert torch.equal(o.view(torch.int32), s.view(torch.int32)), rep
    b.close()


@pytest.mark.parametrize("config", range(lpaici.lib().lpaici_num_tile_configs()))
def test_batch_every_tile_config(setup, config):
    torch, ks, ko, imgs, sig, gam, singles = setup
    outs = [torch.empty_like(x) for x in imgs]
    b = lpaici.Batch(ks, imgs, outs, sig, gam, use_graph=False, tile_config=config)
    b.run()
    torch.cuda.synchronize()
    for o, s in zip(outs, singles):
        assert torch.equal(o.view(torch.int32), s.view(torch.int32))
    b.close()


def test_batch_matches_oracle_and_scale_maps(setup):
    torch, ks, ko, imgs, sig, gam, singles = setup
    sel = [3, 4, 8]
    xs = [imgs[i] for i in sel]
    outs = [torch.empty_like(x) for x in xs]
    maps = [torch.empty((ks.D,) + tuple(x.shape), dtype=torch.uint8, device="cuda") for x in xs]
    b = lpaici.Batch(ks, xs, outs, [sig[i] for i in sel], [gam[i] for i in sel], scale_maps=maps)
    b.run()
    torch.cuda.synchronize()
    for j, i in enumerate(sel):
        ref, rmap, _ = ob.oracle_forward_f32(imgs[i].cpu().numpy(), ko, ks.variances(sig[i]), gam[i], want_map=True)
        assert np.array_equal(outs[j].cpu().numpy().view(np.uint32), ref.view(np.uint32))
        assert np.array_equal(maps[j].cpu().numpy(), rmap)
    b.close()


def test_one_shot_and_errors(setup):
    torch, ks, ko, imgs, sig, gam, singles = setup
    outs = lpaici.forward_batched(ks, imgs, sig, gam)
    for o, s in zip(outs, singles):
        assert torch.equal(o.view(torch.int32), s.view(torch.int32))
    with pytest.raises(lpaici.LpaIciError):
        lpaici.Batch(ks, imgs[:2], outs[:2], [0.1, -1.0], [2.0, 2.0])


@pytest.mark.parametrize("config", [-1] + list(range(lpaici.lib().lpaici_num_tile_configs())))
def test_one_size_plan(setup, config):
    """A plan of images of one size, pitch, sigma and gamma runs the single-image kernel once with a grid
    layer per image: every image equals its single-image call bit for bit, and the scale maps and outputs
    equal the oracle's."""
    torch, ks, ko, imgs, sig, gam, singles = setup
    s, g = sig[5], gam[5]
    xs = [torch.from_numpy(lpaici.add_noise(lpaici.synth_image(173, 131, 2000 + i), s, 77 + i)).cuda()
          for i in range(5)]
    ref = [lpaici.forward(ks, x, s, g) for x in xs]
    outs = [torch.full_like(x, float("nan")) for x in xs]
    maps = [torch.empty((ks.D,) + tuple(x.shape), dtype=torch.uint8, device="cuda") for x in xs]
    b = lpaici.Batch(ks, xs, outs, [s] * len(xs), [g] * len(xs), use_graph=config < 0,
                     tile_config=max(config, -1), scale_maps=maps)
    for rep in range(2):
        for o in outs:
            o.fill_(float("nan"))
        b.run()
        torch.cuda.synchronize()
        for o, r in zip(outs, ref):
            assert torch.equal(o.view(torch.int32), r.view(torch.int32)), rep
    b.close()
    if config in (-1, 0):
        var = ks.variances(s)
        for x, o, m in zip(xs[::2], outs[::2], maps[::2]):
            oref, rmap, _ = ob.oracle_forward_f32(x.cpu().numpy(), ko, var, g, want_map=True)
            assert np.array_equal(o.cpu().numpy().view(np.uint32), oref.view(np.uint32))
            assert np.array_equal(m.cpu().numpy(), rmap)
