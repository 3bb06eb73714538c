"""The large forward + adjoint case at full size: one 8192x8192 synthetic image, the gaussian m=(2,0)
16x7 kernel set, sigma 25/255, gamma 1.5, scale maps recomputed inside the backward.

Full-size checks that need no full-size oracle run:
  * forward and selected scales bit-equal to the FP32 oracle on windows (corner, edge, interior), each
    evaluated by the oracle on the window plus its R-pixel halo (exactly the input those pixels see);
  * adjoint against the FP64 oracle adjoint on crops: the gradient at q reads g and the selection within
    R of q, so the interior of a crop (R from any cut edge) is exact;
  * the adjoint identity sum(g * out) = sum(grad * x) (the frozen-selection map is linear), over the
    whole image.
Tolerance of the adjoint: |grad - ref| <= 2e-5 * max|ref| + 1e-6 (FP32 accumulation, FP64 reference)."""
import numpy as np
import pytest

import lpaici
import oracle_bind as ob
from conftest import GAUSS_M2, kernel_file

pytestmark = [pytest.mark.gpu, pytest.mark.slow]
N = 8192
SIGMA_25 = float(np.float32(25.0) / np.float32(255.0))
GAMMA = 1.5
RTOL = 2e-5


@pytest.fixture(scope="module")
def large():
    import torch

    ks = lpaici.KernelSet.load(kernel_file(GAUSS_M2))
    ko = ob.oracle_load_kernels(kernel_file(GAUSS_M2))
    noisy = lpaici.add_noise(lpaici.synth_image(N, N, 20250910), SIGMA_25, 20250910)
    x = torch.from_numpy(noisy).cuda()
    out, smap = lpaici.forward(ks, x, SIGMA_25, GAMMA, scale_map=True)
    g = torch.randn(N, N, generator=torch.Generator().manual_seed(5)).cuda()
    grad = lpaici.backward(ks, x, g, SIGMA_25, GAMMA)
    torch.cuda.synchronize()
    return dict(ks=ks, ko=ko, noisy=noisy, x=x, out=out, smap=smap, g=g, grad=grad,
                var=ks.variances(SIGMA_25))


@pytest.mark.parametrize("y,x", [(0, 0), (0, 4000), (N - 48, N - 48), (5123, 2977)])
def test_forward_windows_bit_exact(large, y, x):
    R, n = large["ks"].radius, 48
    noisy = large["noisy"]
    y0, x0, y1, x1 = max(0, y - R), max(0, x - R), min(N, y + n + R), min(N, x + n + R)
    ref, ref_map, _ = ob.oracle_forward_f32(noisy[y0:y1, x0:x1], large["ko"], large["var"], GAMMA, want_map=True)
    got = large["out"][y:y + n, x:x + n].cpu().numpy()
    assert np.array_equal(got.view(np.uint32), ref[y - y0:y - y0 + n, x - x0:x - x0 + n].view(np.uint32))
    got_map = large["smap"][:, y:y + n, x:x + n].cpu().numpy()
    assert np.array_equal(got_map, ref_map[:, y - y0:y - y0 + n, x - x0:x - x0 + n])


@pytest.mark.parametrize("y,x", [(0, 0), (3000, 6100), (N - 160, N - 160)])
def test_adjoint_crops_vs_fp64(large, y, x):
    R, c = large["ks"].radius, 160
    g = large["g"][y:y + c, x:x + c].cpu().numpy().astype(np.float64)
    smap = np.ascontiguousarray(large["smap"][:, y:y + c, x:x + c].cpu().numpy())
    ref = ob.oracle_adjoint_f64(large["ko"], large["var"], smap, g)
    got = large["grad"][y:y + c, x:x + c].cpu().numpy()
    # keep pixels at least R from every edge of the crop that is not an edge of the image
    top = 0 if y == 0 else R
    left = 0 if x == 0 else R
    bottom = c if y + c == N else c - R
    right = c if x + c == N else c - R
    a, b = got[top:bottom, left:right], ref[top:bottom, left:right]
    err = np.abs(a - b).max()
    assert err <= RTOL * np.abs(b).max() + 1e-6, (err, np.abs(b).max())


def test_adjoint_identity_full_image(large):
    g, x, out, grad = (large[k].double() for k in ("g", "x", "out", "grad"))
    a = float((g * out).sum())
    b = float((grad * x).sum())
    scale = float((g.abs() * out.abs()).sum())
    assert abs(a - b) <= 1e-5 * scale, (a, b, scale)
