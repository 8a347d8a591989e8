"""One surface split into x-strips (arma_ar_filter_strip + arma_b200.xstrip)
on the GPU.

The ranks of the strip pipeline are emulated one after another on one
device: strip r runs all its time chunks after strip r - 1, reading the
bands strip r - 1 sent (the exchange is the only coupling, so the order of
execution does not change any value; no kernel waits on another launch).
The strips put together are bit-identical to the single-surface FP32 filter.
"""
import numpy as np
import pytest

import arma_b200 as A
from arma_b200 import xstrip as X
import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def split_run(ctx, phi, eps, world, chunk):
    nt, nx, ny = eps.shape
    bands, out = {}, []
    for r, (x0, x1) in enumerate(X.strip_bounds(nx, world)):
        z = torch.from_numpy(np.ascontiguousarray(eps[:, x0:x1])).cuda()
        recv = (lambda a, b, r=r: bands[(r - 1, a)]) if r > 0 else None
        send = (lambda a, b, t, r=r: bands.__setitem__((r, a), t.clone())) if r < world - 1 else None
        X.filter_strip(ctx, phi, z, x0, chunk, recv, send)
        torch.cuda.synchronize()
        out.append(z.cpu().numpy())
    return np.concatenate(out, axis=1)


@pytest.mark.parametrize("shape,order,world,chunk", [
    ((40, 80, 70), (6, 8, 5), 2, 7),
    ((40, 80, 70), (6, 8, 5), 3, 16),
    ((40, 80, 70), (6, 8, 5), 5, 40),
    ((30, 70, 45), (4, 16, 4), 3, 3),     # a 15-row halo: nearly the whole band is read
    ((25, 48, 96), (10, 10, 10), 2, 9),
])
def test_strips_equal_the_whole_surface(ctx, shape, order, world, chunk):
    phi, var = A.ar_fit_analytic(A.ACF_STANDING, order, 1.5, 0.8, [0.05] * 3, [0.5, 0.5])
    eps = O.white_noise(O.mt19937_params(), 5, np.sqrt(var), int(np.prod(shape)))
    eps = eps.reshape(shape).astype(np.float32)
    whole = torch.from_numpy(eps.copy()).cuda()
    ctx.ar_filter(phi, shape, A.FP32C, whole.data_ptr())
    ctx.synchronize()
    got = split_run(ctx, phi, eps, world, chunk)
    assert np.array_equal(got, whole.cpu().numpy())


def test_strip_renorm_scale_matches_the_device_renorm(ctx):
    shape = (33, 80, 37)
    rng = np.random.default_rng(3)
    z = rng.standard_normal(shape).astype(np.float32)
    d = torch.from_numpy(z.copy()).cuda()
    want = ctx.variance_renorm(d.data_ptr(), shape, A.FP32C, 1.7)
    got = X.renorm_scale(torch.from_numpy(z).cuda(), shape, 0, 1.7)
    assert abs(got / want - 1) <= 1e-12


def test_strip_rejects_bad_bands(ctx):
    phi, _ = A.ar_fit_analytic(A.ACF_STANDING, (3, 3, 3), 1.5, 0.8, [0.05] * 3, [0.5, 0.5])
    z = torch.zeros((8, 40, 32), dtype=torch.float32, device="cuda")
    for t0, given in [(0, 8), (0, 40), (8, 16), (-1, 16)]:
        with pytest.raises(A.ArmaError) as e:
            ctx.ar_filter_strip(phi, tuple(z.shape), t0, given, z.data_ptr())
        assert e.value.code == -1
