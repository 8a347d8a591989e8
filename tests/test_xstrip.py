"""One surface split into x-strips, on the CPU: three gloo ranks run the
strip pipeline of arma_b200.xstrip (band send/recv per time chunk, the
renormalisation's all-reduced window sums) with the filter's strip
semantics (given band rows, given history slices) restated directly in
Python in place of the device; the strips put together equal the same
restatement run on the whole surface, value for value."""
import ctypes
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SHAPE = (11, 64, 9)
ORDER = (3, 4, 3)


class StripFilter:
    """arma_ar_filter_strip's semantics restated: slices [0, t0) and rows
    [0, given) are read only; every other point is its noise plus the sum of
    phi(k, i, j) z(t-k, x-i, y-j) over the taps (zero outside the buffer),
    summed in FP64 and stored as float."""

    def ar_filter_strip(self, phi, shape, t0, given, ptr):
        nt, nx, ny = shape
        z = np.ctypeslib.as_array((ctypes.c_float * (nt * nx * ny)).from_address(ptr))
        z = z.reshape(shape)
        pt, px, py = phi.shape
        taps = [(k, i, j, phi[k, i, j]) for k in range(pt) for i in range(px) for j in range(py)
                if (k, i, j) != (0, 0, 0)]
        for t in range(t0, nt):
            for x in range(given, nx):
                for y in range(ny):
                    acc = float(z[t, x, y])
                    for k, i, j, p in taps:
                        if t >= k and x >= i and y >= j:
                            acc += p * float(z[t - k, x - i, y - j])
                    z[t, x, y] = acc


def model():
    rng = np.random.default_rng(7)
    phi = rng.uniform(-0.05, 0.05, ORDER)
    phi[0, 0, 0] = 0.0
    eps = rng.standard_normal(SHAPE).astype(np.float32)
    return phi, eps


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, chunk, q):
    import sys
    from datetime import timedelta
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    from arma_b200 import xstrip as X
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        phi, eps = model()
        x0, x1 = X.strip_bounds(SHAPE[1], world)[rank]
        z = torch.from_numpy(np.ascontiguousarray(eps[:, x0:x1]))
        X.filter_surface(StripFilter(), phi, z, x0, chunk)
        scale = X.renorm_scale(z, SHAPE, x0, 1.3)
        q.put((rank, x0, z.numpy().copy(), scale))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("chunk", [4, 11])
def test_three_gloo_ranks_filter_one_surface_in_strips(chunk):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 3, port, chunk, q)) for r in range(3)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=180) for _ in procs), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    import torch
    from arma_b200 import xstrip as X
    phi, eps = model()
    whole = eps.copy()
    StripFilter().ar_filter_strip(phi, SHAPE, 0, 0, whole.ctypes.data)
    got = np.concatenate([z for _, _, z, _ in res], axis=1)
    assert [x0 for _, x0, _, _ in res] == [0, 16, 32]
    assert np.array_equal(got, whole)
    want = X.renorm_scale(torch.from_numpy(whole), SHAPE, 0, 1.3)
    for *_, s in res:
        assert s == pytest.approx(want, rel=1e-12)


def test_strip_bounds_and_windows():
    from arma_b200 import xstrip as X
    assert X.strip_bounds(70, 3) == [(0, 16), (16, 48), (48, 70)]
    assert X.strip_bounds(64, 4) == [(0, 16), (16, 32), (32, 48), (48, 64)]
    with pytest.raises(ValueError):
        X.strip_bounds(40, 4)
    shape = (9, 70, 13)
    nt, nx, ny = shape
    flat = np.arange(nt * nx * ny).reshape(shape)
    count = (nt - nt // 2) * (nx - nx // 2) * (ny - ny // 2)
    s0 = flat[nt // 2, nx // 2, ny // 2]
    seen = []
    for x0, x1 in X.strip_bounds(nx, 3):
        part = flat[:, x0:x1].reshape(nt, -1)
        for t, lo, hi in X.renorm_window(shape, x0, x1):
            seen += part[t, lo:hi].tolist()
    assert sorted(seen) == list(range(s0, s0 + count))


def test_strip_arguments_are_checked():
    import torch
    from arma_b200 import xstrip as X
    phi, eps = model()
    z = torch.from_numpy(np.ascontiguousarray(eps[:, :16]))
    band = lambda a, b: torch.zeros((b - a, X.BAND, SHAPE[2]))  # noqa: E731
    with pytest.raises(ValueError):   # strips start on the 16-row tile grid
        X.filter_strip(StripFilter(), phi, z, 8, 4, band)
    with pytest.raises(ValueError):   # a strip below the first needs its band
        X.filter_strip(StripFilter(), phi, z, 16, 4)
    with pytest.raises(ValueError):   # the first strip has none
        X.filter_strip(StripFilter(), phi, z, 0, 4, band)
    short = torch.from_numpy(np.ascontiguousarray(eps[:, :8]))
    with pytest.raises(ValueError):   # too few rows to feed the strip below
        X.filter_strip(StripFilter(), phi, short, 0, 4, None, lambda a, b, t: None)


def test_one_slice_chunks_equal_the_whole_surface_in_one_process():
    """The pipeline with the bands handed over in memory, chunks of one slice
    (every chunk's history from earlier chunks only)."""
    import torch
    from arma_b200 import xstrip as X
    phi, eps = model()
    whole = eps.copy()
    StripFilter().ar_filter_strip(phi, SHAPE, 0, 0, whole.ctypes.data)
    bands, out = {}, []
    for r, (x0, x1) in enumerate(X.strip_bounds(SHAPE[1], 2)):
        z = torch.from_numpy(np.ascontiguousarray(eps[:, x0:x1]))
        recv = (lambda a, b, r=r: bands[(r - 1, a)]) if r else None
        send = (lambda a, b, t, r=r: bands.__setitem__((r, a), t.clone())) if r == 0 else None
        X.filter_strip(StripFilter(), phi, z, x0, 1, recv, send)
        out.append(z.numpy())
    assert np.array_equal(np.concatenate(out, axis=1), whole)
