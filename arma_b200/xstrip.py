"""One AR surface split across ranks by rows (x-strips).

A surface too large for one device is cut into strips of rows: rank r owns
rows [x0_r, x1_r), every x0_r a multiple of the FP32 filter's 16 tile rows, so
the tiles of a strip are tiles of the whole surface and the strip's values are
bit-identical to the single-device filter's.  The filter at row x reads rows
x - px + 1 .. x of the same and earlier slices, so strip r depends on the
last 16 rows of strip r - 1 and on nothing below it.  The strips run as a
pipeline over time chunks -- the reference's partition wavefront with halos
(src/generator/ar_model_bscheduler.cc:285-353), recast per rank: for chunk c
rank r receives strip r - 1's last 16 rows of the chunk's slices, filters its
own rows of the chunk with those rows and the previous chunk's last pt - 1
slices given (``arma_ar_filter_strip``), and sends its own last 16 rows on,
while rank r - 1 already filters chunk c + 1.  The only exchange is that band,
16 x chunk x ny floats per chunk and strip boundary: NCCL send/recv between
neighbouring ranks on GPUs, gloo on the CPU.

The variance renormalisation's window (the reference's contiguous view,
src/generator/basic_arma_model.cc:102-106) crosses strips: each rank sums its
part of the window in FP64 and the sums are all-reduced in two passes (the
mean, then the squared deviations).
"""
from __future__ import annotations

import numpy as np

BAND = 16  # the FP32 filter's tile rows: what a strip receives from the one above


def strip_bounds(nx: int, world: int) -> list:
    """Rows [x0, x1) of each of `world` strips: whole 16-row tiles, as even
    as that allows (only the last strip may end in a partial tile)."""
    tiles = (nx + BAND - 1) // BAND
    if world < 1 or tiles < world:
        raise ValueError(f"{nx} rows hold {tiles} tiles of {BAND} rows: too few for {world} strips")
    return [((r * tiles // world) * BAND, min(nx, ((r + 1) * tiles // world) * BAND))
            for r in range(world)]


def filter_strip(ctx, phi, zeta, x0: int, chunk: int, recv_band=None, send_band=None):
    """Filter one strip in place, chunk by chunk.

    zeta: (nt, rows, ny) float32 CUDA tensor holding the strip's white noise
    (rows x0 .. x0 + rows - 1 of the surface).  recv_band(a, b) returns the
    strip above's last 16 rows of slices [a, b) as a (b - a, 16, ny) float32
    CUDA tensor (None for the first strip, x0 = 0); send_band(a, b, rows)
    passes this strip's last 16 rows of slices [a, b) to the strip below
    (None for the last strip).  Returns zeta."""
    import torch

    phi = np.ascontiguousarray(phi, np.float64)
    pt = phi.shape[0]
    hist = pt - 1
    nt, rows, ny = zeta.shape
    if x0 % BAND:
        raise ValueError(f"a strip must start at a multiple of {BAND} rows")
    if (x0 > 0) != (recv_band is not None):
        raise ValueError("only the first strip (x0 = 0) has no strip above")
    if send_band is not None and rows < BAND:
        raise ValueError(f"a strip with a strip below needs at least {BAND} rows")
    band = BAND if x0 > 0 else 0
    band_hist = None  # the band's last `hist` slices
    for a in range(0, nt, chunk):
        b = min(nt, a + chunk)
        h = min(hist, a)
        ext = torch.zeros((h + b - a, band + rows, ny), dtype=torch.float32, device=zeta.device)
        ext[:, band:] = zeta[a - h:b]
        if band:
            cur = recv_band(a, b)
            ext[h:, :band] = cur
            if h:
                ext[:h, :band] = band_hist[-h:]
            if hist:
                band_hist = cur[-hist:] if band_hist is None else torch.cat([band_hist, cur])[-hist:]
        if ext.is_cuda:  # the library works on its own stream
            torch.cuda.current_stream().synchronize()
        ctx.ar_filter_strip(phi, tuple(ext.shape), h, band, ext.data_ptr())
        zeta[a:b] = ext[h:, band:]
        if send_band is not None:
            send_band(a, b, zeta[a:b, rows - BAND:].contiguous())
    return zeta


def filter_surface(ctx, phi, zeta, x0: int, chunk: int, group=None):
    """filter_strip on this rank of `group` (torch.distributed), the band
    exchanged with the neighbouring ranks by send/recv.  Rank r must hold
    the strip strip_bounds(nx, world)[r]."""
    import torch
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    nt, rows, ny = zeta.shape

    def recv(a, b):
        t = torch.empty((b - a, BAND, ny), dtype=torch.float32, device=zeta.device)
        dist.recv(t, src=_global(group, rank - 1), group=group)
        return t

    def send(a, b, t):
        dist.send(t, dst=_global(group, rank + 1), group=group)

    return filter_strip(ctx, phi, zeta, x0, chunk, recv if rank > 0 else None,
                        send if rank < world - 1 else None)


def renorm_window(shape, x0: int, x1: int):
    """This strip's part of the renormalisation window as (t, lo, hi) runs:
    values lo .. hi - 1, in memory order, of the strip's slice t.  The window
    is the numElements() values in memory order from zeta(nt/2, nx/2, ny/2),
    as the reference takes it."""
    nt, nx, ny = shape
    count = (nt - nt // 2) * (nx - nx // 2) * (ny - ny // 2)
    s0 = ((nt // 2) * nx + nx // 2) * ny + ny // 2
    s1 = s0 + count
    runs = []
    for t in range(nt):
        lo = max(s0, (t * nx + x0) * ny)
        hi = min(s1, (t * nx + x1) * ny)
        if lo < hi:
            runs.append((t, lo - (t * nx + x0) * ny, hi - (t * nx + x0) * ny))
    return runs


def renorm_scale(zeta, shape, x0: int, acf0: float, group=None) -> float:
    """sqrt(acf0 / var) with var the unbiased variance of the reference's
    window over the whole surface, from this rank's strip (all-reduced)."""
    import torch
    import torch.distributed as dist

    nt, rows, ny = zeta.shape
    flat = zeta.reshape(nt, rows * ny)
    parts = [flat[t, lo:hi].double() for t, lo, hi in renorm_window(shape, x0, x0 + rows)]
    cat = torch.cat(parts) if parts else torch.zeros(0, dtype=torch.float64, device=zeta.device)
    s = torch.stack([cat.sum(), torch.tensor(float(cat.numel()), dtype=torch.float64,
                                             device=zeta.device)])
    if dist.is_initialized():
        dist.all_reduce(s, group=group)
    mean = s[0] / s[1]
    m2 = ((cat - mean) ** 2).sum().reshape(1)
    if dist.is_initialized():
        dist.all_reduce(m2, group=group)
    var = float(m2.item()) / (float(s[1].item()) - 1.0)
    return float(np.sqrt(acf0 / var))


def _global(group, r):
    import torch.distributed as dist
    return r if group is None else dist.get_global_rank(group, r)
