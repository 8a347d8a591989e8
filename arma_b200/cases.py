"""Single-workload runners for timing and profiling one stage in isolation:

    python -m arma_b200.cases velocity --side 128 --slices 400 --nz 4 [--fp64]
    python -m arma_b200.cases ar --side 256 --slices 256 --order 8 [--surfaces 8]
    python -m arma_b200.cases ma --side 256 --slices 256 --order 20,10,10 [--fp64]

`velocity` generates one propagating-wave surface (order 10^3, FP32
compensated) of `slices` x side x side and times the linear velocity solver
on every slice at nz depth levels in {0, -1, -2, -4, ...}, infinite depth.
`ar` times the batched FP32 AR path on `surfaces` standing-wave surfaces of
the given shape and order.  `ma` times the MA filter (zeta = eps - theta * eps)
of one surface on unit normal noise with random coefficients of the given
order.  Each prints one line with the per-call device
time (CUDA events, three warm-up calls, five timed calls).
"""
from __future__ import annotations

import argparse

import numpy as np


def _timed(ctx, stream, fn, warm=3, reps=5):
    import torch
    for _ in range(warm):
        fn()
    ctx.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def velocity_case(args):
    import torch
    import arma_b200 as A
    from arma_b200 import capi
    ctx = A.Context(0)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    shape = (args.slices, args.side, args.side)
    phi, var = A.ar_fit_analytic(A.ACF_PROPAGATING, (10, 10, 10), 1.0, 0.6, [0.04] * 3, [0.3, 0.2])
    prec, dt = (A.FP64, torch.float64) if args.fp64 else (A.FP32C, torch.float32)
    z = torch.empty(shape, dtype=dt, device="cuda")
    ctx.batch_generate([capi.make_surface(shape, phi, var, 1.0, A.mt19937_params(), 42,
                                          z.data_ptr())], prec)
    zs = [0.0, -1.0, -2.0, -4.0, -8.0, -16.0, -32.0, -64.0][:args.nz]
    out = torch.empty((args.slices, args.nz, args.side, args.side), dtype=dt, device="cuda")
    tidx = list(range(args.slices))
    ms = _timed(ctx, stream, lambda: ctx.velocity_linear(z.data_ptr(), shape, prec, (1.0, 1.0, 1.0),
                                                         float("inf"), zs, tidx, out.data_ptr()))
    pts = args.slices * args.side * args.side
    print(f"velocity {args.slices}x{args.side}x{args.side} nz={args.nz} "
          f"{'fp64' if args.fp64 else 'fp32'}: {ms:.3f} ms/call, {pts / ms / 1e6:.2f} G points/s")
    ctx.close()


def ar_case(args):
    import torch
    import arma_b200 as A
    from arma_b200 import capi
    ctx = A.Context(0)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    shape = (args.slices, args.side, args.side)
    order = (args.order,) * 3
    phi, var = A.ar_fit_analytic(A.ACF_STANDING, order, 1.5, 0.8, [0.05] * 3, [0.5, 0.5])
    bufs = [torch.empty(shape, dtype=torch.float32, device="cuda") for _ in range(args.surfaces)]
    surfs = [capi.make_surface(shape, phi, var, 1.5, A.mt19937_params(), 42 + k, b.data_ptr())
             for k, b in enumerate(bufs)]
    ms = _timed(ctx, stream, lambda: ctx.batch_generate(surfs, A.FP32C))
    pts = args.surfaces * int(np.prod(shape))
    flop = pts * 2.0 * (np.prod(order) - 1)
    print(f"ar {args.surfaces} x {shape} order {order}: {ms:.3f} ms/call, "
          f"{pts / ms / 1e6:.2f} G points/s, {flop / ms / 1e9:.2f} TFLOP/s algorithmic")
    ctx.close()


def ma_case(args):
    import torch
    import arma_b200 as A
    ctx = A.Context(0)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    shape = (args.slices, args.side, args.side)
    order = tuple(int(v) for v in args.order.split(","))
    rng = np.random.default_rng(1)
    theta = rng.normal(0.0, 0.2 / np.sqrt(np.prod(order)), order)
    prec, dt = (A.FP64, torch.float64) if args.fp64 else (A.FP32C, torch.float32)
    eps = torch.randn(shape, dtype=dt, device="cuda")
    z = torch.empty_like(eps)
    ms = _timed(ctx, stream, lambda: ctx.ma_filter(theta, shape, prec, eps.data_ptr(), z.data_ptr()))
    pts = int(np.prod(shape))
    flop = pts * 2.0 * int(np.prod(order))
    print(f"ma {shape} order {order} {'fp64' if args.fp64 else 'fp32'}: {ms:.3f} ms/call, "
          f"{pts / ms / 1e6:.2f} G points/s, {flop / ms / 1e9:.2f} TFLOP/s algorithmic")
    ctx.close()


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m arma_b200.cases")
    sub = ap.add_subparsers(dest="case", required=True)
    v = sub.add_parser("velocity")
    v.add_argument("--side", type=int, default=128)
    v.add_argument("--slices", type=int, default=400)
    v.add_argument("--nz", type=int, default=4)
    v.add_argument("--fp64", action="store_true")
    a = sub.add_parser("ar")
    a.add_argument("--side", type=int, default=256)
    a.add_argument("--slices", type=int, default=256)
    a.add_argument("--order", type=int, default=8)
    a.add_argument("--surfaces", type=int, default=8)
    m = sub.add_parser("ma")
    m.add_argument("--side", type=int, default=256)
    m.add_argument("--slices", type=int, default=256)
    m.add_argument("--order", default="20,10,10")
    m.add_argument("--fp64", action="store_true")
    args = ap.parse_args(argv)
    {"velocity": velocity_case, "ar": ar_case, "ma": ma_case}[args.case](args)


if __name__ == "__main__":
    main()
