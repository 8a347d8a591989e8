"""Error statistics of the FP32 compensated path against the FP64 path.

Both surfaces come from the same seed and parameter set, so the FP64 filter
(the reference's exact summation order) is the oracle for the FP32 one.  The
statistics are computed on the device in FP64 with torch: max-abs and RMS
error of zeta, relative error of its variance and skewness, the ACF error at
small lags (relative to the FP64 variance), and the same max-abs / RMS figures
for velocity potentials.
"""
from __future__ import annotations

import itertools

import torch

DEFAULT_LAGS = tuple(itertools.product(range(3), range(3), range(3)))


def moments(z: torch.Tensor):
    """(variance, skewness) with population normalisation, in FP64."""
    x = z.double().flatten()
    d = x - x.mean()
    var = (d * d).mean()
    skew = (d * d * d).mean() / var.pow(1.5)
    return float(var), float(skew)


def acf(z: torch.Tensor, lags=DEFAULT_LAGS):
    """Direct ACF estimate sum(z(p) z(p + lag)) / count over the overlap, mean
    removed, for non-negative lags (t, x, y)."""
    zz = z.double()
    zz = zz - zz.mean()
    nt, nx, ny = zz.shape
    out = {}
    for a, b, c in lags:
        x = zz[:nt - a, :nx - b, :ny - c]
        y = zz[a:, b:, c:]
        out[(a, b, c)] = float((x * y).mean())
    return out


def field_error(ref: torch.Tensor, got: torch.Tensor):
    """max-abs error, RMS error relative to the RMS of ref, max |ref|."""
    r = ref.double()
    d = got.double() - r
    rms_ref = float(r.pow(2).mean().sqrt())
    return {"max_abs": float(d.abs().max()),
            "rms_rel": float(d.pow(2).mean().sqrt()) / max(rms_ref, 1e-300),
            "max_ref": float(r.abs().max())}


def compare_surfaces(z64: torch.Tensor, z32: torch.Tensor, lags=DEFAULT_LAGS):
    """Error of the FP32 surface against the FP64 one: field errors, relative
    variance and skewness errors, ACF errors relative to the FP64 variance."""
    out = field_error(z64, z32)
    v64, s64 = moments(z64)
    v32, s32 = moments(z32)
    a64, a32 = acf(z64, lags), acf(z32, lags)
    out.update({
        "variance_rel": abs(v32 - v64) / v64,
        "skewness_abs": abs(s32 - s64),
        "skewness_rel": abs(s32 - s64) / max(abs(s64), 1e-12),
        "acf_rel_max": max(abs(a32[k] - a64[k]) for k in lags) / a64[(0, 0, 0)],
        "variance_fp64": v64, "skewness_fp64": s64,
    })
    return out
