"""arma_b200: B200 implementation of the ARMA wavy-surface hot path.

The product is the shared library ``libarma_b200.so`` (sm_100a CUDA kernels
behind the C ABI declared in ``include/arma_b200.h``).  This package is a thin
ctypes binding over that ABI for Python callers and tests; it never falls back
to a CPU implementation -- if the library is missing, importing
:mod:`arma_b200.capi` raises.
"""
from .capi import (  # noqa: F401
    ArmaError, Context, Driver, MtParams, NitTable, Router, Server, server_config, Surface, Tuning,
    lib,
    library_path, nit_table,
    FP64, FP32C, ACF_STANDING, ACF_PROPAGATING,
    NIT_GRAM_CHARLIER, NIT_SKEW_NORMAL, NIT_BISECTION, NIT_LUT,
    acf_eval, auto_covariance, ar_fit, ar_fit_analytic, ar_fit_choi, ma_fit, mt19937_params, mt_create,
    mt_equidistribution, mt_file_count, mt_file_read, mt_file_write, mt_is_primitive, poly_roots,
    validate_process,
)
