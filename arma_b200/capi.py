"""ctypes binding of the arma_b200 C ABI (``include/arma_b200.h``).

Device buffers are passed as raw pointers (``int``), e.g.
``torch.Tensor.data_ptr()``; host arrays are numpy arrays.  Every call checks
the returned status and raises :class:`ArmaError` carrying the library's
message, mirroring the reference's exceptions (``std::runtime_error``,
``std::invalid_argument``, ``PRNG_error``).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
library_path = os.path.join(_HERE, "libarma_b200.so")

FP64, FP32C = 0, 1
ACF_STANDING, ACF_PROPAGATING = 0, 1
FIT_BUNCH_KAUFMAN, FIT_CHOLESKY = 0, 1
NIT_GRAM_CHARLIER, NIT_SKEW_NORMAL = 0, 1
NIT_BISECTION, NIT_LUT = 0, 1
OUTPUT_FLAGS = ("none", "summary", "qq", "waves", "acf", "csv", "blitz", "binary", "surface")

ERRORS = {
    -1: "ARMA_EINVAL", -2: "ARMA_ECUDA", -3: "ARMA_ENOMEM", -4: "ARMA_ETIMEDOUT",
    -5: "ARMA_EIO", -6: "ARMA_EPRNG", -7: "ARMA_ENUMERIC", -8: "ARMA_ENOTSUP",
}

EXPORTS = (
    "arma_version", "arma_last_error", "arma_ctx_create", "arma_ctx_destroy",
    "arma_ctx_set_stream", "arma_ctx_synchronize", "arma_ctx_launch_count",
    "arma_ctx_transfer_bytes",
    "arma_ctx_set_profiling", "arma_ctx_profile", "arma_ctx_profile_reset",
    "arma_mt_file_count", "arma_mt_file_read", "arma_mt_file_write",
    "arma_mt19937_params", "arma_mt_genrand", "arma_acf_eval", "arma_auto_covariance",
    "arma_auto_covariance_device",
    "arma_ar_fit",
    "arma_ar_fit_analytic", "arma_white_noise", "arma_ar_filter",
    "arma_variance_renorm", "arma_nit_apply", "arma_velocity_linear",
    "arma_batch_generate", "arma_batch_generate_host", "arma_ar_filter_fp32c_noalloc",
    "arma_driver_open", "arma_driver_close", "arma_driver_generate", "arma_driver_set_output_dir",
    "arma_selftest_wait",
    "arma_driver_compute_velocity", "arma_driver_write_all", "arma_driver_info",
    "arma_driver_copy", "arma_server_config_default", "arma_server_create",
    "arma_server_destroy", "arma_stream_open", "arma_stream_close", "arma_stream_submit",
    "arma_server_poll", "arma_server_stats_get", "arma_server_last_failure",
    "arma_server_profile", "arma_velocity_linear_batch", "arma_validate_process",
    "arma_poly_roots", "arma_ar_fit_choi", "arma_driver_acf", "arma_velocity_high_amplitude",
    "arma_ma_fit", "arma_ma_filter", "arma_ma_generate", "arma_ctx_set_noise_margin",
    "arma_mt_create", "arma_mt_is_primitive", "arma_mt_equidistribution",
    "arma_batch_generate_nit", "arma_ctx_get_tuning", "arma_ctx_set_tuning", "arma_autotune",
    "arma_router_create", "arma_router_destroy", "arma_router_replicas", "arma_router_stream_open",
    "arma_router_stream_close", "arma_router_stream_submit", "arma_router_poll",
    "arma_router_placement", "arma_router_stats_get", "arma_ar_filter_strip",
)


class ArmaError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{ERRORS.get(code, code)}: {message}")
        self.code = code


class MtParams(C.Structure):
    """dcmt parameter set (``arma_mt_params``)."""

    _fields_ = [
        ("aaa", C.c_uint32), ("mm", C.c_int32), ("nn", C.c_int32),
        ("rr", C.c_int32), ("ww", C.c_int32), ("wmask", C.c_uint32),
        ("umask", C.c_uint32), ("lmask", C.c_uint32), ("shift0", C.c_int32),
        ("shift1", C.c_int32), ("shiftB", C.c_int32), ("shiftC", C.c_int32),
        ("maskB", C.c_uint32), ("maskC", C.c_uint32), ("i", C.c_int32),
    ]

    def as_tuple(self):
        return tuple(getattr(self, f) for f, _ in self._fields_)


class Surface(C.Structure):
    """One surface of a batch (``arma_surface``)."""

    _fields_ = [
        ("shape", C.c_int * 3), ("order", C.c_int * 3),
        ("phi", C.POINTER(C.c_double)), ("var_wn", C.c_double),
        ("acf0", C.c_double), ("mt", MtParams), ("seed", C.c_uint32),
        ("d_zeta", C.c_void_p), ("scale", C.c_double),
    ]


class Tuning(C.Structure):
    """``arma_tuning``: result-invariant speed settings of the batched calls."""

    _fields_ = [
        ("mt_log2_segment", C.c_int), ("ar_ctas_per_sm", C.c_int),
        ("host_groups", C.c_int), ("host_first", C.c_double),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class NitTable(C.Structure):
    """The NIT of one batch surface (``arma_nit_table``); dist < 0: none."""

    _fields_ = [
        ("dist", C.c_int), ("params", C.c_double * 3), ("stdev", C.c_double),
        ("lut_nodes", C.c_int), ("lut_range", C.c_double),
    ]


def nit_table(dist=-1, params=(0.0, 0.0, 0.0), stdev=1.0, lut_nodes=1024, lut_range=5.0):
    t = NitTable()
    t.dist = dist
    t.params = (C.c_double * 3)(*(list(params) + [0.0] * (3 - len(params))))
    t.stdev = stdev
    t.lut_nodes = lut_nodes
    t.lut_range = lut_range
    return t


class VelocityJob(C.Structure):
    """``arma_velocity_job``."""

    _fields_ = [
        ("d_zeta", C.c_void_p), ("d_out", C.c_void_p), ("nt", C.c_int),
        ("t_idx", C.POINTER(C.c_int)), ("ntd", C.c_int), ("dt", C.c_double),
    ]


class ServerConfig(C.Structure):
    """``arma_server_config``."""

    _fields_ = [
        ("chunk_slices", C.c_int), ("max_inflight", C.c_int), ("max_batch", C.c_int),
        ("max_batch_points", C.c_longlong), ("hbm_budget", C.c_size_t), ("velocity", C.c_int),
        ("depth", C.c_double), ("nz", C.c_int), ("z_levels", C.c_double * 8),
        ("noise_margin", C.c_double), ("profile", C.c_int),
    ]


class StreamSpec(C.Structure):
    """``arma_stream_spec``."""

    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("order", C.c_int * 3),
        ("phi", C.POINTER(C.c_double)), ("var_wn", C.c_double), ("acf0", C.c_double),
        ("mt", MtParams), ("seed", C.c_uint32), ("delta", C.c_double * 3),
    ]


class Completion(C.Structure):
    """``arma_completion``."""

    _fields_ = [
        ("request", C.c_uint64), ("stream", C.c_uint64), ("chunk", C.c_uint64),
        ("status", C.c_int), ("batch_size", C.c_int), ("latency_ms", C.c_double),
        ("queue_ms", C.c_double), ("device_ms", C.c_double),
    ]


class ServerStats(C.Structure):
    """``arma_server_stats``."""

    _fields_ = [
        ("submitted", C.c_uint64), ("completed", C.c_uint64), ("batches", C.c_uint64),
        ("redone", C.c_uint64), ("launches", C.c_uint64), ("points", C.c_uint64),
        ("resident_bytes", C.c_size_t), ("budget_bytes", C.c_size_t), ("streams", C.c_int),
        ("resident_streams", C.c_int), ("inflight", C.c_int), ("pending", C.c_int),
        ("launch_ms_total", C.c_double), ("launch_ms_max", C.c_double),
    ]


_lib = None


def lib():
    """Load the product library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(library_path):
            raise ImportError(
                f"{library_path} is missing: build it with `make -C arma_b200` "
                "(there is no CPU fallback)")
        L = C.CDLL(library_path)
        i, d, sz, vp = C.c_int, C.c_double, C.c_size_t, C.c_void_p
        ip, dp = C.POINTER(C.c_int), C.POINTER(C.c_double)
        mp = C.POINTER(MtParams)
        sigs = {
            "arma_version": (i, []),
            "arma_last_error": (i, [C.c_char_p, sz]),
            "arma_ctx_create": (i, [i, C.POINTER(vp)]),
            "arma_ctx_destroy": (i, [vp]),
            "arma_ctx_set_stream": (i, [vp, vp]),
            "arma_ctx_synchronize": (i, [vp]),
            "arma_ctx_launch_count": (i, [vp, C.POINTER(C.c_uint64)]),
            "arma_ctx_transfer_bytes": (i, [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
            "arma_ctx_set_profiling": (i, [vp, i]),
            "arma_ctx_profile": (i, [vp, C.c_char_p, dp, C.POINTER(C.c_uint64)]),
            "arma_ctx_profile_reset": (i, [vp]),
            "arma_mt_file_count": (i, [C.c_char_p, ip]),
            "arma_mt_file_read": (i, [C.c_char_p, i, mp]),
            "arma_mt_file_write": (i, [C.c_char_p, mp, i]),
            "arma_mt19937_params": (i, [mp]),
            "arma_mt_create": (i, [i, i, i, C.c_uint32, mp]),
            "arma_mt_is_primitive": (i, [mp, ip]),
            "arma_mt_equidistribution": (i, [mp, i, ip]),
            "arma_mt_genrand": (i, [vp, mp, C.c_uint32, C.c_uint64, sz, vp]),
            "arma_acf_eval": (i, [i, d, d, dp, dp, dp, ip, dp]),
            "arma_auto_covariance": (i, [dp, ip, dp]),
            "arma_auto_covariance_device": (i, [vp, vp, ip, i, vp]),
            "arma_ar_fit": (i, [dp, ip, ip, i, dp, dp]),
            "arma_ar_fit_analytic": (i, [i, d, d, dp, dp, dp, ip, dp, dp]),
            "arma_white_noise": (i, [vp, mp, C.c_uint32, d, sz, i, vp]),
            "arma_ar_filter": (i, [vp, dp, ip, ip, i, vp]),
            "arma_ar_filter_strip": (i, [vp, dp, ip, ip, i, i, vp]),
            "arma_variance_renorm": (i, [vp, vp, ip, i, d, dp]),
            "arma_nit_apply": (i, [vp, i, dp, d, i, dp, d, i, i, d, sz, i, vp]),
            "arma_velocity_linear": (i, [vp, vp, ip, i, dp, d, dp, i, ip, i, vp]),
            "arma_batch_generate": (i, [vp, C.POINTER(Surface), i, i]),
            "arma_batch_generate_host": (i, [vp, C.POINTER(Surface), i, i]),
            "arma_batch_generate_nit": (i, [vp, C.POINTER(Surface), i, i, C.POINTER(NitTable)]),
            "arma_ctx_get_tuning": (i, [vp, C.POINTER(Tuning)]),
            "arma_ctx_set_tuning": (i, [vp, C.POINTER(Tuning)]),
            "arma_autotune": (i, [vp, C.POINTER(Surface), i, i, i, C.POINTER(Tuning), dp]),
            "arma_ar_filter_fp32c_noalloc": (i, [vp, dp, ip, ip, vp]),
            "arma_driver_open": (i, [C.c_char_p, i, C.POINTER(vp)]),
            "arma_driver_close": (i, [vp]),
            "arma_driver_generate": (i, [vp, vp]),
            "arma_driver_set_output_dir": (i, [vp, C.c_char_p]),
            "arma_selftest_wait": (i, [vp]),
            "arma_driver_compute_velocity": (i, [vp, vp]),
            "arma_driver_write_all": (i, [vp, C.c_char_p]),
            "arma_driver_info": (i, [vp, ip, dp, ip, dp, ip, C.POINTER(C.c_uint)]),
            "arma_driver_copy": (i, [vp, i, dp]),
            "arma_server_config_default": (i, [C.POINTER(ServerConfig)]),
            "arma_server_create": (i, [i, C.POINTER(ServerConfig), C.POINTER(vp)]),
            "arma_server_destroy": (i, [vp]),
            "arma_stream_open": (i, [vp, C.POINTER(StreamSpec), C.POINTER(C.c_uint64)]),
            "arma_stream_close": (i, [vp, C.c_uint64]),
            "arma_stream_submit": (i, [vp, C.c_uint64, vp, vp, C.POINTER(C.c_uint64)]),
            "arma_server_poll": (i, [vp, C.POINTER(Completion), i, i, ip]),
            "arma_server_stats_get": (i, [vp, C.POINTER(ServerStats)]),
            "arma_server_last_failure": (i, [vp, C.c_char_p, sz]),
            "arma_server_profile": (i, [vp, C.c_char_p, dp, C.POINTER(C.c_uint64)]),
            "arma_router_create": (i, [ip, i, C.POINTER(ServerConfig), C.POINTER(vp)]),
            "arma_router_destroy": (i, [vp]),
            "arma_router_replicas": (i, [vp, ip]),
            "arma_router_stream_open": (i, [vp, C.POINTER(StreamSpec), C.POINTER(C.c_uint64)]),
            "arma_router_stream_close": (i, [vp, C.c_uint64]),
            "arma_router_stream_submit": (i, [vp, C.c_uint64, vp, vp, C.POINTER(C.c_uint64)]),
            "arma_router_poll": (i, [vp, C.POINTER(Completion), i, i, ip]),
            "arma_router_placement": (i, [vp, C.c_uint64, ip, ip]),
            "arma_router_stats_get": (i, [vp, i, C.POINTER(ServerStats)]),
            "arma_velocity_linear_batch": (i, [vp, C.POINTER(VelocityJob), i, i, i, i, d, dp, i]),
            "arma_validate_process": (i, [dp, ip, ip]),
            "arma_poly_roots": (i, [dp, i, dp, dp]),
            "arma_ar_fit_choi": (i, [dp, i, i, i, d, i, dp, ip, dp]),
            "arma_driver_acf": (i, [vp, ip, dp, dp]),
            "arma_velocity_high_amplitude": (i, [vp, vp, ip, i, dp, d, dp, i, ip, i, vp]),
            "arma_ma_fit": (i, [dp, ip, ip, dp, dp, ip]),
            "arma_ma_filter": (i, [vp, dp, ip, ip, i, vp, vp]),
            "arma_ma_generate": (i, [vp, C.POINTER(Surface), i, i]),
            "arma_ctx_set_noise_margin": (i, [vp, d]),
        }
        for name, (res, args) in sigs.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(rc: int):
    if rc != 0:
        buf = C.create_string_buffer(1024)
        lib().arma_last_error(buf, len(buf))
        raise ArmaError(rc, buf.value.decode(errors="replace"))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _i3(v):
    return (C.c_int * 3)(*[int(x) for x in v])


def _d(v):
    a = np.ascontiguousarray(v, dtype=np.float64)
    return a, _dp(a)


# ------------------------------------------------------------------ host fit
def acf_eval(kind, shape, amplitude, velocity, alpha, beta, delta=(1.0, 1.0, 1.0)):
    out = np.empty(tuple(shape), np.float64)
    a, ap = _d(alpha)
    b, bp = _d(beta)
    dl, dlp = _d(delta)
    _check(lib().arma_acf_eval(kind, amplitude, velocity, ap, bp, dlp, _i3(shape), _dp(out)))
    return out


def auto_covariance(w):
    """Circular auto-covariance of a 3-D FP64 array (arma::auto_covariance)."""
    w = np.ascontiguousarray(w, np.float64)
    out = np.empty_like(w)
    _check(lib().arma_auto_covariance(_dp(w), _i3(w.shape), _dp(out)))
    return out


def ar_fit(acf, order, method=FIT_CHOLESKY):
    acf = np.ascontiguousarray(acf, np.float64)
    phi = np.empty(tuple(order), np.float64)
    var = C.c_double()
    _check(lib().arma_ar_fit(_dp(acf), _i3(acf.shape), _i3(order), method, _dp(phi), C.byref(var)))
    return phi, var.value


def ar_fit_analytic(kind, order, amplitude, velocity, alpha, beta, delta=(1.0, 1.0, 1.0)):
    phi = np.empty(tuple(order), np.float64)
    var = C.c_double()
    a, ap = _d(alpha)
    b, bp = _d(beta)
    dl, dlp = _d(delta)
    _check(lib().arma_ar_fit_analytic(kind, amplitude, velocity, ap, bp, dlp, _i3(order),
                                      _dp(phi), C.byref(var)))
    return phi, var.value


def ar_fit_choi(acf, max_order=None, determine_order=True, var_epsilon=1e-6, chop=True):
    """Choi's order-recursive solver on a cubic ACF: (phi, var_wn)."""
    acf = np.ascontiguousarray(acf, np.float64)
    n = acf.shape[0]
    if acf.shape != (n, n, n):
        raise ValueError("ACF is not square")
    mo = min(n - 1, max_order if max_order else n - 1)
    buf = np.zeros(mo ** 3)
    order = (C.c_int * 3)()
    var = C.c_double()
    _check(lib().arma_ar_fit_choi(_dp(acf), n, mo, 1 if determine_order else 0, var_epsilon,
                                  1 if chop else 0, _dp(buf), order, C.byref(var)))
    shape = tuple(order)
    return buf[:int(np.prod(shape))].reshape(shape).copy(), var.value


def ma_fit(acf, order):
    """MA coefficients by fixed-point iteration: (theta, var_wn, iterations),
    theta of shape `order` with theta[0, 0, 0] = -1."""
    acf = np.ascontiguousarray(acf, np.float64)
    theta = np.zeros(tuple(order))
    var = C.c_double()
    it = C.c_int()
    _check(lib().arma_ma_fit(_dp(acf), _i3(acf.shape), _i3(order), _dp(theta), C.byref(var),
                             C.byref(it)))
    return theta, var.value, it.value


def validate_process(phi) -> int:
    """Raises ArmaError (ARMA_EINVAL) when the flattened AR polynomial has roots
    inside or on the unit circle; returns the number of such roots (0)."""
    phi = np.ascontiguousarray(phi, np.float64)
    bad = C.c_int()
    rc = lib().arma_validate_process(_dp(phi), _i3(phi.shape), C.byref(bad))
    if rc != 0:
        err = C.create_string_buffer(1024)
        lib().arma_last_error(err, len(err))
        e = ArmaError(rc, err.value.decode(errors="replace"))
        e.bad_roots = bad.value
        raise e
    return bad.value


def poly_roots(c):
    """Complex roots of c[0] + c[1] x + ... + c[n-1] x^(n-1)."""
    c = np.ascontiguousarray(c, np.float64)
    re = np.empty(len(c) - 1)
    im = np.empty(len(c) - 1)
    _check(lib().arma_poly_roots(_dp(c), len(c), _dp(re), _dp(im)))
    return re + 1j * im


def mt19937_params() -> MtParams:
    p = MtParams()
    _check(lib().arma_mt19937_params(C.byref(p)))
    return p


def mt_create(p: int, id: int, seed: int, w: int = 32) -> MtParams:
    """dcmt parameter set of generator `id` with period 2^p - 1
    (``arma_mt_create``)."""
    out = MtParams()
    _check(lib().arma_mt_create(w, p, id, C.c_uint32(seed & 0xffffffff), C.byref(out)))
    return out


def mt_is_primitive(params: MtParams) -> bool:
    r = C.c_int()
    _check(lib().arma_mt_is_primitive(C.byref(params), C.byref(r)))
    return bool(r.value)


def mt_equidistribution(params: MtParams, vmax: int = 32):
    """[k(1), ..., k(vmax)] of the tempered output (``arma_mt_equidistribution``)."""
    k = (C.c_int * vmax)()
    _check(lib().arma_mt_equidistribution(C.byref(params), vmax, k))
    return list(k)


def mt_file_count(path: str) -> int:
    n = C.c_int()
    _check(lib().arma_mt_file_count(path.encode(), C.byref(n)))
    return n.value


def mt_file_read(path: str, index: int) -> MtParams:
    p = MtParams()
    _check(lib().arma_mt_file_read(path.encode(), index, C.byref(p)))
    return p


def mt_file_write(path: str, sets) -> None:
    arr = (MtParams * len(sets))(*sets)
    _check(lib().arma_mt_file_write(path.encode(), arr, len(sets)))


# ------------------------------------------------------------------ device
class Context:
    """An ``arma_ctx`` bound to one CUDA device."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(lib().arma_ctx_create(device, C.byref(h)))
        self._h = h

    def close(self):
        if self._h:
            lib().arma_ctx_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream_ptr: int):
        _check(lib().arma_ctx_set_stream(self._h, C.c_void_p(stream_ptr)))

    def synchronize(self):
        _check(lib().arma_ctx_synchronize(self._h))

    def launch_count(self) -> int:
        n = C.c_uint64()
        _check(lib().arma_ctx_launch_count(self._h, C.byref(n)))
        return n.value

    def transfer_bytes(self):
        """(host->device, device->host) bytes copied by this context's calls."""
        a, b = C.c_uint64(), C.c_uint64()
        _check(lib().arma_ctx_transfer_bytes(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def set_profiling(self, on: bool = True):
        _check(lib().arma_ctx_set_profiling(self._h, 1 if on else 0))

    def profile(self, name: str):
        """(milliseconds, launches) accumulated for one kernel class."""
        ms = C.c_double()
        n = C.c_uint64()
        _check(lib().arma_ctx_profile(self._h, name.encode(), C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def set_noise_margin(self, margin: float):
        """Polar-attempt estimate multiplier of the batched calls (default 1)."""
        _check(lib().arma_ctx_set_noise_margin(self._h, float(margin)))

    def profile_reset(self):
        _check(lib().arma_ctx_profile_reset(self._h))

    def mt_genrand(self, params: MtParams, seed: int, n: int, d_out: int, offset: int = 0):
        _check(lib().arma_mt_genrand(self._h, C.byref(params), seed, offset, n, C.c_void_p(d_out)))

    def white_noise(self, params: MtParams, seed: int, stddev: float, n: int, precision: int,
                    d_out: int):
        _check(lib().arma_white_noise(self._h, C.byref(params), seed, stddev, n, precision,
                                      C.c_void_p(d_out)))

    def ar_filter(self, phi, shape, precision: int, d_zeta: int):
        phi = np.ascontiguousarray(phi, np.float64)
        _check(lib().arma_ar_filter(self._h, _dp(phi), _i3(phi.shape), _i3(shape), precision,
                                    C.c_void_p(d_zeta)))

    def ar_filter_strip(self, phi, shape, t0: int, given_rows: int, d_zeta: int):
        """FP32 filter of one x-strip: rows [0, given_rows) and slices [0, t0)
        of the (nt, nx, ny) float32 buffer are given, the rest holds noise."""
        phi = np.ascontiguousarray(phi, np.float64)
        _check(lib().arma_ar_filter_strip(self._h, _dp(phi), _i3(phi.shape), _i3(shape), t0,
                                          given_rows, C.c_void_p(d_zeta)))

    def variance_renorm(self, d_zeta: int, shape, precision: int, acf0: float) -> float:
        s = C.c_double()
        _check(lib().arma_variance_renorm(self._h, C.c_void_p(d_zeta), _i3(shape), precision,
                                          acf0, C.byref(s)))
        return s.value

    def nit_apply(self, dist: int, params, stdev: float, method: int, n: int, precision: int,
                  d_zeta: int, interval=(0.0, 1.0), eps=1e-6, max_iter=100, lut_nodes=1024,
                  lut_range=5.0):
        p, pp = _d(list(params) + [0.0] * (3 - len(params)))
        iv, ivp = _d(interval)
        _check(lib().arma_nit_apply(self._h, dist, pp, stdev, method, ivp, eps, max_iter,
                                    lut_nodes, lut_range, n, precision, C.c_void_p(d_zeta)))

    def velocity_linear(self, d_zeta: int, shape, precision: int, delta, depth: float,
                        z_levels, t_idx, d_out: int, high_amplitude: bool = False):
        dl, dlp = _d(delta)
        zs, zsp = _d(z_levels)
        ti = np.ascontiguousarray(t_idx, np.int32)
        fn = lib().arma_velocity_high_amplitude if high_amplitude else lib().arma_velocity_linear
        _check(fn(self._h, C.c_void_p(d_zeta), _i3(shape), precision, dlp, depth, zsp, len(zs),
                  ti.ctypes.data_as(C.POINTER(C.c_int)), len(ti), C.c_void_p(d_out)))

    def velocity_linear_batch(self, jobs, nx: int, ny: int, precision: int, depth: float,
                              z_levels):
        """jobs: (d_zeta, d_out, nt, t_idx, dt) per surface of slice shape nx x ny."""
        arr = (VelocityJob * len(jobs))()
        keep = []
        for k, (dz, do, nt, tidx, dt) in enumerate(jobs):
            ti = np.ascontiguousarray(tidx, np.int32)
            keep.append(ti)
            arr[k] = VelocityJob(C.c_void_p(dz), C.c_void_p(do), int(nt),
                                 ti.ctypes.data_as(C.POINTER(C.c_int)), len(ti), float(dt))
        zs, zsp = _d(z_levels)
        _check(lib().arma_velocity_linear_batch(self._h, arr, len(jobs), nx, ny, precision, depth,
                                                zsp, len(zs)))

    def selftest_wait(self):
        """The filter's bounded wait on a flag nothing sets: raises ArmaError
        (ARMA_ETIMEDOUT) after about a second; the context stays usable."""
        _check(lib().arma_selftest_wait(self._h))

    def auto_covariance(self, d_in: int, shape, precision: int, d_out: int):
        """Circular auto-covariance of a device array into FP64 device memory."""
        _check(lib().arma_auto_covariance_device(self._h, C.c_void_p(d_in), _i3(shape), precision,
                                                 C.c_void_p(d_out)))

    def ma_filter(self, theta, shape, precision: int, d_eps: int, d_zeta: int):
        """zeta = eps - sum_{m != 0} theta(m) eps(n - m) on device buffers."""
        theta = np.ascontiguousarray(theta, np.float64)
        _check(lib().arma_ma_filter(self._h, _dp(theta), _i3(theta.shape), _i3(shape), precision,
                                    C.c_void_p(d_eps), C.c_void_p(d_zeta)))

    def ma_generate(self, surfaces, precision: int):
        """Noise + MA filter + renormalisation; each surface's phi holds theta."""
        arr = (Surface * len(surfaces))(*surfaces)
        _check(lib().arma_ma_generate(self._h, arr, len(surfaces), precision))
        for k, s in enumerate(surfaces):
            s.scale = arr[k].scale
        return [arr[k].scale for k in range(len(surfaces))]

    def batch_generate(self, surfaces, precision: int, host: bool = False):
        arr = (Surface * len(surfaces))(*surfaces)
        fn = lib().arma_batch_generate_host if host else lib().arma_batch_generate
        _check(fn(self._h, arr, len(surfaces), precision))
        for k, s in enumerate(surfaces):
            s.scale = arr[k].scale
        return [arr[k].scale for k in range(len(surfaces))]

    def tuning(self) -> "Tuning":
        t = Tuning()
        _check(lib().arma_ctx_get_tuning(self._h, C.byref(t)))
        return t

    def set_tuning(self, t: "Tuning") -> None:
        _check(lib().arma_ctx_set_tuning(self._h, C.byref(t)))

    def autotune(self, surfaces, precision: int, host: bool = False):
        """``arma_autotune``: (chosen Tuning, ms per call or -1 when cached)."""
        arr = (Surface * len(surfaces))(*surfaces)
        t = Tuning()
        ms = C.c_double()
        _check(lib().arma_autotune(self._h, arr, len(surfaces), precision, int(host), C.byref(t),
                                   C.byref(ms)))
        return t, ms.value

    def batch_generate_nit(self, surfaces, precision: int, tables):
        """``arma_batch_generate_nit``: tables[k] from :func:`nit_table`."""
        arr = (Surface * len(surfaces))(*surfaces)
        tab = (NitTable * len(surfaces))(*tables)
        _check(lib().arma_batch_generate_nit(self._h, arr, len(surfaces), precision, tab))
        for k, s in enumerate(surfaces):
            s.scale = arr[k].scale
        return [arr[k].scale for k in range(len(surfaces))]


def ar_filter_fp32c_noalloc(stream_ptr: int, phi, shape, d_zeta: int):
    """Allocation-free FP32 AR filter of one surface on `stream_ptr` (0 = the
    default stream); see ``arma_ar_filter_fp32c_noalloc`` in the header."""
    phi = np.ascontiguousarray(phi, np.float64)
    _check(lib().arma_ar_filter_fp32c_noalloc(C.c_void_p(stream_ptr), _dp(phi), _i3(phi.shape),
                                              _i3(shape), C.c_void_p(d_zeta)))


def make_surface(shape, phi, var_wn, acf0, mt: MtParams, seed: int, buf_ptr: int) -> Surface:
    """Build an ``arma_surface``; keeps a reference to phi on the struct."""
    phi = np.ascontiguousarray(phi, np.float64)
    s = Surface()
    s.shape = (C.c_int * 3)(*shape)
    s.order = (C.c_int * 3)(*phi.shape)
    s.phi = _dp(phi)
    s._phi_ref = phi  # keep alive
    s.var_wn = var_wn
    s.acf0 = acf0
    s.mt = mt
    s.seed = seed
    s.d_zeta = buf_ptr
    s.scale = 0.0
    return s


class Driver:
    """An ``arma_driver``: a parsed ``.arma`` programme (the reference's
    ARMA_driver) -- ``generate_wavy_surface``, ``compute_velocity_potentials``
    and ``write_all`` run through the library."""

    def __init__(self, config: str, is_path: bool = False):
        h = C.c_void_p()
        _check(lib().arma_driver_open(config.encode(), 1 if is_path else 0, C.byref(h)))
        self._h = h

    @classmethod
    def open(cls, path: str) -> "Driver":
        return cls(path, is_path=True)

    def close(self):
        if self._h:
            lib().arma_driver_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        shape, order, vs = (C.c_int * 3)(), (C.c_int * 3)(), (C.c_int * 4)()
        delta = (C.c_double * 3)()
        var = C.c_double()
        fl = C.c_uint()
        _check(lib().arma_driver_info(self._h, shape, delta, order, C.byref(var), vs,
                                      C.byref(fl)))
        return {"shape": tuple(shape), "delta": tuple(delta), "order": tuple(order),
                "var_wn": var.value, "velocity_shape": tuple(vs),
                "output": [n for k, n in enumerate(OUTPUT_FLAGS) if fl.value >> k & 1]}

    def set_output_dir(self, directory: str):
        """Where zeta.bin goes when it is streamed during generation."""
        _check(lib().arma_driver_set_output_dir(self._h, directory.encode()))

    def generate_wavy_surface(self, ctx: Context):
        _check(lib().arma_driver_generate(ctx.handle, self._h))

    def compute_velocity_potentials(self, ctx: Context):
        _check(lib().arma_driver_compute_velocity(ctx.handle, self._h))

    def write_all(self, directory: str = ""):
        _check(lib().arma_driver_write_all(self._h, directory.encode()))

    def _copy(self, what: int, shape) -> np.ndarray:
        out = np.empty(tuple(shape), np.float64)
        _check(lib().arma_driver_copy(self._h, what, _dp(out)))
        return out

    def acf(self):
        """(ACF table, grid step) of the model."""
        shape, delta = (C.c_int * 3)(), (C.c_double * 3)()
        _check(lib().arma_driver_acf(self._h, shape, delta, None))
        out = np.empty(tuple(shape), np.float64)
        _check(lib().arma_driver_acf(self._h, shape, delta, _dp(out)))
        return out, tuple(delta)

    def zeta(self) -> np.ndarray:
        return self._copy(0, self.info()["shape"])

    def phi(self) -> np.ndarray:
        return self._copy(1, self.info()["order"])

    def velocity_potentials(self) -> np.ndarray:
        return self._copy(2, self.info()["velocity_shape"])


def server_config(**kw) -> ServerConfig:
    """Defaults of ``arma_server_config_default`` with keyword overrides
    (``z_levels`` as a sequence sets ``nz`` too)."""
    cfg = ServerConfig()
    _check(lib().arma_server_config_default(C.byref(cfg)))
    for k, v in kw.items():
        if k == "z_levels":
            cfg.nz = len(v)
            for j, z in enumerate(v):
                cfg.z_levels[j] = z
        else:
            setattr(cfg, k, v)
    return cfg


def _stream_spec(nx, ny, phi, var_wn, acf0, mt, seed, delta) -> StreamSpec:
    """``arma_stream_spec`` over `phi` (a float64 C-contiguous array the caller
    keeps alive for the call)."""
    spec = StreamSpec()
    spec.nx, spec.ny = int(nx), int(ny)
    spec.order = (C.c_int * 3)(*phi.shape)
    spec.phi = _dp(phi)
    spec.var_wn = var_wn
    spec.acf0 = acf0
    spec.mt = mt
    spec.seed = seed
    spec.delta = (C.c_double * 3)(*delta)
    return spec


def _completions(buf, n, keep) -> list:
    out = []
    for k in range(n):
        c = buf[k]
        keep.pop(c.request, None)
        out.append({"request": c.request, "stream": c.stream, "chunk": c.chunk,
                    "status": c.status, "batch_size": c.batch_size,
                    "latency_ms": c.latency_ms, "queue_ms": c.queue_ms,
                    "device_ms": c.device_ms})
    return out


class _Requests:
    """Handle life cycle and waiting shared by ``Server`` and ``Router``."""

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def wait(self, count: int, timeout_ms: int = 60000):
        """Poll until `count` completions arrived (raises on timeout)."""
        import time
        got = []
        deadline = time.monotonic() + timeout_ms / 1000.0
        while len(got) < count:
            left = int((deadline - time.monotonic()) * 1000)
            if left <= 0:
                raise TimeoutError(f"{len(got)} of {count} completions")
            got += self.poll(256, min(left, 1000))
        return got


class Server(_Requests):
    """An ``arma_server``: device-resident surface streams served in chunks
    with continuous batching."""

    def __init__(self, device: int = 0, config: ServerConfig | None = None, **kw):
        self.config = config if config is not None else server_config(**kw)
        h = C.c_void_p()
        _check(lib().arma_server_create(device, C.byref(self.config), C.byref(h)))
        self._h = h
        self._keep = {}

    def close(self):
        if self._h:
            _check(lib().arma_server_destroy(self._h))
            self._h = None
            self._keep.clear()

    def open_stream(self, nx, ny, phi, var_wn, acf0, mt: MtParams, seed: int,
                    delta=(1.0, 1.0, 1.0)) -> int:
        phi = np.ascontiguousarray(phi, np.float64)
        spec = _stream_spec(nx, ny, phi, var_wn, acf0, mt, seed, delta)
        sid = C.c_uint64()
        _check(lib().arma_stream_open(self._h, C.byref(spec), C.byref(sid)))
        return sid.value

    def close_stream(self, sid: int):
        _check(lib().arma_stream_close(self._h, sid))

    def submit(self, sid: int, zeta_ptr: int, velocity_ptr: int = 0, keep=None) -> int:
        """Queue the next chunk; the pointers must stay valid until completion
        (``keep`` holds Python references until then)."""
        rid = C.c_uint64()
        _check(lib().arma_stream_submit(self._h, sid, C.c_void_p(zeta_ptr),
                                        C.c_void_p(velocity_ptr or None), C.byref(rid)))
        if keep is not None:
            self._keep[rid.value] = keep
        return rid.value

    def poll(self, max_n: int = 256, timeout_ms: int = 0):
        buf = (Completion * max_n)()
        n = C.c_int()
        _check(lib().arma_server_poll(self._h, buf, max_n, timeout_ms, C.byref(n)))
        return _completions(buf, n.value, self._keep)

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().arma_server_stats_get(self._h, C.byref(st)))
        return {f: getattr(st, f) for f, _ in st._fields_}

    def profile(self, name: str):
        """(milliseconds, scopes) of one kernel class when profiling is on."""
        ms = C.c_double()
        n = C.c_uint64()
        _check(lib().arma_server_profile(self._h, name.encode(), C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def last_failure(self) -> str:
        buf = C.create_string_buffer(1024)
        lib().arma_server_last_failure(self._h, buf, len(buf))
        return buf.value.decode(errors="replace")


class Router(_Requests):
    """An ``arma_router``: one serving replica per listed device (a device may
    be listed more than once).  A stream is placed on the replica with the
    least stream state and stays there; its ids carry the replica index in
    their top 8 bits.  Outputs of a stream must be memory of its replica's
    device or page-locked host memory."""

    def __init__(self, devices=(0,), config: ServerConfig | None = None, **kw):
        self.config = config if config is not None else server_config(**kw)
        devs = (C.c_int * len(devices))(*devices)
        h = C.c_void_p()
        _check(lib().arma_router_create(devs, len(devices), C.byref(self.config), C.byref(h)))
        self._h = h
        self._keep = {}

    def close(self):
        if self._h:
            _check(lib().arma_router_destroy(self._h))
            self._h = None
            self._keep.clear()

    def replicas(self) -> int:
        n = C.c_int()
        _check(lib().arma_router_replicas(self._h, C.byref(n)))
        return n.value

    def open_stream(self, nx, ny, phi, var_wn, acf0, mt: MtParams, seed: int,
                    delta=(1.0, 1.0, 1.0)) -> int:
        phi = np.ascontiguousarray(phi, np.float64)
        spec = _stream_spec(nx, ny, phi, var_wn, acf0, mt, seed, delta)
        sid = C.c_uint64()
        _check(lib().arma_router_stream_open(self._h, C.byref(spec), C.byref(sid)))
        return sid.value

    def close_stream(self, sid: int):
        _check(lib().arma_router_stream_close(self._h, sid))

    def submit(self, sid: int, zeta_ptr: int, velocity_ptr: int = 0, keep=None) -> int:
        rid = C.c_uint64()
        _check(lib().arma_router_stream_submit(self._h, sid, C.c_void_p(zeta_ptr),
                                               C.c_void_p(velocity_ptr or None), C.byref(rid)))
        if keep is not None:
            self._keep[rid.value] = keep
        return rid.value

    def poll(self, max_n: int = 256, timeout_ms: int = 0):
        buf = (Completion * max_n)()
        n = C.c_int()
        _check(lib().arma_router_poll(self._h, buf, max_n, timeout_ms, C.byref(n)))
        return _completions(buf, n.value, self._keep)

    def placement(self, sid: int):
        """(replica index, device) of a stream."""
        rep, dev = C.c_int(), C.c_int()
        _check(lib().arma_router_placement(self._h, sid, C.byref(rep), C.byref(dev)))
        return rep.value, dev.value

    def stats(self, replica: int = 0) -> dict:
        st = ServerStats()
        _check(lib().arma_router_stats_get(self._h, replica, C.byref(st)))
        return {f: getattr(st, f) for f, _ in st._fields_}
