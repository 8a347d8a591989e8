"""CPU oracle for the ARMA wavy-surface hot path -- TEST INFRASTRUCTURE ONLY.

numpy-facing ctypes wrappers over ``oracle/_build/liboracle.so`` (built from
the C++ restatement in this directory by ``make -C oracle``).  The oracle is
the checker: only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` may import it.  The product package never does.

Parity status (see ``oracle.h``): the MT recurrence is pinned against
libstdc++'s ``std::mt19937``; the normal white noise is libstdc++'s own
``std::normal_distribution``; dsysv, Owen T and the skew-normal CDF are pinned
against the reference test-suite's known answers; the AR filter, variance
renormalisation, NIT realisation and linear velocity solver are pinned by
restatement only (the reference ships no golden vectors for them).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_u32p = C.POINTER(C.c_uint32)
_ip = C.POINTER(C.c_int)


class MtParams(C.Structure):
    """dcmt ``mt_struct`` fields in the reference's order (src/parallel_mt.hh:109-123)."""

    _fields_ = [
        ("aaa", C.c_uint32), ("mm", C.c_int32), ("nn", C.c_int32),
        ("rr", C.c_int32), ("ww", C.c_int32), ("wmask", C.c_uint32),
        ("umask", C.c_uint32), ("lmask", C.c_uint32), ("shift0", C.c_int32),
        ("shift1", C.c_int32), ("shiftB", C.c_int32), ("shiftC", C.c_int32),
        ("maskB", C.c_uint32), ("maskC", C.c_uint32), ("i", C.c_int32),
    ]

    def as_tuple(self):
        return tuple(getattr(self, f) for f, _ in self._fields_)


def build(quiet: bool = True) -> str:
    subprocess.run(["make", "-C", _HERE], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        d, i, sz, u32 = C.c_double, C.c_int, C.c_size_t, C.c_uint32
        sig = {
            "orc_acf_standing": (None, [d, d, _dp, _dp, _dp, i, i, i, _dp]),
            "orc_acf_propagating": (None, [d, d, _dp, _dp, _dp, i, i, i, _dp]),
            "orc_ac_matrix": (None, [_dp, i, i, i, i, i, i, _dp]),
            "orc_sysv_upper": (i, [i, _dp, _dp]),
            "orc_cholesky_solve": (i, [i, _dp, _dp]),
            "orc_ar_fit_gauss": (i, [_dp, i, i, i, i, i, i, i, _dp, _dp]),
            "orc_white_noise_variance": (d, [_dp, i, i, i, _dp, i, i, i]),
            "orc_mt_sgenrand": (None, [C.POINTER(MtParams), u32, _u32p]),
            "orc_mt_genrand": (None, [C.POINTER(MtParams), u32, sz, _u32p]),
            "orc_mt19937_params": (None, [C.POINTER(MtParams)]),
            "orc_std_mt19937": (None, [u32, sz, _u32p]),
            "orc_mt_file_count": (i, [C.c_char_p]),
            "orc_mt_file_read": (i, [C.c_char_p, i, C.POINTER(MtParams)]),
            "orc_mt_file_write": (i, [C.c_char_p, C.POINTER(MtParams), i, _u32p]),
            "orc_white_noise": (None, [C.POINTER(MtParams), u32, d, sz, _dp]),
            "orc_white_noise_words": (sz, [C.POINTER(MtParams), u32, sz]),
            "orc_ar_filter": (None, [_dp, i, i, i, _dp, i, i, i]),
            "orc_ma_fit": (i, [_dp, i, i, i, i, i, i, _dp, _dp, _ip]),
            "orc_ma_filter": (None, [_dp, i, i, i, _dp, i, i, i, _dp]),
            "orc_ar_filter_f32": (None, [_fp, i, i, i, _fp, i, i, i]),
            "orc_ar_generate_omp": (i, [_dp, i, i, i, _dp, i, i, i, i,
                                        C.POINTER(MtParams), i, _u32p, d, i, _ip]),
            "orc_partition_shape": (None, [_ip, _ip, i, _ip, _ip]),
            "orc_variance_renorm": (d, [_dp, i, i, i, d]),
            "orc_variance_unbiased": (d, [_dp, sz]),
            "orc_gaussian_cdf": (d, [d, d, d]),
            "orc_owen_t": (d, [d, d]),
            "orc_skew_normal_cdf": (d, [d, d, d, d]),
            "orc_gram_charlier_cdf": (d, [d, d, d]),
            "orc_nit_transform": (None, [_dp, sz, d, i, _dp, d, d, d, i, i]),
            "orc_derivative_t": (None, [_dp, i, i, i, d, i, _dp]),
            "orc_factor_waves": (None, [_dp, i, i, i, d, _dp, _dp]),
            "orc_window_function": (None, [i, i, d, d, d, d, _dp]),
            "orc_fft2": (None, [_dp, _dp, i, i, i]),
            "orc_velocity_linear": (None, [_dp, i, i, i, _dp, d, _dp, i, _ip, i, _dp, i]),
            "orc_velocity_solve": (None, [i, _dp, i, i, i, _dp, d, _dp, i, _ip, i, _dp, i]),
            "orc_write_zeta_bin": (i, [C.c_char_p, _dp, sz]),
            "orc_write_zeta_csv": (i, [C.c_char_p, _dp, i, i, i, _dp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ---------------------------------------------------------------- ACF and fit
def acf(kind: str, shape, amplitude, velocity, alpha, beta, delta=(1.0, 1.0, 1.0)):
    out = np.empty(tuple(shape), np.float64)
    a, b, dl = _f64(alpha), _f64(beta), _f64(delta)
    fn = lib().orc_acf_standing if kind == "standing_wave" else lib().orc_acf_propagating
    fn(amplitude, velocity, _d(a), _d(b), _d(dl), *shape, _d(out))
    return out


def ac_matrix(acf_arr, order):
    acf_arr = _f64(acf_arr)
    P = int(np.prod(order))
    out = np.empty((P, P), np.float64)
    lib().orc_ac_matrix(_d(acf_arr), *acf_arr.shape, *order, _d(out))
    return out


def sysv(a, b):
    a = _f64(a).copy()
    b = _f64(b).copy()
    info = lib().orc_sysv_upper(a.shape[0], _d(a), _d(b))
    if info != 0:
        raise np.linalg.LinAlgError(f"sysv info={info}")
    return b


def ar_fit(acf_arr, order, method: str = "bunch_kaufman"):
    acf_arr = _f64(acf_arr)
    phi = np.empty(tuple(order), np.float64)
    var = C.c_double()
    info = lib().orc_ar_fit_gauss(_d(acf_arr), *acf_arr.shape, *order,
                                  0 if method == "bunch_kaufman" else 1,
                                  _d(phi), C.byref(var))
    if info != 0:
        raise np.linalg.LinAlgError(f"ar fit info={info}")
    return phi, var.value


def white_noise_variance(acf_arr, phi):
    acf_arr, phi = _f64(acf_arr), _f64(phi)
    return lib().orc_white_noise_variance(_d(acf_arr), *acf_arr.shape, _d(phi), *phi.shape)


# ---------------------------------------------------------------- PRNG
def mt19937_params() -> MtParams:
    p = MtParams()
    lib().orc_mt19937_params(C.byref(p))
    return p


def mt_genrand(params: MtParams, seed: int, n: int):
    out = np.empty(n, np.uint32)
    lib().orc_mt_genrand(C.byref(params), seed, n, out.ctypes.data_as(_u32p))
    return out


def std_mt19937(seed: int, n: int):
    out = np.empty(n, np.uint32)
    lib().orc_std_mt19937(seed, n, out.ctypes.data_as(_u32p))
    return out


def mt_file_count(path: str) -> int:
    return lib().orc_mt_file_count(path.encode())


def mt_file_read(path: str, index: int) -> MtParams:
    p = MtParams()
    rc = lib().orc_mt_file_read(path.encode(), index, C.byref(p))
    if rc != 0:
        raise IOError(f"cannot read MT set {index} from {path}: {rc}")
    return p


def white_noise(params: MtParams, seed: int, stddev: float, n: int):
    out = np.empty(n, np.float64)
    lib().orc_white_noise(C.byref(params), seed, stddev, n, _d(out))
    return out


def white_noise_words(params: MtParams, seed: int, n: int) -> int:
    return lib().orc_white_noise_words(C.byref(params), seed, n)


# ---------------------------------------------------------------- AR filter
def ar_filter(zeta, phi):
    """In-place causal AR filter (returns the filtered copy)."""
    z = _f64(zeta).copy()
    phi = _f64(phi)
    lib().orc_ar_filter(_d(z), *z.shape, _d(phi), *phi.shape)
    return z


# ---------------------------------------------------------------- MA model
def ma_fit(acf_arr, order):
    """Fixed-point MA fit: (status, theta, var_wn, iterations)."""
    a = _f64(acf_arr)
    theta = np.zeros(tuple(order))
    var = C.c_double()
    it = C.c_int()
    rc = lib().orc_ma_fit(_d(a), *a.shape, *order, _d(theta), C.byref(var), C.byref(it))
    return rc, theta, var.value, it.value


def ma_filter(eps, theta):
    """Direct MA sum (src/test/convolution-test.cc:17-50)."""
    e = _f64(eps)
    th = _f64(theta)
    z = np.empty_like(e)
    lib().orc_ma_filter(_d(th), *th.shape, _d(e), *e.shape, _d(z))
    return z


def ma_block_shape(signal_shape, kernel_shape, parallelism=2):
    """Convolution::get_block_shape (src/apmath/convolution.hh:146-161) with the
    non-OpenMP parallelism of 2."""
    s = np.asarray(signal_shape)
    k = np.asarray(kernel_shape)
    g1 = np.minimum(s, 4 * k)
    g2 = np.maximum(k, s // parallelism)
    return tuple(int(v) for v in np.minimum(g1, g2) + np.abs(g1 - g2) // 2)


def ma_convolve_fft(eps, theta, parallelism=2):
    """The reference's production MA form: FFT overlap-add of the noise with K =
    -theta, K(0,0,0) = 1, blocks of Convolution::get_block_shape zero-padded by
    the kernel's shape, each block's linear convolution added back at its
    offset and truncated to the surface (src/apmath/convolution.hh:58-130,
    src/generator/ma_model.cc:42-61).  Complex FP64 numpy FFTs."""
    e = _f64(eps)
    kern = -_f64(theta).astype(np.complex128)
    kern[0, 0, 0] = 1.0
    bs = np.asarray(ma_block_shape(e.shape, kern.shape, parallelism))
    pad = np.asarray(kern.shape)
    if np.any(kern.shape > bs) or np.any(bs > np.asarray(e.shape)):
        raise ValueError("bad block size")
    full = tuple(int(v) for v in bs + pad)
    kf = np.fft.fftn(kern, full)
    lim = np.asarray(e.shape)
    nparts = -(-lim // bs)
    out = np.zeros(e.shape, np.complex128)
    for idx in np.ndindex(*nparts):
        off = np.asarray(idx) * bs
        to = np.minimum(lim, off + bs)
        part = np.zeros(full, np.complex128)
        part[tuple(slice(0, int(t - o)) for o, t in zip(off, to))] = \
            e[tuple(slice(int(o), int(t)) for o, t in zip(off, to))]
        res = np.fft.ifftn(np.fft.fftn(part) * kf)
        hi = np.minimum(to + pad, lim)
        out[tuple(slice(int(o), int(h)) for o, h in zip(off, hi))] += \
            res[tuple(slice(0, int(h - o)) for o, h in zip(off, hi))]
    return out.real


def ar_filter_f32(zeta, phi):
    z = np.ascontiguousarray(zeta, np.float32).copy()
    phi = np.ascontiguousarray(phi, np.float32)
    lib().orc_ar_filter_f32(z.ctypes.data_as(_fp), *z.shape, phi.ctypes.data_as(_fp), *phi.shape)
    return z


def ar_filter_omp(zeta, phi, nthreads=0, partition=(0, 0, 0)):
    z = _f64(zeta).copy()
    phi = _f64(phi)
    part = (C.c_int * 3)(*partition)
    rc = lib().orc_ar_generate_omp(_d(z), *z.shape, _d(phi), *phi.shape, 0, None, 0,
                                   None, 0.0, nthreads, part)
    assert rc == 0
    return z


def ar_generate_omp(shape, phi, stddev, params_list, seeds, nthreads, partition=(0, 0, 0)):
    z = np.empty(tuple(shape), np.float64)
    phi = _f64(phi)
    arr = (MtParams * len(params_list))(*params_list)
    sd = np.ascontiguousarray(seeds, np.uint32)
    part = (C.c_int * 3)(*partition)
    rc = lib().orc_ar_generate_omp(_d(z), *z.shape, _d(phi), *phi.shape, 1, arr,
                                   len(params_list), sd.ctypes.data_as(_u32p), stddev,
                                   nthreads, part)
    if rc != 0:
        raise RuntimeError("bad number of MT configs")
    return z


def partition_shape(grid, order, parallelism, user=(0, 0, 0)):
    out = (C.c_int * 3)()
    lib().orc_partition_shape((C.c_int * 3)(*grid), (C.c_int * 3)(*order), parallelism,
                              (C.c_int * 3)(*user), out)
    return tuple(out)


def variance_renorm(zeta, acf0):
    z = _f64(zeta).copy()
    s = lib().orc_variance_renorm(_d(z), *z.shape, acf0)
    return z, s


def variance_unbiased(x):
    x = _f64(x).ravel()
    return lib().orc_variance_unbiased(_d(x), x.size)


# ---------------------------------------------------------------- NIT
def gaussian_cdf(x, mean=0.0, sigma=1.0):
    return lib().orc_gaussian_cdf(x, mean, sigma)


def owen_t(h, a):
    return lib().orc_owen_t(h, a)


def skew_normal_cdf(x, mean, sigma, alpha):
    return lib().orc_skew_normal_cdf(x, mean, sigma, alpha)


def gram_charlier_cdf(x, skewness, kurtosis):
    return lib().orc_gram_charlier_cdf(x, skewness, kurtosis)


def nit_transform(data, stdev, kind, params, interval=(0.0, 1.0), eps=1e-6,
                  max_iter=100, nthreads=0):
    z = _f64(data).copy()
    p = _f64(list(params) + [0.0] * (3 - len(params)))
    lib().orc_nit_transform(_d(z), z.size, stdev, 0 if kind == "gram_charlier" else 1,
                            _d(p), interval[0], interval[1], eps, max_iter, nthreads)
    return z


# ---------------------------------------------------------------- velocity
def derivative_t(zeta, dt, idx_t):
    zeta = _f64(zeta)
    out = np.empty(zeta.shape[1:], np.float64)
    lib().orc_derivative_t(_d(zeta), *zeta.shape, dt, idx_t, _d(out))
    return out


def factor_waves(slice2d, t, dt):
    s = _f64(slice2d)
    kmin = np.empty(2)
    kmax = np.empty(2)
    lib().orc_factor_waves(_d(s), *s.shape, t, dt, _d(kmin), _d(kmax))
    return kmin, kmax


def window_function(nx, ny, wnmax, z, depth):
    out = np.empty((nx, ny), np.float64)
    lib().orc_window_function(nx, ny, wnmax[0], wnmax[1], z, depth, _d(out))
    return out


def fft2(a, sign=-1):
    a = np.asarray(a, np.complex128)
    re = np.ascontiguousarray(a.real).copy()
    im = np.ascontiguousarray(a.imag).copy()
    lib().orc_fft2(_d(re), _d(im), a.shape[0], a.shape[1], sign)
    return re + 1j * im


def velocity_linear(zeta, delta, depth, z_levels, t_idx, nthreads=0):
    zeta = _f64(zeta)
    zs = _f64(z_levels)
    ti = np.ascontiguousarray(t_idx, np.int32)
    dl = _f64(delta)
    out = np.empty((len(ti), len(zs)) + zeta.shape[1:], np.float64)
    lib().orc_velocity_linear(_d(zeta), *zeta.shape, _d(dl), depth, _d(zs), len(zs),
                              ti.ctypes.data_as(_ip), len(ti), _d(out), nthreads)
    return out


def velocity_high_amplitude(zeta, delta, depth, z_levels, t_idx, nthreads=0):
    zeta = _f64(zeta)
    zs = _f64(z_levels)
    ti = np.ascontiguousarray(t_idx, np.int32)
    dl = _f64(delta)
    out = np.empty((len(ti), len(zs)) + zeta.shape[1:], np.float64)
    lib().orc_velocity_solve(1, _d(zeta), *zeta.shape, _d(dl), depth, _d(zs), len(zs),
                             ti.ctypes.data_as(_ip), len(ti), _d(out), nthreads)
    return out


def write_zeta_bin(path, zeta):
    z = _f64(zeta)
    return lib().orc_write_zeta_bin(path.encode(), _d(z), z.size)


def write_zeta_csv(path, zeta, delta):
    z = _f64(zeta)
    dl = _f64(delta)
    return lib().orc_write_zeta_csv(path.encode(), _d(z), *z.shape, _d(dl))
