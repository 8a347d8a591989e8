"""The circular auto-covariance behind the wave-group ACF generator
(``arma_auto_covariance``; arma::auto_covariance, src/arma.cc:81-100, called
by ACF_generator::generate, src/generator/acf_generator.cc:147).

The reference's own test, AutoCovariance.CosineNoDecay
(src/test/auto-covariance-test.cc:49-88), is restated here on its inputs: a
cosine wave 4 cos(2 pi (x - t)) on 21^3 points over [-4.5, 4.5] per axis.  It
checks that the FFT form equals the direct circular sum (the test's
auto_covariance_ref, :13-43) within 1e-3, and that the wave and its
exponentially decayed copy rescaled to the same variance have acf(0,0,0)
within 1e-3 of each other.  Host FP64, no GPU.
"""
import numpy as np
import pytest

import arma_b200 as A


def _variance(w):
    """Unbiased variance (gsl_stats_variance)."""
    return float(np.var(w, ddof=1))


def auto_covariance_ref(w):
    """Direct circular sum: r(i,j,k) = sum w(i1,j1,k1) w((i+i1)%n0, ...) / n."""
    n0, n1, n2 = w.shape
    out = np.empty_like(w)
    for i in range(n0):
        wi = np.roll(w, -i, axis=0)
        for j in range(n1):
            wij = np.roll(wi, -j, axis=1)
            # all k shifts at once: stack of rolls along the last axis
            idx = (np.arange(n2)[:, None] + np.arange(n2)[None, :]) % n2  # (k, k1)
            out[i, j, :] = np.einsum("abk,abqk->q", w, wij[:, :, idx]) / w.size
    return out


def cosine_waves(n=21, r=4.5):
    g = -r + 2.0 * r * np.arange(n) / (n - 1)
    xs, ys, ts = g[:, None, None], g[None, :, None], g[None, None, :]
    wave = 4.0 * np.cos(2.0 * np.pi * (xs + 0.0 * ys - ts)) * np.ones((n, n, n))
    wave_exp = np.exp(-(np.abs(xs) + np.abs(ys) + np.abs(ts))) * wave
    wave_exp *= np.sqrt(_variance(wave) / _variance(wave_exp))
    return wave, wave_exp


def test_cosine_no_decay():
    wave, wave_exp = cosine_waves()
    acf = A.auto_covariance(wave)
    acf_exp = A.auto_covariance(wave_exp)
    assert abs(acf[0, 0, 0] - acf_exp[0, 0, 0]) < 1e-3
    ref = auto_covariance_ref(wave)
    assert np.max(np.abs(acf - ref)) < 1e-3
    # and far inside the reference's tolerance: FP64 FFT against the direct sum
    assert np.max(np.abs(acf - ref)) < 1e-10 * np.max(np.abs(ref))


@pytest.mark.parametrize("shape", [(7, 11, 13), (2, 3, 5), (1, 1, 9), (16, 9, 25), (65, 2, 3),
                                   (17, 19, 4)])
def test_auto_covariance_matches_numpy_fft(shape):
    w = np.random.default_rng(sum(shape)).standard_normal(shape)
    got = A.auto_covariance(w)
    exp = np.fft.ifftn(np.abs(np.fft.fftn(w)) ** 2).real / w.size
    assert np.max(np.abs(got - exp)) < 1e-12 * np.max(np.abs(exp))
    assert got[0, 0, 0] == pytest.approx(np.sum(w * w) / w.size, rel=1e-13)


def test_auto_covariance_small_direct():
    w = np.random.default_rng(3).standard_normal((5, 4, 6))
    assert np.allclose(A.auto_covariance(w), auto_covariance_ref(w), rtol=0, atol=1e-13)


def test_auto_covariance_rejects_bad_arguments():
    lib, C = A.capi.lib(), A.capi.C
    buf = (C.c_double * 8)()
    assert lib.arma_auto_covariance(None, (C.c_int * 3)(2, 2, 2), buf) == -1
    assert lib.arma_auto_covariance(buf, (C.c_int * 3)(2, 0, 2), buf) == -1
