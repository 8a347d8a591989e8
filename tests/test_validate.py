"""A5 validate_process (src/arma.cc:14-70) on CPU: the root finder against
numpy's companion-matrix eigenvalues, and the stationarity verdict on the
flattened AR polynomial 1 - sum_k phi_k x^k."""
import numpy as np
import pytest

import arma_b200 as A


def sorted_roots(r):
    return np.array(sorted(r, key=lambda z: (round(abs(z), 9), round(np.angle(z), 9))))


@pytest.mark.parametrize("n,seed", [(2, 0), (3, 1), (5, 2), (12, 3), (40, 4), (125, 5)])
def test_roots_match_numpy(n, seed):
    c = np.random.default_rng(seed).normal(size=n)
    got = A.poly_roots(c)
    ref = np.roots(c[::-1])  # numpy takes the highest power first
    # residual check (any ordering) and modulus agreement
    for z in got:
        assert abs(np.polyval(c[::-1], z)) <= 1e-8 * np.abs(c).sum() * max(1.0, abs(z)) ** (n - 1)
    assert np.allclose(np.sort(np.abs(got)), np.sort(np.abs(ref)), rtol=1e-7, atol=1e-9)


def test_known_roots():
    # (x - 2)(x + 3)(x - 0.5) = x^3 + 0.5x^2 - 6.5x + 3 -> c = [3, -6.5, 0.5, 1]
    got = sorted_roots(A.poly_roots([3.0, -6.5, 0.5, 1.0]))
    assert np.allclose(sorted(got.real), [-3.0, 0.5, 2.0]) and np.allclose(got.imag, 0)
    # x^2 + 1: roots +-i
    got = A.poly_roots([1.0, 0.0, 1.0])
    assert np.allclose(sorted(got.imag), [-1.0, 1.0]) and np.allclose(got.real, 0)


def test_leading_zero_rejected():
    with pytest.raises(A.ArmaError) as e:
        A.poly_roots([1.0, 2.0, 0.0])
    assert e.value.code == -7 and "leading term" in str(e.value)


def test_stationary_and_not():
    # phi with a single lag: 1 - 0.5 x -> root 2 (stationary)
    phi = np.zeros((2, 1, 1))
    phi[1, 0, 0] = 0.5
    assert A.validate_process(phi) == 0
    phi[1, 0, 0] = 2.0  # root 0.5: inside the unit circle
    with pytest.raises(A.ArmaError) as e:
        A.validate_process(phi)
    assert e.value.code == -1 and "not stationary" in str(e.value) and e.value.bad_roots == 1


def test_validate_matches_numpy_on_fitted_models():
    for kind, args in [(A.ACF_STANDING, (1.5, 0.8, [0.05] * 3, [0.5, 0.5])),
                       (A.ACF_PROPAGATING, (1.0, 0.6, [0.04] * 3, [0.3, 0.2]))]:
        for order in [(2, 2, 2), (3, 3, 3), (4, 3, 2)]:
            phi, _ = A.ar_fit_analytic(kind, order, *args)
            c = -phi.ravel().copy()
            c[0] = 1.0
            bad = int((np.abs(np.roots(c[::-1])) <= 1.0).sum())
            if bad:
                with pytest.raises(A.ArmaError) as e:
                    A.validate_process(phi)
                assert e.value.bad_roots == bad
            else:
                assert A.validate_process(phi) == 0
