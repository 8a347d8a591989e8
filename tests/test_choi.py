"""Choi's order-recursive Yule-Walker solver (A3') against the reference's own
tests (src/test/yule-walker-test.cc:141-234): agreement with Gauss
elimination, automatic order determination and chopping.  The ACFs are the
test file's fixtures restated."""
import numpy as np
import pytest

import arma_b200 as A


def exponential_acf(n):
    a, b, c = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    return 0.9 ** a * 0.88 ** b * 0.95 ** c


def standing_wave_test_acf(n):
    t, x, y = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    alpha, beta = 0.06, 0.8
    acf = np.exp(-alpha * (2 * t + x + y)) * np.cos(2 * beta * t) * np.cos(beta * x) * np.cos(0 * y)
    return acf / acf[0, 0, 0]


@pytest.mark.parametrize("order,variance,tol,gen", [
    (2, 239.2780, 1e-4, exponential_acf),
    (3, 239.2780, 1e-4, exponential_acf),
    (4, 239.2780, 1e-4, exponential_acf),
    (7, 2.0, 1e-2, standing_wave_test_acf),
])
def test_compare_to_gauss_elimination(order, variance, tol, gen):
    acf = variance * gen(order + 1)
    phi, _ = A.ar_fit_choi(acf, max_order=order, determine_order=False, chop=False)
    expected, _ = A.ar_fit(acf, (order, order, order))
    assert phi.shape == expected.shape
    assert np.abs(phi - expected).max() <= tol


def test_determine_the_order():
    acf = 239.2780 * exponential_acf(11)
    phi, _ = A.ar_fit_choi(acf, determine_order=True, var_epsilon=1e-5, chop=False)
    assert phi.shape == (2, 2, 2)


def test_chop():
    acf = 239.2780 * exponential_acf(11)
    phi, _ = A.ar_fit_choi(acf, determine_order=False, chop=True)
    assert phi.shape == (2, 2, 2)


def test_real_case():
    acf = 2.0 * standing_wave_test_acf(11)
    phi, var = A.ar_fit_choi(acf, var_epsilon=1e-5)
    assert phi.shape[2] == 2
    # white-noise variance recomputed from phi as the reference does
    box = acf[:phi.shape[0], :phi.shape[1], :phi.shape[2]]
    assert var == pytest.approx(acf[0, 0, 0] - (phi * box).sum(), rel=1e-12)


def test_exact_separable_model():
    """The exponential ACF is a product of AR(1) ACFs, so the 2x2x2 model is
    exact: 1 - sum phi z^k = (1 - 0.9 z1)(1 - 0.88 z2)(1 - 0.95 z3)."""
    phi, _ = A.ar_fit_choi(239.2780 * exponential_acf(6), chop=False)
    assert phi.shape == (2, 2, 2)
    r = np.array([0.9, 0.88, 0.95])
    exp = np.zeros((2, 2, 2))
    for idx in np.ndindex(2, 2, 2):
        if idx != (0, 0, 0):
            exp[idx] = -np.prod([(-r[d]) if idx[d] else 1.0 for d in range(3)])
    assert np.abs(phi - exp).max() <= 1e-9
