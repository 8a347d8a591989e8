"""The moving-average model on CPU: the fixed-point fit, the oracle's two MA
forms and the `.arma` grammar of `model = MA`.

The fit restates MA_coefficient_solver::solve_fixed_point_iteration
(src/generator/ma_coefficient_solver.cc:36-139); the reference's own solver
test runs it on a 10^3 propagating-wave ACF (amplitude 1, alpha (1,1,1), beta
(0.4,0.4), velocity 0.6, unit steps, no absolute values) at order 5^3
(src/test/ma-coefficient-solver-test.cc:15-42) and passes when it does not
throw.  The reference's convolution test checks its FFT overlap-add MA form
against the direct sum on a 400x8x8 signal and an 8^3 kernel drawn from
normal(0, sqrt 2), max error 1e-4 (src/test/convolution-test.cc:205-241).
Nothing here launches a kernel.
"""
import numpy as np
import pytest

import arma_b200 as A
import oracle as O


def solver_test_acf(shape=(10, 10, 10)):
    i, j, k = np.meshgrid(*(np.arange(n) for n in shape), indexing="ij")
    return np.exp(-(i + j + k)) * np.cos(0.6 * i + 0.4 * j + 0.4 * k)


def lag_products(theta):
    """sum_l theta(ijk + l) theta(l) for every ijk (the fit's right-hand side)."""
    o = theta.shape
    out = np.zeros(o)
    for i in range(o[0]):
        for j in range(o[1]):
            for k in range(o[2]):
                out[i, j, k] = np.sum(theta[i:, j:, k:] * theta[:o[0] - i, :o[1] - j, :o[2] - k])
    return out


def test_reference_solver_case_runs_and_matches_oracle():
    acf = solver_test_acf()
    rc, th_o, var_o, it_o = O.ma_fit(acf, (5, 5, 5))
    assert rc == 0
    th, var, it = A.ma_fit(acf, (5, 5, 5))
    # same sweep order, same summation order: bit-identical
    assert np.array_equal(th, th_o) and var == var_o and it == it_o
    assert th[0, 0, 0] == -1.0 and 1 <= it < 1000
    assert var == pytest.approx(acf[0, 0, 0] / np.sum(th ** 2), rel=1e-14)


@pytest.mark.parametrize("order", [(5, 5, 5), (3, 4, 2), (7, 1, 1), (1, 1, 1), (10, 10, 10)])
def test_fit_stopping_rule(order):
    """The fitted theta solves acf(ijk) = var_wn sum_l theta(ijk + l) theta(l)
    over the order box (the loop stops at a residual or variance change of
    1e-5; the final var_wn is one update later, hence the looser bound)."""
    acf = solver_test_acf()
    th, var, it = A.ma_fit(acf, order)
    rc, th_o, var_o, it_o = O.ma_fit(acf, order)
    assert rc == 0 and np.array_equal(th, th_o) and it == it_o
    resid = np.max(np.abs(acf[:order[0], :order[1], :order[2]] - lag_products(th) * var))
    assert resid <= 2e-5 and it < 1000


def test_fit_order_one_is_white_noise():
    th, var, it = A.ma_fit(solver_test_acf(), (1, 1, 1))
    assert th.shape == (1, 1, 1) and th[0, 0, 0] == -1.0 and var == 1.0


def test_fit_bad_order():
    with pytest.raises(A.ArmaError) as e:
        A.ma_fit(solver_test_acf((4, 4, 4)), (5, 2, 2))
    assert e.value.code == -1 and "bad order" in str(e.value)
    assert O.ma_fit(solver_test_acf((4, 4, 4)), (5, 2, 2))[0] == 1


def test_fit_bad_white_noise_variance():
    acf = 1e-7 * solver_test_acf((4, 4, 4))
    with pytest.raises(A.ArmaError) as e:
        A.ma_fit(acf, (2, 2, 2))
    assert e.value.code == -7 and "bad white noise variance" in str(e.value)
    assert O.ma_fit(acf, (2, 2, 2))[0] == 3


def test_fit_diverges_on_constant_acf():
    """A constant ACF (the analytic propagating wave with zero decay, wave
    numbers and velocity) drives the iteration to non-finite coefficients."""
    acf = np.ones((20, 10, 10))
    with pytest.raises(A.ArmaError) as e:
        A.ma_fit(acf, (20, 10, 10))
    assert e.value.code == -7 and "bad MA model coefficients" in str(e.value)
    assert O.ma_fit(acf, (20, 10, 10))[0] == 2


def test_direct_sum_equals_fft_overlap_add_reference_shapes():
    """The reference's GenerateSurfaceTest: direct sum vs FFT overlap-add."""
    rng = np.random.default_rng(12345)
    kernel = rng.normal(0.0, np.sqrt(2.0), (8, 8, 8))
    signal = rng.normal(0.0, np.sqrt(2.0), (400, 8, 8))
    direct = O.ma_filter(signal, kernel)
    fft = O.ma_convolve_fft(signal, kernel)
    err = np.max(np.abs(direct - fft))
    assert err <= 1e-4                          # the reference's bound
    assert err <= 1e-13 * np.max(np.abs(direct))  # FP64 rounding only


@pytest.mark.parametrize("sig,ker", [((33, 17, 9), (4, 3, 2)), ((20, 40, 40), (20, 10, 10)),
                                     ((64, 5, 7), (32, 1, 1))])
def test_direct_sum_equals_fft_overlap_add_ragged(sig, ker):
    rng = np.random.default_rng(7)
    theta = rng.normal(0.0, 0.1, ker)
    eps = rng.normal(0.0, 1.0, sig)
    d = O.ma_filter(eps, theta)
    f = O.ma_convolve_fft(eps, theta)
    assert np.max(np.abs(d - f)) <= 1e-12 * np.max(np.abs(d))


def test_direct_sum_definition():
    """zeta = eps - sum_{m != 0} theta(m) eps(n - m), zero history (numpy)."""
    rng = np.random.default_rng(3)
    theta = rng.normal(0.0, 0.3, (3, 2, 4))
    eps = rng.normal(0.0, 1.0, (6, 5, 7))
    want = eps.copy()
    for k in range(3):
        for i in range(2):
            for j in range(4):
                if k == i == j == 0:
                    continue
                want[k:, i:, j:] -= theta[k, i, j] * eps[:6 - k, :5 - i, :7 - j]
    assert np.allclose(O.ma_filter(eps, theta), want, rtol=0, atol=1e-13)


# ------------------------------------------------------------- `.arma` grammar
def ma_config(body="", acf=None, transform="none"):
    acf = acf or "func = propagating_wave\n\t\tgrid = (20,10,10) : (10,5,5)"
    return ("model = MA {\n\tout_grid = (200,40,40)\n\toutput = waves,acf,surface\n"
            f"\ttransform = {transform}\n\tacf = {{\n\t\t{acf}\n\t}}\n{body}"
            "\tno_seed = 1\n}\nvelocity_potential_solver = high_amplitude {\n"
            "\tdepth = 12\n\tdomain = from (10,-12) to (10,3) npoints (1,128)\n}\n")


def test_ma_config_parses():
    d = A.Driver(ma_config("\torder = (20,10,10)\n\talgorithm = fixed_point_iteration\n"))
    info = d.info()
    assert info["order"] == (20, 10, 10) and info["shape"] == (200, 40, 40)
    # the output grid is rescaled by 2 pi like the AR model's
    # (src/generator/basic_arma_model.cc:62-66)
    assert info["delta"] == pytest.approx(tuple(2 * np.pi * d_ for d_ in (10 / 19, 5 / 9, 5 / 9)))


def test_ma_default_order_is_acf_shape():
    assert A.Driver(ma_config()).info()["order"] == (20, 10, 10)


def test_ma_order_above_acf_shape():
    with pytest.raises(A.ArmaError) as e:
        A.Driver(ma_config("\torder = (21,10,10)\n"))
    assert e.value.code == -1 and "bad order" in str(e.value)


def test_ma_invalid_algorithm():
    with pytest.raises(A.ArmaError) as e:
        A.Driver(ma_config("\talgorithm = choi_recursive\n"))
    assert e.value.code == -1 and "Invalid MA algorithm: choi_recursive" in str(e.value)
    # newton_raphson is a valid name; generation then reports it unsupported
    A.Driver(ma_config("\talgorithm = newton_raphson\n"))


def test_ma_wave_group_acf_config():
    """The reference's propagating_wave.arma layout (wave-group ACF, order
    (32,1,1))."""
    acf = ("func = cos\n\t\tamplitude = 2\n\t\talpha = (1,0,0)\n\t\tvelocity = 0.01\n"
           "\t\tbeta = (0.1,0)\n\t\tnwaves = (12.5,12.5,12.5)\n\t\tshape = (32,1,1)")
    d = A.Driver(ma_config("\torder = (32,1,1)\n", acf=acf))
    table, _ = d.acf()
    assert table.shape == (32, 1, 1) and d.info()["order"] == (32, 1, 1)
    th, var, it = A.ma_fit(table, (32, 1, 1))
    rc, th_o, var_o, it_o = O.ma_fit(table, (32, 1, 1))
    assert rc == 0 and np.array_equal(th, th_o) and var == var_o
