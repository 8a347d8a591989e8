"""The moving-average model on the GPU against the oracle.

arma_ma_filter = zeta = eps - sum_{m != 0} theta(m) eps(n - m) with zero
history (MA_model::generate_surface, src/generator/ma_model.cc:42-61): FP64
within 1e-12 of max|zeta| of the oracle's direct sum (the kernel accumulates
with FMA in its own tap order; the reference's FFT form differs from the
direct sum by FP64 rounding too), FP32C within RMS 1e-5.  Shapes cover ragged
tiles in t, x and y, the reference's time-only order (32,1,1), order 1 (the
identity), and more taps than one launch's parameter block holds (two
launches adding into the output).  arma_ma_generate and the `.arma` driver
with `model = MA` equal the oracle chain (noise -> direct MA sum ->
renormalisation) on the same coefficients.
"""
import math

import numpy as np
import pytest

import arma_b200 as A
import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def run_filter(ctx, theta, eps, precision):
    dt = torch.float64 if precision == A.FP64 else torch.float32
    e = torch.tensor(eps, dtype=dt, device="cuda")
    z = torch.full_like(e, float("nan"))
    ctx.ma_filter(theta, eps.shape, precision, e.data_ptr(), z.data_ptr())
    ctx.synchronize()
    return z.cpu().numpy().astype(np.float64)


CASES = [
    ((40, 24, 24), (5, 5, 5)),
    ((33, 17, 70), (4, 3, 2)),      # ragged in t (8), x (16) and y (64)
    ((64, 5, 7), (32, 1, 1)),       # time-only, as the reference's propagating_wave.arma
    ((20, 40, 40), (20, 10, 10)),   # the reference's nit-propagating-none order
    ((9, 3, 3), (1, 1, 1)),         # identity
    ((24, 20, 20), (16, 16, 16)),   # 4096 taps: two FP64 launches
    ((40, 20, 20), (32, 16, 16)),   # 8192 taps: three FP64 / two FP32 launches
]


@pytest.mark.parametrize("shape,order", CASES)
def test_ma_filter_fp64(ctx, shape, order):
    rng = np.random.default_rng(hash((shape, order)) % 2**32)
    theta = rng.normal(0.0, 0.2 / math.sqrt(np.prod(order)), order)
    eps = rng.normal(0.0, 1.0, shape)
    ref = O.ma_filter(eps, theta)
    got = run_filter(ctx, theta, eps, A.FP64)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("shape,order", CASES)
def test_ma_filter_fp32c(ctx, shape, order):
    rng = np.random.default_rng(17 + len(shape) + sum(order))
    theta = rng.normal(0.0, 0.2 / math.sqrt(np.prod(order)), order)
    eps = rng.normal(0.0, 1.0, shape).astype(np.float32).astype(np.float64)
    ref = O.ma_filter(eps, theta)
    got = run_filter(ctx, theta, eps, A.FP32C)
    d = got - ref
    assert math.sqrt((d ** 2).mean() / (ref ** 2).mean()) <= 1e-5
    assert np.abs(d).max() <= 1e-4 * np.abs(ref).max()


def test_ma_filter_equals_reference_fft_form(ctx):
    """Against the reference's production form (FFT overlap-add)."""
    rng = np.random.default_rng(5)
    theta = rng.normal(0.0, 0.05, (20, 10, 10))
    eps = rng.normal(0.0, 1.0, (60, 40, 40))
    ref = O.ma_convolve_fft(eps, theta)
    got = run_filter(ctx, theta, eps, A.FP64)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_ma_filter_rejects_overlap(ctx):
    e = torch.zeros((8, 8, 8), dtype=torch.float64, device="cuda")
    with pytest.raises(A.ArmaError) as err:
        ctx.ma_filter(np.zeros((2, 2, 2)), (8, 8, 8), A.FP64, e.data_ptr(), e.data_ptr())
    assert err.value.code == -1 and "overlap" in str(err.value)


def oracle_chain(shape, theta, var, acf0, seed):
    eps = O.white_noise(O.mt19937_params(), seed, math.sqrt(var),
                        int(np.prod(shape))).reshape(shape)
    zeta, scale = O.variance_renorm(O.ma_filter(eps, theta), acf0)
    return zeta, scale


def test_ma_generate_fp64_and_fp32c(ctx):
    i, j, k = np.meshgrid(np.arange(10), np.arange(10), np.arange(10), indexing="ij")
    acf = np.exp(-(i + j + k)) * np.cos(0.6 * i + 0.4 * j + 0.4 * k)
    theta, var, _ = A.ma_fit(acf, (5, 5, 5))
    shapes = [(48, 32, 40), (21, 70, 9)]
    ref = [oracle_chain(s, theta, var, acf[0, 0, 0], 100 + n) for n, s in enumerate(shapes)]
    for prec, dt, tol in [(A.FP64, torch.float64, None), (A.FP32C, torch.float32, 1e-5)]:
        bufs = [torch.empty(s, dtype=dt, device="cuda") for s in shapes]
        surfs = [A.capi.make_surface(s, theta, var, acf[0, 0, 0], A.mt19937_params(), 100 + n,
                                     b.data_ptr()) for n, (s, b) in enumerate(zip(shapes, bufs))]
        scales = ctx.ma_generate(surfs, prec)
        ctx.synchronize()
        for (zr, sr), b, sc in zip(ref, bufs, scales):
            z = b.cpu().numpy().astype(np.float64)
            if tol is None:
                assert np.abs(z - zr).max() <= 1e-12 * np.abs(zr).max()
                assert sc == pytest.approx(sr, rel=1e-12)
            else:
                d = z - zr
                assert math.sqrt((d ** 2).mean() / (zr ** 2).mean()) <= tol


def ma_text(mt, acf, order, extra=""):
    return f"""model = MA {{
	out_grid = (200,40,40)
	acf = {{
		{acf}
	}}
	order = {order}
	algorithm = fixed_point_iteration
	output = none
	transform = none
	validate = 0
	seed = 321
	mt_file = {mt}
{extra}
}}
velocity_potential_solver = high_amplitude {{
	depth = 12
	domain = from (10,-12) to (10,3) npoints (1,16)
}}
"""


PROPAGATING = ("func = propagating_wave\n\t\tgrid = (20,10,10) : (10,5,5)\n\t\tamplitude = 1\n"
               "\t\tvelocity = 0.6\n\t\talpha = (1,1,1)\n\t\tbeta = (0.4,0.4)")


def test_driver_ma_reference_config_diverges(ctx, tmp_path):
    """The reference's nit-propagating-none.arma ACF (propagating_wave on
    (20,10,10) : (10,5,5) with the default amplitude 1, velocity 0, alpha 0,
    beta 0: a constant ACF) makes the fixed-point iteration diverge; the
    oracle's restatement does the same, and the reference throws
    "bad MA model coefficients" there."""
    mt = str(tmp_path / "mt.dat")
    A.mt_file_write(mt, [A.mt19937_params()])
    d = A.Driver(ma_text(mt, "func = propagating_wave\n\t\tgrid = (20,10,10) : (10,5,5)",
                         "(20,10,10)"))
    with pytest.raises(A.ArmaError) as e:
        d.generate_wavy_surface(ctx)
    assert e.value.code == -7 and "bad MA model coefficients" in str(e.value)


def test_driver_ma_end_to_end(ctx, tmp_path):
    """The reference's nit-propagating-none.arma layout (analytic propagating
    ACF 20x10x10, order (20,10,10), 200x40x40, high-amplitude solver) with a
    decaying ACF, through the driver: coefficients equal the oracle fit, the
    surface equals the oracle chain, the velocity equals the oracle solver."""
    mt = str(tmp_path / "mt.dat")
    A.mt_file_write(mt, [A.mt19937_params()])
    d = A.Driver(ma_text(mt, PROPAGATING, "(20,10,10)"))
    d.generate_wavy_surface(ctx)
    acf, _ = d.acf()
    rc, theta, var, _ = O.ma_fit(acf, (20, 10, 10))
    assert rc == 0
    np.testing.assert_array_equal(d.phi(), theta)
    assert d.info()["var_wn"] == pytest.approx(var, rel=1e-14)
    zeta_ref, _ = oracle_chain((200, 40, 40), theta, d.info()["var_wn"], acf[0, 0, 0], 321)
    zeta = d.zeta()
    assert np.abs(zeta - zeta_ref).max() <= 1e-12 * np.abs(zeta_ref).max()
    d.compute_velocity_potentials(ctx)
    info = d.info()
    z = [-12.0 + 15.0 * q / 15 for q in range(16)]
    ref = O.velocity_high_amplitude(zeta, info["delta"], 12.0, z, [10])
    vel = d.velocity_potentials()
    assert np.abs(vel - ref).max() <= 1e-9 * np.abs(ref).max()


def test_driver_ma_wave_group_time_only(ctx, tmp_path):
    """The reference's propagating_wave.arma set-up: a wave-group ACF of shape
    (32,1,1) and order (32,1,1), FP32C."""
    mt = str(tmp_path / "mt.dat")
    A.mt_file_write(mt, [A.mt19937_params()])
    acf_text = ("func = cos\n\t\tamplitude = 2\n\t\talpha = (1,0,0)\n\t\tvelocity = 0.01\n"
                "\t\tbeta = (0.1,0)\n\t\tnwaves = (12.5,12.5,12.5)\n\t\tshape = (32,1,1)")
    d = A.Driver(ma_text(mt, acf_text, "(32,1,1)", "\tprecision = fp32c"))
    d.generate_wavy_surface(ctx)
    acf, _ = d.acf()
    theta, var, _ = A.ma_fit(acf, (32, 1, 1))
    zeta_ref, _ = oracle_chain((200, 40, 40), theta, var, acf[0, 0, 0], 321)
    diff = d.zeta() - zeta_ref
    assert math.sqrt((diff ** 2).mean() / (zeta_ref ** 2).mean()) <= 1e-5


def test_driver_ma_newton_raphson_unsupported(ctx, tmp_path):
    mt = str(tmp_path / "mt.dat")
    A.mt_file_write(mt, [A.mt19937_params()])
    text = ma_text(mt, "func = propagating_wave\n\t\tgrid = (8,8,8) : (4,4,4)", "(4,4,4)")
    d = A.Driver(text.replace("fixed_point_iteration", "newton_raphson"))
    with pytest.raises(A.ArmaError) as e:
        d.generate_wavy_surface(ctx)
    assert e.value.code == -8 and "only fixed_point_iteration is supported" in str(e.value)
