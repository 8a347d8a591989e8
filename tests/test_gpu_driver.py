"""The `.arma` programme end to end on the GPU against the oracle chain.

generate_wavy_surface = ACF -> Yule-Walker fit -> white noise -> AR filter ->
variance renormalisation (-> NIT), compute_velocity_potentials = the linear
solver on the domain's t slices and z levels, write_all = the zeta / phi
files (src/arma_driver.cc:29-178).  Tolerances: FP64 surface 1e-12 relative
to max|zeta| (noise within a few ulp, AR filter bit-exact), velocity 1e-9 of
max|phi|, FP32C surface RMS 1e-5; written files byte-equal to the oracle's
writers on the same values.
"""
import math
import os

import numpy as np
import pytest

import arma_b200 as A
import oracle as O

pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

ACF_LEN = (2.5, 5.0, 5.0)


def write_mt(path):
    A.mt_file_write(str(path), [A.mt19937_params()])
    return str(path)


def config(mt, output="surface,csv,blitz,binary", extra=""):
    return f"""model = AR {{
	out_grid = (40,24,24)
	acf = {{
		func = standing_wave
		grid = (10,10,10) : (2.5,5,5)
		amplitude = 1.5
		velocity = 0.5
		alpha = (0.06,0.06,0.06)
		beta = (0.8,0.8)
	}}
	order = (5,5,5)
	algorithm = gauss_elimination
	output = {output}
	validate = 0
	seed = 1234
	mt_file = {mt}
{extra}
}}
velocity_potential_solver = linear {{
	depth = 12
	domain = from (10,-6) to (30,0) npoints (3,4)
}}
"""


MA_BINARY = """model = MA {{
	out_grid = (40,24,24)
	acf = {{
		func = propagating_wave
		grid = (20,10,10) : (10,5,5)
		amplitude = 1
		velocity = 0.6
		alpha = (1,1,1)
		beta = (0.4,0.4)
	}}
	order = (20,10,10)
	algorithm = fixed_point_iteration
	output = surface,binary
	validate = 0
	seed = 321
	mt_file = {mt}
}}
velocity_potential_solver = linear {{
	depth = 12
	domain = from (10,-6) to (30,0) npoints (3,4)
}}
"""


def oracle_fit():
    delta = [L / 9 for L in ACF_LEN]
    acf = O.acf("standing_wave", (10, 10, 10), 1.5, 0.5, [0.06] * 3, [0.8, 0.8], delta)
    phi, var = O.ar_fit(acf, (5, 5, 5), method="cholesky")
    return acf, phi, var


def oracle_surface(phi, var, acf0, seed=1234):
    """The oracle chain on the driver's own coefficients, so that the surface
    check isolates noise + filter + renormalisation."""
    shape = (40, 24, 24)
    eps = O.white_noise(O.mt19937_params(), seed, math.sqrt(var),
                        int(np.prod(shape))).reshape(shape)
    zeta, _ = O.variance_renorm(O.ar_filter(eps, phi), acf0)
    return zeta


def test_driver_generate_velocity_write(ctx, tmp_path):
    mt = write_mt(tmp_path / "mt.dat")
    d = A.Driver(config(mt))
    out = tmp_path / "out"
    out.mkdir()
    d.set_output_dir(str(out))
    d.generate_wavy_surface(ctx)
    # zeta.bin is streamed while generating: the surface before the variance
    # renormalisation, as the reference's writer thread writes it
    assert sorted(os.listdir(out)) == ["zeta.bin"]
    raw = (out / "zeta.bin").read_bytes()
    acf, phi_ref, var_ref = oracle_fit()
    # the fit is a host LL^T; its rounding differs from the oracle's in the
    # last bits, amplified by the Yule-Walker matrix's condition number
    np.testing.assert_allclose(d.phi(), phi_ref, rtol=0, atol=1e-9)
    assert abs(d.info()["var_wn"] - var_ref) < 1e-12
    zeta_ref = oracle_surface(d.phi(), d.info()["var_wn"], acf[0, 0, 0])
    zeta = d.zeta()
    assert np.abs(zeta - zeta_ref).max() <= 1e-12 * np.abs(zeta_ref).max()
    shape = (40, 24, 24)
    eps = O.white_noise(O.mt19937_params(), 1234, math.sqrt(d.info()["var_wn"]),
                        int(np.prod(shape))).reshape(shape)
    gen = O.ar_filter(eps, d.phi())
    got = np.frombuffer(raw, dtype=">f8").reshape(shape)
    assert np.abs(got - gen).max() <= 1e-12 * np.abs(gen).max()
    assert not np.array_equal(got, zeta)

    d.compute_velocity_potentials(ctx)
    info = d.info()
    assert info["velocity_shape"] == (3, 4, 24, 24)
    vel = d.velocity_potentials()
    t_idx = [10, 20, 30]
    z = [-6.0, -4.0, -2.0, 0.0]
    ref = O.velocity_linear(zeta, info["delta"], 12.0, z, t_idx)
    assert np.abs(vel - ref).max() <= 1e-9 * np.abs(ref).max()

    d.write_all(str(out))
    assert sorted(os.listdir(out)) == ["phi", "phi.csv", "zeta", "zeta.bin", "zeta.csv"]
    assert (out / "zeta.bin").read_bytes() == raw  # not written again
    # an MA model has no writer thread: write_all writes the final surface
    ma = A.Driver(MA_BINARY.format(mt=mt))
    out_ma = tmp_path / "out_ma"
    out_ma.mkdir()
    ma.set_output_dir(str(out_ma))
    ma.generate_wavy_surface(ctx)
    assert os.listdir(out_ma) == []
    ma.write_all(str(out_ma))
    O.write_zeta_bin(str(tmp_path / "ref_ma.bin"), ma.zeta())
    assert (out_ma / "zeta.bin").read_bytes() == (tmp_path / "ref_ma.bin").read_bytes()
    O.write_zeta_csv(str(tmp_path / "ref.csv"), zeta, info["delta"])
    assert (out / "zeta.csv").read_text() == (tmp_path / "ref.csv").read_text()
    head = (out / "zeta").read_text().split("\n", 1)[0]
    assert head == "(0,39) x (0,23) x (0,23)"
    rows = (out / "phi.csv").read_text().splitlines()
    assert rows[0] == "t,z,x,y,phi" and len(rows) == 1 + 3 * 4 * 24 * 24


def test_driver_fp32c_and_nit(ctx, tmp_path):
    mt = write_mt(tmp_path / "mt.dat")
    acf, _, _ = oracle_fit()
    d = A.Driver(config(mt, output="none", extra="\tprecision = fp32c"))
    d.generate_wavy_surface(ctx)
    zeta_ref = oracle_surface(d.phi(), d.info()["var_wn"], acf[0, 0, 0])
    diff = d.zeta() - zeta_ref
    assert math.sqrt((diff ** 2).mean() / (zeta_ref ** 2).mean()) <= 1e-5
    nit = ("\ttransform = nit {\n\t\tdistribution = gram_charlier {\n"
           "\t\t\tskewness = 0.5\n\t\t\tkurtosis = 3.2\n\t\t}\n"
           "\t\tcdf_solver = {\n\t\t\tinterval = [-5,5]\n\t\t\tabsolute_error = 1e-8\n"
           "\t\t\tmax_iterations = 100\n\t\t}\n\t}")
    d = A.Driver(config(mt, output="none", extra=nit))
    d.generate_wavy_surface(ctx)
    ref = O.nit_transform(zeta_ref, math.sqrt(acf[0, 0, 0]), "gram_charlier", (0.5, 3.2),
                          interval=(-5.0, 5.0), eps=1e-8, max_iter=100)
    assert np.abs(d.zeta() - ref).max() <= 2e-8


def test_driver_missing_mt_file(ctx, tmp_path):
    d = A.Driver(config(str(tmp_path / "none.dat")))
    with pytest.raises(A.ArmaError) as e:
        d.generate_wavy_surface(ctx)
    assert e.value.code == -5 and "Mersenne Twister configuration file not found" in str(e.value)


def test_cli_runs(tmp_path):
    from arma_b200.__main__ import main
    mt = write_mt(tmp_path / "mt.dat")
    cfg = tmp_path / "standing.arma"
    cfg.write_text(config(mt, output="surface,binary"))
    out = tmp_path / "o"
    out.mkdir()
    assert main(["-C", str(out), str(cfg)]) == 0
    assert (out / "zeta.bin").stat().st_size == 40 * 24 * 24 * 8


def test_driver_choi_default_algorithm(ctx, tmp_path):
    """Without `algorithm`, the reference fits with Choi's recursive solver on
    the ACF table: the driver's order and phi are the solver's, and the surface
    is the oracle chain on those coefficients."""
    mt = write_mt(tmp_path / "mt.dat")
    text = config(mt, output="none").replace("\talgorithm = gauss_elimination\n", "")
    text = text.replace("alpha = (0.06,0.06,0.06)", "alpha = (0.3,0.3,0.3)")
    d = A.Driver(text)
    d.generate_wavy_surface(ctx)
    delta = [L / 9 for L in ACF_LEN]
    acf = O.acf("standing_wave", (10, 10, 10), 1.5, 0.5, [0.3] * 3, [0.8, 0.8], delta)
    phi, var = A.ar_fit_choi(acf, max_order=5)
    assert d.info()["order"] == phi.shape == (5, 5, 5) and var > 0
    np.testing.assert_array_equal(d.phi(), phi)
    assert d.info()["var_wn"] == var
    zeta_ref = oracle_surface(phi, var, acf[0, 0, 0])
    assert np.abs(d.zeta() - zeta_ref).max() <= 1e-12 * np.abs(zeta_ref).max()


def test_driver_wave_group_acf_end_to_end(ctx, tmp_path):
    """The reference's default model set-up: a wave-group ACF (no `grid`),
    Choi's solver, validate_process on, velocity on slices of non-power-of-two
    sides.  The surface equals the oracle chain on the driver's coefficients
    and the velocity equals the oracle solver."""
    mt = write_mt(tmp_path / "mt.dat")
    text = f"""model = AR {{
	out_grid = (30,40,20)
	acf = {{
		func = standing_wave
		amplitude = 2
		alpha = (1.5,0.3,0.8)
		velocity = 0.5
		beta = (0.125,0)
		nwaves = (1.5,4,1)
		shape = (8,8,8)
	}}
	order = (4,4,4)
	output = none
	validate = 1
	seed = 99
	mt_file = {mt}
}}
velocity_potential_solver = linear {{
	depth = 12
	domain = from (5,-12) to (25,3) npoints (3,6)
}}
"""
    d = A.Driver(text)
    d.generate_wavy_surface(ctx)
    acf, _ = d.acf()
    phi, var = A.ar_fit_choi(acf, max_order=4)
    np.testing.assert_array_equal(d.phi(), phi)
    shape = (30, 40, 20)
    eps = O.white_noise(O.mt19937_params(), 99, math.sqrt(var), int(np.prod(shape))).reshape(shape)
    zeta_ref, _ = O.variance_renorm(O.ar_filter(eps, phi), acf[0, 0, 0])
    zeta = d.zeta()
    assert np.abs(zeta - zeta_ref).max() <= 1e-12 * np.abs(zeta_ref).max()
    d.compute_velocity_potentials(ctx)
    info = d.info()
    zs = list(np.linspace(-12.0, 3.0, 6))
    ref = O.velocity_linear(zeta, info["delta"], 12.0, zs, [5, 15, 25])
    assert np.abs(d.velocity_potentials() - ref).max() <= 1e-9 * np.abs(ref).max()
