"""The `.arma` programme layer on CPU: grammar, registry and shapes.

The expected values restate the reference's parsers: Output_flags
(src/output_flags.cc:53-87, known answers of src/test/output-flags-test.cc),
Grid (src/grid.hh:181-192: no ':' means length n-1), Domain, the parameter
map's "Unknown parameter" error (src/params.cc:30-57), the model / solver
registry (src/register_all.hh:47-68), the output grid rescaling
(src/generator/basic_arma_model.cc:56-66) and the linear solver's depth check
(src/velocity/basic_solver.cc:21-36).  Nothing here launches a kernel.
"""
import math

import numpy as np

import pytest

import arma_b200 as A


def config(ar_body: str = "", acf: str = "", solver: str = "", model: str = "AR",
           solver_name: str = "linear") -> str:
    acf = acf or "func = standing_wave\n\t\tgrid = (10,10,10) : (2.5,5,5)"
    solver = solver or "depth = 12\n\tdomain = from (10,-12) to (10,3) npoints (1,128)"
    return (f"# wavy surface\nmodel = {model} {{\n\tout_grid = (40,24,24)\n"
            f"\tacf = {{\n\t\t{acf}\n\t}}\n{ar_body}\n}}\n"
            f"velocity_potential_solver = {solver_name} {{\n\t{solver}\n}}\n")


def err(text: str):
    with pytest.raises(A.ArmaError) as e:
        A.Driver(text)
    return e.value


@pytest.mark.parametrize("line", [
    "acf,surface,blitz",
    "acf , surface , blitz",
    " acf , surface , blitz ",
    "acf,surface,blitz\n",
])
def test_output_flags_known_answers(line):
    d = A.Driver(config(f"\toutput = {line}\n"))
    assert d.info()["output"] == ["acf", "blitz", "surface"]


@pytest.mark.parametrize("line,expect", [
    ("surface", ["blitz", "surface"]),          # default format
    ("surface,csv", ["csv", "surface"]),
    ("surface,binary,summary", ["summary", "binary", "surface"]),
    ("acf,none,surface", ["blitz", "surface"]),  # none clears what came before
    ("none", []),
])
def test_output_flags_prune_and_none(line, expect):
    assert A.Driver(config(f"\toutput = {line}\n")).info()["output"] == expect


def test_output_flag_invalid():
    e = err(config("\toutput = surface,pdf\n"))
    assert e.code == -1 and "Invalid output flag: pdf" in str(e)


def test_grid_lengths_and_output_step():
    """Output step = 2 pi x ACF step; ACF step = length / (n - 1)."""
    info = A.Driver(config()).info()
    assert info["shape"] == (40, 24, 24)
    for got, length in zip(info["delta"], (2.5, 5.0, 5.0)):
        assert got == pytest.approx(length / 9 * 2 * math.pi, rel=1e-15)
    info = A.Driver(config(acf="func = standing_wave\n\t\tgrid = (5,8,8)")).info()
    for got in info["delta"]:  # no ':' -> length n - 1 -> step 1
        assert got == pytest.approx(2 * math.pi, rel=1e-15)


@pytest.mark.parametrize("order,expect", [
    ("", (10, 10, 10)),              # absent: the ACF shape
    ("\torder = (0,3,3)\n", (10, 10, 10)),
    ("\torder = (7,5,3)\n", (7, 5, 3)),
])
def test_order_defaults_to_acf_shape(order, expect):
    assert A.Driver(config(order)).info()["order"] == expect


def test_order_larger_than_acf_rejected():
    e = err(config("\torder = (11,3,3)\n"))
    assert e.code == -1 and "order" in str(e)


def test_unknown_parameter():
    e = err(config(acf="func = standing_wave\n\t\tgrid = (10,10,10)\n\t\twavelength = (1,2,3)"))
    assert e.code == -1 and 'Unknown parameter: "wavelength"' in str(e)
    e = err(config(acf="func = standing_wave\n\t\tgrid = (10,10,10)\n\t\tnwaves = (1,2,3)"))
    assert e.code == -1 and "grid with nwaves" in str(e)


def test_comments_and_blank_lines():
    text = config("# a comment line\n\n\torder = (3,3,3) \n# another\n")
    assert A.Driver(text).info()["order"] == (3, 3, 3)


@pytest.mark.parametrize("name", ["ARMA", "plain_wave", "LH"])
def test_registered_models_not_built(name):
    e = err(config(model=name))
    assert e.code == -8 and name in str(e)


@pytest.mark.parametrize("name", ["plain", "small_amplitude"])
def test_registered_solvers_not_built(name):
    e = err(config(solver_name=name))
    assert e.code == -8 and name in str(e)


def test_unregistered_names():
    assert err(config(model="XYZ")).code == -1
    assert err(config(solver_name="spectral")).code == -1


def test_missing_solver_and_model():
    text = config()
    no_solver = text[:text.index("velocity_potential_solver")]
    e = err(no_solver)
    assert e.code == -1 and "velocity_potential_solver" in str(e)
    e = err(text[text.index("velocity_potential_solver"):])
    assert e.code == -1 and "generator" in str(e)


def test_bad_acf_function():
    e = err(config(acf="func = cos\n\t\tgrid = (10,10,10)"))
    assert e.code == -1 and 'Bad ACF function name: "cos"' in str(e)


def test_depth_inf_and_min_z():
    A.Driver(config(solver="depth = inf\n\tdomain = from (10,-100) to (10,3) npoints (1,16)"))
    e = err(config(solver="depth = 12\n\tdomain = from (10,-13) to (10,3) npoints (1,16)"))
    assert e.code == -1 and "min(z) is less than -h" in str(e)
    e = err(config(solver="depth = -1\n\tdomain = from (0,0) to (0,0) npoints (1,1)"))
    assert e.code == -1


def test_domain_grammar():
    A.Driver(config(solver="domain = npoints (2,4) to (5,0) from (3,-2)\n\tdepth = 2"))
    e = err(config(solver="depth = 2\n\tdomain = at (0,0) to (1,1) npoints (1,1)"))
    assert e.code == -1 and "bad prefix" in str(e)


def test_nit_transform_grammar():
    gc = ("\ttransform = nit {\n\t\tdistribution = gram_charlier {\n"
          "\t\t\tskewness = 2.25\n\t\t\tkurtosis = 0.4\n\t\t}\n"
          "\t\tcdf_solver = {\n\t\t\tinterval = [-5,5]\n\t\t\tabsolute_error = 1e-4\n"
          "\t\t\tmax_iterations = 50\n\t\t}\n\t}\n")
    A.Driver(config(gc))
    sn = ("\ttransform = nit {\n\t\tdistribution = skew_normal {\n"
          "\t\t\tmean = 0\n\t\t\tstdev = 1\n\t\t\talpha = 1\n\t\t}\n\t}\n")
    A.Driver(config(sn))
    e = err(config("\ttransform = nit {\n\t\tdistribution = weibull {}\n\t}\n"))
    assert "Invalid distribution: weibull" in str(e)
    e = err(config(gc.replace("1e-4", "0")))
    assert e.code == -1 and "absolute_error" in str(e)
    e = err(config(gc.replace("[-5,5]", "[5,-5]")))
    assert e.code == -1 and "interval" in str(e)


def test_extensions_parse():
    A.Driver(config("\tseed = 7\n\tprecision = fp32c\n\tmt_file = /tmp/mt.dat\n"))
    e = err(config("\tprecision = fp16\n"))
    assert e.code == -1 and "precision" in str(e)


def test_open_from_path(tmp_path):
    p = tmp_path / "standing.arma"
    p.write_text(config("\torder = (4,4,4)\n"))
    with A.Driver.open(str(p)) as d:
        assert d.info()["order"] == (4, 4, 4)
    with pytest.raises(A.ArmaError) as e:
        A.Driver.open(str(tmp_path / "missing.arma"))
    assert e.value.code == -5


def test_results_before_generate_are_errors():
    d = A.Driver(config())
    with pytest.raises(A.ArmaError) as e:
        d.zeta()
    assert e.value.code == -1
    d.write_all("")  # no "surface" flag: writes nothing


def test_cli_usage(capsys):
    from arma_b200.__main__ import main
    assert main(["-h"]) == 0
    assert "usage:" in capsys.readouterr().out
    assert main([]) == 1


# ----------------------------------------------------------------- wave-group ACF
def wave_acf_numpy(func, amplitude, velocity, alpha, wavenum, nwaves, shape):
    """The reference's ACF_generator restated with numpy (FFT-based circular
    auto-covariance), src/generator/acf_generator.cc:132-244."""
    n = [2 * s + 1 for s in shape]
    ax = [np.linspace(-r, r, m) for r, m in zip(nwaves, n)]
    t, x, y = np.meshgrid(*ax, indexing="ij")
    kx, ky = wavenum
    th = 2 * np.pi * (kx * x + ky * y - velocity * t)
    if func == "sin":
        w = amplitude * np.sin(th)
    elif func == "cos":
        w = amplitude * np.sin(th + 0.5 * np.pi)
    elif func == "stokes":
        st = 2 * np.pi * amplitude * np.hypot(kx, ky)
        w = amplitude * (np.cos(th) + 0.5 * st * np.cos(2 * th) + 3 / 8 * st * st * np.cos(3 * th))
    else:
        w = amplitude * np.cos(2 * np.pi * (kx * x + ky * y)) * np.cos(2 * np.pi * velocity * t)
    we = w * np.exp(-(np.abs(t * alpha[0]) + np.abs(x * alpha[1]) + np.abs(y * alpha[2])))
    we *= np.sqrt(w.var(ddof=1) / we.var(ddof=1))
    acf = np.fft.ifftn(np.abs(np.fft.fftn(we)) ** 2).real / we.size
    h = [m // 2 for m in n]
    return acf[:h[0], :h[1], :h[2]], tuple(r / (s - 1) for r, s in zip(nwaves, h))


@pytest.mark.parametrize("func,amp,vel,alpha,beta,nwaves,shape", [
    ("cos", 1.0, 1.0, (0.06, 0.06, 0.06), (0.8, 0.0), (1.5, 1.5, 1.5), (8, 8, 8)),
    ("standing_wave", 3.0, 0.5, (2.0, 0.2, 1.0), (0.0625, 0.0), (1.85, 16.0, 1.0), (10, 12, 6)),
    ("sin", 2.0, 0.3, (0.1, 0.1, 0.1), (0.3, 0.4), (2.0, 2.0, 2.0), (7, 9, 11)),
    ("stokes", 0.5, 0.7, (0.05, 0.05, 0.05), (0.2, 0.1), (1.0, 1.5, 2.0), (6, 6, 6)),
])
def test_wave_group_acf_matches_numpy(func, amp, vel, alpha, beta, nwaves, shape):
    acf_text = (f"func = {func}\n\t\tamplitude = {amp}\n\t\tvelocity = {vel}\n"
                f"\t\talpha = ({alpha[0]},{alpha[1]},{alpha[2]})\n\t\tbeta = ({beta[0]},{beta[1]})\n"
                f"\t\tnwaves = ({nwaves[0]},{nwaves[1]},{nwaves[2]})\n"
                f"\t\tshape = ({shape[0]},{shape[1]},{shape[2]})")
    d = A.Driver(config("\torder = (3,3,3)\n", acf=acf_text))
    got, delta = d.acf()
    ref, rdelta = wave_acf_numpy(func, amp, vel, alpha, beta, nwaves, shape)
    assert got.shape == ref.shape == tuple(shape)
    assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()
    assert delta == pytest.approx(rdelta, rel=1e-15)
    # the output step is 2 pi times the ACF step (basic_arma_model.cc:62-66)
    assert d.info()["delta"] == pytest.approx(tuple(2 * np.pi * v for v in rdelta), rel=1e-15)


def test_wave_group_defaults_and_order():
    """No keys at all: cos wave, 16^3 ACF; the order defaults to the ACF shape."""
    d = A.Driver(config("", acf="func = cos"))
    acf, delta = d.acf()
    assert acf.shape == (16, 16, 16) and d.info()["order"] == (16, 16, 16)
    assert delta == pytest.approx((1.5 / 15,) * 3)


def test_wave_group_bad_function():
    e = err(config(acf="func = square"))
    assert e.code == -1 and "Invalid plain wave function: square" in str(e)


def test_high_amplitude_solver_is_built():
    A.Driver(config(solver_name="high_amplitude"))


def test_mutated_configs_parse_or_fail_cleanly():
    """Robustness of the `.arma` parser: 2000 random edits (deleted,
    inserted or replaced grammar tokens and extreme numbers) of valid AR, NIT,
    wave-group MA and high-amplitude configurations either parse or raise
    ArmaError with a message; none crashes the process."""
    import random
    seeds = [
        config(),
        config("\torder = (4,4,4)\n\tseed = 3\n\tprecision = fp32c\n\toutput = acf,surface,blitz\n"),
        config("\ttransform = nit {\n\t\tdistribution = gram_charlier {\n\t\t\tskewness = 2.25\n"
               "\t\t\tkurtosis = 0.4\n\t\t}\n\t\tcdf_solver = {\n\t\t\tinterval = [-5,5]\n"
               "\t\t\tabsolute_error = 1e-4\n\t\t\tmax_iterations = 50\n\t\t}\n\t}\n"),
        config(acf="func = cos\n\t\tamplitude = 2\n\t\talpha = (1,0,0)\n\t\tvelocity = 0.01\n"
                   "\t\tbeta = (0.1,0)\n\t\tnwaves = (12.5,12.5,12.5)\n\t\tshape = (32,1,1)",
               model="MA"),
        config(solver_name="high_amplitude"),
    ]
    tokens = ["{", "}", "(", ")", "[", "]", ",", ":", "=", "\n", "#", " ", "-", "1e309", "nan",
              "inf", "0", "-1", "99999999999", "from", "to", "npoints", "nit", "AR", "MA",
              "grid", "order", "(0,0,0)", "(1,1)", "((", "\t"]
    rng = random.Random(2024)
    parsed = 0
    for _ in range(2000):
        s = list(rng.choice(seeds))
        for _ in range(rng.randint(1, 6)):
            op, pos = rng.random(), rng.randrange(len(s) + 1)
            if op < 0.3 and s:
                del s[min(pos, len(s) - 1)]
            elif op < 0.6:
                s.insert(pos, rng.choice(tokens))
            elif s:
                s[rng.randrange(len(s))] = rng.choice(tokens)
        try:
            with A.Driver("".join(s)) as d:
                d.info()
            parsed += 1
        except A.ArmaError as e:
            assert str(e)
    assert 0 < parsed < 2000
