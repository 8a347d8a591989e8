"""CPU tests of the C ABI: the library loads and exports every entry point the
header declares; the host-side FP64 fit matches the oracle; argument checks
and file handling map to the documented error codes.  No device work."""
import os
import re

import numpy as np
import pytest

import arma_b200 as A
from arma_b200 import capi
import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "arma_b200.h")).read()
    return sorted(set(re.findall(r"^int\s+(arma_\w+)\s*\(", txt, flags=re.M)))


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(capi.EXPORTS)
    assert L.arma_version() == 100


def test_acf_eval_matches_oracle():
    for kind, name in [(A.ACF_STANDING, "standing_wave"), (A.ACF_PROPAGATING, "propagating_wave")]:
        a = A.acf_eval(kind, (5, 6, 7), 1.3, 0.7, [0.05, 0.06, 0.07], [0.4, 0.3], (1.0, 0.5, 2.0))
        b = O.acf(name, (5, 6, 7), 1.3, 0.7, [0.05, 0.06, 0.07], [0.4, 0.3], (1.0, 0.5, 2.0))
        assert np.allclose(a, b, rtol=1e-15, atol=0)


@pytest.mark.parametrize("order", [(2, 2, 2), (3, 4, 5), (7, 7, 7)])
def test_fit_matches_oracle(order):
    acf = O.acf("standing_wave", (8, 8, 8), 1.5, 0.8, [0.05] * 3, [0.5, 0.5])
    phi, var = A.ar_fit(acf, order)
    phio, varo = O.ar_fit(acf, order)  # Bunch-Kaufman, the reference's dsysv
    assert phi[0, 0, 0] == 0.0
    assert np.allclose(phi, phio, rtol=0, atol=1e-9)
    assert abs(var - varo) < 1e-12
    assert abs(var - O.white_noise_variance(acf, phi)) < 1e-14


def test_fit_analytic_standing_equals_table_fit():
    acf = A.acf_eval(A.ACF_STANDING, (7, 7, 7), 1.5, 0.8, [0.05] * 3, [0.5, 0.5])
    phi_t, v_t = A.ar_fit(acf, (7, 7, 7))
    phi_a, v_a = A.ar_fit_analytic(A.ACF_STANDING, (7, 7, 7), 1.5, 0.8, [0.05] * 3, [0.5, 0.5])
    assert np.array_equal(phi_t, phi_a) and v_t == v_a


def test_fit_analytic_propagating_is_spd_and_solves_signed_system():
    import itertools
    order = (4, 4, 4)
    phi, var = A.ar_fit_analytic(A.ACF_PROPAGATING, order, 1.0, 0.6, [0.04] * 3, [0.3, 0.2])
    assert var > 0
    g = lambda t, x, y: np.exp(-0.04 * (abs(t) + abs(x) + abs(y))) * np.cos(0.6 * t + 0.3 * x + 0.2 * y)
    pts = np.array(list(itertools.product(*[range(o) for o in order])))
    D = pts[:, None, :] - pts[None, :, :]
    R = g(D[..., 0], D[..., 1], D[..., 2])
    x = np.linalg.solve(R[1:, 1:], R[1:, 0])
    assert np.allclose(phi.ravel()[1:], x, rtol=0, atol=1e-8)


def test_fit_rejects_indefinite_reference_matrix():
    acf = A.acf_eval(A.ACF_PROPAGATING, (10, 10, 10), 1.0, 0.6, [0.04] * 3, [0.3, 0.2])
    with pytest.raises(capi.ArmaError) as e:
        A.ar_fit(acf, (10, 10, 10))
    assert e.value.code == -7


def test_fit_bad_order():
    acf = np.ones((3, 3, 3))
    with pytest.raises(capi.ArmaError) as e:
        A.ar_fit(acf, (4, 3, 3))
    assert e.value.code == -1 and "order" in str(e.value)


def test_mt_file_roundtrip(tmp_path):
    p = A.mt19937_params()
    sets = []
    for k in range(3):
        q = capi.MtParams.from_buffer_copy(p)
        q.aaa = p.aaa ^ (k << 8)
        sets.append(q)
    path = str(tmp_path / "mt.dat")
    A.mt_file_write(path, sets)
    assert os.path.getsize(path) == 3 * (72 + 624 * 4)
    assert A.mt_file_count(path) == 3
    for k in range(3):
        assert A.mt_file_read(path, k).as_tuple() == sets[k].as_tuple()
    # the oracle reads the same bytes
    assert O.mt_file_count(path) == 3
    assert O.mt_file_read(path, 2).as_tuple() == sets[2].as_tuple()
    with pytest.raises(capi.ArmaError) as e:
        A.mt_file_read(path, 3)
    assert e.value.code == -6  # PRNG_error: too few parameter sets


def test_mt_file_missing():
    with pytest.raises(capi.ArmaError) as e:
        A.mt_file_count("/nonexistent/mt.dat")
    assert e.value.code == -5 and "not found" in str(e.value)


@pytest.mark.parametrize("order", [(16, 16, 4), (14, 16, 2), (2, 18, 3), (3, 3, 14), (17, 1, 1),
                                   (100, 1, 1)])
def test_fp32_filter_rejects_unsupported_order_before_device_work(order):
    """The FP32 tile kernel holds at most 13 x 17 (k, i) tap rows, 17 rows of
    taps per slice and 13 taps per row, and the device filters take at most 16
    per axis (a long time order such as 100 x 1 x 1 would also need more
    shared memory than a block has); other orders answer ARMA_ENOTSUP from the
    argument checks (the buffer pointer is never touched)."""
    with pytest.raises(capi.ArmaError) as e:
        capi.ar_filter_fp32c_noalloc(0, np.zeros(order), (4, 16, 32), 256)
    assert e.value.code == -8 and "not supported" in str(e.value)


@pytest.mark.parametrize("field,value", [("shift0", 0), ("shift1", 0), ("shiftB", -3),
                                         ("shiftC", 32), ("rr", 32), ("mm", 0)])
def test_malformed_mt_parameter_set_rejected(tmp_path, field, value):
    """Tempering shifts outside [1, 31] (the device inverts the tempering by
    a fixed-point iteration that advances by the shift) and malformed
    recurrences are rejected wherever a parameter set is used."""
    p = A.mt19937_params()
    setattr(p, field, value)
    with pytest.raises(capi.ArmaError) as e:
        A.mt_file_write(str(tmp_path / "mt.dat"), [p])
    assert e.value.code == -1 and "bad MT parameter set" in str(e.value)


def test_router_rejects_bad_arguments_without_a_device():
    for devices in ([], list(range(257))):
        with pytest.raises(A.ArmaError) as e:
            A.Router(devices=devices)
        assert e.value.code == -1
