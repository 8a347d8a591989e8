"""GPU parity on the committed dcmt parameter sets and the C1 configuration.

Every committed set -- 16 of period 2^19937 - 1 (nn = 624, mm = 312, rr = 31)
in ``arma_b200/data/mt.dat`` and 16 of period 2^521 - 1 (nn = 17, mm = 8,
rr = 23, the shape of the reference's arma-dcmt default) in
``arma_b200/data/mt521.dat`` -- drives the device generator, the jump-ahead
segment split, the polar white noise and the serving layer's window
untempering, bit-exact with the CPU oracle (MT words and accepted attempts;
noise values within a few ulp, 1e-15 relative).

C1 (the plain FP64 configuration): standing-wave ACF a = 1.5, b = 0.05,
c = 0.8, d = 0.5 on a 7x7x7 lag grid (unit steps), order 7x7x7 from the
FP64 Yule-Walker Cholesky solve, 200 x 40 x 40 output, white noise from the
first set of the 16-set file seeded with 42 (the sequential reference path
draws from mts[0], src/white_noise.hh:48), FP64 filter bit-exact with the
oracle, renormalisation within 1e-12.
"""
import os

import numpy as np
import pytest

import arma_b200 as A
from arma_b200 import capi
import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DATA = os.path.join(ROOT, "arma_b200", "data")
FILES = {"p19937": os.path.join(DATA, "mt.dat"), "p521": os.path.join(DATA, "mt521.dat")}


def sets(name):
    path = FILES[name]
    return [A.mt_file_read(path, k) for k in range(A.mt_file_count(path))]


def oracle_params(p):
    return O.MtParams.from_buffer_copy(p)


@pytest.mark.parametrize("name", ["p19937", "p521"])
def test_words_and_noise_every_set(ctx, name):
    for k, p in enumerate(sets(name)):
        seed = 42 + k
        out = torch.zeros(6000, dtype=torch.int32, device="cuda")
        ctx.mt_genrand(p, seed, 6000, out.data_ptr())
        ctx.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.uint32),
                              O.mt_genrand(oracle_params(p), seed, 6000)), (name, k)
        n = 5001
        ref = O.white_noise(oracle_params(p), seed, 0.7, n)
        z = torch.zeros(n, dtype=torch.float64, device="cuda")
        ctx.white_noise(p, seed, 0.7, n, A.FP64, z.data_ptr())
        ctx.synchronize()
        got = z.cpu().numpy()
        rel = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)
        assert rel.max() <= 1e-15, (name, k, rel.max())


@pytest.mark.parametrize("name,which", [("p19937", [0, 7, 15]), ("p521", [0, 9])])
def test_jump_ahead_segments_every_characteristic_polynomial(ctx, name, which):
    """Streams longer than one 2^20-word segment start each segment from a
    window jumped ahead with the set's own characteristic polynomial."""
    all_sets = sets(name)
    n, offset = (1 << 21) + 3000, (1 << 20) - 1500
    for k in which:
        p = all_sets[k]
        out = torch.zeros(n, dtype=torch.int32, device="cuda")
        ctx.mt_genrand(p, 7 + k, n, out.data_ptr(), offset=offset)
        ctx.synchronize()
        ref = O.mt_genrand(oracle_params(p), 7 + k, offset + n)[offset:]
        assert np.array_equal(out.cpu().numpy().view(np.uint32), ref), (name, k)


@pytest.mark.parametrize("name,k", [("p19937", 3), ("p521", 4)])
def test_stream_chunks_continue_the_generator(ctx, name, k):
    """The serving layer carries each stream's generator from chunk to chunk
    by untempering the last nn words of a chunk's stream (rr = 23 for the
    p = 521 sets); three chunks equal one surface of the same length."""
    p = sets(name)[k]
    phi, var = A.ar_fit_analytic(A.ACF_STANDING, (4, 4, 4), 1.5, 0.8, [0.05] * 3, [0.5, 0.5])
    T, n2 = 16, (48, 64)
    outs = []
    with A.Server(chunk_slices=T, velocity=0, max_inflight=2) as srv:
        sid = srv.open_stream(*n2, phi, var, 0.0, p, 91)
        for _ in range(3):
            z = torch.empty((T,) + n2, dtype=torch.float32, device="cuda")
            srv.submit(sid, z.data_ptr(), 0, keep=(z,))
            outs.append(z)
        got = srv.wait(3)
        assert all(g["status"] == 0 for g in got)
        torch.cuda.synchronize()
    chunks = np.concatenate([z.cpu().numpy() for z in outs])
    ref = torch.empty((3 * T,) + n2, dtype=torch.float32, device="cuda")
    ctx.batch_generate([capi.make_surface(ref.shape, phi, var, 0.0, p, 91, ref.data_ptr())],
                       A.FP32C)
    ctx.synchronize()
    assert np.array_equal(chunks, ref.cpu().numpy())


def test_c1_plain_fp64_configuration(ctx):
    shape, order = (200, 40, 40), (7, 7, 7)
    acf = A.acf_eval(A.ACF_STANDING, order, 1.5, 0.8, [0.05] * 3, [0.5, 0.5])
    oacf = O.acf("standing_wave", order, 1.5, 0.8, [0.05] * 3, [0.5, 0.5])
    assert np.allclose(acf, oacf, rtol=1e-15, atol=1e-15)
    phi, var = A.ar_fit(acf, order, A.capi.FIT_CHOLESKY)
    ophi, ovar = O.ar_fit(oacf, order)  # the reference's dsysv (Bunch-Kaufman) semantics
    assert np.abs(phi - ophi).max() <= 1e-9 and abs(var - ovar) <= 1e-9 * abs(ovar)
    mt = sets("p19937")
    assert len(mt) == 16
    z = torch.empty(shape, dtype=torch.float64, device="cuda")
    s = capi.make_surface(shape, phi, var, 1.5, mt[0], 42, z.data_ptr())
    scale = ctx.batch_generate([s], A.FP64)[0]
    ctx.synchronize()
    eps = O.white_noise(oracle_params(mt[0]), 42, np.sqrt(var), int(np.prod(shape)))
    raw = O.ar_filter(eps.reshape(shape), phi)
    ref, ref_scale = O.variance_renorm(raw, 1.5)
    assert abs(scale - ref_scale) <= 1e-12 * ref_scale
    got = z.cpu().numpy()
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-12)
    # the filter itself is bit-exact: undo the (common) scale
    z2 = torch.as_tensor(eps.reshape(shape)).cuda()
    ctx.ar_filter(phi, shape, A.FP64, z2.data_ptr())
    ctx.synchronize()
    assert np.array_equal(z2.cpu().numpy(), raw)
