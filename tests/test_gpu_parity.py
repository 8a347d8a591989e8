"""GPU parity tests: every device row against the CPU oracle through the C ABI.

Tolerances (stated per test):
  * MT words: bit-exact.
  * white noise: the accepted-attempt pattern is bit-exact; values agree to
    a few ulp, <= 1e-15 relative (device log() vs glibc log()).
  * FP64 AR filter: bit-exact with the oracle given the same noise (same
    summation order, explicitly rounded operations).
  * FP32 compensated AR filter: RMS error <= 1e-5 relative to the FP64 result
    on the same noise (the precision target of the FP32 form); max-abs error
    reported.
  * renormalisation: 1e-12 relative.
  * NIT bisection: 2e-6 absolute (bisection tolerance 1e-6); NIT LUT: 5e-5.
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


def assert_noise_close(got, ref):
    """Same accepted attempts (no misalignment: the relative error would be
    O(1)) and values within a few ulp."""
    rel = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)
    assert rel.max() <= 1e-15, (rel.max(), int(np.argmax(rel)), int((rel > 1e-15).sum()))


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to(dtype).cuda().contiguous()


def test_mt_words_bit_exact(ctx, golden):
    p = A.mt19937_params()
    out = torch.zeros(4096, dtype=torch.int32, device="cuda")
    ctx.mt_genrand(p, 42, 4096, out.data_ptr())
    ctx.synchronize()
    got = out.cpu().numpy().view(np.uint32)
    assert np.array_equal(got, golden["mt19937_seed42"])
    # offset: words [1000, 1500)
    out2 = torch.zeros(500, dtype=torch.int32, device="cuda")
    ctx.mt_genrand(p, 42, 500, out2.data_ptr(), offset=1000)
    ctx.synchronize()
    assert np.array_equal(out2.cpu().numpy().view(np.uint32), golden["mt19937_seed42"][1000:1500])


def test_mt_other_parameter_set_and_seed(ctx):
    p = A.mt19937_params()
    q = capi.MtParams.from_buffer_copy(p)
    q.maskB, q.maskC = 0x9d2c5680 ^ 0x10, 0xefc60000
    for seed in (0, 7, 0xFFFFFFFF):
        out = torch.zeros(3000, dtype=torch.int32, device="cuda")
        ctx.mt_genrand(q, seed, 3000, out.data_ptr())
        ctx.synchronize()
        oq = O.MtParams.from_buffer_copy(q)
        assert np.array_equal(out.cpu().numpy().view(np.uint32), O.mt_genrand(oq, seed, 3000))


@pytest.mark.parametrize("n", [1, 2, 5001, 100000])
def test_white_noise(ctx, n):
    p = A.mt19937_params()
    ref = O.white_noise(O.mt19937_params(), 42, 0.5, n)
    out = torch.zeros(n, dtype=torch.float64, device="cuda")
    ctx.white_noise(p, 42, 0.5, n, A.FP64, out.data_ptr())
    ctx.synchronize()
    got = out.cpu().numpy()
    assert_noise_close(got, ref)
    # float output is the double value rounded
    outf = torch.zeros(n, dtype=torch.float32, device="cuda")
    ctx.white_noise(p, 42, 0.5, n, A.FP32C, outf.data_ptr())
    ctx.synchronize()
    assert np.array_equal(outf.cpu().numpy(), got.astype(np.float32))


def test_white_noise_golden(ctx, golden):
    out = torch.zeros(5001, dtype=torch.float64, device="cuda")
    ctx.white_noise(A.mt19937_params(), 42, 0.5, 5001, A.FP64, out.data_ptr())
    ctx.synchronize()
    assert_noise_close(out.cpu().numpy(), golden["wn_seed42"])


@pytest.mark.parametrize("case", ["333", "777"])
def test_ar64_bit_exact(ctx, golden, case):
    eps, phi = golden["ar_eps_" + case], golden["ar_phi_" + case]
    z = dev(eps)
    ctx.ar_filter(phi, eps.shape, A.FP64, z.data_ptr())
    ctx.synchronize()
    assert np.array_equal(z.cpu().numpy(), golden["ar_zeta_" + case])


@pytest.mark.parametrize("shape,order", [((1, 1, 1), (1, 1, 1)), ((5, 3, 2), (2, 3, 4)),
                                         ((9, 40, 7), (4, 2, 3)), ((30, 33, 65), (5, 5, 5))])
def test_ar64_ragged_and_edge(ctx, shape, order):
    rng = np.random.default_rng(sum(shape) + sum(order))
    phi = rng.uniform(-0.05, 0.05, order)
    phi.flat[0] = 0.0
    eps = rng.standard_normal(shape)
    z = dev(eps)
    ctx.ar_filter(phi, shape, A.FP64, z.data_ptr())
    ctx.synchronize()
    assert np.array_equal(z.cpu().numpy(), O.ar_filter(eps, phi))


def rel_err(a, b):
    d = a.astype(np.float64) - b
    return np.sqrt(np.mean(d * d)) / np.sqrt(np.mean(b * b)), np.abs(d).max()


@pytest.mark.parametrize("shape,order,kind", [
    ((24, 20, 20), (7, 7, 7), "standing"),
    ((40, 50, 70), (4, 6, 8), "standing"),
    ((64, 48, 40), (10, 10, 10), "propagating"),
    ((3, 17, 33), (3, 2, 5), "standing"),
])
def test_ar32c_vs_fp64(ctx, shape, order, kind):
    if kind == "standing":
        phi, var = A.ar_fit_analytic(A.ACF_STANDING, order, 1.5, 0.8, [0.05] * 3, [0.5, 0.5])
    else:
        phi, var = A.ar_fit_analytic(A.ACF_PROPAGATING, order, 1.0, 0.6, [0.04] * 3, [0.3, 0.2])
    eps = O.white_noise(O.mt19937_params(), 11, np.sqrt(var), int(np.prod(shape))).reshape(shape)
    ref = O.ar_filter(eps, phi)
    z = dev(eps.astype(np.float32), torch.float32)
    ctx.ar_filter(phi, shape, A.FP32C, z.data_ptr())
    ctx.synchronize()
    rms, mx = rel_err(z.cpu().numpy(), ref)
    assert rms <= 1e-5, (rms, mx)


def test_renorm(ctx, golden):
    z = dev(golden["ar_zeta_777"])
    s = ctx.variance_renorm(z.data_ptr(), z.shape, A.FP64, 1.5)
    assert abs(s - golden["renorm_scale_777"][0]) <= 1e-12 * s
    assert np.allclose(z.cpu().numpy(), golden["renorm_zeta_777"], rtol=1e-12, atol=0)


def test_nit_bisection(ctx, golden):
    sd = np.sqrt(1.5)
    for dist, params, key in [(A.NIT_GRAM_CHARLIER, [0.3, 3.2], "nit_gc"),
                              (A.NIT_SKEW_NORMAL, [0.0, 1.0, 1.5], "nit_sn")]:
        z = dev(golden["nit_in"])
        ctx.nit_apply(dist, params, sd, A.NIT_BISECTION, z.numel(), A.FP64, z.data_ptr(),
                      interval=(-5, 5))
        ctx.synchronize()
        assert np.abs(z.cpu().numpy() - golden[key]).max() <= 2e-6


def test_nit_lut(ctx, golden):
    sd = np.sqrt(1.5)
    for dist, params, key in [(A.NIT_GRAM_CHARLIER, [0.3, 3.2], "nit_gc"),
                              (A.NIT_SKEW_NORMAL, [0.0, 1.0, 1.5], "nit_sn")]:
        for prec, dt in [(A.FP64, torch.float64), (A.FP32C, torch.float32)]:
            z = dev(golden["nit_in"], dt)
            ctx.nit_apply(dist, params, sd, A.NIT_LUT, z.numel(), prec, z.data_ptr(),
                          lut_nodes=1024, lut_range=5.0)
            ctx.synchronize()
            assert np.abs(z.cpu().numpy() - golden[key]).max() <= 5e-5


def test_batch_fp64_matches_sequential_oracle(ctx):
    p = A.mt19937_params()
    shapes = [(20, 16, 24), (12, 33, 9), (30, 8, 8)]
    orders = [(3, 3, 3), (2, 4, 3), (4, 2, 2)]
    bufs, surfs, refs = [], [], []
    for k, (sh, od) in enumerate(zip(shapes, orders)):
        phi, var = A.ar_fit_analytic(A.ACF_STANDING, od, 1.5, 0.8, [0.05] * 3, [0.5, 0.5])
        b = torch.zeros(sh, dtype=torch.float64, device="cuda")
        bufs.append(b)
        surfs.append(capi.make_surface(sh, phi, var, 1.5, p, 42 + k, b.data_ptr()))
        eps = O.white_noise(O.mt19937_params(), 42 + k, np.sqrt(var), int(np.prod(sh))).reshape(sh)
        refs.append(O.variance_renorm(O.ar_filter(eps, phi), 1.5))
    scales = ctx.batch_generate(surfs, A.FP64)
    for b, (rz, rs), s in zip(bufs, refs, scales):
        assert abs(s - rs) <= 1e-12 * rs
        assert np.allclose(b.cpu().numpy(), rz, rtol=1e-12, atol=1e-12)


def test_batch_fp32c_alone_equals_in_batch(ctx):
    """Each surface of an FP32 batch is the same alone and in the mix."""
    p = A.mt19937_params()
    shapes = [(40, 64, 64), (25, 32, 96), (60, 20, 40), (16, 100, 33)]
    orders = [(4, 4, 4), (6, 4, 8), (3, 5, 4), (8, 8, 8)]
    fits = [A.ar_fit_analytic(A.ACF_STANDING, od, 1.5, 0.8, [0.05] * 3, [0.5, 0.5]) for od in orders]

    def run(idx):
        bufs, surfs = [], []
        for k in idx:
            b = torch.zeros(shapes[k], dtype=torch.float32, device="cuda")
            bufs.append(b)
            phi, var = fits[k]
            surfs.append(capi.make_surface(shapes[k], phi, var, 1.5, p, 100 + k, b.data_ptr()))
        ctx.batch_generate(surfs, A.FP32C)
        return [b.cpu().numpy() for b in bufs]

    together = run([0, 1, 2, 3])
    for k in range(4):
        alone = run([k])[0]
        assert np.array_equal(alone, together[k])
        # and against the FP64 oracle chain on the same noise
        phi, var = fits[k]
        eps = O.white_noise(O.mt19937_params(), 100 + k, np.sqrt(var),
                            int(np.prod(shapes[k]))).reshape(shapes[k])
        ref, _ = O.variance_renorm(O.ar_filter(eps, phi), 1.5)
        rms, mx = rel_err(alone, ref)
        assert rms <= 1e-5, (k, rms, mx)


def test_batch_host_buffers(ctx):
    p = A.mt19937_params()
    phi, var = A.ar_fit_analytic(A.ACF_STANDING, (3, 3, 3), 1.5, 0.8, [0.05] * 3, [0.5, 0.5])
    host = np.zeros((10, 12, 14), np.float64)
    s = capi.make_surface(host.shape, phi, var, 1.5, p, 5, host.ctypes.data)
    ctx.batch_generate([s], A.FP64, host=True)
    eps = O.white_noise(O.mt19937_params(), 5, np.sqrt(var), host.size).reshape(host.shape)
    ref, _ = O.variance_renorm(O.ar_filter(eps, phi), 1.5)
    assert np.allclose(host, ref, rtol=1e-12, atol=1e-12)


def test_batch_host_buffers_fp32_pipelined(ctx):
    """Six FP32 surfaces into host buffers (the grouped path that overlaps the
    device->host copies with the filtering) equal the same batch generated
    into device buffers, bit for bit, scales included."""
    import torch
    p = A.mt19937_params()
    shapes = [(40, 64, 96), (25, 32, 32), (60, 48, 40), (17, 100, 33), (33, 16, 128), (50, 70, 70)]
    fits = [A.ar_fit_analytic(A.ACF_STANDING if k % 2 else A.ACF_PROPAGATING, (4 + k % 3,) * 3,
                              1.5, 0.8, [0.05] * 3, [0.5, 0.5]) for k in range(len(shapes))]
    dev = [torch.empty(sh, dtype=torch.float32, device="cuda") for sh in shapes]
    sd = [capi.make_surface(sh, f[0], f[1], 1.5, p, 300 + k, b.data_ptr())
          for k, (sh, f, b) in enumerate(zip(shapes, fits, dev))]
    sc_dev = ctx.batch_generate(sd, A.FP32C)
    ctx.synchronize()
    host = [torch.zeros(sh, dtype=torch.float32).pin_memory() if k % 2 else np.zeros(sh, np.float32)
            for k, sh in enumerate(shapes)]
    ptr = [h.data_ptr() if k % 2 else h.ctypes.data for k, h in enumerate(host)]
    sh_ = [capi.make_surface(sh, f[0], f[1], 1.5, p, 300 + k, q)
           for k, (sh, f, q) in enumerate(zip(shapes, fits, ptr))]
    sc_host = ctx.batch_generate(sh_, A.FP32C, host=True)
    assert sc_host == sc_dev
    for k in range(len(shapes)):
        h = host[k].numpy() if k % 2 else host[k]
        assert np.array_equal(h, dev[k].cpu().numpy()), k


def test_short_noise_regeneration_is_exact(ctx):
    """With a polar-attempt margin of 0.5 every surface's noise runs short; the
    batched calls then generate such a surface again on its own (device
    buffers, the pipelined host-buffer path, the FP64 path and the MA model)
    and the results equal those at the default margin bit for bit."""
    import torch
    p = A.mt19937_params()
    shapes = [(30, 32, 48), (20, 64, 32), (25, 40, 40), (18, 33, 70), (22, 16, 64)]
    fits = [A.ar_fit_analytic(A.ACF_STANDING, (3 + k % 2,) * 3, 1.5, 0.8, [0.05] * 3, [0.5, 0.5])
            for k in range(len(shapes))]

    def run():
        out = []
        for prec, dt in ((A.FP32C, torch.float32), (A.FP64, torch.float64)):
            dev = [torch.empty(sh, dtype=dt, device="cuda") for sh in shapes]
            sd = [capi.make_surface(sh, f[0], f[1], 1.5, p, 500 + k, b.data_ptr())
                  for k, (sh, f, b) in enumerate(zip(shapes, fits, dev))]
            sc = ctx.batch_generate(sd, prec)
            ctx.synchronize()
            out.append(([b.cpu().numpy() for b in dev], sc))
        host = [np.zeros(sh, np.float32) for sh in shapes]
        sh_ = [capi.make_surface(sh, f[0], f[1], 1.5, p, 500 + k, h.ctypes.data)
               for k, (sh, f, h) in enumerate(zip(shapes, fits, host))]
        out.append(([h.copy() for h in host], ctx.batch_generate(sh_, A.FP32C, host=True)))
        theta, var, _ = A.ma_fit(np.exp(-np.add.outer(np.add.outer(np.arange(6), np.arange(6)),
                                                       np.arange(6)) * 0.7), (3, 3, 3))
        ma = [torch.empty(sh, dtype=torch.float32, device="cuda") for sh in shapes[:2]]
        sm = [capi.make_surface(sh, theta, var, 1.0, p, 700 + k, b.data_ptr())
              for k, (sh, b) in enumerate(zip(shapes[:2], ma))]
        out.append(([b.cpu().numpy() for b in ma], ctx.ma_generate(sm, A.FP32C)))
        return out

    base = run()
    try:
        ctx.set_noise_margin(0.5)
        short = run()
    finally:
        ctx.set_noise_margin(1.0)
    for (za, sa), (zb, sb) in zip(base, short):
        assert sa == sb
        for a, b in zip(za, zb):
            assert np.array_equal(a, b)
    with pytest.raises(capi.ArmaError):
        ctx.set_noise_margin(0.0)


@pytest.mark.parametrize("prec,dt", [(A.FP32C, "float32"), (A.FP64, "float64")])
def test_batch_nit_fused_equals_separate_passes(ctx, prec, dt):
    """The NIT table applied in the renormalisation's scale pass
    (arma_batch_generate_nit) equals the batch call followed by the
    standalone table NIT, bit for bit; a surface without NIT is untouched."""
    p = A.mt19937_params()
    shapes = [(20, 33, 50), (16, 64, 32), (12, 40, 40), (9, 17, 31), (10, 32, 32)]
    fits = [A.ar_fit_analytic(A.ACF_STANDING, (3, 3, 2 + k % 2), 1.5, 0.8, [0.05] * 3, [0.5, 0.5])
            for k in range(len(shapes))]
    specs = [(A.NIT_SKEW_NORMAL, [0.0, 1.0, 1.499]), (A.NIT_GRAM_CHARLIER, [0.3, 3.2, 0.0]),
             None, (A.NIT_SKEW_NORMAL, [0.0, 1.0, 1.499]), (A.NIT_GRAM_CHARLIER, [0.3, 3.2, 0.0])]
    tdt = getattr(torch, dt)

    def surfaces(bufs):
        return [capi.make_surface(sh, f[0], f[1], 1.5, p, 60 + k, b.data_ptr())
                for k, (sh, f, b) in enumerate(zip(shapes, fits, bufs))]

    fused = [torch.empty(sh, dtype=tdt, device="cuda") for sh in shapes]
    tables = [capi.nit_table(sp[0], sp[1], np.sqrt(1.5), 1024, 5.0) if sp else capi.nit_table()
              for sp in specs]
    sc1 = ctx.batch_generate_nit(surfaces(fused), prec, tables)
    sep = [torch.empty(sh, dtype=tdt, device="cuda") for sh in shapes]
    sc2 = ctx.batch_generate(surfaces(sep), prec)
    for sp, b in zip(specs, sep):
        if sp:
            ctx.nit_apply(sp[0], sp[1], float(np.sqrt(1.5)), A.NIT_LUT, b.numel(), prec, b.data_ptr(),
                          lut_nodes=1024, lut_range=5.0)
    ctx.synchronize()
    assert sc1 == sc2
    for a, b in zip(fused, sep):
        assert torch.equal(a, b)


def test_tuning_settings_do_not_change_results(ctx):
    """The MT segment length, the filter's CTAs per SM and the host-output
    group split change the speed only: the same batch comes out bit for bit
    equal under several settings, into device and into host buffers, and the
    autotuner's choice (cached per shape class) is one of them."""
    import torch
    sets = [A.mt_file_read(os.path.join(ROOT, "arma_b200", "data", "mt.dat"), k) for k in range(3)]
    shapes = [(60, 64, 96), (25, 32, 32), (90, 48, 64), (17, 100, 33), (33, 16, 128), (50, 70, 70)]
    fits = [A.ar_fit_analytic(A.ACF_STANDING if k % 2 else A.ACF_PROPAGATING, (4 + k % 3,) * 3,
                              1.5, 0.8, [0.05] * 3, [0.5, 0.5]) for k in range(len(shapes))]
    base = ctx.tuning()

    def run(t, host):
        ctx.set_tuning(t)
        if host:
            out = [np.zeros(sh, np.float32) for sh in shapes]
            ptr = [o.ctypes.data for o in out]
        else:
            out = [torch.empty(sh, dtype=torch.float32, device="cuda") for sh in shapes]
            ptr = [o.data_ptr() for o in out]
        sf = [capi.make_surface(sh, f[0], f[1], 1.5, sets[k % 3], 900 + k, q)
              for k, (sh, f, q) in enumerate(zip(shapes, fits, ptr))]
        sc = ctx.batch_generate(sf, A.FP32C, host=host)
        ctx.synchronize()
        return [o if host else o.cpu().numpy() for o in out], sc, sf

    try:
        ref, ref_sc, _ = run(base, False)
        variants = []
        for mt, ar, g, f in [(16, 1, 2, 0.5), (18, 2, 6, 0.06), (22, 0, 16, 0.03)]:
            t = capi.Tuning()
            t.mt_log2_segment, t.ar_ctas_per_sm, t.host_groups, t.host_first = mt, ar, g, f
            variants.append(t)
        for t in variants:
            for host in (False, True):
                got, sc, _ = run(t, host)
                assert sc == ref_sc
                for a, b in zip(got, ref):
                    assert np.array_equal(a, b), (t.as_dict(), host)
        bad = capi.Tuning()
        bad.mt_log2_segment, bad.ar_ctas_per_sm, bad.host_groups, bad.host_first = 12, 0, 4, 0.3
        with pytest.raises(capi.ArmaError):
            ctx.set_tuning(bad)
        keep, _, sf = run(base, True)  # the surfaces write into `keep`: it must stay alive
        chosen, ms = ctx.autotune(sf, A.FP32C, host=True)
        assert ms > 0.0 and 16 <= chosen.mt_log2_segment <= 22
        again, ms2 = ctx.autotune(sf, A.FP32C, host=True)
        assert ms2 == -1.0 and again.as_dict() == chosen.as_dict()
        del keep
        got, sc, _ = run(chosen, True)
        assert sc == ref_sc and all(np.array_equal(a, b) for a, b in zip(got, ref))
    finally:
        ctx.set_tuning(base)


def test_errors_are_reported(ctx):
    with pytest.raises(capi.ArmaError):
        ctx.ar_filter(np.zeros((2, 2, 2)), (0, 4, 4), A.FP64, 0)
    with pytest.raises(capi.ArmaError):
        ctx.white_noise(A.mt19937_params(), 1, -1.0, 10, A.FP64, 0)


def test_velocity_fp64_golden(ctx, golden):
    """Linear solver, FP64: equal to the oracle up to FFT rounding
    (tolerance 1e-9 of the largest |phi|)."""
    zeta = golden["vel_zeta"]
    ref = golden["vel_phi"]
    z = dev(zeta)
    out = torch.zeros(ref.shape, dtype=torch.float64, device="cuda")
    ctx.velocity_linear(z.data_ptr(), zeta.shape, A.FP64, (1.0, 1.0, 1.0), 12.0,
                        [0.0, -1.0, -2.0], [3, 10], out.data_ptr())
    got = out.cpu().numpy()
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() <= 1e-9 * scale


@pytest.mark.parametrize("shape,depth,zs,tidx", [
    ((12, 32, 64), np.inf, [0.0, -1.0, -2.0, -4.0], [0, 5, 11]),
    ((6, 16, 16), 12.0, [0.0, -3.0], [0, 1, 4, 5]),
    ((3, 64, 32), np.inf, [0.0], [0, 1, 2]),
])
def test_velocity_vs_oracle(ctx, shape, depth, zs, tidx):
    """FP64 within 1e-9 and FP32 within 2e-4 of max|phi| against the oracle,
    including the first/last slice one-sided derivatives and infinite depth."""
    phi, var = A.ar_fit_analytic(A.ACF_PROPAGATING, (3, 3, 3), 1.0, 0.6, [0.04] * 3, [0.3, 0.2])
    eps = O.white_noise(O.mt19937_params(), 3, np.sqrt(var), int(np.prod(shape))).reshape(shape)
    zeta = O.ar_filter(eps, phi)
    ref = O.velocity_linear(zeta, (1.0, 1.0, 1.0), depth, zs, tidx)
    scale = np.abs(ref).max()
    for prec, dt, tol in [(A.FP64, torch.float64, 1e-9), (A.FP32C, torch.float32, 2e-4)]:
        z = dev(zeta, dt)
        out = torch.zeros(ref.shape, dtype=dt, device="cuda")
        ctx.velocity_linear(z.data_ptr(), shape, prec, (1.0, 1.0, 1.0), depth, zs, tidx,
                            out.data_ptr())
        got = out.cpu().numpy().astype(np.float64)
        assert np.abs(got - ref).max() <= tol * scale, (prec, np.abs(got - ref).max() / scale)


@pytest.mark.parametrize("shape,depth,zs,tidx", [
    ((4, 256, 256), np.inf, [0.0, -1.0, -2.0], [0, 1, 3]),  # two-CTA cluster kernel
    ((4, 256, 128), 12.0, [0.0, -1.0], [0, 2, 3]),          # 32768 points in one CTA
    ((4, 128, 256), np.inf, [0.0], [1, 2]),
    ((4, 32, 16), 12.0, [0.0, -2.0], [0, 3]),               # the smallest real-input shape
])
def test_velocity_real_input_kernels_vs_oracle(ctx, shape, depth, zs, tidx):
    """The FP32 real-input kernels (power-of-two slices, rows packed in pairs,
    even part of the window) within 2e-4 of max|phi| of the oracle, with
    several depths (the spectrum reloaded per depth) and both depth kinds."""
    phi, var = A.ar_fit_analytic(A.ACF_PROPAGATING, (3, 3, 3), 1.0, 0.6, [0.04] * 3, [0.3, 0.2])
    eps = O.white_noise(O.mt19937_params(), 5, np.sqrt(var), int(np.prod(shape))).reshape(shape)
    zeta = O.ar_filter(eps, phi)
    ref = O.velocity_linear(zeta, (1.0, 1.0, 1.0), depth, zs, tidx)
    scale = np.abs(ref).max()
    z = dev(zeta, torch.float32)
    out = torch.zeros(ref.shape, dtype=torch.float32, device="cuda")
    ctx.velocity_linear(z.data_ptr(), shape, A.FP32C, (1.0, 1.0, 1.0), depth, zs, tidx,
                        out.data_ptr())
    got = out.cpu().numpy().astype(np.float64)
    assert np.abs(got - ref).max() <= 2e-4 * scale, np.abs(got - ref).max() / scale


@pytest.mark.parametrize("offset,n", [(0, 5_000_000), (3_000_000, 1_500_000), (1_048_570, 20)])
def test_mt_jump_ahead_segments_bit_exact(ctx, offset, n):
    """Streams longer than one 2^20-word segment are split by jump-ahead;
    every word must equal the sequential generator's."""
    p = A.mt19937_params()
    out = torch.zeros(n, dtype=torch.int32, device="cuda")
    ctx.mt_genrand(p, 12345, n, out.data_ptr(), offset=offset)
    ctx.synchronize()
    ref = O.std_mt19937(12345, offset + n)[offset:]
    assert np.array_equal(out.cpu().numpy().view(np.uint32), ref)


def test_mt_non_primitive_set_falls_back_to_sequential(ctx):
    """A parameter set whose recurrence is not full-period has no jump table;
    long streams are then generated sequentially, still bit-exact."""
    p = A.mt19937_params()
    q = capi.MtParams.from_buffer_copy(p)
    q.aaa = 0x12345678
    n = (1 << 20) + 4096
    out = torch.zeros(n, dtype=torch.int32, device="cuda")
    ctx.mt_genrand(q, 9, n, out.data_ptr())
    ctx.synchronize()
    oq = O.MtParams.from_buffer_copy(q)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), O.mt_genrand(oq, 9, n))


def test_white_noise_long_stream(ctx):
    n = 3_000_001
    ref = O.white_noise(O.mt19937_params(), 77, 1.3, n)
    out = torch.zeros(n, dtype=torch.float64, device="cuda")
    ctx.white_noise(A.mt19937_params(), 77, 1.3, n, A.FP64, out.data_ptr())
    ctx.synchronize()
    assert_noise_close(out.cpu().numpy(), ref)


def test_velocity_batch_equals_single_calls(ctx):
    """The batched velocity entry point (several surfaces of one slice shape,
    different lengths and slice lists) gives exactly the per-surface results,
    in FP32 (fused kernel) and FP64 (FFT passes through global memory)."""
    phi, var = A.ar_fit_analytic(A.ACF_STANDING, (4, 4, 4), 1.5, 0.8, [0.05] * 3, [0.5, 0.5])
    specs = [((10, 32, 64), [0, 3, 9]), ((6, 32, 64), [5, 1]), ((3, 32, 64), [2])]
    for prec, dt in [(A.FP32C, torch.float32), (A.FP64, torch.float64)]:
        zs, outs, jobs = [], [], []
        for k, (shape, tidx) in enumerate(specs):
            eps = O.white_noise(O.mt19937_params(), 7 + k, np.sqrt(var), int(np.prod(shape)))
            z = dev(O.ar_filter(eps.reshape(shape), phi), dt)
            o = torch.zeros((len(tidx), 2) + shape[1:], dtype=dt, device="cuda")
            zs.append(z)
            outs.append(o)
            jobs.append((z.data_ptr(), o.data_ptr(), shape[0], tidx, 1.0))
        ctx.velocity_linear_batch(jobs, 32, 64, prec, 12.0, [0.0, -2.0])
        for (shape, tidx), z, o in zip(specs, zs, outs):
            ref = torch.zeros_like(o)
            ctx.velocity_linear(z.data_ptr(), shape, prec, (1.0, 1.0, 1.0), 12.0, [0.0, -2.0], tidx,
                                ref.data_ptr())
            ctx.synchronize()
            assert torch.equal(o, ref)


@pytest.mark.parametrize("prec,dt", [(A.FP32C, torch.float32), (A.FP64, torch.float64)])
def test_velocity_independent_of_line_pieces(ctx, prec, dt):
    """factor_waves cuts each slice's lines into fewer pieces the more slices a
    launch holds (here 3 and 7 pieces per line on the two axes for 3 slices,
    1 and 2 for 1600, with 148 SMs), and joins the pieces' walks afterwards:
    the potentials of every slice are the same bits whichever cut was taken."""
    shape = (1600, 32, 64)
    phi, var = A.ar_fit_analytic(A.ACF_PROPAGATING, (2, 2, 2), 1.0, 0.6, [0.04] * 3, [0.3, 0.2])
    eps = O.white_noise(O.mt19937_params(), 11, np.sqrt(var), int(np.prod(shape))).reshape(shape)
    z = dev(O.ar_filter(eps, phi), dt)
    every = list(range(shape[0]))
    whole = torch.zeros((shape[0], 1) + shape[1:], dtype=dt, device="cuda")
    ctx.velocity_linear(z.data_ptr(), shape, prec, (1.0, 1.0, 1.0), np.inf, [0.0], every,
                        whole.data_ptr())
    for t0 in (0, 1, 797, 1597):
        part = torch.zeros((3, 1) + shape[1:], dtype=dt, device="cuda")
        ctx.velocity_linear(z.data_ptr(), shape, prec, (1.0, 1.0, 1.0), np.inf, [0.0],
                            [t0, t0 + 1, t0 + 2], part.data_ptr())
        ctx.synchronize()
        assert torch.equal(part, whole[t0:t0 + 3]), t0


@pytest.mark.parametrize("shape,depth,zs", [
    ((8, 40, 24), 12.0, [0.0, -3.0]),     # 40 = 4.2.5, 24 = 4.2.3
    ((6, 20, 30), np.inf, [0.0]),         # 30 = 2.3.5
    ((5, 12, 100), np.inf, [0.0, -1.0]),  # 100 = 4.5.5
    ((4, 28, 36), 12.0, [0.0]),           # 28 = 4.7, 36 = 4.3.3
    ((4, 13, 16), np.inf, [0.0]),         # 13: direct-summation radix
    ((3, 200, 100), np.inf, [0.0]),       # FP32 over 16384 points: banded passes
])
def test_velocity_mixed_radix_vs_oracle(ctx, shape, depth, zs):
    """Slice sides that are not powers of two (the reference's GSL mixed-radix
    FFT takes any length): FP64 within 1e-9 and FP32 within 2e-4 of max|phi|
    against the oracle's direct DFT."""
    phi, var = A.ar_fit_analytic(A.ACF_STANDING, (3, 3, 3), 1.5, 0.8, [0.05] * 3, [0.5, 0.5])
    eps = O.white_noise(O.mt19937_params(), 5, np.sqrt(var), int(np.prod(shape))).reshape(shape)
    zeta = O.ar_filter(eps, phi)
    tidx = list(range(shape[0]))
    ref = O.velocity_linear(zeta, (1.0, 1.0, 1.0), depth, zs, tidx)
    scale = np.abs(ref).max()
    for prec, dt, tol in [(A.FP64, torch.float64, 1e-9), (A.FP32C, torch.float32, 2e-4)]:
        z = dev(zeta, dt)
        out = torch.zeros(ref.shape, dtype=dt, device="cuda")
        ctx.velocity_linear(z.data_ptr(), shape, prec, (1.0, 1.0, 1.0), depth, zs, tidx,
                            out.data_ptr())
        got = out.cpu().numpy().astype(np.float64)
        assert np.abs(got - ref).max() <= tol * scale, (prec, np.abs(got - ref).max() / scale)


@pytest.mark.parametrize("shape,depth,zs,amp", [
    ((8, 32, 24), 12.0, [0.0, -2.0], 1.0),
    ((6, 20, 30), np.inf, [0.0], 3.0),       # steep: slopes of order one
    ((4, 200, 100), np.inf, [0.0, -1.0], 2.0),
])
def test_velocity_high_amplitude_vs_oracle(ctx, shape, depth, zs, amp):
    """High_amplitude_solver: the complex slope-corrected input through the
    same window and FFTs; FP64 within 1e-9 and FP32 within 2e-4 of max|phi|,
    with non-unit grid steps for the slopes."""
    phi, var = A.ar_fit_analytic(A.ACF_STANDING, (3, 3, 3), 1.5, 0.8, [0.05] * 3, [0.5, 0.5])
    eps = O.white_noise(O.mt19937_params(), 8, np.sqrt(var), int(np.prod(shape))).reshape(shape)
    zeta = amp * O.ar_filter(eps, phi)
    delta = (0.5, 0.8, 1.25)
    tidx = list(range(shape[0]))
    ref = O.velocity_high_amplitude(zeta, delta, depth, zs, tidx)
    scale = np.abs(ref).max()
    for prec, dt, tol in [(A.FP64, torch.float64, 1e-9), (A.FP32C, torch.float32, 2e-4)]:
        z = dev(zeta, dt)
        out = torch.zeros(ref.shape, dtype=dt, device="cuda")
        ctx.velocity_linear(z.data_ptr(), shape, prec, delta, depth, zs, tidx, out.data_ptr(),
                            high_amplitude=True)
        got = out.cpu().numpy().astype(np.float64)
        assert np.abs(got - ref).max() <= tol * scale, (prec, np.abs(got - ref).max() / scale)


@pytest.mark.gpu
def test_auto_covariance_device(ctx):
    """arma_auto_covariance_device against the host FP64 form (which
    tests/test_acf_gen.py pins to the reference's CosineNoDecay case and to
    numpy) on odd, prime and the generator's 2 n + 1 sides, from FP64 and FP32
    input."""
    rng = np.random.default_rng(11)
    for shape in [(7, 11, 13), (21, 21, 21), (65, 33, 17), (1, 64, 2), (40, 40, 40), (5, 129, 3)]:
        w = rng.standard_normal(shape)
        host = A.auto_covariance(w)
        for prec, dt in [(A.FP64, torch.float64), (A.FP32C, torch.float32)]:
            src = torch.tensor(w, dtype=dt, device="cuda")
            out = torch.empty(shape, dtype=torch.float64, device="cuda")
            ctx.auto_covariance(src.data_ptr(), shape, prec, out.data_ptr())
            ctx.synchronize()
            ref = host if prec == A.FP64 else A.auto_covariance(src.cpu().double().numpy())
            assert np.max(np.abs(out.cpu().numpy() - ref)) <= 1e-12 * np.max(np.abs(ref)), shape
    with pytest.raises(capi.ArmaError) as e:
        big = torch.zeros((2, 2, 1025), dtype=torch.float64, device="cuda")
        ctx.auto_covariance(big.data_ptr(), big.shape, A.FP64, big.data_ptr())
    assert e.value.code == -8


@pytest.mark.gpu
def test_bounded_wait_times_out_and_context_survives(ctx):
    """A device wait that runs out (a tile flag nothing publishes) comes back
    as ARMA_ETIMEDOUT after its poll limit, and the context keeps working."""
    import time
    t0 = time.perf_counter()
    with pytest.raises(capi.ArmaError) as e:
        ctx.selftest_wait()
    assert e.value.code == -4
    assert time.perf_counter() - t0 < 30.0
    phi, var = A.ar_fit_analytic(A.ACF_STANDING, (3, 3, 3), 1.5, 0.8, [0.05] * 3, [0.5, 0.5])
    z = torch.empty((20, 16, 24), dtype=torch.float32, device="cuda")
    ctx.batch_generate([capi.make_surface(z.shape, phi, var, 1.5, A.mt19937_params(), 7,
                                          z.data_ptr())], A.FP32C)
    ctx.synchronize()
    assert torch.isfinite(z).all()
