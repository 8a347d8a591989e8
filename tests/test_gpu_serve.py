"""Serving layer on the GPU: device-resident streams, chunk continuity,
continuous batching, admission by HBM footprint.

Exactness claims (all bit-exact, FP32 outputs):
  * a stream's chunks concatenated == one surface of the same total length
    generated in one batch call with the same seed (no renormalisation);
  * chunk 0 with renormalisation == the batch call on a chunk-sized surface;
    later chunks == the long surface's slices times the first chunk's scale;
  * a chunk's velocity potentials == the linear solver run on the history +
    chunk slices;
  * a stream served alone == the same stream served among others (zeta and
    velocity), whatever the batch composition;
  * a forced noise redo (too few polar attempts) changes nothing.
"""
import numpy as np
import pytest

import arma_b200 as A

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

MT = None


def mt():
    global MT
    if MT is None:
        MT = A.mt19937_params()
    return MT


def model(order=(5, 4, 4), kind=A.ACF_STANDING):
    if kind == A.ACF_STANDING:
        return A.ar_fit_analytic(kind, order, 1.5, 0.8, [0.05] * 3, [0.5, 0.5])
    return A.ar_fit_analytic(kind, order, 1.0, 0.6, [0.04] * 3, [0.3, 0.2])


def one_shot(ctx, shape, phi, var, acf0, seed):
    z = torch.empty(shape, dtype=torch.float32, device="cuda")
    s = A.capi.make_surface(shape, phi, var, acf0, mt(), seed, z.data_ptr())
    scale = ctx.batch_generate([s], A.FP32C)[0]
    ctx.synchronize()
    return z.cpu().numpy(), scale


def run_stream(srv, sid, nchunks, shape2, T, nz=0):
    outs = []
    for _ in range(nchunks):
        z = torch.empty((T,) + shape2, dtype=torch.float32, device="cuda")
        v = torch.empty((T, nz) + shape2, dtype=torch.float32, device="cuda") if nz else None
        srv.submit(sid, z.data_ptr(), v.data_ptr() if nz else 0, keep=(z, v))
        outs.append((z, v))
    return outs


def test_chunks_equal_one_shot(ctx):
    phi, var = model()
    T, n2 = 16, (64, 96)
    with A.Server(chunk_slices=T, velocity=0, max_inflight=2) as srv:
        sid = srv.open_stream(*n2, phi, var, 0.0, mt(), 77)
        outs = run_stream(srv, sid, 3, n2, T)
        got = srv.wait(3)
        assert all(g["status"] == 0 for g in got)
        assert [g["chunk"] for g in got] == [0, 1, 2]
        torch.cuda.synchronize()
        chunks = np.concatenate([z.cpu().numpy() for z, _ in outs])
    ref, _ = one_shot(ctx, (3 * T,) + n2, phi, var, 0.0, 77)
    assert np.array_equal(chunks, ref)


def test_renormalised_chunks(ctx):
    phi, var = model((6, 6, 6), A.ACF_PROPAGATING)
    T, n2 = 32, (64, 64)
    with A.Server(chunk_slices=T, velocity=0) as srv:
        sid = srv.open_stream(*n2, phi, var, 1.0, mt(), 5)
        outs = run_stream(srv, sid, 2, n2, T)
        srv.wait(2)
        torch.cuda.synchronize()
        c0, c1 = (z.cpu().numpy() for z, _ in outs)
    ref0, scale = one_shot(ctx, (T,) + n2, phi, var, 1.0, 5)
    assert np.array_equal(c0, ref0)
    raw, _ = one_shot(ctx, (2 * T,) + n2, phi, var, 0.0, 5)
    assert np.array_equal(c1, (raw[T:].astype(np.float64) * scale).astype(np.float32))


def test_chunk_velocity_is_the_solver_on_history_and_chunk(ctx):
    phi, var = model((4, 4, 4))
    T, n2, H = 16, (64, 64), 3
    delta = (1.0, 1.0, 1.0)
    with A.Server(chunk_slices=T, velocity=1, z_levels=[0.0, -1.0]) as srv:
        sid = srv.open_stream(*n2, phi, var, 0.0, mt(), 11, delta)
        outs = run_stream(srv, sid, 2, n2, T, nz=2)
        srv.wait(2)
        torch.cuda.synchronize()
    (z0, v0), (z1, v1) = outs
    for zz, vv, hist in [(z0, v0, None), (z1, v1, z0[-H:])]:
        buf = zz if hist is None else torch.cat([hist, zz]).contiguous()
        t0 = 0 if hist is None else H
        ref = torch.empty((T, 2) + n2, dtype=torch.float32, device="cuda")
        ctx.velocity_linear(buf.data_ptr(), buf.shape, A.FP32C, delta, float("inf"), [0.0, -1.0],
                            list(range(t0, t0 + T)), ref.data_ptr())
        ctx.synchronize()
        assert torch.equal(vv, ref)


def _mix(srv, target, others, rng):
    """Submit the target stream's chunks interleaved with other streams'
    chunks, some while earlier batches are still on the GPU."""
    outs, keep = [], []
    for c in range(3):
        for sid, n2 in others:
            for _ in range(int(rng.integers(0, 3))):
                z = torch.empty((64,) + n2, dtype=torch.float32, device="cuda")
                v = torch.empty((64, 1) + n2, dtype=torch.float32, device="cuda")
                srv.submit(sid, z.data_ptr(), v.data_ptr(), keep=(z, v))
                keep.append((z, v))
        outs += run_stream(srv, target[0], 1, target[1], 64, nz=1)
    return outs, keep


def test_alone_equals_in_mix(ctx):
    phi, var = model((8, 8, 8))
    n2 = (128, 128)
    with A.Server(chunk_slices=64, velocity=1, z_levels=[0.0], max_inflight=1) as srv:
        sid = srv.open_stream(*n2, phi, var, 1.5, mt(), 2024)
        alone = run_stream(srv, sid, 3, n2, 64, nz=1)
        srv.wait(3)
        torch.cuda.synchronize()
        alone = [(z.cpu(), v.cpu()) for z, v in alone]
    rng = np.random.default_rng(1)
    with A.Server(chunk_slices=64, velocity=1, z_levels=[0.0], max_inflight=3) as srv:
        others = []
        for k, side in enumerate([64, 256, 128, 64, 128]):
            o = (8, 8, 8) if k % 2 else (6, 6, 6)
            p, v = model(o, A.ACF_PROPAGATING if k % 2 else A.ACF_STANDING)
            others.append((srv.open_stream(side, side, p, v, 1.0, mt(), 100 + k), (side, side)))
        sid = srv.open_stream(*n2, phi, var, 1.5, mt(), 2024)
        mixed, keep = _mix(srv, (sid, n2), others, rng)
        srv.wait(3 + len(keep))
        st = srv.stats()
        torch.cuda.synchronize()
    assert st["batches"] < st["completed"]  # requests shared batches
    for (za, va), (zm, vm) in zip(alone, mixed):
        assert torch.equal(za, zm.cpu())
        assert torch.equal(va, vm.cpu())


def test_forced_noise_redo_is_exact(ctx):
    phi, var = model()
    T, n2 = 16, (64, 64)
    res = []
    for margin in (1.0, 0.5):
        with A.Server(chunk_slices=T, velocity=0, noise_margin=margin) as srv:
            sid = srv.open_stream(*n2, phi, var, 1.5, mt(), 9)
            outs = run_stream(srv, sid, 3, n2, T)
            srv.wait(3)
            torch.cuda.synchronize()
            res.append((np.concatenate([z.cpu().numpy() for z, _ in outs]), srv.stats()["redone"]))
    assert res[0][1] == 0 and res[1][1] >= 3
    assert np.array_equal(res[0][0], res[1][0])


def test_admission_by_hbm_footprint():
    phi, var = model()
    T, n2 = 16, (64, 64)
    with A.Server(chunk_slices=T, velocity=0) as srv:
        sid = srv.open_stream(*n2, phi, var, 0.0, mt(), 1)
        run_stream(srv, sid, 1, n2, T)
        srv.wait(1)
        one = srv.stats()["resident_bytes"]
    assert one > 0
    with A.Server(chunk_slices=T, velocity=0, hbm_budget=one + one // 2) as srv:
        s1 = srv.open_stream(*n2, phi, var, 0.0, mt(), 1)
        s2 = srv.open_stream(*n2, phi, var, 0.0, mt(), 2)
        keep = run_stream(srv, s1, 1, n2, T) + run_stream(srv, s2, 1, n2, T)
        first = srv.wait(1)
        assert first[0]["stream"] == s1
        assert srv.poll(8, 500) == []          # s2 waits for memory
        st = srv.stats()
        assert st["pending"] == 1 and st["resident_streams"] == 1
        srv.close_stream(s1)                   # frees s1's state
        second = srv.wait(1)
        assert second[0]["stream"] == s2 and second[0]["status"] == 0
        with pytest.raises(A.ArmaError) as e:  # can never fit
            srv.open_stream(256, 256, phi, var, 0.0, mt(), 3)
        assert e.value.code == -3
        del keep


def test_output_memory_kinds(ctx):
    phi, var = model()
    T, n2 = 16, (64, 64)
    with A.Server(chunk_slices=T, velocity=0) as srv:
        sid = srv.open_stream(*n2, phi, var, 0.0, mt(), 3)
        host = np.empty((T,) + n2, np.float32)
        with pytest.raises(A.ArmaError) as e:
            srv.submit(sid, host.ctypes.data)
        assert e.value.code == -1 and "page-locked" in str(e.value)
        pinned = torch.empty((T,) + n2, dtype=torch.float32).pin_memory()
        srv.submit(sid, pinned.data_ptr(), keep=pinned)
        srv.wait(1)
    ref, _ = one_shot(ctx, (T,) + n2, phi, var, 0.0, 3)
    assert np.array_equal(pinned.numpy(), ref)


def test_open_rejects_bad_streams():
    phi, var = model()
    with A.Server(chunk_slices=8, velocity=1) as srv:
        with pytest.raises(A.ArmaError) as e:
            srv.open_stream(67, 64, phi, var, 0.0, mt(), 1)   # prime side > 64: no FFT plan
        assert e.value.code == -8
        big, bv = model((13, 4, 4))
        with pytest.raises(A.ArmaError) as e:
            srv.open_stream(64, 64, big, bv, 0.0, mt(), 1)     # history > chunk
        assert e.value.code == -1


def test_router_places_by_stream_state_and_serves_exactly(ctx):
    """Two replicas on one device: streams go to the replica with the least
    stream state (nx * ny * (pt - 1 + 2 T) points), ids carry the replica in
    their top 8 bits, one poll merges both replicas' completions, and every
    stream's chunks equal the one-shot surface of the same seed."""
    phi, var = model()                      # pt = 5
    T = 16
    sizes = [(128, 128), (64, 64), (64, 64), (64, 64), (64, 96)]
    with A.Router(devices=[0, 0], chunk_slices=T, velocity=0, max_inflight=2) as r:
        assert r.replicas() == 2
        sids = [r.open_stream(*n2, phi, var, 0.0, mt(), 40 + k) for k, n2 in enumerate(sizes[:4])]
        # 128^2 x 36 = 589,824 on replica 0; each 64^2 x 36 = 147,456 to replica 1
        assert [r.placement(s) for s in sids] == [(0, 0), (1, 0), (1, 0), (1, 0)]
        assert [s >> 56 for s in sids] == [0, 1, 1, 1]
        r.close_stream(sids[0])             # replica 0 now holds nothing
        sids[0] = r.open_stream(*sizes[4], phi, var, 0.0, mt(), 44)
        assert r.placement(sids[0]) == (0, 0)
        outs = {s: run_stream(r, s, 2, n2, T) for s, n2 in zip(sids, [sizes[4]] + sizes[1:4])}
        got = r.wait(2 * len(sids))
        # a closed stream's state is reclaimed by its replica's serving thread
        assert r.stats(0)["streams"] == 1 and r.stats(1)["streams"] == 3
        assert all(g["status"] == 0 for g in got)
        assert sorted(g["stream"] for g in got) == sorted(sids * 2)
        assert all(g["request"] >> 56 == g["stream"] >> 56 for g in got)
        torch.cuda.synchronize()
        chunks = {s: np.concatenate([z.cpu().numpy() for z, _ in o]) for s, o in outs.items()}
        with pytest.raises(A.ArmaError):
            r.placement((1 << 56) | 999)       # no such stream on replica 1
    seeds = [44, 41, 42, 43]
    for s, n2, seed in zip(sids, [sizes[4]] + sizes[1:4], seeds):
        ref, _ = one_shot(ctx, (2 * T,) + n2, phi, var, 0.0, seed)
        assert np.array_equal(chunks[s], ref)
