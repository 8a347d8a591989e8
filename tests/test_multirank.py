"""The N > 1 path on CPU: two gloo ranks, as `torchrun --nproc-per-node 2
bench.py` would run them.  The path shards by surface: every rank draws its
own batch (rank-dependent generator and seeds), no data crosses ranks, and
the only collectives are the barrier and the max-over-ranks reduction of the
timed region, from which the whole-job points/s is formed."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import sys
    from datetime import timedelta
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        batch = bench.make_batch(rank, 16)
        elapsed = 1.0 + rank  # rank 1 is the slow one
        dist.barrier()
        mx = bench.reduce_max(elapsed, "cpu")
        seeds = torch.tensor([s["seed"] for s in batch], dtype=torch.int64)
        gathered = [torch.zeros_like(seeds) for _ in range(world)]
        dist.all_gather(gathered, seeds)
        q.put((rank, mx, bench.points(batch), [g.tolist() for g in gathered],
               bench.shard_value(bench.points(batch), 3, mx, world)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_by_surface():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, mx0, n0, seeds, v0), (r1, mx1, n1, _, v1) = res
    assert mx0 == mx1 == 2.0                       # max over ranks, seen by both
    assert not set(seeds[0]) & set(seeds[1])       # independent realisations
    assert v0 == pytest.approx(2 * n0 * 3 / 2.0)   # whole-job points/s at the slowest rank
    assert n0 != n1 or seeds[0] != seeds[1]


def _scaled(spec):
    """A bench surface scaled down for the CPU oracle (same seed, parameter
    set, order and ACF; shape divided by 16 in t and 8 in x and y)."""
    nt, nx, ny = spec["shape"]
    return dict(spec, shape=(max(8, nt // 16), max(4, nx // 8), max(4, ny // 8)))


def _generate(spec, sets):
    """One surface the way every rank's device path makes it: white noise from
    the surface's own parameter set and seed, the AR filter, renormalisation."""
    import numpy as np
    import oracle as O
    n = int(np.prod(spec["shape"]))
    p = O.MtParams.from_buffer_copy(sets[spec["mtset"] % len(sets)])
    eps = O.white_noise(p, spec["seed"], float(np.sqrt(spec["var"])), n).reshape(spec["shape"])
    z, _ = O.variance_renorm(O.ar_filter(eps, spec["phi"]), spec["acf0"])
    return z


def _shard_rank(rank, world, port, q):
    import hashlib
    import sys
    from datetime import timedelta
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        sets = bench.mt_sets()
        batch = bench.fit_batch([_scaled(s) for s in bench.make_batch(rank, 4)])
        mine = [(s["seed"], s["mtset"], hashlib.sha256(_generate(s, sets).tobytes()).hexdigest())
                for s in batch]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        q.put((rank, gathered))
    finally:
        dist.destroy_process_group()


def test_sharded_surfaces_equal_a_one_rank_run():
    """Two gloo ranks each generate their own surfaces (the CPU oracle standing
    in for the device path).  The union of what they produce equals the same
    surfaces generated one after another in this single process, and no seed
    repeats across ranks."""
    import hashlib
    import sys
    sys.path.insert(0, ROOT)
    import bench
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in procs), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    gathered = res[0][1]
    assert gathered == res[1][1]  # both ranks hold the same view
    sets = bench.mt_sets()
    for rank in range(2):
        batch = bench.fit_batch([_scaled(s) for s in bench.make_batch(rank, 4)])
        one = [(s["seed"], s["mtset"], hashlib.sha256(_generate(s, sets).tobytes()).hexdigest())
               for s in batch]
        assert [tuple(x) for x in gathered[rank]] == one
    seeds = [x[0] for r in gathered for x in r]
    assert len(seeds) == len(set(seeds))
