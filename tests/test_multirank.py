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
