"""The multi-rank path on CPU: two gloo ranks, no GPU.

Covers what bench.py does under torchrun: per-rank shards and seeds, the
max-over-ranks timing reduction, and that the union of per-rank shard results
equals the single-process result (the transform has no cross-signal exchange,
so sharding must not change any output bit).  The per-signal transform here is
the CPU oracle, standing in for the GPU on a machine without one.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp

from mpfft_b200.dist import max_over_ranks, rank_seed, shard_range


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, n, p, total, q):
    import sys
    from datetime import timedelta

    import torch.distributed as dist

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from oracle import oracle as O

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        start, stop = shard_range(total, rank, world)
        f = O.MpFFT(n, p)
        mine = []
        for sig in range(start, stop):
            xr, xi = O.mp_pair(n, p)
            O.fill_uniform(xr, xi, 1000 + sig)
            yr, yi = O.mp_pair(n, p)
            f(xr, xi, yr, yi)
            mine.append((sig, yr.hex(), yi.hex()))
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        t = max_over_ranks(0.25 * (rank + 1))
        if rank == 0:
            q.put((gathered, t, rank_seed(7, 1)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_shard_range_partitions():
    for total in (0, 1, 5, 10, 1023):
        for world in (1, 2, 3, 8):
            got = [shard_range(total, r, world) for r in range(world)]
            assert got[0][0] == 0 and got[-1][1] == total
            assert all(a[1] == b[0] for a, b in zip(got, got[1:]))
            sizes = [b - a for a, b in got]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(4, 2, 2)


def test_two_gloo_ranks_shard_and_reduce(orc):
    n, p, total, world = 16, 64, 5, 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, n, p, total, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    gathered, tmax, seed = q.get(timeout=120)
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    assert tmax == 0.5 and seed == 8
    got = sorted(item for part in gathered for item in part)
    assert [g[0] for g in got] == list(range(total))
    # single-process reference of the same signals
    O = orc
    f = O.MpFFT(n, p)
    for sig, hr, hi in got:
        xr, xi = O.mp_pair(n, p)
        O.fill_uniform(xr, xi, 1000 + sig)
        yr, yi = O.mp_pair(n, p)
        f(xr, xi, yr, yi)
        assert yr.hex() == hr and yi.hex() == hi
