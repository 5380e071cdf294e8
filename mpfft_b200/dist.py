"""Multi-GPU plumbing: the transform shards by signal, so ranks share no data.

Every rank transforms its own signals; the only collective is the reduction
of a timing scalar (max over ranks) and, for a caller that wants one global
batch split across ranks, the contiguous shard each rank owns.  One process
per GPU, torch.distributed for the plumbing (nccl on GPUs, gloo in tests).
"""
from __future__ import annotations


def shard_range(total: int, rank: int, world: int) -> tuple[int, int]:
    """[start, stop) of the signals rank `rank` owns out of `total`
    (contiguous, sizes differ by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of {world}")
    base, extra = divmod(total, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def rank_seed(seed: int, rank: int) -> int:
    """Seed of rank `rank`'s synthetic inputs (distinct signals per rank)."""
    return seed + rank


def max_over_ranks(value: float, device=None) -> float:
    """Largest `value` over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
