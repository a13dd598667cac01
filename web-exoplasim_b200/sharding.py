"""Multi-GPU sharding of independent planets: one process per GPU.

Planets never interact, so a batch of P planets splits into contiguous,
disjoint per-rank slices with no collective on the data path; the only
communication is one reduction of the ranks' device times (max over ranks)
and, optionally, a gather of per-rank results at the end.
"""
from __future__ import annotations


def shard(total: int, rank: int, world: int) -> range:
    """Indices of the planets rank `rank` of `world` steps: contiguous
    slices whose sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(total, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over all ranks of the default process group
    (the job's time is its slowest rank's); the value itself without one."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return value
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return value
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
