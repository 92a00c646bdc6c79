"""Replica sharding of the coarse pass across GPUs, one process per GPU.

The coarse pass shards by particle with no exchange: every particle's
diff2[o][t] block depends only on its own image, the shared (read-only,
replicated) projector and the shared orientation and translation sets, and
its minimum is local.  So ranks split the particles, score them independently
and only the bookkeeping crosses ranks: the total number of evaluations and
the slowest rank's device time.  No collective sits on the data path.

Works with any torch.distributed backend (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations


def particle_range(P_total: int, rank: int, world: int) -> tuple[int, int]:
    """(first, count) of the contiguous particle block of `rank`: the first
    P_total % world ranks take one extra particle."""
    if world <= 0 or not 0 <= rank < world or P_total < 0:
        raise ValueError("bad shard request")
    base, extra = divmod(P_total, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def _reduce(value: float, op: str, dist=None, device=None) -> float:
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def slowest(ms: float, dist=None, device=None) -> float:
    """Device time of the slowest rank (every rank calls it)."""
    return _reduce(ms, "max", dist, device)


def total(units: float, dist=None, device=None) -> float:
    """Units processed by all ranks together (every rank calls it)."""
    return _reduce(units, "sum", dist, device)


def job_rate(units_this_rank: float, ms_this_rank: float, dist=None, device=None) -> float:
    """Whole-job throughput: all ranks' units over the slowest rank's time."""
    u = total(units_this_rank, dist, device)
    t = slowest(ms_this_rank, dist, device)
    return u / (t / 1e3) if t > 0 else 0.0
