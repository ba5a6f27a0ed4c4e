"""One process per GPU: the host-side pieces of running the box-image path on several
GPUs of one node.

The path shards without a data-path collective: independent jobs (served streams,
batched instances, or one whole job per rank) are divided among the ranks, and only the
timing and the totals cross ranks.  `torch.distributed` carries those (NCCL on GPUs,
gloo on CPU); every rank takes the same collective steps in the same order.
"""
from __future__ import annotations


def shard(items, world: int, rank: int) -> list:
    """The items rank `rank` of `world` owns: every world-th item starting at rank, so the
    mix of job kinds and sizes along a stream is spread evenly."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    return list(items)[rank::world]


def _reduce(dist, value: float, op, device) -> float:
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(dist, value: float, device="cpu") -> float:
    """The largest value over all ranks (the slowest rank's time); `value` when dist is None."""
    return value if dist is None else _reduce(dist, value, dist.ReduceOp.MAX, device)


def sum_over_ranks(dist, value: float, device="cpu") -> float:
    """The sum over all ranks (units processed by the whole job); `value` when dist is None."""
    return value if dist is None else _reduce(dist, value, dist.ReduceOp.SUM, device)


def throughput(dist, units: float, seconds: float, device="cpu") -> tuple[float, float, float]:
    """Whole-job throughput: all ranks' units over the slowest rank's time.
    Returns (units per second, total units, slowest seconds)."""
    total = sum_over_ranks(dist, units, device)
    slowest = max_over_ranks(dist, seconds, device)
    return total / slowest, total, slowest
