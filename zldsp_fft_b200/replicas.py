"""Replica execution across GPUs: one process per GPU, no data-path collective.

Every transform of a batch is independent, so a multi-GPU job is N replicas:
each rank transforms its own batch (or its shard of a shared batch) on its own
GPU. The only communication is host-side bookkeeping: a barrier around the
timed region and the maximum of the ranks' elapsed times, so the whole-job
throughput is (bytes of all ranks) / (slowest rank's time). The process group
may be NCCL (GPUs) or gloo (CPU, tests).
"""
from __future__ import annotations


def shard(n_items: int, rank: int, world: int) -> range:
    """Contiguous share of items [0, n_items) for `rank`: sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The maximum of `value` over all ranks of the default process group
    (the value itself when there is none)."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_gbs(bytes_per_rank: float, world: int, elapsed_s_max: float) -> float:
    """Whole-job GB/s of `world` replicas that each moved `bytes_per_rank`."""
    if elapsed_s_max <= 0:
        raise ValueError("elapsed time must be positive")
    return bytes_per_rank * world / elapsed_s_max / 1e9
