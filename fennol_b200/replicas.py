"""Multi-GPU plumbing: one process per GPU, each evaluating its own systems.

The energy/force path has no data exchange between systems, so N GPUs run N
independent replicas (or disjoint shards of a request stream) and the only
collectives are the timing reduction and barriers: the job time is the
largest time over ranks, and the job throughput is the units all ranks
processed divided by that time.
"""

from __future__ import annotations

from typing import List, Sequence, TypeVar

import torch
import torch.distributed as dist

T = TypeVar("T")


def max_over_ranks(value: float, device=None) -> float:
    """The largest ``value`` over all ranks (the value itself without a
    process group).  ``device``: where the reduction tensor lives (a CUDA
    device for NCCL, CPU for gloo)."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_throughput(units_this_rank: float, seconds_this_rank: float, device=None) -> float:
    """Units processed by all ranks divided by the slowest rank's time."""
    units = sum_over_ranks(units_this_rank, device)
    seconds = max_over_ranks(seconds_this_rank, device)
    return units / seconds if seconds > 0 else float("inf")


def shard(items: Sequence[T], rank: int, world: int) -> List[T]:
    """Round-robin share of ``items`` for ``rank`` (every item on exactly one rank)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    return [it for k, it in enumerate(items) if k % world == rank]
