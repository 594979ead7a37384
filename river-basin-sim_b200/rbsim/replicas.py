"""Multi-GPU as independent replicas: whole domains or requests per rank, no data-path collective.

The solver path does not shard a single domain (the reference has no domain
decomposition), so N GPUs run N independent units of work. What crosses ranks is
bookkeeping only: which rank owns which unit, and the job's time as the slowest
rank's time. Both run over any ``torch.distributed`` process group (NCCL on the
GPUs, gloo on the host).
"""

from __future__ import annotations

import heapq
import os
from collections.abc import Sequence

import torch
import torch.distributed as dist


def rank_world() -> tuple[int, int]:
    """(rank, world size) from the launcher's environment; (0, 1) when not launched."""
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))


def shard_units(costs: Sequence[float], world: int) -> list[list[int]]:
    """Assign units to ranks, longest first onto the least-loaded rank (LPT).

    Deterministic: every rank computes the same assignment from the same costs, so
    no rank has to tell another what it owns. Ties go to the lower rank; equal
    costs keep their input order.
    """
    if world < 1:
        raise ValueError(f"world size must be >= 1, got {world}")
    if any(not (c >= 0.0) for c in costs):
        raise ValueError("unit costs must be finite and non-negative")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    for units in out:
        units.sort()
    return out


def _device_of(group) -> torch.device:
    backend = dist.get_backend(group)
    if backend == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(value: float, group=None) -> float:
    """The largest ``value`` over the ranks (the job's time is its slowest rank's)."""
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device_of(group))
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def sum_over_ranks(value: float, group=None) -> float:
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device_of(group))
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t.item())


def whole_job_rate(units: float, seconds: float, group=None) -> tuple[float, float]:
    """(units all ranks processed / slowest rank's seconds, slowest rank's seconds)."""
    total = sum_over_ranks(units, group)
    slowest = max_over_ranks(seconds, group)
    if not slowest > 0.0:
        raise ValueError(f"non-positive job time {slowest}")
    return total / slowest, slowest
