"""Multi-process plumbing for running the operators on several GPUs of one node.

The hot path shards with no exchange: lines along the solved axis are
independent and so are fields, so each rank (one process per GPU, launched by
torchrun) works on its own fields.  Ranks meet only to agree on timings:
a device time is reported as the maximum over ranks, and throughput as the
points of all ranks divided by that time (weak scaling).
"""
from __future__ import annotations

import datetime
import os

import torch


def world() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 120.0):
    """Joins the process group when there is more than one rank; returns
    torch.distributed, or None for a single process."""
    _, size, _ = world()
    if size <= 1:
        return None
    import torch.distributed as dist

    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def max_over_ranks(value: float, dist, device: str | torch.device = "cpu") -> float:
    """The largest value over all ranks (every rank gets it)."""
    if dist is None:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def partition_fields(costs, world_size: int) -> list[list[int]]:
    """Assigns fields to ranks by LPT bin packing (largest first, each to the
    least-loaded rank): the field-level data parallelism of a batch of uneven
    fields.  costs[i] is field i's work (points x the scheme's relative cost);
    returns, per rank, the field indices it runs (each rank then builds its own
    batch of them -- no data moves between ranks)."""
    import heapq

    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world_size)]
    parts: list[list[int]] = [[] for _ in range(world_size)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    for p in parts:
        p.sort()
    return parts


def weak_scaling_rate(points_per_rank: float, world_size: int, max_seconds: float) -> float:
    """Whole-job throughput (points per second) when every rank processed
    points_per_rank points and the slowest took max_seconds."""
    return points_per_rank * world_size / max_seconds
