"""Multi-GPU execution: independent shots on independent GPUs.

Shots never exchange data, so N GPUs run N replicas (one process per GPU,
torch.distributed for the plumbing only).  A batch of shots is split across
ranks by cost (cell-updates = padded cells x steps) with a deterministic
longest-processing-time greedy assignment, so every rank computes the same
partition without communicating.  The only collectives are the timing
barrier and the max-over-ranks of the measured time.
"""
from __future__ import annotations

from typing import Sequence


def shot_cost(cfg) -> int:
    nx, ny, nz = cfg.padded
    return int(nx) * int(ny) * int(nz) * int(cfg.nt)


def shard(costs: Sequence[int], world: int) -> list[list[int]]:
    """Partition shot indices over `world` ranks, balancing total cost."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += costs[i]
    for p in parts:
        p.sort()
    return parts


def my_shots(costs: Sequence[int], rank: int, world: int) -> list[int]:
    return shard(costs, world)[rank]


def max_over_ranks(value: float) -> float:
    """Max of a host float over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
