"""Host-side plumbing for running the solver on several GPUs of one node.

The hot path has no exchange step: right-hand sides (point / noise sources,
shifts of different rational functions) and whole lattices are independent
units, so N GPUs run N independent replicas of the gauge field and split the
units between them.  Nothing crosses NVLink during a solve; torch.distributed
is used only for the start barrier and for the max-over-ranks timing.
"""
from __future__ import annotations

from typing import List, Sequence


def shard_units(costs: Sequence[float], world: int, rank: int) -> List[int]:
    """Indices of the units rank `rank` solves.

    Longest-processing-time-first greedy assignment on the given costs (e.g.
    volume x expected iterations), ties broken by index, so every rank computes
    the same partition without communicating."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    owner = [0] * len(costs)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += float(costs[i])
    return [i for i in range(len(costs)) if owner[i] == rank]


def rank_seed(base: int, rank: int) -> int:
    """Seed of the synthetic source a replica solves (distinct per rank)."""
    return (int(base) + 7919 * int(rank)) & 0xFFFFFFFFFFFFFFFF


def max_over_ranks(value: float) -> float:
    """Maximum of a per-rank time over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
