"""Multi-GPU plumbing: one process per GPU, independent design instances.

The reference is single-GPU, one protein per run (src/main.cu); its generation
loop has no exchange step, so the engine scales by running independent
instances per rank (weak scaling) with no collective on the data path.  Only
the timing uses a collective: the slowest rank's time (MAX all-reduce).
"""
from __future__ import annotations


def replica_seed(base: int, rank: int) -> int:
    """Seed of rank `rank`'s replica (distinct, reproducible streams)."""
    return (base + 0x9E3779B97F4A7C15 * (rank + 1)) & 0xFFFFFFFFFFFFFFFF


def shard_jobs(costs, world: int):
    """Assign jobs (by estimated cost, e.g. HBM bytes or stem-scan cells) to ranks:
    longest job first onto the least-loaded rank, ties to the lower rank.
    Every rank computes the same assignment."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0] * world
    shards = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        shards[r].append(i)
        load[r] += costs[i]
    return [sorted(s) for s in shards]


def max_over_ranks(seconds: float, device=None) -> float:
    """Slowest rank's time (all ranks call this in the same order)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(seconds)
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_results(local: dict) -> dict:
    """Every rank's {job index: result} merged (all ranks call this in the same order;
    a job index appears on exactly one rank)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return dict(local)
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, local)
    merged = {}
    for part in parts:
        for k, v in part.items():
            if k in merged:
                raise ValueError(f"job {k} reported by two ranks")
            merged[k] = v
    return merged


def whole_job_rate(units_per_rank: float, world: int, max_seconds: float) -> float:
    """Aggregate throughput: units processed by all ranks / slowest rank's time."""
    return units_per_rank * world / max_seconds
