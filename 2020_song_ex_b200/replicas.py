"""Replicas across GPUs (one process per GPU): the search does not shard.

Queries are independent and every graph of the reference's workloads fits
one B200, so N GPUs run N replicas: every rank holds the same base and
graph, searches its own queries, and only the timing is reduced (the
maximum over ranks).  No collective touches the data path.
"""
from __future__ import annotations

import os


def env():
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def query_seed(base_seed: int, rank: int):
    """Rank 0 keeps the workload's own queries; rank r > 0 draws its own from
    the same mixture with a separate generator."""
    return None if rank == 0 else base_seed + 7919 * rank


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank scalar (a duration) over all ranks; the value
    itself when not distributed."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_qps(world_size: int, per_rank_queries: int, steps: int, max_seconds: float) -> float:
    """Whole-job throughput: every rank's queries over the slowest rank's time."""
    return world_size * per_rank_queries * steps / max_seconds
