"""Replica layout over GPUs.

The Brownian-dynamics step of one system has no data-parallel split in the
reference (one patch per system, no halo exchange on this path), so N GPUs run
N independent replicas, one process per GPU: rank r simulates its own
system, seeded ``base_seed + r``, with no collective on the data path. The
only cross-rank traffic is the timing reduction: a job's throughput counts
every rank's particle-steps over the slowest rank's device time.
"""
from __future__ import annotations

import os


def rank_env() -> tuple:
    """(world_size, rank, local_rank) from the torch.distributed launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def replica_seed(base_seed: int, rank: int) -> int:
    """Seed of rank `rank`'s replica: independent systems and noise streams."""
    return int(base_seed) + int(rank)


def max_over_ranks(value: float, device=None) -> float:
    """Largest `value` over all ranks (the identity outside a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank: int, steps: int, max_ms: float, world: int) -> float:
    """Whole-job units per second: all ranks' work over the slowest rank's time."""
    return world * units_per_rank * steps / (max_ms / 1e3)
