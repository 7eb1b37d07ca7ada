"""Independent replicas, one per GPU (the step does not shard across GPUs).

Each rank runs its own simulation (or its own share of a request stream) with
no data-path collective; the only cross-rank operations are the timing
reduction -- the slowest rank's device time defines the whole job's time --
and barriers around the timed region.  beamz's CUDA path is single-GPU
(beamz/simulation/kernels.py:1590-1602 rejects sharding for it); its JAX
path would shard z-slabs (beamz/simulation/sharding.py:115-202), which this
engine does not do.
"""

from __future__ import annotations

import os


def world() -> tuple[int, int, int]:
    """(rank, world_size, local_rank) from the launcher's environment."""
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def shard(items, rank: int, world_size: int) -> list:
    """Round-robin share of `items` for `rank` (every item on exactly one rank)."""
    return [x for i, x in enumerate(items) if i % world_size == rank]


def max_over_ranks(value: float, device=None) -> float:
    """The largest `value` over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank: float, max_seconds: float, world_size: int) -> float:
    """Whole-job throughput of `world_size` replicas that each processed
    `units_per_rank` units, timed by the slowest rank."""
    return units_per_rank * world_size / max_seconds
