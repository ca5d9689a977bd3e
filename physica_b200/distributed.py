"""Multi-GPU placement for the PBF path.

One scene does not shard without a halo exchange (the reference has none), so N GPUs run N replicas
of a single-scene workload.  Independent scenes of a batch partition across ranks with no collective on
the data path: `partition_scenes` assigns whole scenes to ranks, balancing particle counts
(longest-processing-time greedy, deterministic), and `max_over_ranks` reduces the per-rank timings.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def partition_scenes(counts: list, world: int) -> list:
    """Scene indices per rank: every scene exactly once, particle totals balanced."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(counts)), key=lambda s: (-counts[s], s))
    loads = [0] * world
    parts = [[] for _ in range(world)]
    for s in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        parts[r].append(s)
        loads[r] += counts[s]
    return [sorted(p) for p in parts]


def max_over_ranks(value: float) -> float:
    """Maximum of a per-rank float over the process group (identity without one)."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return value
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
