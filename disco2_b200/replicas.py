"""Multi-GPU layout: independent disks per rank, no data-path collective.

The single-disk step does not shard (an MPI-style radial split is outside the
path), so N GPUs run N replicas, and a batched sweep of many disks is split
across ranks by disk.  The only collectives are a barrier and the max-over-ranks
of the measured time.
"""
from __future__ import annotations


def partition(cells: list[int], world: int) -> list[list[int]]:
    """Split disks (given by cell count) over `world` ranks, balancing cells:
    largest disk first onto the least-loaded rank (ties -> lowest rank).
    Deterministic, so every rank computes the same assignment."""
    order = sorted(range(len(cells)), key=lambda k: (-cells[k], k))
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda i: (load[i], i))
        parts[r].append(k)
        load[r] += cells[k]
    return [sorted(p) for p in parts]


def max_over_ranks(x: float, device=None) -> float:
    """Maximum of a per-rank float over the default process group (identity
    without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
