"""Process-group helpers for runs with one process per GPU.

A single grid does not shard here (replicas only); parameter sweeps shard by
instance with no collective on the data path.  These helpers cover the host
side: the balanced instance partition and the max-over-ranks reduction used to
time multi-GPU runs.
"""
from __future__ import annotations

import math


def instance_cost(n: int) -> float:
    """Relative cost of one RK4 step of an n^3 instance: the FFT passes scale
    as n^3 log n, the multigrid work as n^3."""
    return float(n) ** 3 * (math.log2(n) + 8.0)


def partition(sizes, world_size: int):
    """Longest-processing-time assignment of instances (given by grid size) to
    ranks; returns one list of instance indices per rank.  Deterministic: ties
    broken by index, so every rank computes the same partition."""
    order = sorted(range(len(sizes)), key=lambda i: (-instance_cost(sizes[i]), i))
    load = [0.0] * world_size
    parts = [[] for _ in range(world_size)]
    for i in order:
        r = min(range(world_size), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += instance_cost(sizes[i])
    return [sorted(p) for p in parts]


def max_over_ranks(x: float, device=None) -> float:
    """Maximum of a float over the default process group (identity without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
