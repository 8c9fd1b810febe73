"""Scene-parallel placement over ranks (one process per GPU).

Scenes are independent, so several GPUs share a set of scenes without any
data-path collective: each rank takes a subset, steps it in its own Batch,
and only metrics cross ranks.  The placement is deterministic (the same on
every rank, no communication needed): longest-processing-time-first by
particle count, ties broken by scene index.
"""
from __future__ import annotations

from typing import List, Sequence


def partition(weights: Sequence[float], world_size: int) -> List[List[int]]:
    """Assign item indices to `world_size` ranks, balancing the summed weight."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(weights)), key=lambda i: (-float(weights[i]), i))
    loads = [0.0] * world_size
    parts: List[List[int]] = [[] for _ in range(world_size)]
    for i in order:
        r = min(range(world_size), key=lambda k: (loads[k], k))
        parts[r].append(i)
        loads[r] += float(weights[i])
    for p in parts:
        p.sort()
    return parts


def scenes_for_rank(scenes, rank: int, world_size: int):
    """The scenes rank `rank` owns (each scene weighted by its particle count)."""
    parts = partition([max(1, s.n) for s in scenes], world_size)
    return [scenes[i] for i in parts[rank]]


def reduce_step_metrics(local_particle_steps: float, local_seconds: float, all_reduce_sum, all_reduce_max):
    """Whole-job particle-steps/s: total work over the slowest rank's time."""
    total = all_reduce_sum(float(local_particle_steps))
    t = all_reduce_max(float(local_seconds))
    return total / t if t > 0 else 0.0, total, t
