"""Sharding a sweep of independent instances over ranks (one process per GPU).

Instances are independent, so a sweep partitions with no data-path
collective: each rank builds a gpe_batch of its own instances.  The
assignment is greedy by estimated cost (N log N points per iteration of the
instance's grid, largest first, to the least-loaded rank) and depends only on
the instance list, so every rank computes the same partition without
communication.  The only exchange is the final gather of per-instance
results, done by the caller (torch.distributed all_gather_object).
"""
from __future__ import annotations

import math


def instance_cost(shape) -> float:
    """Relative cost of one iteration: points * log2(points)."""
    n = 1
    for d in shape:
        n *= int(d)
    return n * math.log2(max(n, 2))


def partition(shapes, world: int):
    """Rank of each instance: greedy longest-processing-time assignment."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(shapes)), key=lambda i: (-instance_cost(shapes[i]), i))
    load = [0.0] * world
    owner = [0] * len(shapes)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += instance_cost(shapes[i])
    return owner


def my_instances(shapes, rank: int, world: int):
    """Indices of the instances rank owns, in instance order."""
    own = partition(shapes, world)
    return [i for i, r in enumerate(own) if r == rank]
