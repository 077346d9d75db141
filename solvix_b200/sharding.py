"""Instance sharding for the batched and served forms on several GPUs.

The models of a batch are independent, so N GPUs split them with no
collective on the data path: every rank computes the same greedy
longest-processing-time assignment from the models' estimated work and
solves its own share.  The estimate is DOF x sqrt(DOF), the Jacobi-PCG
cost growth of these plate and beam models (iterations grow roughly with the
square root of the condition number, which scales with the mesh size).
"""
from __future__ import annotations

import heapq

import numpy as np


def estimated_work(n_dof) -> np.ndarray:
    n = np.asarray(n_dof, dtype=np.float64)
    return n * np.sqrt(n)


def shard_instances(n_dof, world: int):
    """List of `world` index lists; deterministic, disjoint and complete."""
    work = estimated_work(n_dof)
    order = sorted(range(len(work)), key=lambda k: (-work[k], k))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    shards = [[] for _ in range(world)]
    for k in order:
        load, r = heapq.heappop(heap)
        shards[r].append(k)
        heapq.heappush(heap, (load + float(work[k]), r))
    return [sorted(s) for s in shards]


def solve_sharded(items, solve_fn, rank: int, world: int, n_dof=None):
    """Solve ``items`` split over ``world`` ranks and return every result, in
    item order, on every rank.

    Each rank calls ``solve_fn`` on its own shard only (no data crosses
    ranks before that); the per-item results are then exchanged once with
    ``all_gather_object`` over the default process group.  ``n_dof`` gives
    the per-item sizes used for the split (default: ``item.n_dof``).
    """
    sizes = [it.n_dof for it in items] if n_dof is None else list(n_dof)
    mine = shard_instances(sizes, world)[rank]
    local = solve_fn([items[k] for k in mine])
    if world == 1:
        return list(local)
    import torch.distributed as dist
    gathered = [None] * world
    dist.all_gather_object(gathered, (mine, list(local)))
    out = [None] * len(items)
    for idx, res in gathered:
        for k, r in zip(idx, res):
            out[k] = r
    return out
