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
