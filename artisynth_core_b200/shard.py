"""Multi-GPU form of the batched and served paths: independent models are
dealt to ranks (one process per GPU), with no collective on the data path.

* :func:`lpt_partition` -- longest-processing-time bin packing of models by
  their work (elements), deterministic, so every rank computes the same
  assignment without communication;
* :func:`gather_to_root` -- host-side gather of per-rank result objects
  (torch.distributed ``all_gather_object``; works over NCCL and gloo);
* :func:`max_over_ranks` -- the timing rule of multi-GPU measurements: the
  slowest rank's time.

A BackwardEuler step of one model is a coupled solve and is never split
across GPUs; only whole models move.
"""
from __future__ import annotations

import heapq


def lpt_partition(weights, n_ranks: int):
    """Deal items to ranks, heaviest first, each to the least-loaded rank
    (ties: lowest rank, then lowest index).  Returns one ascending index list
    per rank."""
    if n_ranks <= 0:
        raise ValueError("n_ranks must be positive")
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    heap = [(0.0, r) for r in range(n_ranks)]
    heapq.heapify(heap)
    out = [[] for _ in range(n_ranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(weights[i]), r))
    return [sorted(s) for s in out]


def gather_to_root(dist, obj, root: int = 0):
    """Every rank's `obj` in rank order on `root` (None elsewhere); without a
    process group, [obj]."""
    if dist is None:
        return [obj]
    objs = [None] * dist.get_world_size()
    dist.all_gather_object(objs, obj)
    return objs if dist.get_rank() == root else None


def max_over_ranks(dist, value: float) -> float:
    """The largest `value` over ranks (the multi-GPU timing rule)."""
    if dist is None:
        return value
    vals = [None] * dist.get_world_size()
    dist.all_gather_object(vals, float(value))
    return max(vals)
