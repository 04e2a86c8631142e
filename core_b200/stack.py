"""Stacks of interferograms across GPUs and within one GPU.

A stack shards by grid: every interferogram is an independent solve (the DCT
couples the pixels of one grid, nothing couples two grids), so the ranks of a
multi-GPU job take disjoint subsets of the stack and exchange nothing on the
data path.  The reference distributes the same independent per-pair solves as
dask tasks (insardev/insardev/Stack_unwrap2d.py:873-945), serialised on one GPU
by a process lock (:20, :63).

`shard_stack` balances the subsets by estimated work (pixels times expected
iterations), greedily assigning the largest remaining grid to the least
loaded rank; every rank computes the same assignment from the same sizes, so
no communication is needed to agree on it.
"""
from __future__ import annotations

import heapq


def shard_stack(shapes, world_size, work=None):
    """Assign grids to ranks.

    shapes      list of (H, W) per grid
    world_size  number of ranks
    work        optional per-grid weights (default H*W)
    Returns a list of `world_size` lists of grid indices (each sorted).
    """
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    n = len(shapes)
    w = [float(h) * float(x) for h, x in shapes] if work is None else [float(v) for v in work]
    if len(w) != n:
        raise ValueError("work must have one entry per grid")
    order = sorted(range(n), key=lambda i: (-w[i], i))
    heap = [(0.0, r) for r in range(world_size)]
    heapq.heapify(heap)
    out = [[] for _ in range(world_size)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + w[i], r))
    return [sorted(s) for s in out]


def unwrap_stack(phases, weights=None, rank=0, world_size=1, device='auto', **kw):
    """Unwrap this rank's share of a stack with one batched solve.

    Returns {grid index: (unwrapped, conncomp)} for the grids of this rank.
    Keyword arguments are those of `irls_unwrap_2d_batch`.
    """
    from .irls import irls_unwrap_2d_batch
    shapes = [tuple(p.shape) for p in phases]
    mine = shard_stack(shapes, world_size)[rank]
    if not mine:
        return {}
    ws = None if weights is None else [weights[i] for i in mine]
    res = irls_unwrap_2d_batch([phases[i] for i in mine], ws, device=device, **kw)
    return dict(zip(mine, res))
