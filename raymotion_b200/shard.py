"""Splitting a batch of images across ranks (one process per GPU).

The images of a batch are independent - different scenes, views, sizes and
sample counts - so a batch on N GPUs is split by image with no data-path
collective: each rank renders a disjoint subset through its own
``rmcuda_render_batch``, and the ranks meet only to reduce timings and counts
(the slowest rank's time, the sum of path samples).  The reference has no
multi-GPU path (one synchronous Metal command queue, src/engine/metal.mm:365-367).

``partition`` balances the subsets by an estimated cost per image (longest
processing time first: the most expensive image goes to the least loaded
rank), so that the slowest rank - which sets the whole job's time - carries
about 1/N of the work.
"""
from __future__ import annotations

import math


def image_cost(width: int, height: int, spp: int, depth: int, n_tris: int, **_) -> float:
    """Estimated work of one image: path samples x path length bound x BVH depth
    (log2 of the triangle count).  Only the ratios between images matter."""
    return float(width) * float(height) * float(spp) * float(max(depth, 1)) * math.log2(2.0 + float(n_tris))


def partition(costs: list[float], n_ranks: int) -> list[list[int]]:
    """Disjoint index lists, one per rank, covering every item exactly once.

    Greedy longest-processing-time assignment: items in decreasing cost (ties by
    index) each go to the rank with the smallest total so far (ties by rank), so
    the result depends only on the costs.  Each list is returned in increasing
    index order."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be at least 1")
    loads = [0.0] * n_ranks
    parts: list[list[int]] = [[] for _ in range(n_ranks)]
    for i in sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k)):
        r = min(range(n_ranks), key=lambda q: (loads[q], q))
        parts[r].append(i)
        loads[r] += float(costs[i])
    return [sorted(p) for p in parts]


def rank_items(specs: list[dict], rank: int, world: int) -> list[int]:
    """The indices of ``specs`` (dicts with width, height, spp, depth, n_tris)
    that ``rank`` of ``world`` renders."""
    return partition([image_cost(**s) for s in specs], world)[rank]
