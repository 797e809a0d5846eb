"""Pairs across GPUs: one process per GPU, no collective on the data path.

Pairs are independent, so a job's pairs are split across ranks by longest
processing time first on their estimated aggregated cells (each pair goes to
the rank with the least work so far); every rank matches its share with one
batch call on its own GPU. Only the finished maps are exchanged
(``gather=True``: an all-gather of host arrays over the process group, gloo
or NCCL), so every rank ends with all results in the input order.
"""

from __future__ import annotations

import heapq
from typing import Sequence

from .stereo import Matcher


def estimated_cells(pair: dict) -> int:
    """W * H * D of the full label range at level 0 (aligned to 16), the
    work measure of the reference's benchmark; hierarchical pairs aggregate
    less, but in proportion."""
    h, w = pair["left"].shape
    nd = (int(pair["num_disparities"]) + 15) // 16 * 16
    return w * h * nd


def shard_pairs(costs: Sequence[int], world: int) -> list[list[int]]:
    """Indices of the pairs per rank: largest first onto the least-loaded
    rank (ties to the lower rank); each rank's list in ascending order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0, r) for r in range(world)]
    shares: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(s) for s in shares]


def match_sharded(matcher: Matcher, pairs: Sequence[dict], rank: int, world: int, group=None,
                  gather: bool = True):
    """Matches this rank's share of `pairs` (dicts as for
    Matcher.match_stereo_batch). Returns {index: DisparityMap} for the own
    share, or with gather=True the list of all maps in input order."""
    share = shard_pairs([estimated_cells(p) for p in pairs], world)[rank]
    own = matcher.match_stereo_batch([pairs[i] for i in share]) if share else []
    mine = dict(zip(share, own))
    if not gather or world == 1:
        return mine if not gather else [mine[i] for i in range(len(pairs))]
    import torch.distributed as dist

    parts: list = [None] * world
    dist.all_gather_object(parts, mine, group=group)
    merged = {}
    for p in parts:
        merged.update(p)
    return [merged[i] for i in range(len(pairs))]
