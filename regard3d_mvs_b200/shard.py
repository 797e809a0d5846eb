"""Pairs and depth maps across GPUs: one process per GPU.

Pairs are independent, so a job's pairs are split across ranks by longest
processing time first on their estimated aggregated cells (each pair goes to
the rank with the least work so far); every rank matches its share with one
batch call on its own GPU. Only the finished maps are exchanged
(``gather=True``: an all-gather of host arrays over the process group, gloo
or NCCL), so every rank ends with all results in the input order.

The depth stage after the combination shards by view
(``depth_stage_sharded``): refinement is per view; the consistency check of
a view needs its neighbours' prepared maps, so the refined maps are
exchanged once before the checks.
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


def _copy_map(m: dict) -> dict:
    return {k: (v.copy() if hasattr(v, "copy") and not isinstance(v, (list, dict)) else v) for k, v in m.items()}


def depth_stage_sharded(matcher: Matcher, maps: Sequence[dict], images: Sequence[dict],
                        partners: Sequence[Sequence[int]], rank: int, world: int, refine_options=None,
                        consistency_options=None, group=None):
    """The depth stage after the combination across ranks. Views are split by
    pixel count (largest first onto the least-loaded rank); each rank refines
    its share against the views' refinement images (`images[i]`: {camera,
    data}, held by every rank), the refined maps are all-gathered (a check
    needs its neighbours), every rank prepares all maps (cheap and
    deterministic), checks its share against the prepared maps, and the
    results are all-gathered. `maps` are depth-map dicts
    (regard3d_mvs_b200.depth_maps); `partners[i]` refine and check view i.
    Returns (all filtered maps in input order, refinement statistics summed
    over the views, consistency statistics summed over the views), equal to
    refine_depth_map per view followed by filter_depth_maps in one process."""
    from .depth_maps import normalise

    n = len(maps)
    share = shard_pairs([int(m["depth"].size) for m in maps], world)[rank]
    work = [normalise(_copy_map(m)) for m in maps]
    refine_stats = {"input": 0, "refined": 0, "kept": 0, "unconfirmed": 0}
    refined = {}
    for i in share:
        st = matcher.refine_depth_map(work[i], images[i], [images[j] for j in partners[i]], refine_options)
        refine_stats = {k: refine_stats[k] + st[k] for k in refine_stats}
        refined[i] = (work[i]["depth"], work[i]["confidence"])
    # Two collective calls, the same on every rank: the refined maps, then the results.
    exchange = _all_gather if world > 1 else (lambda obj, grp: [obj])
    refine_total = dict.fromkeys(refine_stats, 0)
    for part in exchange((refined, refine_stats), group):
        for i, (d, c) in part[0].items():
            work[i]["depth"], work[i]["confidence"] = d, c
        refine_total = {k: refine_total[k] + part[1][k] for k in refine_total}
    prepared = []
    cons_stats: dict = {}
    for i in range(n):
        p = _copy_map(work[i])
        st = matcher.prepare_depth_map(p, consistency_options)
        if i in share:
            cons_stats = {k: cons_stats.get(k, 0) + v for k, v in st.items()}
        prepared.append(p)
    done = {}
    for i in share:
        out = _copy_map(prepared[i])
        st = matcher.check_consistency(out, [prepared[j] for j in partners[i]], consistency_options)
        cons_stats = {k: cons_stats.get(k, 0) + v for k, v in st.items()}
        done[i] = (out["depth"], out["support"], out["confidence"])
    result = [None] * n
    totals: dict = {}
    for part in exchange((done, cons_stats), group):
        for i, (d, s, c) in part[0].items():
            result[i] = dict(work[i], depth=d, support=s, confidence=c)
        totals = {k: totals.get(k, 0) + v for k, v in part[1].items()}
    return result, refine_total, totals


def _all_gather(obj, group):
    import torch.distributed as dist

    parts: list = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, obj, group=group)
    return parts
