"""Pairs across ranks (regard3d_mvs_b200/shard.py): the longest-processing-time
split, and two gloo ranks on the CPU, each matching its share on the SIMT
emulator, whose gathered maps equal the pairs matched in one process."""

from __future__ import annotations

import datetime
import multiprocessing as mp
import os
import socket

import numpy as np

from conftest import SIMT_LIB
from images import Texture, render_pair, same_disparities
from regard3d_mvs_b200.shard import estimated_cells, shard_pairs
from regard3d_mvs_b200.types import StereoOptions


def test_shard_pairs_balances_and_covers():
    costs = [90, 10, 40, 40, 30, 70, 5, 5]
    for world in (1, 2, 3, 5, 9):
        shares = shard_pairs(costs, world)
        assert len(shares) == world
        assert sorted(i for s in shares for i in s) == list(range(len(costs)))
        loads = [sum(costs[i] for i in s) for s in shares]
        if world <= len(costs):
            # LPT bound: the largest load exceeds the ideal by at most the largest job.
            assert max(loads) <= sum(costs) / world + max(costs)
    assert shard_pairs(costs, 2) == shard_pairs(costs, 2)  # deterministic
    assert shard_pairs([], 3) == [[], [], []]


def _pairs():
    tex = Texture(51)
    out = []
    for i, (w, h, nd, lv) in enumerate(((28, 16, 16, 0), (24, 18, 16, 1), (20, 14, 16, 0), (32, 16, 32, 0))):
        left, right, _ = render_pair(tex, w, h, lambda x, y, i=i: 2.0 + 0.1 * x + i)
        out.append(dict(left=left, right=right, disparity_min=0, num_disparities=nd,
                        options=StereoOptions(levels=lv, tile_size=32)))
    return out


def _rank(rank, world, port, pairs, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        from regard3d_mvs_b200 import Matcher
        from regard3d_mvs_b200.shard import match_sharded

        m = Matcher(SIMT_LIB, host_is_device=True)
        res = match_sharded(m, pairs, rank, world)
        q.put((rank, [(r.disparity, r.confidence, r.cells, r.levels) for r in res]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_their_shares(simt_matcher):
    pairs = _pairs()
    assert len({tuple(s) for s in shard_pairs([estimated_cells(p) for p in pairs], 2)}) == 2
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, pairs, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=600) for _ in procs)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    ref = simt_matcher.match_stereo_batch(pairs)
    for r in (0, 1):
        for (d, c, cells, levels), m in zip(got[r], ref):
            assert same_disparities(d, m.disparity) and np.array_equal(c, m.confidence)
            assert (cells, levels) == (m.cells, m.levels)


def _rank_failing(rank, world, port, pairs, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    if rank == 1:
        os._exit(3)  # leaves between steps, before the exchange
    try:
        from regard3d_mvs_b200 import Matcher
        from regard3d_mvs_b200.shard import match_sharded

        m = Matcher(SIMT_LIB, host_is_device=True)
        match_sharded(m, pairs, rank, world)
        q.put((rank, "finished"))
    except Exception as e:  # noqa: BLE001 - the failure is the expected outcome
        q.put((rank, f"error: {type(e).__name__}"))


def test_lost_rank_ends_the_exchange_with_an_error(simt_matcher):
    """A rank that exits makes the other rank's gather fail (connection
    closed or process-group timeout) instead of waiting for ever."""
    pairs = _pairs()[:2]
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_failing, args=(r, 2, port, pairs, q)) for r in range(2)]
    for p in procs:
        p.start()
    rank, outcome = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
    assert rank == 0 and outcome.startswith("error")
    assert procs[1].exitcode == 3


# ------------------------------------------------------------------ depth stage
def _depth_inputs():
    """Four small views with sparse depths (a few hundred refinement warps)."""
    from regard3d_mvs_b200.multi_view import depth_stage_scene

    scene = depth_stage_scene(4, 40, 30, partners=2)
    rng = np.random.default_rng(5)
    maps, images = [], []
    for i, v in enumerate(scene["views"]):
        keep = np.zeros(v["depth"].shape, bool)
        for _ in range(8):
            y, x = rng.integers(4, 26), rng.integers(4, 36)
            keep[y - 1:y + 2, x - 1:x + 2] = True
        keep[10:20, 10:30] = True  # a block the consistency check sees in the neighbours
        maps.append({"camera": v["camera"], "depth": np.where(keep, v["depth"], 0).astype(np.float32),
                     "confidence": np.zeros(v["depth"].shape, np.float32),
                     "pair_mask": np.ones(v["depth"].shape, np.uint16), "color": v["color"], "view": i,
                     "partners": scene["partners"][i]})
        images.append({"camera": v["camera"], "data": None, "gray": v["gray"]})
    return maps, images, scene["partners"]


def _depth_rank(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=300))
    try:
        from regard3d_mvs_b200 import Matcher
        from regard3d_mvs_b200.depth_maps import RefinementOptions
        from regard3d_mvs_b200.shard import depth_stage_sharded

        m = Matcher(SIMT_LIB, host_is_device=True)
        maps, images, partners = _depth_inputs()
        for im in images:
            im["data"] = m.make_refinement_image(im.pop("gray"))
        res, rst, cst = depth_stage_sharded(m, maps, images, partners, rank, world,
                                            RefinementOptions(radius=2, step=2))
        q.put((rank, [(r["depth"], r["support"]) for r in res], rst, cst))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_run_the_depth_stage(simt_matcher):
    """Refinement of each rank's views, exchange, consistency of each rank's
    views: the same maps and statistics as one process refining every view
    and filtering all maps."""
    from regard3d_mvs_b200.depth_maps import ConsistencyOptions, RefinementOptions

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_depth_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in procs:
        rank, res, rst, cst = q.get(timeout=600)
        got[rank] = (res, rst, cst)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    maps, images, partners = _depth_inputs()
    for im in images:
        im["data"] = simt_matcher.make_refinement_image(im.pop("gray"))
    rst = {"input": 0, "refined": 0, "kept": 0, "unconfirmed": 0}
    for i, mp_ in enumerate(maps):
        st = simt_matcher.refine_depth_map(mp_, images[i], [images[j] for j in partners[i]],
                                           RefinementOptions(radius=2, step=2))
        rst = {k: rst[k] + st[k] for k in rst}
    cst = simt_matcher.filter_depth_maps(maps, partners, ConsistencyOptions())
    assert rst["refined"] > 0 and cst["output"] > 0
    for rank in (0, 1):
        res, r_rst, r_cst = got[rank]
        assert r_rst == rst and r_cst == cst
        for (d, sup), ref in zip(res, maps):
            assert np.array_equal(d, ref["depth"]) and np.array_equal(sup, ref["support"])
