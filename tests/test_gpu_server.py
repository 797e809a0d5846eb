"""The serving loop on the B200: requests of uneven size, label range and
hierarchy depth, submitted from several client threads and run in
continuous batches on two worker streams, give exactly the maps of the same
pairs matched alone; a tight device-memory budget serialises them without
changing any result."""

from __future__ import annotations

import threading

import numpy as np
import pytest

from images import mismatch_report, same_disparities
from regard3d_mvs_b200 import Server, StereoOptions
from test_gpu_parity import _synthetic_pair

pytestmark = pytest.mark.gpu

SPECS = ((640, 480, 128, 0), (768, 512, 256, 3), (400, 300, 96, -1), (1024, 700, 192, 2), (320, 240, 64, 0),
         (900, 600, 128, 1))


@pytest.fixture(scope="module")
def pairs():
    out = []
    for i, (w, h, nd, lv) in enumerate(SPECS):
        left, right = _synthetic_pair(w, h, nd, 30 + i)
        o = StereoOptions(levels=lv, range_radius=0, range_margin=8) if lv else StereoOptions(levels=lv)
        out.append(dict(left=left, right=right, disparity_min=0, num_disparities=nd, options=o))
    return out


@pytest.fixture(scope="module")
def alone(gpu_matcher, pairs):
    return [gpu_matcher.match_stereo(p["left"], p["right"], None, None, 0, p["num_disparities"], p["options"])
            for p in pairs]


def _same(a, b):
    assert same_disparities(a.disparity, b.disparity), mismatch_report(a.disparity, b.disparity)
    assert np.array_equal(a.confidence, b.confidence)
    assert (a.cells, a.levels, a.num_disparities) == (b.cells, b.levels, b.num_disparities)


def test_server_mix_equals_alone(pairs, alone, oracle):
    got, times = {}, {}
    lock = threading.Lock()
    with Server(workers=2, max_batch=3, hbm_budget=16 << 30, scratch_budget=8 << 30) as srv:
        def client(idxs):
            tickets = [(i, srv.submit(**pairs[i])) for i in idxs]
            for i, t in tickets:
                m, tm = srv.wait(t)
                with lock:
                    got[i], times[i] = m, tm

        threads = [threading.Thread(target=client, args=(list(range(k, len(pairs), 3)),)) for k in range(3)]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
    for i, a in enumerate(alone):
        _same(got[i], a)
    assert {t["worker"] for t in times.values()} <= {0, 1}
    # The served maps are the reference's maps too.
    oracle.set_threads(oracle.max_threads())
    for i, p in enumerate(pairs):
        _same(got[i], oracle.match_stereo(p["left"], p["right"], None, None, 0, p["num_disparities"], p["options"]))


def test_server_tight_budget(pairs, alone):
    # Every request is larger than the budget: each runs alone, one at a time.
    with Server(workers=2, max_batch=8, hbm_budget=1) as srv:
        tickets = [srv.submit(**p) for p in pairs]
        res = [srv.wait(t) for t in tickets]
    for a, (m, tm) in zip(alone, res):
        _same(m, a)
        assert tm["batch_size"] == 1


def test_server_keyed_left_image_cached(pairs):
    """A view's partner pairs share its left image under one content key:
    the first request uploads it, the others find it cached (on either
    worker's stream); every map equals the uncached request's."""
    p = pairs[3]
    variants = [dict(p, right=np.roll(p["right"], s, axis=1)) for s in (0, 1, 2, 3)]
    with Server(workers=2, max_batch=1, hbm_budget=16 << 30, scratch_budget=8 << 30) as srv:
        plain = [srv.wait(srv.submit(**q))[0] for q in variants]
    with Server(workers=2, max_batch=2, hbm_budget=16 << 30, scratch_budget=8 << 30, cache_budget=1 << 30) as srv:
        first = srv.wait(srv.submit(**variants[0], left_key=11))
        tickets = [srv.submit(**q, left_key=11) for q in variants[1:]]
        rest = [srv.wait(t) for t in tickets]
    _same(first[0], plain[0])
    assert first[1]["cache_hits"] == 0
    for (m, tm), a in zip(rest, plain[1:]):
        _same(m, a)
        assert tm["cache_hits"] == 1
        assert tm["uploaded_bytes"] == p["right"].size * 2
