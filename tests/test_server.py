"""The serving loop (include/r3dgpu_server.h) on the CPU SIMT emulator: every
result equals the pair matched alone, whatever batch it ran in; admission
keeps the estimated device memory of the running requests within the budget;
invalid requests are refused at submission; destroying a server finishes the
queued requests."""

from __future__ import annotations

import threading

import numpy as np
import pytest

from conftest import SIMT_LIB
from images import Texture, mismatch_report, render_pair, same_disparities
from regard3d_mvs_b200 import Server, StereoError, StereoOptions


def _pairs():
    tex = Texture(41)
    out = []
    for i, (w, h, nd, lv) in enumerate(((32, 18, 16, 0), (28, 22, 16, 1), (24, 16, 16, -1), (36, 18, 16, 1),
                                        (20, 20, 16, 0), (30, 20, 32, 1))):
        left, right, _ = render_pair(tex, w, h, lambda x, y, i=i: 3.0 + 0.05 * x + i)
        out.append(dict(left=left, right=right, disparity_min=0, num_disparities=nd,
                        options=StereoOptions(levels=lv, tile_size=32)))
    return out


def _same(a, b):
    assert same_disparities(a.disparity, b.disparity), mismatch_report(a.disparity, b.disparity)
    assert np.array_equal(a.confidence, b.confidence)
    assert (a.cells, a.levels, a.num_disparities) == (b.cells, b.levels, b.num_disparities)


@pytest.fixture(scope="module")
def pairs():
    return _pairs()


@pytest.fixture(scope="module")
def alone(simt_matcher, pairs):
    """Each pair matched by itself."""
    return [simt_matcher.match_stereo(p["left"], p["right"], None, None, p["disparity_min"], p["num_disparities"],
                                      p["options"]) for p in pairs]


def test_mix_equals_alone(pairs, alone):
    with Server(SIMT_LIB, workers=2, max_batch=3, hbm_budget=1 << 30) as srv:
        tickets = [srv.submit(**p) for p in pairs]
        results = [srv.wait(t) for t in tickets]
    for a, (m, times) in zip(alone, results):
        _same(m, a)
        assert 1 <= times["batch_size"] <= 3 and times["worker"] in (0, 1)
        assert times["total_ms"] >= times["run_ms"] >= 0.0
    assert max(t["batch_size"] for _, t in results) > 1  # some requests did share a batch


def test_budget_admits_one_request_at_a_time(pairs, alone):
    # Every request's estimate exceeds half the budget: no two run together.
    with Server(SIMT_LIB, workers=2, max_batch=8, hbm_budget=(1 << 20) + 150_000) as srv:
        tickets = [srv.submit(**p) for p in pairs[:4]]
        results = [srv.wait(t) for t in tickets]
    for a, (m, times) in zip(alone, results):
        assert 2 * times["device_bytes"] > (1 << 20) + 150_000
        assert times["batch_size"] == 1
        _same(m, a)


def test_concurrent_submitters_and_errors(pairs, alone):
    got = {}
    with Server(SIMT_LIB, workers=2, max_batch=4, hbm_budget=1 << 30) as srv:
        with pytest.raises(StereoError):  # unequal heights: refused at submission
            srv.submit(pairs[0]["left"], pairs[0]["right"][:5], num_disparities=16)
        with pytest.raises(StereoError):  # invalid options
            srv.submit(pairs[0]["left"], pairs[0]["right"], num_disparities=16, options=StereoOptions(p2=9000))
        lock = threading.Lock()

        def client(idx):
            t = srv.submit(**pairs[idx])
            m, _ = srv.wait(t)
            with lock:
                got[idx] = m

        threads = [threading.Thread(target=client, args=(i,)) for i in range(len(pairs))]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
    for i, a in enumerate(alone):
        _same(got[i], a)


def test_destroy_finishes_queued_requests(pairs, alone):
    srv = Server(SIMT_LIB, workers=1, max_batch=1, hbm_budget=1 << 30)
    tickets = [srv.submit(**p) for p in pairs[:3]]
    # The maps are written into the host buffers the requests point to.
    outs = [srv._live[t][1][4] for t in tickets]
    srv.close()
    for a, d in zip(alone, outs):
        assert same_disparities(d, a.disparity)


def test_keyed_images_are_uploaded_once(pairs, alone):
    """Requests that share a keyed left image (a view's partner pairs): the
    image goes to the device once and stays cached; every result equals the
    pair matched alone, and a cache too small for an image falls back to
    staging it."""
    p = pairs[0]
    shifted = [dict(p, right=np.roll(p["right"], s, axis=1)) for s in (0, 1, 2)]
    ref = [alone[0]] + [None, None]
    with Server(SIMT_LIB, workers=2, max_batch=1, hbm_budget=1 << 30, cache_budget=1 << 20) as srv:
        first = srv.wait(srv.submit(**shifted[0], left_key=7))
        rest = [srv.wait(srv.submit(**q, left_key=7)) for q in shifted[1:]]
    _same(first[0], ref[0])
    assert first[1]["cache_hits"] == 0
    assert all(t["cache_hits"] == 1 for _, t in rest)
    nbytes = p["left"].size * 2
    assert all(t["uploaded_bytes"] == nbytes for _, t in rest)  # the right image only
    with Server(SIMT_LIB, workers=1, max_batch=1, hbm_budget=1 << 30) as srv:
        plain = [srv.wait(srv.submit(**q)) for q in shifted[1:]]
    for (a, _), (b, _) in zip(rest, plain):
        _same(a, b)
    with Server(SIMT_LIB, workers=1, max_batch=1, hbm_budget=1 << 30, cache_budget=16) as srv:
        m, t = srv.wait(srv.submit(**shifted[0], left_key=7))
    _same(m, ref[0])
    assert t["cache_hits"] == 0 and t["uploaded_bytes"] == 2 * nbytes
