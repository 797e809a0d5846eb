"""Cancellation of the matcher entry points: the r3dgpu_cancel_token of
include/r3dgpu.h, the counterpart of the reference's per-thread CancelToken
(src/r3d/core/cancel.hpp:36-55) that its thread pool polls before every tile
chunk (src/r3d/core/thread_pool.cpp:53-55). The library polls the token on
the host between hierarchy rounds and waves of tiles, and the chain-pass
kernels read it once per chain block (never waiting on it): a cancelled call
returns R3DGPU_ECANCELLED once its enqueued work has ended, and the next call
after a reset gives the normal result."""

from __future__ import annotations

import threading
import time

import numpy as np
import pytest

from images import Texture, render_pair, same_disparities
from regard3d_mvs_b200 import StereoError
from regard3d_mvs_b200.types import StereoOptions

ECANCELLED = 2


def _pairs():
    tex = Texture(71)
    out = []
    for lv in (0, 1):
        left, right, _ = render_pair(tex, 64, 40, lambda x, y: 6.0 + 0.1 * x)
        out.append(dict(left=left, right=right, disparity_min=0, num_disparities=32,
                        options=StereoOptions(levels=lv, tile_size=32)))
    return out


def _check_cancel_and_reset(m):
    pairs = _pairs()
    ref = m.match_stereo_batch(pairs)
    tok = m.cancel_token()
    try:
        m.set_cancel_token(tok)
        tok.cancel()
        assert tok.requested()
        with pytest.raises(StereoError) as e:
            m.match_stereo_batch(pairs)
        assert e.value.status == ECANCELLED
        with pytest.raises(StereoError) as e:
            m.match_stereo(pairs[0]["left"], pairs[0]["right"], None, None, 0, 32, pairs[0]["options"])
        assert e.value.status == ECANCELLED
        tok.reset()
        got = m.match_stereo_batch(pairs)
        for a, b in zip(got, ref):
            assert same_disparities(a.disparity, b.disparity) and a.cells == b.cells
    finally:
        m.set_cancel_token(None)
        tok.close()


def test_cancel_on_the_emulator(simt_matcher):
    _check_cancel_and_reset(simt_matcher)


@pytest.mark.gpu
def test_cancel_before_the_call(gpu_matcher):
    _check_cancel_and_reset(gpu_matcher)


@pytest.mark.gpu
def test_cancel_during_a_batch(gpu_matcher):
    """A token set from another thread while a long batch runs: the call ends
    early with R3DGPU_ECANCELLED (the kernels stop taking chain blocks), and
    the device and library stay usable."""
    from test_gpu_parity import _synthetic_pair

    left, right = _synthetic_pair(3072, 2048, 256, 5)
    pairs = [dict(left=left, right=right, disparity_min=0, num_disparities=256, options=StereoOptions(levels=0))
             for _ in range(6)]
    m = gpu_matcher
    t0 = time.perf_counter()
    full = m.match_stereo_batch(pairs)
    full_s = time.perf_counter() - t0
    tok = m.cancel_token()
    try:
        m.set_cancel_token(tok)
        timer = threading.Timer(0.1 * full_s, tok.cancel)
        timer.start()
        t0 = time.perf_counter()
        with pytest.raises(StereoError) as e:
            m.match_stereo_batch(pairs)
        cancelled_s = time.perf_counter() - t0
        timer.join()
        assert e.value.status == ECANCELLED
        assert cancelled_s < 0.75 * full_s, (cancelled_s, full_s)
        tok.reset()
        again = m.match_stereo_batch(pairs[:1])
        assert same_disparities(again[0].disparity, full[0].disparity)
    finally:
        m.set_cancel_token(None)
        tok.close()
