"""The CUDA kernel sources, run on the CPU SIMT emulator, against the oracle.

The emulator (tests/simt) compiles the same kernel and host sources as the
product library with every CUDA thread as a fiber: barriers and shuffles
switch fibers, cp.async copies land at their wait, and a barrier that cannot
complete is an error. These tests check kernel logic and index arithmetic
without a GPU; the GPU tests repeat them on the B200.
"""

from __future__ import annotations

import numpy as np
import pytest

from images import Rng, Texture, mismatch_report, random_image, render_pair, same_disparities, to_u16
from regard3d_mvs_b200.types import LabelRanges, StereoOptions, SubpixelMethod


def _same_map(a, b):
    assert same_disparities(a.disparity, b.disparity), mismatch_report(a.disparity, b.disparity)
    assert np.array_equal(a.confidence, b.confidence)
    assert a.cells == b.cells and a.levels == b.levels


def test_census_and_pyramid(simt_matcher, oracle):
    for w in (1, 5, 31, 77):
        img = random_image(w, 13, w)
        assert np.array_equal(simt_matcher.census_transform(img), oracle.census_transform(img))
        assert np.array_equal(simt_matcher.pyramid_down(img), oracle.pyramid_down(img))


@pytest.mark.parametrize("dmin,nd,p2_adapt", [(-3, 16, 0), (2, 48, 12)])
def test_volume(simt_matcher, oracle, dmin, nd, p2_adapt):
    tex = Texture(3)
    left, right, _ = render_pair(tex, 41, 23, lambda x, y: 5.0 + 0.1 * x)
    right = right ^ (random_image(41, 23, 9) & 0x0F00)
    o = StereoOptions(p2=120, p2_adapt=p2_adapt)
    assert np.array_equal(simt_matcher.sgm_cost_volume(left, right, dmin, nd, o),
                          oracle.sgm_cost_volume(left, right, dmin, nd, o))


@pytest.mark.parametrize("shape,nd", [("2,16", 48), ("4,16", 128), ("8,16", 208), ("8,8", 112), ("4,12", 96)])
@pytest.mark.parametrize("p2", [120, 8000])
def test_volume_chain_shapes(simt_matcher, oracle, monkeypatch, shape, nd, p2):
    """Every chain-pass shape selectable by R3DGPU_PATH_SHAPE (lanes per
    chain, label pairs per lane) against the textbook volume, with byte terms
    (P2 <= 255) and with u16 sums (P2 = 8000: sums that wrap)."""
    monkeypatch.setenv("R3DGPU_PATH_SHAPE", shape)
    tex = Texture(19)
    left, right, _ = render_pair(tex, 30, 17, lambda x, y: 7.0 + 0.2 * x)
    o = StereoOptions(p1=20, p2=p2, p2_adapt=0 if p2 > 255 else 6, invalid_cost=40)
    assert np.array_equal(simt_matcher.sgm_cost_volume(left, right, -1, nd, o),
                          oracle.sgm_cost_volume(left, right, -1, nd, o))


@pytest.mark.parametrize("terms", ["0", "1"])
def test_ranged_term_modes(simt_matcher, oracle, monkeypatch, terms):
    """Per-pixel ranges through the chain passes with u16 sums (the default)
    and with byte terms (R3DGPU_RANGED_TERMS=1): volume and a hierarchical
    match against the oracle."""
    monkeypatch.setenv("R3DGPU_RANGED_TERMS", terms)
    tex = Texture(29)
    w, h, nd = 33, 21, 112
    left, right, _ = render_pair(tex, w, h, lambda x, y: 25.0 + 0.4 * x - 0.2 * y)
    r = Rng(37)
    num = np.array([[16 * r.uniform_int(1, 5) for _ in range(w)] for _ in range(h)], np.uint16)
    lo = np.array([[r.uniform_int(0, nd - int(n)) for n in row] for row in num], np.uint16)
    o = StereoOptions(p2=140, p2_adapt=5)
    assert np.array_equal(simt_matcher.sgm_cost_volume(left, right, 1, nd, o, LabelRanges(lo, num)),
                          oracle.sgm_cost_volume(left, right, 1, nd, o, (lo, num)))
    left, right, _ = render_pair(tex, 120, 64, lambda x, y: np.where(x < 50, 9.0, 21.0))
    o = StereoOptions(levels=2, tile_size=48, tile_margin=8, tile_blend=8, range_radius=1)
    a = simt_matcher.match_stereo(left, right, None, None, 0, 48, o)
    b = oracle.match_stereo(left, right, None, None, 0, 48, o)
    assert same_disparities(a.disparity, b.disparity), mismatch_report(a.disparity, b.disparity)
    assert a.cells == b.cells


def test_volume_ranges_and_wrap(simt_matcher, oracle):
    tex = Texture(13)
    w, h, nd = 37, 19, 96
    left, right, _ = render_pair(tex, w, h, lambda x, y: 20.0 + 0.5 * x - 0.3 * y)
    r = Rng(31)
    num = np.array([[16 * r.uniform_int(1, 3) for _ in range(w)] for _ in range(h)], np.uint16)
    lo = np.array([[r.uniform_int(0, nd - int(n)) for n in row] for row in num], np.uint16)
    o = StereoOptions(p2=150, p2_adapt=8)
    assert np.array_equal(simt_matcher.sgm_cost_volume(left, right, -2, nd, o, LabelRanges(lo, num)),
                          oracle.sgm_cost_volume(left, right, -2, nd, o, (lo, num)))
    # Penalties large enough that the sum of 8 paths wraps modulo 2^16, and
    # more than one 64-label chunk per pixel.
    o = StereoOptions(p1=300, p2=8000, p2_adapt=0, invalid_cost=255)
    left, right, _ = render_pair(tex, 24, 9, lambda x, y: 30.0 + 0.2 * x)
    assert np.array_equal(simt_matcher.sgm_cost_volume(left, right, -5, 144, o),
                          oracle.sgm_cost_volume(left, right, -5, 144, o))


@pytest.mark.parametrize("opts", [
    StereoOptions(tile_size=32, tile_margin=4, tile_blend=4, levels=0),
    StereoOptions(tile_size=32, tile_margin=4, tile_blend=4, levels=0, lr_full_match=False, uniqueness=0.1),
    StereoOptions(tile_size=32, tile_margin=4, tile_blend=4, levels=1, subpixel=SubpixelMethod.parabola),
])
def test_match_stereo(simt_matcher, oracle, opts):
    tex = Texture(5)
    left, right, _ = render_pair(tex, 64, 40, lambda x, y: np.where(x < 30, 4.0, 9.5))
    lm = np.full((40, 64), 255, np.uint8)
    lm[:, 56:] = 0
    lm[5, :] = 0
    _same_map(simt_matcher.match_stereo(left, right, lm, None, 0, 16, opts),
              oracle.match_stereo(left, right, lm, None, 0, 16, opts))


def test_widths_and_negative_disparities(simt_matcher, oracle):
    tex = Texture(23)
    wl, wr, h = 50, 66, 24
    yy, xl = np.mgrid[0:h, 0:wl].astype(np.float64)
    yr, xr = np.mgrid[0:h, 0:wr].astype(np.float64)
    left = to_u16(tex(xl, yy))
    right = to_u16(tex(xr - 5.0, yr))
    o = StereoOptions(levels=1, tile_size=32)
    _same_map(simt_matcher.match_stereo(left, right, None, None, -12, 16, o),
              oracle.match_stereo(left, right, None, None, -12, 16, o))


def test_batch_equals_single(simt_matcher):
    tex = Texture(7)
    pairs = []
    for i, (w, h, nd, lv) in enumerate(((48, 32, 16, 0), (40, 36, 32, 1), (24, 20, 16, -1))):
        left, right, _ = render_pair(tex, w, h, lambda x, y: 3.0 + 0.05 * x + i)
        pairs.append(dict(left=left, right=right, num_disparities=nd, options=StereoOptions(levels=lv, tile_size=32)))
    batch = simt_matcher.match_stereo_batch(pairs)
    for p, b in zip(pairs, batch):
        _same_map(b, simt_matcher.match_stereo(p["left"], p["right"], None, None, 0, p["num_disparities"],
                                               p["options"]))


def test_filters_and_ranges(simt_matcher, oracle):
    rng = np.random.default_rng(3)
    d = np.round(rng.normal(20, 3, (30, 40))).astype(np.float32)
    d[rng.random(d.shape) < 0.1] = np.inf
    for size in (2, 6, 40):
        assert same_disparities(simt_matcher.remove_speckles(d.copy(), size, 1.0), oracle.remove_speckles(d, size, 1.0))
    assert same_disparities(simt_matcher.median_filter_3x3(d), oracle.median_filter_3x3(d))
    coarse = np.where(rng.random((10, 20)) < 0.2, np.inf, rng.uniform(3, 20, (10, 20))).astype(np.float32)
    valid = np.full((20, 40), 255, np.uint8)
    valid[2, 3] = 0
    o = StereoOptions(range_radius=1, range_margin=3, range_fill=4)
    for sign, mir in ((-1, False), (1, True)):
        a = simt_matcher.ranges_from_coarse(coarse, 40, 20, valid, valid, 40, sign, 1, 48, o, mir)
        b = oracle.ranges_from_coarse(coarse, 40, 20, valid, valid, 40, sign, 1, 48, o, mir)
        assert np.array_equal(a.lo, b[0]) and np.array_equal(a.num, b[1])


def test_invalid_input_is_rejected(simt_matcher):
    from regard3d_mvs_b200 import StereoError

    img = random_image(16, 8, 1)
    with pytest.raises(StereoError):
        simt_matcher.match_stereo(img, img, None, None, 0, 16, StereoOptions(p2=9000))
    with pytest.raises(StereoError):
        simt_matcher.match_stereo(img, img[:4], None, None, 0, 16)
    with pytest.raises(StereoError):
        simt_matcher.sgm_cost_volume(img, img, 0, 32, None,
                                     LabelRanges(np.zeros((8, 16), np.uint16), np.full((8, 16), 48, np.uint16)))


def _smooth_ranges(w, h, nd, seed, wide_frac=0.08):
    """Per-pixel ranges shaped like a hierarchical level's: lo drifts slowly
    (small shifts between neighbours, now and then a jump), num mostly 16 or
    32, a few wide pixels."""
    rng = np.random.default_rng(seed)
    base = np.cumsum(rng.integers(-1, 2, (h, w)) * (rng.random((h, w)) < 0.3), axis=1)
    base = base + np.cumsum(rng.integers(-2, 3, (h, 1)), axis=0)
    jumps = rng.random((h, w)) < 0.03
    base = base + np.where(jumps, rng.integers(-40, 40, (h, w)), 0)
    num = np.where(rng.random((h, w)) < 0.2, 16, 32)
    wide = rng.random((h, w)) < wide_frac
    num = np.minimum(np.where(wide, rng.choice([48, 64, 96, nd], (h, w)), num), nd).astype(np.int64)
    lo = np.clip(nd // 3 + base, 0, nd - num)
    return lo.astype(np.uint16), num.astype(np.uint16)


@pytest.mark.parametrize("shape,rows", [("4,4", 8), ("8,4", 4), ("4,4", 32), ("8,8", 4), ("16,12", 2), ("32,8", 3)])
def test_ranged_kernel_volume(simt_matcher, oracle, monkeypatch, shape, rows):
    """Ranged kernel: aligned, shifted and bounds-checked predecessor reads,
    wide pixels, band seams (few rows per band), against the textbook volume."""
    monkeypatch.setenv("R3DGPU_RANGED_SHAPE", shape)
    monkeypatch.setenv("R3DGPU_RANGED_ROWS", str(rows))
    tex = Texture(29)
    w, h, nd = 37, 29, 128
    left, right, _ = render_pair(tex, w, h, lambda x, y: 40.0 + 0.3 * x - 0.2 * y)
    lo, num = _smooth_ranges(w, h, nd, 5)
    for o in (StereoOptions(p2=150, p2_adapt=8), StereoOptions(p1=300, p2=8000, p2_adapt=0, invalid_cost=255)):
        assert np.array_equal(simt_matcher.sgm_cost_volume(left, right, -3, nd, o, LabelRanges(lo, num)),
                              oracle.sgm_cost_volume(left, right, -3, nd, o, (lo, num)))


@pytest.mark.parametrize("lr_full", [True, False])
def test_ranged_kernel_hierarchy(simt_matcher, oracle, monkeypatch, lr_full):
    """The hierarchy through the ranged kernel with many bands per tile."""
    monkeypatch.setenv("R3DGPU_RANGED_ROWS", "8")
    tex = Texture(31)
    left, right, _ = render_pair(tex, 72, 52, lambda x, y: np.where(x < 35, 6.0 + 0.05 * y, 17.5))
    o = StereoOptions(levels=2, tile_size=48, tile_margin=8, tile_blend=8, lr_full_match=lr_full, range_radius=1,
                      range_margin=4)
    _same_map(simt_matcher.match_stereo(left, right, None, None, 0, 32, o),
              oracle.match_stereo(left, right, None, None, 0, 32, o))


@pytest.mark.parametrize("opts", [
    StereoOptions(levels=1, range_margin=20, tile_size=32, tile_margin=4, tile_blend=4, uniqueness=0.05),
    StereoOptions(levels=1, range_margin=20, tile_size=32, tile_margin=4, tile_blend=4, lr_full_match=False,
                  subpixel=SubpixelMethod.parabola),
])
def test_ranged_kernel_wide_pixels_wta(simt_matcher, oracle, monkeypatch, opts):
    """Large range margins make most pixels wider than a row's narrow width:
    the warp-cooperative wide path decides the winners, second bests,
    subpixel neighbours and diagonal LR keys."""
    monkeypatch.setenv("R3DGPU_RANGED_ROWS", "8")
    tex = Texture(37)
    left, right, _ = render_pair(tex, 60, 34, lambda x, y: np.where(y < 15, 9.0 + 0.1 * x, 21.0))
    _same_map(simt_matcher.match_stereo(left, right, None, None, 0, 48, opts),
              oracle.match_stereo(left, right, None, None, 0, 48, opts))


def test_speckles_across_union_tiles(simt_matcher, oracle):
    """Segments spanning many 32 x 32 union tiles (smooth ramps, a large
    plateau, thin diagonal strips and noise) against the reference BFS."""
    rng = np.random.default_rng(8)
    h, w = 97, 131
    yy, xx = np.mgrid[0:h, 0:w]
    d = (0.01 * xx + 0.02 * yy).astype(np.float32)                 # one segment crossing every tile
    d[20:70, 40:100] = 30.0                                       # plateau over tile borders
    d[(xx + yy) % 17 == 0] = 50.0                                 # diagonal strips (cut at tile corners)
    noise = rng.random((h, w)) < 0.05
    d[noise] = np.round(rng.normal(10, 5, noise.sum())).astype(np.float32)
    d[rng.random((h, w)) < 0.03] = np.inf
    for size, diff in ((5, 0.5), (40, 1.0), (400, 1.0), (3000, 0.2)):
        assert same_disparities(simt_matcher.remove_speckles(d.copy(), size, diff),
                                oracle.remove_speckles(d, size, diff)), (size, diff)
