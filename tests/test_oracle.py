"""Pins the CPU oracle to the reference's own tests (CPU only).

Each test restates a test of rhiestan/Regard3D_MVS for the matcher path
(tests/test_census.cpp, tests/test_stereo.cpp, tests/test_pyramid.cpp) and
checks the oracle (oracle/r3d_oracle.cpp) against the reference's known
answers and thresholds. The oracle is then the checker of the GPU library.
"""

from __future__ import annotations

import numpy as np
import pytest

from images import Rng, Texture, evaluate_disparity, random_image, render_pair, same_disparities
from regard3d_mvs_b200.types import StereoOptions, SubpixelMethod


def test_census_bit_order(oracle):
    # tests/test_census.cpp:26-43
    img = np.full((7, 9), 100, np.uint16)
    assert oracle.census_transform(img)[3, 4] == 0
    img[3, 4] = 200
    assert oracle.census_transform(img)[3, 4] == (1 << 62) - 1
    img[:] = 100
    img[0, 0] = 50
    assert oracle.census_transform(img)[3, 4] == 1 << 61
    img[0, 0] = 100
    img[6, 8] = 50
    assert oracle.census_transform(img)[3, 4] == 1
    img[6, 8] = 100
    img[3, 5] = 50
    assert oracle.census_transform(img)[3, 4] == 1 << 30


def test_census_replicated_borders(oracle):
    # tests/test_census.cpp:45-65
    img = (10 * np.arange(20, dtype=np.uint16))[None, :].repeat(10, 0)
    c = oracle.census_transform(img)
    assert c[5, 0] == 0
    expected = 0
    for j in range(7):
        for i in range(9):
            if j == 3 and i == 4:
                continue
            expected = (expected << 1) | (1 if i < 4 else 0)
    assert c[5, 10] == expected


def _float_pyramid(img: np.ndarray) -> np.ndarray:
    w = np.array([1, 4, 6, 4, 1], np.float64)
    h, wd = img.shape
    dw, dh = (wd + 1) // 2, (h + 1) // 2
    xs = np.clip(2 * np.arange(dw)[:, None] + np.arange(-2, 3)[None, :], 0, wd - 1)
    ys = np.clip(2 * np.arange(dh)[:, None] + np.arange(-2, 3)[None, :], 0, h - 1)
    t = (img.astype(np.float64)[:, xs] * w).sum(-1)  # h x dw
    return (t[ys, :] * w[None, :, None]).sum(1) / 256.0


def test_pyramid_exact_rounding(oracle):
    # tests/test_pyramid.cpp:58-91 (single channel)
    rng = np.random.default_rng(7)
    u8 = rng.integers(0, 256, (41, 77), dtype=np.uint8)
    a = oracle.pyramid_down(u8)
    assert a.shape == (21, 39)
    b = np.floor(_float_pyramid(u8) + 0.5)
    assert np.array_equal(a.astype(np.float64), b)
    flat = np.full((9, 9), 54321, np.uint16)
    d = oracle.pyramid_down(flat)
    assert d[0, 0] == 54321 and d[4, 4] == 54321


def test_explicit_full_ranges_equal_no_ranges(oracle):
    # tests/test_stereo.cpp:146-150
    tex = Texture(13)
    w, h, nd = 37, 19, 96
    left, right, _ = render_pair(tex, w, h, lambda x, y: 20.0 + 0.5 * x - 0.3 * y)
    o = StereoOptions(p2=150, p2_adapt=8)
    full = (np.zeros((h, w), np.uint16), np.full((h, w), nd, np.uint16))
    assert np.array_equal(oracle.sgm_cost_volume(left, right, -2, nd, o, full),
                          oracle.sgm_cost_volume(left, right, -2, nd, o))


@pytest.mark.parametrize("method", [SubpixelMethod.parabola, SubpixelMethod.equiangular])
def test_slanted_plane_accuracy(oracle, method):
    # tests/test_stereo.cpp:191-212
    tex = Texture(11)
    w, h = 200, 120
    left, right, gt = render_pair(tex, w, h, lambda x, y: 12.3 + 0.04 * x + 0.02 * y)
    r = oracle.match_stereo(left, right, None, None, 0, 32, StereoOptions(subpixel=method))
    assert r.num_disparities == 32
    mask = np.zeros((h, w), np.uint8)
    mask[:, 30:] = 255
    density, bad1, avg = evaluate_disparity(r.disparity, gt, mask)
    assert density > 0.95 and bad1 < 0.01 and avg < 0.2


def test_tiles_consistent(oracle):
    # tests/test_stereo.cpp:214-253 (tiled and whole-image results agree away from the step)
    tex = Texture(5)
    w, h = 150, 90
    left, right, gt = render_pair(tex, w, h, lambda x, y: np.where(x < 70, 6.0, 14.5))
    tiled = oracle.match_stereo(left, right, None, None, 0, 32, StereoOptions(tile_size=48, tile_margin=8, tile_blend=8))
    whole = oracle.match_stereo(left, right, None, None, 0, 32, StereoOptions(tile_size=1024))
    mask = np.zeros((h, w), np.uint8)
    xs = np.arange(w)
    mask[:, (xs >= 20) & (np.abs(xs - 70) > 12)] = 255
    for r in (tiled, whole):
        density, bad1, _ = evaluate_disparity(r.disparity, gt, mask)
        assert density > 0.95 and bad1 < 0.01


def test_masks(oracle):
    # tests/test_stereo.cpp:255-276
    tex = Texture(8)
    left, right, _ = render_pair(tex, 120, 60, lambda x, y: 10.0 + 0 * x)
    lm = np.full((60, 120), 255, np.uint8)
    rm = np.full((60, 120), 255, np.uint8)
    lm[:, 100:] = 0
    rm[:, :40] = 0
    r = oracle.match_stereo(left, right, lm, rm, 0, 32)
    assert not np.isfinite(r.disparity[:, 100:]).any()
    assert not np.isfinite(r.disparity[:, :40]).any()
    good = (np.abs(r.disparity[:, 55:95] - 10.0) < 0.25).sum()
    assert good > 0.95 * 60 * 40


@pytest.mark.parametrize("full", [False, True])
def test_masked_left_pixels_lr(oracle, full):
    # tests/test_stereo.cpp:278-313
    tex = Texture(21)
    left, right, _ = render_pair(tex, 160, 60, lambda x, y: 10.0 + 0 * x)
    rng = Rng(4)
    noise = np.array([[rng.normal(0.0, 3000.0) for _ in range(160)] for _ in range(60)])
    noise2 = np.array([[rng.normal(0.0, 3000.0) for _ in range(160)] for _ in range(60)])
    # The reference draws left and right noise interleaved per pixel.
    noise_l = np.empty((60, 160))
    noise_r = np.empty((60, 160))
    flat = np.concatenate([noise.ravel(), noise2.ravel()])
    noise_l.ravel()[:] = flat[0::2]
    noise_r.ravel()[:] = flat[1::2]
    from images import to_u16

    left = to_u16(left + noise_l)
    right = to_u16(right + noise_r)
    y, x = np.mgrid[0:60, 0:160]
    lmask = np.where(x < 70 + 2 * y, 255, 0).astype(np.uint8)
    valid = int(((lmask > 0) & (x >= 20)).sum())
    o = StereoOptions(lr_full_match=full, tile_size=64)
    r = oracle.match_stereo(left, right, lmask, None, 0, 256, o)
    good = ((lmask > 0) & (x >= 20) & (np.abs(r.disparity - 10.0) < 0.5)).sum()
    assert good > 0.75 * valid


@pytest.mark.parametrize("levels", [0, 1])
@pytest.mark.parametrize("full", [False, True])
def test_lr_different_widths(oracle, levels, full):
    # tests/test_stereo.cpp:315-341
    tex = Texture(23)
    wl, wr, h, d = 150, 190, 60, -7.0
    y, xl = np.mgrid[0:h, 0:wl].astype(np.float64)
    _, xr = np.mgrid[0:h, 0:wr].astype(np.float64)
    from images import to_u16

    left = to_u16(tex(xl, y))
    right = to_u16(tex(xr + d, np.mgrid[0:h, 0:wr][0]))
    r = oracle.match_stereo(left, right, None, None, -20, 32, StereoOptions(lr_full_match=full, levels=levels))
    assert r.levels == levels
    good = (np.abs(r.disparity - d) < 0.25).sum()
    assert good > 0.9 * wl * h


def test_ranges_from_coarse_kat(oracle):
    # tests/test_stereo.cpp:343-400
    wc, hc = 40, 20
    coarse = np.where(np.arange(wc)[None, :] < wc // 2, 10.0, 30.0).astype(np.float32).repeat(hc, 0)
    coarse[5, 5] = np.inf
    coarse[:, 30:] = np.inf
    w, h, dmin, nd = 2 * wc, 2 * hc, 4, 96
    valid = np.full((h, w), 255, np.uint8)
    valid[1, 1] = 0
    o = StereoOptions(range_radius=1, range_margin=3, range_fill=4)
    lo, num = oracle.ranges_from_coarse(coarse, w, h, valid, None, 1000, 1, dmin, nd, o)

    def covers(x, y, a, b):
        return lo[y, x] <= a and lo[y, x] + num[y, x] - 1 >= b

    assert (num % 16 == 0).all() and (lo.astype(int) + num <= nd).all()
    assert covers(10, 30, 20 - dmin - 3, 20 - dmin + 3) and num[30, 10] == 16
    assert covers(10, 10, 20 - dmin - 3, 20 - dmin + 3) and num[10, 10] == 16
    assert covers(39, 20, 20 - dmin - 3, 60 - dmin + 3)
    assert num[1, 1] == 16
    assert covers(62, 20, 60 - dmin - 3, 60 - dmin + 3) and num[20, 62] == 16
    assert lo[20, 78] == 0 and num[20, 78] == nd
    clo, cnum = oracle.ranges_from_coarse(coarse, w, h, valid, None, w, -1, dmin, nd, o)
    assert cnum[30, 10] == 16
    assert clo[30, 30] <= 20 - dmin - 3
    assert clo[30, 30] + cnum[30, 30] - 1 >= 20 - dmin + 3
    assert clo[20, 78] + cnum[20, 78] - 1 < 78 - dmin + 16


def test_hierarchical_equals_full_range(oracle):
    # tests/test_stereo.cpp:402-449
    tex, hidden = Texture(29), Texture(31)
    w, h, step = 480, 300, 300
    y, x = np.mgrid[0:h, 0:w].astype(np.float64)

    def d_fg(x, y):
        return 150.0 + 0.1 * y - 0.05 * x

    def d_bg(x, y):
        return 40.0 + 0.02 * x

    from images import to_u16

    left = to_u16(tex(x, y))
    gt = np.where(x < step, d_fg(x, y), d_bg(x, y)).astype(np.float32)
    xf = x.copy()
    for _ in range(30):
        xf = x + d_fg(xf, y)
    xb = x.copy()
    for _ in range(30):
        xb = x + d_bg(xb, y)
    right = np.where(xf < step, to_u16(tex(xf, y)), np.where(xb >= step, to_u16(tex(xb, y)), to_u16(hidden(xb, y))))
    mask = np.zeros((h, w), np.uint8)
    xs = np.arange(w)
    mask[:, (xs >= 200) & (np.abs(xs - step) > 12)] = 255
    full = oracle.match_stereo(left, right, None, None, 0, 256, StereoOptions(levels=0))
    hier = oracle.match_stereo(left, right, None, None, 0, 256, StereoOptions(levels=-1))
    assert full.levels == 0 and hier.levels >= 1
    assert hier.cells * 3 < full.cells
    sf = evaluate_disparity(full.disparity, gt, mask)
    sh = evaluate_disparity(hier.disparity, gt, mask)
    assert sf[0] > 0.95 and sf[1] < 0.01 and sh[0] > 0.95 and sh[1] < 0.01
    assert sh[0] >= sf[0] - 0.01 and sh[2] <= sf[2] + 0.02


def test_speckle_and_median_kat(oracle):
    # tests/test_stereo.cpp:451-469
    d = np.full((10, 20), 5.0, np.float32)
    d[3, 3] = 20.0
    d[5, 10] = np.inf
    d[0, 15:20] = 30.0
    s = oracle.remove_speckles(d, 6, 1.0)
    assert not np.isfinite(s[3, 3]) and not np.isfinite(s[0, 17]) and s[0, 0] == 5.0
    s = oracle.remove_speckles(d, 5, 1.0)
    assert s[0, 17] == 30.0
    m = oracle.median_filter_3x3(d)
    assert m[3, 3] == 5.0 and not np.isfinite(m[5, 10]) and m[5, 11] == 5.0


def test_automatic_levels(oracle):
    # stereo_matcher.cpp:1105-1122 on the reference bench and config sizes
    assert oracle.automatic_levels(480, 300, 256) >= 1
    assert oracle.automatic_levels(640, 480, 48) == 0
    assert oracle.automatic_levels(3072, 2048, 256) == 3


def test_oracle_rejects_invalid_options(oracle):
    left = random_image(32, 16, 1)
    with pytest.raises(oracle.OracleError):
        oracle.match_stereo(left, left, None, None, 0, 16, StereoOptions(p1=300, p2=200))
    with pytest.raises(oracle.OracleError):
        oracle.match_stereo(left, left, None, None, 0, 0)
    with pytest.raises(oracle.OracleError):
        oracle.match_stereo(left, left[:8], None, None, 0, 16)
