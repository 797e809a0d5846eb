"""GPU parity: the CUDA library (through its C ABI) against the CPU oracle.

Integer outputs (Census codes, aggregated volumes, label ranges, cell
counts) must be bit-exact; disparity maps too, since the library reproduces
the reference's float operations one by one (tolerance 0 here; the contract
bound for subpixel values is 1e-4 px). Cases follow the reference's stereo
tests (tests/test_stereo.cpp) plus the 640x480 / 128-label single-level pair
and a smaller hierarchical pair.
"""

from __future__ import annotations

import numpy as np
import pytest

from images import Rng, Texture, mismatch_report, random_image, render_pair, same_disparities, to_u16
from regard3d_mvs_b200.types import LabelRanges, StereoOptions, SubpixelMethod

pytestmark = pytest.mark.gpu

SUBPIXEL_TOL = 1e-4  # px; disparities are compared exactly, the bound is stated for the record


def _assert_same_map(a, b):
    assert same_disparities(a.disparity, b.disparity), mismatch_report(a.disparity, b.disparity)
    # Confidence 1 - best / second of every accepted pixel, 0 elsewhere
    # (stereo_matcher.cpp:517-520): float ops in the reference's order, exact.
    assert np.array_equal(a.confidence, b.confidence), mismatch_report(a.confidence, b.confidence)
    assert a.cells == b.cells
    assert a.levels == b.levels
    assert a.num_disparities == b.num_disparities


@pytest.mark.parametrize("shape,nd", [("1,8", 16), ("2,8", 32), ("2,16", 48), ("4,8", 64), ("4,12", 96),
                                      ("4,16", 128), ("8,8", 112), ("8,12", 192), ("8,16", 208), ("16,8", 256),
                                      ("16,12", 384), ("16,16", 512), ("32,8", 512), ("32,12", 768)])
@pytest.mark.parametrize("p2", [120, 8000])
def test_volume_chain_shapes(gpu_matcher, oracle, monkeypatch, shape, nd, p2):
    """Every compiled chain-pass shape (lanes per chain, label pairs per lane)
    against the textbook volume, with byte terms (P2 <= 255, intensity-adapted
    penalties) and with u16 sums (P2 = 8000: sums that wrap)."""
    monkeypatch.setenv("R3DGPU_PATH_SHAPE", shape)
    tex = Texture(19)
    left, right, _ = render_pair(tex, 70, 37, lambda x, y: 7.0 + 0.2 * x)
    o = StereoOptions(p1=20, p2=p2, p2_adapt=0 if p2 > 255 else 6, invalid_cost=40)
    assert np.array_equal(gpu_matcher.sgm_cost_volume(left, right, -1, nd, o),
                          oracle.sgm_cost_volume(left, right, -1, nd, o))


@pytest.mark.parametrize("terms", ["0", "1"])
def test_ranged_term_modes(gpu_matcher, oracle, monkeypatch, terms):
    """Per-pixel ranges through the chain passes with u16 sums and with byte
    terms (R3DGPU_RANGED_TERMS): a volume and a hierarchical match."""
    monkeypatch.setenv("R3DGPU_RANGED_TERMS", terms)
    tex = Texture(29)
    w, h, nd = 67, 41, 112
    left, right, _ = render_pair(tex, w, h, lambda x, y: 25.0 + 0.4 * x - 0.2 * y)
    r = Rng(37)
    num = np.array([[16 * r.uniform_int(1, 5) for _ in range(w)] for _ in range(h)], np.uint16)
    lo = np.array([[r.uniform_int(0, nd - int(n)) for n in row] for row in num], np.uint16)
    o = StereoOptions(p2=140, p2_adapt=5)
    assert np.array_equal(gpu_matcher.sgm_cost_volume(left, right, 1, nd, o, LabelRanges(lo, num)),
                          oracle.sgm_cost_volume(left, right, 1, nd, o, (lo, num)))
    left, right, _ = render_pair(tex, 240, 128, lambda x, y: np.where(x < 100, 9.0, 21.0))
    o = StereoOptions(levels=2, tile_size=96, tile_margin=8, tile_blend=8, range_radius=1)
    _assert_same_map(gpu_matcher.match_stereo(left, right, None, None, 0, 48, o),
                     oracle.match_stereo(left, right, None, None, 0, 48, o))


def test_census(gpu_matcher, oracle):
    for w in (1, 5, 16, 31, 64, 77, 640):
        img = random_image(w, 13, w)
        if w % 2 == 0:
            img = (img >> 13).astype(np.uint16)  # 8 levels: many ties
        assert np.array_equal(gpu_matcher.census_transform(img), oracle.census_transform(img))


def test_pyramid(gpu_matcher, oracle):
    for w, h in ((77, 41), (640, 480), (1, 1), (3, 2)):
        img = random_image(w, h, w + h)
        assert np.array_equal(gpu_matcher.pyramid_down(img), oracle.pyramid_down(img))


@pytest.mark.parametrize("p2_adapt", [0, 12])
@pytest.mark.parametrize("dmin,nd", [(-3, 16), (2, 48)])
def test_volume_equals_textbook(gpu_matcher, oracle, p2_adapt, dmin, nd):
    # tests/test_stereo.cpp:87-117
    tex = Texture(3)
    left, right, _ = render_pair(tex, 41, 23, lambda x, y: 5.0 + 0.1 * x)
    noise = random_image(41, 23, 9)
    right = right ^ (noise & 0x0F00)
    o = StereoOptions(p2_adapt=p2_adapt, p2=120)
    assert np.array_equal(gpu_matcher.sgm_cost_volume(left, right, dmin, nd, o),
                          oracle.sgm_cost_volume(left, right, dmin, nd, o))


def test_volume_with_ranges(gpu_matcher, oracle):
    # tests/test_stereo.cpp:119-151
    tex = Texture(13)
    w, h, nd = 37, 19, 96
    left, right, _ = render_pair(tex, w, h, lambda x, y: 20.0 + 0.5 * x - 0.3 * y)
    r = Rng(31)
    num = np.zeros((h, w), np.uint16)
    lo = np.zeros((h, w), np.uint16)
    for y in range(h):
        for x in range(w):
            n = 16 * r.uniform_int(1, 3)
            num[y, x] = n
            lo[y, x] = r.uniform_int(0, nd - n)
    o = StereoOptions(p2=150, p2_adapt=8)
    got = gpu_matcher.sgm_cost_volume(left, right, -2, nd, o, LabelRanges(lo, num))
    assert np.array_equal(got, oracle.sgm_cost_volume(left, right, -2, nd, o, (lo, num)))
    full = LabelRanges(np.zeros((h, w), np.uint16), np.full((h, w), nd, np.uint16))
    assert np.array_equal(gpu_matcher.sgm_cost_volume(left, right, -2, nd, o, full),
                          gpu_matcher.sgm_cost_volume(left, right, -2, nd, o))


def test_volume_large_labels(gpu_matcher, oracle):
    # Several 64-label chunks per pixel and sums that wrap modulo 2^16.
    tex = Texture(17)
    left, right, _ = render_pair(tex, 48, 20, lambda x, y: 30.0 + 0.2 * x)
    o = StereoOptions(p1=300, p2=8000, p2_adapt=0, invalid_cost=255)
    for nd in (208, 400):
        assert np.array_equal(gpu_matcher.sgm_cost_volume(left, right, -5, nd, o),
                              oracle.sgm_cost_volume(left, right, -5, nd, o))


@pytest.mark.parametrize("method", [SubpixelMethod.parabola, SubpixelMethod.equiangular])
def test_slanted_plane(gpu_matcher, oracle, method):
    tex = Texture(11)
    left, right, _ = render_pair(tex, 200, 120, lambda x, y: 12.3 + 0.04 * x + 0.02 * y)
    o = StereoOptions(subpixel=method)
    _assert_same_map(gpu_matcher.match_stereo(left, right, None, None, 0, 32, o),
                     oracle.match_stereo(left, right, None, None, 0, 32, o))


@pytest.mark.parametrize("opts", [
    StereoOptions(tile_size=48, tile_margin=8, tile_blend=8),
    StereoOptions(tile_size=48, tile_margin=8, tile_blend=8, lr_full_match=False),
    StereoOptions(tile_size=1024),
    StereoOptions(tile_size=48, tile_margin=8, tile_blend=0, uniqueness=0.15, subpixel=SubpixelMethod.none),
    StereoOptions(lr_max_diff=-1, speckle_size=0, median=False, levels=1),
])
def test_tiles_and_options(gpu_matcher, oracle, opts):
    tex = Texture(5)
    left, right, _ = render_pair(tex, 150, 90, lambda x, y: np.where(x < 70, 6.0, 14.5))
    _assert_same_map(gpu_matcher.match_stereo(left, right, None, None, 0, 32, opts),
                     oracle.match_stereo(left, right, None, None, 0, 32, opts))


@pytest.mark.parametrize("levels", [0, 1])
def test_masks(gpu_matcher, oracle, levels):
    tex = Texture(8)
    left, right, _ = render_pair(tex, 120, 60, lambda x, y: 10.0 + 0 * x)
    lm = np.full((60, 120), 255, np.uint8)
    rm = np.full((60, 120), 255, np.uint8)
    lm[:, 100:] = 0
    rm[:, :40] = 0
    lm[7, :] = 0  # a fully masked row
    o = StereoOptions(levels=levels)
    _assert_same_map(gpu_matcher.match_stereo(left, right, lm, rm, 0, 32, o),
                     oracle.match_stereo(left, right, lm, rm, 0, 32, o))


@pytest.mark.parametrize("full", [False, True])
def test_masked_wedge_lr(gpu_matcher, oracle, full):
    tex = Texture(21)
    left, right, _ = render_pair(tex, 160, 60, lambda x, y: 10.0 + 0 * x)
    r = Rng(4)
    nl = np.array([r.normal(0.0, 3000.0) for _ in range(2 * 160 * 60)])
    left = to_u16(left + nl[0::2].reshape(60, 160))
    right = to_u16(right + nl[1::2].reshape(60, 160))
    y, x = np.mgrid[0:60, 0:160]
    lmask = np.where(x < 70 + 2 * y, 255, 0).astype(np.uint8)
    o = StereoOptions(lr_full_match=full, tile_size=64)
    _assert_same_map(gpu_matcher.match_stereo(left, right, lmask, None, 0, 256, o),
                     oracle.match_stereo(left, right, lmask, None, 0, 256, o))


@pytest.mark.parametrize("levels", [0, 1])
@pytest.mark.parametrize("full", [False, True])
def test_different_widths_negative_disparities(gpu_matcher, oracle, levels, full):
    tex = Texture(23)
    wl, wr, h, d = 150, 190, 60, -7.0
    yy, xl = np.mgrid[0:h, 0:wl].astype(np.float64)
    yr, xr = np.mgrid[0:h, 0:wr].astype(np.float64)
    left = to_u16(tex(xl, yy))
    right = to_u16(tex(xr + d, yr))
    o = StereoOptions(lr_full_match=full, levels=levels)
    _assert_same_map(gpu_matcher.match_stereo(left, right, None, None, -20, 32, o),
                     oracle.match_stereo(left, right, None, None, -20, 32, o))


def test_ranges_from_coarse(gpu_matcher, oracle):
    wc, hc = 40, 20
    coarse = np.where(np.arange(wc)[None, :] < wc // 2, 10.0, 30.0).astype(np.float32).repeat(hc, 0)
    coarse[5, 5] = np.inf
    coarse[:, 30:] = np.inf
    w, h, dmin, nd = 2 * wc, 2 * hc, 4, 96
    valid = np.full((h, w), 255, np.uint8)
    valid[1, 1] = 0
    o = StereoOptions(range_radius=1, range_margin=3, range_fill=4)
    for fv, pv, pw, sign, mir in ((valid, None, 1000, 1, False), (valid, None, w, -1, False), (None, valid, w, 1, True)):
        a = gpu_matcher.ranges_from_coarse(coarse, w, h, fv, pv, pw, sign, dmin, nd, o, mir)
        b = oracle.ranges_from_coarse(coarse, w, h, fv, pv, pw, sign, dmin, nd, o, mir)
        assert np.array_equal(a.lo, b[0]) and np.array_equal(a.num, b[1])


def test_speckle_and_median(gpu_matcher, oracle):
    rng = np.random.default_rng(3)
    d = np.round(rng.normal(20, 3, (90, 130))).astype(np.float32)
    d[rng.random(d.shape) < 0.1] = np.inf
    for size in (2, 6, 40):
        assert same_disparities(gpu_matcher.remove_speckles(d.copy(), size, 1.0), oracle.remove_speckles(d, size, 1.0))
    assert same_disparities(gpu_matcher.median_filter_3x3(d), oracle.median_filter_3x3(d))


def _synthetic_pair(w, h, nd, seed):
    """Blurred uniform noise, piecewise-planar disparity, bilinear warp, noise."""
    rng = np.random.default_rng(seed)
    base = rng.uniform(0, 255, (h, w + nd + 8))
    k = np.exp(-0.5 * (np.arange(-5, 6) / 1.5) ** 2)
    k /= k.sum()
    base = np.apply_along_axis(lambda r: np.convolve(r, k, mode="same"), 1, base)
    base = np.apply_along_axis(lambda c: np.convolve(c, k, mode="same"), 0, base)
    base = (base - base.min()) / (base.max() - base.min()) * 255.0
    ys, xs = np.mgrid[0:h, 0:w].astype(np.float64)
    seeds = rng.uniform(0, 1, (8, 2)) * [w, h]
    planes = np.stack([rng.uniform(-0.02, 0.02, 8), rng.uniform(-0.02, 0.02, 8), rng.uniform(5, nd - 8, 8)], 1)
    lab = np.argmin((xs[..., None] - seeds[:, 0]) ** 2 + (ys[..., None] - seeds[:, 1]) ** 2, axis=-1)
    disp = np.clip(planes[lab, 0] * xs + planes[lab, 1] * ys + planes[lab, 2], 5, nd - 8)
    left = base[:, :w]
    xsrc = xs + disp
    x0 = np.floor(xsrc).astype(int)
    f = xsrc - x0
    right = base[np.arange(h)[:, None], x0] * (1 - f) + base[np.arange(h)[:, None], x0 + 1] * f
    right = right + rng.normal(0, 2, right.shape)
    L = np.clip(np.round(left), 0, 255).astype(np.uint8)
    R = np.clip(np.round(right), 0, 255).astype(np.uint8)
    return L.astype(np.uint16) * 257, R.astype(np.uint16) * 257


def test_single_level_640x480_128(gpu_matcher, oracle):
    """The reference's CPU-runnable configuration: 640x480, labels 0..127, one level."""
    left, right = _synthetic_pair(640, 480, 128, 1)
    o = StereoOptions(levels=0)
    _assert_same_map(gpu_matcher.match_stereo(left, right, None, None, 0, 128, o),
                     oracle.match_stereo(left, right, None, None, 0, 128, o))


def test_hierarchical_pair(gpu_matcher, oracle):
    """Hierarchy with per-pixel ranges (+-8 around the upsampled coarse disparity)."""
    left, right = _synthetic_pair(768, 512, 256, 2)
    o = StereoOptions(levels=3, range_radius=0, range_margin=8)
    _assert_same_map(gpu_matcher.match_stereo(left, right, None, None, 0, 256, o),
                     oracle.match_stereo(left, right, None, None, 0, 256, o))
    o = StereoOptions(levels=-1)
    _assert_same_map(gpu_matcher.match_stereo(left, right, None, None, 0, 256, o),
                     oracle.match_stereo(left, right, None, None, 0, 256, o))


def _smooth_ranges(w, h, nd, seed, wide_frac=0.05):
    """Ranges shaped like a hierarchical level's: lo drifting slowly, a few
    jumps, num mostly 16 or 32, some wide pixels."""
    rng = np.random.default_rng(seed)
    base = np.cumsum(rng.integers(-1, 2, (h, w)) * (rng.random((h, w)) < 0.3), axis=1)
    base = base + np.cumsum(rng.integers(-2, 3, (h, 1)), axis=0)
    base = base + np.where(rng.random((h, w)) < 0.03, rng.integers(-40, 40, (h, w)), 0)
    num = np.where(rng.random((h, w)) < 0.2, 16, 32)
    num = np.where(rng.random((h, w)) < wide_frac, rng.choice([48, 64, 96, nd], (h, w)), num)
    num = np.minimum(num, nd)
    lo = np.clip(nd // 3 + base, 0, nd - num)
    return lo.astype(np.uint16), num.astype(np.uint16)


@pytest.mark.parametrize("kernel,shape,rows", [("ranged", "4,4", 32), ("ranged", "8,4", 16), ("ranged", "4,4", 8),
                                               ("ranged", "8,4", 64), ("ranged", "8,8", 12), ("ranged", "16,12", 6),
                                               ("ranged", "32,8", 5), ("ranged", "", 0), ("general", "", 0),
                                               ("path", "", 0)])
def test_ranged_volume_kernels(gpu_matcher, oracle, monkeypatch, kernel, shape, rows):
    """Per-pixel ranges through the one-CTA-per-tile ranged kernel (both
    shapes, several band heights: aligned, shifted and bounds-checked
    predecessor reads, wide pixels, seams), the general kernel and the chain
    passes (the default), against the textbook volume."""
    monkeypatch.setenv("R3DGPU_RANGED_KERNEL", kernel)
    if shape:
        monkeypatch.setenv("R3DGPU_RANGED_SHAPE", shape)
        monkeypatch.setenv("R3DGPU_RANGED_ROWS", str(rows))
    left, right = _synthetic_pair(211, 157, 256, 7)
    lo, num = _smooth_ranges(211, 157, 256, 3)
    for o in (StereoOptions(), StereoOptions(p1=300, p2=8000, p2_adapt=0, invalid_cost=255)):
        assert np.array_equal(gpu_matcher.sgm_cost_volume(left, right, -4, 256, o, LabelRanges(lo, num)),
                              oracle.sgm_cost_volume(left, right, -4, 256, o, (lo, num)))


@pytest.mark.parametrize("lr_full", [True, False])
def test_ranged_kernel_hierarchy_shapes(gpu_matcher, oracle, monkeypatch, lr_full):
    """The hierarchy with the wide-range shape and short bands."""
    monkeypatch.setenv("R3DGPU_RANGED_SHAPE", "8,4")
    monkeypatch.setenv("R3DGPU_RANGED_ROWS", "12")
    left, right = _synthetic_pair(500, 380, 192, 4)
    o = StereoOptions(levels=2, range_radius=0, range_margin=8, lr_full_match=lr_full, tile_size=256)
    _assert_same_map(gpu_matcher.match_stereo(left, right, None, None, 0, 192, o),
                     oracle.match_stereo(left, right, None, None, 0, 192, o))


def test_batch_equals_single(gpu_matcher):
    """Pairs of uneven size, range and depth matched together give the same
    maps as matched one by one."""
    pairs = []
    for i, (w, h, nd, lv) in enumerate(((320, 240, 64, 0), (256, 200, 128, 2), (400, 300, 96, -1), (96, 64, 32, 0))):
        left, right = _synthetic_pair(w, h, nd, 10 + i)
        pairs.append(dict(left=left, right=right, disparity_min=0, num_disparities=nd, options=StereoOptions(levels=lv)))
    batch = gpu_matcher.match_stereo_batch(pairs)
    for p, b in zip(pairs, batch):
        s = gpu_matcher.match_stereo(p["left"], p["right"], None, None, 0, p["num_disparities"], p["options"])
        _assert_same_map(b, s)
        assert np.array_equal(b.confidence, s.confidence)


def test_errors(gpu_matcher):
    from regard3d_mvs_b200 import StereoError

    img = random_image(32, 16, 1)
    with pytest.raises(StereoError):
        gpu_matcher.match_stereo(img, img, None, None, 0, 16, StereoOptions(p1=300, p2=200))
    with pytest.raises(StereoError):
        gpu_matcher.match_stereo(img, img, None, None, 0, 0)
    with pytest.raises(StereoError):
        gpu_matcher.match_stereo(img, img[:8], None, None, 0, 16)
    with pytest.raises(StereoError):
        gpu_matcher.match_stereo(img, img, np.zeros((3, 3), np.uint8), None, 0, 16)
    # The context stays usable after errors.
    r = gpu_matcher.match_stereo(img, img, None, None, 0, 16, StereoOptions(levels=0))
    assert r.disparity.shape == (16, 32)


def _bench_pair(spec):
    """A pair of the benchmark lists from the seeded generator (compiled into
    the oracle library from the same source as the CUDA library's), 8-bit
    lifted x257 as the reference's image reader does (io/image_io.hpp:25)."""
    from oracle import oracle

    L, R = oracle.synth_pair(spec["w"], spec["h"], spec["nd"], spec["seed"], spec["textureless"], spec["occluded"])
    return L.astype(np.uint16) * np.uint16(257), R.astype(np.uint16) * np.uint16(257)


def _bench_options(spec):
    return StereoOptions(levels=spec["levels"], range_radius=spec["radius"], range_margin=spec["margin"])


def test_pair_3072x2048_256_four_levels(gpu_matcher, oracle):
    """3072x2048, labels 0..255, 15 % textureless patches, 10 % occluded right
    pixels, 4-level hierarchy with +-8 labels around the upsampled coarser
    disparity (range_radius 0, range_margin 8)."""
    import bench

    spec = bench.workload_pairs("pair3072", 1, 0)[0]
    left, right = _bench_pair(spec)
    o = _bench_options(spec)
    oracle.set_threads(oracle.max_threads())
    got = gpu_matcher.match_stereo(left, right, None, None, 0, spec["nd"], o)
    ref = oracle.match_stereo(left, right, None, None, 0, spec["nd"], o)
    assert got.levels == 3
    _assert_same_map(got, ref)


# Pairs of the 64-pair benchmark batch (bench.py's default seed): the widest
# pair (5775 px, hierarchical, 192 labels), the widest single-level pair
# (5365x4024, 192 labels), a 3194x2396 384-label single-level pair and a
# 5048 px 384-label hierarchical pair.
BATCH64_SEED = 2024
BATCH64_SAMPLE = (63, 50, 48, 15)


def test_batch64_pairs_batched(gpu_matcher, oracle):
    """Pairs of the 64-pair batch workload (up to 6048 wide, 384 labels)
    matched together in one batch call, each against the
    oracle matching it alone."""
    import bench

    specs = bench.workload_pairs("batch64", 64, BATCH64_SEED)
    chosen = [specs[i] for i in BATCH64_SAMPLE]
    assert max(s["w"] for s in chosen) == max(s["w"] for s in specs)
    assert any(s["nd"] == 384 and s["levels"] == 0 for s in chosen)
    assert any(s["nd"] == 384 and s["levels"] == 3 for s in chosen)
    pairs = []
    for s in chosen:
        left, right = _bench_pair(s)
        pairs.append(dict(left=left, right=right, disparity_min=0, num_disparities=s["nd"], options=_bench_options(s)))
    batch = gpu_matcher.match_stereo_batch(pairs)
    oracle.set_threads(oracle.max_threads())
    for p, got in zip(pairs, batch):
        ref = oracle.match_stereo(p["left"], p["right"], None, None, 0, p["num_disparities"], p["options"])
        _assert_same_map(got, ref)


def _device_batch(gpu_matcher, specs):
    """The r3dgpu_pair array of `specs` over device-resident torch buffers
    (stable pointers from call to call), and a reader of the maps."""
    import ctypes

    import torch

    from regard3d_mvs_b200.types import CDisparityMap, CPair, CViewU8, CViewU16, to_c_options

    keep, pairs = [], (CPair * len(specs))()
    for i, (left, right, nd, opts) in enumerate(specs):
        h, w = left.shape
        dl = torch.from_numpy(left.view(np.int16)).cuda()
        dr = torch.from_numpy(right.view(np.int16)).cuda()
        dd = torch.empty((h, w), dtype=torch.float32, device="cuda")
        dc = torch.empty_like(dd)
        keep += [dl, dr, dd, dc]
        p = pairs[i]
        p.left, p.right = CViewU16(dl.data_ptr(), w, h, w), CViewU16(dr.data_ptr(), w, h, w)
        p.left_valid, p.right_valid = CViewU8(), CViewU8()
        p.disparity_min, p.num_disparities = 0, nd
        p.options = to_c_options(opts)
        p.out = CDisparityMap(dd.data_ptr(), dc.data_ptr(), w, 0, 0, 0, 0, 0)

    def run():
        st = gpu_matcher.lib.r3dgpu_match_stereo_batch(pairs, len(specs), ctypes.c_void_p(0))
        assert st == 0, gpu_matcher.lib.r3dgpu_last_error().decode()
        torch.cuda.synchronize()
        return [(keep[4 * i + 2].cpu().numpy().copy(), keep[4 * i + 3].cpu().numpy().copy(), int(pairs[i].out.cells))
                for i in range(len(specs))]

    return run, keep


def test_single_level_track_graph_replays(gpu_matcher, monkeypatch):
    """A batch mixing single-level and hierarchical pairs: its single-level
    track is captured as a CUDA graph on the first call and replayed on the
    next ones; every call's maps and cell counts equal those of the track
    enqueued directly (R3DGPU_GRAPH=0)."""
    specs = []
    for i, (w, h, nd, lv) in enumerate(((320, 240, 64, 0), (256, 200, 128, 2), (400, 300, 96, 0), (96, 64, 32, 0))):
        left, right = _synthetic_pair(w, h, nd, 30 + i)
        specs.append((left, right, nd, StereoOptions(levels=lv)))
    run, _ = _device_batch(gpu_matcher, specs)
    monkeypatch.setenv("R3DGPU_GRAPH", "0")
    want = run()
    monkeypatch.delenv("R3DGPU_GRAPH")
    before = gpu_matcher.launch_count()
    got = [run() for _ in range(3)]  # capture, then two replays
    assert gpu_matcher.launch_count() > before
    for g in got:
        for (d0, c0, n0), (d1, c1, n1) in zip(want, g):
            assert np.array_equal(d0.view(np.uint32), d1.view(np.uint32))
            assert np.array_equal(c0, c1) and n0 == n1
