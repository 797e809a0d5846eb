"""Patch-based depth refinement (src/r3d/mvs/refinement.cpp).

The double-precision oracle is pinned by the reference's refinement test
(tests/test_mvs.cpp:431-508) restated; the refinement images are bit-exact
between the CUDA kernels (on the SIMT emulator) and the oracle; the refined
depths of the kernel agree with the oracle's to rounding (the kernel sums the
window terms in a butterfly instead of a sequential loop): the same pixels
are refined and their depths differ by at most 2e-6 relative. The float
path (fp32: Gauss-Newton terms in float, the objective in double) stays
within 1e-5 relative of the double oracle.
"""

from __future__ import annotations

import numpy as np
import pytest

from mvs_scenes import refinement_scene, relative_depth_rms
from regard3d_mvs_b200.depth_maps import RefinementOptions

BORDER = 12


@pytest.fixture(scope="module")
def scene(oracle):
    return refinement_scene(oracle.make_refinement_image)


def copy_map(m):
    return {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in m.items()}


def test_oracle_defaults_take_only_clear_gains(oracle, scene):
    """test_mvs.cpp:469-474."""
    m, truth, base, views, _ = scene
    m = copy_map(m)
    before = relative_depth_rms(m, truth, BORDER)
    st = oracle.refine_depth_map(m, base, views)
    assert relative_depth_rms(m, truth, BORDER) < before / 3.0
    assert st["refined"] > st["input"] / 2


def test_oracle_matching_images(oracle, scene):
    """test_mvs.cpp:475-487."""
    m, truth, base, views, _ = scene
    m = copy_map(m)
    before = relative_depth_rms(m, truth, BORDER)
    st = oracle.refine_depth_map(m, base, views, RefinementOptions(min_gain=0.0))
    after = relative_depth_rms(m, truth, BORDER)
    assert st["input"] == m["depth"].size
    assert st["refined"] > st["input"] * 8 // 10
    assert after < before / 5.0
    assert m["confidence"][60, 80] > 0.9


def test_oracle_unrelated_images(oracle, scene):
    """test_mvs.cpp:488-507: unconfirmed depths are removed, or kept."""
    m, truth, base, _, wrong = scene
    before = relative_depth_rms(m, truth, BORDER)
    dropped = copy_map(m)
    st = oracle.refine_depth_map(dropped, base, wrong, RefinementOptions(min_ncc=0.5))
    assert st["refined"] < st["input"] / 20
    assert st["unconfirmed"] > st["input"] / 2
    assert (dropped["depth"] > 0).sum() == st["input"] - st["unconfirmed"]
    kept_map = copy_map(m)
    kept = oracle.refine_depth_map(kept_map, base, wrong, RefinementOptions(min_ncc=0.5, drop_unconfirmed=False))
    assert kept["unconfirmed"] == 0
    assert relative_depth_rms(kept_map, truth, BORDER) < before * 1.2


@pytest.mark.parametrize("sigma", [0.0, 1.3])
def test_refinement_image_equals_oracle(simt_matcher, oracle, sigma):
    rng = np.random.default_rng(4)
    gray = (rng.random((37, 53)) * 255).astype(np.float32)
    np.testing.assert_array_equal(simt_matcher.make_refinement_image(gray, sigma).view(np.uint32),
                                  oracle.make_refinement_image(gray, sigma).view(np.uint32))


def sparse(m, seed, clusters=16):
    """Keeps 3 x 3 clusters of valid depth around random pixels (so that the
    slopes see neighbours), the rest invalid: a few hundred warps for the
    emulator."""
    rng = np.random.default_rng(seed)
    out = copy_map(m)
    keep = np.zeros(m["depth"].shape, bool)
    h, w = keep.shape
    for _ in range(clusters):
        y, x = rng.integers(6, h - 6), rng.integers(6, w - 6)
        keep[y - 1:y + 2, x - 1:x + 2] = True
    out["depth"] = np.where(keep, m["depth"], 0).astype(np.float32)
    return out


def compare(a, b, ia, ib, max_rel=2e-6):
    """Same statistics and decisions; refined depths within max_rel."""
    assert ia == ib
    np.testing.assert_array_equal(a["depth"] > 0, b["depth"] > 0)
    valid = b["depth"] > 0
    rel = np.abs(a["depth"][valid].astype(np.float64) - b["depth"][valid]) / b["depth"][valid]
    assert rel.max() <= max_rel, rel.max()
    np.testing.assert_allclose(a["confidence"], b["confidence"], atol=1e-5)
    return rel


@pytest.mark.parametrize("opts", [RefinementOptions(), RefinementOptions(min_gain=0.0, radius=3, step=1),
                                  RefinementOptions(min_ncc=0.5, iterations=3, max_views=2)])
def test_kernel_equals_oracle(simt_matcher, oracle, scene, opts):
    m, _, base, views, _ = scene
    a, b = sparse(m, 1), sparse(m, 1)
    ia = simt_matcher.refine_depth_map(a, base, views, opts)
    ib = oracle.refine_depth_map(b, base, views, opts)
    compare(a, b, ia, ib)
    assert ib["refined"] > 0


def test_kernel_unrelated_views_equal_oracle(simt_matcher, oracle, scene):
    m, _, base, _, wrong = scene
    a, b = sparse(m, 2), sparse(m, 2)
    opts = RefinementOptions(min_ncc=0.5)
    compare(a, b, simt_matcher.refine_depth_map(a, base, wrong, opts), oracle.refine_depth_map(b, base, wrong, opts))


def fp32_error(a, b):
    """Relative depth error of the float path against the double oracle."""
    valid = b["depth"] > 0
    return np.abs(a["depth"][valid].astype(np.float64) - b["depth"][valid]) / b["depth"][valid]


def test_kernel_fp32_close_to_oracle(simt_matcher, oracle, scene):
    """Gauss-Newton terms in float, objective in double: the same decisions,
    depths within 1e-5 relative of the double oracle (measured: one float ulp)."""
    m, _, base, views, _ = scene
    a, b = sparse(m, 3, 40), sparse(m, 3, 40)
    ia = simt_matcher.refine_depth_map(a, base, views, RefinementOptions(min_gain=0.0, radius=3, step=1, fp32=True))
    ib = oracle.refine_depth_map(b, base, views, RefinementOptions(min_gain=0.0, radius=3, step=1))
    assert ia == ib
    np.testing.assert_array_equal(a["depth"] > 0, b["depth"] > 0)
    rel = fp32_error(a, b)
    assert np.percentile(rel, 99) <= 1e-6 and rel.max() <= 1e-5, (np.percentile(rel, 99), rel.max())


def test_kernel_rejects_bad_options(simt_matcher, scene):
    m, _, base, views, _ = scene
    with pytest.raises(Exception, match="invalid window"):
        simt_matcher.refine_depth_map(copy_map(m), base, views, RefinementOptions(radius=0))
    with pytest.raises(Exception, match="225"):
        simt_matcher.refine_depth_map(copy_map(m), base, views, RefinementOptions(radius=8, step=1))


def test_depth_stage_in_one_call_equals_the_steps(simt_matcher):
    """r3dgpu_depth_stage_host equals refine_depth_map per view followed by
    filter_depth_maps (and leaves the inputs' images untouched)."""
    from regard3d_mvs_b200.depth_maps import ConsistencyOptions
    from regard3d_mvs_b200.multi_view import depth_stage_scene

    scene = depth_stage_scene(3, 40, 30, partners=2)
    views, nbs = scene["views"], scene["partners"]
    rng = np.random.default_rng(2)
    images, maps = [], []
    for i, v in enumerate(views):
        images.append({"camera": v["camera"], "data": simt_matcher.make_refinement_image(v["gray"])})
        keep = rng.random(v["depth"].shape) < 0.04
        keep[12:18, 14:26] = True
        maps.append({"camera": v["camera"], "depth": np.where(keep, v["depth"], 0).astype(np.float32),
                     "confidence": np.zeros(v["depth"].shape, np.float32),
                     "pair_mask": np.ones(v["depth"].shape, np.uint16), "color": v["color"], "view": i,
                     "partners": nbs[i]})
    opts = RefinementOptions(radius=2, step=2)
    a = [copy_map(m) for m in maps]
    ra, ca = simt_matcher.depth_stage(a, images, nbs, opts, ConsistencyOptions())
    b = [copy_map(m) for m in maps]
    rb = {"input": 0, "refined": 0, "kept": 0, "unconfirmed": 0}
    for i, m in enumerate(b):
        st = simt_matcher.refine_depth_map(m, images[i], [images[j] for j in nbs[i]], opts)
        rb = {k: rb[k] + st[k] for k in rb}
    cb = simt_matcher.filter_depth_maps(b, nbs, ConsistencyOptions())
    assert ra == rb and ca == cb and rb["refined"] > 0
    for x, y in zip(a, b):
        assert np.array_equal(x["depth"], y["depth"]) and np.array_equal(x["support"], y["support"])
        assert np.array_equal(x["confidence"], y["confidence"])
