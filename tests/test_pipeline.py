"""A view's depth map on the device (r3dgpu_compute_depth_map): the loop of
the reference's compute_depth_map (src/r3d/mvs/multi_stereo.cpp:243-304)
from the rectified pairs on. Every stage is bit-exact against the oracle, so
the composed result equals the oracle's chain (rectify_image of both images
of each pair, match_stereo, combine_pairs) bit for bit."""

from __future__ import annotations

import numpy as np
import pytest

from regard3d_mvs_b200.multi_view import arc_scene, pipeline_scene
from regard3d_mvs_b200.types import MultiStereoOptions, StereoOptions


def oracle_chain(oracle, grid, base, pairs, stereo, multi):
    """rectify_image (base and partner), match_stereo, combine_pairs on the CPU."""
    K = grid["K"]
    cam = {"model": 0, "width": grid["width"], "height": grid["height"], "fx": K[0, 0], "fy": K[1, 1],
           "cx": K[0, 2], "cy": K[1, 2]}
    matched = []
    cells = 0
    for p in pairs:
        left, lmask = oracle.rectify_image(base, cam, grid["R"] @ p["R_rect"].T, p["left"])
        right, rmask = oracle.rectify_image(p["image"], cam, p["R_partner"] @ p["R_rect"].T, p["right"])
        m = oracle.match_stereo(left, right, lmask, rmask, p["disparity_min"], p["num_disparities"], stereo)
        cells += m.cells
        matched.append(dict(p, disparity=m.disparity, confidence=m.confidence))
    return oracle.combine_pairs(grid, matched, multi), cells


def check(matcher, oracle, w, h, f, partners, stereo, multi=None):
    rig, base, pairs = pipeline_scene(w, h, f, partners, seed=4)
    return check_view(matcher, oracle, rig.grid(), base, pairs, stereo, multi)


def check_view(matcher, oracle, grid, base, pairs, stereo, multi=None):
    got, cells = matcher.compute_depth_map(base, grid, pairs, stereo, multi)
    want, want_cells = oracle_chain(oracle, grid, base, pairs, stereo, multi or MultiStereoOptions())
    assert cells == want_cells
    np.testing.assert_array_equal(got.depth.view(np.uint32), want.depth.view(np.uint32))
    np.testing.assert_array_equal(got.confidence.view(np.uint32), want.confidence.view(np.uint32))
    np.testing.assert_array_equal(got.pair_mask, want.pair_mask)
    return got


def test_emulator_equals_oracle_chain(simt_matcher, oracle):
    got = check(simt_matcher, oracle, 96, 72, 90.0, ((0.6, 0.0, 0.0), (-0.5, 0.3, 0.1)),
                StereoOptions(levels=0, tile_size=64))
    assert (got.depth > 0).mean() > 0.2


def test_emulator_arc_scene_view(simt_matcher, oracle):
    """A view of the multi-view arc scene (textured planes, partners on both
    sides, rectified pairs mirrored for partners on the left)."""
    scene = arc_scene(3, 96, 72, planes=6, partners=2, seed=3, arc_deg=12.0)
    v = scene["views"][1]
    got = check_view(simt_matcher, oracle, v["camera"], v["image"], v["pairs"], StereoOptions(levels=0, tile_size=64))
    assert (got.depth > 0).mean() > 0.2


def test_rejects_too_many_pairs(simt_matcher):
    rig, base, pairs = pipeline_scene(32, 24, 30.0, ((0.6, 0.0, 0.0),), seed=1)
    with pytest.raises(Exception, match="at most 16 pairs"):
        simt_matcher.compute_depth_map(base, rig.grid(), pairs * 17)


@pytest.mark.gpu
def test_gpu_equals_oracle_chain(gpu_matcher, oracle):
    got = check(gpu_matcher, oracle, 640, 480, 600.0, ((0.6, 0.0, 0.0), (-0.5, 0.3, 0.1), (0.2, -0.55, 0.0),
                                                       (-0.3, -0.4, 0.2)), StereoOptions())
    assert (got.depth > 0).mean() > 0.3


@pytest.mark.gpu
def test_gpu_arc_scene_view(gpu_matcher, oracle):
    """A central view of an arc scene of textured planes (the depth-stage
    scene's construction at 640x480): the device chain equals the oracle's."""
    scene = arc_scene(6, 640, 480, planes=20, partners=4, seed=5, arc_deg=20.0)
    v = scene["views"][2]
    got = check_view(gpu_matcher, oracle, v["camera"], v["image"], v["pairs"], StereoOptions())
    assert (got.depth > 0).mean() > 0.3
