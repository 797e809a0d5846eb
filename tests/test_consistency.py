"""Geometric consistency of depth maps (src/r3d/mvs/consistency.cpp).

The oracle is pinned by the reference's own tests (tests/test_mvs.cpp:229-324
and :510-591), restated here; the CUDA kernels run on the SIMT emulator and
must equal the oracle bit for bit: depths, support counts and statistics.
"""

from __future__ import annotations

import numpy as np
import pytest

from mvs_scenes import MultiRig, camera, copy_maps, empty_map, plane_depth_map, slanted_plane, synthetic_scene
from regard3d_mvs_b200.depth_maps import ConsistencyOptions


def valid(m, x, y):
    return m["depth"][y, x] > 0


# ------------------------------------------------------------------ reference tests on the oracle
def rig_maps():
    rig = MultiRig()
    plane = slanted_plane(rig.base)
    cam1 = camera(rig.k, rig.partners[0]["rotation"], rig.partners[0]["center"])
    cam2 = camera(rig.k, rig.partners[1]["rotation"], rig.partners[1]["center"])
    maps = [plane_depth_map(rig.base, plane, 0, 1), plane_depth_map(cam1, plane, 1, 0),
            plane_depth_map(cam2, plane, 2, 0)]
    maps[0]["depth"][100:120, 150:170] *= np.float32(1.05)  # a block 5 % too far
    return maps


@pytest.fixture(params=["oracle", "emulator"])
def impl(request, oracle, simt_matcher):
    return oracle if request.param == "oracle" else simt_matcher


def test_independent_support(impl):
    """test_mvs.cpp:243-260."""
    maps = rig_maps()
    opt = ConsistencyOptions(edge_erosion=0, min_views=1, independent_support=True)
    st = impl.filter_depth_maps(maps, [[1, 2], [0, 2], [0, 1]], opt)
    assert st["input"] == st["rejected"] + st["output"]
    assert not np.any(maps[0]["depth"][100:120, 150:170] > 0)
    assert valid(maps[0], 60, 60)
    assert maps[0]["support"][60, 60] == 1  # from map 2 only


def test_mirrored_pairs_alone_are_not_enough(impl):
    """test_mvs.cpp:261-270."""
    maps = rig_maps()
    opt = ConsistencyOptions(edge_erosion=0, min_views=1, independent_support=True)
    impl.filter_depth_maps(maps, [[1], [0], []], opt)
    assert (maps[0]["depth"] > 0).sum() == 0 and (maps[1]["depth"] > 0).sum() == 0


def test_any_support(impl):
    """test_mvs.cpp:271-280."""
    maps = rig_maps()
    opt = ConsistencyOptions(edge_erosion=0, min_views=1, independent_support=False)
    impl.filter_depth_maps(maps, [[1], [0], []], opt)
    assert valid(maps[0], 60, 60) and maps[0]["support"][60, 60] == 1


def test_defaults_two_pairs_or_one_agreeing_view(impl):
    """test_mvs.cpp:281-294."""
    maps = rig_maps()
    maps[2]["partners"] = [0, 1]
    maps[2]["pair_mask"][60, 60] = 3
    impl.filter_depth_maps(maps, [[], [], []], ConsistencyOptions(edge_erosion=0))
    assert (maps[2]["depth"] > 0).sum() == 1
    assert valid(maps[2], 60, 60) and maps[2]["support"][60, 60] == 0


def test_erode_depth_edges_removes_both_sides(impl):
    """test_mvs.cpp:297-312."""
    m = empty_map(10, 5)
    m["depth"][:] = 2.0
    m["depth"][:, 5:] = 3.0
    assert impl.erode_depth_edges(m, 1, 0.05) == 10
    assert not valid(m, 4, 2) and not valid(m, 5, 2) and valid(m, 3, 2) and valid(m, 6, 2)
    assert impl.erode_depth_edges(m, 2, 0.05) == 0


def test_erode_depth_edges_optionally_erodes_hole_borders(impl):
    """test_mvs.cpp:314-324."""
    m = empty_map(9, 9)
    m["depth"][:] = 2.0
    m["depth"][4, 4] = 0.0
    assert impl.erode_depth_edges(m, 1, 0.05) == 0
    assert impl.erode_depth_edges(m, 1, 0.05, True) == 4
    assert not valid(m, 3, 4) and valid(m, 3, 3) and valid(m, 0, 0)


def test_remove_depth_speckles(impl):
    """test_mvs.cpp:510-529."""
    m = empty_map(20, 20)
    m["depth"][:] = 2.0
    m["depth"][2:5, 2:5] = 3.0
    m["depth"][10:14, 10:14] = 2.02
    assert impl.remove_depth_speckles(m, 10, 0.02) == 9
    assert not valid(m, 3, 3) and valid(m, 11, 11)
    assert (m["depth"] > 0).sum() == 400 - 9
    assert impl.remove_depth_speckles(m, 10, 0.02) == 0


def test_remove_weak_depths(impl):
    """test_mvs.cpp:531-563."""
    m = empty_map(40, 40)
    m["depth"][:] = 2.0
    y, x = np.mgrid[0:40, 0:40]
    g = np.where(x >= 20, 128, np.where(((x // 2) + (y // 2)) % 2 == 0, 0, 255)).astype(np.uint8)
    m["color"] = np.repeat(g[..., None], 3, axis=2)
    m["depth"][5:10, 30:35] = 5.0
    seg = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in m.items()}
    opt = ConsistencyOptions(weak_segment=0.05)
    assert impl.remove_weak_depths(seg, opt) == 25
    assert not valid(seg, 32, 7) and valid(seg, 32, 20)
    opt.weak_texture = 0.0
    assert impl.remove_weak_depths(m, opt) == 0
    opt.weak_texture = 4.0
    opt.reject_weak = True
    assert impl.remove_weak_depths(m, opt) == 17 * 40
    assert valid(m, 22, 20) and not valid(m, 23, 20)


def halo_map(valid_end, edge):
    m = empty_map(40, 40)
    x = np.arange(40)[None, :].repeat(40, 0)
    m["depth"] = np.where(x < valid_end, 2.0, 0.0).astype(np.float32)
    g = np.where(edge & (x < 20), 50, 200).astype(np.uint8)
    m["color"] = np.repeat(g[..., None], 3, axis=2)
    return m


def test_remove_depth_halos(impl):
    """test_mvs.cpp:565-591."""
    m = halo_map(26, True)
    assert impl.remove_depth_halos(m, 16, 25) == 6 * 40
    assert valid(m, 19, 20) and not valid(m, 20, 20)
    assert impl.remove_depth_halos(halo_map(26, True), 8, 25) == 0
    assert impl.remove_depth_halos(halo_map(26, True), 9, 25) == 6 * 40
    assert impl.remove_depth_halos(halo_map(20, True), 16, 25) == 0
    assert impl.remove_depth_halos(halo_map(26, False), 16, 25) == 0


# ------------------------------------------------------------------ kernels against the oracle
OPTION_SETS = [
    ConsistencyOptions(),
    ConsistencyOptions(min_views=1, independent_support=True, erode_holes=True, min_confidence=0.2),
    ConsistencyOptions(average_depths=False, weak_segment=0.01, speckle_size=40, halo_px=12, min_evidence=3),
    ConsistencyOptions(reject_weak=True, weak_texture=30.0, halo_px=0, max_reprojection_px=0.7,
                       max_relative_depth_error=0.004),
]


def assert_same_maps(a, b):
    for i, (x, y) in enumerate(zip(a, b)):
        np.testing.assert_array_equal(x["depth"].view(np.uint32), y["depth"].view(np.uint32), err_msg=f"map {i}")
        np.testing.assert_array_equal(x["support"], y["support"], err_msg=f"map {i}")


@pytest.mark.parametrize("k", range(len(OPTION_SETS)))
def test_filter_equals_oracle(simt_matcher, oracle, k):
    maps, nbs = synthetic_scene(4, 96, 72, seed=10 + k)
    a, b = copy_maps(maps), copy_maps(maps)
    sa = simt_matcher.filter_depth_maps(a, nbs, OPTION_SETS[k])
    sb = oracle.filter_depth_maps(b, nbs, OPTION_SETS[k])
    assert sa == sb
    assert_same_maps(a, b)
    assert sb["rejected"] > 0 and sb["output"] > 0


def test_single_steps_equal_oracle(simt_matcher, oracle):
    maps, nbs = synthetic_scene(3, 96, 72, seed=21)
    opt = ConsistencyOptions(weak_segment=0.02, speckle_size=30)
    a, b = copy_maps(maps), copy_maps(maps)
    assert simt_matcher.prepare_depth_map(a[0], opt) == oracle.prepare_depth_map(b[0], opt)
    assert simt_matcher.check_consistency(a[0], a[1:], opt) == oracle.check_consistency(b[0], b[1:], opt)
    assert_same_maps(a, b)
    for call in (lambda impl, m: impl.remove_depth_speckles(m, 25, 0.02),
                 lambda impl, m: impl.remove_depth_halos(m, 10, 30),
                 lambda impl, m: impl.remove_weak_depths(m, ConsistencyOptions(weak_segment=0.05)),
                 lambda impl, m: impl.erode_depth_edges(m, 3, 0.01, True)):
        x, y = copy_maps(maps[1:2]), copy_maps(maps[1:2])
        assert call(simt_matcher, x[0]) == call(oracle, y[0])
        assert_same_maps(x, y)


def test_filter_rejects_bad_arguments(simt_matcher):
    maps, _ = synthetic_scene(2, 32, 24, seed=3)
    with pytest.raises(Exception, match="neighbour index out of range"):
        simt_matcher.filter_depth_maps(maps, [[5], []])
    maps[0]["partners"] = list(range(17))
    with pytest.raises(Exception, match="16"):
        simt_matcher.filter_depth_maps(maps, [[1], [0]])
