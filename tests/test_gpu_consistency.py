"""Geometric consistency on the B200 against the oracle: depths, support
counts and statistics bit for bit (the projection check computes in double
precision in the reference's order; the segment filters' log depths come from
logf, and the scenes keep neighbouring log depths far from the segment step,
so a last-ulp difference between CUDA's and the host's logf cannot move a
segment border)."""

from __future__ import annotations

import pytest

from mvs_scenes import copy_maps, synthetic_scene
from test_consistency import OPTION_SETS, assert_same_maps, rig_maps
from regard3d_mvs_b200.depth_maps import ConsistencyOptions

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("k", range(len(OPTION_SETS)))
def test_filter_equals_oracle(gpu_matcher, oracle, k):
    maps, nbs = synthetic_scene(5, 320, 240, seed=40 + k)
    a, b = copy_maps(maps), copy_maps(maps)
    assert gpu_matcher.filter_depth_maps(a, nbs, OPTION_SETS[k]) == oracle.filter_depth_maps(b, nbs, OPTION_SETS[k])
    assert_same_maps(a, b)


def test_filter_full_size_equals_oracle(gpu_matcher, oracle):
    """Four 2048 x 1536 maps, each checked against its neighbours."""
    maps, nbs = synthetic_scene(4, 2048, 1536, seed=7)
    opt = ConsistencyOptions(speckle_size=100, weak_segment=0.001)
    a, b = copy_maps(maps), copy_maps(maps)
    sa = gpu_matcher.filter_depth_maps(a, nbs, opt)
    sb = oracle.filter_depth_maps(b, nbs, opt)
    assert sa == sb
    assert_same_maps(a, b)
    assert sb["output"] > sb["input"] // 2


def test_reference_cases_on_gpu(gpu_matcher, oracle):
    """tests/test_mvs.cpp:243-260 through the device entry points."""
    maps = rig_maps()
    opt = ConsistencyOptions(edge_erosion=0, min_views=1, independent_support=True)
    a, b = copy_maps(maps), copy_maps(maps)
    assert gpu_matcher.filter_depth_maps(a, [[1, 2], [0, 2], [0, 1]], opt) == \
        oracle.filter_depth_maps(b, [[1, 2], [0, 2], [0, 1]], opt)
    assert_same_maps(a, b)
    assert a[0]["support"][60, 60] == 1


def test_single_steps_equal_oracle(gpu_matcher, oracle):
    maps, _ = synthetic_scene(3, 640, 480, seed=22)
    opt = ConsistencyOptions(weak_segment=0.02, speckle_size=30)
    a, b = copy_maps(maps), copy_maps(maps)
    assert gpu_matcher.prepare_depth_map(a[0], opt) == oracle.prepare_depth_map(b[0], opt)
    assert gpu_matcher.check_consistency(a[0], a[1:], opt) == oracle.check_consistency(b[0], b[1:], opt)
    assert_same_maps(a, b)
    for call in (lambda impl, m: impl.remove_depth_speckles(m, 25, 0.02),
                 lambda impl, m: impl.remove_depth_halos(m, 10, 30),
                 lambda impl, m: impl.remove_weak_depths(m, ConsistencyOptions(weak_segment=0.05)),
                 lambda impl, m: impl.erode_depth_edges(m, 3, 0.01, True)):
        x, y = copy_maps(maps[1:2]), copy_maps(maps[1:2])
        assert call(gpu_matcher, x[0]) == call(oracle, y[0])
        assert_same_maps(x, y)
