"""combine_pairs (src/r3d/mvs/multi_stereo.cpp:74-216): the oracle against the
reference's own tests (tests/test_mvs.cpp:130-226), restated on a rig built
in tests/geometry.py, and the CUDA kernel on the SIMT emulator against the
oracle (bit for bit: depth, confidence and pair mask)."""

from __future__ import annotations

import numpy as np
import pytest

from geometry import Plane, Rig, grid_plane_depth, plane_disparity
from regard3d_mvs_b200.types import MultiStereoOptions


def _inputs(rig, plane, shifts, conf_seed=None):
    pairs = []
    rng = np.random.default_rng(conf_seed) if conf_seed is not None else None
    for p, s in zip(rig.partners, shifts):
        q = rig.rectify(p)
        q["disparity"] = plane_disparity(rig, q, plane, s)
        if rng is not None:
            q["confidence"] = rng.random((rig.h, rig.w)).astype(np.float32)
        pairs.append(q)
    return pairs


def test_oracle_slanted_plane_from_several_pairs(oracle):
    """tests/test_mvs.cpp:130-172: the third pair is wrong by 6 px and is
    outvoted where the other two see the plane."""
    rig, plane = Rig(), Plane()
    m = oracle.combine_pairs(rig.grid(), _inputs(rig, plane, (0.0, 0.0, 6.0)))
    valid = m.depth > 0
    npairs = np.vectorize(lambda v: bin(int(v)).count("1"))(m.pair_mask)
    two = valid & (npairs >= 2)
    assert valid.mean() > 0.5
    assert two.sum() > 0.8 * valid.sum()
    assert not np.any(m.pair_mask[two] & 4)
    truth = grid_plane_depth(rig, plane)
    assert np.max(np.abs(m.depth[two] / truth[two] - 1.0)) < 1e-3


def test_oracle_ties_missing_pairs_and_narrow_angles(oracle):
    """tests/test_mvs.cpp:174-215."""
    rig, plane = Rig(), Plane()
    a = _inputs(rig, plane, (0.0,))
    both = _inputs(rig, plane, (0.0, 5.0))
    single = int((oracle.combine_pairs(rig.grid(), a).depth > 0).sum())
    tie = oracle.combine_pairs(rig.grid(), both)
    assert single > 0
    assert (tie.depth > 0).sum() < single / 2
    for v in tie.pair_mask[tie.depth > 0]:
        assert bin(int(v)).count("1") == 1
    assert (oracle.combine_pairs(rig.grid(), a, MultiStereoOptions(min_pairs=2)).depth > 0).sum() == 0
    # A short baseline: triangulation angles below 3 degrees at about 6 units.
    close = Rig(partners=((0.15, 0.0, 0.0),))
    narrow = _inputs(close, plane, (0.0,))
    assert (oracle.combine_pairs(close.grid(), narrow).depth > 0).sum() == 0
    assert (oracle.combine_pairs(close.grid(), narrow, MultiStereoOptions(min_angle_deg=1.0)).depth > 0).sum() > 0


def test_oracle_sample_disparity(oracle):
    """tests/test_mvs.cpp:217-227."""
    d = np.full((2, 4), 10.0, np.float32)
    d[0, 2] = 10.5
    d[0, 3] = 30.0
    d[1, 3] = np.inf
    got = oracle.sample_disparity(d, [1.5, 2.4, 2.6, -0.6], [0.0, 0.3, 0.6, 0.0])
    assert got[0] == pytest.approx(10.25) and got[1] == pytest.approx(10.5)
    assert np.isinf(got[2]) and np.isinf(got[3])


def _noisy_inputs(rig, plane, seed):
    rng = np.random.default_rng(seed)
    pairs = _inputs(rig, plane, (0.0, 0.4, 6.0), conf_seed=seed)
    for q in pairs:
        d = q["disparity"]
        d += rng.normal(0, 0.3, d.shape).astype(np.float32)
        d[rng.random(d.shape) < 0.1] = np.inf
        d[rng.random(d.shape) < 0.05] += 3.0
    return pairs


@pytest.mark.parametrize("opts", [MultiStereoOptions(), MultiStereoOptions(min_pairs=2, inlier_px=1.0),
                                  MultiStereoOptions(max_reprojection_px=0.3, min_angle_deg=1.0)])
def test_kernel_on_emulator_equals_oracle(simt_matcher, oracle, opts):
    rig, plane = Rig(w=64, h=48, f=60.0), Plane()
    pairs = _noisy_inputs(rig, plane, 3)
    a = simt_matcher.combine_pairs(rig.grid(), pairs, opts)
    b = oracle.combine_pairs(rig.grid(), pairs, opts)
    assert np.array_equal(a.depth, b.depth) and np.array_equal(a.confidence, b.confidence)
    assert np.array_equal(a.pair_mask, b.pair_mask)
    assert (a.depth > 0).mean() > 0.3
