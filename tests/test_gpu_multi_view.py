"""combine_pairs on the B200 against the oracle: depth, confidence and pair
mask bit for bit (the kernel computes in double precision in the reference's
operation order, without contraction)."""

from __future__ import annotations

import numpy as np
import pytest

from geometry import Plane, Rig, grid_plane_depth, plane_disparity
from regard3d_mvs_b200.types import MultiStereoOptions

pytestmark = pytest.mark.gpu


def _pairs(rig, plane, shifts, seed):
    rng = np.random.default_rng(seed)
    out = []
    for p, s in zip(rig.partners, shifts):
        q = rig.rectify(p)
        d = plane_disparity(rig, q, plane, s)
        d += rng.normal(0, 0.3, d.shape).astype(np.float32)
        d[rng.random(d.shape) < 0.08] = np.inf
        d[rng.random(d.shape) < 0.05] += 4.0
        q["disparity"] = d
        q["confidence"] = rng.random(d.shape).astype(np.float32)
        out.append(q)
    return out


@pytest.mark.parametrize("opts", [MultiStereoOptions(), MultiStereoOptions(min_pairs=2, inlier_px=1.0),
                                  MultiStereoOptions(max_reprojection_px=0.25, min_angle_deg=2.0)])
def test_combine_pairs_equals_oracle(gpu_matcher, oracle, opts):
    rig = Rig(w=640, h=480, f=600.0, partners=((0.6, 0.0, 0.0), (-0.5, 0.3, 0.1), (0.2, -0.55, 0.0),
                                                (-0.3, -0.4, 0.2)))
    plane = Plane()
    pairs = _pairs(rig, plane, (0.0, 0.5, 6.0, 0.0), 11)
    a = gpu_matcher.combine_pairs(rig.grid(), pairs, opts)
    b = oracle.combine_pairs(rig.grid(), pairs, opts)
    assert np.array_equal(a.depth, b.depth), int((a.depth != b.depth).sum())
    assert np.array_equal(a.confidence, b.confidence) and np.array_equal(a.pair_mask, b.pair_mask)
    assert (a.depth > 0).mean() > 0.3


def test_combine_pairs_plane_accuracy(gpu_matcher):
    rig, plane = Rig(w=320, h=240, f=300.0), Plane()
    pairs = []
    for p, s in zip(rig.partners, (0.0, 0.0, 6.0)):
        q = rig.rectify(p)
        q["disparity"] = plane_disparity(rig, q, plane, s)
        pairs.append(q)
    m = gpu_matcher.combine_pairs(rig.grid(), pairs)
    two = (m.depth > 0) & (np.vectorize(lambda v: bin(int(v)).count("1"))(m.pair_mask) >= 2)
    truth = grid_plane_depth(rig, plane)
    assert two.mean() > 0.4
    assert np.max(np.abs(m.depth[two] / truth[two] - 1.0)) < 1e-3
    assert not np.any(m.pair_mask[two] & 4)
