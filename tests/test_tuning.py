"""The autotuner's table reaches the launches: entries given through
R3DGPU_TUNING set the band rows of the ranged kernel and the shape of the
full-range kernel (seen in the library's per-launch profile), results stay
identical, and environment overrides take precedence."""

from __future__ import annotations

import ctypes
import json

import numpy as np

from images import Texture, render_pair
from regard3d_mvs_b200.types import CProfile, LabelRanges, StereoOptions


def _launches(m, run):
    lib = m.lib
    lib.r3dgpu_profile_enable(1)
    prof = CProfile()
    lib.r3dgpu_profile_take(ctypes.byref(prof))
    out = run()
    lib.r3dgpu_profile_take(ctypes.byref(prof))
    lib.r3dgpu_profile_enable(0)
    n = lib.r3dgpu_profile_launches(None, 0)
    buf = ctypes.create_string_buffer(int(n) + 1)
    lib.r3dgpu_profile_launches(buf, n + 1)
    return out, [e for e in json.loads(buf.value.decode() or "[]") if e["kernel"] != "sgm_round"]


def test_default_kernels_are_the_chain_passes(simt_matcher):
    """Full-range and ranged tiles go to the chain-pass kernels by default."""
    tex = Texture(61)
    left, right, _ = render_pair(tex, 40, 30, lambda x, y: 6.0 + 0.1 * x)
    pairs = [dict(left=left, right=right, disparity_min=0, num_disparities=32, options=StereoOptions(levels=0)),
             dict(left=left, right=right, disparity_min=0, num_disparities=32, options=StereoOptions(levels=1))]
    _, launches = _launches(simt_matcher, lambda: simt_matcher.match_stereo_batch(pairs))
    kinds = {e["kernel"] for e in launches}
    assert kinds == {"sgm_path_kernel", "sgm_path_ranged_kernel"}, kinds


def test_table_from_environment(simt_matcher, monkeypatch):
    """The table drives the one-CTA-per-tile kernels (selected by the environment)."""
    monkeypatch.setenv("R3DGPU_FULL_KERNEL", "wavefront")
    monkeypatch.setenv("R3DGPU_RANGED_KERNEL", "ranged")
    tex = Texture(61)
    left, right, _ = render_pair(tex, 40, 30, lambda x, y: 6.0 + 0.1 * x)
    pairs = [dict(left=left, right=right, disparity_min=0, num_disparities=32, options=StereoOptions(levels=0))]
    monkeypatch.setenv("R3DGPU_TUNING", "#")
    ref, launches = _launches(simt_matcher, lambda: simt_matcher.match_stereo_batch(pairs))
    assert [e["shape"] for e in launches] == ["8x4/nd32"]
    monkeypatch.setenv("R3DGPU_TUNING", "full 32 16 4 6; ranged 32 8")
    got, launches = _launches(simt_matcher, lambda: simt_matcher.match_stereo_batch(pairs))
    assert [(e["shape"], e["rows"]) for e in launches] == [("16x4/nd32", 6)]
    assert np.array_equal(np.nan_to_num(got[0].disparity, posinf=-1), np.nan_to_num(ref[0].disparity, posinf=-1))
    # Ranged kernel rows, and an environment override that wins over the table.
    lo = np.full((30, 40), 4, np.uint16)
    num = np.full((30, 40), 16, np.uint16)
    _, launches = _launches(simt_matcher, lambda: simt_matcher.match_stereo_batch(pairs))
    monkeypatch.setenv("R3DGPU_FULL_ROWS", "2")
    _, launches = _launches(simt_matcher, lambda: simt_matcher.match_stereo_batch(pairs))
    assert [(e["shape"], e["rows"]) for e in launches] == [("16x4/nd32", 2)]
    vol = simt_matcher.sgm_cost_volume(left, right, 0, 32, StereoOptions(), LabelRanges(lo, num))
    assert vol.size == 16 * 40 * 30


def test_path_shape_from_table(simt_matcher, monkeypatch):
    """A `path` entry sets the chain passes' shape for its label count (seen
    in the per-pass profile), R3DGPU_PATH_SHAPE overrides it, and the maps
    stay identical."""
    tex = Texture(62)
    left, right, _ = render_pair(tex, 40, 30, lambda x, y: 6.0 + 0.1 * x)
    pairs = [dict(left=left, right=right, disparity_min=0, num_disparities=64, options=StereoOptions(levels=0))]

    def shapes(launches):
        return {e["shape"].split("/")[0] for e in launches if e.get("pass")}

    monkeypatch.setenv("R3DGPU_TUNING", "#")
    ref, launches = _launches(simt_matcher, lambda: simt_matcher.match_stereo_batch(pairs))
    assert shapes(launches) == {"4x8"}
    monkeypatch.setenv("R3DGPU_TUNING", "path 64 2 16")
    got, launches = _launches(simt_matcher, lambda: simt_matcher.match_stereo_batch(pairs))
    assert shapes(launches) == {"2x16"}
    assert np.array_equal(np.nan_to_num(got[0].disparity, posinf=-1), np.nan_to_num(ref[0].disparity, posinf=-1))
    monkeypatch.setenv("R3DGPU_PATH_SHAPE", "8,8")
    got, launches = _launches(simt_matcher, lambda: simt_matcher.match_stereo_batch(pairs))
    assert shapes(launches) == {"8x8"}
    assert np.array_equal(np.nan_to_num(got[0].disparity, posinf=-1), np.nan_to_num(ref[0].disparity, posinf=-1))
