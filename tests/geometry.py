"""Test geometry for the multi-view combination (defined in the package,
regard3d_mvs_b200/multi_view.py, where the benchmark uses it too)."""

from regard3d_mvs_b200.multi_view import Plane, Rig, grid_plane_depth, plane_disparity, rot_x, rot_y  # noqa: F401
