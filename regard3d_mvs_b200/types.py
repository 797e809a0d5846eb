"""Option and result types of the matcher, mirroring the reference's C++ types.

``StereoOptions`` and ``DisparityMap`` follow r3d::StereoOptions and
r3d::DisparityMap (rhiestan/Regard3D_MVS, src/r3d/stereo/stereo_matcher.hpp:23-68):
same field names, meanings and defaults. The ctypes structures mirror
include/r3dgpu.h field for field.
"""

from __future__ import annotations

import ctypes
import enum
from dataclasses import dataclass, field

import numpy as np

INVALID_DISPARITY = float("inf")  # kInvalidDisparity, stereo_matcher.hpp:59


class SubpixelMethod(enum.IntEnum):
    """stereo_matcher.hpp:23-27"""

    none = 0
    parabola = 1
    equiangular = 2


@dataclass
class StereoOptions:
    """stereo_matcher.hpp:30-57 (defaults tuned by the reference on Middlebury 2014)."""

    p1: int = 28
    p2: int = 200
    p2_adapt: int = 4
    invalid_cost: int = 31
    subpixel: SubpixelMethod = SubpixelMethod.equiangular
    uniqueness: float = 0.0
    lr_max_diff: int = 1
    lr_full_match: bool = True
    speckle_size: int = 100
    speckle_diff: float = 1.0
    median: bool = True
    levels: int = -1
    range_radius: int = 3
    range_margin: int = 4
    range_fill: int = 64
    tile_size: int = 512
    tile_margin: int = 32
    tile_blend: int = 32
    memory_budget: int = 2 << 30
    scalar_kernels: bool = False  # accepted for interface parity; the GPU build has one kernel path


@dataclass
class DisparityMap:
    """stereo_matcher.hpp:61-68: disparity is x_left - x_right (+inf where unknown)."""

    disparity: np.ndarray
    confidence: np.ndarray
    disparity_min: int = 0
    num_disparities: int = 0
    levels: int = 0
    cells: int = 0


@dataclass
class LabelRanges:
    """stereo_matcher.hpp:73-76: pixel (x, y) searches labels lo .. lo + num - 1."""

    lo: np.ndarray
    num: np.ndarray


class COptions(ctypes.Structure):
    _fields_ = [
        ("p1", ctypes.c_int32),
        ("p2", ctypes.c_int32),
        ("p2_adapt", ctypes.c_int32),
        ("invalid_cost", ctypes.c_int32),
        ("subpixel", ctypes.c_int32),
        ("uniqueness", ctypes.c_float),
        ("lr_max_diff", ctypes.c_int32),
        ("lr_full_match", ctypes.c_int32),
        ("speckle_size", ctypes.c_int32),
        ("speckle_diff", ctypes.c_float),
        ("median", ctypes.c_int32),
        ("levels", ctypes.c_int32),
        ("range_radius", ctypes.c_int32),
        ("range_margin", ctypes.c_int32),
        ("range_fill", ctypes.c_int32),
        ("tile_size", ctypes.c_int32),
        ("tile_margin", ctypes.c_int32),
        ("tile_blend", ctypes.c_int32),
        ("memory_budget", ctypes.c_uint64),
        ("scalar_kernels", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class CViewU16(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("width", ctypes.c_int32), ("height", ctypes.c_int32),
                ("stride", ctypes.c_int64)]


class CViewU8(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("width", ctypes.c_int32), ("height", ctypes.c_int32),
                ("stride", ctypes.c_int64)]


class CDisparityMap(ctypes.Structure):
    _fields_ = [
        ("disparity", ctypes.c_void_p),
        ("confidence", ctypes.c_void_p),
        ("stride", ctypes.c_int64),
        ("disparity_min", ctypes.c_int32),
        ("num_disparities", ctypes.c_int32),
        ("levels", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("cells", ctypes.c_uint64),
    ]


class CPair(ctypes.Structure):
    _fields_ = [
        ("left", CViewU16),
        ("right", CViewU16),
        ("left_valid", CViewU8),
        ("right_valid", CViewU8),
        ("disparity_min", ctypes.c_int32),
        ("num_disparities", ctypes.c_int32),
        ("options", COptions),
        ("out", CDisparityMap),
    ]


class CDepthGrid(ctypes.Structure):
    _fields_ = [
        ("k_inv", ctypes.c_double * 9),
        ("rot_t", ctypes.c_double * 9),
        ("center", ctypes.c_double * 3),
        ("width", ctypes.c_int32),
        ("height", ctypes.c_int32),
    ]


class CPairGeometry(ctypes.Structure):
    _fields_ = [
        ("grid_to_rect", ctypes.c_double * 9),
        ("fb", ctypes.c_double),
        ("offset", ctypes.c_double),
        ("partner_center", ctypes.c_double * 3),
        ("disparity", ctypes.c_void_p),
        ("confidence", ctypes.c_void_p),
        ("width", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("stride", ctypes.c_int64),
    ]


class CMultiStereoOptions(ctypes.Structure):
    _fields_ = [
        ("inlier_px", ctypes.c_double),
        ("max_reprojection_px", ctypes.c_double),
        ("min_angle_deg", ctypes.c_double),
        ("min_pairs", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


@dataclass
class MultiStereoOptions:
    """MultiStereoOptions, src/r3d/mvs/multi_stereo.hpp:25-30."""

    inlier_px: float = 2.0
    max_reprojection_px: float = 1.0
    min_angle_deg: float = 3.0
    min_pairs: int = 1

    def c(self) -> CMultiStereoOptions:
        return CMultiStereoOptions(self.inlier_px, self.max_reprojection_px, self.min_angle_deg, self.min_pairs, 0)


@dataclass
class DepthMap:
    """DepthMap (src/r3d/mvs/depth_map.hpp:17-31): depth 0 = none, pair_mask bit i = pair i used."""

    depth: np.ndarray
    confidence: np.ndarray
    pair_mask: np.ndarray


# Camera models of CameraIntrinsics (src/r3d/core/camera_model.hpp:15-21).
CAMERA_MODELS = {"pinhole": 0, "radial_k1": 1, "radial_k3": 2, "brown_t2": 3, "fisheye": 4}


class CCamera(ctypes.Structure):
    """r3dgpu_camera: CameraIntrinsics, src/r3d/core/camera_model.hpp:32-41."""

    _fields_ = [
        ("model", ctypes.c_int32),
        ("width", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("fx", ctypes.c_double),
        ("fy", ctypes.c_double),
        ("cx", ctypes.c_double),
        ("cy", ctypes.c_double),
        ("params", ctypes.c_double * 5),
    ]


class CPinhole(ctypes.Structure):
    """r3dgpu_pinhole: PinholeIntrinsics of a rectified camera."""

    _fields_ = [
        ("width", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("fx", ctypes.c_double),
        ("fy", ctypes.c_double),
        ("cx", ctypes.c_double),
        ("cy", ctypes.c_double),
    ]


def camera_struct(cam: dict) -> CCamera:
    """CCamera from {model (name or number), width, height, fx, fy, cx, cy, params}."""
    model = cam.get("model", 0)
    model = CAMERA_MODELS[model] if isinstance(model, str) else int(model)
    params = list(cam.get("params", ()))
    if len(params) > 5:
        raise ValueError("at most 5 distortion parameters")
    c = CCamera(model, int(cam["width"]), int(cam["height"]), 0, float(cam["fx"]), float(cam["fy"]),
                float(cam["cx"]), float(cam["cy"]))
    for i, v in enumerate(params):
        c.params[i] = float(v)
    return c


def pinhole_struct(k: dict) -> CPinhole:
    """CPinhole from {width, height, fx, fy, cx, cy}."""
    return CPinhole(int(k["width"]), int(k["height"]), float(k["fx"]), float(k["fy"]), float(k["cx"]),
                    float(k["cy"]))


class CServerConfig(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32),
        ("workers", ctypes.c_int32),
        ("max_batch", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("hbm_budget", ctypes.c_uint64),
        ("scratch_budget", ctypes.c_uint64),
        ("cache_budget", ctypes.c_uint64),
    ]


class CRequest(ctypes.Structure):
    """r3dgpu_request: the fields of r3dgpu_pair, then the images' content keys."""

    _fields_ = CPair._fields_ + [("left_key", ctypes.c_uint64), ("right_key", ctypes.c_uint64)]


class CRequestTimes(ctypes.Structure):
    _fields_ = [
        ("queued_ms", ctypes.c_double),
        ("run_ms", ctypes.c_double),
        ("total_ms", ctypes.c_double),
        ("device_bytes", ctypes.c_uint64),
        ("batch_size", ctypes.c_int32),
        ("worker", ctypes.c_int32),
        ("cache_hits", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("uploaded_bytes", ctypes.c_uint64),
    ]


class CProfile(ctypes.Structure):
    _fields_ = [
        ("sgm_ms", ctypes.c_double),
        ("sgm_launches", ctypes.c_uint64),
        ("sgm_cells", ctypes.c_uint64),
        ("sgm_tiles", ctypes.c_uint64),
        ("sgm_pixels", ctypes.c_uint64),
    ]


class CSynthParams(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("num_disparities", ctypes.c_int32),
        ("seed", ctypes.c_uint32),
        ("blur_sigma", ctypes.c_float),
        ("noise_sigma", ctypes.c_float),
        ("planes", ctypes.c_int32),
        ("textureless_fraction", ctypes.c_float),
        ("occluded_fraction", ctypes.c_float),
    ]


def to_c_options(o) -> COptions:
    """Fills the C struct from a StereoOptions (or any object with its fields)."""
    c = COptions()
    c.p1 = int(o.p1)
    c.p2 = int(o.p2)
    c.p2_adapt = int(o.p2_adapt)
    c.invalid_cost = int(o.invalid_cost)
    c.subpixel = int(o.subpixel)
    c.uniqueness = float(o.uniqueness)
    c.lr_max_diff = int(o.lr_max_diff)
    c.lr_full_match = int(bool(o.lr_full_match))
    c.speckle_size = int(o.speckle_size)
    c.speckle_diff = float(o.speckle_diff)
    c.median = int(bool(o.median))
    c.levels = int(o.levels)
    c.range_radius = int(o.range_radius)
    c.range_margin = int(o.range_margin)
    c.range_fill = int(o.range_fill)
    c.tile_size = int(o.tile_size)
    c.tile_margin = int(o.tile_margin)
    c.tile_blend = int(o.tile_blend)
    c.memory_budget = int(o.memory_budget)
    c.scalar_kernels = int(bool(o.scalar_kernels))
    c.reserved = 0
    return c
