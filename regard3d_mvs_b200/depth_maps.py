"""Depth maps of the multi-view stage over the C ABI: the ctypes structures of
include/r3dgpu.h's depth-map section and their construction from numpy.

A depth map is a dict (the fields of r3d::DepthMap, src/r3d/mvs/depth_map.hpp:17-41):
``camera`` ({width, height, fx, fy, cx, cy, rotation (3x3, world -> camera),
center (3)}), ``depth`` (float32 H x W, 0 = none), ``confidence`` (float32),
``pair_mask`` (uint16), ``support`` (uint8, written by the check), ``color``
(uint8 H x W x 3 or None), ``view`` (int) and ``partners`` (scene view of
each pair bit, at most 16).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, fields

import numpy as np

from .types import CPinhole

MAX_PARTNERS = 16


class CPinholeCamera(ctypes.Structure):
    _fields_ = [
        ("intrinsics", CPinhole),
        ("rotation", ctypes.c_double * 9),
        ("center", ctypes.c_double * 3),
        ("k_inv", ctypes.c_double * 9),
    ]


class CDepthMap(ctypes.Structure):
    _fields_ = [
        ("camera", CPinholeCamera),
        ("depth", ctypes.c_void_p),
        ("confidence", ctypes.c_void_p),
        ("pair_mask", ctypes.c_void_p),
        ("support", ctypes.c_void_p),
        ("color", ctypes.c_void_p),
        ("stride", ctypes.c_int64),
        ("color_stride", ctypes.c_int64),
        ("width", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("view", ctypes.c_uint32),
        ("num_partners", ctypes.c_uint32),
        ("partners", ctypes.c_uint32 * MAX_PARTNERS),
    ]


class CConsistencyOptions(ctypes.Structure):
    _fields_ = [
        ("max_relative_depth_error", ctypes.c_double),
        ("max_reprojection_px", ctypes.c_double),
        ("min_views", ctypes.c_int32),
        ("min_evidence", ctypes.c_int32),
        ("min_confidence", ctypes.c_float),
        ("edge_erosion", ctypes.c_int32),
        ("discontinuity", ctypes.c_double),
        ("erode_holes", ctypes.c_int32),
        ("max_neighbours", ctypes.c_int32),
        ("independent_support", ctypes.c_int32),
        ("average_depths", ctypes.c_int32),
        ("weak_texture", ctypes.c_double),
        ("weak_segment", ctypes.c_double),
        ("reject_weak", ctypes.c_int32),
        ("halo_px", ctypes.c_int32),
        ("halo_colour", ctypes.c_int32),
        ("speckle_size", ctypes.c_int32),
        ("speckle_step", ctypes.c_double),
    ]


class CConsistencyStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in
                ("input", "unconfident", "eroded", "rejected", "weak", "halo", "speckles", "output")]

    def as_dict(self) -> dict:
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


@dataclass
class ConsistencyOptions:
    """ConsistencyOptions, src/r3d/mvs/consistency.hpp:59-78 (same defaults)."""

    max_relative_depth_error: float = 0.01
    max_reprojection_px: float = 2.0
    min_views: int = 0
    min_evidence: int = 2
    min_confidence: float = 0.0
    edge_erosion: int = 1
    discontinuity: float = 0.05
    erode_holes: bool = False
    max_neighbours: int = 8
    independent_support: bool = False
    average_depths: bool = True
    weak_texture: float = 2.0
    weak_segment: float = 0.0
    reject_weak: bool = False
    halo_px: int = 32
    halo_colour: int = 25
    speckle_size: int = 0
    speckle_step: float = 0.02

    def c(self) -> CConsistencyOptions:
        return CConsistencyOptions(*[int(v) if isinstance(v, bool) else v
                                     for v in (getattr(self, f.name) for f in fields(self))])


def k_inverse(cam: dict) -> np.ndarray:
    """K^-1 of a pinhole camera (row-major)."""
    fx, fy, cx, cy = cam["fx"], cam["fy"], cam["cx"], cam["cy"]
    return np.array([[1.0 / fx, 0.0, -cx / fx], [0.0, 1.0 / fy, -cy / fy], [0.0, 0.0, 1.0]])


def c_camera(cam: dict) -> CPinholeCamera:
    c = CPinholeCamera()
    c.intrinsics = CPinhole(int(cam["width"]), int(cam["height"]), float(cam["fx"]), float(cam["fy"]),
                            float(cam["cx"]), float(cam["cy"]))
    for i, v in enumerate(np.asarray(cam["rotation"], np.float64).reshape(9)):
        c.rotation[i] = float(v)
    for i, v in enumerate(np.asarray(cam["center"], np.float64).reshape(3)):
        c.center[i] = float(v)
    k_inv = cam.get("k_inv")
    for i, v in enumerate(np.asarray(k_inverse(cam) if k_inv is None else k_inv, np.float64).reshape(9)):
        c.k_inv[i] = float(v)
    return c


def normalise(m: dict) -> dict:
    """Contiguous arrays of the right types; allocates support if missing."""
    d = np.ascontiguousarray(m["depth"], np.float32)
    h, w = d.shape
    out = dict(m)
    out["depth"] = d
    out["confidence"] = np.ascontiguousarray(m["confidence"], np.float32) if m.get("confidence") is not None \
        else np.zeros((h, w), np.float32)
    out["pair_mask"] = np.ascontiguousarray(m["pair_mask"], np.uint16) if m.get("pair_mask") is not None \
        else np.zeros((h, w), np.uint16)
    out["support"] = m["support"] if isinstance(m.get("support"), np.ndarray) and m["support"].shape == (h, w) \
        and m["support"].dtype == np.uint8 and m["support"].flags.c_contiguous else np.zeros((h, w), np.uint8)
    c = m.get("color")
    out["color"] = None if c is None else np.ascontiguousarray(c, np.uint8).reshape(h, w, 3)
    return out


def c_depth_map(m: dict, ptr) -> CDepthMap:
    """CDepthMap of a normalised map; ptr(array) gives the pointer to use
    (host pointers, or device copies)."""
    h, w = m["depth"].shape
    c = CDepthMap()
    c.camera = c_camera(m["camera"])
    c.depth = ptr(m["depth"])
    c.confidence = ptr(m["confidence"])
    c.pair_mask = ptr(m["pair_mask"])
    c.support = ptr(m["support"])
    c.color = None if m["color"] is None else ptr(m["color"])
    c.stride = w
    c.color_stride = 3 * w
    c.width, c.height = w, h
    c.view = int(m.get("view", 0))
    partners = list(m.get("partners", ()))
    if len(partners) > MAX_PARTNERS:
        raise ValueError("at most 16 partners")
    c.num_partners = len(partners)
    for i, p in enumerate(partners):
        c.partners[i] = int(p)
    return c


def neighbour_lists(neighbours) -> tuple[np.ndarray, np.ndarray]:
    """CSR form (offsets, indices) of per-map neighbour lists."""
    off = np.zeros(len(neighbours) + 1, np.int32)
    for i, nb in enumerate(neighbours):
        off[i + 1] = off[i] + len(nb)
    idx = np.array([j for nb in neighbours for j in nb], np.int32)
    return off, (idx if idx.size else np.zeros(1, np.int32))


# ------------------------------------------------------------------ refinement
class CRefinementOptions(ctypes.Structure):
    _fields_ = [
        ("radius", ctypes.c_int32),
        ("step", ctypes.c_int32),
        ("iterations", ctypes.c_int32),
        ("max_views", ctypes.c_int32),
        ("min_ncc", ctypes.c_double),
        ("max_shift_px", ctypes.c_double),
        ("min_gain", ctypes.c_double),
        ("min_texture", ctypes.c_double),
        ("blur_sigma", ctypes.c_double),
        ("drop_unconfirmed", ctypes.c_int32),
        ("fp32", ctypes.c_int32),
    ]


class CRefinementStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("input", "refined", "kept", "unconfirmed")]

    def as_dict(self) -> dict:
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


class CRefinementImage(ctypes.Structure):
    _fields_ = [("camera", CPinholeCamera), ("data", ctypes.c_void_p), ("stride", ctypes.c_int64)]


@dataclass
class RefinementOptions:
    """RefinementOptions, src/r3d/mvs/refinement.hpp:33-44 (same defaults);
    fp32 computes the window terms in float."""

    radius: int = 4
    step: int = 2
    iterations: int = 6
    max_views: int = 4
    min_ncc: float = 0.3
    max_shift_px: float = 2.0
    min_gain: float = 0.02
    min_texture: float = 1.0
    blur_sigma: float = 0.0
    drop_unconfirmed: bool = True
    fp32: bool = False

    def c(self) -> CRefinementOptions:
        return CRefinementOptions(*[int(v) if isinstance(v, bool) else v
                                    for v in (getattr(self, f.name) for f in fields(self))])


def c_refinement_image(img: dict, ptr) -> CRefinementImage:
    """img: {camera, data (H x W x 3 float32)}."""
    data = img["data"]
    c = CRefinementImage()
    c.camera = c_camera(img["camera"])
    c.data = ptr(data)
    c.stride = 3 * data.shape[1]
    return c


# ------------------------------------------------------------------ .r3dd files
def write_depth_map(lib, path: str, m: dict) -> None:
    """write_depth_map (src/r3d/mvs/depth_map.hpp:58) of a host map."""
    from . import _native

    n = normalise(m)
    if n["color"] is None:
        n["color"] = np.zeros(n["depth"].shape + (3,), np.uint8)
    c = c_depth_map(n, lambda a: a.ctypes.data)
    _native.check(lib, lib.r3dgpu_write_depth_map(str(path).encode(), ctypes.byref(c), 0, None))


def read_depth_map(lib, path: str) -> dict:
    """read_depth_map (src/r3d/mvs/depth_map.hpp:59): a map dict."""
    from . import _native

    c = CDepthMap()
    _native.check(lib, lib.r3dgpu_read_depth_map_info(str(path).encode(), ctypes.byref(c)))
    h, w = c.height, c.width
    m = {"depth": np.empty((h, w), np.float32), "confidence": np.empty((h, w), np.float32),
         "pair_mask": np.empty((h, w), np.uint16), "support": np.empty((h, w), np.uint8),
         "color": np.empty((h, w, 3), np.uint8)}
    c.depth, c.confidence = m["depth"].ctypes.data, m["confidence"].ctypes.data
    c.pair_mask, c.support, c.color = m["pair_mask"].ctypes.data, m["support"].ctypes.data, m["color"].ctypes.data
    c.stride, c.color_stride = w, 3 * w
    _native.check(lib, lib.r3dgpu_read_depth_map(str(path).encode(), ctypes.byref(c)))
    k = c.camera.intrinsics
    m["camera"] = {"width": k.width, "height": k.height, "fx": k.fx, "fy": k.fy, "cx": k.cx, "cy": k.cy,
                   "rotation": np.array(c.camera.rotation[:]).reshape(3, 3), "center": np.array(c.camera.center[:]),
                   "k_inv": np.array(c.camera.k_inv[:]).reshape(3, 3)}
    m["view"] = int(c.view)
    m["partners"] = [int(c.partners[i]) for i in range(c.num_partners)]
    return m
