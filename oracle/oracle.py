"""ctypes access to the CPU oracle (oracle/r3d_oracle.cpp) — TEST INFRASTRUCTURE.

Only the tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg
import this module: it is the checker of the GPU library, never part of the
product. Each function mirrors the reference function it restates
(rhiestan/Regard3D_MVS, src/r3d/stereo/stereo_matcher.hpp and census.hpp).
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle_r3d.so")
_lib = None


def build() -> str:
    """Compiles the oracle with its Makefile (g++, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        i32 = ctypes.c_int
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_set_threads.argtypes = [i32]
        L.orc_max_threads.restype = i32
        L.orc_census.argtypes = [P, i32, i32, P]
        L.orc_pyramid_down_u16.argtypes = [P, i32, i32, P]
        L.orc_pyramid_down_u8.argtypes = [P, i32, i32, P]
        L.orc_automatic_levels.argtypes = [i32, i32, i32]
        L.orc_automatic_levels.restype = i32
        L.orc_sgm_cost_volume.argtypes = [P, i32, i32, P, i32, i32, i32, P, P, P, P, ctypes.c_uint64, P]
        L.orc_ranges_from_coarse.argtypes = [P, i32, i32, i32, i32, P, P, i32, i32, i32, i32, P, i32, P, P]
        L.orc_remove_speckles.argtypes = [P, i32, i32, i32, ctypes.c_float]
        L.orc_median_filter_3x3.argtypes = [P, i32, i32, P]
        L.orc_match_stereo.argtypes = [P, i32, i32, P, i32, P, P, i32, i32, P, P, P, P]
        L.orc_match_tiles.argtypes = [P, i32, i32, P, i32, P, P, i32, i32, P, P, P, i32, P, P, P]
        L.orc_combine_pairs.argtypes = [P, P, i32, P, P, P, P, ctypes.c_int64]
        L.orc_sample_disparity.argtypes = [P, i32, i32, P, P, i32, P]
        L.orc_rectify_image.argtypes = [i32, P, P, P, P, P, P]
        L.orc_distort_pixel.argtypes = [P, P, i32, P]
        L.orc_mvs_last_error.restype = ctypes.c_char_p
        L.orc_filter_depth_maps.argtypes = [P, i32, P, P, P, P]
        L.orc_prepare_depth_map.argtypes = [P, P, P]
        L.orc_check_consistency.argtypes = [P, P, i32, P, P]
        L.orc_erode_depth_edges.argtypes = [P, i32, ctypes.c_double, i32, P]
        L.orc_remove_weak_depths.argtypes = [P, P, P]
        L.orc_remove_depth_halos.argtypes = [P, i32, i32, P]
        L.orc_remove_depth_speckles.argtypes = [P, i32, ctypes.c_double, P]
        L.orc_make_refinement_image.argtypes = [P, i32, i32, ctypes.c_double, P]
        L.orc_refine_depth_map.argtypes = [P, P, ctypes.c_int64, P, i32, i32, P, P, i32, P, P]
        L.r3dgpu_synth_pair.argtypes = [P, P, P, P]
        _lib = L
    return _lib


class OracleError(RuntimeError):
    pass


def _check(rc: int) -> None:
    if rc != 0:
        raise OracleError(lib().orc_last_error().decode())


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _c(a, dtype):
    return None if a is None else np.ascontiguousarray(a, dtype=dtype)


def options_struct(opts):
    """r3dgpu_stereo_options from a StereoOptions-like object (duck typed)."""
    from regard3d_mvs_b200.types import StereoOptions, to_c_options  # layout shared with the product header

    return to_c_options(opts if opts is not None else StereoOptions())


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def max_threads() -> int:
    return int(lib().orc_max_threads())


class _SynthParams(ctypes.Structure):
    # include/r3dgpu_synth.h, r3dgpu_synth_params
    _fields_ = [("width", ctypes.c_int32), ("height", ctypes.c_int32), ("num_disparities", ctypes.c_int32),
                ("seed", ctypes.c_uint32), ("blur_sigma", ctypes.c_float), ("noise_sigma", ctypes.c_float),
                ("planes", ctypes.c_int32), ("textureless_fraction", ctypes.c_float),
                ("occluded_fraction", ctypes.c_float)]


def synth_pair(width: int, height: int, num_disparities: int, seed: int, textureless: float = 0.0,
               occluded: float = 0.0, blur_sigma: float = 1.5, noise_sigma: float = 2.0, planes: int = 8):
    """The seeded benchmark pair (8-bit left and right images) from the
    generator compiled into the oracle library: the same source and the same
    bytes as r3dgpu_synth_pair of the CUDA library, without loading it."""
    p = _SynthParams(int(width), int(height), int(num_disparities), int(seed) & 0xFFFFFFFF, blur_sigma,
                     noise_sigma, int(planes), textureless, occluded)
    left = np.empty((height, width), np.uint8)
    right = np.empty_like(left)
    _check(lib().r3dgpu_synth_pair(ctypes.byref(p), _ptr(left), _ptr(right), None))
    return left, right


def census_transform(img: np.ndarray) -> np.ndarray:
    img = _c(img, np.uint16)
    out = np.empty(img.shape, np.uint64)
    _check(lib().orc_census(_ptr(img), img.shape[1], img.shape[0], _ptr(out)))
    return out


def pyramid_down(img: np.ndarray) -> np.ndarray:
    h, w = img.shape
    if img.dtype == np.uint8:
        img = _c(img, np.uint8)
        out = np.empty(((h + 1) // 2, (w + 1) // 2), np.uint8)
        _check(lib().orc_pyramid_down_u8(_ptr(img), w, h, _ptr(out)))
    else:
        img = _c(img, np.uint16)
        out = np.empty(((h + 1) // 2, (w + 1) // 2), np.uint16)
        _check(lib().orc_pyramid_down_u16(_ptr(img), w, h, _ptr(out)))
    return out


def automatic_levels(w: int, h: int, nd: int) -> int:
    return int(lib().orc_automatic_levels(w, h, nd))


def sgm_cost_volume(left, right, dmin, nd, options=None, ranges=None) -> np.ndarray:
    left = _c(left, np.uint16)
    right = _c(right, np.uint16)
    o = options_struct(options)
    lo = num = None
    if ranges is not None:
        lo = _c(ranges[0], np.uint16)
        num = _c(ranges[1], np.uint16)
    count = ctypes.c_uint64(0)
    h, wl = left.shape
    wr = right.shape[1]
    _check(lib().orc_sgm_cost_volume(_ptr(left), wl, h, _ptr(right), wr, dmin, nd, ctypes.byref(o), _ptr(lo),
                                     _ptr(num), None, 0, ctypes.byref(count)))
    out = np.empty(count.value, np.uint16)
    _check(lib().orc_sgm_cost_volume(_ptr(left), wl, h, _ptr(right), wr, dmin, nd, ctypes.byref(o), _ptr(lo),
                                     _ptr(num), _ptr(out), count.value, ctypes.byref(count)))
    return out


def ranges_from_coarse(coarse, width, height, fine_valid, partner_valid, partner_width, partner_sign, dmin, nd,
                       options=None, mirrored=False):
    coarse = _c(coarse, np.float32)
    fv = _c(fine_valid, np.uint8)
    pv = _c(partner_valid, np.uint8)
    o = options_struct(options)
    lo = np.empty((height, width), np.uint16)
    num = np.empty((height, width), np.uint16)
    _check(lib().orc_ranges_from_coarse(_ptr(coarse), coarse.shape[1], coarse.shape[0], width, height, _ptr(fv),
                                        _ptr(pv), partner_width, partner_sign, dmin, nd, ctypes.byref(o),
                                        int(bool(mirrored)), _ptr(lo), _ptr(num)))
    return lo, num


def remove_speckles(disp: np.ndarray, min_size: int, max_diff: float) -> np.ndarray:
    d = np.array(disp, dtype=np.float32, order="C", copy=True)
    _check(lib().orc_remove_speckles(_ptr(d), d.shape[1], d.shape[0], int(min_size), float(max_diff)))
    return d


def combine_pairs(grid: dict, pairs: list, options=None):
    """r3d::combine_pairs (src/r3d/mvs/multi_stereo.cpp:74-216) on the CPU;
    grid and pairs as in regard3d_mvs_b200.multi_view."""
    from regard3d_mvs_b200.multi_view import c_grid, c_pairs
    from regard3d_mvs_b200.types import DepthMap, MultiStereoOptions

    g = c_grid(grid)
    arr, keep = c_pairs(grid, pairs)
    o = (options or MultiStereoOptions()).c()
    depth = np.empty((g.height, g.width), np.float32)
    conf = np.empty_like(depth)
    mask = np.empty((g.height, g.width), np.uint16)
    _check(lib().orc_combine_pairs(ctypes.byref(g), arr, len(pairs), ctypes.byref(o), _ptr(depth), _ptr(conf),
                                   _ptr(mask), g.width))
    del keep
    return DepthMap(depth, conf, mask)


def sample_disparity(disp: np.ndarray, u, v) -> np.ndarray:
    """r3d::sample_disparity (src/r3d/mvs/multi_stereo.cpp:44-72) at positions (u, v)."""
    d = _c(disp, np.float32)
    u = np.ascontiguousarray(np.atleast_1d(u), np.float64)
    v = np.ascontiguousarray(np.atleast_1d(v), np.float64)
    out = np.empty(u.shape, np.float32)
    _check(lib().orc_sample_disparity(_ptr(d), d.shape[1], d.shape[0], _ptr(u), _ptr(v), u.size, _ptr(out)))
    return out


def distort_pixel(camera: dict, pixels) -> np.ndarray:
    """CameraIntrinsics::distort_pixel (src/r3d/core/camera_model.cpp:142-146)
    of an (n, 2) array of pixels."""
    from regard3d_mvs_b200.types import camera_struct

    cam = camera_struct(camera)
    p = np.ascontiguousarray(np.reshape(pixels, (-1, 2)), np.float64)
    out = np.empty_like(p)
    _check(lib().orc_distort_pixel(ctypes.byref(cam), _ptr(p), len(p), _ptr(out)))
    return out


# ------------------------------------------------------------------ depth-map consistency
# src/r3d/mvs/consistency.cpp:57-485 on host maps (dicts as in
# regard3d_mvs_b200.depth_maps); depth and support are updated in place.
def _mvs_check(rc: int) -> None:
    if rc != 0:
        raise OracleError(lib().orc_mvs_last_error().decode())


def _host_maps(maps):
    from regard3d_mvs_b200.depth_maps import CDepthMap, c_depth_map, normalise

    norm = [normalise(m) for m in maps]
    arr = (CDepthMap * max(1, len(norm)))()
    for i, n in enumerate(norm):
        arr[i] = c_depth_map(n, lambda a: a.ctypes.data)
    return norm, arr


def _back(maps, norm):
    for m, n in zip(maps, norm):
        m["depth"], m["support"] = n["depth"], n["support"]


def filter_depth_maps(maps, neighbours, options=None) -> dict:
    from regard3d_mvs_b200.depth_maps import CConsistencyStats, ConsistencyOptions, neighbour_lists

    norm, arr = _host_maps(maps)
    off, idx = neighbour_lists(neighbours)
    st = CConsistencyStats()
    o = (options or ConsistencyOptions()).c()
    _mvs_check(lib().orc_filter_depth_maps(arr, len(maps), _ptr(off), _ptr(idx), ctypes.byref(o), ctypes.byref(st)))
    _back(maps, norm)
    return st.as_dict()


def prepare_depth_map(m, options=None) -> dict:
    from regard3d_mvs_b200.depth_maps import CConsistencyStats, ConsistencyOptions

    norm, arr = _host_maps([m])
    st = CConsistencyStats()
    o = (options or ConsistencyOptions()).c()
    _mvs_check(lib().orc_prepare_depth_map(ctypes.byref(arr[0]), ctypes.byref(o), ctypes.byref(st)))
    _back([m], norm)
    return st.as_dict()


def check_consistency(m, neighbours, options=None) -> dict:
    from regard3d_mvs_b200.depth_maps import CConsistencyStats, ConsistencyOptions

    norm, arr = _host_maps([m])
    nnorm, nbs = _host_maps(neighbours)
    st = CConsistencyStats()
    o = (options or ConsistencyOptions()).c()
    _mvs_check(lib().orc_check_consistency(ctypes.byref(arr[0]), nbs, len(neighbours), ctypes.byref(o),
                                           ctypes.byref(st)))
    del nnorm
    _back([m], norm)
    return st.as_dict()


def make_refinement_image(gray: np.ndarray, blur_sigma: float = 0.0) -> np.ndarray:
    """make_refinement_image (src/r3d/mvs/refinement.cpp:242-269): H x W x 3."""
    g = _c(gray, np.float32)
    h, w = g.shape
    out = np.empty((h, w, 3), np.float32)
    _mvs_check(lib().orc_make_refinement_image(_ptr(g), w, h, blur_sigma, _ptr(out)))
    return out


def refine_depth_map(m, base, views, options=None) -> dict:
    """refine_depth_map (src/r3d/mvs/refinement.cpp:271-449) in double
    precision; m["depth"] and m["confidence"] are updated in place."""
    from regard3d_mvs_b200.depth_maps import (CRefinementImage, CRefinementStats, RefinementOptions, c_camera,
                                              c_refinement_image)

    depth = np.ascontiguousarray(m["depth"], np.float32)
    conf = np.ascontiguousarray(m["confidence"], np.float32) if m.get("confidence") is not None \
        else np.zeros_like(depth)
    h, w = depth.shape
    host = lambda a: a.ctypes.data  # noqa: E731
    bdata = np.ascontiguousarray(base["data"], np.float32)
    cb = c_refinement_image({"camera": base["camera"], "data": bdata}, host)
    vdata = [np.ascontiguousarray(v["data"], np.float32) for v in views]
    cv = (CRefinementImage * max(1, len(views)))()
    for i, (v, d) in enumerate(zip(views, vdata)):
        cv[i] = c_refinement_image({"camera": v["camera"], "data": d}, host)
    cam = c_camera(m["camera"])
    st = CRefinementStats()
    o = (options or RefinementOptions()).c()
    _mvs_check(lib().orc_refine_depth_map(_ptr(depth), _ptr(conf), w, ctypes.byref(cam), w, h, ctypes.byref(cb), cv,
                                          len(views), ctypes.byref(o), ctypes.byref(st)))
    m["depth"], m["confidence"] = depth, conf
    return st.as_dict()


def _single(m, call) -> int:
    norm, arr = _host_maps([m])
    removed = ctypes.c_uint64(0)
    _mvs_check(call(ctypes.byref(arr[0]), ctypes.byref(removed)))
    _back([m], norm)
    return int(removed.value)


def erode_depth_edges(m, radius: int, discontinuity: float, holes: bool = False) -> int:
    return _single(m, lambda c, r: lib().orc_erode_depth_edges(c, radius, discontinuity, int(holes), r))


def remove_weak_depths(m, options) -> int:
    o = options.c()
    return _single(m, lambda c, r: lib().orc_remove_weak_depths(c, ctypes.byref(o), r))


def remove_depth_halos(m, max_px: int, colour_step: int) -> int:
    return _single(m, lambda c, r: lib().orc_remove_depth_halos(c, max_px, colour_step, r))


def remove_depth_speckles(m, min_size: int, max_relative_step: float) -> int:
    return _single(m, lambda c, r: lib().orc_remove_depth_speckles(c, min_size, max_relative_step, r))


def rectify_image(src: np.ndarray, camera: dict, source_from_target, target: dict):
    """r3d::rectify_image (src/r3d/rectify/rectification.cpp:287-350) on the
    CPU for a one-channel u16 or f32 image; returns (image, valid)."""
    from regard3d_mvs_b200.types import camera_struct, pinhole_struct

    cam, k = camera_struct(camera), pinhole_struct(target)
    is_float = src.dtype == np.float32
    img = _c(src, np.float32 if is_float else np.uint16)
    if img.shape != (cam.height, cam.width):
        raise OracleError(f"rectify_image: image is {img.shape}, camera is {cam.height}x{cam.width}")
    m = np.ascontiguousarray(source_from_target, dtype=np.float64).reshape(9)
    out = np.empty((k.height, k.width), np.float32 if is_float else np.uint16)
    valid = np.empty((k.height, k.width), np.uint8)
    _check(lib().orc_rectify_image(int(is_float), _ptr(img), ctypes.byref(cam), _ptr(m), ctypes.byref(k), _ptr(out),
                                   _ptr(valid)))
    return out, valid


def median_filter_3x3(disp: np.ndarray) -> np.ndarray:
    d = _c(disp, np.float32)
    out = np.empty_like(d)
    _check(lib().orc_median_filter_3x3(_ptr(d), d.shape[1], d.shape[0], _ptr(out)))
    return out


@dataclass
class OracleMap:
    disparity: np.ndarray
    confidence: np.ndarray
    disparity_min: int
    num_disparities: int
    levels: int
    cells: int


def match_stereo(left, right, left_valid=None, right_valid=None, disparity_min=0, num_disparities=64,
                 options=None) -> OracleMap:
    left = _c(left, np.uint16)
    right = _c(right, np.uint16)
    lv = _c(left_valid, np.uint8)
    rv = _c(right_valid, np.uint8)
    o = options_struct(options)
    h, wl = left.shape
    if right.shape[0] != h or left.size == 0 or right.size == 0:
        raise OracleError("stereo: rectified images must be non-empty with equal height")
    disp = np.empty((h, wl), np.float32)
    conf = np.empty((h, wl), np.float32)
    meta = np.zeros(3, np.int64)
    _check(lib().orc_match_stereo(_ptr(left), wl, h, _ptr(right), right.shape[1], _ptr(lv), _ptr(rv),
                                  int(disparity_min), int(num_disparities), ctypes.byref(o), _ptr(disp), _ptr(conf),
                                  _ptr(meta)))
    return OracleMap(disp, conf, int(disparity_min), int(meta[1]), int(meta[0]), int(meta[2]))


def match_tiles(left, right, left_valid=None, right_valid=None, disparity_min=0, num_disparities=64, options=None,
                ranges=None, diagonal_lr=False):
    left = _c(left, np.uint16)
    right = _c(right, np.uint16)
    lv = _c(left_valid, np.uint8)
    rv = _c(right_valid, np.uint8)
    o = options_struct(options)
    lo = num = None
    if ranges is not None:
        lo = _c(ranges[0], np.uint16)
        num = _c(ranges[1], np.uint16)
    h, wl = left.shape
    disp = np.empty((h, wl), np.float32)
    conf = np.empty((h, wl), np.float32)
    cells = ctypes.c_uint64(0)
    _check(lib().orc_match_tiles(_ptr(left), wl, h, _ptr(right), right.shape[1], _ptr(lv), _ptr(rv),
                                 int(disparity_min), int(num_disparities), ctypes.byref(o), _ptr(lo), _ptr(num),
                                 int(bool(diagonal_lr)), _ptr(disp), _ptr(conf), ctypes.byref(cells)))
    return disp, conf, int(cells.value)
