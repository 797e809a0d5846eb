"""Loads the r3dgpu C-ABI library (include/r3dgpu.h) with ctypes.

The product library is ``regard3d_mvs_b200/_lib/libr3dgpu.so``, built for
sm_100a by ``regard3d_mvs_b200/build.py``. There is no CPU fallback: if the
library is missing or no B200 is present, calls fail with an error.
"""

from __future__ import annotations

import ctypes
import os

from .types import (CCamera, CDepthGrid, CDisparityMap, CMultiStereoOptions, COptions, CPair, CPairGeometry, CPinhole, CProfile,
                    CRequest, CRequestTimes, CServerConfig, CSynthParams, CViewU8, CViewU16)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libr3dgpu.so")

STATUS = {
    0: "R3DGPU_OK",
    1: "R3DGPU_EINVAL",
    2: "R3DGPU_ECANCELLED",
    3: "R3DGPU_ENOMEM",
    4: "R3DGPU_EDEVICE",
    5: "R3DGPU_ETIMEOUT",
    6: "R3DGPU_EUNSUPPORTED",
}

# Every symbol include/r3dgpu.h and include/r3dgpu_server.h declare.
EXPORTS = (
    "r3dgpu_last_error",
    "r3dgpu_default_options",
    "r3dgpu_automatic_levels",
    "r3dgpu_set_device",
    "r3dgpu_cancel_token_create",
    "r3dgpu_cancel_token_destroy",
    "r3dgpu_cancel",
    "r3dgpu_cancel_token_reset",
    "r3dgpu_cancel_requested",
    "r3dgpu_set_cancel_token",
    "r3dgpu_match_stereo_host",
    "r3dgpu_match_stereo",
    "r3dgpu_match_stereo_batch",
    "r3dgpu_census_transform",
    "r3dgpu_pyramid_down_u16",
    "r3dgpu_sgm_cost_volume_host",
    "r3dgpu_ranges_from_coarse_host",
    "r3dgpu_remove_speckles_host",
    "r3dgpu_remove_speckles_no_alloc",
    "r3dgpu_median_filter_3x3_host",
    "r3dgpu_rectify_image_u16",
    "r3dgpu_rectify_image_f32",
    "r3dgpu_rectify_image_u16_host",
    "r3dgpu_rectify_image_f32_host",
    "r3dgpu_write_depth_map",
    "r3dgpu_read_depth_map_info",
    "r3dgpu_read_depth_map",
    "r3dgpu_default_refinement_options",
    "r3dgpu_make_refinement_image",
    "r3dgpu_refine_depth_map",
    "r3dgpu_refine_depth_map_host",
    "r3dgpu_compute_depth_map",
    "r3dgpu_depth_stage_host",
    "r3dgpu_default_consistency_options",
    "r3dgpu_prepare_depth_map",
    "r3dgpu_check_consistency",
    "r3dgpu_filter_depth_maps",
    "r3dgpu_filter_depth_maps_host",
    "r3dgpu_erode_depth_edges",
    "r3dgpu_remove_weak_depths",
    "r3dgpu_remove_depth_halos",
    "r3dgpu_remove_depth_speckles",
    "r3dgpu_default_multi_stereo_options",
    "r3dgpu_combine_pairs",
    "r3dgpu_combine_pairs_host",
    "r3dgpu_release_workspace",
    "r3dgpu_launch_count",
    "r3dgpu_profile_enable",
    "r3dgpu_profile_take",
    "r3dgpu_profile_launches",
    # include/r3dgpu_server.h
    "r3dgpu_server_create",
    "r3dgpu_server_submit",
    "r3dgpu_server_wait",
    "r3dgpu_server_pending",
    "r3dgpu_server_destroy",
)


class StereoError(RuntimeError):
    """r3d::Error counterpart: carries the library's status name."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class NativeLibraryMissing(RuntimeError):
    pass


def _declare(L: ctypes.CDLL) -> ctypes.CDLL:
    P = ctypes.c_void_p
    i32 = ctypes.c_int32
    st = ctypes.c_int
    L.r3dgpu_last_error.restype = ctypes.c_char_p
    L.r3dgpu_default_options.argtypes = [ctypes.POINTER(COptions)]
    L.r3dgpu_default_options.restype = None
    L.r3dgpu_automatic_levels.argtypes = [i32, i32, i32]
    L.r3dgpu_automatic_levels.restype = i32
    L.r3dgpu_set_device.argtypes = [i32]
    L.r3dgpu_set_device.restype = st
    L.r3dgpu_cancel_token_create.argtypes = [ctypes.POINTER(P)]
    L.r3dgpu_cancel_token_create.restype = st
    for name in ("r3dgpu_cancel_token_destroy", "r3dgpu_cancel", "r3dgpu_cancel_token_reset",
                 "r3dgpu_set_cancel_token"):
        getattr(L, name).argtypes = [P]
        getattr(L, name).restype = None
    L.r3dgpu_cancel_requested.argtypes = [P]
    L.r3dgpu_cancel_requested.restype = i32
    L.r3dgpu_match_stereo_host.argtypes = [ctypes.POINTER(CViewU16), ctypes.POINTER(CViewU16),
                                           ctypes.POINTER(CViewU8), ctypes.POINTER(CViewU8), i32, i32,
                                           ctypes.POINTER(COptions), ctypes.POINTER(CDisparityMap)]
    L.r3dgpu_match_stereo_host.restype = st
    L.r3dgpu_match_stereo.argtypes = [ctypes.POINTER(CViewU16), ctypes.POINTER(CViewU16), ctypes.POINTER(CViewU8),
                                      ctypes.POINTER(CViewU8), i32, i32, ctypes.POINTER(COptions),
                                      ctypes.POINTER(CDisparityMap), P]
    L.r3dgpu_match_stereo.restype = st
    L.r3dgpu_match_stereo_batch.argtypes = [ctypes.POINTER(CPair), i32, P]
    L.r3dgpu_match_stereo_batch.restype = st
    L.r3dgpu_census_transform.argtypes = [ctypes.POINTER(CViewU16), P, ctypes.c_int64, P]
    L.r3dgpu_census_transform.restype = st
    L.r3dgpu_pyramid_down_u16.argtypes = [ctypes.POINTER(CViewU16), P, ctypes.c_int64, P]
    L.r3dgpu_pyramid_down_u16.restype = st
    L.r3dgpu_sgm_cost_volume_host.argtypes = [ctypes.POINTER(CViewU16), ctypes.POINTER(CViewU16), i32, i32,
                                              ctypes.POINTER(COptions), P, P, P, ctypes.c_uint64,
                                              ctypes.POINTER(ctypes.c_uint64)]
    L.r3dgpu_sgm_cost_volume_host.restype = st
    L.r3dgpu_ranges_from_coarse_host.argtypes = [P, i32, i32, i32, i32, P, P, i32, i32, i32, i32,
                                                 ctypes.POINTER(COptions), i32, P, P]
    L.r3dgpu_ranges_from_coarse_host.restype = st
    L.r3dgpu_remove_speckles_host.argtypes = [P, i32, i32, i32, ctypes.c_float]
    L.r3dgpu_remove_speckles_host.restype = st
    L.r3dgpu_remove_speckles_no_alloc.argtypes = [P, i32, i32, i32, ctypes.c_float, P]
    L.r3dgpu_remove_speckles_no_alloc.restype = st
    L.r3dgpu_median_filter_3x3_host.argtypes = [P, i32, i32, P]
    L.r3dgpu_median_filter_3x3_host.restype = st
    cam, pin, i64 = ctypes.POINTER(CCamera), ctypes.POINTER(CPinhole), ctypes.c_int64
    L.r3dgpu_rectify_image_u16.argtypes = [ctypes.POINTER(CViewU16), cam, P, pin, P, i64, P, i64, P]
    L.r3dgpu_rectify_image_f32.argtypes = [P, i64, cam, P, pin, P, i64, P, i64, P]
    L.r3dgpu_rectify_image_u16_host.argtypes = [ctypes.POINTER(CViewU16), cam, P, pin, P, i64, P, i64]
    L.r3dgpu_rectify_image_f32_host.argtypes = [P, i64, cam, P, pin, P, i64, P, i64]
    for name in ("r3dgpu_rectify_image_u16", "r3dgpu_rectify_image_f32", "r3dgpu_rectify_image_u16_host",
                 "r3dgpu_rectify_image_f32_host"):
        getattr(L, name).restype = st
    from .depth_maps import CConsistencyOptions, CConsistencyStats, CDepthMap

    dm, co, cs, u64p = (ctypes.POINTER(CDepthMap), ctypes.POINTER(CConsistencyOptions),
                        ctypes.POINTER(CConsistencyStats), ctypes.POINTER(ctypes.c_uint64))
    L.r3dgpu_default_consistency_options.argtypes = [co]
    L.r3dgpu_default_consistency_options.restype = None
    L.r3dgpu_prepare_depth_map.argtypes = [dm, co, cs, P]
    L.r3dgpu_check_consistency.argtypes = [dm, dm, i32, co, cs, P]
    L.r3dgpu_filter_depth_maps.argtypes = [dm, i32, P, P, co, cs, P]
    L.r3dgpu_filter_depth_maps_host.argtypes = [dm, i32, P, P, co, cs]
    L.r3dgpu_erode_depth_edges.argtypes = [dm, i32, ctypes.c_double, i32, u64p, P]
    L.r3dgpu_remove_weak_depths.argtypes = [dm, co, u64p, P]
    L.r3dgpu_remove_depth_halos.argtypes = [dm, i32, i32, u64p, P]
    L.r3dgpu_remove_depth_speckles.argtypes = [dm, i32, ctypes.c_double, u64p, P]
    from .depth_maps import CPinholeCamera, CRefinementImage, CRefinementOptions, CRefinementStats

    ro, ri, rs = (ctypes.POINTER(CRefinementOptions), ctypes.POINTER(CRefinementImage),
                  ctypes.POINTER(CRefinementStats))
    L.r3dgpu_default_refinement_options.argtypes = [ro]
    L.r3dgpu_default_refinement_options.restype = None
    L.r3dgpu_make_refinement_image.argtypes = [P, ctypes.c_int64, i32, i32, ctypes.c_double, P, ctypes.c_int64, P]
    L.r3dgpu_refine_depth_map.argtypes = [P, P, ctypes.c_int64, ctypes.POINTER(CPinholeCamera), i32, i32, ri, ri,
                                          i32, ro, rs, P]
    L.r3dgpu_refine_depth_map_host.argtypes = [P, P, ctypes.c_int64, ctypes.POINTER(CPinholeCamera), i32, i32, ri,
                                               ri, i32, ro, rs]
    from .multi_view import CViewPair

    L.r3dgpu_compute_depth_map.argtypes = [ctypes.POINTER(CViewU16), ctypes.POINTER(CCamera),
                                           ctypes.POINTER(CDepthGrid), ctypes.POINTER(CViewPair), i32,
                                           ctypes.POINTER(COptions), ctypes.POINTER(CMultiStereoOptions), P, P, P,
                                           ctypes.c_int64, ctypes.POINTER(ctypes.c_uint64), P]
    L.r3dgpu_compute_depth_map.restype = st
    L.r3dgpu_depth_stage_host.argtypes = [dm, ri, i32, P, P, ro, co, rs, cs]
    L.r3dgpu_depth_stage_host.restype = st
    L.r3dgpu_write_depth_map.argtypes = [ctypes.c_char_p, dm, i32, P]
    L.r3dgpu_read_depth_map_info.argtypes = [ctypes.c_char_p, dm]
    L.r3dgpu_read_depth_map.argtypes = [ctypes.c_char_p, dm]
    for name in ("r3dgpu_write_depth_map", "r3dgpu_read_depth_map_info", "r3dgpu_read_depth_map"):
        getattr(L, name).restype = st
    for name in ("r3dgpu_make_refinement_image", "r3dgpu_refine_depth_map", "r3dgpu_refine_depth_map_host"):
        getattr(L, name).restype = st
    for name in ("r3dgpu_prepare_depth_map", "r3dgpu_check_consistency", "r3dgpu_filter_depth_maps",
                 "r3dgpu_filter_depth_maps_host", "r3dgpu_erode_depth_edges", "r3dgpu_remove_weak_depths",
                 "r3dgpu_remove_depth_halos", "r3dgpu_remove_depth_speckles"):
        getattr(L, name).restype = st
    L.r3dgpu_default_multi_stereo_options.argtypes = [ctypes.POINTER(CMultiStereoOptions)]
    L.r3dgpu_default_multi_stereo_options.restype = None
    for name in ("r3dgpu_combine_pairs", "r3dgpu_combine_pairs_host"):
        f = getattr(L, name)
        f.argtypes = [ctypes.POINTER(CDepthGrid), ctypes.POINTER(CPairGeometry), i32,
                      ctypes.POINTER(CMultiStereoOptions), P, P, P, ctypes.c_int64] + ([P] if name == "r3dgpu_combine_pairs" else [])
        f.restype = st
    L.r3dgpu_release_workspace.argtypes = []
    L.r3dgpu_release_workspace.restype = st
    L.r3dgpu_launch_count.argtypes = []
    L.r3dgpu_launch_count.restype = ctypes.c_uint64
    L.r3dgpu_profile_enable.argtypes = [i32]
    L.r3dgpu_profile_enable.restype = None
    L.r3dgpu_profile_take.argtypes = [ctypes.POINTER(CProfile)]
    L.r3dgpu_profile_take.restype = None
    L.r3dgpu_profile_launches.argtypes = [ctypes.c_char_p, ctypes.c_uint64]
    L.r3dgpu_profile_launches.restype = ctypes.c_uint64
    # The request struct has the layout of r3dgpu_pair.
    L.r3dgpu_server_create.argtypes = [ctypes.POINTER(CServerConfig), ctypes.POINTER(P)]
    L.r3dgpu_server_create.restype = st
    L.r3dgpu_server_submit.argtypes = [P, ctypes.POINTER(CRequest), ctypes.POINTER(ctypes.c_uint64)]
    L.r3dgpu_server_submit.restype = st
    L.r3dgpu_server_wait.argtypes = [P, ctypes.c_uint64, ctypes.c_double, ctypes.POINTER(CRequest),
                                     ctypes.POINTER(CRequestTimes)]
    L.r3dgpu_server_wait.restype = st
    L.r3dgpu_server_pending.argtypes = [P]
    L.r3dgpu_server_pending.restype = i32
    L.r3dgpu_server_destroy.argtypes = [P]
    L.r3dgpu_server_destroy.restype = st
    if hasattr(L, "r3dgpu_synth_pair"):
        L.r3dgpu_synth_pair.argtypes = [ctypes.POINTER(CSynthParams), P, P, P]
        L.r3dgpu_synth_pair.restype = st
    return L


_cache: dict[str, ctypes.CDLL] = {}


def load(path: str | None = None) -> ctypes.CDLL:
    """The library at `path` (default: the in-tree CUDA build)."""
    path = os.path.abspath(path or LIB_PATH)
    if path not in _cache:
        if not os.path.exists(path):
            raise NativeLibraryMissing(
                f"r3dgpu CUDA library not found at {path}; build it with "
                "`python -m regard3d_mvs_b200.build` (nvcc, sm_100a)")
        _cache[path] = _declare(ctypes.CDLL(path))
    return _cache[path]


def check(lib: ctypes.CDLL, status: int) -> None:
    if status != 0:
        raise StereoError(status, lib.r3dgpu_last_error().decode())
