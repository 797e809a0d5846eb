"""Python mirror of the reference matcher interface over the r3dgpu C ABI.

Function names, arguments and error behaviour follow r3d::match_stereo and
its companions (rhiestan/Regard3D_MVS, src/r3d/stereo/stereo_matcher.hpp:82-128,
census.hpp:20, core/pyramid.hpp:21): invalid options or sizes raise
``StereoError`` (r3d::Error). Images are 2-D numpy arrays (uint16 grey, uint8
masks with 255 = valid); 8-bit images must be lifted with ``lift_u8`` (x257,
as the reference's image reader does, src/r3d/io/image_io.hpp:25-26).

All computation runs in the CUDA library; ``Matcher(lib_path=...)`` can bind a
different build of the same C ABI (the tests use that for the CPU emulator of
the kernels).
"""

from __future__ import annotations

import ctypes
from typing import Iterable, Sequence

import numpy as np

from . import _native
from .types import (CDisparityMap, COptions, CPair, CRequest, CRequestTimes, CServerConfig, CViewU8, CViewU16, DisparityMap,
                    LabelRanges, StereoOptions, to_c_options)


def lift_u8(img: np.ndarray) -> np.ndarray:
    """8-bit grey -> 16-bit (v * 257), the reference's rule for 8-bit files."""
    return img.astype(np.uint16) * np.uint16(257)


def _u16(a: np.ndarray) -> np.ndarray:
    a = np.asarray(a)
    if a.ndim != 2:
        raise _native.StereoError(1, "stereo: expected a single-channel image")
    return np.ascontiguousarray(a, dtype=np.uint16)


def _view16(a: np.ndarray | None) -> CViewU16:
    v = CViewU16()
    if a is not None and a.size:
        v.data = a.ctypes.data
        v.height, v.width = a.shape
        v.stride = a.strides[0] // a.itemsize
    return v


def _view8(a: np.ndarray | None) -> CViewU8:
    v = CViewU8()
    if a is not None and a.size:
        v.data = a.ctypes.data
        v.height, v.width = a.shape
        v.stride = a.strides[0] // a.itemsize
    return v


def _opts(options: StereoOptions | None) -> COptions:
    return to_c_options(options if options is not None else StereoOptions())


class Matcher:
    """Binds the matcher functions to one build of the C ABI and one device."""

    def __init__(self, lib_path: str | None = None, device: int = 0, host_is_device: bool = False):
        self.lib = _native.load(lib_path)
        self.device = device
        # True for builds whose "device" memory is host memory (the emulator).
        self.host_is_device = host_is_device
        _native.check(self.lib, self.lib.r3dgpu_set_device(device))

    def _check(self, status: int) -> None:
        _native.check(self.lib, status)

    # ---------------------------------------------------------------- r3d::match_stereo
    def match_stereo(self, left, right, left_valid=None, right_valid=None, disparity_min: int = 0,
                     num_disparities: int = 64, options: StereoOptions | None = None) -> DisparityMap:
        L, R = _u16(left), _u16(right)
        lv = None if left_valid is None else np.ascontiguousarray(left_valid, dtype=np.uint8)
        rv = None if right_valid is None else np.ascontiguousarray(right_valid, dtype=np.uint8)
        h, w = L.shape
        disp = np.empty((h, w), np.float32)
        conf = np.empty((h, w), np.float32)
        out = CDisparityMap()
        out.disparity = disp.ctypes.data
        out.confidence = conf.ctypes.data
        out.stride = w
        o = _opts(options)
        self._check(self.lib.r3dgpu_match_stereo_host(ctypes.byref(_view16(L)), ctypes.byref(_view16(R)),
                                                      ctypes.byref(_view8(lv)), ctypes.byref(_view8(rv)),
                                                      int(disparity_min), int(num_disparities), ctypes.byref(o),
                                                      ctypes.byref(out)))
        return DisparityMap(disp, conf, out.disparity_min, out.num_disparities, out.levels, int(out.cells))

    # ---------------------------------------------------------------- r3d::combine_pairs
    def combine_pairs(self, grid: dict, pairs: list[dict], options=None):
        """Depth map of the grid camera from matched pairs that share its
        centre (see regard3d_mvs_b200.multi_view for the dicts)."""
        from .multi_view import c_grid, c_pairs
        from .types import DepthMap, MultiStereoOptions

        g = c_grid(grid)
        arr, keep = c_pairs(grid, pairs)
        o = (options or MultiStereoOptions()).c()
        depth = np.empty((g.height, g.width), np.float32)
        conf = np.empty_like(depth)
        mask = np.empty((g.height, g.width), np.uint16)
        self._check(self.lib.r3dgpu_combine_pairs_host(ctypes.byref(g), arr, len(pairs), ctypes.byref(o),
                                                       depth.ctypes.data, conf.ctypes.data, mask.ctypes.data,
                                                       g.width))
        del keep
        return DepthMap(depth, conf, mask)

    def depth_stage(self, maps: list[dict], images: Sequence[dict], neighbours: Sequence[Sequence[int]],
                    refine=None, consistency=None) -> tuple[dict, dict]:
        """r3dgpu_depth_stage_host: each view refined against its neighbours'
        refinement images ({camera, data}), then the consistency filter of
        all maps over the same neighbour lists; maps' depth, confidence and
        support are updated in place. Returns (refinement, consistency) statistics."""
        from .depth_maps import (CConsistencyStats, CDepthMap, ConsistencyOptions, CRefinementImage,
                                 CRefinementStats, RefinementOptions, c_depth_map, c_refinement_image,
                                 neighbour_lists, normalise)

        norm = [normalise(m) for m in maps]
        arr = (CDepthMap * max(1, len(norm)))()
        for i, n in enumerate(norm):
            arr[i] = c_depth_map(n, lambda a: a.ctypes.data)
        data = [np.ascontiguousarray(im["data"], np.float32) for im in images]
        imgs = (CRefinementImage * max(1, len(images)))()
        for i, (im, d) in enumerate(zip(images, data)):
            imgs[i] = c_refinement_image({"camera": im["camera"], "data": d}, lambda a: a.ctypes.data)
        off, idx = neighbour_lists(neighbours)
        rst, cst = CRefinementStats(), CConsistencyStats()
        ro = (refine or RefinementOptions()).c()
        co = (consistency or ConsistencyOptions()).c()
        self._check(self.lib.r3dgpu_depth_stage_host(arr, imgs, len(maps), off.ctypes.data, idx.ctypes.data,
                                                     ctypes.byref(ro), ctypes.byref(co), ctypes.byref(rst),
                                                     ctypes.byref(cst)))
        for m, n in zip(maps, norm):
            m["depth"], m["confidence"], m["support"] = n["depth"], n["confidence"], n["support"]
        return rst.as_dict(), cst.as_dict()

    # ---------------------------------------------------------------- a view's depth map
    def compute_depth_map(self, base: np.ndarray, grid: dict, pairs: list[dict], stereo: StereoOptions | None = None,
                          multi=None):
        """r3dgpu_compute_depth_map: rectification, batch matching and
        combination of a view's pairs on the device. `grid` as for
        combine_pairs (pinhole K, R, C, size; also the base camera); each pair
        carries its partner image ("image"), the partner's rotation
        ("R_partner"), the rectification ("R_rect", "K_rect", "baseline",
        "cx_right", "centre", "left" and "right" pinholes) and its disparity
        range. Returns (DepthMap, matched cells)."""
        from .multi_view import CViewPair, c_grid, pair_geometry
        from .types import DepthMap, MultiStereoOptions, camera_struct, pinhole_struct

        keep: list = []
        b = _u16(base)
        h, w = b.shape
        K = np.asarray(grid["K"], np.float64)
        cam = {"model": 0, "width": w, "height": h, "fx": K[0, 0], "fy": K[1, 1], "cx": K[0, 2], "cy": K[1, 2]}
        cb = camera_struct(cam)
        vb = CViewU16(self._to_device(b, keep), w, h, w)
        arr = (CViewPair * max(1, len(pairs)))()
        R_base = np.asarray(grid["R"], np.float64)
        for i, p in enumerate(pairs):
            q = arr[i]
            img = _u16(p["image"])
            ph, pw = img.shape
            q.partner = CViewU16(self._to_device(img, keep), pw, ph, pw)
            q.partner_camera = camera_struct(dict(cam, width=pw, height=ph))
            R_rect = np.asarray(p["R_rect"], np.float64)
            q.base_from_rect[:] = [float(v) for v in (R_base @ R_rect.T).ravel()]
            q.partner_from_rect[:] = [float(v) for v in (np.asarray(p["R_partner"], np.float64) @ R_rect.T).ravel()]
            q.left, q.right = pinhole_struct(p["left"]), pinhole_struct(p["right"])
            q.disparity_min, q.num_disparities = int(p["disparity_min"]), int(p["num_disparities"])
            q.geometry = pair_geometry(grid, p)
        g = c_grid(grid)
        gh, gw = g.height, g.width
        dp, dobj = self._empty_device((gh, gw), keep)
        cp, cobj = self._empty_device((gh, gw), keep)
        mp, mobj = self._empty_device((gh, gw), keep)  # float32-sized buffer holds the u16 mask
        o = _opts(stereo)
        mo = (multi or MultiStereoOptions()).c()
        cells = ctypes.c_uint64(0)
        self._check(self.lib.r3dgpu_compute_depth_map(ctypes.byref(vb), ctypes.byref(cb), ctypes.byref(g), arr,
                                                      len(pairs), ctypes.byref(o), ctypes.byref(mo), dp, cp, mp, gw,
                                                      ctypes.byref(cells), None))
        depth = self._to_host((dp, dobj), (gh, gw))
        conf = self._to_host((cp, cobj), (gh, gw))
        # The u16 mask is dense (gw per row) in the first half of its float-sized buffer.
        mask = np.ascontiguousarray(self._to_host((mp, mobj), (gh, gw))).reshape(-1).view(np.uint16)[:gh * gw]
        mask = mask.reshape(gh, gw)
        return DepthMap(depth.copy(), conf.copy(), mask.copy()), int(cells.value)

    # ---------------------------------------------------------------- r3d::rectify_image
    def rectify_image(self, src: np.ndarray, camera: dict, source_from_target, target: dict):
        """Resamples a one-channel u16 or f32 image of `camera` ({model, width,
        height, fx, fy, cx, cy, params}) into the pinhole camera `target`
        ({width, height, fx, fy, cx, cy}) rotated by R_source R_target^T =
        `source_from_target` about the same centre; returns (image, valid)
        with valid 255 where the target pixel sees the source.
        r3d::rectify_image, src/r3d/rectify/rectification.hpp:75-88."""
        from .types import camera_struct, pinhole_struct

        cam, k = camera_struct(camera), pinhole_struct(target)
        m = np.ascontiguousarray(source_from_target, dtype=np.float64).reshape(9)
        valid = np.empty((k.height, k.width), np.uint8)
        if src.dtype == np.float32:
            img = np.ascontiguousarray(src)
            if img.ndim != 2 or img.shape != (cam.height, cam.width):
                raise _native.StereoError(1, f"rectify_image: image is {img.shape}, camera is "
                                             f"{cam.height}x{cam.width}")
            out = np.empty((k.height, k.width), np.float32)
            st = self.lib.r3dgpu_rectify_image_f32_host(img.ctypes.data, img.shape[1],
                                                         ctypes.byref(cam), m.ctypes.data, ctypes.byref(k),
                                                         out.ctypes.data, k.width, valid.ctypes.data, k.width)
        else:
            img = _u16(src)
            out = np.empty((k.height, k.width), np.uint16)
            view = CViewU16(img.ctypes.data, img.shape[1], img.shape[0], img.shape[1])
            st = self.lib.r3dgpu_rectify_image_u16_host(ctypes.byref(view), ctypes.byref(cam), m.ctypes.data,
                                                         ctypes.byref(k), out.ctypes.data, k.width,
                                                         valid.ctypes.data, k.width)
        self._check(st)
        return out, valid

    # ---------------------------------------------------------------- depth-map consistency
    # src/r3d/mvs/consistency.hpp:97-125. Maps are dicts (regard3d_mvs_b200.depth_maps);
    # their depth and support arrays are updated in place.
    def _device_maps(self, maps: Sequence[dict], keep: list):
        from .depth_maps import CDepthMap, c_depth_map, normalise

        norm = [normalise(m) for m in maps]
        dev: dict[int, object] = {}

        def ptr(a):
            p = self._to_device(a, keep)
            dev[id(a)] = keep[-1]
            return p

        arr = (CDepthMap * max(1, len(norm)))()
        for i, n in enumerate(norm):
            arr[i] = c_depth_map(n, ptr)
        return norm, arr, dev

    def _maps_back(self, maps: Sequence[dict], norm: list, dev: dict) -> None:
        for m, n in zip(maps, norm):
            if not self.host_is_device:
                n["depth"][...] = dev[id(n["depth"])].cpu().numpy()
                n["support"][...] = dev[id(n["support"])].cpu().numpy()
            m["depth"], m["support"] = n["depth"], n["support"]

    def _single(self, m: dict, call) -> int:
        keep: list = []
        norm, arr, dev = self._device_maps([m], keep)
        removed = ctypes.c_uint64(0)
        self._check(call(ctypes.byref(arr[0]), ctypes.byref(removed)))
        self._maps_back([m], norm, dev)
        return int(removed.value)

    def prepare_depth_map(self, m: dict, options=None) -> dict:
        from .depth_maps import CConsistencyStats, ConsistencyOptions

        keep: list = []
        norm, arr, dev = self._device_maps([m], keep)
        st = CConsistencyStats()
        o = (options or ConsistencyOptions()).c()
        self._check(self.lib.r3dgpu_prepare_depth_map(ctypes.byref(arr[0]), ctypes.byref(o), ctypes.byref(st), None))
        self._maps_back([m], norm, dev)
        return st.as_dict()

    def check_consistency(self, m: dict, neighbours: Sequence[dict], options=None) -> dict:
        from .depth_maps import CConsistencyStats, ConsistencyOptions

        keep: list = []
        norm, arr, dev = self._device_maps([m], keep)
        _, nbs, _ = self._device_maps(neighbours, keep)
        st = CConsistencyStats()
        o = (options or ConsistencyOptions()).c()
        self._check(self.lib.r3dgpu_check_consistency(ctypes.byref(arr[0]), nbs, len(neighbours), ctypes.byref(o),
                                                      ctypes.byref(st), None))
        self._maps_back([m], norm, dev)
        return st.as_dict()

    def filter_depth_maps(self, maps: list[dict], neighbours: Sequence[Sequence[int]], options=None) -> dict:
        """filter_depth_maps through the host entry point (copies inside)."""
        from .depth_maps import CConsistencyStats, CDepthMap, ConsistencyOptions, c_depth_map, neighbour_lists, normalise

        norm = [normalise(m) for m in maps]
        arr = (CDepthMap * max(1, len(norm)))()
        for i, n in enumerate(norm):
            arr[i] = c_depth_map(n, lambda a: a.ctypes.data)
        off, idx = neighbour_lists(neighbours)
        st = CConsistencyStats()
        o = (options or ConsistencyOptions()).c()
        self._check(self.lib.r3dgpu_filter_depth_maps_host(arr, len(maps), off.ctypes.data, idx.ctypes.data,
                                                           ctypes.byref(o), ctypes.byref(st)))
        for m, n in zip(maps, norm):
            m["depth"], m["support"] = n["depth"], n["support"]
        return st.as_dict()

    def erode_depth_edges(self, m: dict, radius: int, discontinuity: float, holes: bool = False) -> int:
        return self._single(m, lambda c, r: self.lib.r3dgpu_erode_depth_edges(c, radius, discontinuity, int(holes),
                                                                              r, None))

    def remove_weak_depths(self, m: dict, options) -> int:
        o = options.c()
        return self._single(m, lambda c, r: self.lib.r3dgpu_remove_weak_depths(c, ctypes.byref(o), r, None))

    def remove_depth_halos(self, m: dict, max_px: int, colour_step: int) -> int:
        return self._single(m, lambda c, r: self.lib.r3dgpu_remove_depth_halos(c, max_px, colour_step, r, None))

    def remove_depth_speckles(self, m: dict, min_size: int, max_relative_step: float) -> int:
        return self._single(m, lambda c, r: self.lib.r3dgpu_remove_depth_speckles(c, min_size, max_relative_step, r,
                                                                                  None))

    # ---------------------------------------------------------------- depth refinement
    # src/r3d/mvs/refinement.hpp:53-68.
    def make_refinement_image(self, gray: np.ndarray, blur_sigma: float = 0.0) -> np.ndarray:
        """Intensity and x / y derivatives (H x W x 3 float32) of a float image."""
        g = np.ascontiguousarray(gray, np.float32)
        h, w = g.shape
        keep: list = []
        dg = self._to_device(g, keep)
        ptr, obj = self._empty_device((h, w, 3), keep)
        self._check(self.lib.r3dgpu_make_refinement_image(dg, w, w, h, blur_sigma, ptr, 3 * w, None))
        return self._to_host((ptr, obj), (h, w, 3))

    def refine_depth_map(self, m: dict, base: dict, views: Sequence[dict], options=None) -> dict:
        """Refines m["depth"] and m["confidence"] in place (host entry point).
        base and views: {camera, data (H x W x 3 float32 refinement image)}."""
        from .depth_maps import (CRefinementImage, CRefinementStats, RefinementOptions, c_camera,
                                 c_refinement_image)

        depth = np.ascontiguousarray(m["depth"], np.float32)
        conf = np.ascontiguousarray(m["confidence"], np.float32) if m.get("confidence") is not None \
            else np.zeros_like(depth)
        h, w = depth.shape
        host = lambda a: a.ctypes.data  # noqa: E731
        cb = c_refinement_image({"camera": base["camera"], "data": np.ascontiguousarray(base["data"], np.float32)},
                                host)
        vdata = [np.ascontiguousarray(v["data"], np.float32) for v in views]
        cv = (CRefinementImage * max(1, len(views)))()
        for i, (v, d) in enumerate(zip(views, vdata)):
            cv[i] = c_refinement_image({"camera": v["camera"], "data": d}, host)
        cam = c_camera(m["camera"])
        st = CRefinementStats()
        o = (options or RefinementOptions()).c()
        self._check(self.lib.r3dgpu_refine_depth_map_host(depth.ctypes.data, conf.ctypes.data, w, ctypes.byref(cam), w,
                                                          h, ctypes.byref(cb), cv, len(views), ctypes.byref(o),
                                                          ctypes.byref(st)))
        m["depth"], m["confidence"] = depth, conf
        return st.as_dict()

    # ---------------------------------------------------------------- batched matching
    def match_stereo_batch(self, pairs: Sequence[dict], stream: int | None = None) -> list[DisparityMap]:
        """Matches many pairs in one pass of every stage.

        Each pair is a dict with keys left, right, (left_valid, right_valid,)
        disparity_min, num_disparities, (options). Host arrays are copied to the
        device (through torch on a GPU build) and results copied back.
        """
        keep = []
        cp = (CPair * len(pairs))()
        outs = []
        for i, p in enumerate(pairs):
            L, R = _u16(p["left"]), _u16(p["right"])
            lv = p.get("left_valid")
            rv = p.get("right_valid")
            lv = None if lv is None else np.ascontiguousarray(lv, dtype=np.uint8)
            rv = None if rv is None else np.ascontiguousarray(rv, dtype=np.uint8)
            h, w = L.shape
            dL, dR, dlv, drv = (self._to_device(a, keep) for a in (L, R, lv, rv))
            disp, conf = self._empty_device((h, w), keep), self._empty_device((h, w), keep)
            c = cp[i]
            c.left = CViewU16(dL, w, h, w)
            c.right = CViewU16(dR, R.shape[1], h, R.shape[1])
            c.left_valid = CViewU8(dlv, w, h, w) if lv is not None else CViewU8()
            c.right_valid = CViewU8(drv, R.shape[1], h, R.shape[1]) if rv is not None else CViewU8()
            c.disparity_min = int(p.get("disparity_min", 0))
            c.num_disparities = int(p["num_disparities"])
            c.options = _opts(p.get("options"))
            c.out.disparity = disp[0]
            c.out.confidence = conf[0]
            c.out.stride = w
            outs.append((disp, conf, (h, w)))
        self._check(self.lib.r3dgpu_match_stereo_batch(cp, len(pairs), stream))
        res = []
        for i, (disp, conf, shape) in enumerate(outs):
            res.append(DisparityMap(self._to_host(disp, shape), self._to_host(conf, shape), cp[i].out.disparity_min,
                                    cp[i].out.num_disparities, cp[i].out.levels, int(cp[i].out.cells)))
        return res

    def _to_device(self, a: np.ndarray | None, keep: list):
        if a is None:
            return None
        if self.host_is_device:
            keep.append(a)
            return a.ctypes.data
        import torch

        t = torch.from_numpy(a.view(np.int16) if a.dtype == np.uint16 else a).to(f"cuda:{self.device}")
        keep.append(t)
        return t.data_ptr()

    def _empty_device(self, shape, keep: list):
        if self.host_is_device:
            a = np.empty(shape, np.float32)
            keep.append(a)
            return (a.ctypes.data, a)
        import torch

        t = torch.empty(shape, dtype=torch.float32, device=f"cuda:{self.device}")
        keep.append(t)
        return (t.data_ptr(), t)

    def _to_host(self, d, shape) -> np.ndarray:
        obj = d[1]
        if self.host_is_device:
            return obj
        return obj.cpu().numpy()

    # ---------------------------------------------------------------- companions
    def census_transform(self, img) -> np.ndarray:
        """census.hpp:20: u64 Census code per pixel."""
        I = _u16(img)
        h, w = I.shape
        keep: list = []
        dI = self._to_device(I, keep)
        out = self._empty_u64((h, w), keep)
        v = CViewU16(dI, w, h, w)
        self._check(self.lib.r3dgpu_census_transform(ctypes.byref(v), out[0], w, None))
        return self._u64_to_host(out)

    def pyramid_down(self, img) -> np.ndarray:
        """pyramid.hpp:21: one 2x binomial reduction of a 16-bit image."""
        I = _u16(img)
        h, w = I.shape
        keep: list = []
        dI = self._to_device(I, keep)
        dh, dw = (h + 1) // 2, (w + 1) // 2
        if self.host_is_device:
            out = np.empty((dh, dw), np.uint16)
            ptr = out.ctypes.data
        else:
            import torch

            t = torch.empty((dh, dw), dtype=torch.int16, device=f"cuda:{self.device}")
            ptr = t.data_ptr()
        v = CViewU16(dI, w, h, w)
        self._check(self.lib.r3dgpu_pyramid_down_u16(ctypes.byref(v), ptr, dw, None))
        if self.host_is_device:
            return out
        return t.cpu().numpy().view(np.uint16)

    def _empty_u64(self, shape, keep):
        if self.host_is_device:
            a = np.empty(shape, np.uint64)
            keep.append(a)
            return (a.ctypes.data, a)
        import torch

        t = torch.empty(shape, dtype=torch.int64, device=f"cuda:{self.device}")
        keep.append(t)
        return (t.data_ptr(), t)

    def _u64_to_host(self, d) -> np.ndarray:
        if self.host_is_device:
            return d[1]
        return d[1].cpu().numpy().view(np.uint64)

    def sgm_cost_volume(self, left, right, disparity_min: int, num_disparities: int,
                        options: StereoOptions | None = None, ranges: LabelRanges | None = None) -> np.ndarray:
        """detail::sgm_cost_volume (stereo_matcher.hpp:98-101): the aggregated
        volume of the whole image as one tile, labels of every pixel in
        row-major pixel order."""
        L, R = _u16(left), _u16(right)
        o = _opts(options)
        lo = num = None
        if ranges is not None:
            lo = np.ascontiguousarray(ranges.lo, dtype=np.uint16)
            num = np.ascontiguousarray(ranges.num, dtype=np.uint16)
        count = ctypes.c_uint64(0)
        args = (ctypes.byref(_view16(L)), ctypes.byref(_view16(R)), int(disparity_min), int(num_disparities),
                ctypes.byref(o), None if lo is None else lo.ctypes.data, None if num is None else num.ctypes.data)
        self._check(self.lib.r3dgpu_sgm_cost_volume_host(*args, None, 0, ctypes.byref(count)))
        out = np.empty(count.value, np.uint16)
        self._check(self.lib.r3dgpu_sgm_cost_volume_host(*args, out.ctypes.data, count.value, ctypes.byref(count)))
        return out

    def ranges_from_coarse(self, coarse, width: int, height: int, fine_valid, partner_valid, partner_width: int,
                           partner_sign: int, disparity_min: int, num_disparities: int,
                           options: StereoOptions | None = None, mirrored: bool = False) -> LabelRanges:
        """detail::ranges_from_coarse (stereo_matcher.hpp:121-125)."""
        C = np.ascontiguousarray(coarse, dtype=np.float32)
        fv = None if fine_valid is None else np.ascontiguousarray(fine_valid, dtype=np.uint8)
        pv = None if partner_valid is None else np.ascontiguousarray(partner_valid, dtype=np.uint8)
        lo = np.empty((height, width), np.uint16)
        num = np.empty((height, width), np.uint16)
        o = _opts(options)
        self._check(self.lib.r3dgpu_ranges_from_coarse_host(
            C.ctypes.data, C.shape[1], C.shape[0], width, height, None if fv is None else fv.ctypes.data,
            None if pv is None else pv.ctypes.data, partner_width, partner_sign, disparity_min, num_disparities,
            ctypes.byref(o), int(bool(mirrored)), lo.ctypes.data, num.ctypes.data))
        return LabelRanges(lo, num)

    def remove_speckles(self, disparity: np.ndarray, min_size: int, max_diff: float) -> np.ndarray:
        """stereo_matcher.hpp:89 (in place on a C-contiguous float32 array; returned as well)."""
        d = disparity if (disparity.dtype == np.float32 and disparity.flags.c_contiguous) else \
            np.ascontiguousarray(disparity, dtype=np.float32)
        self._check(self.lib.r3dgpu_remove_speckles_host(d.ctypes.data, d.shape[1], d.shape[0], int(min_size),
                                                         float(max_diff)))
        return d

    def median_filter_3x3(self, disparity: np.ndarray) -> np.ndarray:
        """stereo_matcher.hpp:91"""
        d = np.ascontiguousarray(disparity, dtype=np.float32)
        out = np.empty_like(d)
        self._check(self.lib.r3dgpu_median_filter_3x3_host(d.ctypes.data, d.shape[1], d.shape[0], out.ctypes.data))
        return out

    def automatic_levels(self, width: int, height: int, num_disparities: int) -> int:
        return int(self.lib.r3dgpu_automatic_levels(width, height, num_disparities))

    def launch_count(self) -> int:
        return int(self.lib.r3dgpu_launch_count())

    def cancel_token(self) -> "CancelToken":
        """A new cancellation token (r3dgpu_cancel_token_create)."""
        return CancelToken(self.lib)

    def set_cancel_token(self, token: "CancelToken | None") -> None:
        """Attaches `token` to this thread's later calls (None detaches);
        a cancelled call raises StereoError with R3DGPU_ECANCELLED."""
        self.lib.r3dgpu_set_cancel_token(token.handle if token is not None else None)


class CancelToken:
    """The r3dgpu_cancel_token of include/r3dgpu.h (r3d::CancelToken's
    counterpart): cancel() from any thread, reset() before reuse."""

    def __init__(self, lib):
        self.lib = lib
        h = ctypes.c_void_p()
        _native.check(lib, lib.r3dgpu_cancel_token_create(ctypes.byref(h)))
        self.handle = h

    def cancel(self) -> None:
        self.lib.r3dgpu_cancel(self.handle)

    def reset(self) -> None:
        self.lib.r3dgpu_cancel_token_reset(self.handle)

    def requested(self) -> bool:
        return bool(self.lib.r3dgpu_cancel_requested(self.handle))

    def close(self) -> None:
        if self.handle:
            self.lib.r3dgpu_cancel_token_destroy(self.handle)
            self.handle = ctypes.c_void_p()


_default: Matcher | None = None


class Server:
    """The serving loop of include/r3dgpu_server.h: submit pair requests
    (host arrays) from any thread, wait on their tickets.

    Requests run in continuous batches on `workers` CUDA streams; the
    estimated device memory of the admitted requests stays within
    `hbm_budget` bytes. Each result equals Matcher.match_stereo on the same
    pair, whatever else ran beside it. With `cache_budget` > 0, images
    submitted with a content key (left_key / right_key) stay on the device
    and are uploaded once while cached.
    """

    def __init__(self, lib_path: str | None = None, device: int = 0, workers: int = 2, max_batch: int = 16,
                 hbm_budget: int = 64 << 30, scratch_budget: int = 0, cache_budget: int = 0):
        self.lib = _native.load(lib_path)
        cfg = CServerConfig(device, workers, max_batch, 0, hbm_budget, scratch_budget, cache_budget)
        h = ctypes.c_void_p()
        _native.check(self.lib, self.lib.r3dgpu_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self._live: dict[int, tuple] = {}  # ticket -> (request, host arrays it points into)

    def submit(self, left, right, left_valid=None, right_valid=None, disparity_min: int = 0,
               num_disparities: int = 64, options: StereoOptions | None = None, out=None, left_key: int = 0,
               right_key: int = 0) -> int:
        """Queues a pair. `out` = (disparity, confidence or None): caller-owned
        float32 arrays of the left image's shape (page-locked memory makes the
        copies asynchronous); by default both are allocated here. A nonzero
        key promises that every request with that key has the same image."""
        L, R = _u16(left), _u16(right)
        lv = None if left_valid is None else np.ascontiguousarray(left_valid, dtype=np.uint8)
        rv = None if right_valid is None else np.ascontiguousarray(right_valid, dtype=np.uint8)
        h, w = L.shape
        if out is None:
            disp, conf = np.empty((h, w), np.float32), np.empty((h, w), np.float32)
        else:
            disp, conf = out
            for a in (disp, conf):
                if a is not None and (a.shape != (h, w) or a.dtype != np.float32 or not a.flags.c_contiguous):
                    raise _native.StereoError(1, "server: output arrays must be contiguous float32 of the image shape")
        req = CRequest()
        req.left_key, req.right_key = int(left_key), int(right_key)
        req.left, req.right = _view16(L), _view16(R)
        req.left_valid, req.right_valid = _view8(lv), _view8(rv)
        req.disparity_min, req.num_disparities = int(disparity_min), int(num_disparities)
        req.options = _opts(options)
        req.out.disparity, req.out.stride = disp.ctypes.data, w
        req.out.confidence = conf.ctypes.data if conf is not None else None
        ticket = ctypes.c_uint64()
        _native.check(self.lib, self.lib.r3dgpu_server_submit(self._h, ctypes.byref(req), ctypes.byref(ticket)))
        self._live[ticket.value] = (req, (L, R, lv, rv, disp, conf))
        return ticket.value

    def wait(self, ticket: int, timeout_ms: float = -1.0) -> tuple[DisparityMap, dict]:
        req, arrays = self._live[ticket]
        t = CRequestTimes()
        st = self.lib.r3dgpu_server_wait(self._h, ticket, float(timeout_ms), ctypes.byref(req), ctypes.byref(t))
        if st != 5:  # R3DGPU_ETIMEOUT keeps the ticket
            del self._live[ticket]
        _native.check(self.lib, st)
        disp, conf = arrays[4], arrays[5]
        times = {"queued_ms": t.queued_ms, "run_ms": t.run_ms, "total_ms": t.total_ms,
                 "device_bytes": int(t.device_bytes), "batch_size": t.batch_size, "worker": t.worker,
                 "cache_hits": t.cache_hits, "uploaded_bytes": int(t.uploaded_bytes)}
        return DisparityMap(disp, conf, req.out.disparity_min, req.out.num_disparities, req.out.levels,
                            int(req.out.cells)), times

    def pending(self) -> int:
        return int(self.lib.r3dgpu_server_pending(self._h))

    def close(self) -> None:
        if self._h:
            _native.check(self.lib, self.lib.r3dgpu_server_destroy(self._h))
            self._h = ctypes.c_void_p()
            self._live.clear()

    def __enter__(self) -> "Server":
        return self

    def __exit__(self, *exc) -> None:
        self.close()


def default_matcher() -> Matcher:
    global _default
    if _default is None:
        _default = Matcher()
    return _default


def match_stereo(left, right, left_valid=None, right_valid=None, disparity_min: int = 0, num_disparities: int = 64,
                 options: StereoOptions | None = None) -> DisparityMap:
    return default_matcher().match_stereo(left, right, left_valid, right_valid, disparity_min, num_disparities, options)


def match_stereo_batch(pairs: Sequence[dict]) -> list[DisparityMap]:
    return default_matcher().match_stereo_batch(pairs)


def census_transform(img) -> np.ndarray:
    return default_matcher().census_transform(img)


def pyramid_down(img) -> np.ndarray:
    return default_matcher().pyramid_down(img)


def remove_speckles(disparity: np.ndarray, min_size: int, max_diff: float) -> np.ndarray:
    return default_matcher().remove_speckles(disparity, min_size, max_diff)


def median_filter_3x3(disparity: np.ndarray) -> np.ndarray:
    return default_matcher().median_filter_3x3(disparity)


class detail:  # noqa: N801 — mirrors the reference's r3d::detail namespace
    @staticmethod
    def sgm_cost_volume(left, right, disparity_min, num_disparities, options=None, ranges=None):
        return default_matcher().sgm_cost_volume(left, right, disparity_min, num_disparities, options, ranges)

    @staticmethod
    def ranges_from_coarse(coarse, width, height, fine_valid, partner_valid, partner_width, partner_sign,
                           disparity_min, num_disparities, options=None, mirrored=False):
        return default_matcher().ranges_from_coarse(coarse, width, height, fine_valid, partner_valid, partner_width,
                                                    partner_sign, disparity_min, num_disparities, options, mirrored)

    @staticmethod
    def automatic_levels(width, height, num_disparities):
        return default_matcher().automatic_levels(width, height, num_disparities)
