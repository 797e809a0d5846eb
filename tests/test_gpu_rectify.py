"""rectify_image on the B200 against the oracle.

Every camera model but fisheye is bit-exact: the kernel's operations are the
reference's, in its order, without contraction, and double division and
square root round correctly on both sides. Fisheye projection goes through
atan, whose CUDA and host implementations may differ in the last ulp, so
there the test allows what one ulp of the source position can change: a u16
pixel by one step in a handful of pixels, an f32 pixel by a relative 1e-5.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from test_rectify import MODELS, setup, textured

pytestmark = pytest.mark.gpu


def _compare(got, want, gv, wv, fisheye):
    if not fisheye:
        np.testing.assert_array_equal(gv, wv)
        if got.dtype == np.float32:
            np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
        else:
            np.testing.assert_array_equal(got, want)
        return
    both = (gv == 255) & (wv == 255)
    assert (gv != wv).sum() <= max(2, int(1e-4 * gv.size))
    if got.dtype == np.float32:
        scale = max(1.0, float(np.abs(want[both]).max()))
        assert np.abs(got[both] - want[both]).max() <= 1e-5 * scale
    else:
        diff = np.abs(got[both].astype(np.int32) - want[both].astype(np.int32))
        assert diff.max() <= 1 and (diff > 0).sum() <= max(2, int(1e-3 * both.sum()))


@pytest.mark.parametrize("model", sorted(MODELS))
@pytest.mark.parametrize("tf", [175.0, 70.0, 50.0])
def test_rectify_equals_oracle(gpu_matcher, oracle, model, tf):
    cam, m, target = setup(model, tf)
    for dtype, seed in ((np.uint16, 1), (np.float32, 2)):
        src = textured(cam["height"], cam["width"], dtype, seed + model)
        got, gv = gpu_matcher.rectify_image(src, cam, m, target)
        want, wv = oracle.rectify_image(src, cam, m, target)
        assert (wv == 255).mean() > 0.05
        _compare(got, want, gv, wv, model == 4)


@pytest.mark.parametrize("model,ratio", [(3, 1.0), (2, 2.2), (0, 4.5)])
def test_rectify_full_size_equals_oracle(gpu_matcher, oracle, model, ratio):
    """A 4000x3000 photo into a rectified camera of the same size (pyramid
    level 0), of about half (level 1) and of a quarter (level 2)."""
    w, h = 4000, 3000
    cam = {"model": model, "width": w, "height": h, "fx": 3600.0, "fy": 3602.0, "cx": (w - 1) / 2 + 7,
           "cy": (h - 1) / 2 - 4, "params": MODELS[model]}
    from geometry import rot_x, rot_y

    m = (rot_y(0.04) @ rot_x(-0.015)) @ rot_x(0.02).T
    tw, th = int(round(w * 1.02 / ratio)), int(round(h * 1.02 / ratio))
    target = {"width": tw, "height": th, "fx": 3600.0 / ratio, "fy": 3600.0 / ratio, "cx": (tw - 1) / 2,
              "cy": (th - 1) / 2 + 3}
    src = textured(h, w, np.uint16, 7)
    got, gv = gpu_matcher.rectify_image(src, cam, m, target)
    want, wv = oracle.rectify_image(src, cam, m, target)
    np.testing.assert_array_equal(gv, wv)
    np.testing.assert_array_equal(got, want)
    assert (wv == 255).mean() > 0.8


def test_rectify_device_entry_with_strides(gpu_matcher):
    """The device-pointer entry points on a stream, with padded rows, equal
    the host entry points."""
    import torch

    from regard3d_mvs_b200.types import CViewU16, camera_struct, pinhole_struct

    lib = gpu_matcher.lib
    cam, m, target = setup(3, 90.0, w=333, h=211, tw=301, th=199)
    c, k = camera_struct(cam), pinhole_struct(target)
    mm = np.ascontiguousarray(m).reshape(9)
    stream = torch.cuda.Stream(0)
    for dtype, tdt in ((np.uint16, torch.int16), (np.float32, torch.float32)):
        src = textured(cam["height"], cam["width"], dtype, 5)
        want, wv = gpu_matcher.rectify_image(src, cam, m, target)
        sp, op, vp = cam["width"] + 13, target["width"] + 7, target["width"] + 29
        dsrc = torch.zeros((cam["height"], sp), dtype=tdt, device="cuda:0")
        dsrc[:, :cam["width"]] = torch.from_numpy(src.view(np.int16) if dtype == np.uint16 else src).to("cuda:0")
        dout = torch.full((target["height"], op), 77, dtype=tdt, device="cuda:0")
        dval = torch.full((target["height"], vp), 9, dtype=torch.uint8, device="cuda:0")
        torch.cuda.synchronize(0)
        if dtype == np.uint16:
            view = CViewU16(dsrc.data_ptr(), cam["width"], cam["height"], sp)
            st = lib.r3dgpu_rectify_image_u16(ctypes.byref(view), ctypes.byref(c), mm.ctypes.data, ctypes.byref(k),
                                              dout.data_ptr(), op, dval.data_ptr(), vp, stream.cuda_stream)
        else:
            st = lib.r3dgpu_rectify_image_f32(dsrc.data_ptr(), sp, ctypes.byref(c), mm.ctypes.data, ctypes.byref(k),
                                              dout.data_ptr(), op, dval.data_ptr(), vp, stream.cuda_stream)
        assert st == 0, lib.r3dgpu_last_error().decode()
        out = dout.cpu().numpy()
        val = dval.cpu().numpy()
        got = out[:, :target["width"]]
        got = got.view(np.uint16) if dtype == np.uint16 else got
        np.testing.assert_array_equal(got, want)
        np.testing.assert_array_equal(val[:, :target["width"]], wv)
        assert np.all(out[:, target["width"]:] == 77) and np.all(val[:, target["width"]:] == 9)  # padding untouched
