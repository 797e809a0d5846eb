"""Rectification resampling (r3d::rectify_image, src/r3d/rectify/rectification.cpp:287-350).

The oracle's camera models are pinned to the OpenMVG golden vectors of the
reference's camera-model test (tests/golden/camera_distortion.json, from
tests/test_camera_model.cpp:17-68), and the oracle as a whole to the
reference's rectify_image test (tests/test_rectification.cpp:128-169: a
Gaussian blob drawn at a known rectified position lands there). The CUDA
kernel runs here on the SIMT emulator and must equal the oracle bit for bit,
for every camera model, both pixel types and the pyramid levels chosen for
anti-aliasing.
"""

from __future__ import annotations

import ctypes
import json
import os

import numpy as np
import pytest

from geometry import rot_x, rot_y

HERE = os.path.dirname(os.path.abspath(__file__))

MODELS = {
    0: (),
    1: (-0.09,),
    2: (-0.08, 0.02, -0.003),
    3: (-0.08, 0.02, -0.003, 0.001, -0.0015),
    4: (0.02, -0.01, 0.004, -0.001),
}


def distort(model: int, p, ux, uy):
    """camera_model.cpp:67-100 in numpy (normalised coordinates)."""
    r2 = ux * ux + uy * uy
    if model == 1:
        s = 1.0 + p[0] * r2
        return ux * s, uy * s
    if model == 2:
        s = 1.0 + r2 * (p[0] + r2 * (p[1] + r2 * p[2]))
        return ux * s, uy * s
    if model == 3:
        radial = r2 * (p[0] + r2 * (p[1] + r2 * p[2]))
        tx = p[4] * (r2 + 2 * ux * ux) + 2 * p[3] * ux * uy
        ty = p[3] * (r2 + 2 * uy * uy) + 2 * p[4] * ux * uy
        return ux + ux * radial + tx, uy + uy * radial + ty
    if model == 4:
        r = np.sqrt(r2)
        th = np.arctan(r)
        t2 = th * th
        s = np.where(r > 1e-8, th * (1 + t2 * (p[0] + t2 * (p[1] + t2 * (p[2] + t2 * p[3])))) / np.maximum(r, 1e-300),
                     1.0)
        return ux * s, uy * s
    return ux, uy


def undistort(model: int, p, dx, dy, iters: int = 30):
    """Inverse of distort by Newton steps with a central-difference Jacobian."""
    ux, uy = np.array(dx, np.float64), np.array(dy, np.float64)
    h = 1e-7
    for _ in range(iters):
        fx, fy = distort(model, p, ux, uy)
        rx, ry = fx - dx, fy - dy
        ax, ay = distort(model, p, ux + h, uy)
        bx, by = distort(model, p, ux - h, uy)
        cx, cy = distort(model, p, ux, uy + h)
        ex, ey = distort(model, p, ux, uy - h)
        j11, j21 = (ax - bx) / (2 * h), (ay - by) / (2 * h)
        j12, j22 = (cx - ex) / (2 * h), (cy - ey) / (2 * h)
        det = j11 * j22 - j12 * j21
        ux = ux - (j22 * rx - j12 * ry) / det
        uy = uy - (-j21 * rx + j11 * ry) / det
    return ux, uy


def setup(model: int, tf: float, w: int = 200, h: int = 150, tw: int = 210, th: int = 160):
    """Source camera (w x h, the given model), target pinhole (tw x th, focal
    tf) rotated against it; returns (camera, source_from_target, target)."""
    cam = {"model": model, "width": w, "height": h, "fx": 180.0, "fy": 181.0, "cx": (w - 1) / 2 + 2,
           "cy": (h - 1) / 2 - 1.5, "params": MODELS[model]}
    r_src = rot_y(0.05) @ rot_x(-0.02)
    r_tgt = rot_x(0.03)
    target = {"width": tw, "height": th, "fx": tf, "fy": tf, "cx": (tw - 1) / 2, "cy": (th - 1) / 2 + 1}
    return cam, r_src @ r_tgt.T, target


def textured(h: int, w: int, dtype, seed: int) -> np.ndarray:
    """Smooth texture plus noise, with saturated patches so that the u16
    clamps at 0 and 65535 are reached by bicubic overshoot."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h, 0:w]
    base = 0.5 + 0.3 * np.sin(x / 7.0) * np.cos(y / 5.0) + 0.15 * rng.standard_normal((h, w))
    base[(x // 16 + y // 16) % 5 == 0] = 1.0
    base[(x // 16 + y // 16) % 7 == 0] = 0.0
    if dtype == np.uint16:
        return np.clip(base * 65535, 0, 65535).astype(np.uint16)
    return (base * 1000.0 - 200.0).astype(np.float32)


# ------------------------------------------------------------------ oracle pins
def test_oracle_camera_models_match_openmvg_vectors(oracle):
    """tests/test_camera_model.cpp:71-83: distort_pixel equals OpenMVG's to 1e-9."""
    with open(os.path.join(HERE, "golden", "camera_distortion.json")) as f:
        data = json.load(f)
    assert len(data["vectors"]) == 24
    for v in data["vectors"]:
        cam = data["cameras"][v["model"]]
        got = oracle.distort_pixel(cam, v["pixel"])[0]
        np.testing.assert_allclose(got, v["distorted"], rtol=0, atol=1e-9, err_msg=str(v))


def test_numpy_camera_models_match_openmvg_vectors():
    """The test-side numpy models (used to draw the blob images) against the
    same vectors, undistortion to OpenMVG's 1e-5 (its inverse stops early)."""
    with open(os.path.join(HERE, "golden", "camera_distortion.json")) as f:
        data = json.load(f)
    models = {"radial_k1": 1, "radial_k3": 2, "brown_t2": 3, "fisheye": 4}
    for v in data["vectors"]:
        cam = data["cameras"][v["model"]]
        m, p = models[v["model"]], cam["params"]
        ux, uy = (v["pixel"][0] - cam["cx"]) / cam["fx"], (v["pixel"][1] - cam["cy"]) / cam["fy"]
        dx, dy = distort(m, p, np.float64(ux), np.float64(uy))
        np.testing.assert_allclose([cam["fx"] * dx + cam["cx"], cam["fy"] * dy + cam["cy"]], v["distorted"],
                                   atol=1e-9)
        bx, by = undistort(m, p, np.float64(ux), np.float64(uy), iters=60)
        np.testing.assert_allclose([cam["fx"] * bx + cam["cx"], cam["fy"] * by + cam["cy"]], v["undistorted"],
                                   atol=1e-5)


def blob_source(cam: dict, source_from_target, target: dict, centre) -> np.ndarray:
    """tests/test_rectification.cpp:139-150: a Gaussian blob (sigma 2.5 px)
    centred on a known rectified pixel, drawn in the distorted source."""
    h, w = cam["height"], cam["width"]
    y, x = np.mgrid[0:h, 0:w].astype(np.float64)
    ux, uy = undistort(cam["model"], cam["params"], (x - cam["cx"]) / cam["fx"], (y - cam["cy"]) / cam["fy"])
    m = np.asarray(source_from_target).T  # target_from_source
    rx = m[0, 0] * ux + m[0, 1] * uy + m[0, 2]
    ry = m[1, 0] * ux + m[1, 1] * uy + m[1, 2]
    rz = m[2, 0] * ux + m[2, 1] * uy + m[2, 2]
    px = target["fx"] * rx / rz + target["cx"]
    py = target["fy"] * ry / rz + target["cy"]
    d2 = (px - centre[0]) ** 2 + (py - centre[1]) ** 2
    return (1000.0 * np.exp(-d2 / (2 * 2.5 * 2.5))).astype(np.float32)


@pytest.mark.parametrize("model", [0, 2, 3])
def test_oracle_moves_a_blob_to_its_rectified_position(oracle, model):
    """tests/test_rectification.cpp:128-169, restated."""
    cam, m, target = setup(model, 175.0)
    centre = (0.45 * target["width"] + 0.3, 0.55 * target["height"] - 0.2)
    src = blob_source(cam, m, target, centre)
    rect, valid = oracle.rectify_image(src, cam, m, target)
    assert rect.shape == (target["height"], target["width"])
    y, x = np.mgrid[0:target["height"], 0:target["width"]]
    near = np.hypot(x - centre[0], y - centre[1]) < 12.0
    assert np.all(valid[near] == 255)
    wsum = rect[near].astype(np.float64).sum()
    assert abs((rect[near] * x[near]).sum() / wsum - centre[0]) < 0.05
    assert abs((rect[near] * y[near]).sum() / wsum - centre[1]) < 0.05


def test_oracle_pyramid_level_for_small_targets(oracle):
    """rectification.cpp:297-311: a target with less than 1/1.5 of the source
    resolution samples the 2x-reduced source (pyramid_camera halves K), so a
    constant image stays constant and a checkerboard at the source's Nyquist
    rate averages out instead of aliasing."""
    cam, m, target = setup(0, 70.0)
    flat = np.full((cam["height"], cam["width"]), 321.5, np.float32)
    rect, valid = oracle.rectify_image(flat, cam, m, target)
    assert np.abs(rect[valid == 255] - 321.5).max() < 1e-3  # float weights sum to 1 within a few ulps
    y, x = np.mgrid[0:cam["height"], 0:cam["width"]]
    board = np.where((x + y) % 2 == 0, 1000.0, 0.0).astype(np.float32)
    rect, valid = oracle.rectify_image(board, cam, m, target)
    # Away from the source border, where the pyramid's clamped taps see an
    # uneven share of the two colours.
    core = valid == 255
    for _ in range(4):
        core = core & np.roll(core, 1, 0) & np.roll(core, -1, 0) & np.roll(core, 1, 1) & np.roll(core, -1, 1)
    inner = rect[core]
    assert inner.size > 1000
    assert np.abs(inner - 500.0).max() < 80.0


# ------------------------------------------------------------------ kernel on the emulator
@pytest.mark.parametrize("model", sorted(MODELS))
@pytest.mark.parametrize("tf", [175.0, 70.0, 50.0])
def test_emulator_matches_oracle(simt_matcher, oracle, model, tf):
    """Bit-exact: u16 and f32, no pyramid level (tf 175), one (70) and two (50)."""
    cam, m, target = setup(model, tf)
    for dtype, seed in ((np.uint16, 1), (np.float32, 2)):
        src = textured(cam["height"], cam["width"], dtype, seed + model)
        got, gv = simt_matcher.rectify_image(src, cam, m, target)
        want, wv = oracle.rectify_image(src, cam, m, target)
        assert got.dtype == want.dtype
        np.testing.assert_array_equal(gv, wv)
        assert (wv == 255).mean() > 0.05
        np.testing.assert_array_equal(got.view(np.uint32 if dtype == np.float32 else np.uint16),
                                      want.view(np.uint32 if dtype == np.float32 else np.uint16))


def test_emulator_clamps_u16_overshoot(simt_matcher, oracle):
    """Bicubic overshoot at a 0 / 65535 step is clamped, as to_pixel does."""
    cam, m, target = setup(0, 175.0)
    src = np.zeros((cam["height"], cam["width"]), np.uint16)
    src[:, cam["width"] // 2:] = 65535
    got, _ = simt_matcher.rectify_image(src, cam, m, target)
    want, _ = oracle.rectify_image(src, cam, m, target)
    np.testing.assert_array_equal(got, want)
    assert got.max() == 65535 and got.min() == 0
    ref_f, _ = oracle.rectify_image(src.astype(np.float32), cam, m, target)
    assert ref_f.max() > 65535.5 and ref_f.min() < -0.5  # the overshoot that was clamped


def _status(lib):
    return lib.r3dgpu_last_error().decode()


def test_emulator_rejects_bad_arguments(simt_matcher):
    from regard3d_mvs_b200.types import CCamera, CPinhole, CViewU16, camera_struct, pinhole_struct

    lib = simt_matcher.lib
    cam, m, target = setup(2, 175.0)
    src = textured(cam["height"], cam["width"], np.uint16, 3)
    out = np.empty((target["height"], target["width"]), np.uint16)
    mm = np.ascontiguousarray(m).reshape(9)
    c, k = camera_struct(cam), pinhole_struct(target)

    def call(view, c=c, k=k, ostride=target["width"]):
        return lib.r3dgpu_rectify_image_u16_host(ctypes.byref(view), ctypes.byref(c), mm.ctypes.data,
                                                  ctypes.byref(k), out.ctypes.data, ostride, None, 0)

    good = CViewU16(src.ctypes.data, cam["width"], cam["height"], cam["width"])
    assert call(good) == 0
    wrong = CViewU16(src.ctypes.data, cam["width"] - 1, cam["height"], cam["width"])
    assert call(wrong) == 1 and "camera is 200x150" in _status(lib)
    bad_model = CCamera.from_buffer_copy(c)
    bad_model.model = 9
    assert call(good, c=bad_model) == 1 and "camera model" in _status(lib)
    assert call(good, ostride=10) == 1 and "stride" in _status(lib)
    empty = CPinhole(0, 0, 100.0, 100.0, 0.0, 0.0)
    assert call(good, k=empty) == 0  # nothing to write
    with pytest.raises(Exception, match="rectify_image"):
        simt_matcher.rectify_image(np.zeros((10, 10), np.float32), cam, m, target)
