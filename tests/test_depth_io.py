""".r3dd depth-map files (src/r3d/mvs/depth_map.cpp:135-239, format version 2).

The library's writer and reader are checked against a restatement of the
format in this file (struct packing of the fields the reference writes, in
its order) and by the reference's round-trip test (tests/test_mvs.cpp:357-383).
File I/O is host code: the tests load the CUDA library itself (no device is
touched when the images are host memory) and the emulator build.
"""

from __future__ import annotations

import struct

import numpy as np
import pytest

from mvs_scenes import MultiRig, plane_depth_map, slanted_plane
from regard3d_mvs_b200 import _native
from regard3d_mvs_b200.depth_maps import read_depth_map, write_depth_map


@pytest.fixture(params=["cuda_library", "emulator"])
def lib(request, simt_matcher):
    if request.param == "emulator":
        return simt_matcher.lib
    return _native.load()


def reference_map():
    """test_mvs.cpp:357-364."""
    rig = MultiRig()
    m = plane_depth_map(rig.base, slanted_plane(rig.base), 7, 3)
    m["partners"] = [3, 9]
    m["pair_mask"][6, 5] = 3
    m["support"][8, 7] = 4
    m["depth"][2, 1] = 0.0
    m["color"][..., 2] = np.arange(m["depth"].size, dtype=np.int64).reshape(m["depth"].shape) % 251
    return m


def packed(m) -> bytes:
    """The bytes the reference's write_depth_map produces (depth_map.cpp:135-176)."""
    cam = m["camera"]
    h, w = m["depth"].shape
    out = [b"R3DD", struct.pack("<II", 2, m["view"])]
    out.append(struct.pack("<ii", cam["width"], cam["height"]))
    out.append(struct.pack("<4d", cam["fx"], cam["fy"], cam["cx"], cam["cy"]))
    out.append(struct.pack("<9d", *np.asarray(cam["rotation"], np.float64).ravel()))
    out.append(struct.pack("<3d", *np.asarray(cam["center"], np.float64)))
    out.append(struct.pack("<I", len(m["partners"])) + struct.pack(f"<{len(m['partners'])}I", *m["partners"]))
    out.append(struct.pack("<ii", w, h))
    for key, dt in (("depth", "<f4"), ("confidence", "<f4"), ("pair_mask", "<u2"), ("support", "u1"),
                    ("color", "u1")):
        out.append(np.ascontiguousarray(m[key], dt).tobytes())
    return b"".join(out)


def test_round_trip(lib, tmp_path):
    """test_mvs.cpp:357-383."""
    m = reference_map()
    path = tmp_path / "d.r3dd"
    write_depth_map(lib, path, m)
    r = read_depth_map(lib, path)
    assert r["view"] == 7 and r["partners"] == [3, 9]
    assert r["camera"]["cx"] == m["camera"]["cx"]
    np.testing.assert_array_equal(r["camera"]["rotation"], m["camera"]["rotation"])
    np.testing.assert_array_equal(r["camera"]["center"], m["camera"]["center"])
    for key in ("depth", "confidence", "pair_mask", "support", "color"):
        np.testing.assert_array_equal(r[key], m[key])
    assert bin(int(r["pair_mask"][6, 5])).count("1") == 2


def test_bytes_follow_the_format(lib, tmp_path):
    m = reference_map()
    path = tmp_path / "d.r3dd"
    write_depth_map(lib, path, m)
    assert path.read_bytes() == packed(m)


def test_reads_files_in_the_format(lib, tmp_path):
    m = reference_map()
    m["partners"] = list(range(16))
    path = tmp_path / "r.r3dd"
    path.write_bytes(packed(m))
    r = read_depth_map(lib, path)
    assert r["partners"] == list(range(16))
    for key in ("depth", "confidence", "pair_mask", "support", "color"):
        np.testing.assert_array_equal(r[key], m[key])


def test_rejects_other_files(lib, tmp_path):
    m = reference_map()
    good = packed(m)
    bad_magic = tmp_path / "a.r3dd"
    bad_magic.write_bytes(b"R3DX" + good[4:])
    with pytest.raises(_native.StereoError, match="not an r3d depth map"):
        read_depth_map(lib, bad_magic)
    old = tmp_path / "b.r3dd"
    old.write_bytes(good[:4] + struct.pack("<I", 1) + good[8:])
    with pytest.raises(_native.StereoError, match="not an r3d depth map"):
        read_depth_map(lib, old)
    short = tmp_path / "c.r3dd"
    short.write_bytes(good[: len(good) // 2])
    with pytest.raises(_native.StereoError, match="corrupt depth map"):
        read_depth_map(lib, short)
    many = tmp_path / "d.r3dd"
    head = 4 + 4 + 4 + 8 + 32 + 72 + 24
    many.write_bytes(good[:head] + struct.pack("<I", 17) + good[head + 4:])
    with pytest.raises(_native.StereoError, match="corrupt depth map"):
        read_depth_map(lib, many)
    with pytest.raises(_native.StereoError, match="cannot open"):
        read_depth_map(lib, tmp_path / "missing.r3dd")


@pytest.mark.gpu
def test_device_maps_write_the_same_bytes(gpu_matcher, tmp_path):
    """Device-resident images (a served result) are written as the host map."""
    import ctypes

    import torch

    from regard3d_mvs_b200.depth_maps import c_depth_map, normalise

    m = normalise(reference_map())
    keep = []

    def dev(a):
        t = torch.from_numpy(a.view(np.int16) if a.dtype == np.uint16 else a).to("cuda:0")
        keep.append(t)
        return t.data_ptr()

    c = c_depth_map(m, dev)
    path = tmp_path / "g.r3dd"
    stream = torch.cuda.current_stream(0)
    _native.check(gpu_matcher.lib, gpu_matcher.lib.r3dgpu_write_depth_map(str(path).encode(), ctypes.byref(c), 1,
                                                                          stream.cuda_stream))
    assert path.read_bytes() == packed(m)
