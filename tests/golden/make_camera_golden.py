"""Writes camera_distortion.json: the reference's camera-model golden vectors.

The vectors are OpenMVG's distorted / undistorted pixels for four camera
models, which the reference's own test holds
(tests/test_camera_model.cpp:17-68, make_camera and kReference). This script
reads that file as text (nothing of the reference is compiled or run) and
keeps the cameras and the vectors as JSON, so that the tests run without the
reference tree.

Usage: python tests/golden/make_camera_golden.py path/to/reference
"""

from __future__ import annotations

import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
NUM = r"-?[0-9.]+(?:e-?[0-9]+)?"


def parse(text: str) -> dict:
    body = text[text.index("CameraIntrinsics make_camera"):text.index("struct Reference")]
    base = {
        "width": int(re.search(r"cam\.width = (\d+);", body).group(1)),
        "height": int(re.search(r"cam\.height = (\d+);", body).group(1)),
        "f": float(re.search(rf"cam\.fx = cam\.fy = ({NUM});", body).group(1)),
        "cx": float(re.search(rf"cam\.cx = ({NUM});", body).group(1)),
        "cy": float(re.search(rf"cam\.cy = ({NUM});", body).group(1)),
    }
    cameras = {}
    for m in re.finditer(r"case CameraModel::(\w+):(.*?)break;", body, re.S):
        name, case = m.group(1), m.group(2)
        f = re.search(rf"cam\.fx = cam\.fy = ({NUM});", case)
        params = [float(v) for v in re.search(r"cam\.params = \{([^}]*)\}", case).group(1).split(",")]
        focal = float(f.group(1)) if f else base["f"]
        cameras[name] = {"model": name, "width": base["width"], "height": base["height"], "fx": focal,
                         "fy": focal, "cx": base["cx"], "cy": base["cy"], "params": params}
    vectors = []
    row = re.compile(rf"\{{CameraModel::(\w+), \{{({NUM}), ({NUM})\}}, \{{({NUM}), ({NUM})\}}, "
                     rf"\{{({NUM}), ({NUM})\}}\}}")
    for m in row.finditer(text):
        vectors.append({"model": m.group(1), "pixel": [float(m.group(2)), float(m.group(3))],
                        "distorted": [float(m.group(4)), float(m.group(5))],
                        "undistorted": [float(m.group(6)), float(m.group(7))]})
    return {"source": "tests/test_camera_model.cpp (make_camera, kReference)", "cameras": cameras,
            "vectors": vectors}


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit("usage: make_camera_golden.py <root of a checkout of rhiestan/Regard3D_MVS>")
    ref = sys.argv[1]
    with open(os.path.join(ref, "tests", "test_camera_model.cpp")) as f:
        data = parse(f.read())
    assert len(data["vectors"]) == 24 and len(data["cameras"]) == 4, (len(data["vectors"]), data["cameras"])
    with open(os.path.join(HERE, "camera_distortion.json"), "w") as f:
        json.dump(data, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
