"""Test scenes of the multi-view depth stages (restating the geometry of the
reference's tests/test_mvs.cpp:20-116: rotation(), pinhole_camera(),
test_plane() as slanted_plane(), plane_depth_map(), MultiRig), plus seeded synthetic scenes for
GPU-vs-oracle parity."""

from __future__ import annotations

import numpy as np


def axis_rotation(axis: int, deg: float) -> np.ndarray:
    a = np.deg2rad(deg)
    c, s = np.cos(a), np.sin(a)
    if axis == 0:
        return np.array([[1, 0, 0], [0, c, -s], [0, s, c]])
    if axis == 1:
        return np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]])
    return np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]])


def rotation(rx: float, ry: float, rz: float) -> np.ndarray:
    """test_mvs.cpp:22-28: Rz Ry Rx (angle-axis, degrees)."""
    return axis_rotation(2, rz) @ axis_rotation(1, ry) @ axis_rotation(0, rx)


def pinhole(w=320, h=240, f=280.0, cx=161.2, cy=118.7) -> dict:
    return {"width": w, "height": h, "fx": f, "fy": f, "cx": cx, "cy": cy}


def camera(k: dict, r: np.ndarray, c) -> dict:
    return dict(k, rotation=np.asarray(r, np.float64), center=np.asarray(c, np.float64))


def view_direction(cam: dict) -> np.ndarray:
    return cam["rotation"][2]


class Plane:
    def __init__(self, normal, point):
        self.normal = np.asarray(normal, np.float64)
        self.point = np.asarray(point, np.float64)

    def intersect(self, centre, dirs):
        """Ray parameter t of centre + t * dir (dirs: ... x 3)."""
        return ((self.point - centre) @ self.normal) / (dirs @ self.normal)


def slanted_plane(base: dict) -> Plane:
    """test_mvs.cpp:47-52."""
    vd = view_direction(base)
    n = vd + base["rotation"].T @ np.array([0.3, -0.2, 0.0])
    return Plane(n / np.linalg.norm(n), base["center"] + 5.0 * vd)


def pixel_rays(cam: dict) -> np.ndarray:
    """World directions of unit depth, H x W x 3 (camera.unproject(p, 1) - C)."""
    y, x = np.mgrid[0:cam["height"], 0:cam["width"]].astype(np.float64)
    d = np.stack([(x - cam["cx"]) / cam["fx"], (y - cam["cy"]) / cam["fy"], np.ones_like(x)], -1)
    return d @ cam["rotation"]  # R^T d per pixel


def plane_depth_map(cam: dict, plane: Plane, view: int, partner: int) -> dict:
    """test_mvs.cpp:71-93: exact depths, pair mask bit 0, confidence 0.5,
    colour (200, 100, 50)."""
    h, w = cam["height"], cam["width"]
    depth = plane.intersect(cam["center"], pixel_rays(cam)).astype(np.float32)
    color = np.empty((h, w, 3), np.uint8)
    color[...] = (200, 100, 50)
    return {"camera": cam, "depth": depth, "confidence": np.full((h, w), 0.5, np.float32),
            "pair_mask": np.ones((h, w), np.uint16), "support": np.zeros((h, w), np.uint8), "color": color,
            "view": view, "partners": [partner]}


class MultiRig:
    """test_mvs.cpp:95-113."""

    def __init__(self, scale: float = 1.0):
        self.k = pinhole(int(320 * scale), int(240 * scale), 280.0 * scale, 161.2 * scale, 118.7 * scale)
        self.base = camera(self.k, rotation(2.0, -3.0, 1.0), (0.1, -0.2, 0.0))
        self.partners = []
        for i, off in enumerate(((0.8, 0.05, 0.1), (-0.7, 0.1, 0.0), (0.1, 0.75, -0.1))):
            r = rotation(-1.0 + i, 3.0 - 2.0 * i, -2.0)
            self.partners.append(camera(self.k, r, self.base["center"] + self.base["rotation"].T @ np.array(off)))


def empty_map(w: int, h: int) -> dict:
    """DepthMap::allocate (depth_map.cpp:19-26) with an identity camera."""
    cam = camera(pinhole(w, h, 100.0, w / 2, h / 2), np.eye(3), (0, 0, 0))
    return {"camera": cam, "depth": np.zeros((h, w), np.float32), "confidence": np.zeros((h, w), np.float32),
            "pair_mask": np.zeros((h, w), np.uint16), "support": np.zeros((h, w), np.uint8),
            "color": np.zeros((h, w, 3), np.uint8), "view": 0, "partners": []}


def synthetic_scene(n_views: int, w: int, h: int, seed: int, outliers: float = 0.03, holes: float = 0.02):
    """Views on an arc around two slanted planes; per view the exact depth with
    small noise, a fraction of outliers (+-8 %), holes, pair masks over 4
    partners, and a colour image with edges (so that halos and weak depths
    occur). Neighbouring log depths differ by far less than the 2 % segment
    step or by far more, so a one-ulp logf difference cannot change a segment."""
    rng = np.random.default_rng(seed)
    f = 0.9 * w
    k = pinhole(w, h, f, (w - 1) / 2 + 0.3, (h - 1) / 2 - 0.2)
    views = []
    for i in range(n_views):
        a = np.deg2rad(-12.0 + 24.0 * i / max(1, n_views - 1))
        c = np.array([4.0 * np.sin(a), 0.15 * np.sin(3 * a), -4.0 * np.cos(a) + 4.0])
        z = -c / np.linalg.norm(c) if np.linalg.norm(c) > 0 else np.array([0, 0, 1.0])
        z = np.array([0.0, 0.0, 4.0]) - c
        z /= np.linalg.norm(z)
        xax = np.cross([0.0, 1.0, 0.0], z)
        xax /= np.linalg.norm(xax)
        yax = np.cross(z, xax)
        views.append(camera(k, np.stack([xax, yax, z]), c))
    back = Plane(np.array([0.1, -0.05, -1.0]) / np.linalg.norm([0.1, -0.05, -1.0]), (0, 0, 8.0))
    front = Plane(np.array([-0.3, 0.1, -1.0]) / np.linalg.norm([-0.3, 0.1, -1.0]), (0.4, 0.2, 5.5))
    maps = []
    for i, cam in enumerate(views):
        rays = pixel_rays(cam)
        tb = back.intersect(cam["center"], rays)
        tf = front.intersect(cam["center"], rays)
        pts = cam["center"] + tf[..., None] * rays
        in_front = (np.abs(pts[..., 0] - 0.4) < 1.0) & (np.abs(pts[..., 1] - 0.2) < 0.7)
        t = np.where(in_front, tf, tb)
        d = (t * (1.0 + rng.normal(0, 2e-4, t.shape))).astype(np.float32)
        bad = rng.random(d.shape) < outliers
        d[bad] *= np.where(rng.random(bad.sum()) < 0.5, 1.08, 0.92).astype(np.float32)
        d[rng.random(d.shape) < holes] = 0.0
        d[40:60, 30:70] = 0.0  # a large hole
        color = np.empty(d.shape + (3,), np.uint8)
        color[...] = np.where(in_front[..., None], np.array([60, 80, 90], np.uint8), np.array([190, 170, 150], np.uint8))
        stripes = ((np.arange(w)[None, :] // 6 + np.arange(h)[:, None] // 9) % 4 == 0) & ~in_front
        color[stripes] = (20, 200, 40)
        partners = [j for j in range(n_views) if j != i][:4]
        mask = rng.integers(0, 16, d.shape).astype(np.uint16)
        conf = rng.random(d.shape).astype(np.float32)
        maps.append({"camera": cam, "depth": d, "confidence": conf, "pair_mask": mask,
                     "support": np.zeros(d.shape, np.uint8), "color": color, "view": i, "partners": partners})
    neighbours = [[j for j in range(n_views) if j != i and abs(j - i) <= 2] for i in range(n_views)]
    return maps, neighbours


def copy_maps(maps):
    out = []
    for m in maps:
        c = dict(m)
        for key in ("depth", "confidence", "pair_mask", "support", "color"):
            if c.get(key) is not None:
                c[key] = c[key].copy()
        out.append(c)
    return out


# ------------------------------------------------------------------ refinement scenes
def unit_orthogonal(n: np.ndarray) -> np.ndarray:
    """A unit vector orthogonal to n (the rule of Eigen's unitOrthogonal for 3-vectors)."""
    x, y, z = n
    if abs(x) > 1e-12 * abs(z) or abs(y) > 1e-12 * abs(z):
        inv = 1.0 / np.hypot(x, y)
        return np.array([-y * inv, x * inv, 0.0])
    inv = 1.0 / np.hypot(y, z)
    return np.array([0.0, -z * inv, y * inv])


WAVES = ((31.0, 7.0, 0.3), (-11.0, 23.0, 1.1), (5.0, -13.0, 2.0), (43.0, 29.0, 0.7), (-37.0, 47.0, 2.9))


def render_plane(cam: dict, plane: Plane, phase: float) -> np.ndarray:
    """test_mvs.cpp:386-414: smooth texture on a plane, 4 x 4 supersampled."""
    u = unit_orthogonal(plane.normal)
    v = np.cross(plane.normal, u)
    h, w = cam["height"], cam["width"]
    y, x = np.mgrid[0:h, 0:w].astype(np.float64)
    acc = np.zeros((h, w))
    for sy in range(4):
        for sx in range(4):
            px, py = x - 0.375 + 0.25 * sx, y - 0.375 + 0.25 * sy
            d = np.stack([(px - cam["cx"]) / cam["fx"], (py - cam["cy"]) / cam["fy"], np.ones_like(px)], -1)
            dirs = d @ cam["rotation"]
            t = plane.intersect(cam["center"], dirs)
            xw = cam["center"] + t[..., None] * dirs - plane.point
            pu, pv = xw @ u, xw @ v
            for kx, ky, ph in WAVES:
                acc += np.sin(kx * pu + ky * pv + ph + phase)
    return (128.0 + 20.0 * acc / 16.0).astype(np.float32)


def refinement_scene(make_image, scale: int = 1):
    """test_mvs.cpp:431-467 (at scale 1): the rig's base view cropped to its
    central 160 x 120, a plane at 42 degrees, rendered views, and an SGM-like input
    (constant depth per 4 x 4 block times a smooth error of up to 1 %).
    make_image(gray) builds a refinement image. Returns (map, truth, base,
    views, wrong_views)."""
    rig = MultiRig(scale)
    cam0 = dict(rig.base, width=160 * scale, height=120 * scale, cx=rig.base["cx"] - 80.0 * scale,
                cy=rig.base["cy"] - 60.0 * scale)
    vd = view_direction(rig.base)
    n = vd + rig.base["rotation"].T @ np.array([0.8, 0.4, 0.0])
    plane = Plane(n / np.linalg.norm(n), rig.base["center"] + 5.0 * vd)
    truth = plane_depth_map(cam0, plane, 0, 1)
    base = {"camera": cam0, "data": make_image(render_plane(cam0, plane, 0.0))}
    views = [{"camera": p, "data": make_image(render_plane(p, plane, 0.0))} for p in rig.partners]
    wrong = [{"camera": p, "data": make_image(render_plane(p, plane, 1.7))} for p in rig.partners]
    h, w = truth["depth"].shape
    y, x = np.mgrid[0:h, 0:w]
    block = truth["depth"][np.minimum(y // 4 * 4 + 2, h - 1), np.minimum(x // 4 * 4 + 2, w - 1)]
    depth = (block * (1.0 + 0.01 * np.sin(x / 9.0) * np.cos(y / 13.0)).astype(np.float32)).astype(np.float32)
    m = {"camera": cam0, "depth": depth, "confidence": truth["confidence"].copy()}
    return m, truth, base, views, wrong


def relative_depth_rms(m: dict, truth: dict, border: int) -> float:
    """test_mvs.cpp:416-428."""
    d = m["depth"][border:-border, border:-border].astype(np.float64)
    t = truth["depth"][border:-border, border:-border].astype(np.float64)
    return float(np.sqrt(np.mean(((d - t) / t) ** 2)))
