"""Geometry of the multi-view combination (r3dgpu_combine_pairs) as ctypes
structs.

A grid is a dict with the grid camera's ``K`` (3x3), ``R`` (world -> camera
rotation), ``C`` (centre), ``width`` and ``height``. A pair is a dict with its
rectified left camera (``K_rect``, ``R_rect``), ``baseline``, the right
camera's principal point ``cx_right``, the partner's ``centre`` and the
pair's ``disparity`` (and optional ``confidence``) maps in the rectified left
image: the quantities src/r3d/mvs/multi_stereo.cpp:85-93 derives per pair.
"""

from __future__ import annotations

import ctypes

import numpy as np

from .types import CCamera, CDepthGrid, CPairGeometry, CPinhole, CViewU16


def c_grid(grid: dict) -> CDepthGrid:
    g = CDepthGrid()
    k_inv = np.linalg.inv(np.asarray(grid["K"], np.float64))
    rot_t = np.asarray(grid["R"], np.float64).T
    g.k_inv[:] = [float(v) for v in k_inv.ravel()]
    g.rot_t[:] = [float(v) for v in rot_t.ravel()]
    g.center[:] = [float(v) for v in np.asarray(grid["C"], np.float64)]
    g.width, g.height = int(grid["width"]), int(grid["height"])
    return g


def pair_geometry(grid: dict, p: dict) -> CPairGeometry:
    """The combination geometry of a pair (no maps): grid-to-rectified
    homography K_r R_r R_g^T K_g^-1, f * b, disparity offset, partner centre."""
    q = CPairGeometry()
    k_inv = np.linalg.inv(np.asarray(grid["K"], np.float64))
    r_gt = np.asarray(grid["R"], np.float64).T
    kr = np.asarray(p["K_rect"], np.float64)
    h = kr @ np.asarray(p["R_rect"], np.float64) @ r_gt @ k_inv
    q.grid_to_rect[:] = [float(v) for v in h.ravel()]
    q.fb = float(kr[0, 0] * p["baseline"])
    q.offset = float(kr[0, 2] - p["cx_right"])
    q.partner_center[:] = [float(v) for v in np.asarray(p["centre"], np.float64)]
    return q


def c_pairs(grid: dict, pairs: list[dict]):
    """(array of CPairGeometry with host map pointers, the arrays they point into)."""
    arr = (CPairGeometry * max(len(pairs), 1))()
    keep = []
    for i, p in enumerate(pairs):
        d = np.ascontiguousarray(p["disparity"], np.float32)
        c = p.get("confidence")
        c = None if c is None else np.ascontiguousarray(c, np.float32)
        keep += [d, c]
        arr[i] = pair_geometry(grid, p)
        q = arr[i]
        q.disparity = d.ctypes.data
        q.confidence = None if c is None else c.ctypes.data
        q.height, q.width = d.shape
        q.stride = d.shape[1]
    return arr, keep


# ---------------------------------------------------------------- synthetic views
# A base camera, partner cameras, their rectified pairs (x axis along the
# baseline, optical axis the mean of the two cameras' axes, as
# src/r3d/rectify/rectification.hpp:14-20 describes) and the disparity maps of
# a plane, d = f b / z + (cx_l - cx_r): inputs for tests and benchmarks.


def rot_y(a):
    c, s = np.cos(a), np.sin(a)
    return np.array([[c, 0, -s], [0, 1, 0], [s, 0, c]], np.float64)


def rot_x(a):
    c, s = np.cos(a), np.sin(a)
    return np.array([[1, 0, 0], [0, c, s], [0, -s, c]], np.float64)


class Rig:
    """Base camera at the origin looking along +z (world -> camera rotation
    R), partners around it looking at the scene centre."""

    def __init__(self, w=160, h=120, f=150.0, partners=((0.6, 0.0, 0.0), (-0.5, 0.3, 0.1), (0.2, -0.55, 0.0))):
        self.w, self.h, self.f = w, h, f
        self.K = np.array([[f, 0, (w - 1) / 2.0], [0, f, (h - 1) / 2.0], [0, 0, 1]], np.float64)
        self.R = rot_x(0.02) @ rot_y(-0.03)
        self.C = np.zeros(3)
        self.partners = [(rot_y(-0.06 * np.sign(p[0] + 1e-9)) @ self.R, np.array(p, np.float64)) for p in partners]

    def grid(self):
        return {"K": self.K, "R": self.R, "C": self.C, "width": self.w, "height": self.h}

    def rectify(self, partner, cx_shift=12.0):
        """Rectified pair of the base camera and `partner` (R_p, C_p)."""
        Rp, Cp = partner
        b = Cp - self.C
        x = b / np.linalg.norm(b)
        z_mean = self.R[2] + Rp[2]
        z_mean /= np.linalg.norm(z_mean)
        y = np.cross(z_mean, x)
        y /= np.linalg.norm(y)
        z = np.cross(x, y)
        R_rect = np.stack([x, y, z])
        cx_l, cy = (self.w - 1) / 2.0 + 3.0, (self.h - 1) / 2.0 - 2.0
        K_rect = np.array([[self.f, 0, cx_l], [0, self.f, cy], [0, 0, 1]], np.float64)
        return {"K_rect": K_rect, "R_rect": R_rect, "baseline": float(np.linalg.norm(b)), "cx_right": cx_l - cx_shift,
                "centre": Cp}


class Plane:
    """Points X with n . X = dist."""

    def __init__(self, normal=(0.15, -0.1, -1.0), point=(0.0, 0.0, 6.0)):
        n = np.asarray(normal, np.float64)
        self.n = n / np.linalg.norm(n)
        self.dist = float(self.n @ np.asarray(point, np.float64))

    def depth_along(self, origin, direction):
        """t with origin + t * direction on the plane."""
        return (self.dist - self.n @ origin) / (direction @ self.n)


def plane_disparity(rig: Rig, pair: dict, plane: Plane, shift: float = 0.0) -> np.ndarray:
    """Disparity of the plane in the rectified left image (rig-sized)."""
    K_inv = np.linalg.inv(pair["K_rect"])
    ys, xs = np.mgrid[0:rig.h, 0:rig.w].astype(np.float64)
    pix = np.stack([xs, ys, np.ones_like(xs)], -1)
    dirs = pix @ (pair["R_rect"].T @ K_inv).T  # world directions with unit rectified depth
    t = (plane.dist - plane.n @ rig.C) / (dirs @ plane.n)
    fb = pair["K_rect"][0, 0] * pair["baseline"]
    offset = pair["K_rect"][0, 2] - pair["cx_right"]
    d = fb / t + offset + shift
    d[~(t > 0)] = np.inf
    return d.astype(np.float32)


def grid_plane_depth(rig: Rig, plane: Plane) -> np.ndarray:
    """Depth along the grid camera's optical axis of the plane at every grid pixel."""
    K_inv = np.linalg.inv(rig.K)
    ys, xs = np.mgrid[0:rig.h, 0:rig.w].astype(np.float64)
    pix = np.stack([xs, ys, np.ones_like(xs)], -1)
    dirs = pix @ (rig.R.T @ K_inv).T
    return (plane.dist - plane.n @ rig.C) / (dirs @ plane.n)


# ---------------------------------------------------------------- depth-stage scene
# Views on an arc around a textured slanted plane, for the depth stage after
# the combination (refinement and consistency): each view's camera, its gray
# image (a sum of plane-coordinate sine waves scaled to about 11 px per
# wavelength at any resolution), an SGM-like depth map (constant per 4 x 4
# block times a smooth error of up to 1 %, as the reference's refinement test
# builds, tests/test_mvs.cpp:459-466), its colour, and the 4 nearest views as
# refinement partners and consistency neighbours.
DEPTH_WAVES = ((31.0, 7.0, 0.3), (-11.0, 23.0, 1.1), (5.0, -13.0, 2.0), (43.0, 29.0, 0.7), (-37.0, 47.0, 2.9))


def depth_stage_scene(n_views: int, width: int, height: int, partners: int = 4) -> dict:
    f = 0.9 * width
    target = np.array([0.0, 0.0, 5.0])
    normal = np.array([0.35, -0.2, -1.0])
    normal /= np.linalg.norm(normal)
    wave_scale = f / 280.0
    u = np.cross(normal, [0.0, 1.0, 0.0])
    u /= np.linalg.norm(u)
    v = np.cross(normal, u)
    views = []
    y, x = np.mgrid[0:height, 0:width].astype(np.float64)
    for i in range(n_views):
        a = np.deg2rad(-18.0 + 36.0 * i / max(1, n_views - 1))
        c = np.array([5.0 * np.sin(a), 0.3 * np.cos(3.0 * a), 5.0 - 5.0 * np.cos(a)])
        z = target - c
        z /= np.linalg.norm(z)
        xa = np.cross([0.0, 1.0, 0.0], z)
        xa /= np.linalg.norm(xa)
        r = np.stack([xa, np.cross(z, xa), z])
        cam = {"width": width, "height": height, "fx": f, "fy": f, "cx": (width - 1) / 2 + 0.4,
               "cy": (height - 1) / 2 - 0.3, "rotation": r, "center": c}
        d = np.stack([(x - cam["cx"]) / f, (y - cam["cy"]) / f, np.ones_like(x)], -1) @ r
        t = ((target - c) @ normal) / (d @ normal)
        pts = c + t[..., None] * d - target
        pu, pv = pts @ u, pts @ v
        acc = np.zeros_like(x)
        for kx, ky, ph in DEPTH_WAVES:
            acc += np.sin(wave_scale * (kx * pu + ky * pv) + ph)
        gray = (128.0 + 20.0 * acc).astype(np.float32)
        depth_true = (t * d[..., 2]).astype(np.float32)  # depth along the optical axis
        block = depth_true[np.minimum(y.astype(int) // 4 * 4 + 2, height - 1),
                           np.minimum(x.astype(int) // 4 * 4 + 2, width - 1)]
        depth = (block * (1.0 + 0.01 * np.sin(x / 9.0) * np.cos(y / 13.0))).astype(np.float32)
        g8 = np.clip(gray, 0, 255).astype(np.uint8)
        views.append({"camera": cam, "gray": gray, "depth": depth, "depth_true": depth_true,
                      "color": np.repeat(g8[..., None], 3, axis=2)})
    order = [sorted((j for j in range(n_views) if j != i), key=lambda j: (abs(j - i), j))[:partners]
             for i in range(n_views)]
    return {"views": views, "partners": order}


# ---------------------------------------------------------------- a view's depth map on the device
class CViewPair(ctypes.Structure):
    """r3dgpu_view_pair: one partner pair of r3dgpu_compute_depth_map."""

    _fields_ = [
        ("partner", CViewU16),
        ("partner_camera", CCamera),
        ("base_from_rect", ctypes.c_double * 9),
        ("partner_from_rect", ctypes.c_double * 9),
        ("left", CPinhole),
        ("right", CPinhole),
        ("disparity_min", ctypes.c_int32),
        ("num_disparities", ctypes.c_int32),
        ("geometry", CPairGeometry),
    ]


def pipeline_scene(w: int, h: int, f: float, partners, seed: int = 0, plane=None):
    """A base view and partners of Rig looking at a textured plane: source
    images (u16, pinhole cameras), each pair's rectification (rotations
    R_source R_rect^T, rectified cameras), disparity range and combination
    geometry. Returns (rig, base image, list of pair dicts)."""
    rig = Rig(w=w, h=h, f=f, partners=partners)
    plane = plane or Plane()
    rng = np.random.default_rng(seed)
    u = np.cross(plane.n, [0.0, 1.0, 0.0])
    u /= np.linalg.norm(u)
    v = np.cross(plane.n, u)
    scale = f / 150.0 * 8.0

    def render(R, C):
        K_inv = np.linalg.inv(rig.K)
        ys, xs = np.mgrid[0:h, 0:w].astype(np.float64)
        dirs = np.stack([xs, ys, np.ones_like(xs)], -1) @ (R.T @ K_inv).T
        t = (plane.dist - plane.n @ C) / (dirs @ plane.n)
        pts = C + t[..., None] * dirs
        pu, pv = pts @ u, pts @ v
        acc = np.zeros_like(xs)
        for kx, ky, ph in DEPTH_WAVES:
            acc += np.sin(scale * (kx * pu + ky * pv) / 4.0 + ph)
        img = 128.0 + 22.0 * acc + rng.normal(0, 1.5, acc.shape)
        return (np.clip(img, 0, 255).astype(np.uint16) * 257).astype(np.uint16)

    base = render(rig.R, rig.C)
    pairs = []
    for (Rp, Cp) in rig.partners:
        rp = rig.rectify((Rp, Cp))
        d = plane_disparity(rig, rp, plane)
        fin = d[np.isfinite(d)]
        dmin = int(np.floor(fin.min())) - 8
        nd = (int(np.ceil(fin.max())) + 8 - dmin + 1 + 15) // 16 * 16
        K = rp["K_rect"]
        pairs.append(dict(rp, image=render(Rp, Cp), R_partner=Rp, disparity_min=dmin, num_disparities=nd,
                          left={"width": w, "height": h, "fx": K[0, 0], "fy": K[1, 1], "cx": K[0, 2], "cy": K[1, 2]},
                          right={"width": w, "height": h, "fx": K[0, 0], "fy": K[1, 1], "cx": rp["cx_right"],
                                 "cy": K[1, 2]}))
    return rig, base, pairs


# ---------------------------------------------------------------- an arc of views around textured planes
# A multi-view scene of the full depth stage: n pinhole views on a circular
# arc of radius `radius_m` (2 m) spanning `arc_deg` (neighbours about 3 degrees
# apart for 32 views, so the 4 nearest partners see a pixel under 3 to 7
# degrees, around the combination's minimum triangulation angle) looking at
# the scene centre,
# and `planes` textured rectangles: a back wall behind the centre (so every
# ray meets a surface) and random rectangles in front of it. Every rectangle
# carries its own texture made like the matcher's synthetic pairs: uniform
# noise, Gaussian-blurred with sigma 1.5 texels and stretched to 0..255,
# sampled bilinearly (wrapping) at `texel_m` per texel (by default about
# one texel per pixel at the centre's distance, 1.1 mm for 2048 pixels). Each view gets its
# image (u8, Gaussian noise sigma 2 added), its true depth, and its
# `partners` nearest views on the arc with the pair rectification, disparity
# range and combination geometry that compute_depth_map takes ("image" is
# the 8-bit image lifted to 16 bits, v * 257, as the matcher reads 8-bit
# files; "image8" the 8-bit one). Rendering
# runs in torch on `device` (CPU or CUDA); numbers other than the images are
# float64 numpy.


def _noise_texture(rng, size: int) -> np.ndarray:
    t = rng.random((size, size))
    r = np.arange(-5, 6)
    k = np.exp(-0.5 * (r / 1.5) ** 2)
    k /= k.sum()
    for axis in (0, 1):
        t = np.apply_along_axis(lambda v: np.convolve(np.concatenate([v[-5:], v, v[:5]]), k, mode="valid"), axis, t)
    t = (t - t.min()) / max(t.max() - t.min(), 1e-12) * 255.0
    return t.astype(np.float32)


def _look_at(c, target, up=(0.0, 1.0, 0.0)):
    z = np.asarray(target, np.float64) - c
    z /= np.linalg.norm(z)
    x = np.cross(np.asarray(up, np.float64), z)
    x /= np.linalg.norm(x)
    return np.stack([x, np.cross(z, x), z])


def arc_scene(n_views: int = 32, width: int = 2048, height: int = 1536, planes: int = 20, partners: int = 4,
              seed: int = 0, arc_deg: float = 100.0, radius_m: float = 2.0, texel_m: float | None = None, device=None,
              label_margin: int = 8) -> dict:
    import torch

    dev = torch.device(device or "cpu")
    rng = np.random.default_rng(seed)
    f = 0.9 * width
    if texel_m is None:
        texel_m = radius_m / f  # about one texel per pixel at the scene centre's distance
    K = np.array([[f, 0.0, (width - 1) / 2.0], [0.0, f, (height - 1) / 2.0], [0.0, 0.0, 1.0]])
    centre = np.zeros(3)
    # Rectangles: centre p, in-plane axes e1, e2 (unit), half sizes.
    rects = [(np.array([0.0, 0.0, 1.2]), np.array([1.0, 0.0, 0.0]), np.array([0.0, 1.0, 0.0]), 12.0, 9.0)]
    while len(rects) < planes:
        p = rng.uniform([-0.6, -0.45, -0.6], [0.6, 0.45, 0.6])
        n = np.array([rng.uniform(-0.6, 0.6), rng.uniform(-0.5, 0.5), -1.0])
        n /= np.linalg.norm(n)
        a = rng.uniform(0.0, np.pi)
        e1 = np.cross(n, [0.0, 1.0, 0.0])
        e1 /= np.linalg.norm(e1)
        e2 = np.cross(n, e1)
        e1, e2 = np.cos(a) * e1 + np.sin(a) * e2, -np.sin(a) * e1 + np.cos(a) * e2
        rects.append((p, e1, e2, rng.uniform(0.1, 0.35), rng.uniform(0.1, 0.35)))
    tex_size = 512
    textures = torch.from_numpy(np.stack([_noise_texture(rng, tex_size) for _ in rects])).to(dev)
    span = np.deg2rad(arc_deg)
    cams = []
    for i in range(n_views):
        a = -span / 2 + span * i / max(1, n_views - 1)
        c = np.array([radius_m * np.sin(a), 0.03 * radius_m * np.sin(5.0 * a + 0.3), -radius_m * np.cos(a)])
        cams.append({"K": K, "R": _look_at(c, centre), "C": c, "width": width, "height": height})

    ys, xs = torch.meshgrid(torch.arange(height, device=dev, dtype=torch.float64),
                            torch.arange(width, device=dev, dtype=torch.float64), indexing="ij")
    pix = torch.stack([xs, ys, torch.ones_like(xs)], -1)
    noise_rng = torch.Generator(device="cpu").manual_seed(seed + 1)

    def render(cam):
        m = torch.from_numpy(cam["R"].T @ np.linalg.inv(K)).to(dev)
        d = pix @ m.T  # world directions, unit depth along the optical axis
        C = torch.from_numpy(cam["C"]).to(dev)
        best_t = torch.full((height, width), float("inf"), dtype=torch.float64, device=dev)
        best_i = torch.full((height, width), -1, dtype=torch.int64, device=dev)
        best_u = torch.zeros_like(best_t)
        best_v = torch.zeros_like(best_t)
        for k, (p, e1, e2, hw, hh) in enumerate(rects):
            n = np.cross(e1, e2)
            nt = torch.from_numpy(n).to(dev)
            den = d @ nt
            t = (float(n @ p) - float(n @ cam["C"])) / den
            pts = C + t[..., None] * d - torch.from_numpy(p).to(dev)
            u = pts @ torch.from_numpy(e1).to(dev)
            v = pts @ torch.from_numpy(e2).to(dev)
            hit = (t > 0) & (u.abs() <= hw) & (v.abs() <= hh) & (t < best_t)
            best_t = torch.where(hit, t, best_t)
            best_i = torch.where(hit, torch.full_like(best_i, k), best_i)
            best_u = torch.where(hit, u, best_u)
            best_v = torch.where(hit, v, best_v)
        # Bilinear texture sample with wrap-around.
        tu = (best_u / texel_m) % tex_size
        tv = (best_v / texel_m) % tex_size
        u0, v0 = torch.floor(tu).long(), torch.floor(tv).long()
        fu, fv = (tu - u0).float(), (tv - v0).float()
        u1, v1 = (u0 + 1) % tex_size, (v0 + 1) % tex_size
        ti = best_i.clamp(min=0)
        flat = textures.reshape(len(rects), -1)

        def tap(vv, uu):
            return flat[ti, vv * tex_size + uu]

        val = ((1 - fu) * (1 - fv) * tap(v0, u0) + fu * (1 - fv) * tap(v0, u1) + (1 - fu) * fv * tap(v1, u0) +
               fu * fv * tap(v1, u1))
        noise = torch.randn((height, width), generator=noise_rng).to(dev) * 2.0
        img = torch.clamp(torch.round(val + noise), 0, 255).to(torch.uint8)
        img = torch.where(best_i >= 0, img, torch.zeros_like(img))
        # Depth along the optical axis (d has unit depth).
        return img.cpu().numpy(), best_t.float().cpu().numpy()

    views = []
    for cam in cams:
        img, depth = render(cam)
        views.append({"camera": cam, "image8": img, "image": img.astype(np.uint16) * np.uint16(257), "depth": depth})
    ys_np, xs_np = np.mgrid[0:height, 0:width].astype(np.float64)
    sub = (slice(None, None, 8), slice(None, None, 8))
    for i, v in enumerate(views):
        order = sorted((j for j in range(n_views) if j != i), key=lambda j: (abs(j - i), j))[:partners]
        base = v["camera"]
        # 3-D points of a sub-grid of the view (true depths) for the disparity ranges.
        dirs = np.stack([xs_np[sub], ys_np[sub], np.ones_like(xs_np[sub])], -1) @ (base["R"].T @ np.linalg.inv(K)).T
        pts = base["C"] + v["depth"][sub].astype(np.float64)[..., None] * dirs
        pairs = []
        for j in order:
            other = views[j]["camera"]
            b = other["C"] - base["C"]
            x = b / np.linalg.norm(b)
            z_mean = base["R"][2] + other["R"][2]
            z_mean /= np.linalg.norm(z_mean)
            y = np.cross(z_mean, x)
            y /= np.linalg.norm(y)
            R_rect = np.stack([x, y, np.cross(x, y)])
            K_rect = K.copy()
            q = (pts - base["C"]) @ R_rect.T
            xl = f * q[..., 0] / q[..., 2] + K_rect[0, 2]
            d_true = f * np.linalg.norm(b) / q[..., 2]
            inside = (q[..., 2] > 0) & (xl >= 0) & (xl < width)
            d_true = d_true[inside]
            # The right camera's principal point moves the disparities to start near label_margin.
            cx_right = K_rect[0, 2] - (label_margin - float(np.percentile(d_true, 0.5)))
            offset = K_rect[0, 2] - cx_right
            lo, hi = np.percentile(d_true, 0.5) + offset, np.percentile(d_true, 99.5) + offset
            dmin = int(np.floor(lo)) - label_margin
            nd = (int(np.ceil(hi)) + label_margin - dmin + 1 + 15) // 16 * 16
            pairs.append({"K_rect": K_rect, "R_rect": R_rect, "baseline": float(np.linalg.norm(b)),
                          "cx_right": cx_right, "centre": other["C"], "partner": j,
                          "image": views[j]["image"], "R_partner": other["R"], "disparity_min": dmin,
                          "num_disparities": nd,
                          "left": {"width": width, "height": height, "fx": f, "fy": f, "cx": K_rect[0, 2],
                                   "cy": K_rect[1, 2]},
                          "right": {"width": width, "height": height, "fx": f, "fy": f, "cx": cx_right,
                                    "cy": K_rect[1, 2]}})
        v["pairs"] = pairs
        v["partners"] = order
    return {"views": views, "K": K}
