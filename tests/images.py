"""Synthetic inputs of the reference's stereo tests, restated (test fixtures).

``Rng`` reproduces r3d::test::Rng (rhiestan/Regard3D_MVS, tests/test_util.hpp:19-39):
std::mt19937 with the portable uniform / integer / Box-Muller normal. ``Texture``
and ``render_pair`` follow tests/test_stereo.cpp:18-65 (sum of 24 random
sinusoids; right image rendered by fixed-point inversion of x_r = x_l - d).
Values may differ from the reference's doubles in the last bits (numpy vs
libm sin), which does not matter: every test compares implementations on the
same arrays.
"""

from __future__ import annotations

import math

import numpy as np


class Rng:
    def __init__(self, seed: int):
        self._bg = np.random.MT19937(0)
        self._bg._legacy_seeding(int(seed))

    def _next(self) -> int:
        return int(self._bg.random_raw(1)[0])

    def uniform(self, lo: float, hi: float) -> float:
        return lo + (hi - lo) * ((self._next() + 0.5) / 4294967296.0)

    def uniform_int(self, lo: int, hi: int) -> int:
        return lo + self._next() % (hi - lo + 1)

    def normal(self, mean: float, sigma: float) -> float:
        u1 = self.uniform(0.0, 1.0)
        u2 = self.uniform(0.0, 1.0)
        return mean + sigma * math.sqrt(-2.0 * math.log(u1)) * math.cos(6.283185307179586 * u2)

    def uniform_ints(self, lo: int, hi: int, n: int) -> np.ndarray:
        raw = self._bg.random_raw(n).astype(np.uint64)
        return (lo + (raw % np.uint64(hi - lo + 1)).astype(np.int64)).astype(np.int64)


class Texture:
    def __init__(self, seed: int):
        r = Rng(seed)
        self.fx, self.fy, self.phase, self.amp = [], [], [], []
        for i in range(24):
            fxm = r.uniform(0.05, 0.9)
            self.fx.append(fxm * r.uniform(-1.0, 1.0))
            fym = r.uniform(0.05, 0.9)
            self.fy.append(fym * r.uniform(-1.0, 1.0))
            self.phase.append(r.uniform(0.0, 6.283))
            self.amp.append(1.0 / (1.0 + i * 0.2))
        self.norm = sum(self.amp)

    def __call__(self, x, y):
        x = np.asarray(x, dtype=np.float64)
        y = np.asarray(y, dtype=np.float64)
        v = np.zeros(np.broadcast(x, y).shape)
        for fx, fy, ph, a in zip(self.fx, self.fy, self.phase, self.amp):
            v = v + a * np.sin(fx * x + fy * y + ph)
        return 32768.0 + 30000.0 * v / self.norm * 2.0


def to_u16(v) -> np.ndarray:
    v = np.clip(np.asarray(v, dtype=np.float64), 0.0, 65535.0)
    # std::lround: halves away from zero (values are non-negative here).
    return np.floor(v + 0.5).astype(np.uint16)


def render_pair(tex: Texture, w: int, h: int, disparity):
    """tests/test_stereo.cpp:44-63: left = texture, right(x) = texture(x_l)
    with x_l - d(x_l) = x (20 fixed-point iterations); returns left, right, gt."""
    y, x = np.mgrid[0:h, 0:w].astype(np.float64)
    left = to_u16(tex(x, y))
    gt = np.asarray(disparity(x, y), dtype=np.float32) * np.ones((h, w), np.float32)
    xl = x.copy()
    for _ in range(20):
        xl = x + disparity(xl, y)
    right = to_u16(tex(xl, y))
    return left, right, gt


def random_image(w: int, h: int, seed: int) -> np.ndarray:
    """tests/test_stereo.cpp:65-71: uniform 16-bit noise from Rng."""
    r = Rng(seed)
    return r.uniform_ints(0, 65535, w * h).reshape(h, w).astype(np.uint16)


def same_disparities(a: np.ndarray, b: np.ndarray) -> bool:
    """tests/test_stereo.cpp:73-81: equal values, or both invalid."""
    if a.shape != b.shape:
        return False
    fa, fb = np.isfinite(a), np.isfinite(b)
    return bool(np.array_equal(fa, fb) and np.array_equal(a[fa], b[fb]))


def mismatch_report(a: np.ndarray, b: np.ndarray, n: int = 5) -> str:
    bad = ~((a == b) | (~np.isfinite(a) & ~np.isfinite(b)))
    ys, xs = np.nonzero(bad)
    items = [f"({y},{x}): {a[y, x]} vs {b[y, x]}" for y, x in list(zip(ys, xs))[:n]]
    return f"{int(bad.sum())} mismatches; " + "; ".join(items)


def evaluate_disparity(est: np.ndarray, gt: np.ndarray, mask: np.ndarray | None = None, mask_min: int = 255):
    """r3d::evaluate_disparity (src/r3d/stereo/disparity_eval.cpp:11-64):
    pixels with finite ground truth and mask >= mask_min are evaluated;
    density = estimated / evaluated; bad1 and the mean absolute error over the
    estimated pixels (errors in double)."""
    valid_gt = np.isfinite(gt)
    if mask is not None:
        valid_gt &= mask >= mask_min
    n = int(valid_gt.sum())
    est_ok = valid_gt & np.isfinite(est)
    density = est_ok.sum() / max(n, 1)
    err = np.abs(est[est_ok].astype(np.float64) - gt[est_ok].astype(np.float64))
    bad1 = float((err > 1.0).sum()) / max(int(est_ok.sum()), 1)
    avg = float(err.mean()) if err.size else 0.0
    return density, bad1, avg
