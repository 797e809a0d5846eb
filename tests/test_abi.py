"""The C-ABI library builds, loads and exports every declared entry point (CPU only)."""

from __future__ import annotations

import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header: str) -> set[str]:
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(r3dgpu_[a-z0-9_]+)\s*\(", text))


@pytest.fixture(scope="module")
def cuda_lib():
    from regard3d_mvs_b200 import _native
    from regard3d_mvs_b200.build import build

    build()
    return _native.load()


def test_exports_every_declared_symbol(cuda_lib):
    names = _declared("r3dgpu.h") | _declared("r3dgpu_server.h") | _declared("r3dgpu_synth.h")
    assert len(names) >= 15
    for n in sorted(names):
        assert hasattr(cuda_lib, n), n
    from regard3d_mvs_b200 import _native

    assert set(_native.EXPORTS) <= names


def test_emulator_exports_the_same_matcher_symbols(simt_matcher):
    names = _declared("r3dgpu.h") | _declared("r3dgpu_server.h")
    for n in sorted(names):
        assert hasattr(simt_matcher.lib, n), n


def test_default_options_match_reference_defaults(cuda_lib):
    from regard3d_mvs_b200.types import COptions, StereoOptions, to_c_options

    c = COptions()
    cuda_lib.r3dgpu_default_options(ctypes.byref(c))
    ref = to_c_options(StereoOptions())
    for name, _ in COptions._fields_:
        assert getattr(c, name) == getattr(ref, name), name


def test_automatic_levels_matches_oracle(cuda_lib, oracle):
    for w, h, nd in ((640, 480, 128), (3072, 2048, 256), (480, 300, 256), (6048, 4536, 384), (100, 90, 64)):
        assert cuda_lib.r3dgpu_automatic_levels(w, h, nd) == oracle.automatic_levels(w, h, nd)


def test_synth_is_deterministic(cuda_lib):
    import numpy as np

    from regard3d_mvs_b200.types import CSynthParams

    def gen(seed):
        p = CSynthParams(96, 64, 64, seed, 1.5, 2.0, 8, 0.15, 0.10)
        L = np.empty((64, 96), np.uint8)
        R = np.empty_like(L)
        gt = np.empty((64, 96), np.float32)
        assert cuda_lib.r3dgpu_synth_pair(ctypes.byref(p), L.ctypes.data, R.ctypes.data, gt.ctypes.data) == 0
        return L, R, gt

    a, b = gen(5), gen(5)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    assert not np.array_equal(a[0], gen(6)[0])
    assert a[2].min() >= 5 and a[2].max() <= 64 - 8


def test_no_gpu_fails_loudly_or_runs(cuda_lib):
    """On a machine without a B200 the library reports an error instead of
    computing anything on the CPU."""
    try:
        import torch

        has_gpu = torch.cuda.is_available()
    except Exception:  # noqa: BLE001
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    from regard3d_mvs_b200 import Matcher, StereoError

    with pytest.raises(StereoError):
        Matcher()
