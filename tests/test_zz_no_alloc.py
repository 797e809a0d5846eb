"""r3dgpu_remove_speckles_no_alloc: the speckle filter for callers that
cannot let the library allocate GPU memory.

Such a caller (an application whose own pool allocator owns the device's
memory, or a pipeline that cannot take the device-wide synchronisation of
cudaFree) hands the library a disparity map already in device memory; the
union-find scratch comes from a static device array of the library, capped at
4,194,304 pixels. These tests call the entry point through the C ABI and
compare it with r3dgpu_remove_speckles_host, which allocates its own scratch.

The file is named to be collected last, so that a run stopping at its first
failure has already run every other test.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from images import same_disparities

MAX_PIXELS = 1 << 22


def _speckled(h, w, seed):
    rng = np.random.default_rng(seed)
    d = np.round(rng.normal(20, 3, (h, w))).astype(np.float32)
    d[rng.random(d.shape) < 0.1] = np.inf
    return d


def _status_name(lib, st):
    from regard3d_mvs_b200._native import STATUS

    return f"{STATUS.get(st, st)}: {lib.r3dgpu_last_error().decode()}"


@pytest.mark.gpu
def test_no_alloc_matches_allocating_entry_point(gpu_matcher):
    import torch

    lib = gpu_matcher.lib
    stream = torch.cuda.current_stream(0)
    # Two calls in a row on one stream: the second, smaller map finds the
    # first call's union-find state in the shared array and must not see it.
    for (h, w), size, diff, seed in (((700, 900), 40, 1.0, 11), ((90, 130), 6, 2.0, 12)):
        d = _speckled(h, w, seed)
        expected = gpu_matcher.remove_speckles(d.copy(), size, diff)
        dev = torch.from_numpy(d).to("cuda:0")
        st = lib.r3dgpu_remove_speckles_no_alloc(dev.data_ptr(), w, h, size, diff, stream.cuda_stream)
        assert st == 0, _status_name(lib, st)
        torch.cuda.synchronize(0)
        got = dev.cpu().numpy()
        assert not np.array_equal(got, d)  # the filter removed something
        assert same_disparities(got, expected)


@pytest.mark.gpu
def test_no_alloc_rejects_maps_above_the_static_maximum(gpu_matcher):
    import torch

    lib = gpu_matcher.lib
    dev = torch.zeros(16, device="cuda:0")
    # Rejected on the host before any launch: the map is never touched.
    st = lib.r3dgpu_remove_speckles_no_alloc(dev.data_ptr(), 2049, 2048, 10, 1.0, None)
    assert st == 1, _status_name(lib, st)  # R3DGPU_EINVAL
    assert "static scratch maximum" in lib.r3dgpu_last_error().decode()
    assert 2049 * 2048 > MAX_PIXELS


@pytest.mark.gpu
def test_no_alloc_rejects_memory_of_no_device(gpu_matcher):
    """The map must be device memory of the thread's device: a host array is
    rejected before any launch, and an empty call (the set-up alone) is fine."""
    lib = gpu_matcher.lib
    st = lib.r3dgpu_remove_speckles_no_alloc(None, 0, 0, 10, 1.0, None)
    assert st == 0, _status_name(lib, st)
    host = np.zeros((4, 4), np.float32)
    st = lib.r3dgpu_remove_speckles_no_alloc(host.ctypes.data_as(ctypes.c_void_p), 4, 4, 10, 1.0, None)
    assert st == 1, _status_name(lib, st)  # R3DGPU_EINVAL
    assert "not" in lib.r3dgpu_last_error().decode() and "memory" in lib.r3dgpu_last_error().decode()


def test_no_alloc_on_the_emulator(simt_matcher, oracle):
    """The same entry point on the CPU SIMT emulator, where device memory is
    host memory, against the oracle."""
    lib = simt_matcher.lib
    for (h, w), size, diff, seed in (((40, 60), 6, 1.0, 3), ((23, 31), 3, 2.0, 4)):
        d = _speckled(h, w, seed)
        got = np.ascontiguousarray(d.copy())
        st = lib.r3dgpu_remove_speckles_no_alloc(got.ctypes.data_as(ctypes.c_void_p), w, h, size, diff, None)
        assert st == 0, _status_name(lib, st)
        assert same_disparities(got, oracle.remove_speckles(d, size, diff))
    # Rejected before any work: the small buffer is never read.
    st = lib.r3dgpu_remove_speckles_no_alloc(got.ctypes.data_as(ctypes.c_void_p), 4096, 1025, 10, 1.0, None)
    assert st == 1 and "static scratch maximum" in lib.r3dgpu_last_error().decode()
