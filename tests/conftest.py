"""Shared pytest setup: the `gpu` marker, builds of the oracle and of the
kernel emulator (CPU tests), and the CUDA library (GPU tests)."""

from __future__ import annotations

import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

SIMT_DIR = os.path.join(ROOT, "tests", "simt")
SIMT_LIB = os.path.join(SIMT_DIR, "_build", "libr3dgpu_simt.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 and the CUDA build of the library")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o

    o.build()
    return o


@pytest.fixture(scope="session")
def simt_matcher():
    """The r3dgpu kernels and host code compiled for the CPU SIMT emulator."""
    subprocess.run(["make", "-s", "-C", SIMT_DIR], check=True)
    from regard3d_mvs_b200 import Matcher

    return Matcher(SIMT_LIB, host_is_device=True)


@pytest.fixture(scope="session")
def gpu_matcher():
    """The CUDA library on cuda:0 (fails loudly if it is missing)."""
    from regard3d_mvs_b200 import Matcher
    from regard3d_mvs_b200.build import build

    build()
    return Matcher()
