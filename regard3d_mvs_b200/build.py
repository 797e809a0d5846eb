"""Builds the r3dgpu CUDA library in-tree: regard3d_mvs_b200/_lib/libr3dgpu.so.

nvcc compiles every source for sm_100a only (-gencode
arch=compute_100a,code=sm_100a), with --fmad=false so that float arithmetic is
never contracted (the reference's float results are reproduced operation by
operation). Objects are compiled in parallel and linked with the static CUDA
runtime. Usage: ``python -m regard3d_mvs_b200.build [--force]``.
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
OBJ_DIR = os.path.join(HERE, "_lib", "obj")
LIB = os.path.join(OUT_DIR, "libr3dgpu.so")
SOURCES = ("image_kernels.cu", "sgm.cu", "sgm_full.cu", "sgm_path.cu", "sgm_ranged.cu", "noalloc.cu", "multi_stereo.cu", "rectify.cu", "consistency.cu", "refine.cu", "depth_io.cpp", "pipeline.cpp", "matcher.cpp", "server.cpp", "tuning.cpp", "synth.cpp")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else "nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "--fmad=false", "-std=c++17",
         "-Xcompiler", "-fPIC,-O3", "-Xptxas", "-O3"]


def _deps() -> list[str]:
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh", ".cu", ".cpp"))]
    files.append(os.path.join(HERE, "..", "include", "r3dgpu.h"))
    files.append(os.path.join(HERE, "..", "include", "r3dgpu_synth.h"))
    return files


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str) -> str:
    obj = os.path.join(OBJ_DIR, src + ".o")
    cmd = [NVCC, *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC, "-x", "cu", *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False) -> str:
    os.makedirs(OBJ_DIR, exist_ok=True)
    deps = _deps()
    if not force and not _stale(LIB, deps):
        return LIB
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(_compile, SOURCES))
    cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-cudart", "static", "-o", LIB, *objs,
           "-ldl", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
