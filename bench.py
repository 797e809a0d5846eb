#!/usr/bin/env python
"""Census+SGM throughput on B200: batched pairs vs one pair per call.

Workload (default ``batch64``): 64 rectified pairs of uneven size (width
log-uniform in 1024..6048, aspect 3:2 or 4:3), 8-bit synthetic images lifted
to 16 bit, label ranges drawn from {64, 128, 192, 256, 384}; half of the pairs
use the 4-level hierarchy with +-8 labels around the upsampled coarse
disparity (range_radius 0, range_margin 8), half a single full-range level.
A step matches the whole batch with one call of the batch C ABI. The metric
counts W*H*D cells of the full label range at level 0 per pair (the
reference's convention), in Gcells/s over the whole job.

  value  device-resident inputs and outputs, CUDA events on the launching stream
  e2e    same call with pinned host buffers: the step's host->device copies of
         all images and the device->host read of all disparity maps inside the
         timed region
  per_pair  the same pairs matched one call per pair (the plain GPU matcher)

`python bench.py --impl reference` times the CPU oracle (a restatement of the
reference matcher, all host threads) on a bounded sample of the same pairs.
Under torchrun every rank matches its own batch (weak scaling); the time is
the maximum over ranks.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Census+SGM Gcells/s (W·H·D) batched vs per-pair, bit-exact; p50/p99 latency"
ND_CHOICES = (64, 128, 192, 256, 384)
# Algorithmic HBM bytes of the SGM tile kernel: the forward partial sum S
# (u16) written once and read once per aggregated cell, plus per tile pixel
# the two Census codes read (2 x 8 B) and disparity + confidence written (8 B).
ALG_BYTES_PER_CELL = 4
ALG_BYTES_PER_PIXEL = 24
# Integer operations per aggregated cell (8 paths x ~7 ops, 8 sum adds, cost).
INT_OPS_PER_CELL = 66


def _native_check(lib, status):
    if status != 0:
        raise RuntimeError(lib.r3dgpu_last_error().decode())


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", choices=("batch64", "pair3072", "pair640", "pair1024", "pair2048", "scene32", "combine", "rectify", "depth",
                                           "view"),
                    default="batch64",
                    help="combine / rectify / depth: only the multi-view combination of one view / the "
                         "rectification resampling of one pair / the depth stage after the combination "
                         "(refinement and consistency of 8 views; each its own JSON line)")
    ap.add_argument("--pairs", type=int, default=64)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--no-per-pair", action="store_true")
    ap.add_argument("--no-plain", dest="plain", action="store_false",
                    help="skip the one-pair-per-call run with the one-CTA-per-tile kernels")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serve", dest="serve", action="store_false",
                    help="skip the serving sweep, which runs in a fresh process after the batch")
    ap.add_argument("--serve-only", type=float, default=0.0, metavar="PAIRS_PER_S",
                    help="run only the serving sweep (its saturation run offers 3 x this batch rate); print its JSON")
    ap.add_argument("--serve-seconds", type=float, default=8.0, help="arrival window per load point")
    ap.add_argument("--serve-workers", type=int, default=SERVE_WORKERS, help="serving loop workers (streams)")
    ap.add_argument("--serve-batch", type=int, default=SERVE_MAX_BATCH, help="requests per batch at most")
    return ap.parse_args()


def workload_pairs(name: str, npairs: int, seed: int):
    """(width, height, nd, options dict) per pair, deterministic."""
    rng = np.random.default_rng(seed)
    out = []
    if name == "pair640":
        return [dict(w=640, h=480, nd=128, levels=0, radius=3, margin=4, textureless=0.0, occluded=0.0, seed=seed)]
    if name == "pair1024":
        # One full-range pair, 1024x768, 128 labels (ncu captures of the pass kernels: 0.2 G cells per pass,
        # a working set of several times the L2 and under 2 GB of device memory).
        return [dict(w=1024, h=768, nd=128, levels=0, radius=3, margin=4, textureless=0.0, occluded=0.0, seed=seed)]
    if name == "pair2048":
        # One full-range 2048x1536 pair, the size of a depth-stage view (profiling case of the pass kernels).
        return [dict(w=2048, h=1536, nd=128, levels=0, radius=3, margin=4, textureless=0.0, occluded=0.0, seed=seed)]
    if name == "pair3072":
        return [dict(w=3072, h=2048, nd=256, levels=3, radius=0, margin=8, textureless=0.15, occluded=0.10,
                     seed=seed)]
    for i in range(npairs):
        w = int(round(math.exp(rng.uniform(math.log(1024), math.log(6048)))))
        aspect = 1.5 if rng.random() < 0.5 else 4.0 / 3.0
        h = int(round(w / aspect))
        nd = int(ND_CHOICES[rng.integers(0, len(ND_CHOICES))])
        hier = i % 2 == 1
        out.append(dict(w=w, h=h, nd=nd, levels=3 if hier else 0, radius=0 if hier else 3, margin=8 if hier else 4,
                        textureless=0.0, occluded=0.0, seed=seed * 1000 + i))
    return out


def make_images(lib, spec):
    from regard3d_mvs_b200.types import CSynthParams

    p = CSynthParams(spec["w"], spec["h"], spec["nd"], spec["seed"] & 0xFFFFFFFF, 1.5, 2.0, spec.get("planes", 8),
                     spec["textureless"], spec["occluded"])
    L = np.empty((spec["h"], spec["w"]), np.uint8)
    R = np.empty_like(L)
    st = lib.r3dgpu_synth_pair(ctypes.byref(p), L.ctypes.data, R.ctypes.data, None)
    if st != 0:
        raise RuntimeError(f"synth failed: {st}")
    return L.astype(np.uint16) * np.uint16(257), R.astype(np.uint16) * np.uint16(257)


def options_for(spec):
    from regard3d_mvs_b200.types import StereoOptions

    return StereoOptions(levels=spec["levels"], range_radius=spec["radius"], range_margin=spec["margin"])


def full_range_cells(specs) -> int:
    return sum(s["w"] * s["h"] * ((s["nd"] + 15) // 16 * 16) for s in specs)


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.samples = []
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        for line in out.strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)

    def summary(self):
        if not getattr(self, "samples", None):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(p[0]) for p in self.samples if p[0].replace(".", "").isdigit()]
        mx = [float(p[1]) for p in self.samples if p[1].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[k] for p in self.samples for k in range(4) if p[3 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


PASS_MODES = {0: "first pass (u16 sums)", 1: "accumulate pass (u16 sums)", 2: "last pass (u16 sums, WTA)",
              3: "term pass (byte terms)", 4: "last pass (byte terms, WTA)"}


def pass_traffic_per_cell():
    """DRAM bytes per cell of the chain-pass modes (mode number -> bytes),
    from the committed ncu summaries (profiles/sgm_path_traffic.json)."""
    path = os.path.join(ROOT, "profiles", "sgm_path_traffic.json")
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        d = json.load(f)
    return {int(k): float(v) for k, v in d.get("dram_bytes_per_cell_by_mode", {}).items()}


def pass_roofline(launch_log, peak, peak_kind):
    """Roofline of the dominant kernel, the chain pass (sgm_path_kernel):
    algorithmic bytes of its launches (costs read, sums or byte terms read and
    written, WTA records) over their CUDA-event durations on the launching
    stream; per pass mode as well."""
    passes = [e for e in launch_log if e.get("pass") and e["kernel"] == "sgm_path_kernel"]
    rpasses = [e for e in launch_log if e.get("pass") and e["kernel"] == "sgm_path_ranged_kernel"]
    if not passes:
        return None
    ms = sum(e["ms"] for e in passes)
    nbytes = sum(e["bytes"] for e in passes)
    cells = sum(e["cells"] for e in passes)
    achieved = nbytes / (ms * 1e-3) / 1e9 if ms > 0 else 0.0
    tpc = pass_traffic_per_cell()
    by_mode = {}
    for e in passes:
        mode = int(e["shape"].rsplit("mode", 1)[1])
        b = by_mode.setdefault(mode, {"what": PASS_MODES.get(mode, "?"), "launches": 0, "ms": 0.0, "bytes": 0,
                                      "cells": 0})
        b["launches"] += 1
        b["ms"] += e["ms"]
        b["bytes"] += e["bytes"]
        b["cells"] += e["cells"]
    for b in by_mode.values():
        b["gbs"] = b["bytes"] / (b["ms"] * 1e-3) / 1e9 if b["ms"] > 0 else 0.0
        b["frac"] = b["gbs"] / peak
    traffic = None
    if tpc and all(m in tpc for m in by_mode):
        traffic = sum(tpc[m] * b["cells"] for m, b in by_mode.items()) / len(passes)
    out = {"bound": "hbm", "kernel": "sgm_path_kernel (chain passes of full-range tiles; a launch runs one pass, or the seven term passes of a tile group)", "achieved": achieved,
           "peak": peak, "peak_kind": f"{peak_kind} copy bandwidth", "unit": "GB/s", "frac": achieved / peak,
           "traffic": traffic, "traffic_source": "profiles/sgm_path_traffic.json (ncu DRAM bytes per cell by mode)",
           "launches": len(passes), "avg_launch_ms": ms / len(passes), "alg_bytes_per_launch": nbytes / len(passes),
           "alg_bytes_per_cell": {"first pass": 3, "accumulate pass": 5, "last pass": "3 + 16 per pixel",
                                  "term pass": 2, "last pass (byte terms)": "8 + 16 per pixel"},
           "cells_per_launch": cells / len(passes),
           "by_mode": {str(k): v for k, v in sorted(by_mode.items())}}
    if rpasses:
        rms = sum(e["ms"] for e in rpasses)
        rb = sum(e["bytes"] for e in rpasses)
        out["ranged_pass"] = {"kernel": "sgm_path_ranged_kernel", "achieved": rb / (rms * 1e-3) / 1e9 if rms else 0.0,
                              "frac": (rb / (rms * 1e-3) / 1e9) / peak if rms else 0.0, "launches": len(rpasses),
                              "avg_launch_ms": rms / len(rpasses),
                              "alg_bytes_per_cell": "3 (first) or 5, + 16 per pixel (range record)"}
    return out


def oracle_images(spec):
    """The pair of `spec` from the generator compiled into the oracle library
    (the same source and bytes as the CUDA library's r3dgpu_synth_pair)."""
    from oracle import oracle

    L, R = oracle.synth_pair(spec["w"], spec["h"], spec["nd"], spec["seed"], spec["textureless"], spec["occluded"])
    return L.astype(np.uint16) * np.uint16(257), R.astype(np.uint16) * np.uint16(257)


def cpu_baseline(specs, gpu_maps=None):
    """The oracle on a bounded sample: the smallest pair of the workload,
    full matcher, all host threads. With `gpu_maps` (index -> the GPU
    disparity map of that pair from the timed batch) the oracle's map is also
    compared with the GPU's, bit for bit."""
    from oracle import oracle

    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    idx = min(range(len(specs)), key=lambda i: specs[i]["w"] * specs[i]["h"] * specs[i]["nd"])
    spec = specs[idx]
    L, R = oracle_images(spec)
    t0 = time.perf_counter()
    r = oracle.match_stereo(L, R, None, None, 0, spec["nd"], options_for(spec))
    dt = time.perf_counter() - t0
    cells = spec["w"] * spec["h"] * ((spec["nd"] + 15) // 16 * 16)
    out = {"value": cells / dt / 1e9, "unit": "Gcells/s", "cores": threads, "kind": "port",
           "sample": f"pair {idx}: one {spec['w']}x{spec['h']} pair, {spec['nd']} labels, levels {spec['levels']}, "
                     f"{dt:.2f} s, {r.cells} aggregated cells"}
    if gpu_maps is not None and idx in gpu_maps:
        g = gpu_maps[idx]
        fa, fb = np.isfinite(g), np.isfinite(r.disparity)
        out["bit_exact_vs_oracle"] = bool(np.array_equal(fa, fb) and np.array_equal(g[fa], r.disparity[fb]))
        out["bit_exact_pair"] = idx
    return out


def run_reference(args, rank, world):
    """The CPU oracle (restatement of the reference matcher, all host threads)
    on the workload's own pairs, uncropped: each timed step matches the next
    pair of the list (pairs 0 .. steps - 1); the warm-up steps match the
    smallest pair. Inputs come from the generator compiled into the oracle
    library, so no library of the GPU build is loaded."""
    if rank != 0:
        return
    from oracle import oracle

    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    specs = workload_pairs(args.workload, args.pairs, args.seed)
    small = min(specs, key=lambda s: s["w"] * s["h"] * s["nd"])
    cells = 0
    elapsed = 0.0
    aggregated = 0
    for i in range(args.warmup + args.steps):
        s = small if i < args.warmup else specs[(i - args.warmup) % len(specs)]
        L, R = oracle_images(s)
        t0 = time.perf_counter()
        r = oracle.match_stereo(L, R, None, None, 0, s["nd"], options_for(s))
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            elapsed += dt
            cells += s["w"] * s["h"] * ((s["nd"] + 15) // 16 * 16)
            aggregated += r.cells
    value = cells / elapsed / 1e9
    sample = (f"pairs 0..{args.steps - 1} of the {args.workload} list, uncropped, one pair per step "
              f"({aggregated} aggregated cells); warm-up on its smallest pair")
    line = {"metric": METRIC, "value": value, "unit": "Gcells/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": "synthetic",
            "config": {"workload": args.workload, "sample": sample, "same_pairs_as_gpu_arm": True},
            "cpu_baseline": {"value": value, "unit": "Gcells/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "Gcells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# Multi-view combination (r3dgpu_combine_pairs) of one view: 2048 x 1536 grid,
# 4 partner pairs. Algorithmic bytes per grid pixel: per pair one disparity
# and one confidence sample (4 + 4 B), plus depth, confidence and pair mask
# written (4 + 4 + 2 B).
COMBINE_W, COMBINE_H, COMBINE_PAIRS = 2048, 1536, 4
COMBINE_BYTES_PER_PIXEL = COMBINE_PAIRS * 8 + 10


def measure_combine(lib, dev, stream, steps: int, warmup: int, peak: float) -> dict:
    """Device time of the combination of 4 matched pairs into a depth map,
    the oracle's time on the same view (all host threads) beside it."""
    import torch

    from oracle import oracle as orc
    from regard3d_mvs_b200.multi_view import Plane, Rig, c_grid, c_pairs, plane_disparity
    from regard3d_mvs_b200.types import CPairGeometry, MultiStereoOptions

    rig = Rig(w=COMBINE_W, h=COMBINE_H, f=1800.0,
              partners=((0.6, 0.0, 0.0), (-0.5, 0.3, 0.1), (0.2, -0.55, 0.0), (-0.3, -0.4, 0.2)))
    plane = Plane()
    rng = np.random.default_rng(3)
    pairs = []
    for p, shift in zip(rig.partners, (0.0, 0.5, 6.0, 0.0)):
        q = rig.rectify(p)
        d = plane_disparity(rig, q, plane, shift)
        d += rng.normal(0, 0.3, d.shape).astype(np.float32)
        d[rng.random(d.shape) < 0.08] = np.inf
        q["disparity"] = d
        q["confidence"] = rng.random(d.shape).astype(np.float32)
        pairs.append(q)
    grid = rig.grid()
    g = c_grid(grid)
    harr, keep = c_pairs(grid, pairs)
    darr = (CPairGeometry * COMBINE_PAIRS)()
    dev_maps = []
    for i, q in enumerate(pairs):
        darr[i] = harr[i]
        dd = torch.from_numpy(q["disparity"]).to(dev)
        dc = torch.from_numpy(q["confidence"]).to(dev)
        dev_maps += [dd, dc]
        darr[i].disparity, darr[i].confidence = dd.data_ptr(), dc.data_ptr()
    depth = torch.empty((COMBINE_H, COMBINE_W), dtype=torch.float32, device=dev)
    conf = torch.empty_like(depth)
    mask = torch.empty((COMBINE_H, COMBINE_W), dtype=torch.int16, device=dev)
    o = MultiStereoOptions().c()
    sptr = ctypes.c_void_p(stream.cuda_stream)

    def run():
        _native_check(lib, lib.r3dgpu_combine_pairs(ctypes.byref(g), darr, COMBINE_PAIRS, ctypes.byref(o),
                                                    depth.data_ptr(), conf.data_ptr(), mask.data_ptr(), COMBINE_W,
                                                    sptr))

    for _ in range(warmup):
        run()
    torch.cuda.synchronize(dev)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        run()
    b.record(stream)
    torch.cuda.synchronize(dev)
    ms = a.elapsed_time(b) / steps
    px = COMBINE_W * COMBINE_H
    achieved = COMBINE_BYTES_PER_PIXEL * px / (ms * 1e-3) / 1e9
    t0 = time.perf_counter()
    ref = orc.combine_pairs(grid, pairs)
    cpu_s = time.perf_counter() - t0
    same = bool(np.array_equal(ref.depth, depth.cpu().numpy()))
    return {"workload": f"combine_pairs, {COMBINE_W}x{COMBINE_H} grid, {COMBINE_PAIRS} pairs, plane + noise",
            "value": px / (ms * 1e-3) / 1e9, "unit": "Gpixels/s", "ms": ms, "bit_exact_vs_oracle": same,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "alg_bytes_per_pixel": COMBINE_BYTES_PER_PIXEL},
            "cpu_baseline": {"value": px / cpu_s / 1e9, "unit": "Gpixels/s", "cores": orc.max_threads(),
                             "kind": "port", "sample": "the same view, once"}}


# Rectification resampling (r3dgpu_rectify_image_u16) of both images of a
# pair: 6000 x 4000 u16 photos with brown_t2 distortion into rectified
# cameras of the same focal length (pyramid level 0), 6120 x 4080 targets.
# Algorithmic bytes per launch: the source read once (2 B per source pixel),
# the target image and validity mask written (2 + 1 B per target pixel).
RECT_W, RECT_H = 6000, 4000
RECT_TW, RECT_TH = 6120, 4080
RECT_BYTES_PER_LAUNCH = 2 * RECT_W * RECT_H + 3 * RECT_TW * RECT_TH
L2_FLUSH_BYTES = 256 << 20


def rectify_setup():
    """Cameras, rotations and source images of the rectified pair."""
    from regard3d_mvs_b200.multi_view import rot_x, rot_y

    cams, rots, srcs = [], [], []
    rng = np.random.default_rng(5)
    for i, (ry, rx) in enumerate(((0.04, -0.015), (-0.035, 0.01))):
        cams.append({"model": 3, "width": RECT_W, "height": RECT_H, "fx": 5200.0, "fy": 5203.0,
                     "cx": (RECT_W - 1) / 2 + 11 - 4 * i, "cy": (RECT_H - 1) / 2 - 6,
                     "params": (-0.09, 0.03, -0.004, 0.0008, -0.0011)})
        rots.append((rot_y(ry) @ rot_x(rx)) @ rot_x(0.012).T)
        y, x = np.mgrid[0:RECT_H, 0:RECT_W]
        img = 32768 + 12000 * np.sin(x / 23.0 + i) * np.cos(y / 17.0) + rng.normal(0, 3000, (RECT_H, RECT_W))
        srcs.append(np.clip(img, 0, 65535).astype(np.uint16))
    target = {"width": RECT_TW, "height": RECT_TH, "fx": 5200.0, "fy": 5200.0, "cx": (RECT_TW - 1) / 2,
              "cy": (RECT_TH - 1) / 2 + 2}
    return cams, rots, srcs, target


def measure_rectify(lib, dev, stream, steps: int, warmup: int, peak: float) -> dict:
    """Device time of rectify_image on both images of a pair (L2 flushed
    before each launch), end-to-end time through the host entry point, and
    the oracle on the host's cores on one image."""
    import torch

    from oracle import oracle as orc
    from regard3d_mvs_b200.types import CViewU16, camera_struct, pinhole_struct

    cams, rots, srcs, target = rectify_setup()
    k = pinhole_struct(target)
    cs = [camera_struct(c) for c in cams]
    ms_ = [np.ascontiguousarray(r).reshape(9) for r in rots]
    dsrc = [torch.from_numpy(a.view(np.int16)).to(dev) for a in srcs]
    views = [CViewU16(d.data_ptr(), RECT_W, RECT_H, RECT_W) for d in dsrc]
    dout = [torch.empty((RECT_TH, RECT_TW), dtype=torch.int16, device=dev) for _ in srcs]
    dval = [torch.empty((RECT_TH, RECT_TW), dtype=torch.uint8, device=dev) for _ in srcs]
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    sptr = ctypes.c_void_p(stream.cuda_stream)

    def run(i):
        _native_check(lib, lib.r3dgpu_rectify_image_u16(ctypes.byref(views[i]), ctypes.byref(cs[i]),
                                                        ms_[i].ctypes.data, ctypes.byref(k), dout[i].data_ptr(),
                                                        RECT_TW, dval[i].data_ptr(), RECT_TW, sptr))

    for _ in range(warmup):
        run(0)
        run(1)
    torch.cuda.synchronize(dev)
    total_ms = 0.0
    launches0 = int(lib.r3dgpu_launch_count())
    for _ in range(steps):
        for i in range(2):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            run(i)
            b.record(stream)
            torch.cuda.synchronize(dev)
            total_ms += a.elapsed_time(b)
    launches = int(lib.r3dgpu_launch_count()) - launches0
    ms = total_ms / (2 * steps)  # per launch
    px = RECT_TW * RECT_TH
    achieved = RECT_BYTES_PER_LAUNCH / (ms * 1e-3) / 1e9

    # End to end through the host entry point: pinned host source in, image
    # and mask out, every step.
    hsrc = [torch.from_numpy(a.view(np.int16)).pin_memory() for a in srcs]
    hout = [torch.empty((RECT_TH, RECT_TW), dtype=torch.int16).pin_memory() for _ in srcs]
    hval = [torch.empty((RECT_TH, RECT_TW), dtype=torch.uint8).pin_memory() for _ in srcs]
    hviews = [CViewU16(h.data_ptr(), RECT_W, RECT_H, RECT_W) for h in hsrc]

    def run_host(i):
        _native_check(lib, lib.r3dgpu_rectify_image_u16_host(ctypes.byref(hviews[i]), ctypes.byref(cs[i]),
                                                             ms_[i].ctypes.data, ctypes.byref(k), hout[i].data_ptr(),
                                                             RECT_TW, hval[i].data_ptr(), RECT_TW))

    for _ in range(max(1, warmup)):
        run_host(0)
        run_host(1)
    t0 = time.perf_counter()
    for _ in range(steps):
        run_host(0)
        run_host(1)
    e2e_s = (time.perf_counter() - t0) / (2 * steps)

    got = [dout[i].cpu().numpy().view(np.uint16) for i in range(2)]
    t0 = time.perf_counter()
    ref, ref_valid = orc.rectify_image(srcs[0], cams[0], rots[0], target)
    cpu_s = time.perf_counter() - t0
    same = bool(np.array_equal(ref, got[0]) and np.array_equal(ref_valid, dval[0].cpu().numpy())
                and np.array_equal(hout[1].numpy().view(np.uint16), got[1]))
    return {"workload": f"rectify_image u16, brown_t2 {RECT_W}x{RECT_H} -> {RECT_TW}x{RECT_TH}, level 0, "
                        "both images of a pair",
            "value": px / (ms * 1e-3) / 1e9, "unit": "Gpixels/s", "ms_per_launch": ms, "gpu_launches": launches,
            "bit_exact_vs_oracle": same, "l2": f"flushed before each launch ({L2_FLUSH_BYTES >> 20} MiB write)",
            "e2e": {"value": px / e2e_s / 1e9, "unit": "Gpixels/s", "h2d_bytes_per_step": 2 * 2 * RECT_W * RECT_H,
                    "d2h_bytes_per_step": 2 * 3 * px},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "alg_bytes_per_launch": RECT_BYTES_PER_LAUNCH},
            "cpu_baseline": {"value": px / cpu_s / 1e9, "unit": "Gpixels/s", "cores": orc.max_threads(),
                             "kind": "port", "sample": "one image of the pair, once"}}


# Depth stage after the combination (refinement and consistency):
# 8 views of 2048 x 1536, each refined against its 4 nearest views with a
# 7 x 7 window (radius 3, step 1), then one consistency filter of all 8 maps
# (4 neighbours each). Algorithmic bytes per view: its refinement image and
# the 4 partners' (12 B per pixel each), depth and confidence in and out
# (16 B per pixel), the consistency pass over depth, pair mask, colour and
# support (about 20 B per pixel): about 96 B per pixel.
DEPTH_VIEWS, DEPTH_W, DEPTH_H = 8, 2048, 1536
DEPTH_BYTES_PER_PIXEL = 96
DEPTH_CROP = (512, 384)


def measure_depth(lib, dev, stream, steps: int, warmup: int, peak: float) -> dict:
    """Device time of the depth stage of 8 views (float and double refinement
    paths), end-to-end time through the host entry points, the float path's
    depth error against the double-precision oracle, and the oracle's time,
    both on a crop of one view."""
    import torch

    from oracle import oracle as orc
    from regard3d_mvs_b200.depth_maps import (CConsistencyStats, CDepthMap, ConsistencyOptions, CRefinementImage,
                                              CRefinementStats, RefinementOptions, c_camera, neighbour_lists)
    from regard3d_mvs_b200.multi_view import depth_stage_scene

    scene = depth_stage_scene(DEPTH_VIEWS, DEPTH_W, DEPTH_H)
    views, partners = scene["views"], scene["partners"]
    n, w, h = len(views), DEPTH_W, DEPTH_H
    sptr = ctypes.c_void_p(stream.cuda_stream)
    cams = [c_camera(v["camera"]) for v in views]
    images = []
    for v in views:
        g = torch.from_numpy(v["gray"]).to(dev)
        img = torch.empty((h, w, 3), dtype=torch.float32, device=dev)
        _native_check(lib, lib.r3dgpu_make_refinement_image(g.data_ptr(), w, w, h, 0.0, img.data_ptr(), 3 * w, sptr))
        images.append(img)
    rimg = []
    for i in range(n):
        r = CRefinementImage()
        r.camera, r.data, r.stride = cams[i], images[i].data_ptr(), 3 * w
        rimg.append(r)
    partner_arr = []
    for i in range(n):
        arr = (CRefinementImage * len(partners[i]))()
        for k, j in enumerate(partners[i]):
            arr[k] = rimg[j]
        partner_arr.append(arr)
    pristine = [torch.from_numpy(v["depth"]).to(dev) for v in views]
    depth = [torch.empty_like(d) for d in pristine]
    conf = [torch.zeros_like(d) for d in pristine]
    mask = [torch.full((h, w), 1, dtype=torch.int16, device=dev) for _ in views]
    support = [torch.zeros((h, w), dtype=torch.uint8, device=dev) for _ in views]
    color = [torch.from_numpy(v["color"]).to(dev) for v in views]
    maps = (CDepthMap * n)()
    for i, v in enumerate(views):
        mp = maps[i]
        mp.camera = cams[i]
        mp.depth, mp.confidence = depth[i].data_ptr(), conf[i].data_ptr()
        mp.pair_mask, mp.support, mp.color = mask[i].data_ptr(), support[i].data_ptr(), color[i].data_ptr()
        mp.stride, mp.color_stride, mp.width, mp.height = w, 3 * w, w, h
        mp.view, mp.num_partners = i, len(partners[i])
        for k, j in enumerate(partners[i]):
            mp.partners[k] = j
    off, idx = neighbour_lists(partners)
    copts = ConsistencyOptions().c()
    rstats, cstats = CRefinementStats(), CConsistencyStats()

    def step(opts):
        for i in range(n):
            depth[i].copy_(pristine[i])
        for i in range(n):
            _native_check(lib, lib.r3dgpu_refine_depth_map(depth[i].data_ptr(), conf[i].data_ptr(), w,
                                                           ctypes.byref(cams[i]), w, h, ctypes.byref(rimg[i]),
                                                           partner_arr[i], len(partners[i]), ctypes.byref(opts),
                                                           ctypes.byref(rstats), sptr))
        _native_check(lib, lib.r3dgpu_filter_depth_maps(maps, n, off.ctypes.data, idx.ctypes.data,
                                                        ctypes.byref(copts), ctypes.byref(cstats), sptr))

    def timed(opts):
        for _ in range(warmup):
            step(opts)
        torch.cuda.synchronize(dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = int(lib.r3dgpu_launch_count())
        a.record(stream)
        for _ in range(steps):
            step(opts)
        b.record(stream)
        torch.cuda.synchronize(dev)
        return a.elapsed_time(b) / steps, (int(lib.r3dgpu_launch_count()) - l0) // steps

    f32 = RefinementOptions(radius=3, step=1, fp32=True).c()
    f64 = RefinementOptions(radius=3, step=1).c()
    ms32, launches = timed(f32)
    refine_stats, filter_stats = rstats.as_dict(), cstats.as_dict()
    ms64, _ = timed(f64)
    # Refinement alone (float path), for the kernel's share.
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for i in range(n):
        depth[i].copy_(pristine[i])
    torch.cuda.synchronize(dev)
    a.record(stream)
    for i in range(n):
        _native_check(lib, lib.r3dgpu_refine_depth_map(depth[i].data_ptr(), conf[i].data_ptr(), w,
                                                       ctypes.byref(cams[i]), w, h, ctypes.byref(rimg[i]),
                                                       partner_arr[i], len(partners[i]), ctypes.byref(f32),
                                                       ctypes.byref(rstats), sptr))
    b.record(stream)
    torch.cuda.synchronize(dev)
    refine_ms = a.elapsed_time(b) / n

    # End to end through the host entry points (host maps and images, copies inside).
    himg = [im.cpu().numpy() for im in images]
    hrimg = []
    for i in range(n):
        r = CRefinementImage()
        r.camera, r.data, r.stride = cams[i], himg[i].ctypes.data, 3 * w
        hrimg.append(r)
    hdepth = [np.empty((h, w), np.float32) for _ in views]
    hconf = [np.zeros((h, w), np.float32) for _ in views]
    hmask = [np.ones((h, w), np.uint16) for _ in views]
    hsup = [np.zeros((h, w), np.uint8) for _ in views]
    hmaps = (CDepthMap * n)()
    for i, v in enumerate(views):
        hmaps[i] = maps[i]
        hmaps[i].depth, hmaps[i].confidence = hdepth[i].ctypes.data, hconf[i].ctypes.data
        hmaps[i].pair_mask, hmaps[i].support, hmaps[i].color = hmask[i].ctypes.data, hsup[i].ctypes.data, \
            v["color"].ctypes.data

    def host_step():
        for i in range(n):
            hdepth[i][...] = views[i]["depth"]
            hconf[i][...] = 0.0
        _native_check(lib, lib.r3dgpu_depth_stage_host(hmaps, hrimg_arr, n, off.ctypes.data, idx.ctypes.data,
                                                       ctypes.byref(f32), ctypes.byref(copts), ctypes.byref(rstats),
                                                       ctypes.byref(cstats)))

    hrimg_arr = (CRefinementImage * n)(*hrimg)
    host_step()
    t0 = time.perf_counter()
    for _ in range(max(1, steps // 2)):
        host_step()
    e2e_s = (time.perf_counter() - t0) / max(1, steps // 2)
    # One call per step: every refinement image and map in once (12 + 13 B per
    # pixel), depth, confidence and support out (9 B per pixel).
    h2d = n * 25 * w * h
    d2h = n * 9 * w * h

    # The float path's error and the oracle's time on a crop of view 0.
    cw, ch = DEPTH_CROP
    x0, y0 = (w - cw) // 2, (h - ch) // 2
    cam0 = dict(views[0]["camera"], width=cw, height=ch, cx=views[0]["camera"]["cx"] - x0,
                cy=views[0]["camera"]["cy"] - y0)
    crop_img = np.ascontiguousarray(himg[0][y0:y0 + ch, x0:x0 + cw])
    base = {"camera": cam0, "data": crop_img}
    pviews = [{"camera": views[j]["camera"], "data": himg[j]} for j in partners[0]]
    crop = {"camera": cam0, "depth": np.ascontiguousarray(views[0]["depth"][y0:y0 + ch, x0:x0 + cw]),
            "confidence": np.zeros((ch, cw), np.float32)}
    from regard3d_mvs_b200.stereo import Matcher

    mm = Matcher(device=dev.index or 0)
    g32 = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in crop.items()}
    mm.refine_depth_map(g32, base, pviews, RefinementOptions(radius=3, step=1, fp32=True))
    o64 = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in crop.items()}
    t0 = time.perf_counter()
    ost = orc.refine_depth_map(o64, base, pviews, RefinementOptions(radius=3, step=1))
    cpu_s = time.perf_counter() - t0
    both = (g32["depth"] > 0) & (o64["depth"] > 0)
    rel = np.abs(g32["depth"][both].astype(np.float64) - o64["depth"][both]) / o64["depth"][both]
    flips = int(((g32["depth"] > 0) != (o64["depth"] > 0)).sum())
    achieved = DEPTH_BYTES_PER_PIXEL * w * h / (ms32 / n * 1e-3) / 1e9
    return {"workload": f"depth stage: {n} views {w}x{h}, refinement 7x7 (radius 3, step 1) against 4 views, "
                        "consistency over 4 neighbours",
            "value": n / (ms32 * 1e-3), "unit": "depth maps/s", "ms_per_step": ms32, "dtype": "f32 window terms",
            "f64_path": {"value": n / (ms64 * 1e-3), "ms_per_step": ms64},
            "refine_ms_per_view_f32": refine_ms, "gpu_launches": launches,
            "refinement": refine_stats, "consistency": filter_stats,
            "fp32_vs_f64_oracle": {"sample": f"{cw}x{ch} crop of view 0", "pixels_compared": int(both.sum()),
                                   "decision_flips": flips, "rel_depth_error_p50": float(np.percentile(rel, 50)),
                                   "p99": float(np.percentile(rel, 99)), "max": float(rel.max())},
            "e2e": {"value": n / e2e_s, "unit": "depth maps/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "alg_bytes_per_pixel": DEPTH_BYTES_PER_PIXEL},
            "cpu_baseline": {"value": (cw * ch) / cpu_s / (w * h), "unit": "depth maps/s (refinement only)",
                             "cores": orc.max_threads(), "kind": "port",
                             "sample": f"double-precision refinement of a {cw}x{ch} crop of view 0, scaled to "
                                       f"{w}x{h}", "refined": ost["refined"]}}


# A view's depth map on the device (r3dgpu_compute_depth_map): a 2048 x 1536
# base image and 4 partners of a textured plane, each pair rectified (both
# images), the 4 pairs matched in one batch (reference default options:
# automatic hierarchy, +-4 ranges), combined into the grid's depth map.
VIEW_W, VIEW_H, VIEW_F = 2048, 1536, 1800.0
VIEW_PARTNERS = ((0.6, 0.0, 0.0), (-0.5, 0.3, 0.1), (0.2, -0.55, 0.0), (-0.3, -0.4, 0.2))


def measure_view(lib, dev, stream, steps: int, warmup: int) -> dict:
    """Device time of compute_depth_map for one view (inputs resident), end
    to end through Matcher.compute_depth_map (host images in, maps out), and
    the oracle's chain (rectify, match, combine) on the same view."""
    import torch

    from oracle import oracle as orc
    from regard3d_mvs_b200.multi_view import CViewPair, c_grid, pair_geometry, pipeline_scene
    from regard3d_mvs_b200.stereo import Matcher
    from regard3d_mvs_b200.types import (CViewU16, MultiStereoOptions, StereoOptions, camera_struct, pinhole_struct,
                                         to_c_options)

    rig, base, pairs = pipeline_scene(VIEW_W, VIEW_H, VIEW_F, VIEW_PARTNERS, seed=4)
    w, h = VIEW_W, VIEW_H
    cam = {"model": 0, "width": w, "height": h, "fx": rig.K[0, 0], "fy": rig.K[1, 1], "cx": rig.K[0, 2],
           "cy": rig.K[1, 2]}
    keep = []

    def dev_u16(a):
        t = torch.from_numpy(a.view(np.int16)).to(dev)
        keep.append(t)
        return t.data_ptr()

    cb = camera_struct(cam)
    vb = CViewU16(dev_u16(base), w, h, w)
    arr = (CViewPair * len(pairs))()
    for i, p in enumerate(pairs):
        q = arr[i]
        q.partner = CViewU16(dev_u16(p["image"]), w, h, w)
        q.partner_camera = camera_struct(cam)
        q.base_from_rect[:] = [float(v) for v in (rig.R @ p["R_rect"].T).ravel()]
        q.partner_from_rect[:] = [float(v) for v in (p["R_partner"] @ p["R_rect"].T).ravel()]
        q.left, q.right = pinhole_struct(p["left"]), pinhole_struct(p["right"])
        q.disparity_min, q.num_disparities = p["disparity_min"], p["num_disparities"]
        q.geometry = pair_geometry(rig.grid(), p)
    g = c_grid(rig.grid())
    depth = torch.empty((h, w), dtype=torch.float32, device=dev)
    conf = torch.empty_like(depth)
    mask = torch.empty((h, w), dtype=torch.int16, device=dev)
    so, mo = to_c_options(StereoOptions()), MultiStereoOptions().c()
    cells = ctypes.c_uint64(0)
    sptr = ctypes.c_void_p(stream.cuda_stream)

    def run():
        _native_check(lib, lib.r3dgpu_compute_depth_map(ctypes.byref(vb), ctypes.byref(cb), ctypes.byref(g), arr,
                                                        len(pairs), ctypes.byref(so), ctypes.byref(mo),
                                                        depth.data_ptr(), conf.data_ptr(), mask.data_ptr(), w,
                                                        ctypes.byref(cells), sptr))

    for _ in range(warmup):
        run()
    torch.cuda.synchronize(dev)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = int(lib.r3dgpu_launch_count())
    a.record(stream)
    for _ in range(steps):
        run()
    b.record(stream)
    torch.cuda.synchronize(dev)
    ms = a.elapsed_time(b) / steps
    launches = (int(lib.r3dgpu_launch_count()) - l0) // steps
    full_cells = sum(w * h * p["num_disparities"] for p in pairs)
    m = Matcher(device=dev.index or 0)
    m.compute_depth_map(base, rig.grid(), pairs)
    t0 = time.perf_counter()
    for _ in range(max(1, steps // 2)):
        got, _ = m.compute_depth_map(base, rig.grid(), pairs)
    e2e_s = (time.perf_counter() - t0) / max(1, steps // 2)
    # The oracle's chain on the same view (once).
    t0 = time.perf_counter()
    matched = []
    for p in pairs:
        left, lmask = orc.rectify_image(base, cam, rig.R @ p["R_rect"].T, p["left"])
        right, rmask = orc.rectify_image(p["image"], cam, p["R_partner"] @ p["R_rect"].T, p["right"])
        mt = orc.match_stereo(left, right, lmask, rmask, p["disparity_min"], p["num_disparities"], StereoOptions())
        matched.append(dict(p, disparity=mt.disparity, confidence=mt.confidence))
    ref = orc.combine_pairs(rig.grid(), matched, MultiStereoOptions())
    cpu_s = time.perf_counter() - t0
    same = bool(np.array_equal(ref.depth, got.depth) and np.array_equal(ref.pair_mask, got.pair_mask))
    return {"workload": f"a view's depth map: {w}x{h} base and 4 partners (plane scene), rectify + match (reference "
                        "default options, one batch) + combine on the device",
            "value": 1000.0 / ms, "unit": "depth maps/s", "ms_per_view": ms, "gpu_launches": launches,
            "full_range_cells": full_cells, "aggregated_cells": int(cells.value),
            "label_ranges": [p["num_disparities"] for p in pairs], "bit_exact_vs_oracle": same,
            "valid_fraction": float((got.depth > 0).mean()),
            "e2e": {"value": 1.0 / e2e_s, "unit": "depth maps/s", "h2d_bytes_per_step": 2 * w * h * (1 + len(pairs)),
                    "d2h_bytes_per_step": 10 * w * h},
            "cpu_baseline": {"value": 1.0 / cpu_s, "unit": "depth maps/s", "cores": orc.max_threads(), "kind": "port",
                             "sample": "the same view once: rectify, match_stereo and combine_pairs of the oracle"}}


# The full depth stage of a 32-view scene (2048 x 1536 views on an
# arc of radius 2 m around 20 textured planes, 4 nearest partners per view).
SCENE_VIEWS, SCENE_W, SCENE_H, SCENE_SEED = 32, 2048, 1536, 11
SCENE_CHECK_VIEW = 16  # compared with the oracle's chain (a central view)
SCENE_THREADS = 4  # host threads (one CUDA stream each) running views concurrently


def _scene_env(plain: bool):
    """Kernel selection of the plain GPU path: one CTA per SGM tile (the
    skewed-wavefront kernels), single-track batches."""
    keys = {"R3DGPU_FULL_KERNEL": "wavefront", "R3DGPU_RANGED_KERNEL": "ranged", "R3DGPU_BATCH_TRACKS": "1"}
    if plain:
        os.environ.update(keys)
    else:
        for k in keys:
            os.environ.pop(k, None)


def measure_scene(lib, dev, stream, steps: int, warmup: int) -> dict:
    """The 32-view depth stage end to end on the device: per view compute_depth_map
    (rectification of both images of its 4 pairs, one batch match,
    combination), then the float refinement of every view against its
    partners' refinement images and the consistency filter of the 32 maps;
    the same through the host entry points (e2e), with the plain one-CTA-per-
    tile kernels, one view's depth map against the oracle's chain, the float
    refinement against the double oracle on a crop, and the oracle's time."""
    import torch

    from oracle import oracle as orc
    from regard3d_mvs_b200.depth_maps import (CConsistencyStats, CDepthMap, ConsistencyOptions, CRefinementImage,
                                              CRefinementStats, RefinementOptions, c_camera, neighbour_lists)
    from regard3d_mvs_b200.multi_view import CViewPair, arc_scene, c_grid, pair_geometry
    from regard3d_mvs_b200.stereo import Matcher
    from regard3d_mvs_b200.types import (CViewU16, MultiStereoOptions, StereoOptions, camera_struct, pinhole_struct,
                                         to_c_options)

    scene = arc_scene(SCENE_VIEWS, SCENE_W, SCENE_H, seed=SCENE_SEED, device=dev)
    views = scene["views"]
    n, w, h = len(views), SCENE_W, SCENE_H
    K = scene["K"]
    sptr = ctypes.c_void_p(stream.cuda_stream)
    cam = {"model": 0, "width": w, "height": h, "fx": K[0, 0], "fy": K[1, 1], "cx": K[0, 2], "cy": K[1, 2]}
    cb = camera_struct(cam)
    d_img = [torch.from_numpy(v["image"].view(np.int16)).to(dev) for v in views]
    d_gray = [torch.from_numpy(v["image8"].astype(np.float32)).to(dev) for v in views]
    d_color = [torch.from_numpy(np.repeat(v["image8"][..., None], 3, axis=2)).to(dev) for v in views]
    pcams = [{"width": w, "height": h, "fx": K[0, 0], "fy": K[1, 1], "cx": K[0, 2], "cy": K[1, 2],
              "rotation": v["camera"]["R"], "center": v["camera"]["C"]} for v in views]
    ccams = [c_camera(c) for c in pcams]
    grids = [c_grid(v["camera"]) for v in views]
    vbs = [CViewU16(d_img[i].data_ptr(), w, h, w) for i in range(n)]
    pair_arrs = []
    for i, v in enumerate(views):
        arr = (CViewPair * len(v["pairs"]))()
        for k, p in enumerate(v["pairs"]):
            q = arr[k]
            q.partner = CViewU16(d_img[p["partner"]].data_ptr(), w, h, w)
            q.partner_camera = camera_struct(cam)
            q.base_from_rect[:] = [float(x) for x in (v["camera"]["R"] @ p["R_rect"].T).ravel()]
            q.partner_from_rect[:] = [float(x) for x in (p["R_partner"] @ p["R_rect"].T).ravel()]
            q.left, q.right = pinhole_struct(p["left"]), pinhole_struct(p["right"])
            q.disparity_min, q.num_disparities = p["disparity_min"], p["num_disparities"]
            q.geometry = pair_geometry(v["camera"], p)
        pair_arrs.append(arr)
    depth = [torch.empty((h, w), dtype=torch.float32, device=dev) for _ in views]
    conf = [torch.empty_like(d) for d in depth]
    mask = [torch.empty((h, w), dtype=torch.int16, device=dev) for _ in views]
    support = [torch.zeros((h, w), dtype=torch.uint8, device=dev) for _ in views]
    rimg_t = [torch.empty((h, w, 3), dtype=torch.float32, device=dev) for _ in views]
    so, mo = to_c_options(StereoOptions()), MultiStereoOptions().c()
    rimg = []
    for i in range(n):
        r = CRefinementImage()
        r.camera, r.data, r.stride = ccams[i], rimg_t[i].data_ptr(), 3 * w
        rimg.append(r)
    partners = [v["partners"] for v in views]
    partner_rimg = []
    for i in range(n):
        arr = (CRefinementImage * len(partners[i]))()
        for k, j in enumerate(partners[i]):
            arr[k] = rimg[j]
        partner_rimg.append(arr)
    maps = (CDepthMap * n)()
    for i in range(n):
        mp = maps[i]
        mp.camera = ccams[i]
        mp.depth, mp.confidence = depth[i].data_ptr(), conf[i].data_ptr()
        mp.pair_mask, mp.support, mp.color = mask[i].data_ptr(), support[i].data_ptr(), d_color[i].data_ptr()
        mp.stride, mp.color_stride, mp.width, mp.height = w, 3 * w, w, h
        mp.view, mp.num_partners = i, len(partners[i])
        for k, j in enumerate(partners[i]):
            mp.partners[k] = j
    off, idx = neighbour_lists(partners)
    ropts = RefinementOptions(radius=3, step=1, fp32=True).c()
    copts = ConsistencyOptions().c()
    cstats = CConsistencyStats()
    total_cells = [0] * (1 + SCENE_THREADS)

    # Views run on SCENE_THREADS host threads, each with its own CUDA stream
    # (the library keeps its workspaces per thread): refinement images and
    # depth maps, then (after every view's depth map exists) the refinement,
    # then the consistency filter of all maps on the main stream.
    from concurrent.futures import ThreadPoolExecutor

    streams = [torch.cuda.Stream(dev) for _ in range(SCENE_THREADS)]
    pool = ThreadPoolExecutor(SCENE_THREADS)
    stat_sum: dict = {}

    def per_thread(fn):
        ready = torch.cuda.Event()
        ready.record(stream)
        for st in streams:
            st.wait_event(ready)
        list(pool.map(fn, range(SCENE_THREADS)))
        for st in streams:
            done = torch.cuda.Event()
            done.record(st)
            stream.wait_event(done)

    def maps_part(t):
        sp = ctypes.c_void_p(streams[t].cuda_stream)
        c = ctypes.c_uint64(0)
        cells_t = 0
        for i in range(t, n, SCENE_THREADS):
            _native_check(lib, lib.r3dgpu_make_refinement_image(d_gray[i].data_ptr(), w, w, h, 0.0,
                                                                rimg_t[i].data_ptr(), 3 * w, sp))
            _native_check(lib, lib.r3dgpu_compute_depth_map(ctypes.byref(vbs[i]), ctypes.byref(cb),
                                                            ctypes.byref(grids[i]), pair_arrs[i], len(views[i]["pairs"]),
                                                            ctypes.byref(so), ctypes.byref(mo), depth[i].data_ptr(),
                                                            conf[i].data_ptr(), mask[i].data_ptr(), w, ctypes.byref(c),
                                                            sp))
            cells_t += int(c.value)
        total_cells[t + 1] = cells_t

    def refine_part(t):
        sp = ctypes.c_void_p(streams[t].cuda_stream)
        for i in range(t, n, SCENE_THREADS):
            st = CRefinementStats()
            _native_check(lib, lib.r3dgpu_refine_depth_map(depth[i].data_ptr(), conf[i].data_ptr(), w,
                                                           ctypes.byref(ccams[i]), w, h, ctypes.byref(rimg[i]),
                                                           partner_rimg[i], len(partners[i]), ctypes.byref(ropts),
                                                           ctypes.byref(st), sp))
            stat_sum[i] = st.as_dict()

    def step():
        per_thread(maps_part)
        total_cells[0] = sum(total_cells[1:])
        per_thread(refine_part)
        _native_check(lib, lib.r3dgpu_filter_depth_maps(maps, n, off.ctypes.data, idx.ctypes.data,
                                                        ctypes.byref(copts), ctypes.byref(cstats), sptr))

    def timed(k):
        torch.cuda.synchronize(dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = int(lib.r3dgpu_launch_count())
        a.record(stream)
        for _ in range(k):
            step()
        b.record(stream)
        torch.cuda.synchronize(dev)
        return a.elapsed_time(b) / k, (int(lib.r3dgpu_launch_count()) - l0) // k

    for _ in range(warmup):
        step()
    ms, launches = timed(steps)
    refine_stats = {k: sum(d[k] for d in stat_sum.values()) for k in next(iter(stat_sum.values()))}
    filter_stats = cstats.as_dict()
    kept = float(sum(int((d > 0).sum().item()) for d in depth)) / (n * w * h)
    full_cells = sum(w * h * p["num_disparities"] for v in views for p in v["pairs"])
    # The plain GPU path: the same chain with one CTA per SGM tile.
    _scene_env(True)
    try:
        step()
        plain_ms, _ = timed(1)
    finally:
        _scene_env(False)

    # End to end through the public host API: Matcher.compute_depth_map per
    # view (host images in, maps out), then Matcher.depth_stage (host maps
    # and refinement images in, refined and filtered maps out).
    m = Matcher(device=dev.index or 0)
    hrimg = [t.cpu().numpy() for t in rimg_t]

    def e2e_step():
        hmaps = []
        for i, v in enumerate(views):
            dm, _ = m.compute_depth_map(v["image"], v["camera"], v["pairs"])
            hmaps.append({"camera": pcams[i], "depth": dm.depth, "confidence": dm.confidence,
                          "pair_mask": dm.pair_mask, "color": np.repeat(v["image8"][..., None], 3, axis=2),
                          "view": i, "partners": partners[i]})
        m.depth_stage(hmaps, [{"camera": pcams[i], "data": hrimg[i]} for i in range(n)], partners,
                      RefinementOptions(radius=3, step=1, fp32=True), ConsistencyOptions())
        return hmaps

    e2e_step()
    t0 = time.perf_counter()
    e2e_step()
    e2e_s = time.perf_counter() - t0
    h2d = n * (2 * w * h * 5 + 12 * w * h + 3 * w * h + 10 * w * h)
    d2h = n * (10 * w * h + 9 * w * h)

    # One view against the oracle's chain (rectify both images of every pair,
    # match_stereo, combine_pairs), timed as the CPU baseline of that part.
    c = SCENE_CHECK_VIEW
    v = views[c]
    got, _ = m.compute_depth_map(v["image"], v["camera"], v["pairs"])
    t0 = time.perf_counter()
    matched = []
    for p in v["pairs"]:
        left, lmask = orc.rectify_image(v["image"], cam, v["camera"]["R"] @ p["R_rect"].T, p["left"])
        right, rmask = orc.rectify_image(p["image"], cam, p["R_partner"] @ p["R_rect"].T, p["right"])
        mt = orc.match_stereo(left, right, lmask, rmask, p["disparity_min"], p["num_disparities"], StereoOptions())
        matched.append(dict(p, disparity=mt.disparity, confidence=mt.confidence))
    ref = orc.combine_pairs(v["camera"], matched, MultiStereoOptions())
    chain_s = time.perf_counter() - t0
    same = bool(np.array_equal(ref.depth, got.depth) and np.array_equal(ref.pair_mask, got.pair_mask))
    # Float refinement against the double oracle on a crop of that view (its
    # combined depth map as the initial depths).
    cw, ch = DEPTH_CROP
    x0, y0 = (w - cw) // 2, (h - ch) // 2
    cam_c = dict(pcams[c], width=cw, height=ch, cx=pcams[c]["cx"] - x0, cy=pcams[c]["cy"] - y0)
    base = {"camera": cam_c, "data": np.ascontiguousarray(hrimg[c][y0:y0 + ch, x0:x0 + cw])}
    pviews = [{"camera": pcams[j], "data": hrimg[j]} for j in partners[c]]
    crop = {"camera": cam_c, "depth": np.ascontiguousarray(got.depth[y0:y0 + ch, x0:x0 + cw]),
            "confidence": np.ascontiguousarray(got.confidence[y0:y0 + ch, x0:x0 + cw])}
    g32 = {k: (x.copy() if isinstance(x, np.ndarray) else x) for k, x in crop.items()}
    m.refine_depth_map(g32, base, pviews, RefinementOptions(radius=3, step=1, fp32=True))
    o64 = {k: (x.copy() if isinstance(x, np.ndarray) else x) for k, x in crop.items()}
    t0 = time.perf_counter()
    orc.refine_depth_map(o64, base, pviews, RefinementOptions(radius=3, step=1))
    refine_s = (time.perf_counter() - t0) * (w * h) / (cw * ch)
    both = (g32["depth"] > 0) & (o64["depth"] > 0)
    rel = np.abs(g32["depth"][both].astype(np.float64) - o64["depth"][both]) / o64["depth"][both]
    flips = int(((g32["depth"] > 0) != (o64["depth"] > 0)).sum())
    return {"workload": f"depth stage: {n} views {w}x{h} on an arc of radius 2 m around 20 textured planes, 4 partners "
                        "per view: rectify + match (reference defaults, one batch per view) + combine, FP32 7x7 "
                        "refinement against the 4 partners, consistency over 4 neighbours; views on "
                        f"{SCENE_THREADS} host threads with a CUDA stream each",
            "value": n / (ms * 1e-3), "unit": "depth maps/s", "ms_per_scene": ms, "gpu_launches": launches,
            "full_range_cells": full_cells, "aggregated_cells": total_cells[0],
            "label_ranges": sorted({p["num_disparities"] for vv in views for p in vv["pairs"]}),
            "depth_fraction_kept": kept, "refinement": refine_stats, "consistency": filter_stats,
            "plain_gpu_path": {"value": n / (plain_ms * 1e-3), "unit": "depth maps/s", "ms_per_scene": plain_ms,
                               "kernels": "one CTA per SGM tile (skewed-wavefront kernels), single-track batches"},
            "bit_exact_vs_oracle": {"view": c, "depth_and_pair_mask_equal": same},
            "fp32_vs_f64_oracle": {"sample": f"{cw}x{ch} crop of view {c}", "pixels_compared": int(both.sum()),
                                   "decision_flips": flips,
                                   "rel_depth_error_p50": float(np.percentile(rel, 50)) if rel.size else 0.0,
                                   "p99": float(np.percentile(rel, 99)) if rel.size else 0.0,
                                   "max": float(rel.max()) if rel.size else 0.0, "target": 1e-5},
            "e2e": {"value": n / e2e_s, "unit": "depth maps/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "cpu_baseline": {"value": 1.0 / (chain_s + refine_s), "unit": "depth maps/s", "cores": orc.max_threads(),
                             "kind": "port",
                             "sample": f"view {c} once: the oracle's rectify, match_stereo and combine_pairs "
                                       f"({chain_s:.1f} s), plus its double refinement of a {cw}x{ch} crop scaled "
                                       f"to the view ({refine_s:.1f} s); consistency not included"}}


SERVE_FRACTIONS = (0.1, 0.5, 0.8, 1.0, 1.2)
SERVE_REQUEST_BUDGET = 110 << 30  # of a 150 GB serving budget: 110 GB for admitted requests, 2 x 16 GB worker scratch, 8 GB cache
SERVE_CACHE = 8 << 30
SERVE_WORKERS = 2
SERVE_MAX_BATCH = 16
SERVE_SCENE_VIEWS = 200
SERVE_POOL_VIEWS = 8
SERVE_PARTNERS = 4


def serving_views(lib, n: int, seed: int) -> list[dict]:
    """Distinct views of the serving simulation: sizes, label ranges and
    hierarchy as the 64-pair batch draws them per pair; each view's 4 partner pairs
    share its left image (the generator's left image depends on the seed,
    size and label count only) and differ in the disparity field (plane
    count), so their right images differ."""
    rng = np.random.default_rng(seed)
    views = []
    for v in range(n):
        w = int(round(math.exp(rng.uniform(math.log(1024), math.log(6048)))))
        h = int(round(w / (1.5 if rng.random() < 0.5 else 4.0 / 3.0)))
        nd = int(ND_CHOICES[rng.integers(0, len(ND_CHOICES))])
        hier = v % 2 == 1
        spec = dict(w=w, h=h, nd=nd, levels=3 if hier else 0, radius=0 if hier else 3, margin=8 if hier else 4,
                    textureless=0.0, occluded=0.0, seed=seed * 1000 + v)
        rights, left = [], None
        for k in range(SERVE_PARTNERS):
            L, R = make_images(lib, dict(spec, planes=5 + k))
            left = L if left is None else left
            assert np.array_equal(left, L)
            rights.append(R)
        views.append(dict(spec, left=left, rights=rights))
    return views


def run_serving(args, rate_hint: float) -> dict:
    """Serving: a simulated 200-view scene, each view issuing its 4 partner
    pair requests (Poisson arrivals of requests), through the serving loop
    (continuous batching, admission by a device-memory budget, a view's left
    image uploaded once and kept on the device across its partners by its
    content key). The served saturation is measured first (offered load 3 x
    the batch rate `rate_hint`), then latency percentiles and served
    Gcells/s at fractions of that saturated rate."""
    import torch

    from regard3d_mvs_b200 import Server
    from regard3d_mvs_b200._native import load

    lib = load()
    pool_views = serving_views(lib, SERVE_POOL_VIEWS, args.seed + 17)

    def pinned(a):
        t = torch.from_numpy(a.view(np.int16) if a.dtype == np.uint16 else a).pin_memory()
        return t.numpy().view(a.dtype)

    for v in pool_views:
        v["left"] = pinned(v["left"])
        v["rights"] = [pinned(r) for r in v["rights"]]
        v["outs"] = [[pinned(np.empty((v["h"], v["w"]), np.float32)) for _ in range(2)]
                     for _ in range(SERVE_PARTNERS)]
    # The scene's request sequence: view s uses the images of pool view
    # s % POOL under its own content key (a new view: its left image is not
    # on the device yet), partners in order.
    seq = [(s, s % SERVE_POOL_VIEWS, k) for s in range(SERVE_SCENE_VIEWS) for k in range(SERVE_PARTNERS)]
    cells = {vi: v["w"] * v["h"] * ((v["nd"] + 15) // 16 * 16) for vi, v in enumerate(pool_views)}
    free0, total = torch.cuda.mem_get_info(0)
    peak_used = [total - free0]
    rng = np.random.default_rng(args.seed + 1)
    cursor = [0]
    key_base = [1]

    def submit(srv, s, vi, k):
        v = pool_views[vi]
        out = v["outs"][k].pop() if v["outs"][k] else pinned(np.empty((v["h"], v["w"]), np.float32))
        t = srv.submit(v["left"], v["rights"][k], None, None, 0, v["nd"], options_for(v), out=(out, None),
                       left_key=key_base[0] + s)
        return (vi, k, out, t)

    def run_point(srv, lam: float, seconds: float) -> dict:
        nreq = int(min(max(16, round(lam * seconds)), len(seq)))
        gaps = rng.exponential(1.0 / lam, nreq)
        tickets = []
        t0 = time.perf_counter()
        arrival = t0
        for q in range(nreq):
            arrival += gaps[q]
            delay = arrival - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            s, vi, k = seq[(cursor[0] + q) % len(seq)]
            tickets.append(submit(srv, s, vi, k))
            free, _ = torch.cuda.mem_get_info(0)
            peak_used[0] = max(peak_used[0], total - free)
        cursor[0] += nreq
        key_base[0] += SERVE_SCENE_VIEWS  # keys of a point never match the previous point's
        lat, batch, hits, up = [], [], 0, 0
        for vi, k, out, t in tickets:
            m, tm = srv.wait(t)
            pool_views[vi]["outs"][k].append(out)
            lat.append(tm["total_ms"])
            batch.append(tm["batch_size"])
            hits += tm["cache_hits"]
            up += tm["uploaded_bytes"]
        t1 = time.perf_counter()
        lat = np.array(lat)
        done_cells = sum(cells[vi] for vi, _, _, _ in tickets)
        return {"offered_pairs_per_s": lam, "requests": nreq, "served_pairs_per_s": nreq / (t1 - t0),
                "gcells_per_s": done_cells / (t1 - t0) / 1e9,
                "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                               "p999": float(np.percentile(lat, 99.9)), "max": float(lat.max())},
                "p99_over_p50": float(np.percentile(lat, 99) / np.percentile(lat, 50)),
                "mean_batch": float(np.mean(batch)), "left_image_cache_hits": hits / nreq,
                "uploaded_mb_per_request": up / nreq / 1e6}

    scratch = min(16 << 30, (32 << 30) // args.serve_workers)  # 32 GB of SGM scratch over the workers
    with Server(device=0, workers=args.serve_workers, max_batch=args.serve_batch, hbm_budget=SERVE_REQUEST_BUDGET,
                scratch_budget=scratch, cache_budget=SERVE_CACHE) as srv:
        # Warm-up: the workers allocate their buffers.
        run_point(srv, 4.0 * max(rate_hint, 1.0), 2.0)
        sat = run_point(srv, 3.0 * max(rate_hint, 1.0), args.serve_seconds)
        sat_rate = sat["served_pairs_per_s"]
        points = []
        for frac in SERVE_FRACTIONS:
            pt = run_point(srv, frac * sat_rate, args.serve_seconds)
            pt["load"] = frac
            points.append(pt)
    return {"scene": f"{SERVE_SCENE_VIEWS} views x {SERVE_PARTNERS} partner pairs (images of {SERVE_POOL_VIEWS} "
                     "distinct views drawn like the 64-pair batch; each view's pairs share its left image under the view's content key)",
            "saturated_pairs_per_s": sat_rate, "saturation_run": sat,
            "load_axis": "fraction of the served saturation measured above", "workers": args.serve_workers,
            "max_batch": args.serve_batch, "host_buffers": "page-locked inputs and disparity maps; no confidence maps",
            "request_budget_bytes": SERVE_REQUEST_BUDGET, "worker_scratch_bytes": scratch,
            "image_cache_bytes": SERVE_CACHE, "device_used_peak_gb": peak_used[0] / 1e9, "arrivals": "Poisson",
            "points": points}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.serve_only > 0:
        print(json.dumps(run_serving(args, args.serve_only)), flush=True)
        return

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = dist_mod

    from regard3d_mvs_b200 import Matcher
    from regard3d_mvs_b200.types import CDisparityMap, CPair, CProfile, CViewU8, CViewU16, to_c_options

    m = Matcher(device=local)
    lib = m.lib
    if args.workload == "combine":
        peak, _ = measured_peaks()
        dev0 = torch.device(f"cuda:{local}")
        r = measure_combine(lib, dev0, torch.cuda.current_stream(dev0), args.steps, args.warmup, peak)
        if rank == 0:
            print(json.dumps(dict(r, metric="combine_pairs Gpixels/s", n_gpus=world, steps=args.steps,
                                  warmup=args.warmup, higher_is_better=True, data="synthetic")), flush=True)
        return
    if args.workload == "view":
        dev0 = torch.device(f"cuda:{local}")
        r = measure_view(lib, dev0, torch.cuda.current_stream(dev0), args.steps, args.warmup)
        if rank == 0:
            print(json.dumps(dict(r, metric="depth maps/s", n_gpus=world, steps=args.steps, warmup=args.warmup,
                                  higher_is_better=True, data="synthetic")), flush=True)
        return
    if args.workload == "scene32":
        dev0 = torch.device(f"cuda:{local}")
        r = measure_scene(lib, dev0, torch.cuda.current_stream(dev0), args.steps, args.warmup)
        if rank == 0:
            print(json.dumps(dict(r, metric="depth maps/s", n_gpus=world, steps=args.steps, warmup=args.warmup,
                                  higher_is_better=True, data="synthetic")), flush=True)
        return
    if args.workload == "depth":
        peak, _ = measured_peaks()
        dev0 = torch.device(f"cuda:{local}")
        r = measure_depth(lib, dev0, torch.cuda.current_stream(dev0), args.steps, args.warmup, peak)
        if rank == 0:
            print(json.dumps(dict(r, metric="depth maps/s", n_gpus=world, steps=args.steps, warmup=args.warmup,
                                  higher_is_better=True, data="synthetic")), flush=True)
        return
    if args.workload == "rectify":
        peak, _ = measured_peaks()
        dev0 = torch.device(f"cuda:{local}")
        r = measure_rectify(lib, dev0, torch.cuda.current_stream(dev0), args.steps, args.warmup, peak)
        if rank == 0:
            print(json.dumps(dict(r, metric="rectify_image Gpixels/s", n_gpus=world, steps=args.steps,
                                  warmup=args.warmup, higher_is_better=True, data="synthetic")), flush=True)
        return
    # The job: `pairs` pairs per rank (weak scaling), split across the ranks
    # as the library's multi-GPU path splits a job (shard.shard_pairs:
    # longest processing time first on W x H x D); every rank draws the same
    # list and matches its share.
    all_specs = workload_pairs(args.workload, args.pairs * world, args.seed)
    cells_job = full_range_cells(all_specs)
    if world > 1:
        from regard3d_mvs_b200.shard import shard_pairs

        share = shard_pairs([s["w"] * s["h"] * ((s["nd"] + 15) // 16 * 16) for s in all_specs], world)[rank]
        specs = [all_specs[i] for i in share]
    else:
        specs = all_specs
    host = [make_images(lib, s) for s in specs]
    dev = torch.device(f"cuda:{local}")
    stream = torch.cuda.current_stream(dev)
    sptr = ctypes.c_void_p(stream.cuda_stream)

    # Device-resident inputs and outputs.
    dL = [torch.from_numpy(L.view(np.int16)).to(dev) for L, _ in host]
    dR = [torch.from_numpy(R.view(np.int16)).to(dev) for _, R in host]
    dD = [torch.empty((s["h"], s["w"]), dtype=torch.float32, device=dev) for s in specs]
    dC = [torch.empty((s["h"], s["w"]), dtype=torch.float32, device=dev) for s in specs]
    n = len(specs)
    pairs = (CPair * n)()
    for i, s in enumerate(specs):
        p = pairs[i]
        p.left = CViewU16(dL[i].data_ptr(), s["w"], s["h"], s["w"])
        p.right = CViewU16(dR[i].data_ptr(), s["w"], s["h"], s["w"])
        p.left_valid = CViewU8()
        p.right_valid = CViewU8()
        p.disparity_min = 0
        p.num_disparities = s["nd"]
        p.options = to_c_options(options_for(s))
        p.out = CDisparityMap(dD[i].data_ptr(), dC[i].data_ptr(), s["w"], 0, 0, 0, 0, 0)

    def step():
        st = lib.r3dgpu_match_stereo_batch(pairs, n, sptr)
        if st != 0:
            raise RuntimeError(lib.r3dgpu_last_error().decode())

    def barrier():
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(v: float) -> float:
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    cells_full = full_range_cells(specs)
    for _ in range(args.warmup):
        step()
    barrier()
    lib.r3dgpu_profile_enable(1)
    prof = CProfile()
    lib.r3dgpu_profile_take(ctypes.byref(prof))
    launches0 = lib.r3dgpu_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        barrier()
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        barrier()
    launches = lib.r3dgpu_launch_count() - launches0
    lib.r3dgpu_profile_take(ctypes.byref(prof))
    lib.r3dgpu_profile_enable(0)
    nbytes = lib.r3dgpu_profile_launches(None, 0)
    buf = ctypes.create_string_buffer(int(nbytes) + 1)
    lib.r3dgpu_profile_launches(buf, nbytes + 1)
    launch_log = json.loads(buf.value.decode() or "[]")
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    value = cells_job * args.steps / (ms * 1e-3) / 1e9
    total_cells = sum(int(pairs[i].out.cells) for i in range(n))

    # End to end: pinned host buffers, copies inside the timed region.
    hL = [torch.from_numpy(L.view(np.int16)).pin_memory() for L, _ in host]
    hR = [torch.from_numpy(R.view(np.int16)).pin_memory() for _, R in host]
    hD = [torch.empty((s["h"], s["w"]), dtype=torch.float32).pin_memory() for s in specs]
    h2d = sum(t.numel() * 2 for t in hL) + sum(t.numel() * 2 for t in hR)
    d2h = sum(t.numel() * 4 for t in hD)

    def e2e_step():
        for i in range(n):
            dL[i].copy_(hL[i], non_blocking=True)
            dR[i].copy_(hR[i], non_blocking=True)
        step()
        for i in range(n):
            hD[i].copy_(dD[i], non_blocking=True)

    e2e_step()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    e2e_value = cells_job * args.steps / (e2e_ms * 1e-3) / 1e9

    # Plain GPU matcher: one call per pair (same kernels, no batching).
    per_pair = None
    if not args.no_per_pair:
        lat = []
        barrier()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for i in range(n):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            st = lib.r3dgpu_match_stereo(ctypes.byref(pairs[i].left), ctypes.byref(pairs[i].right),
                                         ctypes.byref(pairs[i].left_valid), ctypes.byref(pairs[i].right_valid),
                                         pairs[i].disparity_min, pairs[i].num_disparities,
                                         ctypes.byref(pairs[i].options), ctypes.byref(pairs[i].out), sptr)
            if st != 0:
                raise RuntimeError(lib.r3dgpu_last_error().decode())
            b.record(stream)
            lat.append((a, b))
        p1.record(stream)
        barrier()
        pp_ms = max_over_ranks(p0.elapsed_time(p1))
        lats = sorted(a.elapsed_time(b) for a, b in lat)
        per_pair = {"value": cells_job / (pp_ms * 1e-3) / 1e9, "unit": "Gcells/s", "ms_per_batch": pp_ms,
                    "latency_ms": {"p50": float(np.percentile(lats, 50)), "p99": float(np.percentile(lats, 99)),
                                   "max": lats[-1]},
                    "kernels": "chain passes (the library's default), one call per pair"}

    # The plain one-pair-per-launch matcher: one CTA per tile (the wavefront
    # kernels, selected by the environment), one call per pair.
    per_pair_plain = None
    if not args.no_per_pair and args.plain:
        os.environ["R3DGPU_FULL_KERNEL"] = "wavefront"
        os.environ["R3DGPU_RANGED_KERNEL"] = "ranged"
        try:
            barrier()
            p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            p0.record(stream)
            for i in range(n):
                st = lib.r3dgpu_match_stereo(ctypes.byref(pairs[i].left), ctypes.byref(pairs[i].right),
                                             ctypes.byref(pairs[i].left_valid), ctypes.byref(pairs[i].right_valid),
                                             pairs[i].disparity_min, pairs[i].num_disparities,
                                             ctypes.byref(pairs[i].options), ctypes.byref(pairs[i].out), sptr)
                if st != 0:
                    raise RuntimeError(lib.r3dgpu_last_error().decode())
            p1.record(stream)
            barrier()
            pl_ms = max_over_ranks(p0.elapsed_time(p1))
        finally:
            del os.environ["R3DGPU_FULL_KERNEL"]
            del os.environ["R3DGPU_RANGED_KERNEL"]
        per_pair_plain = {"value": cells_job / (pl_ms * 1e-3) / 1e9, "unit": "Gcells/s",
                          "ms_per_batch": pl_ms,
                          "kernels": "one CTA per tile (skewed-wavefront kernels), one call per pair"}

    if rank == 0:
        peak, peak_kind = measured_peaks()
        # The SGM launches of a round run concurrently (one stream per kernel
        # shape); the unit of the roofline is a round's SGM stage, timed from
        # its fork to its join on the launching stream.
        rounds = max(sum(1 for e in launch_log if e["kernel"] == "sgm_round"), 1)
        sgm_ms = prof.sgm_ms / rounds
        alg_bytes = (ALG_BYTES_PER_CELL * prof.sgm_cells + ALG_BYTES_PER_PIXEL * prof.sgm_pixels) / rounds
        achieved = alg_bytes / (sgm_ms * 1e-3) / 1e9 if sgm_ms > 0 else 0.0
        sm_count = torch.cuda.get_device_properties(dev).multi_processor_count
        clocks = clk.summary()
        int_peak = sm_count * 128 * (clocks.get("sm_max_mhz") or 1965.0) * 1e6 / 1e12
        int_achieved = INT_OPS_PER_CELL * prof.sgm_cells / max(prof.sgm_ms * 1e-3, 1e-12) / 1e12
        line = {
            "metric": METRIC, "value": value, "unit": "Gcells/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u16", "data": "synthetic",
            "config": {"workload": args.workload, "pairs": len(all_specs), "full_range_cells_per_step": cells_job,
                       "aggregated_cells_per_step": total_cells, "l2": "inputs larger than L2 (126 MB)",
                       "parallelism": f"weak: {args.pairs} x {world} pairs split across {world} rank(s) by "
                                      "longest processing time (shard.shard_pairs), one batch per rank"},
            "e2e": {"value": e2e_value, "unit": "Gcells/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_ms / args.steps},
            "gpu_launches": int(launches),
            "roofline": pass_roofline(launch_log, peak, peak_kind),
            "stage_roofline": {"bound": "hbm", "kernel": "SGM stage of a round (fork to join of its chain-pass waves)",
                               "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                               "alg_bytes_per_cell": ALG_BYTES_PER_CELL, "alg_bytes_per_pixel": ALG_BYTES_PER_PIXEL,
                               "avg_stage_ms": sgm_ms, "stages": rounds, "alg_bytes_per_stage": alg_bytes,
                               "stage_ms_of_first_step": [round(e["ms"], 2) for e in launch_log
                                                          if e["kernel"] == "sgm_round"][:rounds // max(args.steps, 1)],
                               "sgm_share_of_step": prof.sgm_ms / max(ms, 1e-9)},
            "int_roofline": {"ops_per_cell": INT_OPS_PER_CELL, "achieved_tops": int_achieved,
                             "nominal_int32_tops": int_peak, "frac": int_achieved / int_peak},
            "clocks": clocks,
        }
        if line["roofline"] is None:
            line["roofline"] = dict(line["stage_roofline"])
        breakdown = {}
        for e in launch_log:
            if e["kernel"] == "sgm_round" or e.get("pass"):
                continue
            k = f"{e['kernel']}:{e['shape']}"
            b = breakdown.setdefault(k, {"launches": 0, "ms": 0.0, "cells": 0, "tiles": 0})
            b["launches"] += 1
            b["ms"] += e["ms"]
            b["cells"] += e["cells"]
            b["tiles"] += e["tiles"]
        for b in breakdown.values():
            b["gcells_per_s"] = b["cells"] / max(b["ms"], 1e-9) / 1e6
        line["sgm_breakdown"] = breakdown
        if per_pair is not None:
            line["per_pair"] = per_pair
            line["batched_vs_per_pair"] = value / per_pair["value"]
        if per_pair_plain is not None:
            line["per_pair_plain"] = per_pair_plain
            line["batched_vs_plain_per_pair"] = value / per_pair_plain["value"]
        if not args.no_cpu_baseline and world == 1:
            # The CPU baseline and the other stages' lines at N = 1 only.
            gpu_maps = {i: dD[i].cpu().numpy() for i in range(n)
                        if specs[i]["w"] * specs[i]["h"] * specs[i]["nd"] ==
                        min(q["w"] * q["h"] * q["nd"] for q in specs)}
            line["cpu_baseline"] = cpu_baseline(specs, gpu_maps)

            def extra(fn, *a):
                # A failing side measurement is reported in the line, which stands.
                try:
                    return fn(*a)
                except Exception as e:  # noqa: BLE001
                    import traceback

                    traceback.print_exc()
                    return {"error": f"{type(e).__name__}: {e}"}

            line["multi_view"] = extra(measure_combine, lib, dev, stream, args.steps, args.warmup, peak)
            line["rectify"] = extra(measure_rectify, lib, dev, stream, args.steps, args.warmup, peak)
            # The depth stage of a 32-view scene end to end; the
            # separate depth-stage and one-view lines stay available as
            # --workload depth / view.
            line["scene32"] = extra(measure_scene, lib, dev, stream, 2, 1)
        if args.serve and world == 1:
            # In a fresh process, with this one's device memory given back.
            del dL, dR, dD, dC
            _native_check(lib, lib.r3dgpu_release_workspace())
            torch.cuda.empty_cache()
            out = subprocess.run([sys.executable, os.path.abspath(__file__), "--serve-only",
                                  str(n * args.steps / (ms * 1e-3)), "--pairs", str(args.pairs), "--seed",
                                  str(args.seed), "--serve-seconds", str(args.serve_seconds), "--serve-workers",
                                  str(args.serve_workers), "--serve-batch", str(args.serve_batch)],
                                 capture_output=True, text=True)
            if out.returncode == 0:
                line["serving"] = json.loads(out.stdout.strip().splitlines()[-1])
            else:
                # The batch's line stands; the sweep's failure is reported in it.
                sys.stderr.write(out.stderr)
                line["serving"] = {"error": f"serving sweep exited {out.returncode}",
                                   "stderr_tail": out.stderr.strip().splitlines()[-6:]}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
