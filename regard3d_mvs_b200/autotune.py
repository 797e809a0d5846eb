"""Autotuner for the SGM launch shapes: measures candidates on the GPU and
writes the table that the library reads (regard3d_mvs_b200/csrc/tuning.h).

The chain passes' shape (lanes per chain G, label pairs per lane K; rows of
up to 1.5x the label count) is chosen per label count in isolation: the SGM
stage time (fork to join, from the library's CUDA-event profile) of a batch
of four single-level pairs (1536..4096 wide, 4:3) of that label count, the
minimum of three runs per candidate, the built-in default measured before and
after the candidates; a candidate wins when it beats the default by more
than 3 %. With --plain the one-CTA-per-tile kernels' shapes and band rows,
the ranged kernel's band rows per label width and the share of wide pixels a
tile may keep are searched coordinate-wise on a mixed batch drawn like the
batched workload (pairs of uneven size, label counts from {64, 128, 192,
256, 384}, half of them hierarchical), a candidate replacing the current
entry when it shortens the stage by more than 1 %. The table is written only
where it beats the built-in defaults, and entries of the kinds not searched
are kept from the existing table.

    python -m regard3d_mvs_b200.autotune [--out regard3d_mvs_b200/tuning_b200.txt] [--pairs 24] [--plain]
"""

from __future__ import annotations

import argparse
import ctypes
import math
import os
import time

import numpy as np

from . import _native
from .stereo import Matcher
from .types import CDisparityMap, CPair, CProfile, CSynthParams, CViewU8, CViewU16, StereoOptions, to_c_options

HERE = os.path.dirname(os.path.abspath(__file__))
FULL_SHAPES = ((8, 4), (8, 8), (16, 4), (8, 12), (16, 6), (16, 8), (8, 16), (16, 12), (32, 8), (32, 12))
PATH_SHAPES = ((2, 16), (4, 8), (4, 12), (4, 16), (8, 8), (8, 12), (8, 16), (16, 8), (16, 12), (16, 16), (32, 8),
               (32, 12))
FULL_ND = (384, 256, 192, 128, 64)
ROWS = (64, 48, 32, 24, 16)
ND_CHOICES = (64, 128, 192, 256, 384)


def mixed_specs(n: int, seed: int):
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n):
        w = int(round(math.exp(rng.uniform(math.log(1024), math.log(6048)))))
        h = int(round(w / (1.5 if rng.random() < 0.5 else 4.0 / 3.0)))
        nd = int(ND_CHOICES[rng.integers(0, len(ND_CHOICES))])
        hier = i % 2 == 1
        o = StereoOptions(levels=3, range_radius=0, range_margin=8) if hier else StereoOptions(levels=0)
        specs.append((w, h, nd, o))
    return specs


class Bench:
    """Device-resident synthetic pairs and the SGM stage time of one batch call."""

    def __init__(self, specs, seed=99):
        import torch

        self.m = Matcher()
        self.lib = self.m.lib
        dev = torch.device("cuda:0")
        self.keep = []
        self.pairs = (CPair * len(specs))()
        for i, (w, h, nd, opts) in enumerate(specs):
            p = CSynthParams(w, h, nd, seed + i, 1.5, 2.0, 8, 0.0, 0.0)
            L = np.empty((h, w), np.uint8)
            R = np.empty_like(L)
            _native.check(self.lib, self.lib.r3dgpu_synth_pair(ctypes.byref(p), L.ctypes.data, R.ctypes.data, None))
            dl = torch.from_numpy((L.astype(np.uint16) * 257).view(np.int16)).to(dev)
            dr = torch.from_numpy((R.astype(np.uint16) * 257).view(np.int16)).to(dev)
            dd = torch.empty((h, w), dtype=torch.float32, device=dev)
            self.keep += [dl, dr, dd]
            q = self.pairs[i]
            q.left, q.right = CViewU16(dl.data_ptr(), w, h, w), CViewU16(dr.data_ptr(), w, h, w)
            q.left_valid, q.right_valid = CViewU8(), CViewU8()
            q.disparity_min, q.num_disparities = 0, nd
            q.options = to_c_options(opts)
            q.out = CDisparityMap(dd.data_ptr(), None, w, 0, 0, 0, 0, 0)

    def stage_ms(self, table: list[str], reps: int = 2) -> float:
        """Min over reps of the batch's SGM stage time with `table` in force."""
        os.environ["R3DGPU_TUNING"] = ";".join(table) if table else "#"
        best = float("inf")
        for _ in range(reps):
            self.lib.r3dgpu_profile_enable(1)
            prof = CProfile()
            self.lib.r3dgpu_profile_take(ctypes.byref(prof))
            _native.check(self.lib, self.lib.r3dgpu_match_stereo_batch(self.pairs, len(self.pairs), None))
            self.lib.r3dgpu_profile_take(ctypes.byref(prof))
            self.lib.r3dgpu_profile_enable(0)
            self.lib.r3dgpu_profile_launches(None, 0)
            best = min(best, prof.sgm_ms)
        return best


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "tuning_b200.txt"))
    ap.add_argument("--pairs", type=int, default=24)
    ap.add_argument("--seed", type=int, default=77)
    ap.add_argument("--plain", action="store_true", help="also tune the one-CTA-per-tile kernels")
    args = ap.parse_args()
    import torch

    t0 = time.time()
    searched = {"path"} | ({"full", "ranged", "ranged_wide_frac"} if args.plain else set())
    kept = []
    if os.path.exists(args.out):
        with open(args.out) as f:
            for ln in f:
                body = ln.split("#", 1)[0].strip()
                if body and body.split()[0] not in searched:
                    kept.append(body)
    entries: dict[str, str] = {}

    def table(extra=None):
        return kept + list({**entries, **(extra or {})}.values())

    summary = []
    for nd in FULL_ND:
        iso = Bench([(w, (w * 3) // 4, nd, StereoOptions(levels=0)) for w in (1536, 2048, 3072, 4096)],
                    seed=args.seed + nd)
        iso.stage_ms(kept, reps=1)  # allocations
        base = iso.stage_ms(kept, reps=3)
        best, pick = base, None
        for g, k in (s for s in PATH_SHAPES if nd <= 2 * s[0] * s[1] <= 1.5 * nd):
            entry = f"path {nd} {g} {k}"
            ms = iso.stage_ms(kept + [entry], reps=3)
            print(f"{entry}: {ms:.1f} ms (default {base:.1f} ms)", flush=True)
            if ms < best:
                best, pick = ms, entry
        base = min(base, iso.stage_ms(kept, reps=3))
        if pick is not None and best < 0.97 * base:
            entries[f"p{nd}"] = pick
        summary.append(f"{nd} labels: default {base:.1f} ms, {pick or '-'} {best:.1f} ms")
        del iso
    bench = Bench(mixed_specs(args.pairs, args.seed), seed=args.seed)
    bench.stage_ms(kept, reps=1)  # allocations
    best = bench.stage_ms(table(), reps=3)
    if args.plain:
        for nd in FULL_ND:
            for g, k in (s for s in FULL_SHAPES if nd <= 2 * s[0] * s[1] <= 1.5 * nd):
                for rows in ROWS:
                    entry = f"full {nd} {g} {k} {rows}"
                    ms = bench.stage_ms(table({f"f{nd}": entry}))
                    print(f"{entry}: {ms:.1f} ms", flush=True)
                    if ms < best * 0.99:
                        best, entries[f"f{nd}"] = ms, entry
        for width in (32, 64, 128):
            for rows in ROWS:
                entry = f"ranged {width} {rows}"
                ms = bench.stage_ms(table({f"r{width}": entry}))
                print(f"{entry}: {ms:.1f} ms", flush=True)
                if ms < best * 0.99:
                    best, entries[f"r{width}"] = ms, entry
        for frac in (0.0005, 0.001, 0.004, 0.008):
            entry = f"ranged_wide_frac {frac}"
            ms = bench.stage_ms(table({"frac": entry}))
            print(f"{entry}: {ms:.1f} ms", flush=True)
            if ms < best * 0.99:
                best, entries["frac"] = ms, entry
    final = table()
    check_tuned, check_base = bench.stage_ms(final, reps=3), bench.stage_ms(kept, reps=3)
    keep = final if entries and check_tuned < check_base else kept
    verdict = ("" if keep is final else " (no candidate beat the defaults by more than 1 %: defaults kept)"
               if not entries else " (not better: defaults kept)")
    name = torch.cuda.get_device_name(0)
    with open(args.out, "w") as f:
        f.write(f"# SGM launch shapes chosen by regard3d_mvs_b200/autotune.py on {name} ({time.time() - t0:.0f} s):\n")
        f.write(f"# SGM stage of a {args.pairs}-pair mixed batch: defaults {check_base:.1f} ms, "
                f"this table {check_tuned:.1f} ms{verdict}\n")
        for ln in summary:
            f.write(f"# chain passes, 4 single-level pairs of {ln}\n")
        f.write("# fields: path <nd> <G> <K> | full <nd> <G> <K> <rows> | ranged <width> <rows> | "
                "ranged_wide_frac <f> | ranged_general_width <w>\n")
        for ln in keep:
            f.write(ln + "\n")
    print(f"wrote {args.out}: defaults {check_base:.1f} ms, tuned {check_tuned:.1f} ms", flush=True)


if __name__ == "__main__":
    main()
