// The ranged SGM tile kernel (sgm_ranged.cu): tiles whose pixels carry their
// own label ranges (the finer levels of the hierarchy). Launch shapes and the
// layout of its per-CTA global scratch.
#pragma once

#include <cstddef>
#include <cstdint>

#include "sgm.h"

namespace r3dgpu {

constexpr int kSgmRangedThreads = 512;  // largest CTA
constexpr int kSgmRangedVecs = 11;      // path vectors kept per row: V 3, DB 4, DA 2, H 2

// G lanes per tile row, K label pairs per lane: a row holds 2 * G * K labels
// of a pixel at a time ("narrow" pixels fit; wider ones are processed in
// chunks of that size).
struct SgmRangedShape {
  int g_;
  int k_;
};

struct SgmRangedSlot {
  size_t rec_a, rec_b, info, row_start, row_shift, seam, wide, rkeys, sa, cost, total;
  int64_t seam_pix;  // bytes per seam pixel: 16 bytes of meta, then 3 vectors of ndw labels
  int64_t rk;        // right-WTA keys per row
};

// ndw: label capacity of a wide vector (the group's largest per-pixel label
// count, at least the narrow width, a multiple of 16).
R3D_HOSTDEV SgmRangedSlot sgm_ranged_slot_layout(int w, int h, unsigned long long cells, int nd, int ndw, int rows) {
  SgmRangedSlot L{};
  const size_t px = static_cast<size_t>(w) * static_cast<size_t>(h);
  size_t o = 0;
  L.rec_a = o;
  o += sgm_align16(px * 16);
  L.rec_b = o;
  o += sgm_align16(px * 16);
  L.info = o;
  o += sgm_align16(px * 16);
  L.row_start = o;
  o += sgm_align16((static_cast<size_t>(h) + 1) * 4);
  L.row_shift = o;
  o += sgm_align16(static_cast<size_t>(h) * 4);
  L.seam_pix = 16 + 3 * 2 * static_cast<int64_t>(ndw);
  L.seam = o;
  o += sgm_align16(2 * static_cast<size_t>(w) * static_cast<size_t>(L.seam_pix));
  L.wide = o;
  o += sgm_align16(static_cast<size_t>(rows) * kSgmRangedVecs * static_cast<size_t>(ndw) * 2);
  L.rk = static_cast<int64_t>(w) + nd;
  L.rkeys = o;
  o += sgm_align16(static_cast<size_t>(h) * static_cast<size_t>(L.rk) * 4);
  L.sa = o;
  o += sgm_align16(static_cast<size_t>(cells) * 2);
  L.cost = o;
  o += sgm_align16(static_cast<size_t>(cells));
  L.total = o;
  return L;
}

struct SgmRangedPlan {
  SgmRangedShape shape;
  int rows;
};

// Label width of the kernel shape for a tile with the given label statistics
// (kTileStats ints: the largest num, then the pixels above each of
// kTileStatWidths): the narrowest shape that leaves at most a small share of
// the tile's pixels wide (R3DGPU_RANGED_WIDE_FRAC, default 0.002), or the
// shape that R3DGPU_RANGED_SHAPE="G,K" forces for tuning and tests.
int sgm_ranged_width_for(const int* stats, int64_t pixels);
// Kernel shape (G, K) of a label width returned by sgm_ranged_width_for.
SgmRangedShape sgm_ranged_shape_for_width(int width);
// Rows per band (R3DGPU_RANGED_ROWS=n overrides the default for tuning).
SgmRangedPlan sgm_ranged_plan(SgmRangedShape shape, int smem_optin);
int sgm_ranged_smem(SgmRangedShape sh, int rows);
// Wide-vector capacity for a group whose largest per-pixel label count is max_num.
int sgm_ranged_ndw(SgmRangedShape sh, int max_num);
void launch_sgm_ranged(SgmRangedShape sh, const SgmMatch* dm, const SgmJob* dj, int njobs, int rows, int ndw,
                       int grid, unsigned char* scratch, size_t slot_bytes, int* counter, cudaStream_t s);

}  // namespace r3dgpu
