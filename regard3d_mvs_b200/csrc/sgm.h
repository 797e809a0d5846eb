// The SGM tile kernel (sgm.cu): Hamming costs, 8-path aggregation in two
// passes of four paths, winner-takes-all and the acceptance rules of one tile
// of one match, for every tile of a job table in one persistent launch.
#pragma once

#include <cstddef>
#include <cstdint>

#include "kernels.h"

namespace r3dgpu {

constexpr int kSgmMaxRows = 16;    // rows of a band (one warp each), upper bound
constexpr int kSgmPF = 2;          // prefetch distance (pixels) of costs / partial sums / seam
constexpr int kSgmPFSlots = 4;     // per-row prefetch ring slots (power of two, > kSgmPF)
constexpr int kSgmSeamSlots = 8;   // seam ring slots (power of two, >= kSgmPF + 4)
constexpr int kSgmQueue = kSgmPF + 2;  // per-row record queue length

// One match of one level: base image (the left image, or the mirrored right
// image for the right-to-left match) against its partner.
struct SgmMatch {
  const uint16_t* base;  // base image, u16
  int64_t base_stride;
  const uint64_t* cbase;  // Census of the base image
  int64_t cb_stride;
  const uint64_t* cpart;  // Census of the partner image
  int64_t cp_stride;
  const RowInterval* bv;  // valid columns of every base row
  const RowInterval* pv;  // valid columns of every partner row
  const uint16_t* rlo;    // per-pixel label ranges (null: full range)
  const uint16_t* rnum;
  int64_t r_stride;
  int wb, wp, h;
  int dmin, nd;  // nd: aligned label count
  int p1, invalid_cost, subpixel;
  float uniqueness;
  int lr_max_diff, diagonal_lr, confidence;
  int sum_no_carry;   // 1 if 8 paths can never exceed 65535 (plain 32-bit adds of packed sums are exact)
  int term_u8;        // 1 if every P2 of the LUT is <= 255: a path's term L - C fits one byte
  uint16_t lut[256];  // P2 by 8-bit intensity step
};

// One tile of one match.
struct SgmJob {
  int match;
  int x0, y0, w, h;
  int pad_;
  float* disp;  // w * h, tile-local, row-major
  float* conf;  // w * h or null
  unsigned long long* cells;  // receives the tile's label count
  uint16_t* volume;  // optional: aggregated volume S, packed per pixel in row-major pixel order
};

// Per-CTA global scratch of a tile job (offsets in bytes, 16-byte aligned).
struct SgmSlotLayout {
  size_t rec_a, rec_b, info, row_start, row_shift, seam, rkeys, sa, cost, total;
  int64_t seam_pix_bytes;  // bytes of one seam pixel
  int64_t rk;              // right-WTA keys per row
};

R3D_HOSTDEV size_t sgm_align16(size_t v) { return (v + 15) & ~static_cast<size_t>(15); }

R3D_HOSTDEV SgmSlotLayout sgm_slot_layout(int w, int h, unsigned long long cells, int maxc, int nd) {
  SgmSlotLayout L{};
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
  // Seam pixel: 3 path vectors of 64 * maxc + 8 labels, then 16 bytes of meta.
  L.seam_pix_bytes = 3 * (128 * static_cast<int64_t>(maxc) + 16) + 16;
  L.seam = o;
  o += sgm_align16(2 * static_cast<size_t>(w) * static_cast<size_t>(L.seam_pix_bytes));
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

// Shared-memory layout of the kernel (bytes).
struct SgmSmemLayout {
  int vst;          // u16 stride of one path vector: 8 pad + 64 * maxc + 8 pad
  int row_bytes;    // per-row block
  int ring_off, mins_off, meta_off, cbuf_off, sabuf_off;  // within a row block
  int seam_slot_bytes;
  int rows_off, seam_off, total;
};

R3D_HOSTDEV SgmSmemLayout sgm_smem_layout(int maxc, int rows) {
  SgmSmemLayout L{};
  L.vst = 64 * maxc + 16;
  const int vec_bytes = 2 * L.vst;
  L.ring_off = 0;
  L.mins_off = L.ring_off + 11 * vec_bytes;
  L.meta_off = L.mins_off + 48;  // 11 mins (u32), padded
  L.cbuf_off = L.meta_off + 16;  // 4 pixel metas (u32)
  L.sabuf_off = L.cbuf_off + kSgmPFSlots * 64 * maxc;
  L.row_bytes = L.sabuf_off + kSgmPFSlots * 128 * maxc;
  L.seam_slot_bytes = 3 * vec_bytes + 16;
  L.rows_off = 16;  // job id
  L.seam_off = L.rows_off + rows * L.row_bytes;
  L.total = L.seam_off + kSgmSeamSlots * L.seam_slot_bytes;
  return L;
}

// Largest label count per pixel the kernel instantiations support.
constexpr int kSgmMaxLabels = 64 * 16;

// Chunks of 64 labels an instantiation must handle for `max_num` labels.
int sgm_maxc_for(int max_num);
// Rows per band that fit the shared memory of the device.
int sgm_rows_for(int maxc, int smem_optin);

void launch_sgm(const SgmMatch* d_matches, const SgmJob* d_jobs, int njobs, int maxc, int rows, int grid,
                unsigned char* scratch, size_t slot_bytes, int* d_counter, cudaStream_t s);

}  // namespace r3dgpu
