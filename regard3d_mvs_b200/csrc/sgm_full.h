// The full-range SGM tile kernel (sgm_full.cu): launch shapes and the layout
// of its per-CTA global scratch.
#pragma once

#include <cstddef>
#include <cstdint>

#include "sgm.h"

namespace r3dgpu {

constexpr int kSgmFullThreads = 512;  // largest CTA

// G lanes per tile row, K label pairs per lane (2 * G * K >= nd).
struct SgmFullShape {
  int g_;
  int k_;
};

struct SgmFullSlot {
  size_t rec_a, rec_b, info, seam, rkeys, sa, cost, total;
  int64_t seam_pix;  // bytes per seam pixel: 3 vectors of ndpad + 8 labels, 16 bytes of minima
  int64_t rk;        // right-WTA keys per row
};

R3D_HOSTDEV SgmFullSlot sgm_full_slot_layout(int w, int h, int nd, int ndpad) {
  SgmFullSlot L{};
  const size_t px = static_cast<size_t>(w) * static_cast<size_t>(h);
  const size_t cells = px * static_cast<size_t>(nd);
  size_t o = 0;
  L.rec_a = o;
  o += sgm_align16(px * 8);
  L.rec_b = o;
  o += sgm_align16(px * 8);
  L.info = o;
  o += sgm_align16(px * 16);
  L.seam_pix = 3 * 2 * (static_cast<int64_t>(ndpad) + 8) + 16;
  L.seam = o;
  o += sgm_align16(2 * static_cast<size_t>(w) * static_cast<size_t>(L.seam_pix));
  L.rk = static_cast<int64_t>(w) + nd;
  L.rkeys = o;
  o += sgm_align16(static_cast<size_t>(h) * static_cast<size_t>(L.rk) * 4);
  L.sa = o;
  o += sgm_align16(cells * 2);
  L.cost = o;
  o += sgm_align16(cells);
  L.total = o;
  return L;
}

// Launch plan of the full-range kernel for nd labels ({0, 0} shape: more
// labels than the kernel takes). Chosen from the tuned table, or from the
// environment (R3DGPU_FULL_SHAPE="G,K", R3DGPU_FULL_ROWS=n) for tuning runs.
struct SgmFullPlan {
  SgmFullShape shape;
  int rows;
};
SgmFullPlan sgm_full_plan(int nd, int smem_optin);
bool sgm_full_shape_compiled(SgmFullShape sh);
int sgm_full_smem(SgmFullShape sh, int rows);
// Most band rows (a multiple of 32 / G, at most max_rows) that fit the device's shared memory.
int sgm_full_rows(SgmFullShape sh, int smem_optin, int max_rows);
void launch_sgm_full(SgmFullShape sh, int nd, const SgmMatch* dm, const SgmJob* dj, int njobs, int rows, int grid,
                     unsigned char* scratch, size_t slot_bytes, int* counter, cudaStream_t s);

}  // namespace r3dgpu
