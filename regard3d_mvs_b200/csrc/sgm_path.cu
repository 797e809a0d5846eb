// Full-range SGM tiles as eight chain passes.
//
// Semantics are those of sgm.cu (Census costs, the 8-path recurrence with
// sentinel labels, the sum modulo 2^16, winner-takes-all and the acceptance
// rules of rhiestan/Regard3D_MVS src/r3d/stereo/stereo_matcher.cpp:305-353,
// 446-525 and sgm_kernels.cpp:176-263, 387-403). Because the aggregated cost
// is a sum of 8 independent 1-D recurrences restarted at tile borders, each
// path direction is a set of independent chains: the tile's rows for the
// horizontal paths, its columns for the vertical ones and its diagonals for
// the diagonal ones. This file runs them that way:
//
//   cost kernel     u8 costs of every cell of the wave (written once);
//   8 path passes   one launch per direction (and kernel shape); G lanes walk
//                   one chain, K label pairs per lane, 32 / G chains per warp,
//                   the predecessor vector in registers (its d -+ 1 neighbours
//                   across lanes by shuffle), the next pixel's costs and sums
//                   loaded while the current one is computed. The first pass
//                   writes the sum volume, the next six add to it, the last
//                   adds its path and takes the winner-takes-all records;
//   accept kernel   the acceptance rules, subpixel fit and confidence per
//                   pixel, into the tile's disparity and confidence.
//
// No CTA barrier is on the chain's critical path and every tile spreads over
// as many SMs as it has chains, so one small pair fills the GPU as well as a
// batch does. HBM traffic per aggregated cell: 1 B cost write, 8 x 1 B cost
// reads, 2 B + 6 x 4 B + 2 B sum traffic.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "common.cuh"
#include "sgm_path.h"
#include "sgm_simd.cuh"
#include "tuning.h"

namespace r3dgpu {

namespace {

using sgm_simd::group_umin;
using sgm_simd::kSent2;
constexpr float kInfF = __builtin_huge_valf();
constexpr int kPathThreads = 256;

inline size_t align256(size_t v) { return (v + 255) & ~static_cast<size_t>(255); }

// Last job whose prefix value (field selected by `key`) is <= v; jobs are
// ordered so that every prefix is non-decreasing.
template <class Key>
R3D_DEVICE int find_job(const SgmPathJob* jobs, int njobs, int64_t v, Key key) {
  int lo = 0, hi = njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (key(jobs[mid]) <= v) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Whether the caller's cancellation flag is set (read once per chain block,
// by lane 0 for the whole warp; never a wait).
R3D_DEVICE bool cancelled(const int* cancel) {
  int c = 0;
  if (cancel != nullptr) c = *reinterpret_cast<const volatile int*>(cancel);
  return r3dsimt::shfl(static_cast<uint32_t>(c), 0) != 0;
}

// Start pixel and length of chain c of a direction (dx, dy) in a w x h tile;
// length 0 for c past the class's last chain.
R3D_DEVICE void chain_geometry(int cls, int dx, int dy, int w, int h, int64_t c, int& sx, int& sy, int& len) {
  sx = 0;
  sy = 0;
  len = 0;
  if (cls == 0) {
    if (c < h) {
      sx = dx > 0 ? 0 : w - 1;
      sy = static_cast<int>(c);
      len = w;
    }
  } else if (cls == 1) {
    if (c < w) {
      sx = static_cast<int>(c);
      sy = dy > 0 ? 0 : h - 1;
      len = h;
    }
  } else if (c < w) {
    const int ci = static_cast<int>(c);
    sx = dx > 0 ? ci : w - 1 - ci;
    sy = dy > 0 ? 0 : h - 1;
    len = r3dsimt::imin(h, w - ci);
  } else if (c < static_cast<int64_t>(w) + h - 1) {
    const int k = static_cast<int>(c - w + 1);
    sx = dx > 0 ? 0 : w - 1;
    sy = dy > 0 ? k : h - 1 - k;
    len = r3dsimt::imin(w, h - k);
  }
}

// ---------------------------------------------------------------- costs
// C(p, a) of stereo_matcher.cpp:305-353, u8. One warp per tile row: the
// partner Census codes the row can reach (right columns x0 - dmin - nd + 1 ..
// x0 + w - 1 - dmin) are staged in the warp's shared memory, then the lanes
// take 32 consecutive pixels and write 32 labels (one sector) at a time.
constexpr int kCostStage = 2048;  // staged partner codes per warp at most (sgm_path_fits: w + nd - 1 <= 2048)

// `stage_words` (<= kCostStage): the widest staged row of the wave (tile
// width + labels - 1), so that narrow waves run more CTAs per SM.
R3D_GLOBAL void R3D_LAUNCH_BOUNDS(kPathThreads)
    sgm_path_cost_kernel(const SgmMatch* R3D_RESTRICT matches, const SgmPathJob* R3D_RESTRICT jobs, int njobs,
                         int64_t rows, uint8_t* R3D_RESTRICT cost, int stage_words, uint16_t* R3D_RESTRICT ints) {
  R3D_DYNAMIC_SMEM(smem);
  const int lane = static_cast<int>(threadIdx.x & 31u), warp = static_cast<int>(threadIdx.x >> 5);
  const int wpb = static_cast<int>(blockDim.x) >> 5;
  uint64_t* stage = reinterpret_cast<uint64_t*>(smem) + static_cast<size_t>(warp) * stage_words;
  const int64_t nwarps = static_cast<int64_t>(gridDim.x) * wpb;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * wpb + warp; r < rows; r += nwarps) {
    const int j = find_job(jobs, njobs, r, [](const SgmPathJob& q) { return q.row_off; });
    const SgmPathJob& job = jobs[j];
    const SgmMatch& m = matches[job.match];
    const int nd = m.nd, w = job.w;
    const int y = static_cast<int>(r - job.row_off), by = job.y0 + y;
    const RowInterval lv = m.bv[by], rv = m.pv[by];
    const uint64_t* crow = m.cpart + static_cast<int64_t>(by) * m.cp_stride;
    const uint64_t* lrow = m.cbase + static_cast<int64_t>(by) * m.cb_stride;
    // Staged right column xr is stage[xr - xr0]; columns outside the valid
    // right interval are never read (their cost is invalid_cost).
    const int xr0 = job.x0 - m.dmin - nd + 1;
    const int span = w + nd - 1;
    r3dsimt::syncwarp();
    for (int k = lane; k < span; k += 32) {
      const int xr = xr0 + k;
      stage[k] = (xr >= rv.first && xr <= rv.last) ? crow[xr] : 0;
    }
    // The row's base intensities, for the pass kernels.
    {
      const uint16_t* irow = m.base + static_cast<int64_t>(by) * m.base_stride + job.x0;
      uint16_t* iout = ints + job.px_off + static_cast<int64_t>(y) * w;
      for (int x = lane; x < w; x += 32) iout[x] = irow[x];
    }
    r3dsimt::syncwarp();
    const uint32_t inv = static_cast<uint32_t>(m.invalid_cost);
    uint8_t* row_out = cost + job.cell_off + static_cast<int64_t>(y) * w * nd;
    for (int xb = 0; xb < w; xb += 32) {
      const int x = xb + lane;
      if (x >= w) continue;
      const int bx = job.x0 + x;
      const bool inside = bx >= lv.first && bx <= lv.last;
      const uint64_t cl = inside ? lrow[bx] : 0;
      uint8_t* out = row_out + static_cast<int64_t>(x) * nd;
      for (int c = 0; c < nd; c += 32) {
        const int nl = nd - c < 32 ? 16 : 32;  // nd is a multiple of 16
        uint32_t q[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (inside) {
          // Label a = c + k reads right column bx - dmin - a = xr0 + (x + nd - 1 - a).
          const int base = x + nd - 1 - c;
          const int xr_first = bx - m.dmin - c;  // right column of label c; label c + k reads xr_first - k
          if (xr_first <= rv.last && xr_first - (nl - 1) >= rv.first) {
            // Every label of the run reads a valid right column: four costs a
            // word, the two 32-bit popcounts of each Census XOR packed
            // separately by multiply-adds (each byte at most 32, no carries).
#pragma unroll
            for (int w4 = 0; w4 < 8; ++w4) {
              if (4 * w4 < nl) {
                uint32_t lo = 0, hi = 0;
#pragma unroll
                for (int i = 3; i >= 0; --i) {
                  const uint64_t d = cl ^ stage[base - 4 * w4 - i];
                  lo = lo * 256u + static_cast<uint32_t>(r3dsimt::popc(static_cast<uint32_t>(d)));
                  hi = hi * 256u + static_cast<uint32_t>(r3dsimt::popc(static_cast<uint32_t>(d >> 32)));
                }
                q[w4] = lo + hi;
              }
            }
          } else {
#pragma unroll
            for (int k = 0; k < 32; ++k) {
              if (k < nl) {
                const int xr = xr_first - k;
                const bool ok = xr >= rv.first && xr <= rv.last;
                const uint32_t v = ok ? static_cast<uint32_t>(r3dsimt::popc64(cl ^ stage[base - k])) : inv;
                q[k >> 2] |= v << (8 * (k & 3));
              }
            }
          }
        }
        *reinterpret_cast<uint4*>(out + c) = make_uint4(q[0], q[1], q[2], q[3]);
        if (nl == 32) *reinterpret_cast<uint4*>(out + c + 16) = make_uint4(q[4], q[5], q[6], q[7]);
      }
    }
  }
}

// ---------------------------------------------------------------- passes
// Pass modes. With u16 sums (any penalties): the first pass writes the sum
// volume, the next six add to it, the last adds its path and takes the
// winner-takes-all. With byte terms (every P2 <= 255): passes 1..7 write
// their path's term T_r = L_r - C (in [0, P2]) as one byte per cell, and the
// last pass forms S = L_8 + 7 C + sum T_r (at most 8 (255 + 255) < 2^16, so
// the sum modulo 2^16 is the plain sum) and takes the winner-takes-all.
enum PassMode { kFirst = 0, kAccumulate = 1, kLast = 2, kTerm = 3, kLastTerm = 4 };
constexpr int kTermArrays = 7;
// The passes of one launch: n directions, chain blocks of pass q numbered
// from start[q] (start[n] = all blocks), slot = its term array.
struct PassSet {
  int n;
  uint32_t one;  // 1 (see fma_add)
  int cls[kTermArrays], dx[kTermArrays], dy[kTermArrays], slot[kTermArrays];
  int64_t start[kTermArrays + 1];
};
constexpr int kPathStages = 4;  // ring stages of the ranged passes

// Per-halfword a + b modulo 2^16.
R3D_DEVICE uint32_t add2(uint32_t a, uint32_t b, bool no_carry) { return no_carry ? a + b : r3dsimt::vadd2(a, b); }

// a * one + b with one = 1 at run time: an integer multiply-add, which the
// FMA pipe executes, in place of an add on the ALU pipe (the pass kernels'
// packed min, byte permutes and adds keep the ALU pipe the busier one).
R3D_DEVICE uint32_t fma_add(uint32_t a, uint32_t one, uint32_t b) { return a * one + b; }

// v[j] for a runtime j in [0, K): a tree of K - 1 selects on the bits of j
// (a register array cannot be indexed at run time without local memory).
template <int N>
R3D_DEVICE void pick_level(uint32_t* t, bool hi) {
#pragma unroll
  for (int k = 0; 2 * k < N; ++k) t[k] = (2 * k + 1 < N && hi) ? t[2 * k + 1] : t[2 * k];
}
template <int K>
R3D_DEVICE uint32_t pick(const uint32_t (&v)[K], int j) {
  static_assert(K >= 2 && K <= 16, "pick: 2..16 words");
  constexpr int n1 = (K + 1) / 2, n2 = (n1 + 1) / 2, n3 = (n2 + 1) / 2;
  uint32_t t[K];
#pragma unroll
  for (int k = 0; k < K; ++k) t[k] = v[k];
  pick_level<K>(t, (j & 1) != 0);
  if constexpr (n1 > 1) pick_level<n1>(t, (j & 2) != 0);
  if constexpr (n2 > 1) pick_level<n2>(t, (j & 4) != 0);
  if constexpr (n3 > 1) pick_level<n3>(t, (j & 8) != 0);
  return t[0];
}

// Per-warp shared-memory ring of the pass kernels: Stages stages, each with
// one pixel per chain of the bytes the pass reads (Planes bytes per label:
// the cost, plus the u16 sum or the seven byte terms).
// The term passes read one byte per label and keep 8 stages in flight (their
// step is short, so 3 stages ahead left them waiting on DRAM).
// The last pass with byte terms stages eight byte planes per pixel: two
// stages (its step is long, one pixel ahead covers the DRAM latency).
template <int MODE>
struct PathMode {
  static constexpr int kPlanes = MODE == kAccumulate || MODE == kLast ? 3 : (MODE == kLastTerm ? 1 + kTermArrays : 1);
  static constexpr int kStages = MODE == kLastTerm ? 2 : (MODE == kTerm ? 8 : 4);
};
// A stage ends with one 4-byte word per lane: the aligned word of the
// intensities that holds its chain's pixel (every lane copies its own, since
// a cp.async wait covers only the waiting thread's copies).
// CTA size and resident CTAs per SM: 4-warp CTAs for the byte-term last
// pass (its eight-plane ring) and the 16-word term passes (92 registers),
// so that CTAs pack an SM's registers and shared memory finely (the 12-word
// term passes measured 12-19 % slower that way than in two 8-warp CTAs).
template <int G, int K, int MODE>
struct PathRing {
  static constexpr int kThreads = (MODE == kLastTerm || (MODE == kTerm && K >= 16)) ? 128 : kPathThreads;
  static constexpr int kMinBlocks = MODE == kLastTerm ? (K <= 8 ? 6 : 3)
                                    : MODE == kTerm   ? (K <= 8 ? 4 : (K >= 16 ? 5 : 2))
                                                      : (K <= 8 ? 3 : 2);
  static constexpr int ND = 2 * G * K;
  static constexpr int kStages = PathMode<MODE>::kStages;
  static constexpr int kPlaneBytes = (32 / G) * PathMode<MODE>::kPlanes * ND;
  static constexpr int kIntBytes = 32 * 4;
  static constexpr int kStageBytes = kPlaneBytes + kIntBytes;
  static constexpr int kWarpBytes = kStages * kStageBytes;
  // Each warp's rings, then each warp's copy of its match's P2 table.
  static constexpr int kBlockBytes = (kThreads / 32) * (kWarpBytes + 512);
};

// CTAs per SM (PathRing): four 8-warp CTAs for the 8-word term passes (64
// registers, no spills), two for the 12-word ones, five 4-warp CTAs for the
// 16-word ones; six or three 4-warp CTAs for the byte-term last pass; three
// or two 8-warp CTAs for the u16-sum passes.
//
// The step loop is unrolled by the ring depth NS so that ring slots and the
// intensity queue are indexed statically; each chain keeps running pointers
// (advanced by one pixel along the path per step) instead of recomputing
// addresses. The first pixel needs no special case: with a zero predecessor
// vector and a zero minimum, best = 0, so T = 0 and L = C there.
//
// One launch runs the passes of a PassSet: a single pass, or the seven term
// passes of a segment at once (they only read the costs and each writes its
// own term array, so their chain blocks can be taken in any order).
template <int G, int K, int MODE, bool FULL>
R3D_GLOBAL void R3D_LAUNCH_BOUNDS_MIN((PathRing<G, K, MODE>::kThreads), (PathRing<G, K, MODE>::kMinBlocks))
    sgm_path_kernel(const SgmMatch* R3D_RESTRICT matches, const SgmPathJob* R3D_RESTRICT jobs, int njobs,
                    const PassSet ps, const uint8_t* R3D_RESTRICT cost, uint16_t* sum, uint8_t* terms,
                    int64_t tstride, int4* R3D_RESTRICT info, uint32_t* rkeys, const uint16_t* R3D_RESTRICT ints,
                    const int* cancel) {
  constexpr int CPW = 32 / G;  // chains per warp
  constexpr int U = K / 4;     // units of 8 labels per lane
  constexpr int NS = PathRing<G, K, MODE>::kStages;
  constexpr bool kReadsSum = MODE == kAccumulate || MODE == kLast;
  constexpr bool kWta = MODE == kLast || MODE == kLastTerm;
  // K a multiple of 8: a lane's 2 K labels are NV 16-byte aligned pieces of
  // every byte plane (piece v = units 2 v, 2 v + 1, valid together since
  // label counts are multiples of 16).
  constexpr bool kVec = K % 8 == 0;
  constexpr int NV = K / 8;
  R3D_DYNAMIC_SMEM(smem);
  const int lane = static_cast<int>(threadIdx.x & 31u);
  const int gi = lane / G, t = lane % G;
  const int e0 = 2 * t * K;  // first label of the lane
  const int left_lane = (lane + 31) & 31, right_lane = (lane + 1) & 31;
  const int wpb = static_cast<int>(blockDim.x) >> 5;
  const int64_t nwarps = static_cast<int64_t>(gridDim.x) * wpb;
  using Ring = PathRing<G, K, MODE>;
  unsigned char* const ring = smem + static_cast<size_t>(threadIdx.x >> 5) * Ring::kWarpBytes;
  // The warp's copy of the P2 table of the match it works on (256 u16),
  // reloaded when a chain block belongs to another match.
  uint16_t* const lut = reinterpret_cast<uint16_t*>(smem + static_cast<size_t>(wpb) * Ring::kWarpBytes +
                                                    static_cast<size_t>(threadIdx.x >> 5) * 512);
  int lut_match = -1;
  unsigned char* const ring_cost = ring + gi * Ring::ND + e0;
  unsigned char* const ring_sum = ring + CPW * Ring::ND + gi * 2 * Ring::ND + 2 * e0;
  unsigned char* const ring_term = ring + CPW * Ring::ND + gi * Ring::ND + e0;  // + r * CPW * ND
  unsigned char* const ring_int = ring + Ring::kPlaneBytes + lane * 4;
  const int64_t total_blocks = ps.start[ps.n];
  const uint32_t one = ps.one;
  for (int64_t gblk = static_cast<int64_t>(blockIdx.x) * wpb + (threadIdx.x >> 5); gblk < total_blocks;
       gblk += nwarps) {
    if (cancelled(cancel)) break;
    // The pass of the block (static indices only: no local copy of ps).
    int cls = ps.cls[0], dx = ps.dx[0], dy = ps.dy[0], tslot = ps.slot[0];
    int64_t blk = gblk;
#pragma unroll
    for (int q = 1; q < kTermArrays; ++q) {
      if (q < ps.n && gblk >= ps.start[q]) {
        cls = ps.cls[q];
        dx = ps.dx[q];
        dy = ps.dy[q];
        tslot = ps.slot[q];
        blk = gblk - ps.start[q];
      }
    }
    const int j = find_job(jobs, njobs, blk, [cls](const SgmPathJob& q) { return q.blk[cls]; });
    const SgmPathJob& job = jobs[j];
    const SgmMatch& m = matches[job.match];
    if (job.match != lut_match) {  // the same for the whole warp (one chain block)
      r3dsimt::syncwarp();
      for (int k = lane; k < 128; k += 32)
        reinterpret_cast<uint32_t*>(lut)[k] = reinterpret_cast<const uint32_t*>(m.lut)[k];
      r3dsimt::syncwarp();
      lut_match = job.match;
    }
    const int w = job.w, nd = m.nd;
    const uint32_t p1x2 = static_cast<uint32_t>(m.p1) * 0x10001u;
    const bool no_carry = m.sum_no_carry != 0;
    int sx, sy, len;
    chain_geometry(cls, dx, dy, w, job.h, (blk - job.blk[cls]) * CPW + gi, sx, sy, len);
    int maxlen = len;
#pragma unroll
    for (int o = G; o < 32; o <<= 1) maxlen = r3dsimt::imax(maxlen, static_cast<int>(r3dsimt::shfl_xor(maxlen, o)));
    bool uvalid[U];
#pragma unroll
    for (int u = 0; u < U; ++u) uvalid[u] = FULL || e0 + 8 * u < nd;
    // Running offsets (cells, pixels) of the pixel being issued (NS - 1
    // ahead) and of the pixel being computed.
    const int64_t dcell = (static_cast<int64_t>(dy) * w + dx) * nd;
    const int64_t cell0 = job.cell_off + e0 + (static_cast<int64_t>(sy) * w + sx) * nd;
    const uint8_t* c_in = cost + cell0;
    const uint16_t* s_in = sum + cell0;
    const uint8_t* t_in = terms + cell0;
    uint16_t* s_out = sum + cell0;
    uint8_t* t_out = terms + cell0 + static_cast<int64_t>(tslot) * tstride;
    int64_t px_out = job.px_off + static_cast<int64_t>(sy) * w + sx;
    const int64_t dpx = static_cast<int64_t>(dy) * w + dx;
    // Intensity of the pixel being issued (each lane copies the aligned
    // 4-byte word holding it into the stage), and the parity of the
    // chain's first pixel (which half of a staged word holds the intensity:
    // pixel i's parity is par0 ^ (i & dpar)).
    const uint16_t* i_iss = ints + job.px_off + static_cast<int64_t>(sy) * w + sx;
    const uint32_t par0 = static_cast<uint32_t>(reinterpret_cast<uintptr_t>(i_iss) >> 1) & 1u;
    const uint32_t dpar = static_cast<uint32_t>(dpx) & 1u;
    int x = sx, y = sy;

    auto issue = [&](int i, int st) {
      if (i < len) {
        unsigned char* rc = ring_cost + st * Ring::kStageBytes;
        if constexpr (kVec) {
#pragma unroll
          for (int v = 0; v < NV; ++v) {
            if (uvalid[2 * v]) {
              r3dsimt::cp_async16(rc + 16 * v, c_in + 16 * v);
              if constexpr (kReadsSum) {
                r3dsimt::cp_async16(ring_sum + st * Ring::kStageBytes + 32 * v, s_in + 16 * v);
                r3dsimt::cp_async16(ring_sum + st * Ring::kStageBytes + 32 * v + 16, s_in + 16 * v + 8);
              }
              if constexpr (MODE == kLastTerm) {
#pragma unroll
                for (int r = 0; r < kTermArrays; ++r)
                  r3dsimt::cp_async16(ring_term + st * Ring::kStageBytes + r * CPW * Ring::ND + 16 * v,
                                      t_in + r * tstride + 16 * v);
              }
            }
          }
        } else {
#pragma unroll
          for (int u = 0; u < U; ++u) {
            if (uvalid[u]) {
              r3dsimt::cp_async8(rc + 8 * u, c_in + 8 * u);
              if constexpr (kReadsSum) r3dsimt::cp_async16(ring_sum + st * Ring::kStageBytes + 16 * u, s_in + 8 * u);
              if constexpr (MODE == kLastTerm) {
#pragma unroll
                for (int r = 0; r < kTermArrays; ++r)
                  r3dsimt::cp_async8(ring_term + st * Ring::kStageBytes + r * CPW * Ring::ND + 8 * u,
                                     t_in + r * tstride + 8 * u);
              }
            }
          }
        }
        r3dsimt::cp_async4(ring_int + st * Ring::kStageBytes,
                           reinterpret_cast<const void*>(reinterpret_cast<uintptr_t>(i_iss) & ~uintptr_t{3}));
      }
      r3dsimt::cp_async_commit();
      c_in += dcell;
      if constexpr (kReadsSum) s_in += dcell;
      if constexpr (MODE == kLastTerm) t_in += dcell;
      i_iss += dpx;
    };
#pragma unroll
    for (int k = 0; k < NS - 1; ++k) issue(k, k);
    uint32_t prev[K];
#pragma unroll
    for (int k = 0; k < K; ++k) prev[k] = 0;
    uint32_t pmin = 0;
    // Intensities and P2. With four stages or more, the next pixel's stage
    // has landed when this pixel is computed, so the P2 of the step into the
    // next pixel is looked up one step ahead, off the step's critical path
    // (iprev is then this pixel's intensity); with two stages the P2 of the
    // step into this pixel is looked up in its step (iprev is the previous
    // pixel's intensity). The first step's P2 is unused: its predecessor
    // vector is zero.
    constexpr bool kAheadP2 = NS >= 4;
    int iprev = 0;
    uint32_t p2next = 0;
    if constexpr (kAheadP2) {
      r3dsimt::cp_async_wait<NS - 2>();  // the first of the NS - 1 stages in flight
      const uint32_t iw0 = *reinterpret_cast<const uint32_t*>(ring_int);
      iprev = static_cast<int>((iw0 >> (16u * par0)) & 0xFFFFu);
    }

    auto step = [&](const int i, const int q) {
      const bool on = i < len;
      constexpr int kNext = NS - 1;
      issue(i + kNext, (q + kNext) % NS);
      uint32_t pen;
      if constexpr (kAheadP2) {
        r3dsimt::cp_async_wait<NS - 2>();  // this pixel's stage and the next one's
        const uint32_t iw = *reinterpret_cast<const uint32_t*>(ring_int + ((q + 1) % NS) * Ring::kStageBytes);
        const int inext =
            static_cast<int>((iw >> (16u * ((par0 ^ (static_cast<uint32_t>(i + 1) & dpar)) & 1u))) & 0xFFFFu);
        pen = pmin + p2next;
        const int dn = inext - iprev;
        p2next = lut[(dn < 0 ? -dn : dn) >> 8];
        iprev = inext;
      } else {
        r3dsimt::cp_async_wait<NS - 1>();
        const uint32_t iw = *reinterpret_cast<const uint32_t*>(ring_int + q * Ring::kStageBytes);
        const int icur =
            static_cast<int>((iw >> (16u * ((par0 ^ (static_cast<uint32_t>(i) & dpar)) & 1u))) & 0xFFFFu);
        const int dn = icur - iprev;
        iprev = icur;
        pen = pmin + lut[(dn < 0 ? -dn : dn) >> 8];
      }
      const unsigned char* sc = ring_cost + q * Ring::kStageBytes;
      uint2 craw[U];
      if constexpr (kVec) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const uint4 w4 = uvalid[2 * v] ? *reinterpret_cast<const uint4*>(sc + 16 * v) : make_uint4(0, 0, 0, 0);
          craw[2 * v] = make_uint2(w4.x, w4.y);
          craw[2 * v + 1] = make_uint2(w4.z, w4.w);
        }
      } else {
#pragma unroll
        for (int u = 0; u < U; ++u)
          craw[u] = uvalid[u] ? *reinterpret_cast<const uint2*>(sc + 8 * u) : make_uint2(0, 0);
      }
      uint32_t c2[K];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        c2[4 * u + 0] = r3dsimt::perm(craw[u].x, 0u, 0x4140u);
        c2[4 * u + 1] = r3dsimt::perm(craw[u].x, 0u, 0x4342u);
        c2[4 * u + 2] = r3dsimt::perm(craw[u].y, 0u, 0x4140u);
        c2[4 * u + 3] = r3dsimt::perm(craw[u].y, 0u, 0x4342u);
      }
      // out = L_r = C + T_r with T_r = best - min L(q).
      const uint32_t pen2 = pen * 0x10001u;
      const uint32_t negmp = pmin * 0xFFFEFFFFu;  // -(pmin in both halves) modulo 2^32
      const uint32_t hl = r3dsimt::shfl(prev[K - 1], left_lane);
      const uint32_t hr = r3dsimt::shfl(prev[0], right_lane);
      uint32_t wv[K + 2];
      wv[0] = t > 0 ? hl : kSent2;
#pragma unroll
      for (int k = 0; k < K; ++k) wv[1 + k] = prev[k];
      wv[K + 1] = t + 1 < G ? hr : kSent2;
      uint32_t out[K], tr[K];
      uint32_t mprev = r3dsimt::perm(wv[0], wv[1], 0x5432u);
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const uint32_t mnext = r3dsimt::perm(wv[k + 1], wv[k + 2], 0x5432u);
        const uint32_t nb = r3dsimt::vmin2(mprev, mnext);
        const uint32_t best = r3dsimt::vmin2(wv[k + 1], r3dsimt::vaddmin2(nb, p1x2, pen2));
        tr[k] = fma_add(best, one, negmp);
        out[k] = fma_add(tr[k], one, c2[k]);
        mprev = mnext;
      }
      // Minimum over the lane's labels (a tree), then over the chain's lanes.
      uint32_t mm[K];
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (!uvalid[k / 4]) out[k] = kSent2;
        mm[k] = out[k];
      }
#pragma unroll
      for (int s = 1; s < K; s <<= 1) {
#pragma unroll
        for (int k = 0; k + s < K; k += 2 * s) mm[k] = r3dsimt::vmin2(mm[k], mm[k + s]);
      }
      pmin = group_umin<G>(r3dsimt::umin(mm[0] & 0xFFFFu, mm[0] >> 16));
      uint32_t s[K];
      if constexpr (MODE == kFirst) {
        if (on) {
#pragma unroll
          for (int u = 0; u < U; ++u)
            if (uvalid[u])
              r3dsimt::st_stream(reinterpret_cast<uint4*>(s_out + 8 * u),
                                 make_uint4(out[4 * u], out[4 * u + 1], out[4 * u + 2], out[4 * u + 3]));
        }
      } else if constexpr (MODE == kTerm) {
        if (on) {
          if constexpr (kVec) {
#pragma unroll
            for (int v = 0; v < NV; ++v)
              if (uvalid[2 * v])
                r3dsimt::st_stream(reinterpret_cast<uint4*>(t_out + 16 * v),
                                   make_uint4(r3dsimt::perm(tr[8 * v], tr[8 * v + 1], 0x6420u),
                                              r3dsimt::perm(tr[8 * v + 2], tr[8 * v + 3], 0x6420u),
                                              r3dsimt::perm(tr[8 * v + 4], tr[8 * v + 5], 0x6420u),
                                              r3dsimt::perm(tr[8 * v + 6], tr[8 * v + 7], 0x6420u)));
          } else {
#pragma unroll
            for (int u = 0; u < U; ++u)
              if (uvalid[u])
                r3dsimt::st_stream8(reinterpret_cast<uint2*>(t_out + 8 * u),
                                    make_uint2(r3dsimt::perm(tr[4 * u], tr[4 * u + 1], 0x6420u),
                                               r3dsimt::perm(tr[4 * u + 2], tr[4 * u + 3], 0x6420u)));
          }
        }
      } else if constexpr (MODE == kLastTerm) {
        // S = L_8 + 7 C + sum of the seven byte terms (no halfword overflows).
#pragma unroll
        for (int k = 0; k < K; ++k) s[k] = out[k] + 7u * c2[k];
        const unsigned char* stt = ring_term + q * Ring::kStageBytes;
#pragma unroll
        for (int r = 0; r < kTermArrays; ++r) {
          uint2 tw[U];
          if constexpr (kVec) {
#pragma unroll
            for (int v = 0; v < NV; ++v) {
              const uint4 w4 = uvalid[2 * v] ? *reinterpret_cast<const uint4*>(stt + r * CPW * Ring::ND + 16 * v)
                                             : make_uint4(0, 0, 0, 0);
              tw[2 * v] = make_uint2(w4.x, w4.y);
              tw[2 * v + 1] = make_uint2(w4.z, w4.w);
            }
          } else {
#pragma unroll
            for (int u = 0; u < U; ++u)
              tw[u] = uvalid[u] ? *reinterpret_cast<const uint2*>(stt + r * CPW * Ring::ND + 8 * u) : make_uint2(0, 0);
          }
#pragma unroll
          for (int u = 0; u < U; ++u) {
            s[4 * u + 0] = fma_add(r3dsimt::perm(tw[u].x, 0u, 0x4140u), one, s[4 * u + 0]);
            s[4 * u + 1] = fma_add(r3dsimt::perm(tw[u].x, 0u, 0x4342u), one, s[4 * u + 1]);
            s[4 * u + 2] = fma_add(r3dsimt::perm(tw[u].y, 0u, 0x4140u), one, s[4 * u + 2]);
            s[4 * u + 3] = fma_add(r3dsimt::perm(tw[u].y, 0u, 0x4342u), one, s[4 * u + 3]);
          }
        }
      } else {
        const unsigned char* ss = ring_sum + q * Ring::kStageBytes;
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const uint4 sraw = uvalid[u] ? *reinterpret_cast<const uint4*>(ss + 16 * u) : make_uint4(0, 0, 0, 0);
          s[4 * u + 0] = add2(sraw.x, out[4 * u + 0], no_carry);
          s[4 * u + 1] = add2(sraw.y, out[4 * u + 1], no_carry);
          s[4 * u + 2] = add2(sraw.z, out[4 * u + 2], no_carry);
          s[4 * u + 3] = add2(sraw.w, out[4 * u + 3], no_carry);
        }
        if constexpr (MODE == kAccumulate) {
          if (on) {
#pragma unroll
            for (int u = 0; u < U; ++u)
              if (uvalid[u])
                r3dsimt::st_stream(reinterpret_cast<uint4*>(s_out + 8 * u),
                                   make_uint4(s[4 * u], s[4 * u + 1], s[4 * u + 2], s[4 * u + 3]));
          }
        }
      }
      if constexpr (kWta) {
        // Winner-takes-all over the total sums (sgm_kernels.cpp:332-358):
        // the first minimum, the second best outside +-1, and S at kb -+ 1.
        // Labels of units past nd count as 0xFFFF (they follow every valid
        // label, so they never come first among equal minima); with byte
        // terms their sum is the sentinel 0x7FFF, above every valid S (at
        // most 8 (255 + 255)), which serves as well.
        uint32_t sv[K];
#pragma unroll
        for (int k = 0; k < K; ++k) sv[k] = (MODE == kLastTerm || uvalid[k / 4]) ? s[k] : 0xFFFFFFFFu;
        // The lane's minimum and its first label, as one key S << 16 | label
        // whose minimum over the lane group is (bcost, kb).
        uint32_t mv = sv[0];
#pragma unroll
        for (int k = 1; k < K; ++k) mv = r3dsimt::vmin2(mv, sv[k]);
        const uint32_t lmin = r3dsimt::umin(mv & 0xFFFFu, mv >> 16);
        // Per word min(S - lmin, 1) is 0 in the halves at the minimum (every
        // half is >= lmin, so the subtraction borrows nothing).
        const uint32_t l2 = lmin * 0x10001u;
        uint32_t miss = 0;
#pragma unroll
        for (int k = 0; k < K; ++k) miss |= r3dsimt::vmin2(sv[k] - l2, 0x00010001u) << k;
        const uint32_t hit = ~miss & (((1u << K) - 1u) * 0x10001u);
        const uint32_t he = hit & 0xFFFFu, ho = hit >> 16;
        const uint32_t fe = he != 0 ? static_cast<uint32_t>(2 * (r3dsimt::ffs(he) - 1)) : 0xFFFFu;
        const uint32_t fo = ho != 0 ? static_cast<uint32_t>(2 * (r3dsimt::ffs(ho) - 1) + 1) : 0xFFFFu;
        const uint32_t key = group_umin<G>((lmin << 16) | (r3dsimt::umin(fe, fo) + static_cast<uint32_t>(e0)));
        const uint32_t bcost = key >> 16;
        const int kb = static_cast<int>(key & 0xFFFFu);
        // The second best outside kb -+ 1. Label kb - 1 lies in the lane's
        // word wa = (kb - 1 - e0) >> 1 (arithmetic shift; out of [0, K) in
        // other lanes): its high half only when kb - 1 - e0 is odd, then kb and
        // kb + 1 fill word wa + 1; its both halves when even, then kb + 1 is the
        // low half of word wa + 1.
        const int wo = kb - 1 - e0;
        const int wa = wo >> 1;
        const uint32_t mask_a = (wo & 1) ? 0xFFFF0000u : 0xFFFFFFFFu;
        const uint32_t mask_b = (wo & 1) ? 0xFFFFFFFFu : 0x0000FFFFu;
        uint32_t sec2 = 0xFFFFFFFFu;
#pragma unroll
        for (int k = 0; k < K; ++k) {
          const uint32_t m = (k == wa ? mask_a : 0u) | (k == wa + 1 ? mask_b : 0u);
          sec2 = r3dsimt::vmin2(sec2, sv[k] | m);
        }
        const uint32_t sec = group_umin<G>(r3dsimt::umin(sec2 & 0xFFFFu, sec2 >> 16));
        const int km = kb > 0 ? kb - 1 : 0, kp = kb + 1 < nd ? kb + 1 : nd - 1;
        const int base_lane = gi * G;
        uint32_t vm = pick<K>(s, (km % (2 * K)) >> 1);
        uint32_t vp = pick<K>(s, (kp % (2 * K)) >> 1);
        vm = r3dsimt::shfl(vm, (base_lane + km / (2 * K)) & 31);
        vp = r3dsimt::shfl(vp, (base_lane + kp / (2 * K)) & 31);
        const uint32_t sm = (km & 1) ? (vm >> 16) : (vm & 0xFFFFu);
        const uint32_t sp = (kp & 1) ? (vp >> 16) : (vp & 0xFFFFu);
        if (on) {
          if (t == 0)
            info[px_out] = make_int4(static_cast<int>(static_cast<uint32_t>(kb) | (bcost << 16)),
                                     static_cast<int>(sec | (sm << 16)), static_cast<int>(sp), 0);
          if (job.volume != nullptr) {
            uint16_t* vb = job.volume + (static_cast<int64_t>(y) * w + x) * nd + e0;
#pragma unroll
            for (int u = 0; u < U; ++u)
              if (uvalid[u])
                *reinterpret_cast<uint4*>(vb + 8 * u) = make_uint4(s[4 * u], s[4 * u + 1], s[4 * u + 2], s[4 * u + 3]);
          }
          if (m.diagonal_lr) {
            // Right-view WTA along the diagonal (sgm_kernels.cpp:349-356): the
            // smallest (S, x) key per right column.
            const RowInterval lv = m.bv[job.y0 + y];
            const int bx = job.x0 + x;
            if (bx >= lv.first && bx <= lv.last) {
              uint32_t* keys = rkeys + job.rk_off + static_cast<int64_t>(y) * (w + nd);
              const int b0 = x + nd - 1;
#pragma unroll
              for (int k = 0; k < K; ++k) {
                if (uvalid[k / 4]) {
                  const int e = e0 + 2 * k;
                  atomicMin(keys + (b0 - e), ((s[k] & 0xFFFFu) << 16) | static_cast<uint32_t>(x));
                  atomicMin(keys + (b0 - e - 1), (s[k] & 0xFFFF0000u) | static_cast<uint32_t>(x));
                }
              }
            }
          }
        }
      }
      (void)s;
#pragma unroll
      for (int k = 0; k < K; ++k) prev[k] = out[k];
      if constexpr (MODE == kFirst || MODE == kAccumulate) s_out += dcell;
      if constexpr (MODE == kTerm) t_out += dcell;
      if constexpr (kWta) {
        px_out += dpx;
        x += dx;
        y += dy;
      }
    };
    for (int i0 = 0; i0 < maxlen; i0 += NS) {
#pragma unroll
      for (int q = 0; q < NS; ++q)
        if (i0 + q < maxlen) step(i0 + q, q);
    }
    r3dsimt::cp_async_wait<0>();
  }
}

// ---------------------------------------------------------------- acceptance
// stereo_matcher.cpp:474-523 with lo = 0, num = nd for every pixel.
R3D_GLOBAL void R3D_LAUNCH_BOUNDS(kPathThreads)
    sgm_path_accept_kernel(const SgmMatch* R3D_RESTRICT matches, const SgmPathJob* R3D_RESTRICT jobs, int njobs,
                           int64_t pixels, const int4* R3D_RESTRICT info, const uint32_t* R3D_RESTRICT rkeys) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < pixels; i += stride) {
    const int j = find_job(jobs, njobs, i, [](const SgmPathJob& q) { return q.px_off; });
    const SgmPathJob& job = jobs[j];
    const SgmMatch& m = matches[job.match];
    const int nd = m.nd, w = job.w;
    const int p = static_cast<int>(i - job.px_off);
    const int y = p / w, x = p - (p / w) * w;
    const int bx = job.x0 + x, by = job.y0 + y;
    const RowInterval lv = m.bv[by];
    float d = kInfF, cf = 0.0F;
    if (bx >= lv.first && bx <= lv.last) {
      const int4 in = info[i];
      const int best = in.x & 0xFFFF;
      const uint32_t bcost = static_cast<uint32_t>(in.x) >> 16;
      const uint32_t sec = static_cast<uint32_t>(in.y) & 0xFFFFu;
      const uint32_t sm = static_cast<uint32_t>(in.y) >> 16;
      const uint32_t sp = static_cast<uint32_t>(in.z);
      const RowInterval rv = m.pv[by];
      const int xr = bx - m.dmin - best;
      bool ok = xr >= rv.first && xr <= rv.last;
      if (ok && m.diagonal_lr) {
        const uint32_t key = rkeys[job.rk_off + static_cast<int64_t>(y) * (w + nd) + (x - best + nd - 1)];
        const int rb = key == 0xFFFFFFFFu ? 0xFFFF : static_cast<int>(key & 0xFFFFu) - x + best;
        const int diff = rb - best;
        if ((diff < 0 ? -diff : diff) > m.lr_max_diff) ok = false;
      }
      const float best_cost = static_cast<float>(bcost);
      if (ok && m.uniqueness > 0.0F && sec != 0xFFFFu &&
          best_cost > __fmul_rn(__fsub_rn(1.0F, m.uniqueness), static_cast<float>(sec)))
        ok = false;
      if (ok) {
        float delta = 0.0F;
        if (best > 0 && best < nd - 1)
          delta = sgm_simd::subpixel_delta(m.subpixel, static_cast<float>(sm), best_cost, static_cast<float>(sp));
        d = __fadd_rn(static_cast<float>(m.dmin + best), delta);
        if (m.confidence)
          cf = (sec != 0xFFFFu && sec > 0u) ? __fsub_rn(1.0F, __fdiv_rn(best_cost, static_cast<float>(sec))) : 0.0F;
      }
    }
    job.disp[p] = d;
    if (job.conf != nullptr) job.conf[p] = cf;
    if (p == 0) *job.cells = static_cast<unsigned long long>(w) * static_cast<unsigned long long>(job.h) * nd;
  }
}

// ================================================================ ranged tiles
// Per-pixel label ranges (lo, num; num a multiple of 16): the same passes on
// costs and sums packed per tile (pixel after pixel, num labels each).

// Per wave row: the in-row exclusive prefix of num (the pixel's cell offset
// before its row start is added), the range and the base intensity of every
// pixel as one 16-byte record {offset, lo | num << 16, intensity, 0}; the
// row's label total and its right-WTA shift max(lo + num - 1 - x).
R3D_GLOBAL void R3D_LAUNCH_BOUNDS(kPathThreads)
    sgm_path_ranged_rows_kernel(const SgmMatch* R3D_RESTRICT matches, const SgmPathJob* R3D_RESTRICT jobs, int njobs,
                                int64_t rows, int4* R3D_RESTRICT rec, int* R3D_RESTRICT rowsum,
                                int* R3D_RESTRICT rowshift) {
  const int lane = static_cast<int>(threadIdx.x & 31u);
  const int wpb = static_cast<int>(blockDim.x) >> 5;
  const int64_t nwarps = static_cast<int64_t>(gridDim.x) * wpb;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * wpb + (threadIdx.x >> 5); r < rows; r += nwarps) {
    const int j = find_job(jobs, njobs, r, [](const SgmPathJob& q) { return q.row_off; });
    const SgmPathJob& job = jobs[j];
    const SgmMatch& m = matches[job.match];
    const int y = static_cast<int>(r - job.row_off), by = job.y0 + y, w = job.w;
    int run = 0, shift = -0x7FFFFFFF;
    for (int xb = 0; xb < w; xb += 32) {
      const int x = xb + lane;
      int lo = 0, num = 0, iv = 0;
      if (x < w) {
        const int64_t ri = static_cast<int64_t>(by) * m.r_stride + job.x0 + x;
        lo = m.rlo[ri];
        num = m.rnum[ri];
        iv = m.base[static_cast<int64_t>(by) * m.base_stride + job.x0 + x];
        shift = r3dsimt::imax(shift, lo + num - 1 - x);
      }
      int incl = num;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = static_cast<int>(r3dsimt::shfl(static_cast<uint32_t>(incl), lane >= o ? lane - o : lane));
        if (lane >= o) incl += v;
      }
      if (x < w)
        rec[job.px_off + static_cast<int64_t>(y) * w + x] =
            make_int4(run + incl - num, lo | (num << 16), iv, 0);
      run += static_cast<int>(r3dsimt::shfl(static_cast<uint32_t>(incl), 31));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
      shift = r3dsimt::imax(shift, static_cast<int>(r3dsimt::shfl_xor(static_cast<uint32_t>(shift), o)));
    if (lane == 0) {
      rowsum[r] = run;
      rowshift[r] = shift;
    }
  }
}

// Per tile: exclusive prefix of the row totals (the cell offset of each row).
R3D_GLOBAL void R3D_LAUNCH_BOUNDS(kPathThreads)
    sgm_path_ranged_rowstart_kernel(const SgmPathJob* R3D_RESTRICT jobs, int njobs, const int* R3D_RESTRICT rowsum,
                                    int* R3D_RESTRICT rowstart) {
  const int lane = static_cast<int>(threadIdx.x & 31u);
  const int wpb = static_cast<int>(blockDim.x) >> 5;
  for (int j = static_cast<int>(blockIdx.x) * wpb + static_cast<int>(threadIdx.x >> 5); j < njobs;
       j += static_cast<int>(gridDim.x) * wpb) {
    const SgmPathJob& job = jobs[j];
    int carry = 0;
    for (int yb = 0; yb < job.h; yb += 32) {
      const int y = yb + lane;
      const int v = y < job.h ? rowsum[job.row_off + y] : 0;
      int incl = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int u = static_cast<int>(r3dsimt::shfl(static_cast<uint32_t>(incl), lane >= o ? lane - o : lane));
        if (lane >= o) incl += u;
      }
      if (y < job.h) rowstart[job.row_off + y] = carry + incl - v;
      carry += static_cast<int>(r3dsimt::shfl(static_cast<uint32_t>(incl), 31));
    }
    if (lane == 0) *job.cells = static_cast<unsigned long long>(carry);
  }
}

// Per pixel: the final cell offset (row start added) and the u8 costs of its
// num labels, C(p, lo + j) of stereo_matcher.cpp:305-353.
R3D_GLOBAL void R3D_LAUNCH_BOUNDS(kPathThreads)
    sgm_path_ranged_cost_kernel(const SgmMatch* R3D_RESTRICT matches, const SgmPathJob* R3D_RESTRICT jobs, int njobs,
                                int64_t pixels, int4* R3D_RESTRICT rec, const int* R3D_RESTRICT rowstart,
                                uint8_t* R3D_RESTRICT cost) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < pixels; i += stride) {
    const int j = find_job(jobs, njobs, i, [](const SgmPathJob& q) { return q.px_off; });
    const SgmPathJob& job = jobs[j];
    const SgmMatch& m = matches[job.match];
    const int p = static_cast<int>(i - job.px_off);
    const int y = p / job.w, x = p - y * job.w;
    int4 rc = rec[i];
    rc.x += rowstart[job.row_off + y];
    rec[i] = rc;
    const int lo = rc.y & 0xFFFF, num = static_cast<int>(static_cast<uint32_t>(rc.y) >> 16);
    const int bx = job.x0 + x, by = job.y0 + y;
    const RowInterval lv = m.bv[by], rv = m.pv[by];
    const bool inside = bx >= lv.first && bx <= lv.last;
    const uint64_t cl = inside ? m.cbase[static_cast<int64_t>(by) * m.cb_stride + bx] : 0;
    const uint64_t* crow = m.cpart + static_cast<int64_t>(by) * m.cp_stride;
    const int safe = rv.first > 0 ? rv.first : 0;
    const uint32_t inv = static_cast<uint32_t>(m.invalid_cost);
    uint8_t* out = cost + job.cell_off + rc.x;
    for (int c = 0; c < num; c += 16) {
      uint32_t q[4] = {0, 0, 0, 0};
      if (inside) {
        const int xr0 = bx - m.dmin - lo - c;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          const int xr = xr0 - k;
          const bool ok = xr >= rv.first && xr <= rv.last;
          const uint64_t cr = crow[ok ? xr : safe];
          const uint32_t v = ok ? static_cast<uint32_t>(r3dsimt::popc64(cl ^ cr)) : inv;
          q[k >> 2] |= v << (8 * (k & 3));
        }
      }
      *reinterpret_cast<uint4*>(out + c) = make_uint4(q[0], q[1], q[2], q[3]);
    }
  }
}

// Labels of a chain's predecessor vector kept in shared memory (u32 words of
// two labels); wider vectors continue in the chain's global overflow. A
// buffer holds a sentinel word before the vector (index -1) and one after it
// (index nw, written with the vector), so that a vector of at most
// kRangedSmemWords words is read at a clamped index without bounds checks.
// The buffers of a warp's chains are kRangedSmemStride words apart (odd, so
// that the chains of a warp start in different banks).
constexpr int kRangedSmemWords = 32;
// Ranged pass CTAs have 4 warps: about 15 KB of shared memory per warp
// (ring, records, predecessor buffers), so that three CTAs fit an SM.
constexpr int kRangedThreads = 128;
constexpr int kRangedSmemStride = kRangedSmemWords + 3;

// Ring of the ranged passes: D stages of chunk 0's bytes (kPlanes bytes per
// label: cost, plus the u16 sum or the seven byte terms) and 2 D record slots.
template <int G, int K, int MODE>
struct RangedRing {
  static constexpr int CH = 2 * G * K;  // labels per chunk
  static constexpr int CPW = 32 / G;
  // Two stages for the passes that stage several planes (the accumulate
  // pass: cost and sum; the byte-term last pass: eight planes), four for
  // the one-plane passes: less shared memory per warp, more warps per SM.
  static constexpr int D = MODE == kLastTerm || MODE == kAccumulate ? 2 : kPathStages;
  static constexpr int kPlanes = MODE == kAccumulate ? 3 : (MODE == kLastTerm ? 1 + kTermArrays : 1);
  static constexpr int kDataStage = CPW * kPlanes * CH;
  static constexpr int kData = D * kDataStage;
  static constexpr int kRec = 2 * D * 32 * 16;  // one record slot per lane and stage
  static constexpr int kPrev = CPW * 2 * kRangedSmemStride * 4;
  static constexpr int kLut = 512;  // the warp's copy of its match's P2 table
  static constexpr int kWarpBytes = kData + kRec + kPrev + kLut;
  static constexpr int kBlockBytes = (kRangedThreads / 32) * kWarpBytes;
};

template <int G, int K, int MODE>
R3D_GLOBAL void R3D_LAUNCH_BOUNDS(kRangedThreads)
    sgm_path_ranged_kernel(const SgmMatch* R3D_RESTRICT matches, const SgmPathJob* R3D_RESTRICT jobs, int njobs,
                           const PassSet ps, const int4* R3D_RESTRICT rec, const uint8_t* R3D_RESTRICT cost,
                           uint16_t* sum, uint8_t* terms, int64_t tstride, uint32_t* ovf, int64_t ovf_words,
                           const int* cancel) {
  // Modes: kFirst / kAccumulate write or add u16 sums; kTerm writes the
  // pass's byte terms; kLastTerm writes S = L_8 + 7 C + sum of the seven
  // terms as the u16 sum (read by the per-pixel winner-takes-all).
  using R = RangedRing<G, K, MODE>;
  constexpr int CPW = R::CPW, U = K / 4, CH = R::CH, D = R::D;
  constexpr bool kReadsSum = MODE == kAccumulate;
  R3D_DYNAMIC_SMEM(smem);
  const int lane = static_cast<int>(threadIdx.x & 31u), warp = static_cast<int>(threadIdx.x >> 5);
  const int gi = lane / G, t = lane % G;
  const int e0 = 2 * t * K;  // first label of the lane within a chunk
  const int wpb = static_cast<int>(blockDim.x) >> 5;
  const int64_t nwarps = static_cast<int64_t>(gridDim.x) * wpb;
  unsigned char* wb = smem + static_cast<size_t>(warp) * R::kWarpBytes;
  int4* recs = reinterpret_cast<int4*>(wb + R::kData);
  // Buffer b of this lane's chain: words (b * CPW + gi) * kRangedSmemStride onwards.
  uint32_t* prevw = reinterpret_cast<uint32_t*>(wb + R::kData + R::kRec) + gi * kRangedSmemStride;
  uint16_t* const lut = reinterpret_cast<uint16_t*>(wb + R::kData + R::kRec + R::kPrev);
  int lut_match = -1;
  uint32_t* ovfc = ovf + (static_cast<int64_t>(blockIdx.x) * wpb * CPW + warp * CPW + gi) * 2 * ovf_words;
  auto stage_cost = [&](int st) -> unsigned char* { return wb + st * R::kDataStage + gi * CH + e0; };
  auto stage_sum = [&](int st) -> unsigned char* {
    return wb + st * R::kDataStage + CPW * CH + gi * 2 * CH + 2 * e0;
  };
  auto stage_term = [&](int st, int r) -> unsigned char* {
    return wb + st * R::kDataStage + (1 + r) * CPW * CH + gi * CH + e0;
  };
  // Word idx (labels 2 idx, 2 idx + 1) of buffer b of the predecessor vector
  // (nw words long): two sentinels outside it.
  // The shared-memory word is read unconditionally (at a wrapped, in-bounds
  // index); only the rare words of wide vectors go to the overflow.
  auto qword = [&](int b, int idx, int nw) -> uint32_t {
    const uint32_t* vec = prevw + b * CPW * kRangedSmemStride + 1;
    if (nw <= kRangedSmemWords) return vec[r3dsimt::imax(r3dsimt::imin(idx, nw), -1)];
    uint32_t v = vec[idx & (kRangedSmemWords - 1)];
    if (idx >= kRangedSmemWords && idx < nw) v = ovfc[b * ovf_words + (idx - kRangedSmemWords)];
    return (idx < 0 || idx >= nw) ? kSent2 : v;
  };
  auto put_word = [&](int b, int idx, uint32_t v) {
    if (idx < kRangedSmemWords) prevw[b * CPW * kRangedSmemStride + 1 + idx] = v;
    else ovfc[b * ovf_words + (idx - kRangedSmemWords)] = v;
  };
  const int64_t total_blocks = ps.start[ps.n];
  const uint32_t one = ps.one;
  for (int64_t gblk = static_cast<int64_t>(blockIdx.x) * wpb + warp; gblk < total_blocks; gblk += nwarps) {
    if (cancelled(cancel)) break;
    // The pass of the block (static indices only: no local copy of ps).
    int cls = ps.cls[0], dx = ps.dx[0], dy = ps.dy[0], tslot = ps.slot[0];
    int64_t blk = gblk;
#pragma unroll
    for (int q = 1; q < kTermArrays; ++q) {
      if (q < ps.n && gblk >= ps.start[q]) {
        cls = ps.cls[q];
        dx = ps.dx[q];
        dy = ps.dy[q];
        tslot = ps.slot[q];
        blk = gblk - ps.start[q];
      }
    }
    const int j = find_job(jobs, njobs, blk, [cls](const SgmPathJob& q) { return q.blk[cls]; });
    const SgmPathJob& job = jobs[j];
    const SgmMatch& m = matches[job.match];
    if (job.match != lut_match) {  // the same for the whole warp (one chain block)
      r3dsimt::syncwarp();
      for (int k = lane; k < 128; k += 32)
        reinterpret_cast<uint32_t*>(lut)[k] = reinterpret_cast<const uint32_t*>(m.lut)[k];
      r3dsimt::syncwarp();
      lut_match = job.match;
    }
    const int w = job.w;
    const uint32_t p1x2 = static_cast<uint32_t>(m.p1) * 0x10001u;
    const bool no_carry = m.sum_no_carry != 0;
    int sx, sy, len;
    chain_geometry(cls, dx, dy, w, job.h, (blk - job.blk[cls]) * CPW + gi, sx, sy, len);
    int maxlen = len;
#pragma unroll
    for (int o = G; o < 32; o <<= 1) maxlen = r3dsimt::imax(maxlen, static_cast<int>(r3dsimt::shfl_xor(maxlen, o)));
    const uint8_t* cbase = cost + job.cell_off;
    uint16_t* sbase = sum + job.cell_off;
    uint8_t* tbase = terms + job.cell_off;
    const int4* rbase = rec + job.px_off;
    auto pix = [&](int i) -> int { return (sy + i * dy) * w + sx + i * dx; };
    auto issue_rec = [&](int i) {
      if (i < len) r3dsimt::cp_async16(&recs[(i & (2 * D - 1)) * 32 + lane], rbase + pix(i));
    };
    auto issue_data = [&](int i, int4 r) {
      if (i >= len) return;
      const int off = r.x, num = static_cast<int>(static_cast<uint32_t>(r.y) >> 16);
      const int st = i & (D - 1);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (e0 + 8 * u < num) {
          r3dsimt::cp_async8(stage_cost(st) + 8 * u, cbase + off + e0 + 8 * u);
          if constexpr (kReadsSum) r3dsimt::cp_async16(stage_sum(st) + 16 * u, sbase + off + e0 + 8 * u);
          if constexpr (MODE == kLastTerm) {
#pragma unroll
            for (int r = 0; r < kTermArrays; ++r)
              r3dsimt::cp_async8(stage_term(st, r) + 8 * u, tbase + r * tstride + off + e0 + 8 * u);
          }
        }
      }
    };
    // The leading sentinels of both buffers (read from the second pixel on,
    // after the first step's warp barrier).
    if (t == 0) {
      prevw[0] = kSent2;
      prevw[CPW * kRangedSmemStride] = kSent2;
    }
    // Records of the first 2 D - 1 pixels now, the first D - 1 pixels' data in flight.
#pragma unroll
    for (int k = 0; k < 2 * D - 1; ++k)
      if (k < len) recs[k * 32 + lane] = rbase[pix(k)];
#pragma unroll
    for (int k = 0; k < D - 1; ++k) {
      issue_data(k, recs[k * 32 + lane]);
      r3dsimt::cp_async_commit();
    }
    uint32_t pmin = 0, lutv = 0;
    int lo_q = 0, num_q = 0;
    for (int i = 0; i < maxlen; ++i) {
      const bool on = i < len;
      // One wait per step: the group of step i - D + 1 (this pixel's data)
      // and the older one holding record i + D - 1 are complete when at most
      // the D - 2 most recent groups are still in flight. The slots refilled
      // here (record and data of the previous pixel) are no longer read.
      r3dsimt::cp_async_wait<D - 2>();
      const int4 rc = recs[(i & (2 * D - 1)) * 32 + lane];
      const int4 rn = recs[((i + D - 1) & (2 * D - 1)) * 32 + lane];
      issue_rec(i + 2 * D - 1);
      issue_data(i + D - 1, rn);
      r3dsimt::cp_async_commit();
      const int off = rc.x, lo = rc.y & 0xFFFF, icur = rc.z;
      const int num = on ? static_cast<int>(static_cast<uint32_t>(rc.y) >> 16) : 0;
      // Chunks of this pixel's range: the same for the chain's G lanes (one
      // pixel), and the chunk loop holds no warp-wide operation.
      const int nchw = (num + CH - 1) / CH;
      const int sh = lo - lo_q, nwq = num_q >> 1;
      const int cur = i & 1, prv = cur ^ 1;
      uint32_t pen2 = 0, negmp = 0;
      if (i > 0) {
        const uint32_t pen = pmin + lutv;
        pen2 = pen | (pen << 16);
        negmp = 0u - (pmin | (pmin << 16));
      }
      {
        // The next step's P2, loaded one step ahead from the next pixel's
        // record (landed: it was issued 2 D - 1 steps ahead). Past the end of
        // the chain that record slot holds an older or an unwritten record,
        // so the table index is clamped to the table.
        const int dn = recs[((i + 1) & (2 * D - 1)) * 32 + lane].z - icur;
        const uint32_t di = static_cast<uint32_t>(dn < 0 ? -dn : dn) >> 8;
        lutv = lut[di < 255u ? di : 255u];
      }
      uint32_t pm = kSent2;
      for (int c = 0; c < nchw; ++c) {
        const int j0 = c * CH + e0;
        bool uv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) uv[u] = j0 + 8 * u < num;
        uint2 craw[U];
        uint4 sraw[U];
        uint32_t tsum[K];  // kLastTerm: sum of the seven byte terms per label pair
#pragma unroll
        for (int k = 0; k < K; ++k) tsum[k] = 0;
#pragma unroll
        for (int u = 0; u < U; ++u) {
          craw[u] = make_uint2(0, 0);
          sraw[u] = make_uint4(0, 0, 0, 0);
          if (uv[u]) {
            if (c == 0) {
              const int st = i & (D - 1);
              craw[u] = *reinterpret_cast<const uint2*>(stage_cost(st) + 8 * u);
              if constexpr (kReadsSum) sraw[u] = *reinterpret_cast<const uint4*>(stage_sum(st) + 16 * u);
            } else {
              craw[u] = *reinterpret_cast<const uint2*>(cbase + off + j0 + 8 * u);
              if constexpr (kReadsSum)
                sraw[u] = r3dsimt::ld_stream(reinterpret_cast<const uint4*>(sbase + off + j0 + 8 * u));
            }
            if constexpr (MODE == kLastTerm) {
#pragma unroll
              for (int r = 0; r < kTermArrays; ++r) {
                const uint2 tw = c == 0 ? *reinterpret_cast<const uint2*>(stage_term(i & (D - 1), r) + 8 * u)
                                        : *reinterpret_cast<const uint2*>(tbase + r * tstride + off + j0 + 8 * u);
                tsum[4 * u + 0] = fma_add(r3dsimt::perm(tw.x, 0u, 0x4140u), one, tsum[4 * u + 0]);
                tsum[4 * u + 1] = fma_add(r3dsimt::perm(tw.x, 0u, 0x4342u), one, tsum[4 * u + 1]);
                tsum[4 * u + 2] = fma_add(r3dsimt::perm(tw.y, 0u, 0x4140u), one, tsum[4 * u + 2]);
                tsum[4 * u + 3] = fma_add(r3dsimt::perm(tw.y, 0u, 0x4342u), one, tsum[4 * u + 3]);
              }
            }
          }
        }
        uint32_t c2[K];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          c2[4 * u + 0] = r3dsimt::perm(craw[u].x, 0u, 0x4140u);
          c2[4 * u + 1] = r3dsimt::perm(craw[u].x, 0u, 0x4342u);
          c2[4 * u + 2] = r3dsimt::perm(craw[u].y, 0u, 0x4140u);
          c2[4 * u + 3] = r3dsimt::perm(craw[u].y, 0u, 0x4342u);
        }
        uint32_t out[K], tr[K];
        if (i == 0) {
#pragma unroll
          for (int k = 0; k < K; ++k) {
            tr[k] = 0;
            out[k] = c2[k];
          }
        } else {
          // Predecessor labels j0 + sh - 2 .. j0 + sh + 2 K + 1 (its own
          // indexing), sentinels outside its range, realigned by one label
          // when the shift is odd.
          const int b = j0 + sh - 2;
          const int f = b >> 1;
          uint32_t qw[K + 3];
#pragma unroll
          for (int k = 0; k < K + 3; ++k) qw[k] = qword(prv, f + k, nwq);
          uint32_t wv[K + 2];
          if (b & 1) {
#pragma unroll
            for (int k = 0; k < K + 2; ++k) wv[k] = r3dsimt::perm(qw[k], qw[k + 1], 0x5432u);
          } else {
#pragma unroll
            for (int k = 0; k < K + 2; ++k) wv[k] = qw[k];
          }
          uint32_t mprev = r3dsimt::perm(wv[0], wv[1], 0x5432u);
#pragma unroll
          for (int k = 0; k < K; ++k) {
            const uint32_t mnext = r3dsimt::perm(wv[k + 1], wv[k + 2], 0x5432u);
            const uint32_t nb = r3dsimt::vmin2(mprev, mnext);
            const uint32_t best = r3dsimt::vmin2(wv[k + 1], r3dsimt::vaddmin2(nb, p1x2, pen2));
            tr[k] = fma_add(best, one, negmp);
            out[k] = fma_add(tr[k], one, c2[k]);
            mprev = mnext;
          }
        }
#pragma unroll
        for (int k = 0; k < K; ++k) {
          if (!uv[k / 4]) out[k] = kSent2;
          pm = r3dsimt::vmin2(pm, out[k]);
          if (uv[k / 4]) put_word(cur, (j0 >> 1) + k, out[k]);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (!uv[u]) continue;
          if constexpr (MODE == kTerm) {
            r3dsimt::st_stream8(reinterpret_cast<uint2*>(tbase + tslot * tstride + off + j0 + 8 * u),
                                make_uint2(r3dsimt::perm(tr[4 * u], tr[4 * u + 1], 0x6420u),
                                           r3dsimt::perm(tr[4 * u + 2], tr[4 * u + 3], 0x6420u)));
            continue;
          }
          uint4 v;
          if constexpr (MODE == kFirst) {
            v = make_uint4(out[4 * u], out[4 * u + 1], out[4 * u + 2], out[4 * u + 3]);
          } else if constexpr (MODE == kLastTerm) {
            v = make_uint4(out[4 * u] + 7u * c2[4 * u] + tsum[4 * u],
                           out[4 * u + 1] + 7u * c2[4 * u + 1] + tsum[4 * u + 1],
                           out[4 * u + 2] + 7u * c2[4 * u + 2] + tsum[4 * u + 2],
                           out[4 * u + 3] + 7u * c2[4 * u + 3] + tsum[4 * u + 3]);
          } else {
            v = make_uint4(add2(sraw[u].x, out[4 * u], no_carry), add2(sraw[u].y, out[4 * u + 1], no_carry),
                           add2(sraw[u].z, out[4 * u + 2], no_carry), add2(sraw[u].w, out[4 * u + 3], no_carry));
          }
          r3dsimt::st_stream(reinterpret_cast<uint4*>(sbase + off + j0 + 8 * u), v);
        }
      }
      pmin = group_umin<G>(r3dsimt::umin(pm & 0xFFFFu, pm >> 16));
      // The trailing sentinel of the vector just written.
      if (t == 0 && (num >> 1) <= kRangedSmemWords) prevw[cur * CPW * kRangedSmemStride + 1 + (num >> 1)] = kSent2;
      r3dsimt::syncwarp();
      if (on) {
        lo_q = lo;
        num_q = num;
      }
    }
    r3dsimt::cp_async_wait<0>();
    r3dsimt::syncwarp();
  }
}

// Per pixel: winner-takes-all over the total sums (sgm_kernels.cpp:332-358;
// first minimum, second best outside +-1, S at kb -+ 1 within the range),
// the optional volume copy and the right-view keys of the diagonal check.
R3D_GLOBAL void R3D_LAUNCH_BOUNDS(kPathThreads)
    sgm_path_ranged_wta_kernel(const SgmMatch* R3D_RESTRICT matches, const SgmPathJob* R3D_RESTRICT jobs, int njobs,
                               int64_t pixels, const int4* R3D_RESTRICT rec, const uint16_t* R3D_RESTRICT sum,
                               const int* R3D_RESTRICT rowshift, int4* R3D_RESTRICT info, uint32_t* rkeys) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < pixels; i += stride) {
    const int j = find_job(jobs, njobs, i, [](const SgmPathJob& q) { return q.px_off; });
    const SgmPathJob& job = jobs[j];
    const SgmMatch& m = matches[job.match];
    const int p = static_cast<int>(i - job.px_off);
    const int y = p / job.w, x = p - y * job.w;
    const int4 rc = rec[i];
    const int lo = rc.y & 0xFFFF, num = static_cast<int>(static_cast<uint32_t>(rc.y) >> 16);
    const uint16_t* sp16 = sum + job.cell_off + rc.x;
    uint32_t kmin = 0xFFFFFFFFu;
    for (int c = 0; c < num; c += 8) {
      const uint4 v = *reinterpret_cast<const uint4*>(sp16 + c);
      const uint32_t wv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const uint32_t e = static_cast<uint32_t>(c + 2 * k);
        kmin = r3dsimt::umin(kmin, r3dsimt::umin(((wv[k] & 0xFFFFu) << 16) | e, (wv[k] & 0xFFFF0000u) | (e + 1)));
      }
      if (job.volume != nullptr) *reinterpret_cast<uint4*>(job.volume + rc.x + c) = v;
    }
    const int kb = static_cast<int>(kmin & 0xFFFFu);
    const uint32_t bcost = kmin >> 16;
    uint32_t sec = 0xFFFFu;
    for (int e = 0; e < num; ++e)
      if (e + 1 < kb || e > kb + 1) sec = r3dsimt::umin(sec, sp16[e]);
    const int km = kb > 0 ? kb - 1 : 0;
    const int kp = kb + 1 < num ? kb + 1 : (num > 0 ? num - 1 : 0);
    const uint32_t sm = sp16[km], spv = sp16[kp];
    info[i] = make_int4(static_cast<int>(static_cast<uint32_t>(lo + kb) | (bcost << 16)),
                        static_cast<int>(sec | (sm << 16)), static_cast<int>(spv), 0);
    if (m.diagonal_lr) {
      const RowInterval lv = m.bv[job.y0 + y];
      const int bx = job.x0 + x;
      if (bx >= lv.first && bx <= lv.last) {
        uint32_t* keys = rkeys + job.rk_off + static_cast<int64_t>(y) * (job.w + m.nd);
        const int base = x - lo + rowshift[job.row_off + y];
        for (int e = 0; e < num; ++e)
          atomicMin(keys + (base - e), (static_cast<uint32_t>(sp16[e]) << 16) | static_cast<uint32_t>(x));
      }
    }
  }
}

// Acceptance rules with per-pixel ranges (stereo_matcher.cpp:474-523): as
// the full-range kernel's, plus the rejection of a minimum on the edge of a
// reduced range (:501-503).
R3D_GLOBAL void R3D_LAUNCH_BOUNDS(kPathThreads)
    sgm_path_ranged_accept_kernel(const SgmMatch* R3D_RESTRICT matches, const SgmPathJob* R3D_RESTRICT jobs,
                                  int njobs, int64_t pixels, const int4* R3D_RESTRICT rec,
                                  const int4* R3D_RESTRICT info, const uint32_t* R3D_RESTRICT rkeys,
                                  const int* R3D_RESTRICT rowshift) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < pixels; i += stride) {
    const int j = find_job(jobs, njobs, i, [](const SgmPathJob& q) { return q.px_off; });
    const SgmPathJob& job = jobs[j];
    const SgmMatch& m = matches[job.match];
    const int w = job.w;
    const int p = static_cast<int>(i - job.px_off);
    const int y = p / w, x = p - y * w;
    const int bx = job.x0 + x, by = job.y0 + y;
    const RowInterval lv = m.bv[by];
    float d = kInfF, cf = 0.0F;
    if (bx >= lv.first && bx <= lv.last) {
      const int4 in = info[i];
      const int4 rc = rec[i];
      const int lo = rc.y & 0xFFFF, num = static_cast<int>(static_cast<uint32_t>(rc.y) >> 16);
      const int best = in.x & 0xFFFF;
      const uint32_t bcost = static_cast<uint32_t>(in.x) >> 16;
      const uint32_t sec = static_cast<uint32_t>(in.y) & 0xFFFFu;
      const uint32_t sm = static_cast<uint32_t>(in.y) >> 16;
      const uint32_t sp = static_cast<uint32_t>(in.z);
      const int jb = best - lo;
      const RowInterval rv = m.pv[by];
      const int xr = bx - m.dmin - best;
      bool ok = xr >= rv.first && xr <= rv.last;
      if ((jb == 0 && lo > 0) || (jb == num - 1 && lo + num < m.nd)) ok = false;
      if (ok && m.diagonal_lr) {
        const uint32_t key =
            rkeys[job.rk_off + static_cast<int64_t>(y) * (w + m.nd) + (x - best + rowshift[job.row_off + y])];
        const int rb = key == 0xFFFFFFFFu ? 0xFFFF : static_cast<int>(key & 0xFFFFu) - x + best;
        const int diff = rb - best;
        if ((diff < 0 ? -diff : diff) > m.lr_max_diff) ok = false;
      }
      const float best_cost = static_cast<float>(bcost);
      if (ok && m.uniqueness > 0.0F && sec != 0xFFFFu &&
          best_cost > __fmul_rn(__fsub_rn(1.0F, m.uniqueness), static_cast<float>(sec)))
        ok = false;
      if (ok) {
        float delta = 0.0F;
        if (jb > 0 && jb < num - 1)
          delta = sgm_simd::subpixel_delta(m.subpixel, static_cast<float>(sm), best_cost, static_cast<float>(sp));
        d = __fadd_rn(static_cast<float>(m.dmin + best), delta);
        if (m.confidence)
          cf = (sec != 0xFFFFu && sec > 0u) ? __fsub_rn(1.0F, __fdiv_rn(best_cost, static_cast<float>(sec))) : 0.0F;
      }
    }
    job.disp[p] = d;
    if (job.conf != nullptr) job.conf[p] = cf;
  }
}

// ---------------------------------------------------------------- launches
// Pass order: the first pass writes the sums, the last takes the WTA.
struct Pass {
  int cls, dx, dy;
};
constexpr Pass kPasses[8] = {{0, 1, 0},  {1, 0, 1},   {2, 1, 1},  {2, -1, 1},
                             {1, 0, -1}, {2, -1, -1}, {2, 1, -1}, {0, -1, 0}};

template <class Kernel>
int resident_grid(Kernel kernel, int sms, int64_t work_items, int per_block, size_t smem = 0,
                  int threads = kPathThreads) {
  int per_sm = 1;
  R3D_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
  const int64_t need = (work_items + per_block - 1) / per_block;
  const int64_t resident = static_cast<int64_t>(sms) * (per_sm > 0 ? per_sm : 1);
  return static_cast<int>(need < resident ? (need > 0 ? need : 1) : resident);
}

// Algorithmic HBM bytes of one pass over `cells` cells of `pixels` pixels:
// costs read, sums read (not by the first pass) and written (not by the
// full-range last pass, which writes the WTA records instead); byte terms:
// one written per cell by passes 1..7, seven read by the last pass.
uint64_t pass_bytes(int mode, bool ranged, const SgmPathSegment& g) {
  const uint64_t c = static_cast<uint64_t>(g.cells), px = static_cast<uint64_t>(g.pixels);
  if (mode == kFirst) return 3 * c;
  if (mode == kTerm) return 2 * c;
  if (mode == kLastTerm) return (1 + kTermArrays) * c + 16 * px;
  if (mode == kLast && !ranged) return 3 * c + 16 * px;
  return 5 * c;
}

template <int G, int K, int MODE, bool FULL = false>
void launch_pass(const PassSet& ps, const SgmMatch* dm, const SgmPathJob* jobs, int njobs, const uint8_t* cost,
                 uint16_t* sum, uint8_t* terms, int64_t tstride, int4* info, uint32_t* rkeys, const uint16_t* ints,
                 int sms, cudaStream_t s, const SgmPathSegment& seg, const int* cancel) {
  const cudaEvent_t ev0 = profile_on() ? profile_mark(s) : nullptr;
  auto* k = sgm_path_kernel<G, K, MODE, FULL>;
  constexpr size_t smem = PathRing<G, K, MODE>::kBlockBytes;
  static thread_local int configured[64] = {};
  int dev = 0;
  R3D_CUDA(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 64 && !configured[dev]) {
    R3D_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    configured[dev] = 1;
  }
  const int64_t nb = ps.start[ps.n];
  constexpr int threads = PathRing<G, K, MODE>::kThreads;
  R3D_LAUNCH(k, dim3(resident_grid(k, sms, nb, threads / 32, smem, threads)), dim3(threads), smem, s, dm, jobs, njobs,
             ps, cost, sum, terms, tstride, info, rkeys, ints, cancel);
  launched("sgm_path_kernel");
  if (ev0 != nullptr) {
    char shape[32];
    std::snprintf(shape, sizeof(shape), "%dx%d/mode%d", G, K, MODE);
    const uint64_t n = static_cast<uint64_t>(ps.n);
    profile_pass(ev0, profile_mark(s), "sgm_path_kernel", shape, n * static_cast<uint64_t>(seg.cells),
                 n * static_cast<uint64_t>(seg.pixels), n * pass_bytes(MODE, false, seg));
  }
}

// Passes q of kPasses in `qs` (count n) as one PassSet.
PassSet pass_set(const SgmPathSegment& g, const int* qs, int n) {
  PassSet ps{};
  ps.one = 1;
  int64_t start = 0;
  for (int i = 0; i < n; ++i) {
    const Pass& p = kPasses[qs[i]];
    ps.cls[ps.n] = p.cls;
    ps.dx[ps.n] = p.dx;
    ps.dy[ps.n] = p.dy;
    ps.slot[ps.n] = qs[i];
    ps.start[ps.n] = start;
    start += g.blocks[p.cls];
    ++ps.n;
  }
  ps.start[ps.n] = start;
  return ps;
}

template <int G, int K>
void launch_passes(const SgmMatch* dm, const SgmPathJob* jobs, const SgmPathSegment& g, const uint8_t* cost,
                   uint16_t* sum, uint8_t* terms, int64_t tstride, int4* info, uint32_t* rkeys, const uint16_t* ints,
                   int sms, cudaStream_t s, const int* cancel) {
  for (int q = 0; q < 8; ++q)
    if (g.blocks[kPasses[q].cls] <= 0) return;  // no pixels: every class has chains otherwise
  if (terms != nullptr) {
    // The seven term passes in one launch, then the last pass, which finds
    // all seven term arrays written.
    const int qs[kTermArrays] = {0, 1, 2, 3, 4, 5, 6};
    const int last = 7;
    // Segments whose matches fill every label unit take the kernels without
    // the per-unit validity selects.
    if (g.full != 0) {
      launch_pass<G, K, kTerm, true>(pass_set(g, qs, kTermArrays), dm, jobs, g.count, cost, sum, terms, tstride, info,
                                     rkeys, ints, sms, s, g, cancel);
      launch_pass<G, K, kLastTerm, true>(pass_set(g, &last, 1), dm, jobs, g.count, cost, sum, terms, tstride, info,
                                         rkeys, ints, sms, s, g, cancel);
    } else {
      launch_pass<G, K, kTerm>(pass_set(g, qs, kTermArrays), dm, jobs, g.count, cost, sum, terms, tstride, info,
                               rkeys, ints, sms, s, g, cancel);
      launch_pass<G, K, kLastTerm>(pass_set(g, &last, 1), dm, jobs, g.count, cost, sum, terms, tstride, info, rkeys,
                                   ints, sms, s, g, cancel);
    }
    return;
  }
  for (int q = 0; q < 8; ++q) {
    const PassSet ps = pass_set(g, &q, 1);
    if (q == 0)
      launch_pass<G, K, kFirst>(ps, dm, jobs, g.count, cost, sum, terms, tstride, info, rkeys, ints, sms, s, g,
                                cancel);
    else if (q < 7)
      launch_pass<G, K, kAccumulate>(ps, dm, jobs, g.count, cost, sum, terms, tstride, info, rkeys, ints, sms, s, g,
                                     cancel);
    else
      launch_pass<G, K, kLast>(ps, dm, jobs, g.count, cost, sum, terms, tstride, info, rkeys, ints, sms, s, g,
                               cancel);
  }
}

// Shapes compiled into the library (lanes per chain G, label pairs per lane K).
#define R3D_PATH_SHAPES(X) \
  X(1, 8)                  \
  X(2, 8)                  \
  X(2, 12)                 \
  X(2, 16)                 \
  X(4, 8)                  \
  X(4, 12)                 \
  X(4, 16)                 \
  X(8, 8)                  \
  X(8, 12)                 \
  X(8, 16)                 \
  X(16, 8)                 \
  X(16, 12)                \
  X(16, 16)                \
  X(32, 8)                 \
  X(32, 12)

}  // namespace

bool sgm_path_enabled() {
  const char* e = std::getenv("R3DGPU_FULL_KERNEL");
  return !(e != nullptr && std::strcmp(e, "wavefront") == 0);
}

namespace {
bool path_shape_compiled(int g, int k) {
  bool found = false;
#define R3D_SHAPE(gg, kk) found = found || (g == gg && k == kk);
  R3D_PATH_SHAPES(R3D_SHAPE)
#undef R3D_SHAPE
  return found;
}
}  // namespace

SgmPathShape sgm_path_shape(int nd) {
  // A compiled shape from R3DGPU_PATH_SHAPE ("G,K": any label count it
  // covers) or the tuning table (an entry for exactly this label count),
  // else the narrowest row of 8 or 12 label pairs per lane, ties to fewer
  // lanes per chain.
  if (const char* e = std::getenv("R3DGPU_PATH_SHAPE")) {
    int g = 0, k = 0;
    if (std::sscanf(e, "%d,%d", &g, &k) == 2 && path_shape_compiled(g, k) && 2 * g * k >= nd) return {g, k};
  }
  const auto it = tuning().path.find(nd);
  if (it != tuning().path.end() && path_shape_compiled(it->second.g, it->second.k) &&
      2 * it->second.g * it->second.k >= nd)
    return {it->second.g, it->second.k};
  SgmPathShape best{0, 0};
  int best_nd = 1 << 30;
#define R3D_SHAPE(g, k)                                       \
  if (k != 16 && 2 * g * k >= nd && 2 * g * k < best_nd) { \
    best = SgmPathShape{g, k};                                \
    best_nd = 2 * g * k;                                      \
  }
  R3D_PATH_SHAPES(R3D_SHAPE)
#undef R3D_SHAPE
  return best;
}

SgmPathBuffers sgm_path_buffers(int64_t cells, int64_t pixels, int64_t keys, bool terms) {
  SgmPathBuffers b{};
  size_t o = 0;
  b.cost = o;
  o += align256(static_cast<size_t>(cells));
  b.sum = o;
  b.term_stride = terms ? static_cast<int64_t>(align256(static_cast<size_t>(cells))) : 0;
  b.terms = b.sum;
  o += terms ? static_cast<size_t>(kTermArrays) * static_cast<size_t>(b.term_stride)
             : align256(static_cast<size_t>(cells) * 2);
  b.info = o;
  o += align256(static_cast<size_t>(pixels) * 16);
  b.rkeys = o;
  o += align256(static_cast<size_t>(keys) * 4);
  // The tiles' base intensities, pixel after pixel, and 16 bytes more: the
  // pass kernels copy the aligned 4-byte word holding a pixel's intensity.
  b.ints = o;
  o += align256(static_cast<size_t>(pixels) * 2 + 16);
  b.total = o;
  return b;
}

void launch_sgm_path_wave(const SgmMatch* dm, const SgmPathWave& wave, int sms, cudaStream_t s) {
  if (wave.njobs <= 0 || wave.cells <= 0) return;
  const SgmPathBuffers B = sgm_path_buffers(wave.cells, wave.pixels, wave.keys, wave.terms != 0);
  uint8_t* cost = wave.buffer + B.cost;
  uint16_t* sum = reinterpret_cast<uint16_t*>(wave.buffer + B.sum);
  uint8_t* terms = wave.terms != 0 ? wave.buffer + B.terms : nullptr;
  int4* info = reinterpret_cast<int4*>(wave.buffer + B.info);
  uint32_t* rkeys = reinterpret_cast<uint32_t*>(wave.buffer + B.rkeys);
  uint16_t* ints = reinterpret_cast<uint16_t*>(wave.buffer + B.ints);
  if (wave.keys > 0) R3D_CUDA(cudaMemsetAsync(rkeys, 0xFF, static_cast<size_t>(wave.keys) * 4, s));
  {
    constexpr size_t max_smem = static_cast<size_t>(kPathThreads / 32) * kCostStage * 8;
    static thread_local int configured[64] = {};
    int dev = 0;
    R3D_CUDA(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && !configured[dev]) {
      R3D_CUDA(cudaFuncSetAttribute(sgm_path_cost_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(max_smem)));
      configured[dev] = 1;
    }
    const int words = wave.max_span > 0 && wave.max_span <= kCostStage ? (wave.max_span + 1) & ~1 : kCostStage;
    const size_t smem = static_cast<size_t>(kPathThreads / 32) * words * 8;
    R3D_LAUNCH(sgm_path_cost_kernel,
               dim3(resident_grid(sgm_path_cost_kernel, sms, wave.rows, kPathThreads / 32, smem)),
               dim3(kPathThreads), smem, s, dm, wave.jobs, wave.njobs, wave.rows, cost, words, ints);
    launched("sgm_path_cost_kernel");
  }
  for (int q = 0; q < wave.nsegs; ++q) {
    const SgmPathSegment& g = wave.segs[q];
    const SgmPathJob* jobs = wave.jobs + g.first;
    bool done = false;
#define R3D_SHAPE(gg, kk)                                                                                     \
  if (!done && g.shape.g_ == gg && g.shape.k_ == kk) {                                                        \
    launch_passes<gg, kk>(dm, jobs, g, cost, sum, terms, B.term_stride, info, rkeys, ints, sms, s, wave.cancel); \
    done = true;                                                                                              \
  }
    R3D_PATH_SHAPES(R3D_SHAPE)
#undef R3D_SHAPE
    if (!done) fail(R3DGPU_EINVAL, "stereo: bad path kernel shape");
  }
  R3D_LAUNCH(sgm_path_accept_kernel, dim3(resident_grid(sgm_path_accept_kernel, sms, wave.pixels, kPathThreads)),
             dim3(kPathThreads), 0, s, dm, wave.jobs, wave.njobs, wave.pixels, info, rkeys);
  launched("sgm_path_accept_kernel");
}

// ---------------------------------------------------------------- ranged launches
namespace {

// Largest number of resident CTAs per SM any ranged pass kernel is launched
// with (the overflow has one slot per resident chain).
constexpr int kRangedMaxPerSm = 6;

template <int G, int K, int MODE>
void launch_ranged_pass(const PassSet& ps, const SgmMatch* dm, const SgmPathJob* jobs, int njobs, const int4* rec,
                        const uint8_t* cost, uint16_t* sum, uint8_t* terms, int64_t tstride, uint32_t* ovf,
                        int64_t ovf_words, int sms, cudaStream_t s, const SgmPathSegment& seg, const int* cancel) {
  const cudaEvent_t ev0 = profile_on() ? profile_mark(s) : nullptr;
  auto* k = sgm_path_ranged_kernel<G, K, MODE>;
  constexpr size_t smem = RangedRing<G, K, MODE>::kBlockBytes;
  static thread_local int configured[64] = {};
  int dev = 0;
  R3D_CUDA(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 64 && !configured[dev]) {
    R3D_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    configured[dev] = 1;
  }
  const int64_t nb = ps.start[ps.n];
  int grid = resident_grid(k, sms, nb, kRangedThreads / 32, smem, kRangedThreads);
  grid = grid < sms * kRangedMaxPerSm ? grid : sms * kRangedMaxPerSm;
  R3D_LAUNCH(k, dim3(grid), dim3(kRangedThreads), smem, s, dm, jobs, njobs, ps, rec, cost, sum, terms, tstride, ovf,
             ovf_words, cancel);
  launched("sgm_path_ranged_kernel");
  if (ev0 != nullptr) {
    char shape[32];
    std::snprintf(shape, sizeof(shape), "%dx%d/mode%d", G, K, MODE);
    // Per pixel and pass also the 16-byte record (range and cell offset).
    const uint64_t n = static_cast<uint64_t>(ps.n);
    const uint64_t alg = MODE == kLastTerm ? (1 + kTermArrays + 2) * static_cast<uint64_t>(seg.cells)
                                           : pass_bytes(MODE, true, seg);
    profile_pass(ev0, profile_mark(s), "sgm_path_ranged_kernel", shape, n * static_cast<uint64_t>(seg.cells),
                 n * static_cast<uint64_t>(seg.pixels), n * (alg + 16 * static_cast<uint64_t>(seg.pixels)));
  }
}

template <int G, int K>
void launch_ranged_passes(const SgmMatch* dm, const SgmPathJob* jobs, const SgmPathSegment& g, const int4* rec,
                          const uint8_t* cost, uint16_t* sum, uint8_t* terms, int64_t tstride, uint32_t* ovf,
                          int64_t ovf_words, int sms, cudaStream_t s, const int* cancel) {
  for (int q = 0; q < 8; ++q)
    if (g.blocks[kPasses[q].cls] <= 0) return;  // no pixels: every class has chains otherwise
  if (terms != nullptr) {
    // Byte terms: the seven term passes in one launch, then the last pass
    // (the total sum).
    const int qs[kTermArrays] = {0, 1, 2, 3, 4, 5, 6};
    const int last = 7;
    launch_ranged_pass<G, K, kTerm>(pass_set(g, qs, kTermArrays), dm, jobs, g.count, rec, cost, sum, terms, tstride,
                                    ovf, ovf_words, sms, s, g, cancel);
    launch_ranged_pass<G, K, kLastTerm>(pass_set(g, &last, 1), dm, jobs, g.count, rec, cost, sum, terms, tstride, ovf,
                                        ovf_words, sms, s, g, cancel);
    return;
  }
  for (int q = 0; q < 8; ++q) {
    const PassSet ps = pass_set(g, &q, 1);
    if (q == 0)
      launch_ranged_pass<G, K, kFirst>(ps, dm, jobs, g.count, rec, cost, sum, terms, tstride, ovf, ovf_words, sms, s,
                                       g, cancel);
    else
      launch_ranged_pass<G, K, kAccumulate>(ps, dm, jobs, g.count, rec, cost, sum, terms, tstride, ovf, ovf_words, sms,
                                            s, g, cancel);
  }
}

}  // namespace

bool sgm_path_ranged_enabled() {
  const char* e = std::getenv("R3DGPU_RANGED_KERNEL");
  return e == nullptr || std::strcmp(e, "path") == 0;
}

SgmPathShape sgm_path_ranged_shape(int over32, int64_t pixels) {
  // 32-label chunks unless more than a tenth of the tile's pixels need two.
  return static_cast<int64_t>(over32) * 10 > pixels ? SgmPathShape{4, 8} : SgmPathShape{2, 8};
}

SgmPathBuffers sgm_path_ranged_buffers(int64_t cells, int64_t pixels, int64_t keys, int64_t rows, int maxnum,
                                       int sms, bool terms) {
  SgmPathBuffers b = sgm_path_buffers(cells, pixels, keys, false);
  size_t o = b.total;
  // Byte terms of the ranged passes come in addition to the u16 sum (which
  // the last pass writes for the per-pixel winner-takes-all).
  b.terms = o;
  b.term_stride = terms ? static_cast<int64_t>(align256(static_cast<size_t>(cells))) : 0;
  o += static_cast<size_t>(kTermArrays) * static_cast<size_t>(b.term_stride);
  b.rec = o;
  o += align256(static_cast<size_t>(pixels) * 16);
  b.rowsum = o;
  o += align256(static_cast<size_t>(rows) * 4);
  b.rowstart = o;
  o += align256(static_cast<size_t>(rows) * 4);
  b.rowshift = o;
  o += align256(static_cast<size_t>(rows) * 4);
  b.overflow_words = maxnum > 2 * kRangedSmemWords ? (maxnum - 2 * kRangedSmemWords + 1) / 2 : 0;
  b.overflow = o;
  // One slot (two buffers) per resident chain: at most 16 chains per warp.
  const int64_t slots = static_cast<int64_t>(sms) * kRangedMaxPerSm * (kPathThreads / 32) * 16;
  o += align256(static_cast<size_t>(slots) * 2 * static_cast<size_t>(b.overflow_words) * 4);
  b.total = o;
  return b;
}

void launch_sgm_path_ranged_wave(const SgmMatch* dm, const SgmPathRangedWave& wave, int sms, cudaStream_t s) {
  if (wave.njobs <= 0 || wave.pixels <= 0) return;
  const SgmPathBuffers B =
      sgm_path_ranged_buffers(wave.cells, wave.pixels, wave.keys, wave.rows, wave.maxnum, sms, wave.terms != 0);
  uint8_t* cost = wave.buffer + B.cost;
  uint16_t* sum = reinterpret_cast<uint16_t*>(wave.buffer + B.sum);
  uint8_t* terms = wave.terms != 0 ? wave.buffer + B.terms : nullptr;
  int4* info = reinterpret_cast<int4*>(wave.buffer + B.info);
  uint32_t* rkeys = reinterpret_cast<uint32_t*>(wave.buffer + B.rkeys);
  int4* rec = reinterpret_cast<int4*>(wave.buffer + B.rec);
  int* rowsum = reinterpret_cast<int*>(wave.buffer + B.rowsum);
  int* rowstart = reinterpret_cast<int*>(wave.buffer + B.rowstart);
  int* rowshift = reinterpret_cast<int*>(wave.buffer + B.rowshift);
  uint32_t* ovf = reinterpret_cast<uint32_t*>(wave.buffer + B.overflow);
  if (wave.keys > 0) R3D_CUDA(cudaMemsetAsync(rkeys, 0xFF, static_cast<size_t>(wave.keys) * 4, s));
  R3D_LAUNCH(sgm_path_ranged_rows_kernel,
             dim3(resident_grid(sgm_path_ranged_rows_kernel, sms, wave.rows, kPathThreads / 32)), dim3(kPathThreads),
             0, s, dm, wave.jobs, wave.njobs, wave.rows, rec, rowsum, rowshift);
  launched("sgm_path_ranged_rows_kernel");
  R3D_LAUNCH(sgm_path_ranged_rowstart_kernel,
             dim3(resident_grid(sgm_path_ranged_rowstart_kernel, sms, wave.njobs, kPathThreads / 32)),
             dim3(kPathThreads), 0, s, wave.jobs, wave.njobs, rowsum, rowstart);
  launched("sgm_path_ranged_rowstart_kernel");
  R3D_LAUNCH(sgm_path_ranged_cost_kernel,
             dim3(resident_grid(sgm_path_ranged_cost_kernel, sms, wave.pixels, kPathThreads)), dim3(kPathThreads), 0,
             s, dm, wave.jobs, wave.njobs, wave.pixels, rec, rowstart, cost);
  launched("sgm_path_ranged_cost_kernel");
  for (int q = 0; q < wave.nsegs; ++q) {
    const SgmPathSegment& g = wave.segs[q];
    const SgmPathJob* jobs = wave.jobs + g.first;
    if (g.shape.g_ == 2 && g.shape.k_ == 8)
      launch_ranged_passes<2, 8>(dm, jobs, g, rec, cost, sum, terms, B.term_stride, ovf, B.overflow_words, sms, s,
                                 wave.cancel);
    else if (g.shape.g_ == 4 && g.shape.k_ == 8)
      launch_ranged_passes<4, 8>(dm, jobs, g, rec, cost, sum, terms, B.term_stride, ovf, B.overflow_words, sms, s,
                                 wave.cancel);
    else
      fail(R3DGPU_EINVAL, "stereo: bad ranged path kernel shape");
  }
  R3D_LAUNCH(sgm_path_ranged_wta_kernel,
             dim3(resident_grid(sgm_path_ranged_wta_kernel, sms, wave.pixels, kPathThreads)), dim3(kPathThreads), 0,
             s, dm, wave.jobs, wave.njobs, wave.pixels, rec, sum, rowshift, info, rkeys);
  launched("sgm_path_ranged_wta_kernel");
  R3D_LAUNCH(sgm_path_ranged_accept_kernel,
             dim3(resident_grid(sgm_path_ranged_accept_kernel, sms, wave.pixels, kPathThreads)), dim3(kPathThreads),
             0, s, dm, wave.jobs, wave.njobs, wave.pixels, rec, info, rkeys, rowshift);
  launched("sgm_path_ranged_accept_kernel");
}

}  // namespace r3dgpu
