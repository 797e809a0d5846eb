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
#include <cstdlib>
#include <cstring>

#include "common.cuh"
#include "sgm_path.h"
#include "sgm_simd.cuh"

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
// C(p, a) of stereo_matcher.cpp:305-353 for 8 labels per item, u8.
R3D_GLOBAL void R3D_LAUNCH_BOUNDS(kPathThreads)
    sgm_path_cost_kernel(const SgmMatch* R3D_RESTRICT matches, const SgmPathJob* R3D_RESTRICT jobs, int njobs,
                         int64_t items, uint8_t* R3D_RESTRICT cost) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < items; i += stride) {
    const int64_t cell = 8 * i;
    const int j = find_job(jobs, njobs, cell, [](const SgmPathJob& q) { return q.cell_off; });
    const SgmPathJob& job = jobs[j];
    const SgmMatch& m = matches[job.match];
    const int nd = m.nd;
    const int64_t local = cell - job.cell_off;
    const int p = static_cast<int>(local / nd);
    const int b = static_cast<int>(local - static_cast<int64_t>(p) * nd) >> 3;
    const int y = p / job.w, x = p - (p / job.w) * job.w;
    const int bx = job.x0 + x, by = job.y0 + y;
    const RowInterval lv = m.bv[by], rv = m.pv[by];
    uint32_t lo4 = 0, hi4 = 0;
    if (bx >= lv.first && bx <= lv.last) {
      const uint64_t cl = m.cbase[static_cast<int64_t>(by) * m.cb_stride + bx];
      const uint64_t* crow = m.cpart + static_cast<int64_t>(by) * m.cp_stride;
      const int xr0 = bx - m.dmin - 8 * b;
      const int safe = rv.first > 0 ? rv.first : 0;
      uint32_t c[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int xr = xr0 - k;
        const bool ok = xr >= rv.first && xr <= rv.last;
        const uint64_t cr = crow[ok ? xr : safe];
        c[k] = ok ? static_cast<uint32_t>(r3dsimt::popc64(cl ^ cr)) : static_cast<uint32_t>(m.invalid_cost);
      }
      lo4 = c[0] | (c[1] << 8) | (c[2] << 16) | (c[3] << 24);
      hi4 = c[4] | (c[5] << 8) | (c[6] << 16) | (c[7] << 24);
    }
    *reinterpret_cast<uint2*>(cost + cell) = make_uint2(lo4, hi4);
  }
}

// ---------------------------------------------------------------- passes
enum PassMode { kFirst = 0, kAccumulate = 1, kLast = 2 };

// Per-halfword a + b modulo 2^16.
R3D_DEVICE uint32_t add2(uint32_t a, uint32_t b, bool no_carry) { return no_carry ? a + b : r3dsimt::vadd2(a, b); }

template <int G, int K, int MODE>
R3D_GLOBAL void R3D_LAUNCH_BOUNDS(kPathThreads)
    sgm_path_kernel(const SgmMatch* R3D_RESTRICT matches, const SgmPathJob* R3D_RESTRICT jobs, int njobs, int cls,
                    int dx, int dy, int64_t total_blocks, const uint8_t* R3D_RESTRICT cost, uint16_t* sum,
                    int4* R3D_RESTRICT info, uint32_t* rkeys) {
  constexpr int CPW = 32 / G;  // chains per warp
  constexpr int U = K / 4;     // units of 8 labels per lane
  const int lane = static_cast<int>(threadIdx.x & 31u);
  const int gi = lane / G, t = lane % G;
  const int e0 = 2 * t * K;  // first label of the lane
  const int left_lane = (lane + 31) & 31, right_lane = (lane + 1) & 31;
  const int wpb = static_cast<int>(blockDim.x) >> 5;
  const int64_t nwarps = static_cast<int64_t>(gridDim.x) * wpb;
  for (int64_t blk = static_cast<int64_t>(blockIdx.x) * wpb + (threadIdx.x >> 5); blk < total_blocks; blk += nwarps) {
    const int j = find_job(jobs, njobs, blk, [cls](const SgmPathJob& q) { return q.blk[cls]; });
    const SgmPathJob& job = jobs[j];
    const SgmMatch& m = matches[job.match];
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
    for (int u = 0; u < U; ++u) uvalid[u] = e0 + 8 * u < nd;
    const uint8_t* cbase = cost + job.cell_off + e0;
    uint16_t* sbase = sum + job.cell_off + e0;
    const uint16_t* img = m.base + static_cast<int64_t>(job.y0) * m.base_stride + job.x0;

    // Data of the current and the next pixel of the chain.
    uint2 craw[U], cnext[U];
    uint4 sraw[U], snext[U];
    int icur = 0, inext = 0;
    auto load = [&](int i, uint2 (&cr)[U], uint4 (&sr)[U], int& iv) {
      if (i >= len) return;
      const int x = sx + i * dx, y = sy + i * dy;
      const int64_t cell = static_cast<int64_t>(y * w + x) * nd;
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (uvalid[u]) {
          cr[u] = *reinterpret_cast<const uint2*>(cbase + cell + 8 * u);
          if constexpr (MODE != kFirst) sr[u] = r3dsimt::ld_stream(reinterpret_cast<const uint4*>(sbase + cell + 8 * u));
        }
      }
      iv = img[static_cast<int64_t>(y) * m.base_stride + x];
    };
#pragma unroll
    for (int u = 0; u < U; ++u) {
      craw[u] = make_uint2(0, 0);
      cnext[u] = make_uint2(0, 0);
      sraw[u] = make_uint4(0, 0, 0, 0);
      snext[u] = make_uint4(0, 0, 0, 0);
    }
    load(0, craw, sraw, icur);
    uint32_t prev[K];
#pragma unroll
    for (int k = 0; k < K; ++k) prev[k] = kSent2;
    uint32_t pmin = 0;
    int iprev = 0;
    for (int i = 0; i < maxlen; ++i) {
      const bool on = i < len;
      load(i + 1, cnext, snext, inext);
      uint32_t c2[K];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        c2[4 * u + 0] = r3dsimt::perm(craw[u].x, 0u, 0x4140u);
        c2[4 * u + 1] = r3dsimt::perm(craw[u].x, 0u, 0x4342u);
        c2[4 * u + 2] = r3dsimt::perm(craw[u].y, 0u, 0x4140u);
        c2[4 * u + 3] = r3dsimt::perm(craw[u].y, 0u, 0x4342u);
      }
      uint32_t out[K];
      if (i == 0) {
        // First pixel of the chain: no predecessor inside the tile, L = C.
#pragma unroll
        for (int k = 0; k < K; ++k) out[k] = c2[k];
      } else {
        const int dI = icur - iprev;
        const uint32_t pen = pmin + m.lut[(dI < 0 ? -dI : dI) >> 8];
        const uint32_t pen2 = pen | (pen << 16);
        const uint32_t negmp = 0u - (pmin | (pmin << 16));
        const uint32_t hl = r3dsimt::shfl(prev[K - 1], left_lane);
        const uint32_t hr = r3dsimt::shfl(prev[0], right_lane);
        uint32_t wv[K + 2];
        wv[0] = t > 0 ? hl : kSent2;
#pragma unroll
        for (int k = 0; k < K; ++k) wv[1 + k] = prev[k];
        wv[K + 1] = t + 1 < G ? hr : kSent2;
        uint32_t mprev = r3dsimt::perm(wv[0], wv[1], 0x5432u);
#pragma unroll
        for (int k = 0; k < K; ++k) {
          const uint32_t mnext = r3dsimt::perm(wv[k + 1], wv[k + 2], 0x5432u);
          const uint32_t nb = r3dsimt::vmin2(mprev, mnext);
          const uint32_t best = r3dsimt::vmin2(wv[k + 1], r3dsimt::vaddmin2(nb, p1x2, pen2));
          out[k] = best + c2[k] + negmp;
          mprev = mnext;
        }
      }
      uint32_t mk = kSent2;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (!uvalid[k / 4]) out[k] = kSent2;
        mk = r3dsimt::vmin2(mk, out[k]);
      }
      pmin = group_umin<G>(r3dsimt::umin(mk & 0xFFFFu, mk >> 16));
      const int x = sx + i * dx, y = sy + i * dy;
      const int64_t cell = static_cast<int64_t>(y * w + x) * nd;
      if constexpr (MODE == kFirst) {
        if (on) {
#pragma unroll
          for (int u = 0; u < U; ++u)
            if (uvalid[u])
              r3dsimt::st_stream(reinterpret_cast<uint4*>(sbase + cell + 8 * u),
                                 make_uint4(out[4 * u], out[4 * u + 1], out[4 * u + 2], out[4 * u + 3]));
        }
      } else {
        uint32_t s[K];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          s[4 * u + 0] = add2(sraw[u].x, out[4 * u + 0], no_carry);
          s[4 * u + 1] = add2(sraw[u].y, out[4 * u + 1], no_carry);
          s[4 * u + 2] = add2(sraw[u].z, out[4 * u + 2], no_carry);
          s[4 * u + 3] = add2(sraw[u].w, out[4 * u + 3], no_carry);
        }
        if constexpr (MODE == kAccumulate) {
          if (on) {
#pragma unroll
            for (int u = 0; u < U; ++u)
              if (uvalid[u])
                r3dsimt::st_stream(reinterpret_cast<uint4*>(sbase + cell + 8 * u),
                                   make_uint4(s[4 * u], s[4 * u + 1], s[4 * u + 2], s[4 * u + 3]));
          }
        } else {
          // Winner-takes-all over the total sums (sgm_kernels.cpp:332-358):
          // the first minimum, the second best outside +-1, and S at kb -+ 1.
          uint32_t kmin = 0xFFFFFFFFu;
#pragma unroll
          for (int k = 0; k < K; ++k) {
            if (uvalid[k / 4]) {
              const uint32_t e = static_cast<uint32_t>(e0 + 2 * k);
              kmin = r3dsimt::umin(kmin, r3dsimt::umin(((s[k] & 0xFFFFu) << 16) | e, (s[k] & 0xFFFF0000u) | (e + 1)));
            }
          }
          kmin = group_umin<G>(kmin);
          const int kb = static_cast<int>(kmin & 0xFFFFu);
          const uint32_t bcost = kmin >> 16;
          uint32_t sec = 0xFFFFu;
#pragma unroll
          for (int k = 0; k < K; ++k) {
            if (uvalid[k / 4]) {
              const int e = e0 + 2 * k;
              if (e + 1 < kb || e > kb + 1) sec = r3dsimt::umin(sec, s[k] & 0xFFFFu);
              if (e + 2 < kb || e + 1 > kb + 1) sec = r3dsimt::umin(sec, s[k] >> 16);
            }
          }
          sec = group_umin<G>(sec);
          const int km = kb > 0 ? kb - 1 : 0, kp = kb + 1 < nd ? kb + 1 : nd - 1;
          const int jm = (km % (2 * K)) >> 1, jp = (kp % (2 * K)) >> 1;
          uint32_t vm = 0, vp = 0;
#pragma unroll
          for (int k = 0; k < K; ++k) {
            if (k == jm) vm = s[k];
            if (k == jp) vp = s[k];
          }
          const int base_lane = gi * G;
          vm = r3dsimt::shfl(vm, (base_lane + km / (2 * K)) & 31);
          vp = r3dsimt::shfl(vp, (base_lane + kp / (2 * K)) & 31);
          const uint32_t sm = (km & 1) ? (vm >> 16) : (vm & 0xFFFFu);
          const uint32_t sp = (kp & 1) ? (vp >> 16) : (vp & 0xFFFFu);
          if (on) {
            if (t == 0)
              info[job.px_off + static_cast<int64_t>(y) * w + x] =
                  make_int4(static_cast<int>(static_cast<uint32_t>(kb) | (bcost << 16)),
                            static_cast<int>(sec | (sm << 16)), static_cast<int>(sp), 0);
            if (job.volume != nullptr) {
              uint16_t* vb = job.volume + cell + e0;
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
      }
#pragma unroll
      for (int k = 0; k < K; ++k) prev[k] = out[k];
      iprev = icur;
      icur = inext;
#pragma unroll
      for (int u = 0; u < U; ++u) {
        craw[u] = cnext[u];
        sraw[u] = snext[u];
      }
    }
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

// ---------------------------------------------------------------- launches
// Pass order: the first pass writes the sums, the last takes the WTA.
struct Pass {
  int cls, dx, dy;
};
constexpr Pass kPasses[8] = {{0, 1, 0},  {1, 0, 1},   {2, 1, 1},  {2, -1, 1},
                             {1, 0, -1}, {2, -1, -1}, {2, 1, -1}, {0, -1, 0}};

template <class Kernel>
int resident_grid(Kernel kernel, int sms, int64_t work_items, int per_block) {
  int per_sm = 1;
  R3D_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kPathThreads, 0));
  const int64_t need = (work_items + per_block - 1) / per_block;
  const int64_t resident = static_cast<int64_t>(sms) * (per_sm > 0 ? per_sm : 1);
  return static_cast<int>(need < resident ? (need > 0 ? need : 1) : resident);
}

template <int G, int K>
void launch_passes(const SgmMatch* dm, const SgmPathJob* jobs, int njobs, const int64_t (&blocks)[kPathClasses],
                   const uint8_t* cost, uint16_t* sum, int4* info, uint32_t* rkeys, int sms, cudaStream_t s) {
  for (int q = 0; q < 8; ++q) {
    const Pass ps = kPasses[q];
    const int64_t nb = blocks[ps.cls];
    if (nb <= 0) continue;
    if (q == 0) {
      auto* k = sgm_path_kernel<G, K, kFirst>;
      R3D_LAUNCH(k, dim3(resident_grid(k, sms, nb, kPathThreads / 32)), dim3(kPathThreads), 0, s, dm, jobs, njobs,
                 ps.cls, ps.dx, ps.dy, nb, cost, sum, info, rkeys);
    } else if (q < 7) {
      auto* k = sgm_path_kernel<G, K, kAccumulate>;
      R3D_LAUNCH(k, dim3(resident_grid(k, sms, nb, kPathThreads / 32)), dim3(kPathThreads), 0, s, dm, jobs, njobs,
                 ps.cls, ps.dx, ps.dy, nb, cost, sum, info, rkeys);
    } else {
      auto* k = sgm_path_kernel<G, K, kLast>;
      R3D_LAUNCH(k, dim3(resident_grid(k, sms, nb, kPathThreads / 32)), dim3(kPathThreads), 0, s, dm, jobs, njobs,
                 ps.cls, ps.dx, ps.dy, nb, cost, sum, info, rkeys);
    }
    launched("sgm_path_kernel");
  }
}

// Shapes compiled into the library (lanes per chain G, label pairs per lane K).
#define R3D_PATH_SHAPES(X) \
  X(1, 8)                  \
  X(2, 8)                  \
  X(2, 12)                 \
  X(4, 8)                  \
  X(4, 12)                 \
  X(8, 8)                  \
  X(8, 12)                 \
  X(16, 8)                 \
  X(16, 12)                \
  X(32, 8)                 \
  X(32, 12)

}  // namespace

bool sgm_path_enabled() {
  const char* e = std::getenv("R3DGPU_FULL_KERNEL");
  return !(e != nullptr && std::strcmp(e, "wavefront") == 0);
}

SgmPathShape sgm_path_shape(int nd) {
  SgmPathShape best{0, 0};
  int best_nd = 1 << 30;
#define R3D_SHAPE(g, k)                           \
  if (2 * g * k >= nd && 2 * g * k < best_nd) { \
    best = SgmPathShape{g, k};                    \
    best_nd = 2 * g * k;                          \
  }
  R3D_PATH_SHAPES(R3D_SHAPE)
#undef R3D_SHAPE
  return best;
}

SgmPathBuffers sgm_path_buffers(int64_t cells, int64_t pixels, int64_t keys) {
  SgmPathBuffers b{};
  size_t o = 0;
  b.cost = o;
  o += align256(static_cast<size_t>(cells));
  b.sum = o;
  o += align256(static_cast<size_t>(cells) * 2);
  b.info = o;
  o += align256(static_cast<size_t>(pixels) * 16);
  b.rkeys = o;
  o += align256(static_cast<size_t>(keys) * 4);
  b.total = o;
  return b;
}

void launch_sgm_path_wave(const SgmMatch* dm, const SgmPathWave& wave, int sms, cudaStream_t s) {
  if (wave.njobs <= 0 || wave.cells <= 0) return;
  const SgmPathBuffers B = sgm_path_buffers(wave.cells, wave.pixels, wave.keys);
  uint8_t* cost = wave.buffer + B.cost;
  uint16_t* sum = reinterpret_cast<uint16_t*>(wave.buffer + B.sum);
  int4* info = reinterpret_cast<int4*>(wave.buffer + B.info);
  uint32_t* rkeys = reinterpret_cast<uint32_t*>(wave.buffer + B.rkeys);
  if (wave.keys > 0) R3D_CUDA(cudaMemsetAsync(rkeys, 0xFF, static_cast<size_t>(wave.keys) * 4, s));
  {
    const int64_t items = wave.cells / 8;
    R3D_LAUNCH(sgm_path_cost_kernel, dim3(resident_grid(sgm_path_cost_kernel, sms, items, kPathThreads)),
               dim3(kPathThreads), 0, s, dm, wave.jobs, wave.njobs, items, cost);
    launched("sgm_path_cost_kernel");
  }
  for (int q = 0; q < wave.nsegs; ++q) {
    const SgmPathSegment& g = wave.segs[q];
    const SgmPathJob* jobs = wave.jobs + g.first;
    bool done = false;
#define R3D_SHAPE(gg, kk)                                                                                     \
  if (!done && g.shape.g_ == gg && g.shape.k_ == kk) {                                                        \
    launch_passes<gg, kk>(dm, jobs, g.count, g.blocks, cost, sum, info, rkeys, sms, s);                       \
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

}  // namespace r3dgpu
