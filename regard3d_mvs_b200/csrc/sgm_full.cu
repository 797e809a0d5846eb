// SGM tile kernel for full-range tiles (every pixel searches the same nd
// labels): the computation of sgm.cu (see its header for the semantics and
// the reference citations), specialised so that the per-pixel label count is
// a compile-time shape.
//
// Layout. G lanes handle one tile row (32 / G rows per warp); lane t holds the
// K label pairs 2tK .. 2tK + 2K - 1 of its row's current pixel, contiguous,
// so that a pixel vector is read and written with 64/128-bit shared-memory
// accesses and the d -+ 1 neighbours come from the lane's own registers plus
// one word from each side. Rows are skewed by two pixels (pixel u of band row
// r at step u + 2r), and the bands of a tile run back to back as one
// wavefront: a row starts its next band as soon as it leaves the current one,
// so the rows drain and fill once per tile rather than once per band. The
// horizontal path stays in registers (its predecessor
// is the row's previous pixel; the two boundary words come by shuffle); the
// vertical and the two diagonal paths go to shared-memory rings of depth 3, 4
// and 2, read by the row below two, three and one steps later. The last row
// of a band also writes them to a global seam that the first row of the next
// band streams back with cp.async. Costs (u8) are computed per tile into the
// CTA's global scratch, forward partial sums (u16) are stored there too, and
// both are prefetched two pixels ahead with cp.async. Every instruction of a
// step is executed by all 32 lanes of a warp (rows idle at the tile's first
// and last steps compute on clamped addresses and store nothing), so shuffles
// never diverge.
#include <cstdio>
#include <cstdlib>

#include "common.cuh"
#include "sgm.h"
#include "sgm_full.h"
#include "sgm_simd.cuh"
#include "tuning.h"

namespace r3dgpu {

namespace {

using sgm_simd::group_umin;
using sgm_simd::group_vmin2;
using sgm_simd::kSent2;
using sgm_simd::load_words;
using sgm_simd::store_words;
constexpr float kInfF = __builtin_huge_valf();

template <int G, int K>
struct FullCfg {
  static constexpr int ND = 2 * G * K;  // padded label count
  static constexpr int VS = ND + 16;    // u16 stride of a shared vector (8 pad, ND, 8 pad)
  static constexpr int RPW = 32 / G;    // rows per warp
  static constexpr int SEAMV = ND + 8;  // u16 length of a global seam vector
};

// Ring vectors of a row: V slots 0..2, DB slots 3..6, DA slots 7..8 (minima likewise).
constexpr int kVec = 9;

// Shared-memory layout (bytes).
template <int G, int K>
struct FullSmem {
  using C = FullCfg<G, K>;
  static constexpr int vec_bytes = 2 * C::VS;
  static constexpr int ring_off = 0;
  static constexpr int mins_off = kVec * vec_bytes;
  static constexpr int cbuf_off = mins_off + 48;
  static constexpr int sabuf_off = cbuf_off + kSgmPFSlots * C::ND;
  static constexpr int row_bytes = sabuf_off + kSgmPFSlots * 2 * C::ND;
  static constexpr int seam_slot_bytes = 3 * vec_bytes + 16;
  static constexpr int rows_off = 16;
  R3D_HOSTDEV static int seam_off(int rows) { return rows_off + rows * row_bytes; }
  R3D_HOSTDEV static int total(int rows) { return seam_off(rows) + kSgmSeamSlots * seam_slot_bytes; }
};

template <int G, int K>
struct FullPass {
  const SgmMatch* m;
  unsigned char* smem;
  int rows;  // band rows
  int dir;
  int w, h, nd;
  const int2* recs;     // penalties, pass-local order
  const uint8_t* cost;  // image order, nd per pixel
  uint16_t* sa;         // forward partial sums, image order
  int4* info;           // image order
  unsigned char* seam;  // two seam buffers
  int64_t seam_pix;     // bytes per seam pixel
  uint32_t* rkeys;
  int64_t rk;
  int x0, y0;
  uint16_t* volume;
};

template <int G, int K>
R3D_DEVICE uint16_t* ring_vec(unsigned char* smem, int r, int v) {
  using S = FullSmem<G, K>;
  return reinterpret_cast<uint16_t*>(smem + S::rows_off + r * S::row_bytes + S::ring_off + v * S::vec_bytes) + 8;
}

template <int G, int K>
R3D_DEVICE uint32_t* ring_mins(unsigned char* smem, int r) {
  using S = FullSmem<G, K>;
  return reinterpret_cast<uint32_t*>(smem + S::rows_off + r * S::row_bytes + S::mins_off);
}

template <int G, int K>
R3D_DEVICE uint16_t* seam_vec_s(unsigned char* smem, int rows, int s, int path) {
  using S = FullSmem<G, K>;
  return reinterpret_cast<uint16_t*>(smem + S::seam_off(rows) + s * S::seam_slot_bytes + path * S::vec_bytes) + 8;
}

template <int G, int K>
R3D_DEVICE uint32_t* seam_meta_s(unsigned char* smem, int rows, int s) {
  using S = FullSmem<G, K>;
  return reinterpret_cast<uint32_t*>(smem + S::seam_off(rows) + s * S::seam_slot_bytes + 3 * S::vec_bytes);
}

template <int G, int K>
R3D_DEVICE uint16_t* gseam_vec_f(unsigned char* seam, int64_t pix, int u, int path) {
  return reinterpret_cast<uint16_t*>(seam + u * pix) + path * FullCfg<G, K>::SEAMV;
}

template <int G, int K>
R3D_DEVICE uint32_t* gseam_meta_f(unsigned char* seam, int64_t pix, int u) {
  return reinterpret_cast<uint32_t*>(seam + u * pix + 3 * 2 * FullCfg<G, K>::SEAMV);
}

template <int G, int K, bool MASKED>
R3D_DEVICE void run_full_pass(const FullPass<G, K>& a) {
  using C = FullCfg<G, K>;
  using S = FullSmem<G, K>;
  const int lane = static_cast<int>(threadIdx.x & 31u);
  const int warp = static_cast<int>(threadIdx.x >> 5);
  const int gi = lane / G;  // row within the warp
  const int t = lane % G;   // lane within the row
  const int r = warp * C::RPW + gi;
  const SgmMatch& m = *a.m;
  const uint32_t p1x2 = static_cast<uint32_t>(m.p1) * 0x10001u;
  const bool no_carry = m.sum_no_carry != 0;
  const int nd = a.nd;
  const int e0 = 2 * t * K;  // first label of the lane
  uint32_t maskbits = 0;     // words with labels >= nd (MASKED shapes only)
  if constexpr (MASKED) {
#pragma unroll
    for (int j = 0; j < K; ++j)
      if (e0 + 2 * j >= nd) maskbits |= 1u << j;
  }
  uint32_t* mins = ring_mins<G, K>(a.smem, r);
  uint8_t* cbuf = a.smem + S::rows_off + r * S::row_bytes + S::cbuf_off;
  uint16_t* sabuf = reinterpret_cast<uint16_t*>(a.smem + S::rows_off + r * S::row_bytes + S::sabuf_off);
  const int rup = r > 0 ? r - 1 : 0;
  uint32_t* mins_up = ring_mins<G, K>(a.smem, rup);
  const int left_lane = (lane + 31) & 31, right_lane = (lane + 1) & 31;

  // Bands follow one another without a pause: band row r handles its local
  // step L (pixel u = L mod P of band L / P) at CTA step L + 2r, so the first
  // rows of band b + 1 start while the lower rows of band b finish. The period
  // P is at least the tile width and at least 2 rows + kSgmPF: the last row of
  // band b writes seam pixel u at step bP + u + 2(rows - 1), strictly before
  // the first row of band b + 1 prefetches it at step (b + 1)P + u - kSgmPF - 1.
  // Ring, prefetch and seam slots are indexed by L, which advances by one
  // across a band change, so consecutive steps never share a slot.
  {
    const int R = a.rows;
    const int nb = (a.h + R - 1) / R;
    const int P = r3dsimt::imax(a.w, 2 * R + kSgmPF);
    struct Pos {
      int b, u, L;  // band, pixel (negative before the row's first step), local step
    };
    auto adv = [&](Pos p, int k) -> Pos {
      p.u += k;
      p.L += k;
      if (p.u >= P) {
        p.u -= P;
        ++p.b;
      }
      return p;
    };
    auto valid = [&](const Pos& p) -> bool { return p.u >= 0 && p.u < a.w && p.b * R + r < a.h; };
    auto row_of = [&](const Pos& p) -> int { return r3dsimt::imin(p.b * R + r, a.h - 1); };  // clamped
    auto pixel_off = [&](const Pos& p) -> int64_t {
      const int v = row_of(p);
      const int y = a.dir > 0 ? v : a.h - 1 - v;
      const int uc = p.u < 0 ? 0 : (p.u >= a.w ? a.w - 1 : p.u);
      const int x = a.dir > 0 ? uc : a.w - 1 - uc;
      return (static_cast<int64_t>(y) * a.w + x) * nd;
    };
    auto prefetch = [&](const Pos& p) {
      if (!valid(p)) return;
      const int64_t off = pixel_off(p);
      const int slot = p.L & (kSgmPFSlots - 1);
      for (int q = t; q < nd / 16; q += G) r3dsimt::cp_async16(cbuf + slot * C::ND + 16 * q, a.cost + off + 16 * q);
      if (a.dir < 0)
        for (int q = t; q < nd / 8; q += G) r3dsimt::cp_async16(sabuf + slot * C::ND + 8 * q, a.sa + off + 8 * q);
    };
    auto prefetch_seam = [&](const Pos& p) {
      if (r != 0 || p.b == 0 || !valid(p)) return;
      unsigned char* gseam_in = a.seam + static_cast<size_t>((p.b + 1) & 1) * a.w * a.seam_pix;
      const int s = p.L & (kSgmSeamSlots - 1);
      constexpr int pieces = (2 * C::SEAMV) / 16;
      for (int q = t; q < 3 * pieces + 1; q += G) {
        if (q < 3 * pieces) {
          const int path = q / pieces, k = q % pieces;
          r3dsimt::cp_async16(seam_vec_s<G, K>(a.smem, a.rows, s, path) + 8 * k,
                              gseam_vec_f<G, K>(gseam_in, a.seam_pix, p.u, path) + 8 * k);
        } else {
          r3dsimt::cp_async16(seam_meta_s<G, K>(a.smem, a.rows, s), gseam_meta_f<G, K>(gseam_in, a.seam_pix, p.u));
        }
      }
    };
    auto rec_at = [&](const Pos& p) -> int2 {
      return valid(p) ? a.recs[static_cast<int64_t>(p.b * R + r) * a.w + p.u] : make_int2(0, 0);
    };

    Pos cur{0, -2 * r, -2 * r};
    int2 q0 = rec_at(cur), q1 = rec_at(adv(cur, 1)), q2 = rec_at(adv(cur, 2));
#pragma unroll
    for (int g = 0; g < kSgmPF; ++g) {
      prefetch(adv(cur, g));
      if (g == 0) prefetch_seam(cur);
      prefetch_seam(adv(cur, g + 1));
      r3dsimt::cp_async_commit();
    }
    uint32_t hprev[K];  // horizontal path of the row's previous pixel
#pragma unroll
    for (int j = 0; j < K; ++j) hprev[j] = kSent2;
    uint32_t hmin = 0;
    const int last_rows = a.h - (nb - 1) * R;
    int steps = (nb - 1) * P + a.w + 2 * (last_rows - 1);
    if (nb > 1) steps = r3dsimt::imax(steps, (nb - 2) * P + a.w + 2 * (R - 1));
    const int Lend = steps - 2 * r;  // this row's local step at the CTA's last step, plus one
    for (; cur.L < Lend; cur = adv(cur, 1)) {
      const int u = cur.u;
      const bool active = valid(cur);
      const int uc = u < 0 ? 0 : (u >= a.w ? a.w - 1 : u);  // clamped for addressing
      const int v = row_of(cur);
      const int Lc = cur.L < 0 ? 0 : cur.L;  // slot index
      const bool seam_out = active && r == R - 1 && (cur.b + 1) * R < a.h;
      unsigned char* gseam_out = a.seam + static_cast<size_t>(cur.b & 1) * a.w * a.seam_pix;
      r3dsimt::cp_async_wait<kSgmPF - 1>();
      r3dsimt::syncthreads();
      const int2 rec = q0;
      const int pslot = Lc & (kSgmPFSlots - 1);
      uint32_t c2[K];
      {
        const uint8_t* cb = cbuf + pslot * C::ND + e0;
#pragma unroll
        for (int j = 0; j < K; ++j) {
          const uint32_t b = *reinterpret_cast<const uint16_t*>(cb + 2 * j);
          c2[j] = r3dsimt::perm(b, 0u, 0x4140u);
        }
      }
      uint32_t sum[K];
#pragma unroll
      for (int j = 0; j < K; ++j) sum[j] = 0;
      const bool has_up = v > 0;
      const bool hasp[4] = {uc > 0, has_up, has_up && uc > 0, has_up && uc + 1 < a.w};
      const uint32_t p2v[4] = {static_cast<uint32_t>(rec.x) & 0xFFFFu, static_cast<uint32_t>(rec.x) >> 16,
                               static_cast<uint32_t>(rec.y) & 0xFFFFu, static_cast<uint32_t>(rec.y) >> 16};
      const uint16_t* qv[4];
      uint32_t qmin[4];
      qv[0] = nullptr;
      qmin[0] = hmin;
      if (r > 0) {
        const int u3 = Lc % 3, udb = (Lc + 3) & 3, uda = (Lc + 1) & 1;
        qv[1] = ring_vec<G, K>(a.smem, rup, u3);
        qmin[1] = mins_up[u3];
        qv[2] = ring_vec<G, K>(a.smem, rup, 3 + udb);
        qmin[2] = mins_up[3 + udb];
        qv[3] = ring_vec<G, K>(a.smem, rup, 7 + uda);
        qmin[3] = mins_up[7 + uda];
      } else {
        const int sV = Lc & (kSgmSeamSlots - 1), sDB = (Lc + kSgmSeamSlots - 1) & (kSgmSeamSlots - 1),
                  sDA = (Lc + 1) & (kSgmSeamSlots - 1);
        qv[1] = seam_vec_s<G, K>(a.smem, a.rows, sV, 0);
        qmin[1] = seam_meta_s<G, K>(a.smem, a.rows, sV)[0];
        qv[2] = seam_vec_s<G, K>(a.smem, a.rows, sDB, 1);
        qmin[2] = seam_meta_s<G, K>(a.smem, a.rows, sDB)[1];
        qv[3] = seam_vec_s<G, K>(a.smem, a.rows, sDA, 2);
        qmin[3] = seam_meta_s<G, K>(a.smem, a.rows, sDA)[2];
      }
      const int ovec[4] = {0, Lc % 3, 3 + (Lc & 3), 7 + (Lc & 1)};
      // Boundary words of the horizontal predecessor (all lanes shuffle).
      const uint32_t hl = r3dsimt::shfl(hprev[K - 1], left_lane);
      const uint32_t hr = r3dsimt::shfl(hprev[0], right_lane);
      uint32_t pmin[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        uint32_t out[K];
        uint32_t mk = kSent2;
        if (!hasp[k]) {
#pragma unroll
          for (int j = 0; j < K; ++j) out[j] = c2[j];
        } else {
          uint32_t wv[K + 2];
          if (k == 0) {
            wv[0] = t > 0 ? hl : kSent2;
#pragma unroll
            for (int j = 0; j < K; ++j) wv[1 + j] = hprev[j];
            wv[K + 1] = t + 1 < G ? hr : kSent2;
          } else {
            load_words<K>(reinterpret_cast<const uint32_t*>(qv[k]) + t * K, wv);
          }
          const uint32_t pen = qmin[k] + p2v[k];
          const uint32_t pen2 = pen | (pen << 16);
          const uint32_t negmp = 0u - (qmin[k] | (qmin[k] << 16));
          uint32_t mprev = r3dsimt::perm(wv[0], wv[1], 0x5432u);
#pragma unroll
          for (int j = 0; j < K; ++j) {
            const uint32_t mnext = r3dsimt::perm(wv[j + 1], wv[j + 2], 0x5432u);
            const uint32_t nb = r3dsimt::vmin2(mprev, mnext);
            const uint32_t best = r3dsimt::vmin2(wv[j + 1], r3dsimt::vaddmin2(nb, p1x2, pen2));
            out[j] = best + c2[j] + negmp;
            mprev = mnext;
          }
        }
#pragma unroll
        for (int j = 0; j < K; ++j) {
          if constexpr (MASKED) {
            if (maskbits & (1u << j)) out[j] = kSent2;
          }
          mk = r3dsimt::vmin2(mk, out[j]);
          sum[j] += out[j];
        }
        if (k == 0) {
          if (active) {
#pragma unroll
            for (int j = 0; j < K; ++j) hprev[j] = out[j];
          }
        } else if (active) {
          store_words<K>(reinterpret_cast<uint32_t*>(ring_vec<G, K>(a.smem, r, ovec[k])) + t * K, out);
          if (seam_out)
            store_words<K>(reinterpret_cast<uint32_t*>(gseam_vec_f<G, K>(gseam_out, a.seam_pix, uc, k - 1)) + t * K,
                           out);
        }
        pmin[k] = r3dsimt::umin(mk & 0xFFFFu, mk >> 16);
      }
      const uint32_t m01 = group_vmin2<G>(pmin[0] | (pmin[1] << 16));
      const uint32_t m23 = group_vmin2<G>(pmin[2] | (pmin[3] << 16));
      if (active) {
        hmin = m01 & 0xFFFFu;
        if (t == 0) {
          mins[Lc % 3] = m01 >> 16;
          mins[3 + (Lc & 3)] = m23 & 0xFFFFu;
          mins[7 + (Lc & 1)] = m23 >> 16;
        }
        if (seam_out && t < 4) {
          // Tail sentinels of the seam vectors and the minima.
#pragma unroll
          for (int k = 0; k < 3; ++k)
            reinterpret_cast<uint32_t*>(gseam_vec_f<G, K>(gseam_out, a.seam_pix, uc, k))[C::ND / 2 + t] = kSent2;
          if (t == 0) {
            uint32_t* gm = gseam_meta_f<G, K>(gseam_out, a.seam_pix, uc);
            gm[0] = m01 >> 16;
            gm[1] = m23 & 0xFFFFu;
            gm[2] = m23 >> 16;
            gm[3] = 0;
          }
        }
      }
      const int64_t off = pixel_off(cur);
      if (a.dir > 0) {
        if (active) {
          uint32_t* sa32 = reinterpret_cast<uint32_t*>(a.sa + off) + t * K;
          if (!MASKED || e0 + 2 * K <= nd) {
            store_words<K>(sa32, sum);
          } else {
#pragma unroll
            for (int j = 0; j < K; ++j)
              if (!(maskbits & (1u << j))) sa32[j] = sum[j];
          }
        }
      } else {
        // Total sums and winner-takes-all.
        const uint32_t* sb = reinterpret_cast<const uint32_t*>(sabuf + pslot * C::ND) + t * K;
        uint32_t kmin = 0xFFFFFFFFu;
#pragma unroll
        for (int j = 0; j < K; ++j) {
          sum[j] = no_carry ? sb[j] + sum[j] : r3dsimt::vadd2(sb[j], sum[j]);
          if (!(maskbits & (1u << j))) {
            const uint32_t e = static_cast<uint32_t>(e0 + 2 * j);
            kmin = r3dsimt::umin(kmin, r3dsimt::umin(((sum[j] & 0xFFFFu) << 16) | e, (sum[j] & 0xFFFF0000u) | (e + 1)));
          }
        }
        if (active && a.volume != nullptr) {
          uint32_t* v32 = reinterpret_cast<uint32_t*>(a.volume + off) + t * K;
#pragma unroll
          for (int j = 0; j < K; ++j)
            if (!(maskbits & (1u << j))) v32[j] = sum[j];
        }
        kmin = group_umin<G>(kmin);
        const int kb = static_cast<int>(kmin & 0xFFFFu);
        const uint32_t bcost = kmin >> 16;
        uint32_t sec = 0xFFFFu;
#pragma unroll
        for (int j = 0; j < K; ++j) {
          if (!(maskbits & (1u << j))) {
            const int e = e0 + 2 * j;
            if (e + 1 < kb || e > kb + 1) sec = r3dsimt::umin(sec, sum[j] & 0xFFFFu);
            if (e + 2 < kb || e + 1 > kb + 1) sec = r3dsimt::umin(sec, sum[j] >> 16);
          }
        }
        sec = group_umin<G>(sec);
        // S at kb - 1 and kb + 1 from the lanes that hold them (kb is
        // uniform within the row group).
        const int km = kb > 0 ? kb - 1 : 0, kp = kb + 1 < nd ? kb + 1 : nd - 1;
        const int jm = (km % (2 * K)) >> 1, jp = (kp % (2 * K)) >> 1;
        uint32_t vm = 0, vp = 0;
#pragma unroll
        for (int j = 0; j < K; ++j) {
          if (j == jm) vm = sum[j];
          if (j == jp) vp = sum[j];
        }
        const int base_lane = gi * G;
        vm = r3dsimt::shfl(vm, (base_lane + km / (2 * K)) & 31);
        vp = r3dsimt::shfl(vp, (base_lane + kp / (2 * K)) & 31);
        const uint32_t sm = (km & 1) ? (vm >> 16) : (vm & 0xFFFFu);
        const uint32_t sp = (kp & 1) ? (vp >> 16) : (vp & 0xFFFFu);
        const int x = a.w - 1 - uc, yy = a.h - 1 - v;  // image-order tile coordinates
        if (active && t == 0) {
          a.info[static_cast<int64_t>(yy) * a.w + x] =
              make_int4(static_cast<int>(static_cast<uint32_t>(kb) | (bcost << 16)),
                        static_cast<int>(sec | (sm << 16)), static_cast<int>(sp), 0);
        }
        if (active && m.diagonal_lr) {
          const RowInterval lv = m.bv[a.y0 + yy];
          const int bx = a.x0 + x;
          if (bx >= lv.first && bx <= lv.last) {
            uint32_t* keys = a.rkeys + static_cast<int64_t>(yy) * a.rk;
            // The right-WTA shift of a full-range row is max_x (nd - 1 - x) = nd - 1.
            const int b0 = x + nd - 1;
#pragma unroll
            for (int j = 0; j < K; ++j) {
              if (!(maskbits & (1u << j))) {
                const int e = e0 + 2 * j;
                atomicMin(keys + (b0 - e), ((sum[j] & 0xFFFFu) << 16) | static_cast<uint32_t>(x));
                atomicMin(keys + (b0 - e - 1), (sum[j] & 0xFFFF0000u) | static_cast<uint32_t>(x));
              }
            }
          }
        }
      }
      // Next prefetches (possibly the next band's first pixels) and the penalty queue.
      prefetch(adv(cur, kSgmPF));
      prefetch_seam(adv(cur, kSgmPF + 1));
      r3dsimt::cp_async_commit();
      q0 = q1;
      q1 = q2;
      q2 = rec_at(adv(cur, 3));
    }
    r3dsimt::cp_async_wait<0>();
    r3dsimt::fence();
    r3dsimt::syncthreads();
  }
}

template <int G, int K, bool MASKED>
R3D_GLOBAL void R3D_LAUNCH_BOUNDS(kSgmFullThreads)
    sgm_full_kernel(const SgmMatch* R3D_RESTRICT matches, const SgmJob* R3D_RESTRICT jobs, int njobs, int rows,
                    unsigned char* scratch, size_t slot_bytes, int* counter) {
  using C = FullCfg<G, K>;
  R3D_DYNAMIC_SMEM(smem);
  const int nthreads = static_cast<int>(blockDim.x);
  const int tid = static_cast<int>(threadIdx.x);
  unsigned char* slot = scratch + static_cast<size_t>(blockIdx.x) * slot_bytes;
  int* job_id = reinterpret_cast<int*>(smem);

  // Sentinel pads of every shared vector (never overwritten later).
  {
    const int nvec = rows * kVec + kSgmSeamSlots * 3;
    for (int i = tid; i < nvec * 16; i += nthreads) {
      const int vi = i >> 4, k = i & 15;
      uint16_t* vec;
      if (vi < rows * kVec) {
        vec = ring_vec<G, K>(smem, vi / kVec, vi % kVec) - 8;
      } else {
        const int s = (vi - rows * kVec) / 3, p = (vi - rows * kVec) % 3;
        vec = seam_vec_s<G, K>(smem, rows, s, p) - 8;
      }
      vec[k < 8 ? k : 8 + C::ND + (k - 8)] = 0x7FFF;
    }
  }

  while (true) {
    r3dsimt::syncthreads();
    if (tid == 0) *job_id = atomicAdd(counter, 1);
    r3dsimt::syncthreads();
    const int jid = *job_id;
    if (jid >= njobs) break;
    const SgmJob job = jobs[jid];
    const SgmMatch& m = matches[job.match];
    const int w = job.w, h = job.h, nd = m.nd;
    const int64_t npx = static_cast<int64_t>(w) * h;
    const unsigned long long cells = static_cast<unsigned long long>(npx) * static_cast<unsigned long long>(nd);
    const SgmFullSlot L = sgm_full_slot_layout(w, h, nd, C::ND);
    int2* rec_a = reinterpret_cast<int2*>(slot + L.rec_a);
    int2* rec_b = reinterpret_cast<int2*>(slot + L.rec_b);
    int4* info = reinterpret_cast<int4*>(slot + L.info);
    uint8_t* cost = slot + L.cost;
    uint16_t* sa = reinterpret_cast<uint16_t*>(slot + L.sa);
    unsigned char* seam = slot + L.seam;
    uint32_t* rkeys = reinterpret_cast<uint32_t*>(slot + L.rkeys);

    // ---- Penalties of both passes (P2 of the 4 paths; 0 without predecessor).
    const uint16_t* img = m.base;
    const int64_t ist = m.base_stride;
    for (int64_t i = tid; i < npx; i += nthreads) {
      const int y = static_cast<int>(i / w), x = static_cast<int>(i - static_cast<int64_t>(y) * w);
      const int bx = job.x0 + x, by = job.y0 + y;
      const int I = img[static_cast<int64_t>(by) * ist + bx];
      auto pen = [&](int qx, int qy) -> uint32_t {
        const int dI = I - static_cast<int>(img[static_cast<int64_t>(job.y0 + qy) * ist + job.x0 + qx]);
        return m.lut[(dI < 0 ? -dI : dI) >> 8];
      };
      const uint32_t aH = x > 0 ? pen(x - 1, y) : 0u;
      const uint32_t aV = y > 0 ? pen(x, y - 1) : 0u;
      const uint32_t aDB = (x > 0 && y > 0) ? pen(x - 1, y - 1) : 0u;
      const uint32_t aDA = (x + 1 < w && y > 0) ? pen(x + 1, y - 1) : 0u;
      const uint32_t bH = x + 1 < w ? pen(x + 1, y) : 0u;
      const uint32_t bV = y + 1 < h ? pen(x, y + 1) : 0u;
      const uint32_t bDB = (x + 1 < w && y + 1 < h) ? pen(x + 1, y + 1) : 0u;
      const uint32_t bDA = (x > 0 && y + 1 < h) ? pen(x - 1, y + 1) : 0u;
      rec_a[i] = make_int2(static_cast<int>(aH | (aV << 16)), static_cast<int>(aDB | (aDA << 16)));
      rec_b[static_cast<int64_t>(h - 1 - y) * w + (w - 1 - x)] =
          make_int2(static_cast<int>(bH | (bV << 16)), static_cast<int>(bDB | (bDA << 16)));
    }
    if (m.diagonal_lr) {
      const int64_t nk = static_cast<int64_t>(h) * L.rk;
      for (int64_t i = tid; i < nk; i += nthreads) rkeys[i] = 0xFFFFFFFFu;
    }
    // ---- Hamming costs: items of 8 labels (8 independent Census loads),
    //      two items per iteration.
    {
      const int blocks = nd / 8;
      const int64_t items = npx * blocks;
      auto item = [&](int64_t i) {
        const int64_t p = i / blocks;
        const int b = static_cast<int>(i - p * blocks);
        const int y = static_cast<int>(p / w), x = static_cast<int>(p - static_cast<int64_t>(y) * w);
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
        *reinterpret_cast<uint2*>(cost + p * nd + 8 * b) = make_uint2(lo4, hi4);
      };
      int64_t i = tid;
      for (; i + nthreads < items; i += 2 * static_cast<int64_t>(nthreads)) {
        item(i);
        item(i + nthreads);
      }
      if (i < items) item(i);
    }
    r3dsimt::fence();
    r3dsimt::syncthreads();

    FullPass<G, K> pa;
    pa.m = &m;
    pa.smem = smem;
    pa.rows = rows;
    pa.w = w;
    pa.h = h;
    pa.nd = nd;
    pa.cost = cost;
    pa.sa = sa;
    pa.info = info;
    pa.seam = seam;
    pa.seam_pix = L.seam_pix;
    pa.rkeys = rkeys;
    pa.rk = L.rk;
    pa.x0 = job.x0;
    pa.y0 = job.y0;
    pa.volume = job.volume;
    pa.dir = 1;
    pa.recs = rec_a;
    run_full_pass<G, K, MASKED>(pa);
    pa.dir = -1;
    pa.recs = rec_b;
    run_full_pass<G, K, MASKED>(pa);

    // ---- Acceptance rules and outputs (stereo_matcher.cpp:474-523), lo = 0, num = nd.
    for (int64_t i = tid; i < npx; i += nthreads) {
      const int y = static_cast<int>(i / w), x = static_cast<int>(i - static_cast<int64_t>(y) * w);
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
          const uint32_t key = rkeys[static_cast<int64_t>(y) * L.rk + (x - best + nd - 1)];
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
      job.disp[i] = d;
      if (job.conf != nullptr) job.conf[i] = cf;
    }
    if (tid == 0) *job.cells = cells;
  }
}

template <int G, int K, bool MASKED>
void launch_full_instance(const SgmMatch* dm, const SgmJob* dj, int njobs, int rows, int grid, unsigned char* scratch,
                          size_t slot_bytes, int* counter, cudaStream_t s) {
  using S = FullSmem<G, K>;
  const size_t smem = static_cast<size_t>(S::total(rows));
  static thread_local int configured[64] = {};
  int dev = 0;
  R3D_CUDA(cudaGetDevice(&dev));
  auto* kernel = sgm_full_kernel<G, K, MASKED>;
  if (dev >= 0 && dev < 64 && configured[dev] < static_cast<int>(smem)) {
    R3D_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    configured[dev] = static_cast<int>(smem);
  }
  const int threads = rows / FullCfg<G, K>::RPW * 32;
  R3D_LAUNCH(kernel, dim3(grid), dim3(threads), smem, s, dm, dj, njobs, rows, scratch, slot_bytes, counter);
  launched("sgm_full_kernel");
}

// Shapes compiled into the library (lanes per row G, label pairs per lane K).
#define R3D_FULL_SHAPES(X) \
  X(8, 4)                  \
  X(8, 8)                  \
  X(16, 4)                 \
  X(8, 12)                 \
  X(16, 6)                 \
  X(16, 8)                 \
  X(8, 16)                 \
  X(16, 12)                \
  X(32, 8)                 \
  X(32, 12)

}  // namespace

SgmFullPlan sgm_full_plan(int nd, int smem_optin) {
  SgmFullPlan p{{0, 0}, 0};
  // Default shapes: the most labels per lane that compile without spills.
  if (nd <= 64) p.shape = {8, 4};
  else if (nd <= 128) p.shape = {8, 8};
  else if (nd <= 192) p.shape = {8, 12};
  else if (nd <= 256) p.shape = {16, 8};
  else if (nd <= 384) p.shape = {16, 12};
  else if (nd <= 512) p.shape = {32, 8};
  else if (nd <= 768) p.shape = {32, 12};
  else return p;
  int max_rows = 1 << 20;
  // The autotuner's entry for this label count, if any.
  {
    const auto& table = tuning().full;
    const auto it = table.find(nd);
    if (it != table.end() && 2 * it->second.g * it->second.k >= nd &&
        sgm_full_shape_compiled({it->second.g, it->second.k})) {
      p.shape = {it->second.g, it->second.k};
      max_rows = it->second.rows;
    }
  }
  if (const char* e = std::getenv("R3DGPU_FULL_SHAPE")) {
    int g = 0, k = 0;
    if (std::sscanf(e, "%d,%d", &g, &k) == 2 && 2 * g * k >= nd && sgm_full_shape_compiled({g, k})) p.shape = {g, k};
  }
  if (const char* e = std::getenv("R3DGPU_FULL_ROWS")) max_rows = std::max(32 / p.shape.g_, std::atoi(e));
  p.rows = sgm_full_rows(p.shape, smem_optin, max_rows);
  return p;
}

int sgm_full_smem(SgmFullShape sh, int rows) {
#define R3D_SHAPE(g, k) \
  if (sh.g_ == g && sh.k_ == k) return FullSmem<g, k>::total(rows);
  R3D_FULL_SHAPES(R3D_SHAPE)
#undef R3D_SHAPE
  fail(R3DGPU_EINVAL, "stereo: bad full-range kernel shape");
}

bool sgm_full_shape_compiled(SgmFullShape sh) {
#define R3D_SHAPE(g, k) \
  if (sh.g_ == g && sh.k_ == k) return true;
  R3D_FULL_SHAPES(R3D_SHAPE)
#undef R3D_SHAPE
  return false;
}

int sgm_full_rows(SgmFullShape sh, int smem_optin, int max_rows) {
  const int rpw = 32 / sh.g_;
  for (int warps = kSgmFullThreads / 32; warps >= 1; --warps) {
    const int rows = warps * rpw;
    if (rows <= max_rows && sgm_full_smem(sh, rows) <= smem_optin) return rows;
  }
  fail(R3DGPU_EUNSUPPORTED, "stereo: label count needs more shared memory than the device has");
}

void launch_sgm_full(SgmFullShape sh, int nd, const SgmMatch* dm, const SgmJob* dj, int njobs, int rows, int grid,
                     unsigned char* scratch, size_t slot_bytes, int* counter, cudaStream_t s) {
#define R3D_SHAPE(g, k)                                                                               \
  if (sh.g_ == g && sh.k_ == k) {                                                                     \
    if (nd == 2 * g * k)                                                                              \
      launch_full_instance<g, k, false>(dm, dj, njobs, rows, grid, scratch, slot_bytes, counter, s); \
    else                                                                                              \
      launch_full_instance<g, k, true>(dm, dj, njobs, rows, grid, scratch, slot_bytes, counter, s);  \
    return;                                                                                           \
  }
  R3D_FULL_SHAPES(R3D_SHAPE)
#undef R3D_SHAPE
  fail(R3DGPU_EINVAL, "stereo: bad full-range kernel shape");
}

}  // namespace r3dgpu
