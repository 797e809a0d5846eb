// SGM tile kernel for ranged tiles: every pixel searches its own label range
// [lo, lo + num) (the finer levels of the hierarchy, where the ranges come
// from the coarser level's disparities). The computation is that of sgm.cu
// (see its header for the semantics and the reference citations); this
// kernel is laid out for the range statistics of those levels, where most
// pixels carry 16 or 32 labels, neighbours nearly always share their range
// or differ by a few labels, and a few pixels (depth edges, unmatched
// regions) carry hundreds.
//
// Layout. As in sgm_full.cu, G lanes handle one tile row (32 / G rows per
// warp), lane t holding the K label pairs 2tK .. 2tK + 2K - 1 of the row's
// current pixel, rows are skewed by two pixels per row, and a tile's bands
// run back to back as one wavefront. A pixel whose
// range fits the row's ND = 2GK labels ("narrow") keeps its four path
// vectors in shared-memory rings of ND labels; the vectors of a row are
// separated by 16 sentinel labels. A narrow predecessor whose lo differs from
// the pixel's by at most 12 labels is read as K + 3 words at the shifted
// position and realigned with a funnel shift, the pads supplying the
// sentinels, so that every row of a warp runs the same instructions whatever
// its shift; anything else (a larger shift, or a wide predecessor) is read
// label by label with bounds checks. A pixel with more than ND labels
// ("wide") is processed by its row's lanes in chunks of ND labels, its path
// vectors going to a per-row ring in the CTA's global scratch. All loads of
// a pixel (or chunk) are issued before its stores. Labels outside a range
// hold 0x7FFF, which never wins against the P2 term, so every value stays
// exact without saturating arithmetic.
#include <cstdio>
#include <cstdlib>

#include "common.cuh"
#include "sgm.h"
#include "sgm_ranged.h"
#include "sgm_simd.cuh"
#include "tuning.h"

namespace r3dgpu {

namespace {

using sgm_simd::group_umin;
using sgm_simd::group_vmin2;
using sgm_simd::kSent2;
using sgm_simd::store_words;
constexpr uint32_t kSent = 0x7FFFu;
constexpr float kInfF = __builtin_huge_valf();
constexpr int kPad = 16;       // sentinel labels between the shared vectors of a row
constexpr int kMaxShift = 12;  // largest |lo - qlo| the shifted read serves within the pads

template <int G, int K>
struct RangedCfg {
  static constexpr int ND = 2 * G * K;    // labels of a narrow pixel
  static constexpr int VS = ND + kPad;    // u16 stride of the shared vectors
  static constexpr int RPW = 32 / G;      // rows per warp
  static constexpr int MAXT = K >= 8 ? 256 : kSgmRangedThreads;  // CTA size cap (registers per thread)
};

// Vector indices of a row (shared ring, global wide ring and minima alike):
// V 0..2, DB 3..6, DA 7..8, H 9..10, by the producing pixel u.
R3D_DEVICE int vec_v(int u) { return u % 3; }
R3D_DEVICE int vec_db(int u) { return 3 + (u & 3); }
R3D_DEVICE int vec_da(int u) { return 7 + (u & 1); }
R3D_DEVICE int vec_h(int u) { return 9 + (u & 1); }

// Shared-memory layout (bytes). Row block: [pad v0 pad v1 ... v10 pad]
// (u16), 11 minima, 4 metas (lo | num << 16 by u % 4), prefetch slots of
// costs and forward sums. Seam slot: [pad V pad DB pad DA pad], then
// {minV, minDB, minDA, lo | num << 16}.
template <int G, int K>
struct RangedSmem {
  using C = RangedCfg<G, K>;
  static constexpr int ring_bytes = 2 * (kPad + kSgmRangedVecs * C::VS);
  static constexpr int mins_off = ring_bytes;
  static constexpr int meta_off = mins_off + 48;
  static constexpr int cbuf_off = meta_off + 16;
  static constexpr int sabuf_off = cbuf_off + kSgmPFSlots * C::ND;
  static constexpr int row_bytes = sabuf_off + kSgmPFSlots * 2 * C::ND;
  static constexpr int seam_vec_bytes = 2 * (kPad + 3 * C::VS);
  static constexpr int seam_slot_bytes = seam_vec_bytes + 16;
  static constexpr int rows_off = 16;
  static_assert(ring_bytes % 16 == 0 && row_bytes % 16 == 0 && seam_slot_bytes % 16 == 0, "16-byte layout");
  R3D_HOSTDEV static int seam_off(int rows) { return rows_off + rows * row_bytes; }
  R3D_HOSTDEV static int total(int rows) { return seam_off(rows) + kSgmSeamSlots * seam_slot_bytes; }
};

template <int G, int K>
R3D_DEVICE uint16_t* rvec(unsigned char* smem, int r, int v) {
  using S = RangedSmem<G, K>;
  return reinterpret_cast<uint16_t*>(smem + S::rows_off + r * S::row_bytes) + kPad + v * RangedCfg<G, K>::VS;
}
template <int G, int K>
R3D_DEVICE uint32_t* rmins(unsigned char* smem, int r) {
  using S = RangedSmem<G, K>;
  return reinterpret_cast<uint32_t*>(smem + S::rows_off + r * S::row_bytes + S::mins_off);
}
template <int G, int K>
R3D_DEVICE uint32_t* rmeta(unsigned char* smem, int r) {
  using S = RangedSmem<G, K>;
  return reinterpret_cast<uint32_t*>(smem + S::rows_off + r * S::row_bytes + S::meta_off);
}
template <int G, int K>
R3D_DEVICE uint16_t* seam_vec_s(unsigned char* smem, int rows, int s, int path) {
  using S = RangedSmem<G, K>;
  return reinterpret_cast<uint16_t*>(smem + S::seam_off(rows) + s * S::seam_slot_bytes) + kPad +
         path * RangedCfg<G, K>::VS;
}
template <int G, int K>
R3D_DEVICE uint32_t* seam_meta_s(unsigned char* smem, int rows, int s) {
  using S = RangedSmem<G, K>;
  return reinterpret_cast<uint32_t*>(smem + S::seam_off(rows) + s * S::seam_slot_bytes + S::seam_vec_bytes);
}
// Global seam pixel u: 16 bytes of meta, then the V, DB and DA vectors of ndw labels.
R3D_DEVICE uint32_t* gseam_meta(unsigned char* seam, int64_t pix, int u) {
  return reinterpret_cast<uint32_t*>(seam + u * pix);
}
R3D_DEVICE uint16_t* gseam_vec(unsigned char* seam, int64_t pix, int u, int path, int ndw) {
  return reinterpret_cast<uint16_t*>(seam + u * pix + 16) + path * ndw;
}

// A path predecessor: its vector (shared when narrow, global when wide),
// range and minimum.
struct Pred {
  const uint16_t* s;
  const uint16_t* g;
  int lo, num;
  uint32_t qmin;
};

template <int ND>
R3D_DEVICE uint32_t pred_at(const Pred& q, int j) {
  if (q.num <= ND) return (j >= 0 && j < ND) ? static_cast<uint32_t>(q.s[j]) : kSent;
  return (j >= 0 && j < q.num) ? static_cast<uint32_t>(__ldcg(q.g + j)) : kSent;
}

// Packed neighbour minimum min(q[j-1], q[j+1]) and middle q[j] of the label
// pair whose first label sits at q's index j (bounds-checked reads).
template <int ND>
R3D_DEVICE void pred_pair(const Pred& q, int j, uint32_t& nb, uint32_t& mid) {
  const uint32_t a = pred_at<ND>(q, j - 1), b = pred_at<ND>(q, j), c = pred_at<ND>(q, j + 1), d = pred_at<ND>(q, j + 2);
  nb = r3dsimt::vmin2(a | (b << 16), c | (d << 16));
  mid = b | (c << 16);
}

// L of one path for the lane's K label pairs of a narrow pixel (labels at or
// beyond num are set to the sentinel by the caller). Called by all lanes of
// the warp: when no row of the warp has a shifted or out-of-reach
// predecessor, the predecessor is read with aligned vector loads; otherwise
// rows read K + 3 words at their shift and realign them with a funnel shift,
// and rows whose predecessor is wide or shifted beyond the pads read label
// by label with bounds checks.
template <int G, int K>
R3D_DEVICE void path_narrow(const Pred& q, bool has, uint32_t p2, int lo, int t, uint32_t p1x2,
                            const uint32_t (&c2)[K], uint32_t (&out)[K]) {
  constexpr int ND = RangedCfg<G, K>::ND;
  const int e0 = 2 * t * K;
  const int shift = lo - q.lo;
  const bool near = q.num <= ND && shift >= -kMaxShift && shift <= kMaxShift;
  const int mode = !has ? 0 : (!near ? 3 : (shift != 0 ? 2 : 1));
  const uint32_t unaligned = r3dsimt::ballot(mode >= 2);
  const uint32_t pen = q.qmin + p2;
  const uint32_t pen2 = pen | (pen << 16);
  const uint32_t negmp = 0u - (q.qmin | (q.qmin << 16));
  const uint32_t* q32 = reinterpret_cast<const uint32_t*>(q.s);
  uint32_t nb[K], mid[K];
  if (unaligned == 0) {
    uint32_t wv[K + 2];
    sgm_simd::load_words<K>(q32 + t * K, wv);
    uint32_t mprev = r3dsimt::perm(wv[0], wv[1], 0x5432u);
#pragma unroll
    for (int j = 0; j < K; ++j) {
      const uint32_t mnext = r3dsimt::perm(wv[j + 1], wv[j + 2], 0x5432u);
      nb[j] = r3dsimt::vmin2(mprev, mnext);
      mid[j] = wv[j + 1];
      mprev = mnext;
    }
  } else if (mode != 3) {
    // Words from label e0 + sh - 2 (rounded down to even) on, realigned so
    // that X[j] holds labels e0 + sh - 2 + 2j and the next one.
    const int sh = mode == 0 ? 0 : shift;
    const int ws = (e0 + sh - 2) >> 1;
    const uint32_t fs = static_cast<uint32_t>(sh & 1) << 4;
    uint32_t W[K + 3];
#pragma unroll
    for (int j = 0; j < K + 3; ++j) W[j] = q32[ws + j];
    uint32_t X[K + 2];
#pragma unroll
    for (int j = 0; j < K + 2; ++j) X[j] = r3dsimt::funnel_r(W[j], W[j + 1], fs);
    uint32_t mprev = r3dsimt::perm(X[0], X[1], 0x5432u);
#pragma unroll
    for (int j = 0; j < K; ++j) {
      const uint32_t mnext = r3dsimt::perm(X[j + 1], X[j + 2], 0x5432u);
      nb[j] = r3dsimt::vmin2(mprev, mnext);
      mid[j] = X[j + 1];
      mprev = mnext;
    }
  } else {
#pragma unroll
    for (int j = 0; j < K; ++j) pred_pair<ND>(q, e0 + 2 * j + shift, nb[j], mid[j]);
  }
#pragma unroll
  for (int j = 0; j < K; ++j)
    out[j] = has ? r3dsimt::vmin2(mid[j], r3dsimt::vaddmin2(nb[j], p1x2, pen2)) + c2[j] + negmp : c2[j];
}

struct RangedPass {
  const SgmMatch* m;
  unsigned char* smem;
  int rows;
  int dir;
  int w, h, ndw;
  const int4* recs;     // {cell offset, lo | num << 16, P2 of H | V << 16, P2 of DB | DA << 16}, pass order
  const uint8_t* cost;  // packed per pixel, image order
  uint16_t* sa;         // forward partial sums (and the totals of wide pixels)
  int4* info;           // image order
  unsigned char* seam;  // two seam buffers
  int64_t seam_pix;
  uint16_t* wide;       // rows x 11 vectors of ndw labels
  uint32_t* rkeys;
  int64_t rk;
  const int* row_shift;
  int x0, y0;
  uint16_t* volume;
};

// Predecessors of band row rr's pixel uc (band-local row rr, tile row vv,
// ring slot index lc): H from the row itself (its previous pixel's range
// hl/hn and minimum hm), V, DB and DA from the row above, or from the seam
// for the band's first row.
template <int G, int K>
R3D_DEVICE void build_preds(const RangedPass& a, unsigned char* gseam_in, int rr, int uc, int lc, int vv, int hl,
                            int hn, uint32_t hm, Pred (&pr)[4], bool (&hasp)[4]) {
  const bool has_up = vv > 0;
  hasp[0] = uc > 0;
  hasp[1] = has_up;
  hasp[2] = has_up && uc > 0;
  hasp[3] = has_up && uc + 1 < a.w;
  const uint16_t* wide_r = a.wide + static_cast<int64_t>(rr) * kSgmRangedVecs * a.ndw;
  const int vh = vec_h(lc + 1);  // pixel uc - 1
  pr[0] = Pred{rvec<G, K>(a.smem, rr, vh), wide_r + vh * a.ndw, hl, hn, hm};
  if (rr > 0) {
    const int rup = rr - 1;
    const uint32_t* meta_up = rmeta<G, K>(a.smem, rup);
    const uint32_t* mins_up = rmins<G, K>(a.smem, rup);
    const uint16_t* wide_up = wide_r - static_cast<int64_t>(kSgmRangedVecs) * a.ndw;
    const int iv = vec_v(lc), idb = vec_db(lc + 3), ida = vec_da(lc + 1);
    const uint32_t mv = meta_up[lc & 3], mdb = meta_up[(lc + 3) & 3], mda = meta_up[(lc + 1) & 3];
    pr[1] = Pred{rvec<G, K>(a.smem, rup, iv), wide_up + iv * a.ndw, static_cast<int>(mv & 0xFFFFu),
                 static_cast<int>(mv >> 16), mins_up[iv]};
    pr[2] = Pred{rvec<G, K>(a.smem, rup, idb), wide_up + idb * a.ndw, static_cast<int>(mdb & 0xFFFFu),
                 static_cast<int>(mdb >> 16), mins_up[idb]};
    pr[3] = Pred{rvec<G, K>(a.smem, rup, ida), wide_up + ida * a.ndw, static_cast<int>(mda & 0xFFFFu),
                 static_cast<int>(mda >> 16), mins_up[ida]};
  } else {
    const int sv = lc & (kSgmSeamSlots - 1), sdb = (lc + kSgmSeamSlots - 1) & (kSgmSeamSlots - 1),
              sda = (lc + 1) & (kSgmSeamSlots - 1);
    const int ul = uc > 0 ? uc - 1 : 0, ur = uc + 1 < a.w ? uc + 1 : uc;
    const uint32_t* mv = seam_meta_s<G, K>(a.smem, a.rows, sv);
    const uint32_t* mdb = seam_meta_s<G, K>(a.smem, a.rows, sdb);
    const uint32_t* mda = seam_meta_s<G, K>(a.smem, a.rows, sda);
    pr[1] = Pred{seam_vec_s<G, K>(a.smem, a.rows, sv, 0), gseam_vec(gseam_in, a.seam_pix, uc, 0, a.ndw),
                 static_cast<int>(mv[3] & 0xFFFFu), static_cast<int>(mv[3] >> 16), mv[0]};
    pr[2] = Pred{seam_vec_s<G, K>(a.smem, a.rows, sdb, 1), gseam_vec(gseam_in, a.seam_pix, ul, 1, a.ndw),
                 static_cast<int>(mdb[3] & 0xFFFFu), static_cast<int>(mdb[3] >> 16), mdb[1]};
    pr[3] = Pred{seam_vec_s<G, K>(a.smem, a.rows, sda, 2), gseam_vec(gseam_in, a.seam_pix, ur, 2, a.ndw),
                 static_cast<int>(mda[3] & 0xFFFFu), static_cast<int>(mda[3] >> 16), mda[2]};
  }
}

R3D_DEVICE uint32_t warp_vmin2(uint32_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = r3dsimt::vmin2(v, r3dsimt::shfl_xor(v, o));
  return v;
}
R3D_DEVICE uint32_t warp_umin(uint32_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = r3dsimt::umin(v, r3dsimt::shfl_xor(v, o));
  return v;
}

template <int G, int K>
R3D_DEVICE void run_ranged_pass(const RangedPass& a) {
  using C = RangedCfg<G, K>;
  using S = RangedSmem<G, K>;
  constexpr int ND = C::ND;
  const int lane = static_cast<int>(threadIdx.x & 31u);
  const int warp = static_cast<int>(threadIdx.x >> 5);
  const int gi = lane / G;
  const int t = lane % G;
  const int r = warp * C::RPW + gi;
  const SgmMatch& m = *a.m;
  const uint32_t p1x2 = static_cast<uint32_t>(m.p1) * 0x10001u;
  const bool no_carry = m.sum_no_carry != 0;
  const int e0 = 2 * t * K;
  uint32_t* mins = rmins<G, K>(a.smem, r);
  uint32_t* meta = rmeta<G, K>(a.smem, r);
  uint8_t* cbuf = a.smem + S::rows_off + r * S::row_bytes + S::cbuf_off;
  uint16_t* sabuf = reinterpret_cast<uint16_t*>(a.smem + S::rows_off + r * S::row_bytes + S::sabuf_off);

  // Bands follow one another without a pause: band row r handles its local
  // step L (pixel u = L mod P of band L / P) at CTA step L + 2r, so the first
  // rows of band b + 1 start while the lower rows of band b finish. The period
  // P is at least the tile width and at least 2 rows + kSgmPF: the last row of
  // band b writes seam pixel u at step bP + u + 2(rows - 1), strictly before
  // the first row of band b + 1 prefetches it at step (b + 1)P + u - kSgmPF - 1.
  // Ring, prefetch and seam slots are indexed by L, which advances by one
  // across a band change, so consecutive steps never share a slot. The rows
  // of a warp can be in different bands, so wide pixels take their band from
  // the row that owns them.
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
    auto seam_buf = [&](int b) -> unsigned char* {
      return a.seam + static_cast<size_t>(b & 1) * a.w * a.seam_pix;
    };
    auto prefetch = [&](const Pos& p, const int4& rec) {
      if (!valid(p)) return;
      const int num = static_cast<int>(static_cast<uint32_t>(rec.y) >> 16);
      if (num > ND) return;  // wide pixels read global memory directly
      const int slot = p.L & (kSgmPFSlots - 1);
      for (int q = t; q < num / 16; q += G) r3dsimt::cp_async16(cbuf + slot * ND + 16 * q, a.cost + rec.x + 16 * q);
      if (a.dir < 0)
        for (int q = t; q < num / 8; q += G) r3dsimt::cp_async16(sabuf + slot * ND + 8 * q, a.sa + rec.x + 8 * q);
    };
    auto prefetch_seam = [&](const Pos& p) {
      if (r != 0 || p.b == 0 || !valid(p)) return;
      unsigned char* gseam_in = seam_buf(p.b + 1);
      const int s = p.L & (kSgmSeamSlots - 1);
      constexpr int pieces = ND / 8;
      for (int q = t; q < 3 * pieces + 1; q += G) {
        if (q < 3 * pieces) {
          const int path = q / pieces, k = q % pieces;
          r3dsimt::cp_async16(seam_vec_s<G, K>(a.smem, a.rows, s, path) + 8 * k,
                              gseam_vec(gseam_in, a.seam_pix, p.u, path, a.ndw) + 8 * k);
        } else {
          r3dsimt::cp_async16(seam_meta_s<G, K>(a.smem, a.rows, s), gseam_meta(gseam_in, a.seam_pix, p.u));
        }
      }
    };
    auto rec_at = [&](const Pos& p) -> int4 {
      return valid(p) ? a.recs[static_cast<int64_t>(p.b * R + r) * a.w + p.u] : make_int4(0, 0, 0, 0);
    };

    Pos cur{0, -2 * r, -2 * r};
    int4 q0 = rec_at(cur), q1 = rec_at(adv(cur, 1)), q2 = rec_at(adv(cur, 2));
    prefetch(cur, q0);
    prefetch_seam(cur);
    prefetch_seam(adv(cur, 1));
    r3dsimt::cp_async_commit();
    prefetch(adv(cur, 1), q1);
    prefetch_seam(adv(cur, 2));
    r3dsimt::cp_async_commit();

    uint32_t hmin = 0;  // range and minimum of the row's previous pixel
    int hlo = 0, hnum = 0;
    const int last_rows = a.h - (nb - 1) * R;
    int steps = (nb - 1) * P + a.w + 2 * (last_rows - 1);
    if (nb > 1) steps = r3dsimt::imax(steps, (nb - 2) * P + a.w + 2 * (R - 1));
    const int Lend = steps - 2 * r;  // this row's local step at the CTA's last step, plus one
    for (; cur.L < Lend; cur = adv(cur, 1)) {
      const int u = cur.u;
      const bool active = valid(cur);
      const int uc = u < 0 ? 0 : (u >= a.w ? a.w - 1 : u);
      const int v = r3dsimt::imin(cur.b * R + r, a.h - 1);  // clamped for addressing
      const int Lc = cur.L < 0 ? 0 : cur.L;                  // slot index
      const int yy = a.h - 1 - v;                            // image-order tile row (backward pass)
      const bool seam_out = active && r == R - 1 && (cur.b + 1) * R < a.h;
      unsigned char* gseam_in = seam_buf(cur.b + 1);
      unsigned char* gseam_out = seam_buf(cur.b);
      r3dsimt::cp_async_wait<kSgmPF - 1>();
      r3dsimt::syncthreads();
      const int4 rec = q0;
      const int off = rec.x;
      const int lo = rec.y & 0xFFFF;
      const int num = active ? static_cast<int>(static_cast<uint32_t>(rec.y) >> 16) : 0;
      const bool wide = num > ND;
      const int pslot = Lc & (kSgmPFSlots - 1);
      Pred pr[4];
      bool hasp[4];
      build_preds<G, K>(a, gseam_in, r, uc, Lc, v, hlo, hnum, hmin, pr, hasp);
      const uint32_t p2v[4] = {static_cast<uint32_t>(rec.z) & 0xFFFFu, static_cast<uint32_t>(rec.z) >> 16,
                               static_cast<uint32_t>(rec.w) & 0xFFFFu, static_cast<uint32_t>(rec.w) >> 16};
      const int ovec[4] = {vec_h(Lc), vec_v(Lc), vec_db(Lc), vec_da(Lc)};
      const int x = a.w - 1 - uc;  // image-order tile column (backward pass)
      bool lr_row = false;
      int lr_base = 0;
      if (a.dir < 0 && m.diagonal_lr) {
        const RowInterval lv = m.bv[a.y0 + yy];
        const int bx = a.x0 + x;
        lr_row = bx >= lv.first && bx <= lv.last;
        lr_base = x - lo + a.row_shift[yy];
      }

      // ---- Narrow pixels: all four paths first (loads only), then the stores.
      uint32_t pm[4];
      uint32_t sum[K];
#pragma unroll
      for (int j = 0; j < K; ++j) sum[j] = 0;
      uint32_t kmin = 0xFFFFFFFFu;
      {
        uint32_t c2[K];
        const uint8_t* cb = cbuf + pslot * ND + e0;
#pragma unroll
        for (int j = 0; j < K; ++j) {
          const uint32_t b = *reinterpret_cast<const uint16_t*>(cb + 2 * j);
          c2[j] = r3dsimt::perm(b, 0u, 0x4140u);
        }
        uint32_t out[4][K];
#pragma unroll
        for (int k = 0; k < 4; ++k) path_narrow<G, K>(pr[k], hasp[k] && !wide, p2v[k], lo, t, p1x2, c2, out[k]);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          uint32_t mk = kSent2;
#pragma unroll
          for (int j = 0; j < K; ++j) {
            if (e0 + 2 * j >= num) out[k][j] = kSent2;
            mk = r3dsimt::vmin2(mk, out[k][j]);
            sum[j] += out[k][j];
          }
          pm[k] = mk;
          if (active && !wide) {
            store_words<K>(reinterpret_cast<uint32_t*>(rvec<G, K>(a.smem, r, ovec[k])) + t * K, out[k]);
            if (k > 0 && seam_out)
              store_words<K>(reinterpret_cast<uint32_t*>(gseam_vec(gseam_out, a.seam_pix, uc, k - 1, a.ndw)) + t * K,
                             out[k]);
          }
        }
      }
      if (!wide) {
        if (a.dir > 0) {
          if (active) {
            uint32_t* sa32 = reinterpret_cast<uint32_t*>(a.sa + off) + t * K;
            if (e0 + 2 * K <= num) {
              store_words<K>(sa32, sum);
            } else {
#pragma unroll
              for (int j = 0; j < K; ++j)
                if (e0 + 2 * j < num) sa32[j] = sum[j];
            }
          }
        } else {
          uint32_t* keys = a.rkeys + static_cast<int64_t>(yy) * a.rk;
          const uint32_t* sb = reinterpret_cast<const uint32_t*>(sabuf + pslot * ND) + t * K;
#pragma unroll
          for (int j = 0; j < K; ++j) {
            sum[j] = no_carry ? sb[j] + sum[j] : r3dsimt::vadd2(sb[j], sum[j]);
            const int e = e0 + 2 * j;
            if (e < num) {
              const uint32_t ue = static_cast<uint32_t>(e);
              kmin = r3dsimt::umin(kmin, r3dsimt::umin(((sum[j] & 0xFFFFu) << 16) | ue, (sum[j] & 0xFFFF0000u) | (ue + 1)));
              if (a.volume != nullptr) reinterpret_cast<uint32_t*>(a.volume + off)[e >> 1] = sum[j];
              if (lr_row) {
                atomicMin(keys + (lr_base - e), ((sum[j] & 0xFFFFu) << 16) | static_cast<uint32_t>(x));
                atomicMin(keys + (lr_base - e - 1), (sum[j] & 0xFFFF0000u) | static_cast<uint32_t>(x));
              }
            }
          }
        }
      }

      // ---- Wide pixels: the whole warp takes the wide pixels of its rows one
      //      after the other, 2K labels per lane per chunk; loads come before
      //      the stores of a chunk. Results go to the row's own lanes.
      uint32_t wsec = 0xFFFFu, wsm = 0, wsp = 0;
      uint32_t wmask = r3dsimt::ballot(wide && t == 0);
      while (wmask != 0u) {
        const int src = r3dsimt::ffs(wmask) - 1;
        wmask &= wmask - 1u;
        const int gw = src / G;
        const int rw = warp * C::RPW + gw;
        const int ucw = static_cast<int>(r3dsimt::shfl(static_cast<uint32_t>(uc), src));
        const int lcw = static_cast<int>(r3dsimt::shfl(static_cast<uint32_t>(Lc), src));
        const int bw = static_cast<int>(r3dsimt::shfl(static_cast<uint32_t>(cur.b), src));
        const int offw = static_cast<int>(r3dsimt::shfl(static_cast<uint32_t>(off), src));
        const int low = static_cast<int>(r3dsimt::shfl(static_cast<uint32_t>(lo), src));
        const int numw = static_cast<int>(r3dsimt::shfl(static_cast<uint32_t>(num), src));
        const uint32_t recz = r3dsimt::shfl(static_cast<uint32_t>(rec.z), src);
        const uint32_t recw = r3dsimt::shfl(static_cast<uint32_t>(rec.w), src);
        const int hlw = static_cast<int>(r3dsimt::shfl(static_cast<uint32_t>(hlo), src));
        const int hnw = static_cast<int>(r3dsimt::shfl(static_cast<uint32_t>(hnum), src));
        const uint32_t hmw = r3dsimt::shfl(hmin, src);
        const int vw = bw * R + rw;
        Pred pw[4];
        bool hw[4];
        build_preds<G, K>(a, seam_buf(bw + 1), rw, ucw, lcw, vw, hlw, hnw, hmw, pw, hw);
        const bool seam_w = rw == R - 1 && (bw + 1) * R < a.h;
        unsigned char* gseam_out_w = seam_buf(bw);
        const int ovw[4] = {vec_h(lcw), vec_v(lcw), vec_db(lcw), vec_da(lcw)};
        uint16_t* wide_w = a.wide + static_cast<int64_t>(rw) * kSgmRangedVecs * a.ndw;
        const uint32_t p2w[4] = {recz & 0xFFFFu, recz >> 16, recw & 0xFFFFu, recw >> 16};
        uint32_t pen2[4], negmp[4], pmw[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const uint32_t pen = pw[k].qmin + p2w[k];
          pen2[k] = pen | (pen << 16);
          negmp[k] = 0u - (pw[k].qmin | (pw[k].qmin << 16));
          pmw[k] = kSent2;
        }
        const int yyw = a.h - 1 - vw, xw = a.w - 1 - ucw;
        bool lrw = false;
        int lrbw = 0;
        if (a.dir < 0 && m.diagonal_lr) {
          const RowInterval lv = m.bv[a.y0 + yyw];
          const int bx = a.x0 + xw;
          lrw = bx >= lv.first && bx <= lv.last;
          lrbw = xw - low + a.row_shift[yyw];
        }
        uint32_t* keysw = a.rkeys + static_cast<int64_t>(yyw) * a.rk;
        uint32_t* sa32 = reinterpret_cast<uint32_t*>(a.sa + offw);
        uint32_t kminw = 0xFFFFFFFFu;
        for (int i = 2 * K * lane; i < numw; i += 64 * K) {
          uint32_t cc[K], prev[K];
          uint32_t L[4][K];
#pragma unroll
          for (int j = 0; j < K; ++j) {
            const int e = i + 2 * j < numw ? i + 2 * j : i;
            cc[j] = r3dsimt::perm(*reinterpret_cast<const uint16_t*>(a.cost + offw + e), 0u, 0x4140u);
            prev[j] = a.dir < 0 ? __ldcg(sa32 + (e >> 1)) : 0u;
          }
#pragma unroll
          for (int k = 0; k < 4; ++k) {
#pragma unroll
            for (int j = 0; j < K; ++j) {
              uint32_t nb = 0, mid = 0;
              if (hw[k]) pred_pair<ND>(pw[k], i + 2 * j + low - pw[k].lo, nb, mid);
              L[k][j] = hw[k] ? r3dsimt::vmin2(mid, r3dsimt::vaddmin2(nb, p1x2, pen2[k])) + cc[j] + negmp[k] : cc[j];
            }
          }
#pragma unroll
          for (int j = 0; j < K; ++j) {
            const int e = i + 2 * j;
            if (e < numw) {
              uint32_t sw = 0;
#pragma unroll
              for (int k = 0; k < 4; ++k) {
                pmw[k] = r3dsimt::vmin2(pmw[k], L[k][j]);
                sw += L[k][j];
                reinterpret_cast<uint32_t*>(wide_w + ovw[k] * a.ndw)[e >> 1] = L[k][j];
                if (k > 0 && seam_w)
                  reinterpret_cast<uint32_t*>(gseam_vec(gseam_out_w, a.seam_pix, ucw, k - 1, a.ndw))[e >> 1] = L[k][j];
              }
              if (a.dir > 0) {
                sa32[e >> 1] = sw;
              } else {
                const uint32_t tot = no_carry ? prev[j] + sw : r3dsimt::vadd2(prev[j], sw);
                sa32[e >> 1] = tot;
                const uint32_t ue = static_cast<uint32_t>(e);
                kminw = r3dsimt::umin(kminw, r3dsimt::umin(((tot & 0xFFFFu) << 16) | ue, (tot & 0xFFFF0000u) | (ue + 1)));
                if (a.volume != nullptr) reinterpret_cast<uint32_t*>(a.volume + offw)[e >> 1] = tot;
                if (lrw) {
                  atomicMin(keysw + (lrbw - e), ((tot & 0xFFFFu) << 16) | static_cast<uint32_t>(xw));
                  atomicMin(keysw + (lrbw - e - 1), (tot & 0xFFFF0000u) | static_cast<uint32_t>(xw));
                }
              }
            }
          }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) pmw[k] = warp_vmin2(pmw[k]);
        uint32_t secw = 0xFFFFu, smw = 0, spw = 0;
        if (a.dir < 0) {
          kminw = warp_umin(kminw);
          r3dsimt::syncwarp();  // totals of the other lanes visible
          const int kb = static_cast<int>(kminw & 0xFFFFu);
          for (int i = 2 * K * lane; i < numw; i += 64 * K) {
#pragma unroll
            for (int j = 0; j < K; ++j) {
              const int e = i + 2 * j;
              if (e < numw) {
                const uint32_t tot = __ldcg(sa32 + (e >> 1));
                if (e + 1 < kb || e > kb + 1) secw = r3dsimt::umin(secw, tot & 0xFFFFu);
                if (e + 2 < kb || e + 1 > kb + 1) secw = r3dsimt::umin(secw, tot >> 16);
              }
            }
          }
          secw = warp_umin(secw);
          smw = __ldcg(a.sa + offw + (kb > 0 ? kb - 1 : 0));
          spw = __ldcg(a.sa + offw + (kb + 1 < numw ? kb + 1 : numw - 1));
        }
        if (gi == gw) {
#pragma unroll
          for (int k = 0; k < 4; ++k) pm[k] = pmw[k];
          kmin = kminw;
          wsec = secw;
          wsm = smw;
          wsp = spw;
        }
      }

      r3dsimt::syncwarp();
      uint32_t pmin[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) pmin[k] = r3dsimt::umin(pm[k] & 0xFFFFu, pm[k] >> 16);
      const uint32_t m01 = group_vmin2<G>(pmin[0] | (pmin[1] << 16));
      const uint32_t m23 = group_vmin2<G>(pmin[2] | (pmin[3] << 16));
      if (active) {
        hmin = m01 & 0xFFFFu;
        hlo = lo;
        hnum = num;
        if (t == 0) {
          mins[ovec[1]] = m01 >> 16;
          mins[ovec[2]] = m23 & 0xFFFFu;
          mins[ovec[3]] = m23 >> 16;
          meta[Lc & 3] = static_cast<uint32_t>(lo) | (static_cast<uint32_t>(num) << 16);
          if (seam_out) {
            uint32_t* gm = gseam_meta(gseam_out, a.seam_pix, uc);
            gm[0] = m01 >> 16;
            gm[1] = m23 & 0xFFFFu;
            gm[2] = m23 >> 16;
            gm[3] = static_cast<uint32_t>(lo) | (static_cast<uint32_t>(num) << 16);
          }
        }
      }
      if (a.dir < 0) {
        // Winner-takes-all: first minimum, second best outside +-1, S at kb -+ 1.
        kmin = group_umin<G>(kmin);
        const int kb = static_cast<int>(kmin & 0xFFFFu);
        const uint32_t bcost = kmin >> 16;
        uint32_t sec = 0xFFFFu;
        if (!wide) {
#pragma unroll
          for (int j = 0; j < K; ++j) {
            const int e = e0 + 2 * j;
            if (e < num) {
              if (e + 1 < kb || e > kb + 1) sec = r3dsimt::umin(sec, sum[j] & 0xFFFFu);
              if (e + 2 < kb || e + 1 > kb + 1) sec = r3dsimt::umin(sec, sum[j] >> 16);
            }
          }
        }
        sec = group_umin<G>(sec);
        const int km = kb > 0 ? kb - 1 : 0;
        const int kp = kb + 1 < num ? kb + 1 : (num > 0 ? num - 1 : 0);
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
        uint32_t sm = (km & 1) ? (vm >> 16) : (vm & 0xFFFFu);
        uint32_t sp = (kp & 1) ? (vp >> 16) : (vp & 0xFFFFu);
        if (wide) {
          sec = wsec;
          sm = wsm;
          sp = wsp;
        }
        if (active && t == 0) {
          a.info[static_cast<int64_t>(yy) * a.w + x] =
              make_int4(static_cast<int>(static_cast<uint32_t>(lo + kb) | (bcost << 16)),
                        static_cast<int>(sec | (sm << 16)), static_cast<int>(sp), 0);
        }
      }
      // Next prefetches and the record queue.
      prefetch(adv(cur, kSgmPF), q2);
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

R3D_DEVICE uint32_t warp_sum_excl(uint32_t v, uint32_t& total) {
  const int lane = static_cast<int>(r3dsimt::lane_id());
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = r3dsimt::shfl(x, lane - o < 0 ? lane : lane - o);
    if (lane >= o) x += y;
  }
  total = r3dsimt::shfl(x, 31);
  return x - v;
}

template <int G, int K>
R3D_GLOBAL void R3D_LAUNCH_BOUNDS((RangedCfg<G, K>::MAXT))
    sgm_ranged_kernel(const SgmMatch* R3D_RESTRICT matches, const SgmJob* R3D_RESTRICT jobs, int njobs, int rows,
                      int ndw, unsigned char* scratch, size_t slot_bytes, int* counter) {
  R3D_DYNAMIC_SMEM(smem);
  const int nthreads = static_cast<int>(blockDim.x);
  const int tid = static_cast<int>(threadIdx.x);
  const int warp = tid >> 5, lane = tid & 31;
  const int nwarps = nthreads >> 5;
  unsigned char* slot = scratch + static_cast<size_t>(blockIdx.x) * slot_bytes;
  int* job_id = reinterpret_cast<int*>(smem);

  // Sentinel pads between the shared vectors (never overwritten later):
  // 12 per row block, 4 per seam slot, kPad labels each.
  {
    const int npads = rows * (kSgmRangedVecs + 1) + kSgmSeamSlots * 4;
    for (int i = tid; i < npads * kPad; i += nthreads) {
      const int pi = i / kPad, k = i % kPad;
      uint16_t* pad;
      if (pi < rows * (kSgmRangedVecs + 1)) {
        pad = rvec<G, K>(smem, pi / (kSgmRangedVecs + 1), pi % (kSgmRangedVecs + 1)) - kPad;
      } else {
        const int q = pi - rows * (kSgmRangedVecs + 1);
        pad = seam_vec_s<G, K>(smem, rows, q / 4, q % 4) - kPad;
      }
      pad[k] = static_cast<uint16_t>(kSent);
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
    const int w = job.w, h = job.h;
    const int64_t npx = static_cast<int64_t>(w) * h;
    // ---- P1: per row, label ranges, in-row offsets, totals and the
    //          right-WTA shift (max of lo + num - 1 - x). The cell-sized
    //          arrays of the layout are placed once the cell count is known.
    SgmRangedSlot L = sgm_ranged_slot_layout(w, h, 0ull, m.nd, ndw, rows);
    int4* rec_a = reinterpret_cast<int4*>(slot + L.rec_a);
    int4* rec_b = reinterpret_cast<int4*>(slot + L.rec_b);
    int4* info = reinterpret_cast<int4*>(slot + L.info);
    uint32_t* row_start = reinterpret_cast<uint32_t*>(slot + L.row_start);
    int* row_shift = reinterpret_cast<int*>(slot + L.row_shift);
    for (int y = warp; y < h; y += nwarps) {
      const int by = job.y0 + y;
      uint32_t run = 0;
      int shift = -0x7FFFFFFF;
      for (int xb = 0; xb < w; xb += 32) {
        const int x = xb + lane;
        int lo = 0, num = 0;
        if (x < w) {
          if (m.rlo != nullptr) {
            lo = m.rlo[static_cast<int64_t>(by) * m.r_stride + job.x0 + x];
            num = m.rnum[static_cast<int64_t>(by) * m.r_stride + job.x0 + x];
          } else {
            num = m.nd;
          }
          shift = r3dsimt::imax(shift, lo + num - 1 - x);
        }
        uint32_t total = 0;
        const uint32_t excl = warp_sum_excl(static_cast<uint32_t>(num), total);
        if (x < w)
          rec_a[static_cast<int64_t>(y) * w + x] = make_int4(static_cast<int>(run + excl), lo | (num << 16), 0, 0);
        run += total;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
        shift = r3dsimt::imax(shift, static_cast<int>(r3dsimt::shfl_xor(static_cast<uint32_t>(shift), o)));
      if (lane == 0) {
        row_start[y + 1] = run;
        row_shift[y] = shift;
      }
    }
    r3dsimt::syncthreads();
    // ---- P2: row starts.
    if (warp == 0) {
      uint32_t carry = 0;
      for (int yb = 0; yb < h; yb += 32) {
        const int y = yb + lane;
        const uint32_t tv = y < h ? row_start[y + 1] : 0u;
        uint32_t total = 0;
        const uint32_t excl = warp_sum_excl(tv, total);
        if (y < h) row_start[y + 1] = carry + excl + tv;
        carry += total;
      }
      if (lane == 0) row_start[0] = 0;
    }
    r3dsimt::syncthreads();
    const unsigned long long cells = row_start[h];
    L = sgm_ranged_slot_layout(w, h, cells, m.nd, ndw, rows);
    uint8_t* cost = slot + L.cost;
    uint16_t* sa = reinterpret_cast<uint16_t*>(slot + L.sa);
    unsigned char* seam = slot + L.seam;
    uint16_t* wide = reinterpret_cast<uint16_t*>(slot + L.wide);
    uint32_t* rkeys = reinterpret_cast<uint32_t*>(slot + L.rkeys);

    // ---- P3: records of both passes (cell offset, range, P2 of the 4 paths).
    const uint16_t* img = m.base;
    const int64_t ist = m.base_stride;
    for (int64_t i = tid; i < npx; i += nthreads) {
      const int y = static_cast<int>(i / w), x = static_cast<int>(i - static_cast<int64_t>(y) * w);
      const int4 r0 = rec_a[i];
      const int off = static_cast<int>(row_start[y] + static_cast<uint32_t>(r0.x));
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
      rec_a[i] = make_int4(off, r0.y, static_cast<int>(aH | (aV << 16)), static_cast<int>(aDB | (aDA << 16)));
      rec_b[static_cast<int64_t>(h - 1 - y) * w + (w - 1 - x)] =
          make_int4(off, r0.y, static_cast<int>(bH | (bV << 16)), static_cast<int>(bDB | (bDA << 16)));
    }
    if (m.diagonal_lr) {
      const int64_t nk = static_cast<int64_t>(h) * L.rk;
      for (int64_t i = tid; i < nk; i += nthreads) rkeys[i] = 0xFFFFFFFFu;
    }
    r3dsimt::syncthreads();

    // ---- P4: Hamming costs, one lane per pixel, 16 labels per store.
    for (int y = warp; y < h; y += nwarps) {
      const int by = job.y0 + y;
      const RowInterval lv = m.bv[by], rv = m.pv[by];
      const uint64_t* crow = m.cpart + static_cast<int64_t>(by) * m.cp_stride;
      const uint64_t* lrow = m.cbase + static_cast<int64_t>(by) * m.cb_stride;
      const int safe = rv.first > 0 ? rv.first : 0;
      for (int x = lane; x < w; x += 32) {
        const int4 rc = rec_a[static_cast<int64_t>(y) * w + x];
        const int lo = rc.y & 0xFFFF, num = static_cast<int>(static_cast<uint32_t>(rc.y) >> 16);
        const int bx = job.x0 + x;
        const bool inside = bx >= lv.first && bx <= lv.last;
        const uint64_t cl = inside ? lrow[bx] : 0ull;
        for (int k0 = 0; k0 < num; k0 += 16) {
          uint32_t wd[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            uint32_t word = 0;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
              const int xr = bx - m.dmin - (lo + k0 + 4 * q + b);
              const bool ok = xr >= rv.first && xr <= rv.last;
              const uint64_t cr = crow[ok ? xr : safe];
              const uint32_t c = !inside ? 0u
                                         : (ok ? static_cast<uint32_t>(r3dsimt::popc64(cl ^ cr))
                                               : static_cast<uint32_t>(m.invalid_cost));
              word |= c << (8 * b);
            }
            wd[q] = word;
          }
          *reinterpret_cast<uint4*>(cost + rc.x + k0) = make_uint4(wd[0], wd[1], wd[2], wd[3]);
        }
      }
    }
    r3dsimt::fence();
    r3dsimt::syncthreads();

    // ---- Passes.
    RangedPass pa;
    pa.m = &m;
    pa.smem = smem;
    pa.rows = rows;
    pa.w = w;
    pa.h = h;
    pa.ndw = ndw;
    pa.cost = cost;
    pa.sa = sa;
    pa.info = info;
    pa.seam = seam;
    pa.seam_pix = L.seam_pix;
    pa.wide = wide;
    pa.rkeys = rkeys;
    pa.rk = L.rk;
    pa.row_shift = row_shift;
    pa.x0 = job.x0;
    pa.y0 = job.y0;
    pa.volume = job.volume;
    pa.dir = 1;
    pa.recs = rec_a;
    run_ranged_pass<G, K>(pa);
    pa.dir = -1;
    pa.recs = rec_b;
    run_ranged_pass<G, K>(pa);

    // ---- Acceptance rules and outputs (stereo_matcher.cpp:474-523).
    for (int64_t i = tid; i < npx; i += nthreads) {
      const int y = static_cast<int>(i / w), x = static_cast<int>(i - static_cast<int64_t>(y) * w);
      const int bx = job.x0 + x, by = job.y0 + y;
      const RowInterval lv = m.bv[by];
      float d = kInfF, cf = 0.0F;
      if (bx >= lv.first && bx <= lv.last) {
        const int4 in = info[i];
        const int4 rc = rec_a[i];
        const int lo = rc.y & 0xFFFF, num = static_cast<int>(static_cast<uint32_t>(rc.y) >> 16);
        const int best = in.x & 0xFFFF;
        const uint32_t bcost = static_cast<uint32_t>(in.x) >> 16;
        const uint32_t sec = static_cast<uint32_t>(in.y) & 0xFFFFu;
        const uint32_t sm = static_cast<uint32_t>(in.y) >> 16;
        const uint32_t sp = static_cast<uint32_t>(in.z);
        const int j = best - lo;
        const RowInterval rv = m.pv[by];
        const int xr = bx - m.dmin - best;
        bool ok = xr >= rv.first && xr <= rv.last;
        if ((j == 0 && lo > 0) || (j == num - 1 && lo + num < m.nd)) ok = false;
        if (ok && m.diagonal_lr) {
          const uint32_t key = rkeys[static_cast<int64_t>(y) * L.rk + (x - best + row_shift[y])];
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
          if (j > 0 && j < num - 1)
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

template <int G, int K>
void launch_ranged_instance(const SgmMatch* dm, const SgmJob* dj, int njobs, int rows, int ndw, int grid,
                            unsigned char* scratch, size_t slot_bytes, int* counter, cudaStream_t s) {
  using S = RangedSmem<G, K>;
  const size_t smem = static_cast<size_t>(S::total(rows));
  static thread_local int configured[64] = {};
  int dev = 0;
  R3D_CUDA(cudaGetDevice(&dev));
  auto* kernel = sgm_ranged_kernel<G, K>;
  if (dev >= 0 && dev < 64 && configured[dev] < static_cast<int>(smem)) {
    R3D_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    configured[dev] = static_cast<int>(smem);
  }
  const int threads = rows / RangedCfg<G, K>::RPW * 32;
  R3D_LAUNCH(kernel, dim3(grid), dim3(threads), smem, s, dm, dj, njobs, rows, ndw, scratch, slot_bytes, counter);
  launched("sgm_ranged_kernel");
}

// Shapes compiled into the library (lanes per row G, label pairs per lane K).
#define R3D_RANGED_SHAPES(X) \
  X(4, 4)                    \
  X(8, 4)                    \
  X(8, 8)                    \
  X(8, 12)                   \
  X(16, 8)                   \
  X(16, 12)                  \
  X(32, 8)                   \
  X(32, 12)

bool ranged_shape_compiled(SgmRangedShape sh) {
#define R3D_SHAPE(g, k) \
  if (sh.g_ == g && sh.k_ == k) return true;
  R3D_RANGED_SHAPES(R3D_SHAPE)
#undef R3D_SHAPE
  return false;
}

}  // namespace

int sgm_ranged_smem(SgmRangedShape sh, int rows) {
#define R3D_SHAPE(g, k) \
  if (sh.g_ == g && sh.k_ == k) return RangedSmem<g, k>::total(rows);
  R3D_RANGED_SHAPES(R3D_SHAPE)
#undef R3D_SHAPE
  fail(R3DGPU_EINVAL, "stereo: bad ranged kernel shape");
}

namespace {

// Label widths of the compiled shapes, narrowest first.
constexpr int kRangedWidths[] = {32, 64, 128, 192, 256, 384, 512, 768};
constexpr SgmRangedShape kRangedShapes[] = {{4, 4}, {8, 4}, {8, 8}, {8, 12}, {16, 8}, {16, 12}, {32, 8}, {32, 12}};

}  // namespace

int sgm_ranged_width_for(const int* stats, int64_t pixels) {
  if (const char* e = std::getenv("R3DGPU_RANGED_SHAPE")) {
    int g = 0, k = 0;
    if (std::sscanf(e, "%d,%d", &g, &k) == 2 && ranged_shape_compiled({g, k})) return 2 * g * k;
  }
  double frac = tuning().ranged_wide_frac >= 0.0 ? tuning().ranged_wide_frac : 0.002;
  if (const char* e = std::getenv("R3DGPU_RANGED_WIDE_FRAC")) frac = std::atof(e);
  const double allowed = frac * static_cast<double>(pixels);
  // stats[1 + i]: pixels with more labels than tile_stat_width(i).
  for (int i = 0; i < kTileStats - 1; ++i)
    if (kRangedWidths[i] == tile_stat_width(i) && static_cast<double>(stats[1 + i]) <= allowed) return kRangedWidths[i];
  return kRangedWidths[kTileStats - 1];
}

SgmRangedShape sgm_ranged_shape_for_width(int width) {
  for (int i = 0; i < kTileStats; ++i)
    if (kRangedWidths[i] == width) return kRangedShapes[i];
  fail(R3DGPU_EINVAL, "stereo: no ranged kernel shape for width " + std::to_string(width));
}

SgmRangedPlan sgm_ranged_plan(SgmRangedShape shape, int smem_optin) {
  SgmRangedPlan p{shape, 32};
  {
    const auto it = tuning().ranged_rows.find(2 * shape.g_ * shape.k_);
    if (it != tuning().ranged_rows.end()) p.rows = it->second;
  }
  const int rpw = 32 / p.shape.g_;
  const int max_rows = (p.shape.k_ >= 8 ? 256 : kSgmRangedThreads) / 32 * rpw;
  if (const char* e = std::getenv("R3DGPU_RANGED_ROWS")) p.rows = std::atoi(e);
  p.rows = std::max(rpw, std::min(p.rows, max_rows)) / rpw * rpw;
  while (p.rows > rpw && sgm_ranged_smem(p.shape, p.rows) > smem_optin) p.rows -= rpw;
  if (sgm_ranged_smem(p.shape, p.rows) > smem_optin)
    fail(R3DGPU_EUNSUPPORTED, "stereo: ranged kernel needs more shared memory than the device has");
  return p;
}

int sgm_ranged_ndw(SgmRangedShape sh, int max_num) {
  const int nd = 2 * sh.g_ * sh.k_;
  return std::max(nd, (max_num + 15) / 16 * 16);
}

void launch_sgm_ranged(SgmRangedShape sh, const SgmMatch* dm, const SgmJob* dj, int njobs, int rows, int ndw,
                       int grid, unsigned char* scratch, size_t slot_bytes, int* counter, cudaStream_t s) {
#define R3D_SHAPE(g, k)                                                                             \
  if (sh.g_ == g && sh.k_ == k) {                                                                   \
    launch_ranged_instance<g, k>(dm, dj, njobs, rows, ndw, grid, scratch, slot_bytes, counter, s); \
    return;                                                                                         \
  }
  R3D_RANGED_SHAPES(R3D_SHAPE)
#undef R3D_SHAPE
  fail(R3DGPU_EINVAL, "stereo: bad ranged kernel shape");
}

}  // namespace r3dgpu
