// SGM tile kernel: one persistent launch processes a table of tile jobs (tiles
// of one or many matches, pairs and levels). A CTA takes a job, computes its
// per-pixel records and Hamming costs, runs the forward pass (paths from the
// left, top, top-left and top-right predecessors) and the backward pass (the
// mirrored four paths) and finally the winner-takes-all with the reference's
// acceptance rules, writing the tile's disparity and confidence.
//
// Semantics (rhiestan/Regard3D_MVS src/r3d/stereo/):
//   C(p, a)  = popcount(census_left(p) ^ census_right(x - dmin - a)), or
//              invalid_cost outside the row's valid right columns, or 0 for
//              every label of a left pixel outside the valid left columns
//              (stereo_matcher.cpp:305-353);
//   L(p, a)  = C(p, a) + min(Lq(a), Lq(a -+ 1) + P1, min_k Lq(k) + P2) - min_k Lq(k)
//              per path, Lq infinite outside q's range, L = C without a
//              predecessor inside the tile (sgm_kernels.cpp:176-263, 387-403);
//   S(p, a)  = sum of the 8 paths modulo 2^16;
//   WTA      = first minimum, second best outside +-1, subpixel fit and the
//              acceptance rules of stereo_matcher.cpp:446-525.
// Because S is a sum, each path is an independent 1-D recurrence; only the
// data layout below is this implementation's own.
//
// Layout. A band of R tile rows is processed by R warps, warp r owning row r
// and walking it one pixel per step, two pixels behind the warp above (pixel
// u of row r at step u + 2r), so that its vertical and diagonal predecessors
// have been produced one to three steps earlier. Every pixel's 4 path vectors
// go to shared-memory rings of its row (depths 2, 3, 4 and 2: the ages at
// which they are read); the last row of a band also writes them to a global
// seam that the first row of the next band streams back with cp.async. Labels
// are packed two per 32-bit register (lane l holds labels 64c + 2l, 2l + 1 of
// chunk c) and updated with 16x2 SIMD min instructions. A label outside the
// pixel's range is stored as 0x7FFF, which never wins against the P2 term
// (at most 16257), so no saturating arithmetic is needed and every value
// stays exact. Costs (u8) and forward partial sums (u16) live in the CTA's
// global scratch slot and are prefetched two pixels ahead with cp.async.
#include "common.cuh"
#include "sgm.h"

namespace r3dgpu {

namespace {

constexpr uint32_t kSent = 0x7FFFu;
constexpr uint32_t kSent2 = 0x7FFF7FFFu;
constexpr float kInfF = __builtin_huge_valf();

// Shared-memory views of one row block. The 11 path vectors of a row are
// consecutive: H (2 slots), V (3), DB (4), DA (2).
struct RowView {
  uint16_t* ring;  // payload index 0 of vector 0
  int vst;
  uint32_t* mins;  // [0..1] H, [2..4] V, [5..8] DB, [9..10] DA
  uint32_t* meta;  // [4]: lo | num << 16 of the pixel produced at u % 4
  uint8_t* cbuf;   // [kSgmPFSlots][64 * maxc]
  uint16_t* sabuf; // [kSgmPFSlots][64 * maxc]
  R3D_DEVICE uint16_t* vec(int i) const { return ring + i * vst; }
  R3D_DEVICE uint16_t* H(int s) const { return vec(s); }
  R3D_DEVICE uint16_t* V(int s) const { return vec(2 + s); }
  R3D_DEVICE uint16_t* DB(int s) const { return vec(5 + s); }
  R3D_DEVICE uint16_t* DA(int s) const { return vec(9 + s); }
};

R3D_DEVICE RowView row_view(unsigned char* smem, const SgmSmemLayout& L, int r) {
  unsigned char* b = smem + L.rows_off + r * L.row_bytes;
  RowView v;
  v.ring = reinterpret_cast<uint16_t*>(b + L.ring_off) + 8;
  v.vst = L.vst;
  v.mins = reinterpret_cast<uint32_t*>(b + L.mins_off);
  v.meta = reinterpret_cast<uint32_t*>(b + L.meta_off);
  v.cbuf = b + L.cbuf_off;
  v.sabuf = reinterpret_cast<uint16_t*>(b + L.sabuf_off);
  return v;
}

// Seam slot s: 3 vectors (V, DB, DA), then meta {minV, minDB, minDA, lo | num << 16}.
R3D_DEVICE uint16_t* seam_vec(unsigned char* smem, const SgmSmemLayout& L, int s, int path) {
  return reinterpret_cast<uint16_t*>(smem + L.seam_off + s * L.seam_slot_bytes) + path * L.vst + 8;
}
R3D_DEVICE uint32_t* seam_meta(unsigned char* smem, const SgmSmemLayout& L, int s) {
  return reinterpret_cast<uint32_t*>(smem + L.seam_off + s * L.seam_slot_bytes + 3 * 2 * L.vst);
}

// Global seam pixel u: 3 vectors of 64 * maxc + 8 labels, then the meta.
R3D_DEVICE uint16_t* gseam_vec(unsigned char* seam, int64_t pix_bytes, int u, int path, int maxc) {
  return reinterpret_cast<uint16_t*>(seam + u * pix_bytes) + path * (64 * maxc + 8);
}
R3D_DEVICE uint32_t* gseam_meta(unsigned char* seam, int64_t pix_bytes, int u, int maxc) {
  return reinterpret_cast<uint32_t*>(seam + u * pix_bytes + 3 * (128 * maxc + 16));
}

R3D_DEVICE uint32_t warp_min_u32(uint32_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = r3dsimt::umin(v, r3dsimt::shfl_xor(v, o));
  return v;
}

R3D_DEVICE uint32_t warp_vmin2(uint32_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = r3dsimt::vmin2(v, r3dsimt::shfl_xor(v, o));
  return v;
}

R3D_DEVICE uint32_t warp_sum_excl(uint32_t v, uint32_t& total) {
  // Inclusive scan by shuffles, then exclusive.
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

// Path input: predecessor vector (payload index 0), its range and minimum.
struct PathIn {
  const uint16_t* q;
  int qlo, qnum;
  uint32_t qmin;
  uint32_t p2;
  bool has;
};

// Packed q values at labels (e - 1, e), (e, e + 1), (e + 1, e + 2) of the
// current pixel, e = 64c + 2 * lane, for a predecessor whose range differs.
R3D_DEVICE void read_shifted(const PathIn& in, int e, int shift, uint32_t& minus, uint32_t& mid, uint32_t& plus) {
  const int i = e + shift;
  auto rd = [&](int idx) -> uint32_t {
    return static_cast<unsigned>(idx) < static_cast<unsigned>(in.qnum) ? static_cast<uint32_t>(in.q[idx]) : kSent;
  };
  const uint32_t a = rd(i - 1), b = rd(i), c = rd(i + 1), d = rd(i + 2);
  minus = a | (b << 16);
  mid = b | (c << 16);
  plus = c | (d << 16);
}

template <int MAXC>
struct PassArgs {
  const SgmMatch* m;
  unsigned char* smem;
  SgmSmemLayout sl;
  int dir;
  int w, h, rows;
  const int4* recs;      // pass-local order
  const uint8_t* cost;   // global scratch
  uint16_t* sa;          // global scratch (forward partial sums)
  int4* info;            // WTA per pixel (image order)
  unsigned char* seam;   // two seam buffers
  int64_t seam_pix_bytes;
  uint32_t* rkeys;
  int64_t rk;
  const int* row_shift;
  int x0, y0;
  uint16_t* volume;  // optional full-volume output (backward pass)
};

// Issues the cp.async copies of pixel u of a row (costs, and forward partial
// sums in the backward pass) into prefetch slot u % kSgmPFSlots.
template <int MAXC>
R3D_DEVICE void prefetch_pixel(const PassArgs<MAXC>& a, const RowView& me, int u, const int4& rec, int lane) {
  if (u >= a.w) return;
  const int off = rec.x;
  const int num = rec.y >> 16;
  const int slot = u & (kSgmPFSlots - 1);
  uint8_t* cdst = me.cbuf + slot * 64 * MAXC;
  const uint8_t* csrc = a.cost + off;
  for (int p = lane; p < num / 16; p += 32) r3dsimt::cp_async16(cdst + 16 * p, csrc + 16 * p);
  if (a.dir < 0) {
    uint16_t* sdst = me.sabuf + slot * 64 * MAXC;
    const uint16_t* ssrc = a.sa + off;
    for (int p = lane; p < num / 8; p += 32) r3dsimt::cp_async16(sdst + 8 * p, ssrc + 8 * p);
  }
}

// Issues the copies of seam pixel u (the previous band's last row): the
// three full-length vectors (payload and tail) and the meta. Fixed size, so
// that no load has to complete before the copies are issued.
template <int MAXC>
R3D_DEVICE void prefetch_seam(const PassArgs<MAXC>& a, const unsigned char* gseam, int u, int lane) {
  if (u >= a.w) return;
  const int s = u & (kSgmSeamSlots - 1);
  constexpr int pieces = 8 * MAXC + 1;  // 64 * MAXC + 8 labels in 16-byte pieces
  unsigned char* g = const_cast<unsigned char*>(gseam);
  for (int p = lane; p < 3 * pieces + 1; p += 32) {
    if (p < 3 * pieces) {
      const int path = p / pieces, k = p % pieces;
      r3dsimt::cp_async16(seam_vec(a.smem, a.sl, s, path) + 8 * k, gseam_vec(g, a.seam_pix_bytes, u, path, MAXC) + 8 * k);
    } else {
      r3dsimt::cp_async16(seam_meta(a.smem, a.sl, s), gseam_meta(g, a.seam_pix_bytes, u, MAXC));
    }
  }
}

// One pass over the tile (dir = +1 forward, -1 backward), band by band.
template <int MAXC>
R3D_DEVICE void run_pass(const PassArgs<MAXC>& a) {
  const int warp = static_cast<int>(threadIdx.x >> 5);
  const int lane = static_cast<int>(threadIdx.x & 31u);
  const SgmMatch& m = *a.m;
  const uint32_t p1x2 = static_cast<uint32_t>(m.p1) * 0x10001u;
  const RowView me = row_view(a.smem, a.sl, warp);
  const RowView up = row_view(a.smem, a.sl, warp > 0 ? warp - 1 : 0);
  int band = 0;
  for (int v0 = 0; v0 < a.h; v0 += a.rows, ++band) {
    const int Rb = r3dsimt::imin(a.rows, a.h - v0);
    const int r = warp;
    const bool in_band = r < Rb;
    const int v = v0 + r;
    const bool seam_in = in_band && r == 0 && v0 > 0;
    const bool seam_out = in_band && r == Rb - 1 && v0 + Rb < a.h;
    const unsigned char* gseam_in = a.seam + static_cast<size_t>((band + 1) & 1) * a.w * a.seam_pix_bytes;
    unsigned char* gseam_out = a.seam + static_cast<size_t>(band & 1) * a.w * a.seam_pix_bytes;
    const int4* rrow = a.recs + static_cast<int64_t>(v) * a.w;

    int4 q[kSgmQueue];
    if (in_band) {
#pragma unroll
      for (int i = 0; i < kSgmQueue; ++i) q[i] = i < a.w ? rrow[i] : make_int4(0, 0, 0, 0);
#pragma unroll
      for (int g = 0; g < kSgmPF; ++g) {
        prefetch_pixel<MAXC>(a, me, g, q[g], lane);
        if (seam_in) {
          if (g == 0) prefetch_seam<MAXC>(a, gseam_in, 0, lane);
          prefetch_seam<MAXC>(a, gseam_in, g + 1, lane);
        }
        r3dsimt::cp_async_commit();
      }
    }
    const int steps = a.w + 2 * (Rb - 1);
    for (int t = 0; t < steps; ++t) {
      const int u = t - 2 * r;
      const bool active = in_band && u >= 0 && u < a.w;
      if (active) r3dsimt::cp_async_wait<kSgmPF - 1>();
      r3dsimt::syncthreads();
      if (active) {
        const int4 rec = q[0];
        const int off = rec.x;
        const int lo = rec.y & 0xFFFF;
        const int num = static_cast<int>(static_cast<uint32_t>(rec.y) >> 16);
        const int nc = (num + 63) >> 6;
        const bool has_up = v > 0;

        // Predecessors: H = own pixel u-1; V / DB / DA = row above (or the
        // seam) at pixels u, u-1, u+1.
        PathIn pin[4];
        pin[0].has = u > 0;
        pin[1].has = has_up;
        pin[2].has = has_up && u > 0;
        pin[3].has = has_up && u + 1 < a.w;
        pin[0].p2 = static_cast<uint32_t>(rec.z) & 0xFFFFu;
        pin[1].p2 = static_cast<uint32_t>(rec.z) >> 16;
        pin[2].p2 = static_cast<uint32_t>(rec.w) & 0xFFFFu;
        pin[3].p2 = static_cast<uint32_t>(rec.w) >> 16;
        {
          const int um1 = (u + 3) & 3;  // (u - 1) mod 4 for u >= 0
          pin[0].q = me.H((u + 1) & 1);
          pin[0].qmin = me.mins[(u + 1) & 1];
          const uint32_t mt = me.meta[um1];
          pin[0].qlo = static_cast<int>(mt & 0xFFFFu);
          pin[0].qnum = static_cast<int>(mt >> 16);
        }
        if (r > 0) {
          const int u3 = u % 3;
          pin[1].q = up.V(u3);
          pin[1].qmin = up.mins[2 + u3];
          const uint32_t m1 = up.meta[u & 3];
          pin[1].qlo = static_cast<int>(m1 & 0xFFFFu);
          pin[1].qnum = static_cast<int>(m1 >> 16);
          const int udb = (u + 3) & 3;
          pin[2].q = up.DB(udb);
          pin[2].qmin = up.mins[5 + udb];
          const uint32_t m2 = up.meta[udb];
          pin[2].qlo = static_cast<int>(m2 & 0xFFFFu);
          pin[2].qnum = static_cast<int>(m2 >> 16);
          const int uda = (u + 1) & 1;
          pin[3].q = up.DA(uda);
          pin[3].qmin = up.mins[9 + uda];
          const uint32_t m3 = up.meta[(u + 1) & 3];
          pin[3].qlo = static_cast<int>(m3 & 0xFFFFu);
          pin[3].qnum = static_cast<int>(m3 >> 16);
        } else {
          const int sV = u & (kSgmSeamSlots - 1), sDB = (u + kSgmSeamSlots - 1) & (kSgmSeamSlots - 1),
                    sDA = (u + 1) & (kSgmSeamSlots - 1);
          const uint32_t* mV = seam_meta(a.smem, a.sl, sV);
          const uint32_t* mDB = seam_meta(a.smem, a.sl, sDB);
          const uint32_t* mDA = seam_meta(a.smem, a.sl, sDA);
          pin[1].q = seam_vec(a.smem, a.sl, sV, 0);
          pin[1].qmin = mV[0];
          pin[1].qlo = static_cast<int>(mV[3] & 0xFFFFu);
          pin[1].qnum = static_cast<int>(mV[3] >> 16);
          pin[2].q = seam_vec(a.smem, a.sl, sDB, 1);
          pin[2].qmin = mDB[1];
          pin[2].qlo = static_cast<int>(mDB[3] & 0xFFFFu);
          pin[2].qnum = static_cast<int>(mDB[3] >> 16);
          pin[3].q = seam_vec(a.smem, a.sl, sDA, 2);
          pin[3].qmin = mDA[2];
          pin[3].qlo = static_cast<int>(mDA[3] & 0xFFFFu);
          pin[3].qnum = static_cast<int>(mDA[3] >> 16);
        }

        // Output vectors of this pixel.
        const int ovec[4] = {u & 1, 2 + u % 3, 5 + (u & 3), 9 + (u & 1)};
        const int pslot = u & (kSgmPFSlots - 1);
        const uint8_t* cb = me.cbuf + pslot * 64 * MAXC;

        uint32_t c2[MAXC];
        uint32_t sum[MAXC];
#pragma unroll
        for (int c = 0; c < MAXC; ++c) {
          sum[c] = 0;
          c2[c] = 0;
          if (c < nc) {
            const uint32_t b = *reinterpret_cast<const uint16_t*>(cb + 64 * c + 2 * lane);
            c2[c] = r3dsimt::perm(b, 0u, 0x4140u);
          }
        }
        uint32_t pmin[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const PathIn& in = pin[k];
          uint32_t* o32 = reinterpret_cast<uint32_t*>(me.vec(ovec[k]));
          uint32_t mk = kSent2;
          uint32_t* g32 = nullptr;
          if (seam_out && k > 0)
            g32 = reinterpret_cast<uint32_t*>(gseam_vec(gseam_out, a.seam_pix_bytes, u, k - 1, MAXC));
          if (!in.has) {
#pragma unroll
            for (int c = 0; c < MAXC; ++c) {
              if (c < nc) {
                const int e = 64 * c + 2 * lane;
                const uint32_t L = e < num ? c2[c] : kSent2;
                o32[e >> 1] = L;
                if (g32) g32[e >> 1] = L;
                mk = r3dsimt::vmin2(mk, L);
                sum[c] += L;
              }
            }
          } else {
            const uint32_t pen = in.qmin + in.p2;
            const uint32_t pen2 = pen | (pen << 16);
            const uint32_t negmp = 0u - (in.qmin | (in.qmin << 16));
            const bool fast = in.qlo == lo && in.qnum == num;
            const uint32_t* q32 = reinterpret_cast<const uint32_t*>(in.q);
            const int shift = lo - in.qlo;
#pragma unroll
            for (int c = 0; c < MAXC; ++c) {
              if (c < nc) {
                const int e = 64 * c + 2 * lane;
                uint32_t minus, mid, plus;
                if (fast) {
                  const uint32_t wlo = q32[(e >> 1) - 1], wmid = q32[e >> 1], whi = q32[(e >> 1) + 1];
                  minus = r3dsimt::perm(wlo, wmid, 0x5432u);
                  mid = wmid;
                  plus = r3dsimt::perm(wmid, whi, 0x5432u);
                } else {
                  read_shifted(in, e, shift, minus, mid, plus);
                }
                const uint32_t nb = r3dsimt::vmin2(minus, plus);
                const uint32_t tpen = r3dsimt::vmin2(nb + p1x2, pen2);
                const uint32_t best = r3dsimt::vmin2(mid, tpen);
                uint32_t L = best + c2[c] + negmp;
                if (e >= num) L = kSent2;
                o32[e >> 1] = L;
                if (g32) g32[e >> 1] = L;
                mk = r3dsimt::vmin2(mk, L);
                sum[c] += L;
              }
            }
          }
          if (nc < MAXC && lane < 4) {
            o32[32 * nc + lane] = kSent2;  // labels 64nc .. 64nc + 7
            if (g32) g32[32 * nc + lane] = kSent2;
          }
          if (nc == MAXC && g32 && lane < 4) g32[32 * MAXC + lane] = kSent2;
          pmin[k] = r3dsimt::umin(mk & 0xFFFFu, mk >> 16);
        }
        const uint32_t m01 = warp_vmin2(pmin[0] | (pmin[1] << 16));
        const uint32_t m23 = warp_vmin2(pmin[2] | (pmin[3] << 16));
        if (lane == 0) {
          me.mins[u & 1] = m01 & 0xFFFFu;
          me.mins[2 + u % 3] = m01 >> 16;
          me.mins[5 + (u & 3)] = m23 & 0xFFFFu;
          me.mins[9 + (u & 1)] = m23 >> 16;
          me.meta[u & 3] = static_cast<uint32_t>(lo) | (static_cast<uint32_t>(num) << 16);
          if (seam_out) {
            uint32_t* gm = gseam_meta(gseam_out, a.seam_pix_bytes, u, MAXC);
            gm[0] = m01 >> 16;
            gm[1] = m23 & 0xFFFFu;
            gm[2] = m23 >> 16;
            gm[3] = static_cast<uint32_t>(lo) | (static_cast<uint32_t>(num) << 16);
          }
        }

        if (a.dir > 0) {
          // Forward pass: store the partial sums of the four paths.
          uint32_t* sa32 = reinterpret_cast<uint32_t*>(a.sa + off);
#pragma unroll
          for (int c = 0; c < MAXC; ++c) {
            const int e = 64 * c + 2 * lane;
            if (c < nc && e < num) sa32[e >> 1] = sum[c];
          }
        } else {
          // Backward pass: total sums, winner-takes-all.
          const uint16_t* sb = me.sabuf + pslot * 64 * MAXC;
          uint32_t kmin = 0xFFFFFFFFu;
#pragma unroll
          for (int c = 0; c < MAXC; ++c) {
            const int e = 64 * c + 2 * lane;
            if (c < nc) {
              sum[c] = r3dsimt::vadd2(*reinterpret_cast<const uint32_t*>(sb + e), sum[c]);
              if (e < num) {
                const uint32_t klo = ((sum[c] & 0xFFFFu) << 16) | static_cast<uint32_t>(e);
                const uint32_t khi = (sum[c] & 0xFFFF0000u) | static_cast<uint32_t>(e + 1);
                kmin = r3dsimt::umin(kmin, r3dsimt::umin(klo, khi));
              }
            }
          }
          if (a.volume != nullptr) {
            uint32_t* v32 = reinterpret_cast<uint32_t*>(a.volume + off);
#pragma unroll
            for (int c = 0; c < MAXC; ++c) {
              const int e = 64 * c + 2 * lane;
              if (c < nc && e < num) v32[e >> 1] = sum[c];
            }
          }
          kmin = warp_min_u32(kmin);
          const int kb = static_cast<int>(kmin & 0xFFFFu);
          const uint32_t bcost = kmin >> 16;
          uint32_t sec = 0xFFFFu;
#pragma unroll
          for (int c = 0; c < MAXC; ++c) {
            const int e = 64 * c + 2 * lane;
            if (c < nc && e < num) {
              if (e + 1 < kb || e > kb + 1) sec = r3dsimt::umin(sec, sum[c] & 0xFFFFu);
              if (e + 2 < kb || e + 1 > kb + 1) sec = r3dsimt::umin(sec, sum[c] >> 16);
            }
          }
          sec = warp_min_u32(sec);
          uint32_t sm = 0, sp = 0;
          if (kb > 0 && kb < num - 1) {
            // S at labels kb - 1 and kb + 1 from the lanes that hold them.
            uint32_t vm = 0, vp = 0;
            const int cm = (kb - 1) >> 6, cp = (kb + 1) >> 6;
#pragma unroll
            for (int c = 0; c < MAXC; ++c) {
              if (c == cm) vm = sum[c];
              if (c == cp) vp = sum[c];
            }
            vm = r3dsimt::shfl(vm, ((kb - 1) & 63) >> 1);
            vp = r3dsimt::shfl(vp, ((kb + 1) & 63) >> 1);
            sm = ((kb - 1) & 1) ? (vm >> 16) : (vm & 0xFFFFu);
            sp = ((kb + 1) & 1) ? (vp >> 16) : (vp & 0xFFFFu);
          }
          const int x = a.w - 1 - u, y = a.h - 1 - v;  // image-order tile coordinates
          if (lane == 0) {
            a.info[static_cast<int64_t>(y) * a.w + x] =
                make_int4(static_cast<int>(static_cast<uint32_t>(lo + kb) | (bcost << 16)),
                          static_cast<int>(sec | (sm << 16)), static_cast<int>(sp), 0);
          }
          if (m.diagonal_lr) {
            const RowInterval lv = m.bv[a.y0 + y];
            const int bx = a.x0 + x;
            if (bx >= lv.first && bx <= lv.last) {
              uint32_t* keys = a.rkeys + static_cast<int64_t>(y) * a.rk;
              const int base = x - lo + a.row_shift[y];
#pragma unroll
              for (int c = 0; c < MAXC; ++c) {
                const int e = 64 * c + 2 * lane;
                if (c < nc && e < num) {
                  atomicMin(keys + (base - e), ((sum[c] & 0xFFFFu) << 16) | static_cast<uint32_t>(x));
                  atomicMin(keys + (base - e - 1), (sum[c] & 0xFFFF0000u) | static_cast<uint32_t>(x));
                }
              }
            }
          }
        }

        // Next prefetches, record queue.
        prefetch_pixel<MAXC>(a, me, u + kSgmPF, q[kSgmPF], lane);
        if (seam_in) prefetch_seam<MAXC>(a, gseam_in, u + kSgmPF + 1, lane);
        r3dsimt::cp_async_commit();
#pragma unroll
        for (int i = 0; i + 1 < kSgmQueue; ++i) q[i] = q[i + 1];
        q[kSgmQueue - 1] = u + kSgmQueue < a.w ? rrow[u + kSgmQueue] : make_int4(0, 0, 0, 0);
      }
    }
    r3dsimt::cp_async_wait<0>();
    r3dsimt::fence();
    r3dsimt::syncthreads();
  }
}

R3D_DEVICE float subpixel_offset(int method, float sm, float s0, float sp) {
  float delta = 0.0F;
  if (method == R3DGPU_SUBPIXEL_PARABOLA) {
    const float denom = __fadd_rn(__fsub_rn(sm, __fmul_rn(2.0F, s0)), sp);
    delta = denom > 0.0F ? __fdiv_rn(__fsub_rn(sm, sp), __fmul_rn(2.0F, denom)) : 0.0F;
  } else if (method == R3DGPU_SUBPIXEL_EQUIANGULAR) {
    const float a = __fsub_rn(sm, s0), b = __fsub_rn(sp, s0);
    const float slope = a < b ? b : a;
    delta = slope > 0.0F ? __fdiv_rn(__fsub_rn(sm, sp), __fmul_rn(2.0F, slope)) : 0.0F;
  }
  return delta < -0.5F ? -0.5F : (delta > 0.5F ? 0.5F : delta);
}

template <int MAXC>
R3D_GLOBAL void R3D_LAUNCH_BOUNDS(kSgmMaxRows * 32)
    sgm_tile_kernel(const SgmMatch* R3D_RESTRICT matches, const SgmJob* R3D_RESTRICT jobs, int njobs, int rows,
                    unsigned char* scratch, size_t slot_bytes, int* counter) {
  R3D_DYNAMIC_SMEM(smem);
  const SgmSmemLayout sl = sgm_smem_layout(MAXC, rows);
  const int nthreads = static_cast<int>(blockDim.x);
  const int tid = static_cast<int>(threadIdx.x);
  const int warp = tid >> 5, lane = tid & 31;
  unsigned char* slot = scratch + static_cast<size_t>(blockIdx.x) * slot_bytes;
  int* job_id = reinterpret_cast<int*>(smem);

  // Sentinel pads of every shared path vector (never overwritten later).
  {
    const int nvec = rows * 11 + kSgmSeamSlots * 3;
    for (int i = tid; i < nvec * 16; i += nthreads) {
      const int vi = i >> 4, k = i & 15;
      uint16_t* vec;
      if (vi < rows * 11) {
        vec = reinterpret_cast<uint16_t*>(smem + sl.rows_off + (vi / 11) * sl.row_bytes + sl.ring_off) +
              (vi % 11) * sl.vst;
      } else {
        const int s = (vi - rows * 11) / 3, p = (vi - rows * 11) % 3;
        vec = reinterpret_cast<uint16_t*>(smem + sl.seam_off + s * sl.seam_slot_bytes) + p * sl.vst;
      }
      const int idx = k < 8 ? k : 8 + 64 * MAXC + (k - 8);
      vec[idx] = static_cast<uint16_t>(kSent);
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
    //          right-WTA shift (max of lo + num - 1 - x).
    // The scratch layout needs the tile's cell count, which is known only
    // after P2; the layout's fixed-size part does not depend on it, so P1/P2
    // use it with cells = 0 and the cell-sized arrays are placed after P2.
    SgmSlotLayout L = sgm_slot_layout(w, h, 0ull, MAXC, m.nd);
    int4* rec_a = reinterpret_cast<int4*>(slot + L.rec_a);
    int4* rec_b = reinterpret_cast<int4*>(slot + L.rec_b);
    int4* info = reinterpret_cast<int4*>(slot + L.info);
    uint32_t* row_start = reinterpret_cast<uint32_t*>(slot + L.row_start);
    int* row_shift = reinterpret_cast<int*>(slot + L.row_shift);
    for (int y = warp; y < h; y += rows) {
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
          rec_a[static_cast<int64_t>(y) * w + x] =
              make_int4(static_cast<int>(run + excl), lo | (num << 16), 0, 0);
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
        const uint32_t t = y < h ? row_start[y + 1] : 0u;
        uint32_t total = 0;
        const uint32_t excl = warp_sum_excl(t, total);
        if (y < h) row_start[y + 1] = carry + excl + t;
        carry += total;
      }
      if (lane == 0) row_start[0] = 0;
    }
    r3dsimt::syncthreads();
    const unsigned long long cells = row_start[h];
    L = sgm_slot_layout(w, h, cells, MAXC, m.nd);
    uint8_t* cost = slot + L.cost;
    uint16_t* sa = reinterpret_cast<uint16_t*>(slot + L.sa);
    unsigned char* seam = slot + L.seam;
    uint32_t* rkeys = reinterpret_cast<uint32_t*>(slot + L.rkeys);

    // ---- P3: records of both passes (offset, range, P2 of the 4 paths).
    const uint16_t* img = m.base;
    const int64_t ist = m.base_stride;
    for (int64_t i = tid; i < npx; i += nthreads) {
      const int y = static_cast<int>(i / w), x = static_cast<int>(i % w);
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

    // ---- P4: Hamming costs, one warp per row, lanes over label pairs.
    for (int y = warp; y < h; y += rows) {
      const int by = job.y0 + y;
      const RowInterval lv = m.bv[by], rv = m.pv[by];
      const uint64_t* crow = m.cpart + static_cast<int64_t>(by) * m.cp_stride;
      for (int x = 0; x < w; ++x) {
        const int4 rc = rec_a[static_cast<int64_t>(y) * w + x];
        const int lo = rc.y & 0xFFFF, num = static_cast<int>(static_cast<uint32_t>(rc.y) >> 16);
        const int bx = job.x0 + x;
        const bool outside = bx < lv.first || bx > lv.last;
        const uint64_t cl = m.cbase[static_cast<int64_t>(by) * m.cb_stride + bx];
        for (int k = 2 * lane; k < num; k += 64) {
          const int xr = bx - m.dmin - (lo + k);
          uint32_t c0 = 0, c1 = 0;
          if (!outside) {
            c0 = (xr >= rv.first && xr <= rv.last) ? static_cast<uint32_t>(r3dsimt::popc64(cl ^ crow[xr]))
                                                   : static_cast<uint32_t>(m.invalid_cost);
            c1 = (xr - 1 >= rv.first && xr - 1 <= rv.last)
                     ? static_cast<uint32_t>(r3dsimt::popc64(cl ^ crow[xr - 1]))
                     : static_cast<uint32_t>(m.invalid_cost);
          }
          *reinterpret_cast<uint16_t*>(cost + rc.x + k) = static_cast<uint16_t>(c0 | (c1 << 8));
        }
      }
    }
    r3dsimt::fence();
    r3dsimt::syncthreads();

    // ---- Passes.
    PassArgs<MAXC> pa;
    pa.m = &m;
    pa.smem = smem;
    pa.sl = sl;
    pa.w = w;
    pa.h = h;
    pa.rows = rows;
    pa.cost = cost;
    pa.sa = sa;
    pa.info = info;
    pa.seam = seam;
    pa.seam_pix_bytes = L.seam_pix_bytes;
    pa.rkeys = rkeys;
    pa.rk = L.rk;
    pa.row_shift = row_shift;
    pa.x0 = job.x0;
    pa.y0 = job.y0;
    pa.volume = job.volume;
    pa.dir = 1;
    pa.recs = rec_a;
    run_pass<MAXC>(pa);
    pa.dir = -1;
    pa.recs = rec_b;
    run_pass<MAXC>(pa);

    // ---- Acceptance rules and outputs (stereo_matcher.cpp:474-523).
    for (int64_t i = tid; i < npx; i += nthreads) {
      const int y = static_cast<int>(i / w), x = static_cast<int>(i % w);
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
            delta = subpixel_offset(m.subpixel, static_cast<float>(sm), best_cost, static_cast<float>(sp));
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

template <int MAXC>
void launch_instance(const SgmMatch* d_matches, const SgmJob* d_jobs, int njobs, int rows, int grid,
                     unsigned char* scratch, size_t slot_bytes, int* d_counter, cudaStream_t s) {
  const size_t smem = static_cast<size_t>(sgm_smem_layout(MAXC, rows).total);
  // Raise the kernel's dynamic shared-memory limit when a launch needs more
  // than any earlier one (per device; the attribute is per function).
  static thread_local int configured[64] = {};
  int dev = 0;
  R3D_CUDA(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 64 && configured[dev] < static_cast<int>(smem)) {
    R3D_CUDA(cudaFuncSetAttribute(sgm_tile_kernel<MAXC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem)));
    configured[dev] = static_cast<int>(smem);
  }
  R3D_LAUNCH(sgm_tile_kernel<MAXC>, dim3(grid), dim3(rows * 32), smem, s, d_matches, d_jobs, njobs, rows, scratch,
             slot_bytes, d_counter);
  launched("sgm_tile_kernel");
}

}  // namespace

int sgm_maxc_for(int max_num) {
  const int c = (max_num + 63) / 64;
  if (c <= 1) return 1;
  if (c <= 2) return 2;
  if (c <= 3) return 3;
  if (c <= 4) return 4;
  if (c <= 6) return 6;
  if (c <= 8) return 8;
  if (c <= 12) return 12;
  if (c <= 16) return 16;
  fail(R3DGPU_EUNSUPPORTED, "stereo: more than " + std::to_string(kSgmMaxLabels) + " labels per pixel");
}

int sgm_rows_for(int maxc, int smem_optin) {
  for (int r = kSgmMaxRows; r >= 1; --r)
    if (sgm_smem_layout(maxc, r).total <= smem_optin) return r;
  fail(R3DGPU_EUNSUPPORTED, "stereo: label count needs more shared memory than the device has");
}

void launch_sgm(const SgmMatch* d_matches, const SgmJob* d_jobs, int njobs, int maxc, int rows, int grid,
                unsigned char* scratch, size_t slot_bytes, int* d_counter, cudaStream_t s) {
  switch (maxc) {
    case 1: launch_instance<1>(d_matches, d_jobs, njobs, rows, grid, scratch, slot_bytes, d_counter, s); break;
    case 2: launch_instance<2>(d_matches, d_jobs, njobs, rows, grid, scratch, slot_bytes, d_counter, s); break;
    case 3: launch_instance<3>(d_matches, d_jobs, njobs, rows, grid, scratch, slot_bytes, d_counter, s); break;
    case 4: launch_instance<4>(d_matches, d_jobs, njobs, rows, grid, scratch, slot_bytes, d_counter, s); break;
    case 6: launch_instance<6>(d_matches, d_jobs, njobs, rows, grid, scratch, slot_bytes, d_counter, s); break;
    case 8: launch_instance<8>(d_matches, d_jobs, njobs, rows, grid, scratch, slot_bytes, d_counter, s); break;
    case 12: launch_instance<12>(d_matches, d_jobs, njobs, rows, grid, scratch, slot_bytes, d_counter, s); break;
    case 16: launch_instance<16>(d_matches, d_jobs, njobs, rows, grid, scratch, slot_bytes, d_counter, s); break;
    default: fail(R3DGPU_EINVAL, "stereo: bad label chunk count");
  }
}

}  // namespace r3dgpu
