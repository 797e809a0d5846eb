// CPU oracle of the R3DMVS Census+SGM matcher — TEST INFRASTRUCTURE ONLY.
//
// This file restates, in plain C++ written for this project, what the
// reference matcher computes (rhiestan/Regard3D_MVS, src/r3d/stereo/ and
// src/r3d/core/pyramid.cpp). It is the checker for the GPU library: only the
// tests, the smoke check and bench.py's CPU-baseline leg may load it. The
// product never calls it.
//
// The reference cannot be compiled here (its sources need Highway 1.2.0 and
// Eigen 3.4.0, which are absent), so parity is pinned instead by the
// reference's own known-answer tests and invariants, restated in
// tests/test_oracle.py (Census bit order and borders, pyramid rounding,
// ranges_from_coarse, speckle/median values, slanted-plane accuracy, the
// textbook-volume identity).
//
// Aggregation is the reference's textbook form (sgm_cost_volume_reference,
// src/r3d/stereo/stereo_matcher.cpp:1280-1362): each of the 8 paths
// separately, in int arithmetic, labels outside a range are "infinite",
// restarted at every tile border; the reference's tests assert that its
// production kernels give the same volume (tests/test_stereo.cpp:87-151).
//
// Floating point follows the reference compiled for baseline x86-64 (no FMA):
// build with -ffp-contract=off.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/r3dgpu.h"

namespace orc {

using Options = r3dgpu_stereo_options;
constexpr float kInvalid = std::numeric_limits<float>::infinity();
constexpr int kInf = 1 << 28;  // L of a label outside a range (stereo_matcher.cpp:1313)

struct Failure : std::runtime_error {
  using std::runtime_error::runtime_error;
};

thread_local std::string g_error;

int align16(int n) { return (n + 15) / 16 * 16; }

template <class T>
struct Img {
  int w = 0, h = 0;
  std::vector<T> px;
  Img() = default;
  Img(int w_, int h_, T v = T{}) : w(w_), h(h_), px(static_cast<size_t>(w_) * h_, v) {}
  T& operator()(int x, int y) { return px[static_cast<size_t>(y) * w + x]; }
  const T& operator()(int x, int y) const { return px[static_cast<size_t>(y) * w + x]; }
  bool empty() const { return w == 0 || h == 0; }
};

template <class T>
Img<T> wrap(const T* p, int w, int h) {
  Img<T> m;
  if (p == nullptr) return m;
  m.w = w;
  m.h = h;
  m.px.assign(p, p + static_cast<size_t>(w) * h);
  return m;
}

// ---------------------------------------------------------------- census
// census.hpp:11-16, census.cpp:20-35, 104-113: 9x7 window, neighbours in
// raster order without the centre, first neighbour in bit 61, bit set when the
// neighbour is darker than the centre, borders replicated (census.cpp:151-153).
Img<uint64_t> census(const Img<uint16_t>& im) {
  Img<uint64_t> out(im.w, im.h);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < im.h; ++y) {
    for (int x = 0; x < im.w; ++x) {
      const uint16_t c = im(x, y);
      uint64_t bits = 0;
      for (int j = 0; j < 7; ++j) {
        const int yy = std::clamp(y + j - 3, 0, im.h - 1);
        for (int i = 0; i < 9; ++i) {
          if (j == 3 && i == 4) continue;
          const int xx = std::clamp(x + i - 4, 0, im.w - 1);
          bits = (bits << 1) | (im(xx, yy) < c ? 1u : 0u);
        }
      }
      out(x, y) = bits;
    }
  }
  return out;
}

// ---------------------------------------------------------------- pyramid
// pyramid.cpp:33-85: [1 4 6 4 1] horizontally then vertically with u32 sums,
// (s + 128) >> 8, clamped borders, size ceil(w/2) x ceil(h/2).
template <class T>
Img<T> pyramid_down(const Img<T>& s) {
  const int w = s.w, h = s.h, dw = (w + 1) / 2, dh = (h + 1) / 2;
  Img<uint32_t> tmp(dw, h);
  for (int y = 0; y < h; ++y) {
    for (int x = 0; x < dw; ++x) {
      const int c = 2 * x;
      auto v = [&](int xx) { return static_cast<uint32_t>(s(std::clamp(xx, 0, w - 1), y)); };
      tmp(x, y) = v(c - 2) + v(c + 2) + 4u * (v(c - 1) + v(c + 1)) + 6u * v(c);
    }
  }
  Img<T> out(dw, dh);
  for (int y = 0; y < dh; ++y) {
    const int c = 2 * y;
    for (int x = 0; x < dw; ++x) {
      auto v = [&](int yy) { return tmp(x, std::clamp(yy, 0, h - 1)); };
      out(x, y) = static_cast<T>((v(c - 2) + v(c + 2) + 4u * (v(c - 1) + v(c + 1)) + 6u * v(c) + 128u) >> 8);
    }
  }
  return out;
}

// stereo_matcher.cpp:892-900
Img<uint8_t> reduce_mask(const Img<uint8_t>& m) {
  Img<uint8_t> r = pyramid_down(m);
  for (auto& v : r.px) v = v >= 128 ? 255 : 0;
  return r;
}

template <class T>
Img<T> mirror(const Img<T>& m) {
  Img<T> r(m.w, m.h);
  for (int y = 0; y < m.h; ++y)
    for (int x = 0; x < m.w; ++x) r(x, y) = m(m.w - 1 - x, y);
  return r;
}

// ---------------------------------------------------------------- context
struct Interval {
  int first = 0, last = -1;
};

// stereo_matcher.cpp:43-67: valid columns [first, last] of each row (mask >= 128).
std::vector<Interval> intervals(const Img<uint8_t>& mask, int w, int h) {
  std::vector<Interval> rows(h, Interval{0, w - 1});
  if (mask.empty()) return rows;
  for (int y = 0; y < h; ++y) {
    Interval r;
    int x = 0;
    while (x < w && mask(x, y) < 128) ++x;
    if (x < w) {
      r.first = x;
      int e = w - 1;
      while (mask(e, y) < 128) --e;
      r.last = e;
    }
    rows[y] = r;
  }
  return rows;
}

// stereo_matcher.cpp:69-79
std::array<uint16_t, 256> p2_lut(const Options& o) {
  std::array<uint16_t, 256> t{};
  for (int di = 0; di < 256; ++di) {
    int p2 = o.p2;
    if (o.p2_adapt > 0) p2 = std::max(o.p1 + 1, o.p2 * o.p2_adapt / (o.p2_adapt + di));
    t[di] = static_cast<uint16_t>(p2);
  }
  return t;
}

// stereo_matcher.cpp:81-95
void check_options(const Options& o) {
  if (o.p1 < 0 || o.p2 < o.p1 || o.p2 > 8000) throw Failure("stereo: invalid penalties");
  if (o.invalid_cost < 0 || o.invalid_cost > 255) throw Failure("stereo: invalid_cost outside [0, 255]");
  if (o.tile_size < 16 || o.tile_margin < 0 || o.tile_blend < 0) throw Failure("stereo: invalid tiling");
  if (o.levels < -1 || o.levels > 12 || o.range_radius < 0 || o.range_margin < 0 || o.range_fill < 0)
    throw Failure("stereo: invalid hierarchy");
}

struct Ranges {
  Img<uint16_t> lo, num;
};

// stereo_matcher.cpp:97-111
void check_ranges(const Ranges& r, int w, int h, int nd) {
  if (r.lo.w != w || r.lo.h != h || r.num.w != w || r.num.h != h) throw Failure("stereo: label ranges size");
  for (size_t i = 0; i < r.lo.px.size(); ++i) {
    const int lo = r.lo.px[i], n = r.num.px[i];
    if (n <= 0 || n % 16 != 0 || lo + n > nd) throw Failure("stereo: invalid label range");
  }
}

struct Ctx {
  Img<uint16_t> base, partner;         // base (matched) image and its partner
  Img<uint64_t> cb, cp;                // their census images
  std::vector<Interval> bv, pv;        // valid row intervals
  int dmin = 0, nd = 0;                // nd: aligned label count
  const Ranges* ranges = nullptr;
  std::array<uint16_t, 256> lut{};
  Options o{};
  bool diagonal_lr = false;
  bool confidence = true;
  int lo(int x, int y) const { return ranges ? ranges->lo(x, y) : 0; }
  int num(int x, int y) const { return ranges ? ranges->num(x, y) : nd; }
};

// stereo_matcher.cpp:128-163
Ctx make_ctx(const Img<uint16_t>& base, const Img<uint16_t>& partner, const Img<uint8_t>& bmask,
             const Img<uint8_t>& pmask, int dmin, int nd, const Ranges* ranges, const Options& o) {
  check_options(o);
  if (base.h != partner.h || base.empty() || partner.empty()) throw Failure("stereo: image sizes");
  if (!bmask.empty() && (bmask.w != base.w || bmask.h != base.h)) throw Failure("stereo: left mask size");
  if (!pmask.empty() && (pmask.w != partner.w || pmask.h != partner.h)) throw Failure("stereo: right mask size");
  if (nd <= 0) throw Failure("stereo: no disparities to search");
  Ctx c;
  c.base = base;
  c.partner = partner;
  c.cb = census(base);
  c.cp = census(partner);
  c.bv = intervals(bmask, base.w, base.h);
  c.pv = intervals(pmask, partner.w, partner.h);
  c.dmin = dmin;
  c.nd = align16(nd);
  if (ranges) check_ranges(*ranges, base.w, base.h, c.nd);
  c.ranges = ranges;
  c.lut = p2_lut(o);
  c.o = o;
  return c;
}

// ---------------------------------------------------------------- tiles
struct Tile {
  int x0 = 0, y0 = 0, w = 0, h = 0;
  int c0x = 0, c1x = 0, c0y = 0, c1y = 0;  // core
};

// stereo_matcher.cpp:545-552
std::vector<int> split(int size, int tile) {
  const int n = std::max(1, (size + tile - 1) / tile);
  std::vector<int> b(n + 1);
  for (int i = 0; i <= n; ++i) b[i] = static_cast<int>(static_cast<long long>(size) * i / n);
  return b;
}

// stereo_matcher.cpp:555-568
uint64_t count_cells(const Ctx& c, int x0, int y0, int x1, int y1) {
  if (!c.ranges) return static_cast<uint64_t>(x1 - x0) * static_cast<uint64_t>(y1 - y0) * c.nd;
  uint64_t s = 0;
  for (int y = y0; y < y1; ++y)
    for (int x = x0; x < x1; ++x) s += c.ranges->num(x, y);
  return s;
}

// stereo_matcher.cpp:571-578
size_t estimated_tile_bytes(const Ctx& c, int x0, int y0, int x1, int y1, size_t right_width) {
  const size_t cells = static_cast<size_t>(count_cells(c, x0, y0, x1, y1));
  const size_t w = static_cast<size_t>(x1 - x0), h = static_cast<size_t>(y1 - y0);
  const size_t row_cells = cells / std::max<size_t>(h, 1);
  return cells * 2 + row_cells * 2 + 6 * (row_cells + w * 2 * 8) * 2 + w * h * 32 + (w + right_width + 16) * (h + 6) * 8;
}

// stereo_matcher.cpp:619-650
std::vector<Tile> tile_layout(const Ctx& c) {
  const Options& o = c.o;
  const int W = c.base.w, H = c.base.h;
  const int ext = o.tile_margin + (o.tile_blend + 1) / 2;
  auto layout = [&](int ts) {
    std::vector<Tile> t;
    const auto bx = split(W, ts), by = split(H, ts);
    for (size_t j = 0; j + 1 < by.size(); ++j)
      for (size_t i = 0; i + 1 < bx.size(); ++i) {
        Tile tl;
        tl.x0 = std::max(0, bx[i] - ext);
        const int x1 = std::min(W, bx[i + 1] + ext);
        tl.y0 = std::max(0, by[j] - ext);
        const int y1 = std::min(H, by[j + 1] + ext);
        tl.w = x1 - tl.x0;
        tl.h = y1 - tl.y0;
        tl.c0x = bx[i];
        tl.c1x = bx[i + 1];
        tl.c0y = by[j];
        tl.c1y = by[j + 1];
        t.push_back(tl);
      }
    return t;
  };
  auto max_bytes = [&](const std::vector<Tile>& ts) {
    size_t m = 0;
    for (const Tile& t : ts)
      m = std::max(m, estimated_tile_bytes(c, t.x0, t.y0, t.x0 + t.w, t.y0 + t.h, static_cast<size_t>(c.partner.w)));
    return m;
  };
  int ts = o.tile_size;
  auto tiles = layout(ts);
  while (ts > 64 && max_bytes(tiles) > o.memory_budget) {
    ts /= 2;
    tiles = layout(ts);
  }
  return tiles;
}

// ---------------------------------------------------------------- aggregation
// Packed per-pixel labels of a tile (row-major pixel order).
struct TileLabels {
  int w = 0, h = 0;
  std::vector<int> lo, num;
  std::vector<size_t> off;  // [w*h + 1]
  int max_num = 0;
};

TileLabels tile_labels(const Ctx& c, const Tile& t) {
  TileLabels L;
  L.w = t.w;
  L.h = t.h;
  const size_t n = static_cast<size_t>(t.w) * t.h;
  L.lo.resize(n);
  L.num.resize(n);
  L.off.assign(n + 1, 0);
  for (int y = 0; y < t.h; ++y)
    for (int x = 0; x < t.w; ++x) {
      const size_t i = static_cast<size_t>(y) * t.w + x;
      L.lo[i] = c.lo(t.x0 + x, t.y0 + y);
      L.num[i] = c.num(t.x0 + x, t.y0 + y);
      L.off[i + 1] = L.off[i] + L.num[i];
      L.max_num = std::max(L.max_num, L.num[i]);
    }
  return L;
}

// Matching costs of a tile (stereo_matcher.cpp:305-353): Hamming distance of
// the Census codes; labels whose right column lies outside the row's valid
// right interval cost invalid_cost; left pixels outside the valid left
// interval cost 0 for every label.
std::vector<uint8_t> tile_costs(const Ctx& c, const Tile& t, const TileLabels& L) {
  std::vector<uint8_t> C(L.off.back());
  const auto inv = static_cast<uint8_t>(c.o.invalid_cost);
  for (int y = 0; y < t.h; ++y) {
    const int by = t.y0 + y;
    const Interval lv = c.bv[by], rv = c.pv[by];
    for (int x = 0; x < t.w; ++x) {
      const int bx = t.x0 + x;
      const size_t i = static_cast<size_t>(y) * t.w + x;
      uint8_t* out = C.data() + L.off[i];
      if (bx < lv.first || bx > lv.last) {
        std::fill(out, out + L.num[i], uint8_t{0});
        continue;
      }
      const uint64_t cl = c.cb(bx, by);
      for (int k = 0; k < L.num[i]; ++k) {
        const int xr = bx - c.dmin - (L.lo[i] + k);
        out[k] = (xr >= rv.first && xr <= rv.last) ? static_cast<uint8_t>(__builtin_popcountll(cl ^ c.cp(xr, by))) : inv;
      }
    }
  }
  return C;
}

// One path step: L(p, a) = C(p, a) + min(Lq(a), Lq(a-1)+P1, Lq(a+1)+P1, minq+P2) - minq,
// Lq infinite outside q's range (stereo_matcher.cpp:1334-1341). `lq` holds
// q's values at p's labels a = lo-1 .. lo+num (index a - lo + 1).
inline void path_step(const int* lq, int minq, int p1, int p2, const uint8_t* cost, int num, int* lp, int& minp) {
  int m = std::numeric_limits<int>::max();
  const int pen = minq + p2;
  for (int k = 0; k < num; ++k) {
    const int nb = std::min(lq[k], lq[k + 2]) + p1;
    const int best = std::min(std::min(lq[k + 1], nb), pen);
    const int v = static_cast<int>(cost[k]) + best - minq;
    lp[k] = v;
    m = std::min(m, v);
  }
  minp = m;
}

// Aggregated volume S of a tile: the 8 paths of the textbook, restarted at the
// tile border, summed modulo 2^16 (the reference casts the int sum to u16).
std::vector<uint16_t> aggregate_tile(const Ctx& c, const Tile& t, const TileLabels& L) {
  const std::vector<uint8_t> C = tile_costs(c, t, L);
  std::vector<uint16_t> S(L.off.back(), 0);
  const int w = t.w, h = t.h, D = L.max_num;
  const int stride = D + 2;  // one "infinite" label on each side
  std::vector<int> prev(static_cast<size_t>(w) * stride), cur(static_cast<size_t>(w) * stride);
  std::vector<int> prev_min(w), cur_min(w);
  std::vector<int> lq(D + 2);
  const int dirs[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {-1, -1}, {-1, 1}, {1, -1}};
  for (const auto& d : dirs) {
    const int dx = d[0], dy = d[1];
    for (int iy = 0; iy < h; ++iy) {
      const int y = dy >= 0 ? iy : h - 1 - iy;
      for (int ix = 0; ix < w; ++ix) {
        const int x = dx >= 0 ? ix : w - 1 - ix;
        const size_t i = static_cast<size_t>(y) * w + x;
        const int lo = L.lo[i], num = L.num[i];
        const uint8_t* cost = C.data() + L.off[i];
        int* lp = cur.data() + static_cast<size_t>(x) * stride + 1;
        const int qx = x - dx, qy = y - dy;
        int m;
        if (qx < 0 || qy < 0 || qx >= w || qy >= h) {
          m = std::numeric_limits<int>::max();
          for (int k = 0; k < num; ++k) {
            lp[k] = cost[k];
            m = std::min(m, lp[k]);
          }
        } else {
          const size_t qi = static_cast<size_t>(qy) * w + qx;
          const std::vector<int>& qbuf = dy == 0 ? cur : prev;
          const int* q = qbuf.data() + static_cast<size_t>(qx) * stride + 1;
          const int qlo = L.lo[qi], qnum = L.num[qi];
          const int minq = dy == 0 ? cur_min[qx] : prev_min[qx];
          for (int k = -1; k <= num; ++k) {
            const int a = lo + k - qlo;
            lq[k + 1] = (a >= 0 && a < qnum) ? q[a] : kInf;
          }
          const int p2 = c.lut[std::abs(int{c.base(t.x0 + x, t.y0 + y)} - int{c.base(t.x0 + qx, t.y0 + qy)}) >> 8];
          path_step(lq.data(), minq, c.o.p1, p2, cost, num, lp, m);
        }
        cur_min[x] = m;
        uint16_t* s = S.data() + L.off[i];
        for (int k = 0; k < num; ++k) s[k] = static_cast<uint16_t>(s[k] + lp[k]);
      }
      if (dy != 0) {
        std::swap(prev, cur);
        std::swap(prev_min, cur_min);
      }
    }
  }
  return S;
}

// ---------------------------------------------------------------- selection
struct TileResult {
  Tile t;
  std::vector<float> disp, conf;
  uint64_t cells = 0;
};

// stereo_matcher.cpp:426-436
float subpixel_offset(int method, float sm, float s0, float sp) {
  float delta = 0.0F;
  if (method == R3DGPU_SUBPIXEL_PARABOLA) {
    const float denom = sm - 2.0F * s0 + sp;
    delta = denom > 0.0F ? (sm - sp) / (2.0F * denom) : 0.0F;
  } else if (method == R3DGPU_SUBPIXEL_EQUIANGULAR) {
    const float slope = std::max(sm - s0, sp - s0);
    delta = slope > 0.0F ? (sm - sp) / (2.0F * slope) : 0.0F;
  }
  return std::clamp(delta, -0.5F, 0.5F);
}

// Winner-takes-all and the acceptance rules of stereo_matcher.cpp:446-525 with
// the row WTA of sgm_kernels.cpp:405-438 (first minimum; second best outside
// best +- 1; right-image WTA along the diagonal keeps the first strict minimum).
void select_disparities(const Ctx& c, const TileLabels& L, const std::vector<uint16_t>& S, TileResult& r) {
  const Tile& t = r.t;
  const Options& o = c.o;
  const int w = t.w;
  r.disp.assign(static_cast<size_t>(w) * t.h, kInvalid);
  if (c.confidence) r.conf.assign(static_cast<size_t>(w) * t.h, 0.0F);
  std::vector<uint16_t> rc, rb;
  std::vector<int> bestv(w), costv(w), secv(w);
  for (int y = 0; y < t.h; ++y) {
    const int by = t.y0 + y;
    const size_t row = static_cast<size_t>(y) * w;
    long shift = 0;
    if (c.diagonal_lr) {
      long top = 0;
      shift = std::numeric_limits<long>::min();
      for (int x = 0; x < w; ++x) {
        shift = std::max<long>(shift, L.lo[row + x] + L.num[row + x] - 1 - x);
        top = std::max<long>(top, x - L.lo[row + x]);
      }
      rc.assign(static_cast<size_t>(top + shift + 1), 0xFFFF);
      rb.assign(rc.size(), 0xFFFF);
    }
    const Interval lv = c.bv[by], rv = c.pv[by];
    const int xb = std::clamp(lv.first - t.x0, 0, w);
    const int xe = std::clamp(lv.last + 1 - t.x0, xb, w);
    for (int x = xb; x < xe; ++x) {
      const size_t i = row + x;
      const uint16_t* s = S.data() + L.off[i];
      const int n = L.num[i], lo = L.lo[i];
      int kb = 0;
      for (int k = 1; k < n; ++k)
        if (s[k] < s[kb]) kb = k;
      int sec = 0xFFFF;
      for (int k = 0; k < n; ++k)
        if (k + 1 < kb || k > kb + 1) sec = std::min<int>(sec, s[k]);
      bestv[x] = lo + kb;
      costv[x] = s[kb];
      secv[x] = sec;
      if (c.diagonal_lr) {
        for (int k = 0; k < n; ++k) {
          const size_t ri = static_cast<size_t>(x - lo - k + shift);
          if (s[k] < rc[ri]) {
            rc[ri] = s[k];
            rb[ri] = static_cast<uint16_t>(lo + k);
          }
        }
      }
    }
    for (int x = xb; x < xe; ++x) {
      const size_t i = row + x;
      const uint16_t* s = S.data() + L.off[i];
      const int best = bestv[x], j = best - L.lo[i], n = L.num[i];
      const unsigned second = static_cast<unsigned>(secv[x]);
      const int xr = t.x0 + x - c.dmin - best;
      if (xr < rv.first || xr > rv.last) continue;
      if ((j == 0 && L.lo[i] > 0) || (j == n - 1 && L.lo[i] + n < c.nd)) continue;
      if (c.diagonal_lr && std::abs(int{rb[static_cast<size_t>(x - best + shift)]} - best) > o.lr_max_diff) continue;
      const float best_cost = static_cast<float>(costv[x]);
      if (o.uniqueness > 0.0F && second != 0xFFFFu && best_cost > (1.0F - o.uniqueness) * static_cast<float>(second))
        continue;
      float delta = 0.0F;
      if (j > 0 && j < n - 1) delta = subpixel_offset(o.subpixel, s[j - 1], best_cost, s[j + 1]);
      r.disp[i] = static_cast<float>(c.dmin + best) + delta;
      if (c.confidence)
        r.conf[i] = second != 0xFFFFu && second > 0 ? 1.0F - best_cost / static_cast<float>(second) : 0.0F;
    }
  }
}

// stereo_matcher.cpp:530-543
float axis_weight(int v, int c0, int c1, int size, int blend_px) {
  const float blend = static_cast<float>(blend_px);
  float w = 1.0F;
  const float pos = static_cast<float>(v) + 0.5F;
  if (c0 > 0)
    w = std::min(w, blend_px > 0 ? std::clamp((pos - static_cast<float>(c0) + 0.5F * blend) / blend, 0.0F, 1.0F)
                                 : (v >= c0 ? 1.0F : 0.0F));
  if (c1 < size)
    w = std::min(w, blend_px > 0 ? std::clamp((static_cast<float>(c1) + 0.5F * blend - pos) / blend, 0.0F, 1.0F)
                                 : (v < c1 ? 1.0F : 0.0F));
  return w;
}

struct Map {
  Img<float> disp, conf;
  uint64_t cells = 0;
};

// Tiles, per-tile selection and blending (stereo_matcher.cpp:613-771).
Map match_tiles(const Ctx& c) {
  const std::vector<Tile> layout = tile_layout(c);
  std::vector<TileResult> res(layout.size());
#pragma omp parallel for schedule(dynamic, 1)
  for (size_t ti = 0; ti < layout.size(); ++ti) {
    res[ti].t = layout[ti];
    const TileLabels L = tile_labels(c, layout[ti]);
    const std::vector<uint16_t> S = aggregate_tile(c, layout[ti], L);
    select_disparities(c, L, S, res[ti]);
    res[ti].cells = L.off.back();
  }
  const int W = c.base.w, H = c.base.h, blend = c.o.tile_blend;
  Map out;
  for (const auto& r : res) out.cells += r.cells;
  out.disp = Img<float>(W, H, kInvalid);
  if (c.confidence) out.conf = Img<float>(W, H, 0.0F);
  std::vector<std::vector<float>> colw(res.size());
  for (size_t i = 0; i < res.size(); ++i) {
    const Tile& t = res[i].t;
    colw[i].resize(t.w);
    for (int x = 0; x < t.w; ++x) colw[i][x] = axis_weight(t.x0 + x, t.c0x, t.c1x, W, blend);
  }
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H; ++y) {
    std::vector<float> wsum(W, 0.0F), wall(W, 0.0F), dsum(W, 0.0F), csum(W, 0.0F), wbest(W, 0.0F), dbest(W, kInvalid);
    for (size_t i = 0; i < res.size(); ++i) {
      const TileResult& r = res[i];
      const Tile& t = r.t;
      if (y < t.y0 || y >= t.y0 + t.h) continue;
      const float wy = axis_weight(y, t.c0y, t.c1y, H, blend);
      if (wy <= 0.0F) continue;
      const size_t row = static_cast<size_t>(y - t.y0) * t.w;
      for (int x = 0; x < t.w; ++x) {
        const float wg = wy * colw[i][x];
        if (wg <= 0.0F) continue;
        const int px = t.x0 + x;
        wall[px] += wg;
        const float dv = r.disp[row + x];
        if (std::isfinite(dv)) {
          wsum[px] += wg;
          dsum[px] += wg * dv;
          if (c.confidence) csum[px] += wg * r.conf[row + x];
          if (wg > wbest[px]) {
            wbest[px] = wg;
            dbest[px] = dv;
          }
        }
      }
    }
    for (int x = 0; x < W; ++x) {
      float dv = kInvalid;
      if (wsum[x] > 0.0F && wsum[x] >= 0.5F * wall[x]) {
        dv = dsum[x] / wsum[x];
        if (std::abs(dv - dbest[x]) > 1.0F) dv = dbest[x];
        if (c.confidence) out.conf(x, y) = csum[x] / wsum[x];
      }
      out.disp(x, y) = dv;
    }
  }
  return out;
}

// ---------------------------------------------------------------- checks and filters
// stereo_matcher.cpp:777-782
bool lr_differ(const Img<float>& map, const Img<float>& other, int x, int y, int sign, int max_diff) {
  const float d = map(x, y);
  const int xo = static_cast<int>(std::lround(static_cast<float>(x) + static_cast<float>(sign) * d));
  const float dother = xo >= 0 && xo < other.w ? other(xo, y) : kInvalid;
  return !std::isfinite(dother) || std::abs(d - dother) > static_cast<float>(max_diff);
}

std::vector<uint8_t> lr_mismatch(const Img<float>& map, const Img<float>& other, int sign, int max_diff) {
  std::vector<uint8_t> bad(map.px.size(), 0);
  for (int y = 0; y < map.h; ++y)
    for (int x = 0; x < map.w; ++x)
      if (std::isfinite(map(x, y)) && lr_differ(map, other, x, y, sign, max_diff)) bad[static_cast<size_t>(y) * map.w + x] = 1;
  return bad;
}

void apply_bad(Img<float>& map, const std::vector<uint8_t>& bad) {
  for (size_t i = 0; i < bad.size(); ++i)
    if (bad[i]) map.px[i] = kInvalid;
}

// stereo_matcher.cpp:919-970: segments of 4-neighbours with |step| <= max_diff
// (breadth first; the segments are the connected components of that relation).
void remove_speckles(Img<float>& d, int min_size, float max_diff) {
  if (min_size <= 1 || d.empty()) return;
  const int w = d.w;
  const size_t n = d.px.size();
  std::vector<uint8_t> seen(n, 0);
  std::vector<uint32_t> seg;
  for (size_t s = 0; s < n; ++s) {
    if (seen[s] || !std::isfinite(d.px[s])) continue;
    seg.clear();
    seg.push_back(static_cast<uint32_t>(s));
    seen[s] = 1;
    for (size_t head = 0; head < seg.size(); ++head) {
      const size_t i = seg[head];
      const float v = d.px[i];
      const int x = static_cast<int>(i % w);
      auto visit = [&](size_t j) {
        if (!seen[j] && std::abs(d.px[j] - v) <= max_diff) {
          seen[j] = 1;
          seg.push_back(static_cast<uint32_t>(j));
        }
      };
      if (x > 0) visit(i - 1);
      if (x + 1 < w) visit(i + 1);
      if (i >= static_cast<size_t>(w)) visit(i - w);
      if (i + w < n) visit(i + w);
    }
    if (static_cast<int>(seg.size()) < min_size)
      for (uint32_t i : seg) d.px[i] = kInvalid;
  }
}

// stereo_matcher.cpp:972-1021: median of the valid values of the 3x3
// neighbourhood; an even count averages the two middle values. (The
// reference's 9-value sorting network returns the same middle value.)
Img<float> median3x3(const Img<float>& d) {
  Img<float> out(d.w, d.h);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < d.h; ++y) {
    for (int x = 0; x < d.w; ++x) {
      const float c = d(x, y);
      if (!std::isfinite(c)) {
        out(x, y) = c;
        continue;
      }
      float v[9];
      int n = 0;
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int qx = x + dx, qy = y + dy;
          if (qx >= 0 && qy >= 0 && qx < d.w && qy < d.h && std::isfinite(d(qx, qy))) v[n++] = d(qx, qy);
        }
      for (int a = 1; a < n; ++a)  // insertion sort of at most 9 values
        for (int b = a; b > 0 && v[b] < v[b - 1]; --b) std::swap(v[b], v[b - 1]);
      float m = v[n / 2];
      if (n % 2 == 0) m = 0.5F * (m + v[n / 2 - 1]);
      out(x, y) = m;
    }
  }
  return out;
}

void post_filter(Img<float>& d, const Options& o, int speckle) {
  remove_speckles(d, speckle, o.speckle_diff);
  if (o.median) d = median3x3(d);
}

// ---------------------------------------------------------------- ranges
// stereo_matcher.cpp:1124-1267
Ranges ranges_from_coarse(const Img<float>& coarse, int width, int height, const Img<uint8_t>& fine_valid,
                          const Img<uint8_t>& partner_valid, int partner_width, int partner_sign, int dmin, int nd,
                          const Options& o, bool mirrored) {
  const int wc = coarse.w, hc = coarse.h;
  if (wc != (width + 1) / 2 || hc != (height + 1) / 2) throw Failure("stereo: coarse map size");
  const float inf = std::numeric_limits<float>::infinity();
  const int r = o.range_radius;
  Img<float> hmin(wc, hc), hmax(wc, hc);
  for (int y = 0; y < hc; ++y)
    for (int x = 0; x < wc; ++x) {
      float mn = inf, mx = -inf;
      for (int k = std::max(0, x - r); k <= std::min(wc - 1, x + r); ++k) {
        const float v = coarse(k, y);
        if (std::isfinite(v)) {
          mn = std::min(mn, v);
          mx = std::max(mx, v);
        }
      }
      hmin(x, y) = mn;
      hmax(x, y) = mx;
    }
  Img<float> cmin(wc, hc), cmax(wc, hc);
  for (int y = 0; y < hc; ++y)
    for (int x = 0; x < wc; ++x) {
      float mn = inf, mx = -inf;
      for (int k = std::max(0, y - r); k <= std::min(hc - 1, y + r); ++k) {
        mn = std::min(mn, hmin(x, k));
        mx = std::max(mx, hmax(x, k));
      }
      cmin(x, y) = mn;
      cmax(x, y) = mx;
    }
  std::vector<Img<float>> pmin{cmin}, pmax{cmax};
  while ((2 << pmin.size()) <= 2 * o.range_fill && pmin.back().w > 1) {
    const Img<float>& a = pmin.back();
    const Img<float>& b = pmax.back();
    const int nw = (a.w + 1) / 2, nh = (a.h + 1) / 2;
    Img<float> mn(nw, nh), mx(nw, nh);
    for (int y = 0; y < nh; ++y)
      for (int x = 0; x < nw; ++x) {
        const int x1 = std::min(2 * x + 1, a.w - 1), y1 = std::min(2 * y + 1, a.h - 1);
        mn(x, y) = std::min(std::min(a(2 * x, 2 * y), a(x1, 2 * y)), std::min(a(2 * x, y1), a(x1, y1)));
        mx(x, y) = std::max(std::max(b(2 * x, 2 * y), b(x1, 2 * y)), std::max(b(2 * x, y1), b(x1, y1)));
      }
    pmin.push_back(std::move(mn));
    pmax.push_back(std::move(mx));
  }
  for (int y = 0; y < hc; ++y)
    for (int x = 0; x < wc; ++x) {
      if (pmin[0](x, y) != inf) continue;
      for (size_t k = 1; k < pmin.size(); ++k) {
        const Img<float>& a = pmin[k];
        const Img<float>& b = pmax[k];
        const int bx = x >> k, by = y >> k;
        float mn = inf, mx = -inf;
        for (int qy = std::max(0, by - 1); qy <= std::min(a.h - 1, by + 1); ++qy)
          for (int qx = std::max(0, bx - 1); qx <= std::min(a.w - 1, bx + 1); ++qx) {
            mn = std::min(mn, a(qx, qy));
            mx = std::max(mx, b(qx, qy));
          }
        if (mn != inf) {
          cmin(x, y) = mn;
          cmax(x, y) = mx;
          break;
        }
      }
    }
  const int n_all = align16(nd);
  Ranges out{Img<uint16_t>(width, height), Img<uint16_t>(width, height)};
  const std::vector<Interval> pr_rows = intervals(partner_valid, partner_width, height);
  for (int y = 0; y < height; ++y) {
    const Interval pr = pr_rows[y];
    const int cy0 = y / 2, cy1 = std::min(cy0 + 1, hc - 1);
    for (int x = 0; x < width; ++x) {
      const int cx0 = x / 2, cx1 = std::min(cx0 + 1, wc - 1);
      const float mn = std::min(std::min(cmin(cx0, cy0), cmin(cx1, cy0)), std::min(cmin(cx0, cy1), cmin(cx1, cy1)));
      const float mx = std::max(std::max(cmax(cx0, cy0), cmax(cx1, cy0)), std::max(cmax(cx0, cy1), cmax(cx1, cy1)));
      int lo = 0, hi = n_all - 1;
      if (mn != inf) {
        lo = static_cast<int>(std::floor(2.0F * mn)) - dmin - o.range_margin;
        hi = static_cast<int>(std::ceil(2.0F * mx)) - dmin + o.range_margin;
      }
      const int mlo = (partner_sign < 0 ? x - pr.last : pr.first - x) - dmin;
      const int mhi = (partner_sign < 0 ? x - pr.first : pr.last - x) - dmin;
      lo = std::max(lo, mlo);
      hi = std::min(hi, mhi);
      if (lo > hi || pr.last < pr.first || (!fine_valid.empty() && fine_valid(x, y) < 128)) hi = lo;
      lo = std::clamp(lo, 0, n_all - 1);
      hi = std::clamp(hi, lo, n_all - 1);
      const int n = std::min(n_all, (hi - lo + 16) / 16 * 16);
      lo = std::clamp(lo - (n - (hi - lo + 1)) / 2, 0, n_all - n);
      const int xo = mirrored ? width - 1 - x : x;
      out.lo(xo, y) = static_cast<uint16_t>(lo);
      out.num(xo, y) = static_cast<uint16_t>(n);
    }
  }
  return out;
}

// ---------------------------------------------------------------- hierarchy
// stereo_matcher.cpp:889-890
int floor_shift(int v, int k) { return v >= 0 ? v >> k : -((-v + (1 << k) - 1) >> k); }
int ceil_shift(int v, int k) { return -floor_shift(-v, k); }

// stereo_matcher.cpp:1105-1122
int automatic_levels(int width, int height, int nd) {
  int levels = 0, w = width, h = height, n = nd;
  while (levels < 8) {
    const int nw = (w + 1) / 2, nh = (h + 1) / 2;
    if (std::min(nw, nh) < 96 || n <= 48) break;
    w = nw;
    h = nh;
    n = (n + 1) / 2;
    ++levels;
  }
  return levels;
}

struct Level {
  Img<uint16_t> left, right;
  Img<uint8_t> lv, rv;
  int dmin = 0, nd = 0;
};

struct LevelOut {
  Map left;
  Img<float> right;
};

// stereo_matcher.cpp:831-886
LevelOut match_level(const Level& in, const Ranges* lr, const Ranges* rr, bool need_right, int speckle, const Options& o) {
  Ctx ctx = make_ctx(in.left, in.right, in.lv, in.rv, in.dmin, in.nd, lr, o);
  const bool check_lr = o.lr_max_diff >= 0;
  ctx.diagonal_lr = check_lr && !o.lr_full_match;
  LevelOut out;
  out.left = match_tiles(ctx);
  if (check_lr && o.lr_full_match) {
    const int wl = in.left.w, wr = in.right.w;
    Ctx rctx = make_ctx(mirror(in.right), mirror(in.left), in.rv.empty() ? Img<uint8_t>() : mirror(in.rv),
                        in.lv.empty() ? Img<uint8_t>() : mirror(in.lv), in.dmin + wr - wl, in.nd, rr, o);
    rctx.diagonal_lr = false;
    rctx.confidence = false;
    Map rmap = match_tiles(rctx);
    out.left.cells += rmap.cells;
    out.right = Img<float>(wr, in.right.h);
    for (int y = 0; y < in.right.h; ++y)
      for (int x = 0; x < wr; ++x) out.right(x, y) = rmap.disp(wr - 1 - x, y) - static_cast<float>(wr - wl);
    if (need_right) {
      const std::vector<uint8_t> rbad = lr_mismatch(out.right, out.left.disp, 1, o.lr_max_diff);
      apply_bad(out.left.disp, lr_mismatch(out.left.disp, out.right, -1, o.lr_max_diff));
      apply_bad(out.right, rbad);
      post_filter(out.right, o, speckle);
    } else {
      apply_bad(out.left.disp, lr_mismatch(out.left.disp, out.right, -1, o.lr_max_diff));
      out.right = Img<float>();
    }
  }
  post_filter(out.left.disp, o, speckle);
  return out;
}

struct Result {
  Map map;
  int levels = 0, nd = 0;
};

// stereo_matcher.cpp:1023-1095
Result match_stereo(const Img<uint16_t>& left, const Img<uint16_t>& right, const Img<uint8_t>& lvalid,
                    const Img<uint8_t>& rvalid, int dmin, int nd, const Options& o) {
  check_options(o);
  if (nd <= 0) throw Failure("stereo: no disparities to search");
  const int levels = o.levels >= 0 ? o.levels : automatic_levels(left.w, left.h, nd);
  const bool lr_full = o.lr_max_diff >= 0 && o.lr_full_match;
  const int dmax = dmin + nd - 1;
  std::vector<Level> lv(levels + 1);
  lv[0].left = left;
  lv[0].right = right;
  lv[0].lv = lvalid;
  lv[0].rv = rvalid;
  for (int l = 1; l <= levels; ++l) {
    lv[l].left = pyramid_down(lv[l - 1].left);
    lv[l].right = pyramid_down(lv[l - 1].right);
    if (!lvalid.empty()) lv[l].lv = reduce_mask(lv[l - 1].lv);
    if (!rvalid.empty()) lv[l].rv = reduce_mask(lv[l - 1].rv);
  }
  for (int l = 0; l <= levels; ++l) {
    lv[l].dmin = floor_shift(dmin, l);
    lv[l].nd = align16(ceil_shift(dmax, l) - lv[l].dmin + 1);
  }
  LevelOut coarse;
  uint64_t cells = 0;
  for (int l = levels; l >= 0; --l) {
    const Level& in = lv[l];
    const int speckle = o.speckle_size >> (2 * l);
    if (l == levels) {
      coarse = match_level(in, nullptr, nullptr, lr_full && l > 0, speckle, o);
    } else {
      const Ranges lr = ranges_from_coarse(coarse.left.disp, in.left.w, in.left.h, in.lv, in.rv, in.right.w, -1,
                                           in.dmin, in.nd, o, false);
      Ranges rr;
      if (lr_full)
        rr = ranges_from_coarse(coarse.right, in.right.w, in.right.h, in.rv, in.lv, in.left.w, 1, in.dmin, in.nd, o, true);
      coarse = match_level(in, &lr, lr_full ? &rr : nullptr, lr_full && l > 0, speckle, o);
    }
    cells += coarse.left.cells;
  }
  Result r;
  r.map = std::move(coarse.left);
  r.map.cells = cells;
  r.levels = levels;
  r.nd = align16(nd);
  return r;
}

template <class F>
int guarded(F&& f) {
  try {
    g_error.clear();
    f();
    return 0;
  } catch (const Failure& e) {
    g_error = e.what();
    return 1;
  } catch (const std::bad_alloc&) {
    g_error = "out of memory";
    return 3;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 1;
  }
}

}  // namespace orc

// ---------------------------------------------------------------- C ABI (ctypes)
// ---------------------------------------------------------------- multi-view
// combine_pairs and sample_disparity (src/r3d/mvs/multi_stereo.cpp:44-216),
// in the reference's operation order; the geometry (Eigen-derived matrices in
// the reference) comes precomputed in r3dgpu_depth_grid / r3dgpu_pair_geometry.
namespace orc {

float sample_disparity(const r3dgpu_pair_geometry& g, double u, double v) {  // multi_stereo.cpp:44-72
  const int w = g.width, h = g.height;
  if (!(u > -0.5 && v > -0.5 && u < w - 0.5 && v < h - 0.5)) return kInvalid;
  const int x0 = std::clamp(static_cast<int>(std::floor(u)), 0, w - 1);
  const int y0 = std::clamp(static_cast<int>(std::floor(v)), 0, h - 1);
  const int x1 = std::min(x0 + 1, w - 1);
  const int y1 = std::min(y0 + 1, h - 1);
  auto at = [&](int x, int y) { return g.disparity[static_cast<int64_t>(y) * g.stride + x]; };
  const float d00 = at(x0, y0), d10 = at(x1, y0), d01 = at(x0, y1), d11 = at(x1, y1);
  if (std::isfinite(d00) && std::isfinite(d10) && std::isfinite(d01) && std::isfinite(d11)) {
    const float lo = std::min({d00, d10, d01, d11});
    const float hi = std::max({d00, d10, d01, d11});
    if (hi - lo <= 1.0F) {
      const auto fx = static_cast<float>(std::clamp(u - x0, 0.0, 1.0));
      const auto fy = static_cast<float>(std::clamp(v - y0, 0.0, 1.0));
      const float top = d00 + fx * (d10 - d00);
      const float bottom = d01 + fx * (d11 - d01);
      return top + fy * (bottom - top);
    }
  }
  const int xn = std::clamp(static_cast<int>(std::lround(u)), 0, w - 1);
  const int yn = std::clamp(static_cast<int>(std::lround(v)), 0, h - 1);
  return at(xn, yn);
}

// 3x3 (row-major) times (x, y, z), each row summed left to right.
void mat_vec(const double* m, double x, double y, double z, double* out) {
  for (int i = 0; i < 3; ++i) out[i] = m[3 * i] * x + m[3 * i + 1] * y + m[3 * i + 2] * z;
}

void normalize3(double* v) {
  const double n = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
  if (n > 0.0) {
    const double s = std::sqrt(n);
    for (int k = 0; k < 3; ++k) v[k] /= s;
  }
}

void combine_pairs(const r3dgpu_depth_grid& grid, const r3dgpu_pair_geometry* geo, int count,
                   const r3dgpu_multi_stereo_options& options, float* depth, float* confidence, uint16_t* mask,
                   int64_t stride) {  // multi_stereo.cpp:74-216
  constexpr int kMaxPairs = 16;
  if (count > kMaxPairs) throw Failure("combine_pairs: at most 16 pairs per view");
  struct Candidate {
    double w = 0.0, k = 0.0;
    float confidence = 0.0F;
    int pair = 0;
  };
  const double cos_min_angle = std::cos(options.min_angle_deg * 3.14159265358979323846 / 180.0);
  const int min_pairs = std::max(1, options.min_pairs);
  const int w = grid.width, h = grid.height;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 8)
#endif
  for (int yy = 0; yy < h; ++yy) {
    Candidate cand[kMaxPairs];
    int used[kMaxPairs];
    for (int x = 0; x < w; ++x) {
      const int64_t o = static_cast<int64_t>(yy) * stride + x;
      depth[o] = 0.0F;
      confidence[o] = 0.0F;
      mask[o] = 0;
      int n = 0;
      for (int i = 0; i < count; ++i) {
        const r3dgpu_pair_geometry& g = geo[i];
        double r[3];
        mat_vec(g.grid_to_rect, x, yy, 1.0, r);
        const double c = r[2];
        if (!(c > 1e-9)) continue;
        const double u = r[0] / c;
        const double v = r[1] / c;
        const float d = sample_disparity(g, u, v);
        if (!std::isfinite(d) || d <= g.offset) continue;
        Candidate& cd = cand[n++];
        cd.k = g.fb / c;
        cd.w = (d - g.offset) / cd.k;
        cd.pair = i;
        cd.confidence = 0.0F;
        if (g.confidence != nullptr) {
          const int xn = std::clamp(static_cast<int>(std::lround(u)), 0, g.width - 1);
          const int yn = std::clamp(static_cast<int>(std::lround(v)), 0, g.height - 1);
          cd.confidence = g.confidence[static_cast<int64_t>(yn) * g.stride + xn];
        }
      }
      if (n < min_pairs) continue;
      int best = -1, best_support = 0;
      float best_conf = -1.0F;
      for (int i = 0; i < n; ++i) {
        int support = 0;
        float conf = 0.0F;
        for (int j = 0; j < n; ++j) {
          if (std::abs(cand[j].k * (cand[j].w - cand[i].w)) <= options.inlier_px) {
            ++support;
            conf += cand[j].confidence;
          }
        }
        if (support > best_support || (support == best_support && conf > best_conf)) {
          best = i;
          best_support = support;
          best_conf = conf;
        }
      }
      int m = 0;
      for (int j = 0; j < n; ++j)
        if (std::abs(cand[j].k * (cand[j].w - cand[best].w)) <= options.inlier_px) used[m++] = j;
      double w_opt = 0.0;
      while (m > 0) {
        double sw = 0.0, swx = 0.0;
        for (int t = 0; t < m; ++t) {
          const Candidate& cd = cand[used[t]];
          sw += cd.k * cd.k;
          swx += cd.k * cd.k * cd.w;
        }
        w_opt = swx / sw;
        int worst = -1;
        double worst_res = options.max_reprojection_px;
        for (int t = 0; t < m; ++t) {
          const Candidate& cd = cand[used[t]];
          const double res = std::abs(cd.k * (cd.w - w_opt));
          if (res > worst_res) {
            worst_res = res;
            worst = t;
          }
        }
        if (worst < 0) break;
        used[worst] = used[--m];
      }
      const bool majority = m > n - m || (m >= 2 && m >= n - m);
      if (m < min_pairs || !majority || !(w_opt > 0.0)) continue;
      const double z = 1.0 / w_opt;
      double a[3], ray[3], xw[3], tb[3];
      mat_vec(grid.k_inv, x, yy, 1.0, a);
      mat_vec(grid.rot_t, a[0], a[1], a[2], ray);
      for (int k = 0; k < 3; ++k) xw[k] = grid.center[k] + z * ray[k];
      for (int k = 0; k < 3; ++k) tb[k] = grid.center[k] - xw[k];
      normalize3(tb);
      bool wide = false;
      float conf = 0.0F;
      uint16_t msk = 0;
      for (int t = 0; t < m; ++t) {
        const Candidate& cd = cand[used[t]];
        msk = static_cast<uint16_t>(msk | (1U << cd.pair));
        double tp[3];
        for (int k = 0; k < 3; ++k) tp[k] = geo[cd.pair].partner_center[k] - xw[k];
        normalize3(tp);
        wide = wide || (tb[0] * tp[0] + tb[1] * tp[1] + tb[2] * tp[2]) <= cos_min_angle;
        conf += cd.confidence;
      }
      if (!wide) continue;
      depth[o] = static_cast<float>(z);
      confidence[o] = conf / static_cast<float>(m);
      mask[o] = msk;
    }
  }
}

// ---------------------------------------------------------------- rectification
// rectify_image (src/r3d/rectify/rectification.cpp:287-350) for one-channel
// u16 and f32 images: pyramid level for anti-aliasing, target ray rotated
// into the source camera, projection through the camera model
// (src/r3d/core/camera_model.cpp:67-100, 148-151), Catmull-Rom bicubic
// sampling with clamped taps (src/r3d/core/sampling.hpp:15-55).

// pyramid.cpp:33-83 with float accumulators: sums of the horizontal pass kept
// per row, then the vertical pass, times 1/256.
Img<float> pyramid_down_f32(const Img<float>& s) {
  const int w = s.w, h = s.h, dw = (w + 1) / 2, dh = (h + 1) / 2;
  Img<float> tmp(dw, h);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < dw; ++x) {
      const int c = 2 * x;
      auto v = [&](int xx) { return s(std::clamp(xx, 0, w - 1), y); };
      tmp(x, y) = v(c - 2) + v(c + 2) + 4.0F * (v(c - 1) + v(c + 1)) + 6.0F * v(c);
    }
  Img<float> out(dw, dh);
  for (int y = 0; y < dh; ++y) {
    const int c = 2 * y;
    for (int x = 0; x < dw; ++x) {
      auto v = [&](int yy) { return tmp(x, std::clamp(yy, 0, h - 1)); };
      out(x, y) = (v(c - 2) + v(c + 2) + 4.0F * (v(c - 1) + v(c + 1)) + 6.0F * v(c)) * (1.0F / 256.0F);
    }
  }
  return out;
}

Img<uint16_t> level_down(const Img<uint16_t>& s) { return pyramid_down(s); }
Img<float> level_down(const Img<float>& s) { return pyramid_down_f32(s); }

// camera_model.cpp:67-100.
void distort(const r3dgpu_camera& c, double ux, double uy, double& dx, double& dy) {
  const double r2 = ux * ux + uy * uy;
  const double* p = c.params;
  dx = ux;
  dy = uy;
  if (c.model == 1) {
    dx = ux * (1.0 + p[0] * r2);
    dy = uy * (1.0 + p[0] * r2);
  } else if (c.model == 2) {
    const double f = 1.0 + r2 * (p[0] + r2 * (p[1] + r2 * p[2]));
    dx = ux * f;
    dy = uy * f;
  } else if (c.model == 3) {
    const double radial = r2 * (p[0] + r2 * (p[1] + r2 * p[2]));
    dx = ux + ux * radial + (p[4] * (r2 + 2.0 * ux * ux) + 2.0 * p[3] * ux * uy);
    dy = uy + uy * radial + (p[3] * (r2 + 2.0 * uy * uy) + 2.0 * p[4] * ux * uy);
  } else if (c.model == 4) {
    const double r = std::sqrt(r2);
    if (r > 1e-8) {
      const double th = std::atan(r), th2 = th * th;
      const double f = th * (1.0 + th2 * (p[0] + th2 * (p[1] + th2 * (p[2] + th2 * p[3])))) / r;
      dx = ux * f;
      dy = uy * f;
    }
  }
}

// sampling.hpp:21-26.
std::array<float, 4> cubic_weights(float t) {
  const float t2 = t * t, t3 = t2 * t;
  return {-0.5F * t3 + t2 - 0.5F * t, 1.5F * t3 - 2.5F * t2 + 1.0F, -1.5F * t3 + 2.0F * t2 + 0.5F * t,
          0.5F * t3 - 0.5F * t2};
}

// rectification.cpp:140-148.
template <class T>
T to_pixel(float v) {
  if constexpr (std::is_floating_point_v<T>) {
    return v;
  } else {
    return static_cast<T>(std::clamp(std::round(v), 0.0F, 65535.0F));
  }
}

template <class T>
void rectify(const Img<T>& src, const r3dgpu_camera& cam, const double* m, const r3dgpu_pinhole& k, T* out,
             uint8_t* valid) {
  if (src.w != cam.width || src.h != cam.height) throw Failure("rectify_image: image and camera sizes differ");
  int level = 0;
  while (cam.fx / k.fx > 1.5 * std::ldexp(1.0, level) && (cam.width >> (level + 1)) >= 16 &&
         (cam.height >> (level + 1)) >= 16)
    ++level;
  Img<T> img = src;
  for (int l = 0; l < level; ++l) img = level_down(img);
  r3dgpu_camera c = cam;
  const double scale = std::ldexp(1.0, -level);
  c.fx *= scale;
  c.fy *= scale;
  c.cx *= scale;
  c.cy *= scale;
#pragma omp parallel for schedule(static)
  for (int y = 0; y < k.height; ++y) {
    const double ry = (y - k.cy) / k.fy;
    for (int x = 0; x < k.width; ++x) {
      const double rx = (x - k.cx) / k.fx;
      double r[3];
      for (int i = 0; i < 3; ++i) r[i] = m[3 * i] * rx + m[3 * i + 1] * ry + m[3 * i + 2] * 1.0;
      bool inside = r[2] > 1e-9;
      double sx = 0.0, sy = 0.0;
      if (inside) {
        double dx, dy;
        distort(c, r[0] / r[2], r[1] / r[2], dx, dy);
        sx = c.fx * dx + c.cx;
        sy = c.fy * dy + c.cy;
        inside = sx >= -0.5 && sy >= -0.5 && sx <= img.w - 0.5 && sy <= img.h - 0.5;
      }
      T v{};
      if (inside) {
        const double flx = std::floor(sx), fly = std::floor(sy);
        const auto wx = cubic_weights(static_cast<float>(sx - flx));
        const auto wy = cubic_weights(static_cast<float>(sy - fly));
        const int x0 = static_cast<int>(flx) - 1, y0 = static_cast<int>(fly) - 1;
        float acc_y = 0.0F;
        for (int j = 0; j < 4; ++j) {
          const int yy = std::clamp(y0 + j, 0, img.h - 1);
          float acc = 0.0F;
          for (int i = 0; i < 4; ++i) acc += wx[i] * static_cast<float>(img(std::clamp(x0 + i, 0, img.w - 1), yy));
          acc_y += wy[j] * acc;
        }
        v = to_pixel<T>(acc_y);
      }
      out[static_cast<size_t>(y) * k.width + x] = v;
      if (valid != nullptr) valid[static_cast<size_t>(y) * k.width + x] = inside ? 255 : 0;
    }
  }
}

}  // namespace orc

extern "C" {

const char* orc_last_error() { return orc::g_error.c_str(); }

void orc_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n > 0 ? n : omp_get_num_procs());
#else
  (void)n;
#endif
}

int orc_max_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

int orc_census(const uint16_t* img, int w, int h, uint64_t* out) {
  return orc::guarded([&] {
    const auto c = orc::census(orc::wrap(img, w, h));
    std::copy(c.px.begin(), c.px.end(), out);
  });
}

int orc_pyramid_down_u16(const uint16_t* img, int w, int h, uint16_t* out) {
  return orc::guarded([&] {
    if (w <= 0 || h <= 0) throw orc::Failure("pyramid_down: empty image");
    const auto p = orc::pyramid_down(orc::wrap(img, w, h));
    std::copy(p.px.begin(), p.px.end(), out);
  });
}

int orc_pyramid_down_u8(const uint8_t* img, int w, int h, uint8_t* out) {
  return orc::guarded([&] {
    if (w <= 0 || h <= 0) throw orc::Failure("pyramid_down: empty image");
    const auto p = orc::pyramid_down(orc::wrap(img, w, h));
    std::copy(p.px.begin(), p.px.end(), out);
  });
}

int orc_automatic_levels(int w, int h, int nd) { return orc::automatic_levels(w, h, nd); }

// Whole image as one tile (stereo_matcher.cpp:1269-1278) or the textbook
// volume (1280-1362); identical by construction here, both entries exist so
// that the tests can state the reference's identity.
int orc_sgm_cost_volume(const uint16_t* left, int wl, int h, const uint16_t* right, int wr, int dmin, int nd,
                        const r3dgpu_stereo_options* o, const uint16_t* rlo, const uint16_t* rnum, uint16_t* out,
                        uint64_t cap, uint64_t* count) {
  return orc::guarded([&] {
    orc::Ranges R;
    const orc::Ranges* rp = nullptr;
    if (rlo && rnum) {
      R.lo = orc::wrap(rlo, wl, h);
      R.num = orc::wrap(rnum, wl, h);
      rp = &R;
    }
    orc::Ctx c = orc::make_ctx(orc::wrap(left, wl, h), orc::wrap(right, wr, h), {}, {}, dmin, nd, rp, *o);
    orc::Tile t{0, 0, wl, h, 0, wl, 0, h};
    const orc::TileLabels L = orc::tile_labels(c, t);
    const auto S = orc::aggregate_tile(c, t, L);
    *count = S.size();
    if (out) {
      if (cap < S.size()) throw orc::Failure("sgm_cost_volume: output too small");
      std::copy(S.begin(), S.end(), out);
    }
  });
}

int orc_ranges_from_coarse(const float* coarse, int wc, int hc, int w, int h, const uint8_t* fine_valid,
                           const uint8_t* partner_valid, int partner_width, int partner_sign, int dmin, int nd,
                           const r3dgpu_stereo_options* o, int mirrored, uint16_t* lo, uint16_t* num) {
  return orc::guarded([&] {
    const auto r = orc::ranges_from_coarse(orc::wrap(coarse, wc, hc), w, h, orc::wrap(fine_valid, w, h),
                                           orc::wrap(partner_valid, partner_width, h), partner_width, partner_sign,
                                           dmin, nd, *o, mirrored != 0);
    std::copy(r.lo.px.begin(), r.lo.px.end(), lo);
    std::copy(r.num.px.begin(), r.num.px.end(), num);
  });
}

int orc_remove_speckles(float* d, int w, int h, int min_size, float max_diff) {
  return orc::guarded([&] {
    auto m = orc::wrap(d, w, h);
    orc::remove_speckles(m, min_size, max_diff);
    std::copy(m.px.begin(), m.px.end(), d);
  });
}

int orc_median_filter_3x3(const float* d, int w, int h, float* out) {
  return orc::guarded([&] {
    const auto m = orc::median3x3(orc::wrap(d, w, h));
    std::copy(m.px.begin(), m.px.end(), out);
  });
}

// r3d::match_stereo; masks may be NULL (all valid). meta[0] = levels,
// meta[1] = aligned label count, meta[2] = aggregated cells.
int orc_match_stereo(const uint16_t* left, int wl, int h, const uint16_t* right, int wr, const uint8_t* lvalid,
                     const uint8_t* rvalid, int dmin, int nd, const r3dgpu_stereo_options* o, float* disp, float* conf,
                     int64_t* meta) {
  return orc::guarded([&] {
    const auto r = orc::match_stereo(orc::wrap(left, wl, h), orc::wrap(right, wr, h), orc::wrap(lvalid, wl, h),
                                     orc::wrap(rvalid, wr, h), dmin, nd, *o);
    std::copy(r.map.disp.px.begin(), r.map.disp.px.end(), disp);
    if (conf) std::copy(r.map.conf.px.begin(), r.map.conf.px.end(), conf);
    meta[0] = r.levels;
    meta[1] = r.nd;
    meta[2] = static_cast<int64_t>(r.map.cells);
  });
}

// One level's left match before checks and filters (tiles, selection and
// blending only), for localising a mismatch.
int orc_match_tiles(const uint16_t* left, int wl, int h, const uint16_t* right, int wr, const uint8_t* lvalid,
                    const uint8_t* rvalid, int dmin, int nd, const r3dgpu_stereo_options* o, const uint16_t* rlo,
                    const uint16_t* rnum, int diagonal_lr, float* disp, float* conf, uint64_t* cells) {
  return orc::guarded([&] {
    orc::Ranges R;
    const orc::Ranges* rp = nullptr;
    if (rlo && rnum) {
      R.lo = orc::wrap(rlo, wl, h);
      R.num = orc::wrap(rnum, wl, h);
      rp = &R;
    }
    orc::Ctx c = orc::make_ctx(orc::wrap(left, wl, h), orc::wrap(right, wr, h), orc::wrap(lvalid, wl, h),
                               orc::wrap(rvalid, wr, h), dmin, nd, rp, *o);
    c.diagonal_lr = diagonal_lr != 0;
    const auto m = orc::match_tiles(c);
    std::copy(m.disp.px.begin(), m.disp.px.end(), disp);
    if (conf) std::copy(m.conf.px.begin(), m.conf.px.end(), conf);
    *cells = m.cells;
  });
}

// combine_pairs on host maps (pairs' disparity/confidence pointers are host pointers).
int orc_combine_pairs(const r3dgpu_depth_grid* grid, const r3dgpu_pair_geometry* pairs, int count,
                      const r3dgpu_multi_stereo_options* options, float* depth, float* confidence, uint16_t* mask,
                      int64_t stride) {
  return orc::guarded([&] { orc::combine_pairs(*grid, pairs, count, *options, depth, confidence, mask, stride); });
}

// rectify_image of a contiguous host image (u16, or f32 when is_float) into
// contiguous host outputs; `valid` may be NULL.
int orc_rectify_image(int is_float, const void* src, const r3dgpu_camera* cam, const double* m,
                      const r3dgpu_pinhole* k, void* out, uint8_t* valid) {
  return orc::guarded([&] {
    if (is_float)
      orc::rectify(orc::wrap(static_cast<const float*>(src), cam->width, cam->height), *cam, m, *k,
                   static_cast<float*>(out), valid);
    else
      orc::rectify(orc::wrap(static_cast<const uint16_t*>(src), cam->width, cam->height), *cam, m, *k,
                   static_cast<uint16_t*>(out), valid);
  });
}

// distort_pixel (src/r3d/core/camera_model.cpp:142-146) at n pixels
// (xy pairs), for the camera-model golden vectors.
int orc_distort_pixel(const r3dgpu_camera* cam, const double* px, int n, double* out) {
  return orc::guarded([&] {
    for (int i = 0; i < n; ++i) {
      double dx, dy;
      orc::distort(*cam, (px[2 * i] - cam->cx) / cam->fx, (px[2 * i + 1] - cam->cy) / cam->fy, dx, dy);
      out[2 * i] = cam->fx * dx + cam->cx;
      out[2 * i + 1] = cam->fy * dy + cam->cy;
    }
  });
}

// sample_disparity at n positions.
int orc_sample_disparity(const float* disp, int w, int h, const double* u, const double* v, int n, float* out) {
  return orc::guarded([&] {
    r3dgpu_pair_geometry g{};
    g.disparity = disp;
    g.width = w;
    g.height = h;
    g.stride = w;
    for (int i = 0; i < n; ++i) out[i] = orc::sample_disparity(g, u[i], v[i]);
  });
}

}  // extern "C"
