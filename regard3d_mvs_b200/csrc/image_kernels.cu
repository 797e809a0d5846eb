// Per-pixel image kernels of the matcher: Census, pyramid, masks, left-right
// check, speckle filter, median filter, label ranges and tile blending.
// Float arithmetic is written operation by operation with round-to-nearest
// intrinsics (no contraction), so results equal the reference's scalar code.
#include <cmath>
#include <cstdint>

#include "common.cuh"
#include "kernels.h"

namespace r3dgpu {

namespace {

constexpr float kInf = __builtin_huge_valf();

R3D_DEVICE int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ------------------------------------------------------------------ census
// 9x7 Census (census.cpp:20-35, 104-113): the 62 neighbours in raster order,
// first in bit 61, bit = neighbour < centre; borders replicated.
constexpr int kCBX = 32, kCBY = 8;

R3D_GLOBAL void R3D_LAUNCH_BOUNDS(kCBX* kCBY) census_kernel(const uint16_t* __restrict__ img, int64_t stride, int w,
                                                           int h, uint64_t* __restrict__ out, int64_t ostride) {
  R3D_DYNAMIC_SMEM(smem_raw);
  auto tile = reinterpret_cast<uint16_t(*)[kCBX + 8]>(smem_raw);
  const int x0 = blockIdx.x * kCBX, y0 = blockIdx.y * kCBY;
  for (int i = threadIdx.y * kCBX + threadIdx.x; i < (kCBY + 6) * (kCBX + 8); i += kCBX * kCBY) {
    const int ty = i / (kCBX + 8), tx = i % (kCBX + 8);
    const int gx = clampi(x0 + tx - 4, 0, w - 1), gy = clampi(y0 + ty - 3, 0, h - 1);
    tile[ty][tx] = img[static_cast<int64_t>(gy) * stride + gx];
  }
  r3dsimt::syncthreads();
  const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
  if (x >= w || y >= h) return;
  const uint16_t c = tile[threadIdx.y + 3][threadIdx.x + 4];
  uint64_t bits = 0;
#pragma unroll
  for (int j = 0; j < 7; ++j) {
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      if (j == 3 && i == 4) continue;
      bits = (bits << 1) | static_cast<uint64_t>(tile[threadIdx.y + j][threadIdx.x + i] < c);
    }
  }
  out[static_cast<int64_t>(y) * ostride + x] = bits;
}

// ------------------------------------------------------------------ pyramid
// [1 4 6 4 1]^2 / 256 with clamped borders and exact rounding (pyramid.cpp:33-85).
template <class T>
R3D_DEVICE uint32_t pyr_sum(const T* __restrict__ in, int64_t stride, int w, int h, int x, int y) {
  const int wt[5] = {1, 4, 6, 4, 1};
  uint32_t acc = 0;
#pragma unroll
  for (int j = 0; j < 5; ++j) {
    const T* row = in + static_cast<int64_t>(clampi(2 * y + j - 2, 0, h - 1)) * stride;
    uint32_t hs = 0;
#pragma unroll
    for (int i = 0; i < 5; ++i) hs += wt[i] * static_cast<uint32_t>(row[clampi(2 * x + i - 2, 0, w - 1)]);
    acc += wt[j] * hs;
  }
  return acc;
}

R3D_GLOBAL void pyramid_u16_kernel(const uint16_t* __restrict__ in, int64_t istride, int w, int h,
                                   uint16_t* __restrict__ out, int64_t ostride, int dw, int dh) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= dw || y >= dh) return;
  out[static_cast<int64_t>(y) * ostride + x] = static_cast<uint16_t>((pyr_sum(in, istride, w, h, x, y) + 128u) >> 8);
}

R3D_GLOBAL void reduce_mask_kernel(const uint8_t* __restrict__ in, int64_t istride, int w, int h,
                                   uint8_t* __restrict__ out, int64_t ostride, int dw, int dh) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= dw || y >= dh) return;
  const uint32_t v = (pyr_sum(in, istride, w, h, x, y) + 128u) >> 8;
  out[static_cast<int64_t>(y) * ostride + x] = v >= 128u ? 255 : 0;
}

template <class T>
R3D_GLOBAL void mirror_kernel(const T* __restrict__ in, int64_t istride, int w, int h, T* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  out[static_cast<int64_t>(y) * w + x] = in[static_cast<int64_t>(y) * istride + (w - 1 - x)];
}

// ------------------------------------------------------------------ row intervals
// stereo_matcher.cpp:43-67: one warp per row finds the first and last column
// with mask >= 128.
R3D_GLOBAL void intervals_kernel(const uint8_t* __restrict__ mask, int64_t stride, int w, int h,
                                 RowInterval* __restrict__ out) {
  const int y = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (y >= h) return;
  if (mask == nullptr) {
    if (lane == 0) out[y] = RowInterval{0, w - 1};
    return;
  }
  const uint8_t* row = mask + static_cast<int64_t>(y) * stride;
  int first = w, last = -1;
  for (int x = lane; x < w; x += 32) {
    if (row[x] >= 128) {
      first = r3dsimt::imin(first, x);
      last = r3dsimt::imax(last, x);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    first = r3dsimt::imin(first, static_cast<int>(r3dsimt::shfl_xor(static_cast<uint32_t>(first), o)));
    last = r3dsimt::imax(last, static_cast<int>(r3dsimt::shfl_xor(static_cast<uint32_t>(last), o)));
  }
  if (lane == 0) out[y] = first < w ? RowInterval{first, last} : RowInterval{0, -1};
}

// ------------------------------------------------------------------ left-right check
// stereo_matcher.cpp:777-805: xo = lround(x + sign * d); mismatch if the other
// map is invalid there or differs by more than max_diff.
R3D_GLOBAL void lr_check_kernel(const float* __restrict__ map, const float* __restrict__ other, int w, int h, int wo,
                                int sign, int max_diff, uint8_t* __restrict__ bad) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  const float d = map[static_cast<int64_t>(y) * w + x];
  uint8_t b = 0;
  if (r3dsimt::finitef(d)) {
    const float pos = __fadd_rn(static_cast<float>(x), __fmul_rn(static_cast<float>(sign), d));
    const long xo = lroundf(pos);
    const float dother = xo >= 0 && xo < wo ? other[static_cast<int64_t>(y) * wo + xo] : kInf;
    b = (!r3dsimt::finitef(dother) || fabsf(__fsub_rn(d, dother)) > static_cast<float>(max_diff)) ? 1 : 0;
  }
  bad[static_cast<int64_t>(y) * w + x] = b;
}

R3D_GLOBAL void apply_bad_kernel(float* __restrict__ map, const uint8_t* __restrict__ bad, int64_t n) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n && bad[i]) map[i] = kInf;
}

// ------------------------------------------------------------------ speckles
// Segments of 4-neighbours whose disparities differ by at most max_diff
// (stereo_matcher.cpp:919-970) are the connected components of that
// symmetric relation; they are found with a lock-free union-find (roots are
// always the smallest index of a set, so every pointer chain decreases).
R3D_DEVICE int uf_root(const int* parent, int x) {
  int p = __ldcg(parent + x);
  while (p != x) {
    x = p;
    p = __ldcg(parent + x);
  }
  return x;
}

R3D_DEVICE void uf_unite(int* parent, int a, int b) {
  while (true) {
    a = uf_root(parent, a);
    b = uf_root(parent, b);
    if (a == b) return;
    if (a > b) {
      const int t = a;
      a = b;
      b = t;
    }
    const int old = atomicCAS(parent + b, b, a);
    if (old == b) return;
    b = old;
  }
}

// Tiles of 32 x 32 pixels are united in shared memory first (local indices
// in row-major order, so a local root is also the smallest global index of
// its part of the segment); only pixels on tile borders then unite across
// tiles in global memory.
constexpr int kUfTile = 32;

R3D_DEVICE int uf_root_local(volatile int* par, int x) {
  int p = par[x];
  while (p != x) {
    x = p;
    p = par[x];
  }
  return x;
}

R3D_DEVICE void uf_unite_local(int* par, int a, int b) {
  while (true) {
    a = uf_root_local(par, a);
    b = uf_root_local(par, b);
    if (a == b) return;
    if (a > b) {
      const int t = a;
      a = b;
      b = t;
    }
    const int old = atomicCAS(par + b, b, a);
    if (old == b) return;
    b = old;
  }
}

// Per tile: local union, then parent[p] = global index of p's local root and
// size[p] = 0 for every pixel of the tile.
R3D_GLOBAL void uf_tile_kernel(const float* __restrict__ d, int w, int h, float max_diff, int* parent, int* size) {
  R3D_DYNAMIC_SMEM(smem);
  int* par = reinterpret_cast<int*>(smem);
  float* dv = reinterpret_cast<float*>(smem + sizeof(int) * kUfTile * kUfTile);
  const int tx0 = static_cast<int>(blockIdx.x) * kUfTile, ty0 = static_cast<int>(blockIdx.y) * kUfTile;
  const int tw = r3dsimt::imin(kUfTile, w - tx0), th = r3dsimt::imin(kUfTile, h - ty0);
  const int nt = static_cast<int>(blockDim.x);
  for (int i = static_cast<int>(threadIdx.x); i < kUfTile * kUfTile; i += nt) {
    const int lx = i % kUfTile, ly = i / kUfTile;
    par[i] = i;
    dv[i] = (lx < tw && ly < th) ? d[static_cast<int64_t>(ty0 + ly) * w + tx0 + lx] : kInf;
  }
  r3dsimt::syncthreads();
  for (int i = static_cast<int>(threadIdx.x); i < kUfTile * kUfTile; i += nt) {
    const int lx = i % kUfTile, ly = i / kUfTile;
    const float v = dv[i];
    if (lx >= tw || ly >= th || !r3dsimt::finitef(v)) continue;
    if (lx + 1 < tw && fabsf(__fsub_rn(dv[i + 1], v)) <= max_diff) uf_unite_local(par, i, i + 1);
    if (ly + 1 < th && fabsf(__fsub_rn(dv[i + kUfTile], v)) <= max_diff) uf_unite_local(par, i, i + kUfTile);
  }
  r3dsimt::syncthreads();
  for (int i = static_cast<int>(threadIdx.x); i < kUfTile * kUfTile; i += nt) {
    const int lx = i % kUfTile, ly = i / kUfTile;
    if (lx >= tw || ly >= th) continue;
    const int r = uf_root_local(par, i);
    const int64_t g = static_cast<int64_t>(ty0 + ly) * w + tx0 + lx;
    parent[g] = (ty0 + r / kUfTile) * w + tx0 + r % kUfTile;
    size[g] = 0;
  }
}

// Unions across tile borders: the pixel pairs straddling a vertical tile
// boundary, then those straddling a horizontal one.
R3D_GLOBAL void uf_border_kernel(const float* __restrict__ d, int w, int h, float max_diff, int* parent) {
  const int64_t nvx = static_cast<int64_t>((w - 1) / kUfTile) * h;  // vertical boundaries x all rows
  const int64_t nhy = static_cast<int64_t>((h - 1) / kUfTile) * w;  // horizontal boundaries x all columns
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  int a = -1, b = -1;
  if (i < nvx) {
    const int y = static_cast<int>(i % h), k = static_cast<int>(i / h);
    const int x = (k + 1) * kUfTile - 1;
    a = y * w + x;
    b = a + 1;
  } else if (i < nvx + nhy) {
    const int64_t j = i - nvx;
    const int x = static_cast<int>(j % w), k = static_cast<int>(j / w);
    const int y = (k + 1) * kUfTile - 1;
    a = y * w + x;
    b = a + w;
  } else {
    return;
  }
  const float u = d[a], v = d[b];
  if (r3dsimt::finitef(u) && fabsf(__fsub_rn(v, u)) <= max_diff) uf_unite(parent, a, b);
}

// Segment sizes: the lanes of a warp whose pixels share a root add their
// count with one atomic; every pixel's parent becomes its root.
R3D_GLOBAL void uf_count_kernel(const float* __restrict__ d, int64_t n, int* parent, int* size) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const bool ok = i < n && r3dsimt::finitef(d[i]);
  const int r = ok ? uf_root(parent, static_cast<int>(i)) : -1;
  const uint32_t peers = r3dsimt::match_any(static_cast<uint32_t>(r));
  if (ok) {
    parent[i] = r;
    if (static_cast<int>(r3dsimt::lane_id()) == r3dsimt::ffs(peers) - 1)
      atomicAdd(size + r, r3dsimt::popc64(peers));
  }
}

R3D_GLOBAL void uf_filter_kernel(float* __restrict__ d, int64_t n, const int* parent, const int* size, int min_size) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n || !r3dsimt::finitef(d[i])) return;
  const int r = uf_root(parent, static_cast<int>(i));
  if (__ldcg(size + r) < min_size) d[i] = kInf;
}

// ------------------------------------------------------------------ median
// stereo_matcher.cpp:972-1021: median of the valid values of the 3x3
// neighbourhood; an even count averages the two middle values.
R3D_GLOBAL void median_kernel(const float* __restrict__ in, int w, int h, float* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  const float c = in[static_cast<int64_t>(y) * w + x];
  if (!r3dsimt::finitef(c)) {
    out[static_cast<int64_t>(y) * w + x] = c;
    return;
  }
  float v[9];
  int n = 0;
#pragma unroll
  for (int dy = -1; dy <= 1; ++dy) {
#pragma unroll
    for (int dx = -1; dx <= 1; ++dx) {
      const int qx = x + dx, qy = y + dy;
      if (qx >= 0 && qy >= 0 && qx < w && qy < h) {
        const float q = in[static_cast<int64_t>(qy) * w + qx];
        if (r3dsimt::finitef(q)) v[n++] = q;
      }
    }
  }
  for (int a = 1; a < n; ++a) {
    const float key = v[a];
    int b = a - 1;
    while (b >= 0 && v[b] > key) {
      v[b + 1] = v[b];
      --b;
    }
    v[b + 1] = key;
  }
  float m = v[n / 2];
  if ((n & 1) == 0) m = __fmul_rn(0.5F, __fadd_rn(m, v[n / 2 - 1]));
  out[static_cast<int64_t>(y) * w + x] = m;
}

R3D_GLOBAL void unmirror_offset_kernel(const float* __restrict__ in, int w, int h, float offset,
                                       float* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  out[static_cast<int64_t>(y) * w + x] = __fsub_rn(in[static_cast<int64_t>(y) * w + (w - 1 - x)], offset);
}

R3D_GLOBAL void copy2d_kernel(const float* __restrict__ in, int64_t istride, int w, int h, float* __restrict__ out,
                              int64_t ostride) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  out[static_cast<int64_t>(y) * ostride + x] = in[static_cast<int64_t>(y) * istride + x];
}

// ------------------------------------------------------------------ ranges
// stereo_matcher.cpp:1124-1267.
R3D_GLOBAL void range_hminmax_kernel(const float* __restrict__ coarse, int wc, int hc, int r, float* __restrict__ hmin,
                                     float* __restrict__ hmax) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= wc || y >= hc) return;
  float mn = kInf, mx = -kInf;
  const int k1 = r3dsimt::imin(wc - 1, x + r);
  for (int k = r3dsimt::imax(0, x - r); k <= k1; ++k) {
    const float v = coarse[y * wc + k];
    if (r3dsimt::finitef(v)) {
      mn = fminf(mn, v);
      mx = fmaxf(mx, v);
    }
  }
  hmin[y * wc + x] = mn;
  hmax[y * wc + x] = mx;
}

R3D_GLOBAL void range_vminmax_kernel(const float* __restrict__ hmin, const float* __restrict__ hmax, int wc, int hc,
                                     int r, float* __restrict__ cmin, float* __restrict__ cmax,
                                     float* __restrict__ pmin0, float* __restrict__ pmax0) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= wc || y >= hc) return;
  float mn = kInf, mx = -kInf;
  const int k1 = r3dsimt::imin(hc - 1, y + r);
  for (int k = r3dsimt::imax(0, y - r); k <= k1; ++k) {
    mn = fminf(mn, hmin[k * wc + x]);
    mx = fmaxf(mx, hmax[k * wc + x]);
  }
  cmin[y * wc + x] = mn;
  cmax[y * wc + x] = mx;
  pmin0[y * wc + x] = mn;
  pmax0[y * wc + x] = mx;
}

R3D_GLOBAL void range_pyr_kernel(const float* __restrict__ amin, const float* __restrict__ amax, int aw, int ah,
                                 float* __restrict__ omin, float* __restrict__ omax, int nw, int nh) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= nw || y >= nh) return;
  const int x1 = r3dsimt::imin(2 * x + 1, aw - 1), y1 = r3dsimt::imin(2 * y + 1, ah - 1);
  omin[y * nw + x] = fminf(fminf(amin[2 * y * aw + 2 * x], amin[2 * y * aw + x1]),
                           fminf(amin[y1 * aw + 2 * x], amin[y1 * aw + x1]));
  omax[y * nw + x] = fmaxf(fmaxf(amax[2 * y * aw + 2 * x], amax[2 * y * aw + x1]),
                           fmaxf(amax[y1 * aw + 2 * x], amax[y1 * aw + x1]));
}

struct PyrLevels {
  const float* mn[16];
  const float* mx[16];
  int w[16], h[16];
  int count;
};

R3D_GLOBAL void range_fill_kernel(PyrLevels p, int wc, int hc, float* __restrict__ cmin, float* __restrict__ cmax) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= wc || y >= hc) return;
  if (p.mn[0][y * wc + x] != kInf) return;
  for (int k = 1; k < p.count; ++k) {
    const int bx = x >> k, by = y >> k, aw = p.w[k], ah = p.h[k];
    float mn = kInf, mx = -kInf;
    for (int qy = r3dsimt::imax(0, by - 1); qy <= r3dsimt::imin(ah - 1, by + 1); ++qy)
      for (int qx = r3dsimt::imax(0, bx - 1); qx <= r3dsimt::imin(aw - 1, bx + 1); ++qx) {
        mn = fminf(mn, p.mn[k][qy * aw + qx]);
        mx = fmaxf(mx, p.mx[k][qy * aw + qx]);
      }
    if (mn != kInf) {
      cmin[y * wc + x] = mn;
      cmax[y * wc + x] = mx;
      return;
    }
  }
}

R3D_GLOBAL void range_final_kernel(const float* __restrict__ cmin, const float* __restrict__ cmax, int wc, int hc,
                                   int w, int h, const uint8_t* __restrict__ fine_valid, int64_t fv_stride,
                                   const RowInterval* __restrict__ prow, RangeParams p, uint16_t* __restrict__ lo_out,
                                   uint16_t* __restrict__ num_out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  const RowInterval pr = prow[y];
  const int cy0 = y / 2, cy1 = r3dsimt::imin(cy0 + 1, hc - 1), cx0 = x / 2, cx1 = r3dsimt::imin(cx0 + 1, wc - 1);
  const float mn = fminf(fminf(cmin[cy0 * wc + cx0], cmin[cy0 * wc + cx1]), fminf(cmin[cy1 * wc + cx0], cmin[cy1 * wc + cx1]));
  const float mx = fmaxf(fmaxf(cmax[cy0 * wc + cx0], cmax[cy0 * wc + cx1]), fmaxf(cmax[cy1 * wc + cx0], cmax[cy1 * wc + cx1]));
  int lo = 0, hi = p.n_all - 1;
  if (mn != kInf) {
    lo = static_cast<int>(floorf(__fmul_rn(2.0F, mn))) - p.dmin - p.margin;
    hi = static_cast<int>(ceilf(__fmul_rn(2.0F, mx))) - p.dmin + p.margin;
  }
  const int mlo = (p.partner_sign < 0 ? x - pr.last : pr.first - x) - p.dmin;
  const int mhi = (p.partner_sign < 0 ? x - pr.first : pr.last - x) - p.dmin;
  lo = r3dsimt::imax(lo, mlo);
  hi = r3dsimt::imin(hi, mhi);
  if (lo > hi || pr.last < pr.first || (fine_valid != nullptr && fine_valid[static_cast<int64_t>(y) * fv_stride + x] < 128))
    hi = lo;
  lo = clampi(lo, 0, p.n_all - 1);
  hi = clampi(hi, lo, p.n_all - 1);
  const int n = r3dsimt::imin(p.n_all, (hi - lo + 16) / 16 * 16);
  lo = clampi(lo - (n - (hi - lo + 1)) / 2, 0, p.n_all - n);
  const int xo = p.mirrored ? w - 1 - x : x;
  lo_out[static_cast<int64_t>(y) * w + xo] = static_cast<uint16_t>(lo);
  num_out[static_cast<int64_t>(y) * w + xo] = static_cast<uint16_t>(n);
}

// ------------------------------------------------------------------ blend
// stereo_matcher.cpp:530-543
R3D_DEVICE float axis_weight(int v, int c0, int c1, int size, int blend_px) {
  const float blend = static_cast<float>(blend_px);
  float w = 1.0F;
  const float pos = __fadd_rn(static_cast<float>(v), 0.5F);
  if (c0 > 0) {
    float t;
    if (blend_px > 0) {
      t = __fdiv_rn(__fadd_rn(__fsub_rn(pos, static_cast<float>(c0)), __fmul_rn(0.5F, blend)), blend);
      t = fminf(fmaxf(t, 0.0F), 1.0F);
    } else {
      t = v >= c0 ? 1.0F : 0.0F;
    }
    w = fminf(w, t);
  }
  if (c1 < size) {
    float t;
    if (blend_px > 0) {
      t = __fdiv_rn(__fsub_rn(__fadd_rn(static_cast<float>(c1), __fmul_rn(0.5F, blend)), pos), blend);
      t = fminf(fmaxf(t, 0.0F), 1.0F);
    } else {
      t = v < c1 ? 1.0F : 0.0F;
    }
    w = fminf(w, t);
  }
  return w;
}

// stereo_matcher.cpp:700-766: weighted mean over the tiles covering a pixel,
// accumulated in tile-index order; valid if the valid weight is at least half
// of all weight; the dominant tile wins when the mean is more than 1 px away.
R3D_GLOBAL void blend_kernel(const BlendTile* __restrict__ tiles, int ntiles, int tiles_x, int w, int h, int blend,
                             int mirror_out, float offset, float* __restrict__ out_disp, float* __restrict__ out_conf,
                             int64_t ostride) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  float wsum = 0.0F, wall = 0.0F, dsum = 0.0F, csum = 0.0F, wbest = 0.0F, dbest = kInf;
  const int tiles_y = ntiles / tiles_x;
  for (int j = 0; j < tiles_y; ++j) {
    const BlendTile& t0 = tiles[j * tiles_x];
    if (y < t0.y0 || y >= t0.y0 + t0.h) continue;
    const float wy = axis_weight(y, t0.c0y, t0.c1y, h, blend);
    if (wy <= 0.0F) continue;
    for (int i = 0; i < tiles_x; ++i) {
      const BlendTile& t = tiles[j * tiles_x + i];
      if (x < t.x0 || x >= t.x0 + t.w) continue;
      const float wg = __fmul_rn(wy, axis_weight(x, t.c0x, t.c1x, w, blend));
      if (wg <= 0.0F) continue;
      const int64_t ti = static_cast<int64_t>(y - t.y0) * t.w + (x - t.x0);
      wall = __fadd_rn(wall, wg);
      const float dv = t.disp[ti];
      if (r3dsimt::finitef(dv)) {
        wsum = __fadd_rn(wsum, wg);
        dsum = __fadd_rn(dsum, __fmul_rn(wg, dv));
        if (out_conf != nullptr) csum = __fadd_rn(csum, __fmul_rn(wg, t.conf[ti]));
        if (wg > wbest) {
          wbest = wg;
          dbest = dv;
        }
      }
    }
  }
  float dv = kInf, cv = 0.0F;
  if (wsum > 0.0F && wsum >= __fmul_rn(0.5F, wall)) {
    dv = __fdiv_rn(dsum, wsum);
    if (fabsf(__fsub_rn(dv, dbest)) > 1.0F) dv = dbest;
    if (out_conf != nullptr) cv = __fdiv_rn(csum, wsum);
  }
  const int xo = mirror_out ? w - 1 - x : x;
  out_disp[static_cast<int64_t>(y) * ostride + xo] = __fsub_rn(dv, offset);
  if (out_conf != nullptr) out_conf[static_cast<int64_t>(y) * ostride + xo] = cv;
}

// ------------------------------------------------------------------ tile cells
R3D_GLOBAL void tile_cells_kernel(const uint16_t* R3D_RESTRICT rnum, int64_t stride, const int4* R3D_RESTRICT tiles,
                                  unsigned long long* R3D_RESTRICT cells, int* R3D_RESTRICT stats) {
  R3D_DYNAMIC_SMEM(smem_raw);
  unsigned long long* ssum = reinterpret_cast<unsigned long long*>(smem_raw);
  int* sst = reinterpret_cast<int*>(smem_raw + 8 * 32);  // [warp][kTileStats]
  // Block (tile, slice): the slice's rows of the tile, a warp per row, the
  // lanes over its columns; the slices' results meet in atomics (the
  // launcher zeroes the outputs).
  const int4 t = tiles[blockIdx.x];
  unsigned long long s = 0;
  int st[kTileStats] = {};
  const int nwarps = static_cast<int>(blockDim.x >> 5);
  for (int y = static_cast<int>(blockIdx.y) * nwarps + static_cast<int>(threadIdx.x >> 5); y < t.w;
       y += static_cast<int>(gridDim.y) * nwarps) {
    const uint16_t* row = rnum + static_cast<int64_t>(t.y + y) * stride + t.x;
    for (int x = static_cast<int>(threadIdx.x & 31u); x < t.z; x += 32) {
      const int v = row[x];
      s += static_cast<unsigned long long>(v);
      st[0] = r3dsimt::imax(st[0], v);
#pragma unroll
      for (int k = 1; k < kTileStats; ++k) st[k] += v > tile_stat_width(k - 1) ? 1 : 0;
    }
  }
  // Warp reduction (64-bit sum as two 32-bit halves), then across warps.
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const uint32_t lo = r3dsimt::shfl_xor(static_cast<uint32_t>(s), o);
    const uint32_t hi = r3dsimt::shfl_xor(static_cast<uint32_t>(s >> 32), o);
    s += (static_cast<unsigned long long>(hi) << 32) | lo;
    st[0] = r3dsimt::imax(st[0], static_cast<int>(r3dsimt::shfl_xor(static_cast<uint32_t>(st[0]), o)));
#pragma unroll
    for (int k = 1; k < kTileStats; ++k) st[k] += static_cast<int>(r3dsimt::shfl_xor(static_cast<uint32_t>(st[k]), o));
  }
  const int warp = static_cast<int>(threadIdx.x >> 5), lane = static_cast<int>(threadIdx.x & 31u);
  if (lane == 0) {
    ssum[warp] = s;
#pragma unroll
    for (int k = 0; k < kTileStats; ++k) sst[warp * kTileStats + k] = st[k];
  }
  r3dsimt::syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long tot = 0;
    int out[kTileStats] = {};
    for (int i = 0; i < static_cast<int>(blockDim.x >> 5); ++i) {
      tot += ssum[i];
      out[0] = r3dsimt::imax(out[0], sst[i * kTileStats]);
      for (int k = 1; k < kTileStats; ++k) out[k] += sst[i * kTileStats + k];
    }
    atomicAdd(cells + blockIdx.x, tot);
    atomicMax(stats + static_cast<int64_t>(blockIdx.x) * kTileStats, out[0]);
    for (int k = 1; k < kTileStats; ++k) atomicAdd(stats + static_cast<int64_t>(blockIdx.x) * kTileStats + k, out[k]);
  }
}

dim3 grid2d(int w, int h, dim3 b) { return dim3(ceil_div(w, b.x), ceil_div(h, b.y)); }

}  // namespace

std::atomic<uint64_t>& launch_counter() {
  static std::atomic<uint64_t> c{0};
  return c;
}

void launch_census(const uint16_t* img, int64_t stride, int w, int h, uint64_t* out, int64_t ostride, cudaStream_t s) {
  if (w <= 0 || h <= 0) return;
  R3D_LAUNCH(census_kernel, dim3(ceil_div(w, kCBX), ceil_div(h, kCBY)), dim3(kCBX, kCBY), (kCBY + 6) * (kCBX + 8) * sizeof(uint16_t), s, img, stride, w, h, out, ostride);
  launched("census_kernel");
}

void launch_pyramid_u16(const uint16_t* in, int64_t istride, int w, int h, uint16_t* out, int64_t ostride,
                        cudaStream_t s) {
  const int dw = (w + 1) / 2, dh = (h + 1) / 2;
  const dim3 b(32, 8);
  R3D_LAUNCH(pyramid_u16_kernel, grid2d(dw, dh, b), b, 0, s, in, istride, w, h, out, ostride, dw, dh);
  launched("pyramid_u16_kernel");
}

void launch_reduce_mask(const uint8_t* in, int64_t istride, int w, int h, uint8_t* out, int64_t ostride,
                        cudaStream_t s) {
  const int dw = (w + 1) / 2, dh = (h + 1) / 2;
  const dim3 b(32, 8);
  R3D_LAUNCH(reduce_mask_kernel, grid2d(dw, dh, b), b, 0, s, in, istride, w, h, out, ostride, dw, dh);
  launched("reduce_mask_kernel");
}

void launch_mirror_u16(const uint16_t* in, int64_t istride, int w, int h, uint16_t* out, cudaStream_t s) {
  const dim3 b(32, 8);
  R3D_LAUNCH(mirror_kernel<uint16_t>, grid2d(w, h, b), b, 0, s, in, istride, w, h, out);
  launched("mirror_kernel<u16>");
}

void launch_mirror_u8(const uint8_t* in, int64_t istride, int w, int h, uint8_t* out, cudaStream_t s) {
  const dim3 b(32, 8);
  R3D_LAUNCH(mirror_kernel<uint8_t>, grid2d(w, h, b), b, 0, s, in, istride, w, h, out);
  launched("mirror_kernel<u8>");
}

void launch_intervals(const uint8_t* mask, int64_t stride, int w, int h, RowInterval* out, cudaStream_t s) {
  R3D_LAUNCH(intervals_kernel, ceil_div(h, 8), 256, 0, s, mask, stride, w, h, out);
  launched("intervals_kernel");
}

void launch_lr_check(const float* map, const float* other, int w, int h, int wo, int sign, int max_diff, uint8_t* bad,
                     cudaStream_t s) {
  const dim3 b(32, 8);
  R3D_LAUNCH(lr_check_kernel, grid2d(w, h, b), b, 0, s, map, other, w, h, wo, sign, max_diff, bad);
  launched("lr_check_kernel");
}

void launch_apply_bad(float* map, const uint8_t* bad, int64_t n, cudaStream_t s) {
  R3D_LAUNCH(apply_bad_kernel, static_cast<unsigned>(ceil_div64(n, 256)), 256, 0, s, map, bad, n);
  launched("apply_bad_kernel");
}

void launch_segments(const float* d, int w, int h, float max_diff, int* parent, int* size, cudaStream_t s) {
  const int64_t n = static_cast<int64_t>(w) * h;
  const dim3 tiles(static_cast<unsigned>(ceil_div64(w, kUfTile)), static_cast<unsigned>(ceil_div64(h, kUfTile)));
  R3D_LAUNCH(uf_tile_kernel, tiles, 256, 2 * sizeof(int) * kUfTile * kUfTile, s, d, w, h, max_diff, parent, size);
  launched("uf_tile_kernel");
  const int64_t nb = static_cast<int64_t>((w - 1) / kUfTile) * h + static_cast<int64_t>((h - 1) / kUfTile) * w;
  if (nb > 0) {
    R3D_LAUNCH(uf_border_kernel, static_cast<unsigned>(ceil_div64(nb, 256)), 256, 0, s, d, w, h, max_diff, parent);
    launched("uf_border_kernel");
  }
  const unsigned g1 = static_cast<unsigned>(ceil_div64(n, 256));
  R3D_LAUNCH(uf_count_kernel, g1, 256, 0, s, d, n, parent, size);
  launched("uf_count_kernel");
}

void launch_remove_speckles(float* d, int w, int h, int min_size, float max_diff, int* scratch, cudaStream_t s) {
  if (min_size <= 1 || w <= 0 || h <= 0) return;
  const int64_t n = static_cast<int64_t>(w) * h;
  int* parent = scratch;
  int* size = scratch + n;
  launch_segments(d, w, h, max_diff, parent, size, s);
  const unsigned g1 = static_cast<unsigned>(ceil_div64(n, 256));
  R3D_LAUNCH(uf_filter_kernel, g1, 256, 0, s, d, n, parent, size, min_size);
  launched("uf_filter_kernel");
}

void launch_median3x3(const float* in, int w, int h, float* out, cudaStream_t s) {
  const dim3 b(32, 8);
  R3D_LAUNCH(median_kernel, grid2d(w, h, b), b, 0, s, in, w, h, out);
  launched("median_kernel");
}

void launch_unmirror_offset(const float* in, int w, int h, float offset, float* out, cudaStream_t s) {
  const dim3 b(32, 8);
  R3D_LAUNCH(unmirror_offset_kernel, grid2d(w, h, b), b, 0, s, in, w, h, offset, out);
  launched("unmirror_offset_kernel");
}

void launch_copy2d_f32(const float* in, int64_t istride, int w, int h, float* out, int64_t ostride, cudaStream_t s) {
  const dim3 b(32, 8);
  R3D_LAUNCH(copy2d_kernel, grid2d(w, h, b), b, 0, s, in, istride, w, h, out, ostride);
  launched("copy2d_kernel");
}

int64_t ranges_scratch_floats(int wc, int hc, int fill) {
  // hmin, hmax, cmin, cmax, then the min / max pyramid (level 0 included).
  int64_t total = 4LL * wc * hc;
  int aw = wc, ah = hc;
  int levels = 1;
  total += 2LL * aw * ah;
  while ((2 << levels) <= 2 * fill && aw > 1) {
    aw = (aw + 1) / 2;
    ah = (ah + 1) / 2;
    total += 2LL * aw * ah;
    ++levels;
  }
  return total;
}

void launch_ranges_from_coarse(const float* coarse, int wc, int hc, int w, int h, const uint8_t* fine_valid,
                               int64_t fv_stride, const RowInterval* partner_rows, const RangeParams& p, float* scratch,
                               uint16_t* lo, uint16_t* num, cudaStream_t s) {
  const dim3 b(32, 8);
  const int64_t n = static_cast<int64_t>(wc) * hc;
  float* hmin = scratch;
  float* hmax = hmin + n;
  float* cmin = hmax + n;
  float* cmax = cmin + n;
  float* cur = cmax + n;
  PyrLevels pl{};
  pl.mn[0] = cur;
  pl.mx[0] = cur + n;
  pl.w[0] = wc;
  pl.h[0] = hc;
  pl.count = 1;
  R3D_LAUNCH(range_hminmax_kernel, grid2d(wc, hc, b), b, 0, s, coarse, wc, hc, p.radius, hmin, hmax);
  launched("range_hminmax_kernel");
  R3D_LAUNCH(range_vminmax_kernel, grid2d(wc, hc, b), b, 0, s, hmin, hmax, wc, hc, p.radius, cmin, cmax, cur, cur + n);
  launched("range_vminmax_kernel");
  cur += 2 * n;
  int aw = wc, ah = hc;
  while ((2 << pl.count) <= 2 * p.fill && aw > 1) {
    if (pl.count >= 16) fail(R3DGPU_EUNSUPPORTED, "ranges: fill pyramid deeper than 16 levels");
    const int nw = (aw + 1) / 2, nh = (ah + 1) / 2;
    float* omin = cur;
    float* omax = cur + static_cast<int64_t>(nw) * nh;
    R3D_LAUNCH(range_pyr_kernel, grid2d(nw, nh, b), b, 0, s, pl.mn[pl.count - 1], pl.mx[pl.count - 1], aw, ah, omin, omax, nw, nh);
    launched("range_pyr_kernel");
    pl.mn[pl.count] = omin;
    pl.mx[pl.count] = omax;
    pl.w[pl.count] = nw;
    pl.h[pl.count] = nh;
    ++pl.count;
    cur += 2LL * nw * nh;
    aw = nw;
    ah = nh;
  }
  R3D_LAUNCH(range_fill_kernel, grid2d(wc, hc, b), b, 0, s, pl, wc, hc, cmin, cmax);
  launched("range_fill_kernel");
  R3D_LAUNCH(range_final_kernel, grid2d(w, h, b), b, 0, s, cmin, cmax, wc, hc, w, h, fine_valid, fv_stride, partner_rows, p,
                                                   lo, num);
  launched("range_final_kernel");
}

void launch_blend(const BlendTile* tiles, int ntiles, int tiles_x, const int* /*bx*/, const int* /*by*/, int w, int h,
                  int blend, int mirror_out, float offset, float* out_disp, float* out_conf, int64_t ostride,
                  cudaStream_t s) {
  const dim3 b(32, 8);
  R3D_LAUNCH(blend_kernel, grid2d(w, h, b), b, 0, s, tiles, ntiles, tiles_x, w, h, blend, mirror_out, offset, out_disp,
                                             out_conf, ostride);
  launched("blend_kernel");
}

void launch_tile_cells(const uint16_t* rnum, int64_t stride, const int4* tiles, int ntiles, unsigned long long* cells,
                       int* stats, cudaStream_t s) {
  if (ntiles <= 0) return;
  R3D_CUDA(cudaMemsetAsync(cells, 0, sizeof(unsigned long long) * ntiles, s));
  R3D_CUDA(cudaMemsetAsync(stats, 0, sizeof(int) * kTileStats * ntiles, s));
  // Enough slices per tile for several blocks per SM over all tiles.
  const int slices = ntiles >= 296 ? 1 : (592 + ntiles - 1) / ntiles;
  R3D_LAUNCH(tile_cells_kernel, dim3(ntiles, slices > 32 ? 32 : slices), dim3(256), 8 * 32 + 4 * kTileStats * 8, s, rnum,
             stride, tiles, cells, stats);
  launched("tile_cells_kernel");
}

}  // namespace r3dgpu
