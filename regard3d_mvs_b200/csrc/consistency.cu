// Multi-view geometric consistency of depth maps (r3dgpu_prepare_depth_map,
// r3dgpu_check_consistency, r3dgpu_filter_depth_maps and the single filters),
// the reference's src/r3d/mvs/consistency.cpp:57-487.
//
// Every stage is per pixel: one thread per pixel in 32 x 8 blocks, warp rows
// along x so that depth rows are read coalesced. Removal counts are summed
// per warp (ballot + popcount) into device counters that the host reads once
// per call. The projection check computes in double precision with the
// reference's operations in its order (no contraction), so kept depths,
// averaged depths and support counts equal a CPU restatement bit for bit.
// The two segment filters (weak-texture segments and speckles) label the
// segments of the log-depth map with the union-find of the disparity speckle
// filter; their only operation that a CPU may round differently is logf.
#include <cmath>
#include <string>
#include <vector>

#include "common.cuh"
#include "geom.cuh"
#include "kernels.h"
#include "api_guard.h"
#include "matcher_internal.h"

namespace r3dgpu {
namespace {

constexpr float kInfF = __builtin_huge_valf();

enum Counter : int { kUnconfident, kEroded, kRejected, kWeak, kHalo, kSpeckles, kValid, kOutput, kRemoved, kCounters };

R3D_DEVICE void count_warp(unsigned long long* counter, bool pred) {
  const uint32_t b = r3dsimt::ballot(pred);
  if (r3dsimt::lane_id() == 0 && b != 0) atomicAdd(counter, static_cast<unsigned long long>(r3dsimt::popc64(b)));
}

R3D_DEVICE int64_t at(const r3dgpu_depth_map& m, int x, int y) { return static_cast<int64_t>(y) * m.stride + x; }


// ------------------------------------------------------------------ prepare
// consistency.cpp:438-447 (confidence) and the valid-pixel count.
R3D_GLOBAL void confidence_kernel(r3dgpu_depth_map m, float min_confidence, unsigned long long* counters) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  const bool in = x < m.width && y < m.height;
  bool valid = false, cut = false;
  if (in) {
    float* d = m.depth + at(m, x, y);
    valid = *d > 0.0F;
    if (valid && min_confidence > 0.0F && m.confidence[at(m, x, y)] < min_confidence) {
      *d = 0.0F;
      cut = true;
    }
  }
  count_warp(counters + kValid, valid);
  count_warp(counters + kUnconfident, cut);
}

R3D_GLOBAL void count_valid_kernel(r3dgpu_depth_map m, unsigned long long* counter) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  count_warp(counter, x < m.width && y < m.height && m.depth[at(m, x, y)] > 0.0F);
}

// consistency.cpp:57-83: a valid pixel is an edge when a 4-neighbour's depth
// differs by more than jump * min (or, with holes, is invalid).
R3D_GLOBAL void edge_kernel(r3dgpu_depth_map m, float jump, int holes, uint8_t* edge) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= m.width || y >= m.height) return;
  const float z = m.depth[at(m, x, y)];
  bool e = false;
  if (z > 0.0F) {
    auto differs = [&](int nx, int ny) {
      if (nx < 0 || ny < 0 || nx >= m.width || ny >= m.height) return false;
      const float zn = m.depth[at(m, nx, ny)];
      return zn > 0.0F ? fabsf(__fsub_rn(zn, z)) > __fmul_rn(jump, fminf(z, zn)) : holes != 0;
    };
    e = differs(x - 1, y) || differs(x + 1, y) || differs(x, y - 1) || differs(x, y + 1);
  }
  edge[static_cast<int64_t>(y) * m.width + x] = e ? 1 : 0;
}

// consistency.cpp:84-108: valid pixels within (r - 1) of an edge go.
R3D_GLOBAL void erode_kernel(r3dgpu_depth_map m, const uint8_t* edge, int r, unsigned long long* counter) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  bool removed = false;
  if (x < m.width && y < m.height) {
    float* d = m.depth + at(m, x, y);
    if (*d > 0.0F) {
      const int y0 = r3dsimt::imax(y - r, 0), y1 = r3dsimt::imin(y + r, m.height - 1);
      const int x0 = r3dsimt::imax(x - r, 0), x1 = r3dsimt::imin(x + r, m.width - 1);
      for (int v = y0; v <= y1 && !removed; ++v)
        for (int u = x0; u <= x1 && !removed; ++u) removed = edge[static_cast<int64_t>(v) * m.width + u] != 0;
      if (removed) *d = 0.0F;
    }
  }
  count_warp(counter, removed);
}

// ------------------------------------------------------------------ check
struct Neighbour {
  r3dgpu_depth_map map;
  uint16_t bit_m;  // bit of the pair (m, n) in m's pair mask
  uint16_t bit_n;  // bit of the pair (n, m) in n's pair mask
};

struct CheckParams {
  float rel_tol;
  double reproj_tol2;
  int min_views, min_evidence, independent, average;
};

// consistency.cpp:449-534 for one pixel: project its point into every
// neighbour, compare depths, project the neighbour's depth back, count the
// agreeing views; then reject or average.
R3D_GLOBAL void check_kernel(r3dgpu_depth_map m, const Neighbour* R3D_RESTRICT nbs, int count, CheckParams p,
                             float* out, unsigned long long* counter) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  bool rejected = false;
  if (x < m.width && y < m.height) {
    const float z = m.depth[at(m, x, y)];
    float result = z;
    int agree = 0;
    if (z > 0.0F) {
      const r3dgpu_pinhole_camera& c = m.camera;
      const double px = x, py = y, zd = z;
      const double a0 = row3(c.k_inv, 0, px, py, 1.0), a1 = row3(c.k_inv, 1, px, py, 1.0),
                   a2 = row3(c.k_inv, 2, px, py, 1.0);
      double xw[3];
      for (int i = 0; i < 3; ++i) xw[i] = c.center[i] + col3(c.rotation, i, a0, a1, a2) * zd;
      double depth_sum = zd;
      const uint16_t mask = m.pair_mask != nullptr ? m.pair_mask[at(m, x, y)] : 0;
      for (int j = 0; j < count; ++j) {
        const Neighbour& nb = nbs[j];
        const r3dgpu_depth_map& n = nb.map;
        if (n.width == 0) continue;
        const r3dgpu_pinhole_camera& cn = n.camera;
        const double d0 = xw[0] - cn.center[0], d1 = xw[1] - cn.center[1], d2 = xw[2] - cn.center[2];
        const double xc0 = row3(cn.rotation, 0, d0, d1, d2), xc1 = row3(cn.rotation, 1, d0, d1, d2),
                     xc2 = row3(cn.rotation, 2, d0, d1, d2);
        if (!(xc2 > 0.0)) continue;
        const double inv_z = 1.0 / xc2;
        const double qx = cn.intrinsics.fx * xc0 * inv_z + cn.intrinsics.cx;
        const double qy = cn.intrinsics.fy * xc1 * inv_z + cn.intrinsics.cy;
        const long long ix = llround(qx), iy = llround(qy);
        if (ix < 0 || iy < 0 || ix >= n.width || iy >= n.height) continue;
        const int64_t ni = static_cast<int64_t>(iy) * n.stride + ix;
        const float zn = n.depth[ni];
        if (zn <= 0.0F || fabsf(__fsub_rn(zn, static_cast<float>(xc2))) > __fmul_rn(p.rel_tol, zn)) continue;
        // n.point(ix, iy) = R_n^T unproject(ix, iy, zn) + C_n (camera.hpp:47-50, 74-76).
        const double znd = zn;
        const double u0 = (static_cast<double>(ix) - cn.intrinsics.cx) / cn.intrinsics.fx * znd;
        const double u1 = (static_cast<double>(iy) - cn.intrinsics.cy) / cn.intrinsics.fy * znd;
        double back[3];
        for (int i = 0; i < 3; ++i) back[i] = col3(cn.rotation, i, u0, u1, znd) + cn.center[i];
        const double e0 = back[0] - c.center[0], e1 = back[1] - c.center[1], e2 = back[2] - c.center[2];
        const double b0 = row3(c.rotation, 0, e0, e1, e2), b1 = row3(c.rotation, 1, e0, e1, e2),
                     b2 = row3(c.rotation, 2, e0, e1, e2);
        if (!(b2 > 0.0)) continue;
        const double inv_b = 1.0 / b2;
        const double dx = (c.intrinsics.fx * b0 * inv_b + c.intrinsics.cx) - px;
        const double dy = (c.intrinsics.fy * b1 * inv_b + c.intrinsics.cy) - py;
        if (dx * dx + dy * dy > p.reproj_tol2) continue;
        if (p.independent && nb.bit_m != 0 && mask == nb.bit_m) {
          if (nb.bit_n != 0 && n.pair_mask != nullptr && n.pair_mask[ni] == nb.bit_n) continue;
        }
        ++agree;
        depth_sum += b2;
      }
      const int support = agree < 255 ? agree : 255;
      const int pairs = r3dsimt::popc64(mask);
      if (support < p.min_views || support + pairs < p.min_evidence) {
        result = 0.0F;
        rejected = true;
      } else if (p.average) {
        result = static_cast<float>(depth_sum / (agree + 1));
      }
      if (m.support != nullptr) m.support[at(m, x, y)] = static_cast<uint8_t>(support);
    } else if (m.support != nullptr) {
      m.support[at(m, x, y)] = 0;
    }
    out[static_cast<int64_t>(y) * m.width + x] = result;
  }
  count_warp(counter, rejected);
}

// ------------------------------------------------------------------ weak depths
// consistency.cpp:138-163: a valid pixel is weak when the grey level of its
// clamped 7 x 7 colour window varies by less than max_var.
R3D_GLOBAL void weak_kernel(const float* depth, int w, int h, const uint8_t* color, int64_t cstride, double max_var,
                            uint8_t* weak) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  const int64_t i = static_cast<int64_t>(y) * w + x;
  uint8_t out = 0;
  if (depth[i] > 0.0F) {
    double sum = 0.0, sum2 = 0.0;
    int count = 0;
    for (int v = r3dsimt::imax(y - 3, 0); v <= r3dsimt::imin(y + 3, h - 1); ++v) {
      const uint8_t* row = color + static_cast<int64_t>(v) * cstride;
      for (int u = r3dsimt::imax(x - 3, 0); u <= r3dsimt::imin(x + 3, w - 1); ++u) {
        const double g = (0.299 * row[3 * u] + 0.587 * row[3 * u + 1]) + 0.114 * row[3 * u + 2];
        sum += g;
        sum2 += g * g;
        ++count;
      }
    }
    const double mean = sum / count;
    out = sum2 / count - mean * mean < max_var ? 1 : 0;
  }
  weak[i] = out;
}

// Log depth (+inf where invalid), the map the segment filters label.
R3D_GLOBAL void log_depth_kernel(const float* depth, int64_t n, float* out) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float z = depth[i];
  out[i] = z > 0.0F ? logf(z) : kInfF;
}

// Per segment root: the number of weak pixels (warp-aggregated like the sizes).
R3D_GLOBAL void weak_count_kernel(const float* logd, const uint8_t* weak, int64_t n, const int* parent, int* weak_count) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const bool ok = i < n && r3dsimt::finitef(logd[i]) && weak[i] != 0;
  const int r = ok ? parent[i] : -1;
  const uint32_t peers = r3dsimt::match_any(static_cast<uint32_t>(r));
  if (ok && static_cast<int>(r3dsimt::lane_id()) == r3dsimt::ffs(peers) - 1)
    atomicAdd(weak_count + r, r3dsimt::popc64(peers));
}

// consistency.cpp:216-223: a segment smaller than max_size whose pixels are
// at least half weak goes.
R3D_GLOBAL void weak_segment_kernel(float* depth, const float* logd, int64_t n, const int* parent, const int* size,
                                    const int* weak_count, long long max_size, unsigned long long* counter) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  bool removed = false;
  if (i < n && r3dsimt::finitef(logd[i])) {
    const int r = parent[i];
    const long long sz = size[r];
    if (sz < max_size && 2LL * weak_count[r] >= sz) {
      depth[i] = 0.0F;
      removed = true;
    }
  }
  count_warp(counter, removed);
}

// depth = 0 where flag[i] != 0 (flags of valid pixels only), counted.
R3D_GLOBAL void apply_flags_kernel(float* depth, const uint8_t* flag, int64_t n, unsigned long long* counter) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const bool removed = i < n && flag[i] != 0;
  if (removed) depth[i] = 0.0F;
  count_warp(counter, removed);
}

// ------------------------------------------------------------------ halos
// consistency.cpp:247-276: a hole is a pixel whose clamped 5 x 5
// neighbourhood has no valid depth.
R3D_GLOBAL void hole_kernel(const float* depth, int w, int h, uint8_t* hole) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  bool empty = true;
  for (int v = r3dsimt::imax(y - 2, 0); v <= r3dsimt::imin(y + 2, h - 1) && empty; ++v)
    for (int u = r3dsimt::imax(x - 2, 0); u <= r3dsimt::imin(x + 2, w - 1) && empty; ++u)
      empty = depth[static_cast<int64_t>(v) * w + u] <= 0.0F;
  hole[static_cast<int64_t>(y) * w + x] = empty ? 1 : 0;
}

// consistency.cpp:277-331: in one of 8 directions, pixels of this colour
// lead to a hole within max_px, and in the opposite direction a pixel of
// another colour follows before the depths end.
R3D_GLOBAL void halo_kernel(const float* depth, int w, int h, const uint8_t* color, int64_t cstride,
                            const uint8_t* hole, int max_px, int colour_step, uint8_t* halo) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  const int64_t i = static_cast<int64_t>(y) * w + x;
  uint8_t flag = 0;
  if (depth[i] > 0.0F) {
    const uint8_t* c0 = color + static_cast<int64_t>(y) * cstride + 3 * x;
    auto differs = [&](int u, int v) {
      const uint8_t* c1 = color + static_cast<int64_t>(v) * cstride + 3 * u;
      for (int c = 0; c < 3; ++c)
        if (abs(static_cast<int>(c1[c]) - static_cast<int>(c0[c])) >= colour_step) return true;
      return false;
    };
    const int dirs[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {1, -1}, {-1, 1}, {-1, -1}};
    for (int k = 0; k < 8 && flag == 0; ++k) {
      const int dx = dirs[k][0], dy = dirs[k][1];
      int to_hole = 0;
      for (int s = 1; s <= max_px; ++s) {
        const int u = x + s * dx, v = y + s * dy;
        if (u < 0 || v < 0 || u >= w || v >= h || differs(u, v)) break;
        if (hole[static_cast<int64_t>(v) * w + u] != 0) {
          to_hole = s;
          break;
        }
      }
      if (to_hole == 0) continue;
      for (int s = 1; s <= max_px - to_hole; ++s) {
        const int u = x - s * dx, v = y - s * dy;
        if (u < 0 || v < 0 || u >= w || v >= h) break;
        if (differs(u, v)) {
          flag = 1;
          break;
        }
        if (depth[static_cast<int64_t>(v) * w + u] <= 0.0F) break;
      }
    }
  }
  halo[i] = flag;
}

// ------------------------------------------------------------------ speckles
// consistency.cpp:112-131: depth = 0 where the speckle filter of the log
// depth removed the value.
R3D_GLOBAL void speckle_apply_kernel(float* depth, const float* logd, int64_t n, unsigned long long* counter) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const bool removed = i < n && depth[i] > 0.0F && !r3dsimt::finitef(logd[i]);
  if (removed) depth[i] = 0.0F;
  count_warp(counter, removed);
}

// ------------------------------------------------------------------ host side
dim3 grid_of(int w, int h) { return dim3(static_cast<unsigned>(ceil_div(w, 32)), static_cast<unsigned>(ceil_div(h, 8))); }
unsigned grid1(int64_t n) { return static_cast<unsigned>(ceil_div64(n, 256)); }

// Per-thread device scratch of the filters.
struct Scratch {
  DeviceBuffer<unsigned long long> counters;
  DeviceBuffer<uint8_t> flags, flags2;
  DeviceBuffer<float> logd, work;
  DeviceBuffer<int> uf;
  DeviceBuffer<Neighbour> nbs;
};

Scratch& scratch() {
  thread_local Scratch s;
  s.counters.reserve(kCounters);
  return s;
}

void check_map(const r3dgpu_depth_map* m, const char* what) {
  if (m == nullptr) fail(R3DGPU_EINVAL, std::string(what) + ": null depth map");
  if (m->width < 0 || m->height < 0) fail(R3DGPU_EINVAL, std::string(what) + ": negative size");
  if (m->width > 0 && m->height > 0 && (m->depth == nullptr || m->stride < m->width))
    fail(R3DGPU_EINVAL, std::string(what) + ": no depth image or its stride is below the width");
  if (m->color != nullptr && m->color_stride < 3LL * m->width)
    fail(R3DGPU_EINVAL, std::string(what) + ": colour stride below 3 x width");
  if (m->num_partners > R3DGPU_MAX_PARTNERS)
    fail(R3DGPU_EINVAL, std::string(what) + ": more than 16 partners");
}

void check_options(const r3dgpu_consistency_options& o) {
  if (o.halo_px < 0 || o.edge_erosion < 0) fail(R3DGPU_EINVAL, "consistency: negative erosion or halo distance");
}

r3dgpu_consistency_options options_or_default(const r3dgpu_consistency_options* o) {
  r3dgpu_consistency_options out{};
  if (o != nullptr) return *o;
  r3dgpu_default_consistency_options(&out);
  return out;
}

// A contiguous w x h working copy of the map's depth (the segment and halo
// filters index pixels as y * w + x).
void to_work(const r3dgpu_depth_map& m, float* work, cudaStream_t s) {
  R3D_CUDA(cudaMemcpy2DAsync(work, sizeof(float) * m.width, m.depth, sizeof(float) * m.stride,
                             sizeof(float) * m.width, m.height, cudaMemcpyDeviceToDevice, s));
}
void from_work(const r3dgpu_depth_map& m, const float* work, cudaStream_t s) {
  R3D_CUDA(cudaMemcpy2DAsync(m.depth, sizeof(float) * m.stride, work, sizeof(float) * m.width,
                             sizeof(float) * m.width, m.height, cudaMemcpyDeviceToDevice, s));
}

void erode(const r3dgpu_depth_map& m, int radius, double discontinuity, bool holes, unsigned long long* counter,
           cudaStream_t s) {
  if (radius <= 0 || m.width == 0 || m.height == 0) return;
  Scratch& sc = scratch();
  sc.flags.reserve(static_cast<size_t>(m.width) * m.height);
  uint8_t* edge = sc.flags.get();
  const dim3 b(32, 8);
  R3D_LAUNCH(edge_kernel, grid_of(m.width, m.height), b, 0, s, m, static_cast<float>(discontinuity), holes ? 1 : 0,
             edge);
  launched("edge_kernel");
  R3D_LAUNCH(erode_kernel, grid_of(m.width, m.height), b, 0, s, m, edge, radius - 1, counter);
  launched("erode_kernel");
}

// The filters after the check work on a contiguous depth `d` (w x h).
void weak_filter(float* d, const r3dgpu_depth_map& m, const r3dgpu_consistency_options& o,
                 unsigned long long* counter, cudaStream_t s) {
  const int w = m.width, h = m.height;
  const bool segments = o.weak_segment > 0.0;
  if (o.weak_texture <= 0.0 || (!segments && !o.reject_weak) || m.color == nullptr || w == 0 || h == 0) return;
  Scratch& sc = scratch();
  const int64_t n = static_cast<int64_t>(w) * h;
  sc.flags.reserve(n);
  uint8_t* weak = sc.flags.get();
  const dim3 b(32, 8);
  R3D_LAUNCH(weak_kernel, grid_of(w, h), b, 0, s, d, w, h, m.color, m.color_stride,
             o.weak_texture * o.weak_texture, weak);
  launched("weak_kernel");
  if (o.reject_weak) {
    R3D_LAUNCH(apply_flags_kernel, grid1(n), 256, 0, s, d, weak, n, counter);
    launched("apply_flags_kernel");
    return;
  }
  sc.logd.reserve(n);
  sc.uf.reserve(3 * n);
  float* logd = sc.logd.get();
  int* parent = sc.uf.get();
  int* size = parent + n;
  int* weak_count = size + n;
  R3D_CUDA(cudaMemsetAsync(weak_count, 0, sizeof(int) * n, s));
  R3D_LAUNCH(log_depth_kernel, grid1(n), 256, 0, s, d, n, logd);
  launched("log_depth_kernel");
  launch_segments(logd, w, h, static_cast<float>(std::log1p(o.speckle_step)), parent, size, s);
  R3D_LAUNCH(weak_count_kernel, grid1(n), 256, 0, s, logd, weak, n, parent, weak_count);
  launched("weak_count_kernel");
  const auto max_size = static_cast<long long>(static_cast<size_t>(o.weak_segment * static_cast<double>(n)));
  R3D_LAUNCH(weak_segment_kernel, grid1(n), 256, 0, s, d, logd, n, parent, size, weak_count, max_size, counter);
  launched("weak_segment_kernel");
}

void halo_filter(float* d, const r3dgpu_depth_map& m, int max_px, int colour_step, unsigned long long* counter,
                 cudaStream_t s) {
  const int w = m.width, h = m.height;
  if (max_px <= 0 || m.color == nullptr || w == 0 || h == 0) return;
  Scratch& sc = scratch();
  const int64_t n = static_cast<int64_t>(w) * h;
  sc.flags.reserve(n);
  sc.flags2.reserve(n);
  uint8_t* hole = sc.flags.get();
  uint8_t* halo = sc.flags2.get();
  const dim3 b(32, 8);
  R3D_LAUNCH(hole_kernel, grid_of(w, h), b, 0, s, d, w, h, hole);
  launched("hole_kernel");
  R3D_LAUNCH(halo_kernel, grid_of(w, h), b, 0, s, d, w, h, m.color, m.color_stride, hole, max_px, colour_step, halo);
  launched("halo_kernel");
  R3D_LAUNCH(apply_flags_kernel, grid1(n), 256, 0, s, d, halo, n, counter);
  launched("apply_flags_kernel");
}

void speckle_filter(float* d, int w, int h, int min_size, double max_relative_step, unsigned long long* counter,
                    cudaStream_t s) {
  if (min_size <= 1 || w == 0 || h == 0) return;
  Scratch& sc = scratch();
  const int64_t n = static_cast<int64_t>(w) * h;
  sc.logd.reserve(n);
  sc.uf.reserve(3 * n);
  float* logd = sc.logd.get();
  R3D_LAUNCH(log_depth_kernel, grid1(n), 256, 0, s, d, n, logd);
  launched("log_depth_kernel");
  launch_remove_speckles(logd, w, h, min_size, static_cast<float>(std::log1p(max_relative_step)), sc.uf.get(), s);
  R3D_LAUNCH(speckle_apply_kernel, grid1(n), 256, 0, s, d, logd, n, counter);
  launched("speckle_apply_kernel");
}

uint16_t pair_bit(const r3dgpu_depth_map& m, uint32_t view) {
  for (uint32_t i = 0; i < m.num_partners; ++i)
    if (m.partners[i] == view) return static_cast<uint16_t>(1u << i);
  return 0;
}

// Check of `m` against `nbs` (prepared maps); the checked depth goes to the
// contiguous `out` (w x h), filtered there by the weak, halo and speckle steps.
void check_into(const r3dgpu_depth_map& m, const r3dgpu_depth_map* const* nbs, int count,
                const r3dgpu_consistency_options& o, float* out, unsigned long long* counters, cudaStream_t s) {
  if (count > R3DGPU_MAX_NEIGHBOURS)
    fail(R3DGPU_EINVAL, "check_consistency: " + std::to_string(count) + " neighbours (at most " +
                            std::to_string(R3DGPU_MAX_NEIGHBOURS) + ")");
  if (m.width == 0 || m.height == 0) return;
  Scratch& sc = scratch();
  std::vector<Neighbour> host(static_cast<size_t>(count));
  for (int j = 0; j < count; ++j) {
    host[j].map = *nbs[j];
    host[j].bit_m = pair_bit(m, nbs[j]->view);
    host[j].bit_n = pair_bit(*nbs[j], m.view);
  }
  sc.nbs.reserve(R3DGPU_MAX_NEIGHBOURS);
  if (count > 0)
    R3D_CUDA(cudaMemcpyAsync(sc.nbs.get(), host.data(), sizeof(Neighbour) * count, cudaMemcpyHostToDevice, s));
  CheckParams p{static_cast<float>(o.max_relative_depth_error), o.max_reprojection_px * o.max_reprojection_px,
                o.min_views, o.min_evidence, o.independent_support, o.average_depths};
  const dim3 b(32, 8);
  const Neighbour* dnbs = sc.nbs.get();
  R3D_LAUNCH(check_kernel, grid_of(m.width, m.height), b, 0, s, m, dnbs, count, p, out, counters + kRejected);
  launched("check_kernel");
  weak_filter(out, m, o, counters + kWeak, s);
  halo_filter(out, m, o.halo_px, o.halo_colour, counters + kHalo, s);
  speckle_filter(out, m.width, m.height, o.speckle_size, o.speckle_step, counters + kSpeckles, s);
}

void read_counters(unsigned long long* host, cudaStream_t s) {
  R3D_CUDA(cudaMemcpyAsync(host, scratch().counters.get(), sizeof(unsigned long long) * kCounters,
                           cudaMemcpyDeviceToHost, s));
  R3D_CUDA(cudaStreamSynchronize(s));
}

void zero_counters(cudaStream_t s) {
  R3D_CUDA(cudaMemsetAsync(scratch().counters.get(), 0, sizeof(unsigned long long) * kCounters, s));
}

void prepare(const r3dgpu_depth_map& m, const r3dgpu_consistency_options& o, cudaStream_t s) {
  if (m.width == 0 || m.height == 0) return;
  unsigned long long* c = scratch().counters.get();
  const dim3 b(32, 8);
  R3D_LAUNCH(confidence_kernel, grid_of(m.width, m.height), b, 0, s, m, o.min_confidence, c);
  launched("confidence_kernel");
  erode(m, o.edge_erosion, o.discontinuity, o.erode_holes != 0, c + kEroded, s);
}

void count_output(const r3dgpu_depth_map& m, cudaStream_t s) {
  if (m.width == 0 || m.height == 0) return;
  const dim3 b(32, 8);
  unsigned long long* c = scratch().counters.get() + kOutput;
  R3D_LAUNCH(count_valid_kernel, grid_of(m.width, m.height), b, 0, s, m, c);
  launched("count_valid_kernel");
}

// Device filter of `count` maps (device pointers in `maps`).
void filter_maps(r3dgpu_depth_map* maps, int count, const int32_t* off, const int32_t* idx,
                 const r3dgpu_consistency_options& o, r3dgpu_consistency_stats* stats, cudaStream_t s) {
  if (count < 0 || (count > 0 && (maps == nullptr || off == nullptr)))
    fail(R3DGPU_EINVAL, "filter_depth_maps: null argument");
  for (int i = 0; i < count; ++i) {
    check_map(&maps[i], "filter_depth_maps");
    if (off[i + 1] < off[i]) fail(R3DGPU_EINVAL, "filter_depth_maps: neighbour offsets decrease");
    for (int k = off[i]; k < off[i + 1]; ++k)
      if (idx == nullptr || idx[k] < 0 || idx[k] >= count)
        fail(R3DGPU_EINVAL, "filter_depth_maps: neighbour index out of range");
  }
  check_options(o);
  zero_counters(s);
  for (int i = 0; i < count; ++i) prepare(maps[i], o, s);
  // All checks read the prepared maps; their results wait in one buffer.
  std::vector<size_t> at_px(static_cast<size_t>(count) + 1, 0);
  for (int i = 0; i < count; ++i) at_px[i + 1] = at_px[i] + static_cast<size_t>(maps[i].width) * maps[i].height;
  Scratch& sc = scratch();
  sc.work.reserve(at_px[count] > 0 ? at_px[count] : 1);
  std::vector<const r3dgpu_depth_map*> nb;
  for (int i = 0; i < count; ++i) {
    nb.clear();
    for (int k = off[i]; k < off[i + 1]; ++k) nb.push_back(&maps[idx[k]]);
    check_into(maps[i], nb.data(), static_cast<int>(nb.size()), o, sc.work.get() + at_px[i], sc.counters.get(), s);
  }
  for (int i = 0; i < count; ++i) {
    if (maps[i].width == 0 || maps[i].height == 0) continue;
    from_work(maps[i], sc.work.get() + at_px[i], s);
    count_output(maps[i], s);
  }
  unsigned long long c[kCounters];
  read_counters(c, s);
  if (stats != nullptr)
    *stats = r3dgpu_consistency_stats{c[kValid], c[kUnconfident], c[kEroded], c[kRejected],
                                      c[kWeak],  c[kHalo],        c[kSpeckles], c[kOutput]};
}

// The single post-check filters run on a contiguous working copy of the depth.
template <class F>
r3dgpu_status single_filter(r3dgpu_depth_map* map, const char* what, uint64_t* removed, void* stream, F&& run) {
  return guard([&] {
    check_map(map, what);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    zero_counters(s);
    if (map->width > 0 && map->height > 0) {
      Scratch& sc = scratch();
      sc.work.reserve(static_cast<size_t>(map->width) * map->height);
      to_work(*map, sc.work.get(), s);
      run(sc.work.get(), sc.counters.get() + kRemoved, s);
      from_work(*map, sc.work.get(), s);
    }
    unsigned long long c[kCounters];
    read_counters(c, s);
    if (removed != nullptr) *removed = c[kRemoved];
  });
}

// Device copies of host maps (depth, confidence, pair mask, support, colour)
// in one per-thread staging buffer, followed by `extra` bytes for the caller;
// download() copies depth, support and, if asked, confidence back.
struct HostMaps {
  r3dgpu_depth_map* host;
  int count;
  std::vector<r3dgpu_depth_map> dev;
  unsigned char* extra = nullptr;

  HostMaps(r3dgpu_depth_map* maps, int n, size_t extra_bytes, cudaStream_t s) : host(maps), count(n) {
    if (n < 0 || (n > 0 && maps == nullptr)) fail(R3DGPU_EINVAL, "filter_depth_maps: null argument");
    for (int i = 0; i < n; ++i) check_map(&maps[i], "filter_depth_maps");
    auto up = [](size_t b) { return (b + 255) & ~static_cast<size_t>(255); };
    size_t bytes = extra_bytes;
    for (int i = 0; i < n; ++i) {
      const size_t px = static_cast<size_t>(maps[i].width) * maps[i].height;
      bytes += up(4 * px) + up(4 * px) + up(2 * px) + up(px) + (maps[i].color ? up(3 * px) : 0);
    }
    thread_local DeviceBuffer<unsigned char> io;
    io.reserve(bytes > 0 ? bytes : 1);
    unsigned char* p = io.get();
    auto take = [&](size_t b) {
      unsigned char* at = p;
      p += up(b);
      return at;
    };
    dev.assign(maps, maps + n);
    for (int i = 0; i < n; ++i) {
      const r3dgpu_depth_map& h = maps[i];
      r3dgpu_depth_map& d = dev[i];
      const size_t w = static_cast<size_t>(h.width), px = w * h.height;
      d.stride = h.width;
      d.depth = reinterpret_cast<float*>(take(4 * px));
      d.confidence = reinterpret_cast<float*>(take(4 * px));
      d.pair_mask = reinterpret_cast<uint16_t*>(take(2 * px));
      d.support = reinterpret_cast<uint8_t*>(take(px));
      if (h.color != nullptr) {
        d.color = take(3 * px);
        d.color_stride = 3 * h.width;
      }
      if (px == 0) continue;
      R3D_CUDA(cudaMemcpy2DAsync(d.depth, 4 * w, h.depth, 4 * h.stride, 4 * w, h.height, cudaMemcpyHostToDevice, s));
      if (h.confidence != nullptr)
        R3D_CUDA(cudaMemcpy2DAsync(d.confidence, 4 * w, h.confidence, 4 * h.stride, 4 * w, h.height,
                                   cudaMemcpyHostToDevice, s));
      else
        R3D_CUDA(cudaMemsetAsync(d.confidence, 0, 4 * px, s));
      if (h.pair_mask != nullptr)
        R3D_CUDA(cudaMemcpy2DAsync(d.pair_mask, 2 * w, h.pair_mask, 2 * h.stride, 2 * w, h.height,
                                   cudaMemcpyHostToDevice, s));
      else
        R3D_CUDA(cudaMemsetAsync(d.pair_mask, 0, 2 * px, s));
      if (h.color != nullptr)
        R3D_CUDA(cudaMemcpy2DAsync(const_cast<uint8_t*>(d.color), 3 * w, h.color, h.color_stride, 3 * w, h.height,
                                   cudaMemcpyHostToDevice, s));
    }
    extra = p;
  }

  void download(bool confidence, cudaStream_t s) {
    for (int i = 0; i < count; ++i) {
      const r3dgpu_depth_map& h = host[i];
      const r3dgpu_depth_map& d = dev[i];
      const size_t w = static_cast<size_t>(h.width);
      if (w == 0 || h.height == 0) continue;
      R3D_CUDA(cudaMemcpy2DAsync(h.depth, 4 * h.stride, d.depth, 4 * w, 4 * w, h.height, cudaMemcpyDeviceToHost, s));
      if (confidence && h.confidence != nullptr)
        R3D_CUDA(cudaMemcpy2DAsync(h.confidence, 4 * h.stride, d.confidence, 4 * w, 4 * w, h.height,
                                   cudaMemcpyDeviceToHost, s));
      if (h.support != nullptr)
        R3D_CUDA(cudaMemcpy2DAsync(h.support, h.stride, d.support, w, w, h.height, cudaMemcpyDeviceToHost, s));
    }
    R3D_CUDA(cudaStreamSynchronize(s));
  }
};

}  // namespace
}  // namespace r3dgpu

using namespace r3dgpu;

extern "C" {

void r3dgpu_default_consistency_options(r3dgpu_consistency_options* out) {
  if (out == nullptr) return;
  *out = r3dgpu_consistency_options{0.01, 2.0, 0, 2, 0.0F, 1, 0.05, 0, 8, 0, 1, 2.0, 0.0, 0, 32, 25, 0, 0.02};
}

r3dgpu_status r3dgpu_prepare_depth_map(r3dgpu_depth_map* map, const r3dgpu_consistency_options* options,
                                       r3dgpu_consistency_stats* stats, void* stream) {
  return guard([&] {
    check_map(map, "prepare_depth_map");
    const r3dgpu_consistency_options o = options_or_default(options);
    check_options(o);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    zero_counters(s);
    prepare(*map, o, s);
    unsigned long long c[kCounters];
    read_counters(c, s);
    if (stats != nullptr) {
      stats->input += c[kValid];
      stats->unconfident += c[kUnconfident];
      stats->eroded += c[kEroded];
    }
  });
}

r3dgpu_status r3dgpu_check_consistency(r3dgpu_depth_map* map, const r3dgpu_depth_map* neighbours, int32_t count,
                                       const r3dgpu_consistency_options* options, r3dgpu_consistency_stats* stats,
                                       void* stream) {
  return guard([&] {
    check_map(map, "check_consistency");
    if (count < 0 || (count > 0 && neighbours == nullptr)) fail(R3DGPU_EINVAL, "check_consistency: null neighbours");
    for (int j = 0; j < count; ++j) check_map(&neighbours[j], "check_consistency");
    const r3dgpu_consistency_options o = options_or_default(options);
    check_options(o);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    zero_counters(s);
    std::vector<const r3dgpu_depth_map*> nb;
    for (int j = 0; j < count; ++j) nb.push_back(&neighbours[j]);
    Scratch& sc = scratch();
    if (map->width > 0 && map->height > 0) {
      sc.work.reserve(static_cast<size_t>(map->width) * map->height);
      check_into(*map, nb.data(), count, o, sc.work.get(), sc.counters.get(), s);
      from_work(*map, sc.work.get(), s);
      count_output(*map, s);
    }
    unsigned long long c[kCounters];
    read_counters(c, s);
    if (stats != nullptr) {
      stats->rejected += c[kRejected];
      stats->weak += c[kWeak];
      stats->halo += c[kHalo];
      stats->speckles += c[kSpeckles];
      stats->output += c[kOutput];
    }
  });
}

r3dgpu_status r3dgpu_filter_depth_maps(r3dgpu_depth_map* maps, int32_t count, const int32_t* neighbour_offset,
                                       const int32_t* neighbour_index, const r3dgpu_consistency_options* options,
                                       r3dgpu_consistency_stats* stats, void* stream) {
  return guard([&] {
    filter_maps(maps, count, neighbour_offset, neighbour_index, options_or_default(options), stats,
                static_cast<cudaStream_t>(stream));
  });
}

r3dgpu_status r3dgpu_filter_depth_maps_host(r3dgpu_depth_map* maps, int32_t count, const int32_t* neighbour_offset,
                                            const int32_t* neighbour_index,
                                            const r3dgpu_consistency_options* options,
                                            r3dgpu_consistency_stats* stats) {
  return guard([&] {
    cudaStream_t s = nullptr;
    HostMaps hm(maps, count, 0, s);
    filter_maps(hm.dev.data(), count, neighbour_offset, neighbour_index, options_or_default(options), stats, s);
    hm.download(false, s);
  });
}

r3dgpu_status r3dgpu_depth_stage_host(r3dgpu_depth_map* maps, const r3dgpu_refinement_image* images, int32_t count,
                                      const int32_t* neighbour_offset, const int32_t* neighbour_index,
                                      const r3dgpu_refinement_options* refine,
                                      const r3dgpu_consistency_options* consistency,
                                      r3dgpu_refinement_stats* refine_stats,
                                      r3dgpu_consistency_stats* consistency_stats) {
  return guard([&] {
    if (count > 0 && (images == nullptr || neighbour_offset == nullptr))
      fail(R3DGPU_EINVAL, "depth_stage: null argument");
    cudaStream_t s = nullptr;
    auto image_bytes = [&](int i) {
      return sizeof(float) * 3 * static_cast<size_t>(images[i].camera.intrinsics.width) *
             images[i].camera.intrinsics.height;
    };
    size_t extra = 0;
    for (int i = 0; i < count; ++i) extra += (image_bytes(i) + 255) & ~static_cast<size_t>(255);
    HostMaps hm(maps, count, extra, s);
    // Every refinement image once.
    std::vector<r3dgpu_refinement_image> dimg(images, images + count);
    unsigned char* at = hm.extra;
    for (int i = 0; i < count; ++i) {
      const int w = images[i].camera.intrinsics.width, h = images[i].camera.intrinsics.height;
      if (w > 0 && h > 0) {
        if (images[i].data == nullptr || images[i].stride < 3LL * w)
          fail(R3DGPU_EINVAL, "depth_stage: image " + std::to_string(i) + " has no data");
        R3D_CUDA(cudaMemcpy2DAsync(at, sizeof(float) * 3 * w, images[i].data, sizeof(float) * images[i].stride,
                                   sizeof(float) * 3 * w, h, cudaMemcpyHostToDevice, s));
      }
      dimg[i].data = reinterpret_cast<const float*>(at);
      dimg[i].stride = 3LL * w;
      at += (image_bytes(i) + 255) & ~static_cast<size_t>(255);
    }
    r3dgpu_refinement_stats total{};
    std::vector<r3dgpu_refinement_image> views;
    for (int i = 0; i < count; ++i) {
      if (neighbour_offset[i + 1] < neighbour_offset[i]) fail(R3DGPU_EINVAL, "depth_stage: neighbour offsets decrease");
      views.clear();
      for (int k = neighbour_offset[i]; k < neighbour_offset[i + 1]; ++k) {
        if (neighbour_index == nullptr || neighbour_index[k] < 0 || neighbour_index[k] >= count)
          fail(R3DGPU_EINVAL, "depth_stage: neighbour index out of range");
        views.push_back(dimg[neighbour_index[k]]);
      }
      r3dgpu_depth_map& d = hm.dev[i];
      r3dgpu_refinement_stats st{};
      const r3dgpu_status rs = r3dgpu_refine_depth_map(d.depth, d.confidence, d.stride, &d.camera, d.width, d.height,
                                                       &dimg[i], views.data(), static_cast<int32_t>(views.size()),
                                                       refine, &st, s);
      if (rs != R3DGPU_OK) fail(rs, r3dgpu_last_error());
      total.input += st.input;
      total.refined += st.refined;
      total.kept += st.kept;
      total.unconfirmed += st.unconfirmed;
    }
    filter_maps(hm.dev.data(), count, neighbour_offset, neighbour_index, options_or_default(consistency),
                consistency_stats, s);
    hm.download(true, s);
    if (refine_stats != nullptr) *refine_stats = total;
  });
}

r3dgpu_status r3dgpu_erode_depth_edges(r3dgpu_depth_map* map, int32_t radius, double discontinuity, int32_t holes,
                                       uint64_t* removed, void* stream) {
  return guard([&] {
    check_map(map, "erode_depth_edges");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    zero_counters(s);
    erode(*map, radius, discontinuity, holes != 0, scratch().counters.get() + kRemoved, s);
    unsigned long long c[kCounters];
    read_counters(c, s);
    if (removed != nullptr) *removed = c[kRemoved];
  });
}

r3dgpu_status r3dgpu_remove_weak_depths(r3dgpu_depth_map* map, const r3dgpu_consistency_options* options,
                                        uint64_t* removed, void* stream) {
  const r3dgpu_consistency_options o = options_or_default(options);
  return single_filter(map, "remove_weak_depths", removed, stream, [&](float* d, unsigned long long* c, cudaStream_t s) {
    weak_filter(d, *map, o, c, s);
  });
}

r3dgpu_status r3dgpu_remove_depth_halos(r3dgpu_depth_map* map, int32_t max_px, int32_t colour_step,
                                        uint64_t* removed, void* stream) {
  return single_filter(map, "remove_depth_halos", removed, stream, [&](float* d, unsigned long long* c, cudaStream_t s) {
    halo_filter(d, *map, max_px, colour_step, c, s);
  });
}

r3dgpu_status r3dgpu_remove_depth_speckles(r3dgpu_depth_map* map, int32_t min_size, double max_relative_step,
                                           uint64_t* removed, void* stream) {
  return single_filter(map, "remove_depth_speckles", removed, stream,
                       [&](float* d, unsigned long long* c, cudaStream_t s) {
                         speckle_filter(d, map->width, map->height, min_size, max_relative_step, c, s);
                       });
}

}  // extern "C"
