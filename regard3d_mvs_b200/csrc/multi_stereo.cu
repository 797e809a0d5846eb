// Combination of matched pairs into a depth map (r3dgpu_combine_pairs): one
// thread per grid pixel, in double precision as the reference
// (src/r3d/mvs/multi_stereo.cpp:74-216), every operation in the reference's
// order and without contraction (the library is built with --fmad=false),
// so that depths are bit-identical to a CPU restatement.
//
// Per pixel: each pair's homography gives the rectified position (u, v) and
// the depth ratio c; the pair's disparity there (bilinear inside a surface,
// else the nearest pixel, multi_stereo.cpp:44-72) gives a candidate inverse
// depth w with d = k * w + offset, k = fb / c. The candidate with the most
// agreeing candidates (|k_j (w_j - w_i)| <= inlier_px; ties: the larger
// summed confidence) selects the inliers; a weighted least-squares w (weights
// k^2) drops its worst pair while a residual exceeds max_reprojection_px.
// The pixel keeps the depth 1 / w if enough pairs remain, they outnumber the
// others (or two on a tie), and one of them sees the point under at least
// min_angle_deg.
#include <cmath>
#include <string>

#include "common.cuh"
#include "geom.cuh"
#include "api_guard.h"
#include "matcher_internal.h"

namespace r3dgpu {
namespace {

constexpr int kMaxPairs = 16;  // multi_stereo.cpp:23
constexpr float kInfF = __builtin_huge_valf();

R3D_DEVICE int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// multi_stereo.cpp:44-72
R3D_DEVICE float sample_disparity(const r3dgpu_pair_geometry& g, double u, double v) {
  const int w = g.width, h = g.height;
  if (!(u > -0.5 && v > -0.5 && u < w - 0.5 && v < h - 0.5)) return kInfF;
  const int x0 = clampi(static_cast<int>(floor(u)), 0, w - 1);
  const int y0 = clampi(static_cast<int>(floor(v)), 0, h - 1);
  const int x1 = x0 + 1 < w ? x0 + 1 : w - 1;
  const int y1 = y0 + 1 < h ? y0 + 1 : h - 1;
  const float d00 = g.disparity[y0 * g.stride + x0];
  const float d10 = g.disparity[y0 * g.stride + x1];
  const float d01 = g.disparity[y1 * g.stride + x0];
  const float d11 = g.disparity[y1 * g.stride + x1];
  if (r3dsimt::finitef(d00) && r3dsimt::finitef(d10) && r3dsimt::finitef(d01) && r3dsimt::finitef(d11)) {
    const float lo = fminf(fminf(d00, d10), fminf(d01, d11));
    const float hi = fmaxf(fmaxf(d00, d10), fmaxf(d01, d11));
    if (__fsub_rn(hi, lo) <= 1.0F) {
      const double ux = u - x0, vy = v - y0;
      const float fx = static_cast<float>(ux < 0.0 ? 0.0 : (ux > 1.0 ? 1.0 : ux));
      const float fy = static_cast<float>(vy < 0.0 ? 0.0 : (vy > 1.0 ? 1.0 : vy));
      const float top = __fadd_rn(d00, __fmul_rn(fx, __fsub_rn(d10, d00)));
      const float bottom = __fadd_rn(d01, __fmul_rn(fx, __fsub_rn(d11, d01)));
      return __fadd_rn(top, __fmul_rn(fy, __fsub_rn(bottom, top)));
    }
  }
  const int xn = clampi(static_cast<int>(llround(u)), 0, w - 1);
  const int yn = clampi(static_cast<int>(llround(v)), 0, h - 1);
  return g.disparity[yn * g.stride + xn];
}


struct Cand {
  double w, k;
  float conf;
  int pair;
};

R3D_GLOBAL void combine_pairs_kernel(r3dgpu_depth_grid grid, const r3dgpu_pair_geometry* R3D_RESTRICT pairs,
                                     int count, r3dgpu_multi_stereo_options o, double cos_min_angle, float* depth,
                                     float* confidence, uint16_t* pair_mask, int64_t stride) {
  const int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= static_cast<int64_t>(grid.width) * grid.height) return;
  const int y = static_cast<int>(idx / grid.width), x = static_cast<int>(idx - static_cast<int64_t>(y) * grid.width);
  const int64_t out = static_cast<int64_t>(y) * stride + x;
  depth[out] = 0.0F;
  confidence[out] = 0.0F;
  pair_mask[out] = 0;
  const double px = x, py = y;
  Cand cand[kMaxPairs];
  int n = 0;
  for (int i = 0; i < count; ++i) {
    const r3dgpu_pair_geometry& g = pairs[i];
    const double rx = row3(g.grid_to_rect, 0, px, py, 1.0);
    const double ry = row3(g.grid_to_rect, 1, px, py, 1.0);
    const double c = row3(g.grid_to_rect, 2, px, py, 1.0);
    if (!(c > 1e-9)) continue;
    const double u = rx / c, v = ry / c;
    const float d = sample_disparity(g, u, v);
    if (!r3dsimt::finitef(d) || static_cast<double>(d) <= g.offset) continue;
    Cand& cd = cand[n++];
    cd.k = g.fb / c;
    cd.w = (static_cast<double>(d) - g.offset) / cd.k;
    cd.pair = i;
    cd.conf = 0.0F;
    if (g.confidence != nullptr) {
      const int xn = clampi(static_cast<int>(llround(u)), 0, g.width - 1);
      const int yn = clampi(static_cast<int>(llround(v)), 0, g.height - 1);
      cd.conf = g.confidence[yn * g.stride + xn];
    }
  }
  const int min_pairs = o.min_pairs > 1 ? o.min_pairs : 1;
  if (n < min_pairs) return;
  int best = -1, best_support = 0;
  float best_conf = -1.0F;
  for (int i = 0; i < n; ++i) {
    int support = 0;
    float conf = 0.0F;
    for (int j = 0; j < n; ++j) {
      if (fabs(cand[j].k * (cand[j].w - cand[i].w)) <= o.inlier_px) {
        ++support;
        conf = __fadd_rn(conf, cand[j].conf);
      }
    }
    if (support > best_support || (support == best_support && conf > best_conf)) {
      best = i;
      best_support = support;
      best_conf = conf;
    }
  }
  int used[kMaxPairs];
  int m = 0;
  for (int j = 0; j < n; ++j)
    if (fabs(cand[j].k * (cand[j].w - cand[best].w)) <= o.inlier_px) used[m++] = j;
  double w_opt = 0.0;
  while (m > 0) {
    double sw = 0.0, swx = 0.0;
    for (int t = 0; t < m; ++t) {
      const Cand& cd = cand[used[t]];
      sw += cd.k * cd.k;
      swx += cd.k * cd.k * cd.w;
    }
    w_opt = swx / sw;
    int worst = -1;
    double worst_res = o.max_reprojection_px;
    for (int t = 0; t < m; ++t) {
      const Cand& cd = cand[used[t]];
      const double res = fabs(cd.k * (cd.w - w_opt));
      if (res > worst_res) {
        worst_res = res;
        worst = t;
      }
    }
    if (worst < 0) break;
    used[worst] = used[--m];
  }
  const bool majority = m > n - m || (m >= 2 && m >= n - m);
  if (m < min_pairs || !majority || !(w_opt > 0.0)) return;
  const double z = 1.0 / w_opt;
  // ray = R^T (K^-1 (x, y, 1)): world direction with unit depth in the grid camera.
  const double ax = row3(grid.k_inv, 0, px, py, 1.0), ay = row3(grid.k_inv, 1, px, py, 1.0),
               az = row3(grid.k_inv, 2, px, py, 1.0);
  const double ray[3] = {row3(grid.rot_t, 0, ax, ay, az), row3(grid.rot_t, 1, ax, ay, az),
                         row3(grid.rot_t, 2, ax, ay, az)};
  double xw[3], tb[3];
  for (int k = 0; k < 3; ++k) xw[k] = grid.center[k] + z * ray[k];
  for (int k = 0; k < 3; ++k) tb[k] = grid.center[k] - xw[k];
  {
    const double nn = (tb[0] * tb[0] + tb[1] * tb[1]) + tb[2] * tb[2];
    if (nn > 0.0) {
      const double s = sqrt(nn);
      for (int k = 0; k < 3; ++k) tb[k] = tb[k] / s;
    }
  }
  bool wide = false;
  float conf = 0.0F;
  uint32_t mask = 0;
  for (int t = 0; t < m; ++t) {
    const Cand& cd = cand[used[t]];
    mask |= 1u << cd.pair;
    const double* pc = pairs[cd.pair].partner_center;
    double tp[3] = {pc[0] - xw[0], pc[1] - xw[1], pc[2] - xw[2]};
    const double nn = (tp[0] * tp[0] + tp[1] * tp[1]) + tp[2] * tp[2];
    if (nn > 0.0) {
      const double s = sqrt(nn);
      for (int k = 0; k < 3; ++k) tp[k] = tp[k] / s;
    }
    const double dot = (tb[0] * tp[0] + tb[1] * tp[1]) + tb[2] * tp[2];
    wide = wide || dot <= cos_min_angle;
    conf = __fadd_rn(conf, cd.conf);
  }
  if (!wide) return;
  depth[out] = static_cast<float>(z);
  confidence[out] = __fdiv_rn(conf, static_cast<float>(m));
  pair_mask[out] = static_cast<uint16_t>(mask);
}

void check_args(const r3dgpu_depth_grid* grid, const r3dgpu_pair_geometry* pairs, int count, float* depth,
                float* confidence, uint16_t* mask, int64_t stride) {
  if (grid == nullptr || (count > 0 && pairs == nullptr) || depth == nullptr || confidence == nullptr ||
      mask == nullptr)
    fail(R3DGPU_EINVAL, "combine_pairs: null argument");
  if (count < 0 || count > kMaxPairs)
    fail(R3DGPU_EINVAL, "combine_pairs: at most " + std::to_string(kMaxPairs) + " pairs per view (" +
                            std::to_string(count) + " given)");
  if (grid->width < 0 || grid->height < 0 || stride < grid->width)
    fail(R3DGPU_EINVAL, "combine_pairs: bad grid size or stride");
  for (int i = 0; i < count; ++i)
    if (pairs[i].disparity == nullptr || pairs[i].width <= 0 || pairs[i].height <= 0 ||
        pairs[i].stride < pairs[i].width)
      fail(R3DGPU_EINVAL, "combine_pairs: pair " + std::to_string(i) + " has no disparity map");
}

void launch_combine(const r3dgpu_depth_grid& grid, const r3dgpu_pair_geometry* dpairs, int count,
                    const r3dgpu_multi_stereo_options& o, float* depth, float* confidence, uint16_t* mask,
                    int64_t stride, cudaStream_t s) {
  const int64_t n = static_cast<int64_t>(grid.width) * grid.height;
  if (n == 0) return;
  const double cos_min = cos(o.min_angle_deg * 3.14159265358979323846 / 180.0);
  R3D_LAUNCH(combine_pairs_kernel, static_cast<unsigned>(ceil_div64(n, 256)), 256, 0, s, grid, dpairs, count, o,
             cos_min, depth, confidence, mask, stride);
  launched("combine_pairs_kernel");
}

}  // namespace
}  // namespace r3dgpu

using namespace r3dgpu;

extern "C" {

void r3dgpu_default_multi_stereo_options(r3dgpu_multi_stereo_options* out) {
  if (out == nullptr) return;
  *out = r3dgpu_multi_stereo_options{2.0, 1.0, 3.0, 1, 0};
}

r3dgpu_status r3dgpu_combine_pairs(const r3dgpu_depth_grid* grid, const r3dgpu_pair_geometry* pairs, int32_t count,
                                   const r3dgpu_multi_stereo_options* options, float* depth, float* confidence,
                                   uint16_t* pair_mask, int64_t stride, void* stream) {
  return guard([&] {
    check_args(grid, pairs, count, depth, confidence, pair_mask, stride);
    r3dgpu_multi_stereo_options o{};
    if (options != nullptr) {
      o = *options;
    } else {
      r3dgpu_default_multi_stereo_options(&o);
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    thread_local DeviceBuffer<r3dgpu_pair_geometry> dp;
    dp.reserve(kMaxPairs);
    if (count > 0)
      R3D_CUDA(cudaMemcpyAsync(dp.get(), pairs, sizeof(r3dgpu_pair_geometry) * count, cudaMemcpyHostToDevice, s));
    launch_combine(*grid, dp.get(), count, o, depth, confidence, pair_mask, stride, s);
    R3D_CUDA(cudaStreamSynchronize(s));
  });
}

r3dgpu_status r3dgpu_combine_pairs_host(const r3dgpu_depth_grid* grid, const r3dgpu_pair_geometry* pairs,
                                        int32_t count, const r3dgpu_multi_stereo_options* options, float* depth,
                                        float* confidence, uint16_t* pair_mask, int64_t stride) {
  return guard([&] {
    check_args(grid, pairs, count, depth, confidence, pair_mask, stride);
    cudaStream_t s = nullptr;
    const int w = grid->width, h = grid->height;
    size_t bytes = static_cast<size_t>(w) * h * (4 + 4 + 2) + 1024;
    for (int i = 0; i < count; ++i)
      bytes += (pairs[i].confidence ? 8 : 4) * static_cast<size_t>(pairs[i].width) * pairs[i].height + 512;
    thread_local DeviceBuffer<unsigned char> io;
    io.reserve(bytes);
    unsigned char* p = io.get();
    auto take = [&](size_t n) {
      unsigned char* at = p;
      p += (n + 255) & ~static_cast<size_t>(255);
      return at;
    };
    r3dgpu_pair_geometry dev[kMaxPairs];
    for (int i = 0; i < count; ++i) {
      dev[i] = pairs[i];
      const int pw = pairs[i].width, ph = pairs[i].height;
      float* dd = reinterpret_cast<float*>(take(4 * static_cast<size_t>(pw) * ph));
      R3D_CUDA(cudaMemcpy2DAsync(dd, 4 * pw, pairs[i].disparity, 4 * pairs[i].stride, 4 * pw, ph,
                                 cudaMemcpyHostToDevice, s));
      dev[i].disparity = dd;
      if (pairs[i].confidence != nullptr) {
        float* dc = reinterpret_cast<float*>(take(4 * static_cast<size_t>(pw) * ph));
        R3D_CUDA(cudaMemcpy2DAsync(dc, 4 * pw, pairs[i].confidence, 4 * pairs[i].stride, 4 * pw, ph,
                                   cudaMemcpyHostToDevice, s));
        dev[i].confidence = dc;
      }
      dev[i].stride = pw;
    }
    float* od = reinterpret_cast<float*>(take(4 * static_cast<size_t>(w) * h));
    float* oc = reinterpret_cast<float*>(take(4 * static_cast<size_t>(w) * h));
    uint16_t* om = reinterpret_cast<uint16_t*>(take(2 * static_cast<size_t>(w) * h));
    const r3dgpu_status st = r3dgpu_combine_pairs(grid, dev, count, options, od, oc, om, w, s);
    if (st != R3DGPU_OK) fail(st, r3dgpu_last_error());
    R3D_CUDA(cudaMemcpy2DAsync(depth, 4 * stride, od, 4 * static_cast<size_t>(w), 4 * static_cast<size_t>(w), h,
                               cudaMemcpyDeviceToHost, s));
    R3D_CUDA(cudaMemcpy2DAsync(confidence, 4 * stride, oc, 4 * static_cast<size_t>(w), 4 * static_cast<size_t>(w), h,
                               cudaMemcpyDeviceToHost, s));
    R3D_CUDA(cudaMemcpy2DAsync(pair_mask, 2 * stride, om, 2 * static_cast<size_t>(w), 2 * static_cast<size_t>(w), h,
                               cudaMemcpyDeviceToHost, s));
    R3D_CUDA(cudaStreamSynchronize(s));
  });
}

}  // extern "C"
