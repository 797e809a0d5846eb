// CPU oracle of the R3DMVS depth-map stages after the matcher — TEST
// INFRASTRUCTURE ONLY (loaded by the tests, the smoke check and bench.py's
// CPU-baseline leg; the product never calls it).
//
// Restates, in plain C++ written for this project, the geometric consistency
// check of depth maps (rhiestan/Regard3D_MVS src/r3d/mvs/consistency.cpp:
// erode_depth_edges :57-110, remove_depth_speckles :112-136,
// remove_weak_depths :138-227, remove_depth_halos :229-341,
// prepare_depth_map :343-360, check_consistency :362-453,
// filter_depth_maps :455-485) and the patch-based depth refinement
// (src/r3d/mvs/refinement.cpp: evaluate_view :46-152, centre_motion
// :155-165, initial_slope :167-196, gaussian_blur :198-238,
// make_refinement_image :242-269, refine_depth_map :271-449) in double
// precision with sequential sums; the reference's Eigen LDLT solve is
// restated as LDL^T with symmetric diagonal pivoting. Maps are r3dgpu_depth_map structs with host
// pointers. Segments are found by breadth-first search in raster order, as
// the reference does; doubles follow the reference's operation order (no
// contraction, -ffp-contract=off).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "../include/r3dgpu.h"

extern "C" int orc_remove_speckles(float* disp, int w, int h, int min_size, float max_diff);
extern "C" const char* orc_last_error();

namespace omvs {

using Map = r3dgpu_depth_map;
constexpr float kInf = std::numeric_limits<float>::infinity();

thread_local std::string g_error;

float& depth(const Map& m, int x, int y) { return m.depth[static_cast<int64_t>(y) * m.stride + x]; }
bool valid(const Map& m, int x, int y) { return depth(m, x, y) > 0.0F; }
const uint8_t* rgb(const Map& m, int x, int y) { return m.color + static_cast<int64_t>(y) * m.color_stride + 3 * x; }

uint64_t num_valid(const Map& m) {
  uint64_t n = 0;
  for (int y = 0; y < m.height; ++y)
    for (int x = 0; x < m.width; ++x) n += valid(m, x, y) ? 1 : 0;
  return n;
}

// :57-110
uint64_t erode_depth_edges(const Map& m, int radius, double discontinuity, bool holes) {
  if (radius <= 0) return 0;
  const int w = m.width, h = m.height;
  const auto jump = static_cast<float>(discontinuity);
  std::vector<uint8_t> edge(static_cast<size_t>(w) * h, 0);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      const float z = depth(m, x, y);
      if (z <= 0.0F) continue;
      auto differs = [&](int nx, int ny) {
        if (nx < 0 || ny < 0 || nx >= w || ny >= h) return false;
        const float zn = depth(m, nx, ny);
        return zn > 0.0F ? std::abs(zn - z) > jump * std::min(z, zn) : holes;
      };
      if (differs(x - 1, y) || differs(x + 1, y) || differs(x, y - 1) || differs(x, y + 1))
        edge[static_cast<size_t>(y) * w + x] = 1;
    }
  const int r = radius - 1;
  uint64_t removed = 0;
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      if (depth(m, x, y) <= 0.0F) continue;
      bool near = false;
      for (int dy = -r; dy <= r && !near; ++dy)
        for (int dx = -r; dx <= r && !near; ++dx) {
          const int nx = x + dx, ny = y + dy;
          near = nx >= 0 && ny >= 0 && nx < w && ny < h && edge[static_cast<size_t>(ny) * w + nx] != 0;
        }
      if (near) {
        depth(m, x, y) = 0.0F;  // the edge flags above are final, so in-place removal is safe
        ++removed;
      }
    }
  return removed;
}

std::vector<float> log_depth(const Map& m) {
  std::vector<float> d(static_cast<size_t>(m.width) * m.height);
  for (int y = 0; y < m.height; ++y)
    for (int x = 0; x < m.width; ++x) {
      const float z = depth(m, x, y);
      d[static_cast<size_t>(y) * m.width + x] = z > 0.0F ? std::log(z) : kInf;
    }
  return d;
}

// :112-136
uint64_t remove_depth_speckles(const Map& m, int min_size, double max_relative_step) {
  if (min_size <= 1 || m.width == 0) return 0;
  std::vector<float> d = log_depth(m);
  if (orc_remove_speckles(d.data(), m.width, m.height, min_size, static_cast<float>(std::log1p(max_relative_step))) != 0)
    throw std::runtime_error(orc_last_error());
  uint64_t removed = 0;
  for (int y = 0; y < m.height; ++y)
    for (int x = 0; x < m.width; ++x)
      if (depth(m, x, y) > 0.0F && !std::isfinite(d[static_cast<size_t>(y) * m.width + x])) {
        depth(m, x, y) = 0.0F;
        ++removed;
      }
  return removed;
}

// :138-227
uint64_t remove_weak_depths(const Map& m, const r3dgpu_consistency_options& o) {
  const int w = m.width, h = m.height;
  const bool segments = o.weak_segment > 0.0;
  if (o.weak_texture <= 0.0 || (!segments && !o.reject_weak) || m.color == nullptr || w == 0) return 0;
  const double max_var = o.weak_texture * o.weak_texture;
  const size_t n = static_cast<size_t>(w) * h;
  std::vector<uint8_t> weak(n, 0);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      if (depth(m, x, y) <= 0.0F) continue;
      double sum = 0.0, sum2 = 0.0;
      int count = 0;
      for (int v = std::max(y - 3, 0); v <= std::min(y + 3, h - 1); ++v)
        for (int u = std::max(x - 3, 0); u <= std::min(x + 3, w - 1); ++u) {
          const uint8_t* c = rgb(m, u, v);
          const double g = 0.299 * c[0] + 0.587 * c[1] + 0.114 * c[2];
          sum += g;
          sum2 += g * g;
          ++count;
        }
      const double mean = sum / count;
      if (sum2 / count - mean * mean < max_var) weak[static_cast<size_t>(y) * w + x] = 1;
    }
  uint64_t removed = 0;
  if (o.reject_weak) {
    for (size_t i = 0; i < n; ++i)
      if (weak[i] != 0) {
        depth(m, static_cast<int>(i % w), static_cast<int>(i / w)) = 0.0F;
        ++removed;
      }
    return removed;
  }
  const auto max_size = static_cast<size_t>(o.weak_segment * static_cast<double>(n));
  const auto max_step = static_cast<float>(std::log1p(o.speckle_step));
  const std::vector<float> d = log_depth(m);
  std::vector<uint8_t> seen(n, 0);
  std::vector<uint32_t> seg;
  for (size_t start = 0; start < n; ++start) {
    if (seen[start] != 0 || !std::isfinite(d[start])) continue;
    seg.assign(1, static_cast<uint32_t>(start));
    seen[start] = 1;
    size_t weak_count = 0;
    for (size_t head = 0; head < seg.size(); ++head) {
      const size_t i = seg[head];
      weak_count += weak[i];
      const int x = static_cast<int>(i % w);
      auto visit = [&](size_t j) {
        if (seen[j] == 0 && std::abs(d[j] - d[i]) <= max_step) {
          seen[j] = 1;
          seg.push_back(static_cast<uint32_t>(j));
        }
      };
      if (x > 0) visit(i - 1);
      if (x + 1 < w) visit(i + 1);
      if (i >= static_cast<size_t>(w)) visit(i - w);
      if (i + w < n) visit(i + w);
    }
    if (seg.size() < max_size && 2 * weak_count >= seg.size()) {
      for (const uint32_t i : seg) depth(m, static_cast<int>(i % w), static_cast<int>(i / w)) = 0.0F;
      removed += seg.size();
    }
  }
  return removed;
}

// :229-341
uint64_t remove_depth_halos(const Map& m, int max_px, int colour_step) {
  const int w = m.width, h = m.height;
  if (max_px <= 0 || m.color == nullptr || w == 0) return 0;
  const size_t n = static_cast<size_t>(w) * h;
  std::vector<uint8_t> hole(n, 0);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      bool empty = true;
      for (int v = std::max(y - 2, 0); v <= std::min(y + 2, h - 1) && empty; ++v)
        for (int u = std::max(x - 2, 0); u <= std::min(x + 2, w - 1) && empty; ++u) empty = depth(m, u, v) <= 0.0F;
      hole[static_cast<size_t>(y) * w + x] = empty ? 1 : 0;
    }
  auto differs = [&](int x0, int y0, int x1, int y1) {
    const uint8_t* a = rgb(m, x0, y0);
    const uint8_t* b = rgb(m, x1, y1);
    for (int c = 0; c < 3; ++c)
      if (std::abs(static_cast<int>(a[c]) - static_cast<int>(b[c])) >= colour_step) return true;
    return false;
  };
  const int dirs[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {1, -1}, {-1, 1}, {-1, -1}};
  std::vector<uint8_t> halo(n, 0);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      if (depth(m, x, y) <= 0.0F) continue;
      for (const auto& dir : dirs) {
        int to_hole = 0;
        for (int s = 1; s <= max_px; ++s) {
          const int u = x + s * dir[0], v = y + s * dir[1];
          if (u < 0 || v < 0 || u >= w || v >= h || differs(u, v, x, y)) break;
          if (hole[static_cast<size_t>(v) * w + u] != 0) {
            to_hole = s;
            break;
          }
        }
        if (to_hole == 0) continue;
        bool edge = false;
        for (int s = 1; s <= max_px - to_hole; ++s) {
          const int u = x - s * dir[0], v = y - s * dir[1];
          if (u < 0 || v < 0 || u >= w || v >= h) break;
          if (differs(u, v, x, y)) {
            edge = true;
            break;
          }
          if (depth(m, u, v) <= 0.0F) break;
        }
        if (edge) {
          halo[static_cast<size_t>(y) * w + x] = 1;
          break;
        }
      }
    }
  uint64_t removed = 0;
  for (size_t i = 0; i < n; ++i)
    if (halo[i] != 0) {
      depth(m, static_cast<int>(i % w), static_cast<int>(i / w)) = 0.0F;
      ++removed;
    }
  return removed;
}

void prepare(const Map& m, const r3dgpu_consistency_options& o, r3dgpu_consistency_stats& st) {
  st.input += num_valid(m);
  if (o.min_confidence > 0.0F)
    for (int y = 0; y < m.height; ++y)
      for (int x = 0; x < m.width; ++x)
        if (depth(m, x, y) > 0.0F && m.confidence[static_cast<int64_t>(y) * m.stride + x] < o.min_confidence) {
          depth(m, x, y) = 0.0F;
          ++st.unconfident;
        }
  st.eroded += erode_depth_edges(m, o.edge_erosion, o.discontinuity, o.erode_holes != 0);
}

uint16_t pair_bit(const Map& m, uint32_t view) {
  for (uint32_t i = 0; i < m.num_partners; ++i)
    if (m.partners[i] == view) return static_cast<uint16_t>(1u << i);
  return 0;
}

// R v and R^T v for a row-major 3x3 R.
void mul(const double* r, const double* v, double* out) {
  for (int i = 0; i < 3; ++i) out[i] = r[3 * i] * v[0] + r[3 * i + 1] * v[1] + r[3 * i + 2] * v[2];
}
void mul_t(const double* r, const double* v, double* out) {
  for (int i = 0; i < 3; ++i) out[i] = r[i] * v[0] + r[3 + i] * v[1] + r[6 + i] * v[2];
}

// :362-453. `m` is checked against `nbs`; its depth may alias no neighbour.
void check(const Map& m, const Map* const* nbs, int count, const r3dgpu_consistency_options& o,
           r3dgpu_consistency_stats& st) {
  const int w = m.width, h = m.height;
  std::vector<uint8_t> support(static_cast<size_t>(w) * h, 0);
  std::vector<float> averaged(static_cast<size_t>(w) * h, 0.0F);
  const auto rel_tol = static_cast<float>(o.max_relative_depth_error);
  const double tol2 = o.max_reprojection_px * o.max_reprojection_px;
  const r3dgpu_pinhole_camera& c = m.camera;
#pragma omp parallel for schedule(static)
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      const float z = depth(m, x, y);
      if (z <= 0.0F) continue;
      const double pix[3] = {static_cast<double>(x), static_cast<double>(y), 1.0};
      double a[3], ray[3], xw[3];
      mul(c.k_inv, pix, a);
      mul_t(c.rotation, a, ray);
      for (int i = 0; i < 3; ++i) xw[i] = c.center[i] + ray[i] * static_cast<double>(z);
      int agree = 0;
      double depth_sum = z;
      const uint16_t mask = m.pair_mask ? m.pair_mask[static_cast<int64_t>(y) * m.stride + x] : 0;
      for (int j = 0; j < count; ++j) {
        const Map& n = *nbs[j];
        if (n.width == 0) continue;
        const uint16_t bit_m = pair_bit(m, n.view);
        const r3dgpu_pinhole_camera& cn = n.camera;
        const double rel[3] = {xw[0] - cn.center[0], xw[1] - cn.center[1], xw[2] - cn.center[2]};
        double xc[3];
        mul(cn.rotation, rel, xc);
        if (!(xc[2] > 0.0)) continue;
        const double inv_z = 1.0 / xc[2];
        const double qx = cn.intrinsics.fx * xc[0] * inv_z + cn.intrinsics.cx;
        const double qy = cn.intrinsics.fy * xc[1] * inv_z + cn.intrinsics.cy;
        const long long ix = std::llround(qx), iy = std::llround(qy);
        if (ix < 0 || iy < 0 || ix >= n.width || iy >= n.height) continue;
        const int64_t ni = iy * n.stride + ix;
        const float zn = n.depth[ni];
        if (zn <= 0.0F || std::abs(zn - static_cast<float>(xc[2])) > rel_tol * zn) continue;
        const double cam[3] = {(static_cast<double>(ix) - cn.intrinsics.cx) / cn.intrinsics.fx * zn,
                               (static_cast<double>(iy) - cn.intrinsics.cy) / cn.intrinsics.fy * zn,
                               static_cast<double>(zn)};
        double back[3], bc[3];
        mul_t(cn.rotation, cam, back);
        for (int i = 0; i < 3; ++i) back[i] += cn.center[i];
        const double rel2[3] = {back[0] - c.center[0], back[1] - c.center[1], back[2] - c.center[2]};
        mul(c.rotation, rel2, bc);
        if (!(bc[2] > 0.0)) continue;
        const double inv_b = 1.0 / bc[2];
        const double px = c.intrinsics.fx * bc[0] * inv_b + c.intrinsics.cx;
        const double py = c.intrinsics.fy * bc[1] * inv_b + c.intrinsics.cy;
        const double dx = px - x, dy = py - y;
        if (dx * dx + dy * dy > tol2) continue;
        if (o.independent_support && bit_m != 0 && mask == bit_m) {
          const uint16_t bit_n = pair_bit(n, m.view);
          if (bit_n != 0 && n.pair_mask && n.pair_mask[ni] == bit_n) continue;
        }
        ++agree;
        depth_sum += bc[2];
      }
      averaged[static_cast<size_t>(y) * w + x] = static_cast<float>(depth_sum / (agree + 1));
      support[static_cast<size_t>(y) * w + x] = static_cast<uint8_t>(std::min(agree, 255));
    }
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      if (depth(m, x, y) <= 0.0F) continue;
      const int sup = support[static_cast<size_t>(y) * w + x];
      const int pairs = m.pair_mask ? __builtin_popcount(m.pair_mask[static_cast<int64_t>(y) * m.stride + x]) : 0;
      if (sup < o.min_views || sup + pairs < o.min_evidence) {
        depth(m, x, y) = 0.0F;
        ++st.rejected;
      } else if (o.average_depths) {
        depth(m, x, y) = averaged[static_cast<size_t>(y) * w + x];
      }
    }
  if (m.support)
    for (int y = 0; y < h; ++y)
      for (int x = 0; x < w; ++x) m.support[static_cast<int64_t>(y) * m.stride + x] = support[static_cast<size_t>(y) * w + x];
  st.weak += remove_weak_depths(m, o);
  st.halo += remove_depth_halos(m, o.halo_px, o.halo_colour);
  st.speckles += remove_depth_speckles(m, o.speckle_size, o.speckle_step);
  st.output += num_valid(m);
}

// :455-485: prepare all, then check copies of the maps against the prepared
// originals, then replace the depths.
void filter(Map* maps, int count, const int32_t* off, const int32_t* idx, const r3dgpu_consistency_options& o,
            r3dgpu_consistency_stats& st) {
  st = r3dgpu_consistency_stats{};
  for (int i = 0; i < count; ++i) prepare(maps[i], o, st);
  std::vector<std::vector<float>> copies(static_cast<size_t>(count));
  std::vector<Map> filtered(maps, maps + count);
  for (int i = 0; i < count; ++i) {
    copies[i].resize(static_cast<size_t>(maps[i].width) * maps[i].height);
    for (int y = 0; y < maps[i].height; ++y)
      for (int x = 0; x < maps[i].width; ++x) copies[i][static_cast<size_t>(y) * maps[i].width + x] = depth(maps[i], x, y);
    filtered[i].depth = copies[i].data();
    filtered[i].stride = maps[i].width;  // the copy's pair mask and support below are dense too
  }
  std::vector<std::vector<uint16_t>> masks(static_cast<size_t>(count));
  std::vector<std::vector<uint8_t>> supports(static_cast<size_t>(count));
  for (int i = 0; i < count; ++i) {
    const size_t px = static_cast<size_t>(maps[i].width) * maps[i].height;
    masks[i].assign(px, 0);
    supports[i].assign(px, 0);
    if (maps[i].pair_mask)
      for (int y = 0; y < maps[i].height; ++y)
        for (int x = 0; x < maps[i].width; ++x)
          masks[i][static_cast<size_t>(y) * maps[i].width + x] = maps[i].pair_mask[static_cast<int64_t>(y) * maps[i].stride + x];
    filtered[i].pair_mask = masks[i].data();
    filtered[i].support = supports[i].data();
    filtered[i].confidence = nullptr;  // not read by the check
  }
  std::vector<const Map*> nb;
  for (int i = 0; i < count; ++i) {
    nb.clear();
    for (int k = off[i]; k < off[i + 1]; ++k) nb.push_back(&maps[idx[k]]);
    check(filtered[i], nb.data(), static_cast<int>(nb.size()), o, st);
  }
  for (int i = 0; i < count; ++i)
    for (int y = 0; y < maps[i].height; ++y)
      for (int x = 0; x < maps[i].width; ++x) {
        const size_t k = static_cast<size_t>(y) * maps[i].width + x;
        depth(maps[i], x, y) = copies[i][k];
        if (maps[i].support) maps[i].support[static_cast<int64_t>(y) * maps[i].stride + x] = supports[i][k];
      }
}


// ---------------------------------------------------------------- refinement
namespace ref {

constexpr int kMaxSamples = 225;
constexpr int kMaxViews = 8;
constexpr double kDiscontinuity = 0.05;

struct Geo {
  double m[9], b[3];
  const float* data;
  int64_t stride;
  int w, h;
};

struct Sample {
  double dx, dy, sx, sy;
};

struct Res {
  bool valid = false;
  double ncc = 0.0;
  double h[3][3] = {};
  double g[3] = {};
};

double row3(const double* m, int i, double x, double y, double z) { return m[3 * i] * x + m[3 * i + 1] * y + m[3 * i + 2] * z; }

// refinement.cpp:46-152
Res evaluate_view(const Geo& geo, double x, double y, const double* th, const std::vector<Sample>& samples,
                  const double* n0, bool jac) {
  Res res;
  const double max_x = geo.w - 1, max_y = geo.h - 1;
  const double hc[3] = {row3(geo.m, 0, x, y, 1.0), row3(geo.m, 1, x, y, 1.0), row3(geo.m, 2, x, y, 1.0)};
  const int n = static_cast<int>(samples.size());
  double v[kMaxSamples], dv[kMaxSamples];
  double sum = 0.0;
  for (int s = 0; s < n; ++s) {
    const Sample& sm = samples[s];
    const double wq = th[0] + th[1] * sm.sx + th[2] * sm.sy;
    double h[3];
    for (int i = 0; i < 3; ++i) h[i] = hc[i] + geo.m[3 * i] * sm.dx + geo.m[3 * i + 1] * sm.dy + geo.b[i] * wq;
    if (!(h[2] > 0.0)) return res;
    const double inv_z = 1.0 / h[2];
    const double px = h[0] * inv_z, py = h[1] * inv_z;
    if (!(px >= 0.0 && py >= 0.0 && px < max_x && py < max_y)) return res;
    const int ix = static_cast<int>(px), iy = static_cast<int>(py);
    const double fx = px - ix, fy = py - iy;
    const float* r0 = geo.data + iy * geo.stride + 3 * ix;
    const float* r1 = r0 + geo.stride;
    double val[3];
    for (int c = 0; c < 3; ++c)
      val[c] = (1.0 - fy) * ((1.0 - fx) * r0[c] + fx * r0[3 + c]) + fy * ((1.0 - fx) * r1[c] + fx * r1[3 + c]);
    v[s] = val[0];
    sum += val[0];
    if (jac) {
      const double dpx = (geo.b[0] - px * geo.b[2]) * inv_z;
      const double dpy = (geo.b[1] - py * geo.b[2]) * inv_z;
      dv[s] = val[1] * dpx + val[2] * dpy;
    }
  }
  const double mean = sum / n;
  double norm2 = 0.0;
  for (int s = 0; s < n; ++s) {
    v[s] -= mean;
    norm2 += v[s] * v[s];
  }
  if (!(norm2 > 1e-6 * n)) return res;
  const double inv_norm = 1.0 / std::sqrt(norm2);
  double ncc = 0.0;
  for (int s = 0; s < n; ++s) {
    v[s] *= inv_norm;
    ncc += v[s] * n0[s];
  }
  res.valid = true;
  res.ncc = ncc;
  if (!jac) return res;
  double dmean[3] = {0.0, 0.0, 0.0};
  for (int s = 0; s < n; ++s) {
    const double e[3] = {1.0, samples[s].sx, samples[s].sy};
    for (int i = 0; i < 3; ++i) dmean[i] += dv[s] * e[i];
  }
  for (double& d : dmean) d /= n;
  double proj[3] = {0.0, 0.0, 0.0};
  for (int s = 0; s < n; ++s) {
    const double e[3] = {1.0, samples[s].sx, samples[s].sy};
    for (int i = 0; i < 3; ++i) proj[i] += v[s] * (dv[s] * e[i] - dmean[i]);
  }
  for (int s = 0; s < n; ++s) {
    const double e[3] = {1.0, samples[s].sx, samples[s].sy};
    double j[3];
    for (int i = 0; i < 3; ++i) j[i] = ((dv[s] * e[i] - dmean[i]) - v[s] * proj[i]) * inv_norm;
    for (int a = 0; a < 3; ++a) {
      for (int b = 0; b < 3; ++b) res.h[a][b] += j[a] * j[b];
      res.g[a] += j[a] * (v[s] - n0[s]);
    }
  }
  return res;
}

// refinement.cpp:155-165
double centre_motion(const Geo& g, double x, double y, double w) {
  double h[3];
  for (int i = 0; i < 3; ++i) h[i] = row3(g.m, i, x, y, 1.0) + g.b[i] * w;
  if (!(h[2] > 0.0)) return 0.0;
  const double px = h[0] / h[2], py = h[1] / h[2];
  return std::hypot(g.b[0] - px * g.b[2], g.b[1] - py * g.b[2]) / h[2];
}

// refinement.cpp:167-196
double initial_slope(const std::vector<float>& depth, int w, int h, int x, int y, int ax, int ay) {
  const float z = depth[static_cast<size_t>(y) * w + x];
  auto neighbour = [&](int k, double& wn) {
    const int nx = x + k * ax, ny = y + k * ay;
    if (nx < 0 || ny < 0 || nx >= w || ny >= h) return false;
    const float zn = depth[static_cast<size_t>(ny) * w + nx];
    if (!(zn > 0.0F) || std::abs(zn - z) > kDiscontinuity * std::min(z, zn)) return false;
    wn = 1.0 / zn;
    return true;
  };
  double wp = 0.0, wm = 0.0;
  const bool p = neighbour(1, wp), m = neighbour(-1, wm);
  const double w0 = 1.0 / z;
  if (p && m) return 0.5 * (wp - wm);
  if (p) return wp - w0;
  if (m) return w0 - wm;
  return 0.0;
}

// -(H + damping)^-1 g by LDL^T with symmetric diagonal pivoting.
void solve_damped(const double (&hh)[3][3], const double* gg, double* delta) {
  double a[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a[i][j] = hh[i][j];
  for (int i = 0; i < 3; ++i) a[i][i] = a[i][i] * (1.0 + 1e-6) + 1e-12;
  int perm[3] = {0, 1, 2};
  double l[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}, d[3];
  for (int k = 0; k < 3; ++k) {
    int piv = k;
    for (int i = k + 1; i < 3; ++i)
      if (std::abs(a[i][i]) > std::abs(a[piv][piv])) piv = i;
    if (piv != k) {
      for (int j = 0; j < 3; ++j) std::swap(a[k][j], a[piv][j]);
      for (int i = 0; i < 3; ++i) std::swap(a[i][k], a[i][piv]);
      for (int j = 0; j < k; ++j) std::swap(l[k][j], l[piv][j]);
      std::swap(perm[k], perm[piv]);
    }
    d[k] = a[k][k];
    for (int i = k + 1; i < 3; ++i) l[i][k] = d[k] != 0.0 ? a[i][k] / d[k] : 0.0;
    for (int i = k + 1; i < 3; ++i)
      for (int j = k + 1; j <= i; ++j) {
        a[i][j] -= l[i][k] * d[k] * l[j][k];
        a[j][i] = a[i][j];
      }
  }
  double y[3];
  for (int i = 0; i < 3; ++i) {
    y[i] = gg[perm[i]];
    for (int j = 0; j < i; ++j) y[i] -= l[i][j] * y[j];
  }
  for (int i = 0; i < 3; ++i) y[i] = d[i] != 0.0 ? y[i] / d[i] : 0.0;
  for (int i = 2; i >= 0; --i)
    for (int j = i + 1; j < 3; ++j) y[i] -= l[j][i] * y[j];
  for (int i = 0; i < 3; ++i) delta[perm[i]] = -y[i];
}

void mat3(const double* a, const double* b, double* out) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) out[3 * i + j] = a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j] + a[3 * i + 2] * b[6 + j];
}

Geo geometry(const r3dgpu_pinhole_camera& c0, const r3dgpu_refinement_image& v) {
  const r3dgpu_pinhole_camera& cj = v.camera;
  const double kj[9] = {cj.intrinsics.fx, 0.0, cj.intrinsics.cx, 0.0, cj.intrinsics.fy, cj.intrinsics.cy, 0.0, 0.0, 1.0};
  double r0t[9], kr[9], krr[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r0t[3 * i + j] = c0.rotation[3 * j + i];
  Geo g{};
  mat3(kj, cj.rotation, kr);
  mat3(kr, r0t, krr);
  mat3(krr, c0.k_inv, g.m);
  const double dc[3] = {c0.center[0] - cj.center[0], c0.center[1] - cj.center[1], c0.center[2] - cj.center[2]};
  for (int i = 0; i < 3; ++i) g.b[i] = kr[3 * i] * dc[0] + kr[3 * i + 1] * dc[1] + kr[3 * i + 2] * dc[2];
  g.data = v.data;
  g.stride = v.stride;
  g.w = cj.intrinsics.width;
  g.h = cj.intrinsics.height;
  return g;
}

// refinement.cpp:271-449
void refine(float* depth, float* conf, int64_t stride, const r3dgpu_pinhole_camera& cam, int w, int h,
            const r3dgpu_refinement_image& base, const r3dgpu_refinement_image* views, int num_views,
            const r3dgpu_refinement_options& o, r3dgpu_refinement_stats& st) {
  st = r3dgpu_refinement_stats{};
  if (o.radius < 1 || o.step < 1 || o.iterations < 0) throw std::runtime_error("refinement: invalid window");
  if (base.camera.intrinsics.width != w || base.camera.intrinsics.height != h)
    throw std::runtime_error("refinement: base image does not match the depth map");
  std::vector<Sample> samples;
  for (int dy = -o.radius; dy <= o.radius; dy += o.step)
    for (int dx = -o.radius; dx <= o.radius; dx += o.step)
      samples.push_back({static_cast<double>(dx), static_cast<double>(dy), static_cast<double>(dx) / o.radius,
                         static_cast<double>(dy) / o.radius});
  if (samples.size() > static_cast<size_t>(kMaxSamples)) throw std::runtime_error("refinement: window too large");
  std::vector<Geo> geos;
  for (int j = 0; j < num_views && static_cast<int>(geos.size()) < std::min(o.max_views, kMaxViews); ++j)
    geos.push_back(geometry(cam, views[j]));
  const int nv = static_cast<int>(geos.size());
  const int r = o.radius;
  std::vector<float> input(static_cast<size_t>(w) * h);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) input[static_cast<size_t>(y) * w + x] = depth[y * stride + x];
  const int n = static_cast<int>(samples.size());
  uint64_t c_input = 0, c_refined = 0, c_unconfirmed = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : c_input, c_refined, c_unconfirmed)
  for (int y = 0; y < h; ++y) {
    double n0[kMaxSamples];
    int used[kMaxViews];
    for (int x = 0; x < w; ++x) {
      const float z0 = input[static_cast<size_t>(y) * w + x];
      if (!(z0 > 0.0F)) continue;
      ++c_input;
      conf[y * stride + x] = 0.0F;
      if (nv == 0 || x < r || y < r || x >= w - r || y >= h - r) continue;
      double sum = 0.0;
      for (int s = 0; s < n; ++s) {
        n0[s] = base.data[(y + static_cast<int>(samples[s].dy)) * base.stride + 3 * (x + static_cast<int>(samples[s].dx))];
        sum += n0[s];
      }
      const double mean = sum / n;
      double norm2 = 0.0;
      for (int s = 0; s < n; ++s) {
        n0[s] -= mean;
        norm2 += n0[s] * n0[s];
      }
      if (norm2 < o.min_texture * o.min_texture * n) continue;
      const double inv_norm = 1.0 / std::sqrt(norm2);
      for (int s = 0; s < n; ++s) n0[s] *= inv_norm;
      const double w0 = 1.0 / z0;
      const double theta0[3] = {w0, r * initial_slope(input, w, h, x, y, 1, 0), r * initial_slope(input, w, h, x, y, 0, 1)};
      const double xd = x, yd = y;
      int m = 0;
      double s0 = 0.0;
      for (int j = 0; j < nv; ++j) {
        const Res vr = evaluate_view(geos[j], xd, yd, theta0, samples, n0, false);
        if (vr.valid && vr.ncc >= o.min_ncc) {
          used[m++] = j;
          s0 += vr.ncc;
        }
      }
      if (m == 0) {
        if (o.drop_unconfirmed) {
          depth[y * stride + x] = 0.0F;
          ++c_unconfirmed;
        }
        continue;
      }
      s0 /= m;
      conf[y * stride + x] = static_cast<float>(s0);
      double max_motion = 0.0;
      for (int t = 0; t < m; ++t) max_motion = std::max(max_motion, centre_motion(geos[used[t]], xd, yd, w0));
      auto evaluate = [&](const double* th, double (&hh)[3][3], double* gg) {
        for (auto& row : hh)
          for (double& v : row) v = 0.0;
        for (int i = 0; i < 3; ++i) gg[i] = 0.0;
        double score = 0.0;
        for (int t = 0; t < m; ++t) {
          const Res vr = evaluate_view(geos[used[t]], xd, yd, th, samples, n0, true);
          if (!vr.valid) return -std::numeric_limits<double>::infinity();
          score += vr.ncc;
          for (int a = 0; a < 3; ++a) {
            for (int b = 0; b < 3; ++b) hh[a][b] += vr.h[a][b];
            gg[a] += vr.g[a];
          }
        }
        return score / m;
      };
      double hh[3][3], gg[3];
      double best[3] = {theta0[0], theta0[1], theta0[2]};
      double best_score = evaluate(best, hh, gg);
      if (!std::isfinite(best_score)) continue;
      double scale = 1.0;
      for (int it = 0; it < o.iterations; ++it) {
        double delta[3];
        solve_damped(hh, gg, delta);
        if (!(std::isfinite(delta[0]) && std::isfinite(delta[1]) && std::isfinite(delta[2]))) break;
        const double motion = max_motion * (std::abs(delta[0]) + std::abs(delta[1]) + std::abs(delta[2]));
        if (motion > 1.0)
          for (double& d : delta) d /= motion;
        for (double& d : delta) d *= scale;
        if (max_motion * (std::abs(delta[0]) + std::abs(delta[1]) + std::abs(delta[2])) < 1e-3) break;
        double h2[3][3], g2[3];
        const double cand[3] = {best[0] + delta[0], best[1] + delta[1], best[2] + delta[2]};
        const double score = evaluate(cand, h2, g2);
        if (score > best_score) {
          std::copy(cand, cand + 3, best);
          best_score = score;
          std::copy(&h2[0][0], &h2[0][0] + 9, &hh[0][0]);
          std::copy(g2, g2 + 3, gg);
          scale = 1.0;
        } else {
          scale *= 0.25;
        }
      }
      if (best_score > s0 + o.min_gain && best[0] > 0.0 && max_motion * std::abs(best[0] - w0) <= o.max_shift_px) {
        depth[y * stride + x] = static_cast<float>(1.0 / best[0]);
        conf[y * stride + x] = static_cast<float>(best_score);
        ++c_refined;
      }
    }
  }
  st.input = c_input;
  st.refined = c_refined;
  st.unconfirmed = c_unconfirmed;
  st.kept = c_input - c_refined - c_unconfirmed;
}

// refinement.cpp:198-269
void make_image(const float* gray_in, int w, int h, double sigma, float* out) {
  std::vector<float> blurred;
  const float* gray = gray_in;
  if (sigma > 0.0) {
    const int r = std::max(1, static_cast<int>(std::ceil(3.0 * sigma)));
    std::vector<float> k(static_cast<size_t>(2 * r + 1));
    float ksum = 0.0F;
    for (int i = -r; i <= r; ++i) {
      k[i + r] = static_cast<float>(std::exp(-0.5 * i * i / (sigma * sigma)));
      ksum += k[i + r];
    }
    for (float& v : k) v /= ksum;
    std::vector<float> tmp(static_cast<size_t>(w) * h);
    blurred.assign(static_cast<size_t>(w) * h, 0.0F);
    for (int y = 0; y < h; ++y)
      for (int x = 0; x < w; ++x) {
        float acc = 0.0F;
        for (int i = -r; i <= r; ++i) acc += k[i + r] * gray_in[static_cast<size_t>(y) * w + std::clamp(x + i, 0, w - 1)];
        tmp[static_cast<size_t>(y) * w + x] = acc;
      }
    for (int y = 0; y < h; ++y)
      for (int i = -r; i <= r; ++i) {
        const float* row = &tmp[static_cast<size_t>(std::clamp(y + i, 0, h - 1)) * w];
        for (int x = 0; x < w; ++x) blurred[static_cast<size_t>(y) * w + x] += k[i + r] * row[x];
      }
    gray = blurred.data();
  }
  for (int y = 0; y < h; ++y) {
    const float* row = gray + static_cast<size_t>(y) * w;
    const float* up = gray + static_cast<size_t>(std::max(y - 1, 0)) * w;
    const float* down = gray + static_cast<size_t>(std::min(y + 1, h - 1)) * w;
    const float sy = (y > 0 && y < h - 1) ? 0.5F : 1.0F;
    float* o = out + static_cast<size_t>(y) * 3 * w;
    for (int x = 0; x < w; ++x) {
      const int xl = std::max(x - 1, 0), xr = std::min(x + 1, w - 1);
      o[3 * x] = row[x];
      o[3 * x + 1] = (row[xr] - row[xl]) / static_cast<float>(std::max(xr - xl, 1));
      o[3 * x + 2] = (down[x] - up[x]) * (h > 1 ? sy : 0.0F);
    }
  }
}

}  // namespace ref

template <class F>
int guarded(F&& f) {
  try {
    g_error.clear();
    f();
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 1;
  }
}

}  // namespace omvs

extern "C" {

const char* orc_mvs_last_error() { return omvs::g_error.c_str(); }

int orc_filter_depth_maps(r3dgpu_depth_map* maps, int count, const int32_t* off, const int32_t* idx,
                          const r3dgpu_consistency_options* o, r3dgpu_consistency_stats* st) {
  return omvs::guarded([&] { omvs::filter(maps, count, off, idx, *o, *st); });
}

int orc_prepare_depth_map(r3dgpu_depth_map* map, const r3dgpu_consistency_options* o, r3dgpu_consistency_stats* st) {
  return omvs::guarded([&] { omvs::prepare(*map, *o, *st); });
}

int orc_check_consistency(r3dgpu_depth_map* map, const r3dgpu_depth_map* nbs, int count,
                          const r3dgpu_consistency_options* o, r3dgpu_consistency_stats* st) {
  return omvs::guarded([&] {
    std::vector<const r3dgpu_depth_map*> p;
    for (int j = 0; j < count; ++j) p.push_back(&nbs[j]);
    omvs::check(*map, p.data(), count, *o, *st);
  });
}

int orc_erode_depth_edges(r3dgpu_depth_map* map, int radius, double discontinuity, int holes, uint64_t* removed) {
  return omvs::guarded([&] { *removed = omvs::erode_depth_edges(*map, radius, discontinuity, holes != 0); });
}

int orc_remove_weak_depths(r3dgpu_depth_map* map, const r3dgpu_consistency_options* o, uint64_t* removed) {
  return omvs::guarded([&] { *removed = omvs::remove_weak_depths(*map, *o); });
}

int orc_remove_depth_halos(r3dgpu_depth_map* map, int max_px, int colour_step, uint64_t* removed) {
  return omvs::guarded([&] { *removed = omvs::remove_depth_halos(*map, max_px, colour_step); });
}

// make_refinement_image of a contiguous gray image into out (3 floats per pixel).
int orc_make_refinement_image(const float* gray, int w, int h, double sigma, float* out) {
  return omvs::guarded([&] { omvs::ref::make_image(gray, w, h, sigma, out); });
}

// refine_depth_map on host maps (depth, confidence at `stride`) and host images.
int orc_refine_depth_map(float* depth, float* conf, int64_t stride, const r3dgpu_pinhole_camera* cam, int w, int h,
                         const r3dgpu_refinement_image* base, const r3dgpu_refinement_image* views, int num_views,
                         const r3dgpu_refinement_options* o, r3dgpu_refinement_stats* st) {
  return omvs::guarded([&] { omvs::ref::refine(depth, conf, stride, *cam, w, h, *base, views, num_views, *o, *st); });
}

int orc_remove_depth_speckles(r3dgpu_depth_map* map, int min_size, double step, uint64_t* removed) {
  return omvs::guarded([&] { *removed = omvs::remove_depth_speckles(*map, min_size, step); });
}

}  // extern "C"
