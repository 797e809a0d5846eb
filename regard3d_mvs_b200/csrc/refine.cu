// Patch-based depth refinement (r3dgpu_refine_depth_map) and its input images
// (r3dgpu_make_refinement_image), the reference's src/r3d/mvs/refinement.cpp.
//
// One warp per depth-map pixel. The window samples (25 for the default 9 x 9
// window at step 2, 49 for a 7 x 7 window at step 1, at most 225) are spread
// over the lanes: each lane warps, samples and normalises its samples, and
// every sum of the NCC and of the Gauss-Newton terms is an xor-butterfly
// reduction. After a butterfly every lane holds the same bits (the partial
// sums meet in mirrored order, and IEEE addition commutes), so the per-pixel
// control flow — view selection, the damped Gauss-Newton loop with step
// shrinking, the acceptance test — is uniform over the warp and runs in every
// lane, with no shared memory and no barriers. The window terms compute in
// double precision as the reference does; with fp32 = 1 the Gauss-Newton
// terms (Jacobian, J^T J, J^T e: the bulk of the work) are float while the
// objective that decides which steps are taken (sampled values, window
// normalisation, NCC) and the 3 x 3 LDL^T solve stay double. Sums run in a different order than the
// reference's sequential loops, so results agree with a double-precision CPU
// restatement to rounding, not bit for bit.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "geom.cuh"
#include "kernels.h"
#include "api_guard.h"
#include "matcher_internal.h"

namespace r3dgpu {
namespace {

constexpr int kMaxSamples = 225;  // refinement.cpp:21
constexpr int kMaxViews = 8;      // refinement.cpp:22
constexpr double kDiscontinuity = 0.05;
enum : int { kInput, kRefined, kUnconfirmed, kCounters };

// Plane-induced warp into a view (refinement.cpp:24-30): h = m (qx, qy, 1) + b w(q).
struct ViewGeo {
  double m[9];  // K_j R_j R_0^T K_0^-1, row-major
  double b[3];  // K_j R_j (C_0 - C_j)
  const float4* data;  // (intensity, d/dx, d/dy, 0) per pixel, repacked from the 3-channel image
  int64_t stride;      // in pixels
  int width, height;
};

struct Params {
  int width, height;
  int radius, step, side, n;  // `side` samples per window row, n = side^2
  int iterations, num_views;
  double min_ncc, max_shift_px, min_gain, min_texture2n;
  int drop_unconfirmed;
};

template <class T>
R3D_DEVICE T shfl_xor_t(T v, int mask) {
  uint32_t w[sizeof(T) / 4];
  memcpy(w, &v, sizeof(T));
  for (int i = 0; i < static_cast<int>(sizeof(T) / 4); ++i) w[i] = r3dsimt::shfl_xor(w[i], mask);
  memcpy(&v, w, sizeof(T));
  return v;
}

// The value of lane `src` (every lane reads one source lane).
template <class T>
R3D_DEVICE T shfl_t(T v, int src) {
  uint32_t w[sizeof(T) / 4];
  memcpy(w, &v, sizeof(T));
  for (int i = 0; i < static_cast<int>(sizeof(T) / 4); ++i) w[i] = r3dsimt::shfl(w[i], src);
  memcpy(&v, w, sizeof(T));
  return v;
}

// Butterfly sums of K values over aligned groups of `width` lanes (masks
// below width), and from there across the groups (masks width .. 16). After
// each, all lanes of a group (or of the warp) hold the same bits: the partial
// sums meet in mirrored order and IEEE addition commutes.
template <class T, int K>
R3D_DEVICE void sums_below(T (&v)[K], int width) {
  for (int m = 1; m < width; m <<= 1) {
#pragma unroll
    for (int i = 0; i < K; ++i) v[i] += shfl_xor_t(v[i], m);
  }
}

template <class T, int K>
R3D_DEVICE void sums_from(T (&v)[K], int width) {
  for (int m = width; m < 32; m <<= 1) {
#pragma unroll
    for (int i = 0; i < K; ++i) v[i] += shfl_xor_t(v[i], m);
  }
}

template <class T>
R3D_DEVICE T warp_sum(T v) {
  T a[1] = {v};
  sums_below(a, 32);
  return a[0];
}

// Finite (neither infinite nor NaN): v - v is 0 exactly then, NaN otherwise.
R3D_DEVICE bool finite_d(double v) { return v - v == 0.0; }


// Smallest power of two >= m (m in 1..8): the number of lane groups.
R3D_DEVICE int groups_for(int m) { return m <= 1 ? 1 : (m <= 2 ? 2 : (m <= 4 ? 4 : 8)); }

// Per warp in shared memory: the normalised base window n0[s] and the
// window coordinates (offset / radius) of each window column.
constexpr int kWarpTableDoubles = kMaxSamples + 16;

// One view's terms at plane theta (refinement.cpp:46-152), computed by the
// `gsize` lanes of a group: lane `gl` of the group takes the window samples
// gl, gl + gsize, ... NCC of the warped window with the normalised base
// window and, with JAC, J^T J (xx xy xz yy yz zz) and J^T e of
// sum (n_q - n0_q)^2 in (w, a, b). `valid` is false if a sample leaves the
// image or the window has no texture. All lanes of the group return the same
// values; `active` false (a group without a view) returns zeros and valid.
//
// One pass: the lanes accumulate raw moments and one butterfly sums them.
// With v = (raw - mean) / |raw - mean| (sum v = 0, sum v^2 = 1),
// a = dv (1, sx, sy), d = a - mean(a) and p = sum v d, the reference's terms
// are ncc = sum raw n0 / |raw - mean| (n0 has zero mean),
// J^T J = (sum d d^T - p p^T) / |raw - mean|^2 and
// J^T e = (p ncc - sum a n0) / |raw - mean|. The objective moments are double
// (intensities shifted by `shift`, the base window's mean, to keep the
// variance well conditioned); the Jacobian moments are T.
template <class T, bool JAC>
R3D_DEVICE void evaluate_group(const ViewGeo& g, bool active, double x, double y, const double* theta,
                               const Params& p, const double* table, double shift, int gl, int gsize, bool& valid,
                               double& ncc_out, double* hh, double* gg) {
  double ob[3] = {0.0, 0.0, 0.0};
  T jm[15];
#pragma unroll
  for (int i = 0; i < 15; ++i) jm[i] = T(0);
  bool bad = false;
  if (active) {
    const T b0 = static_cast<T>(g.b[0]), b1 = static_cast<T>(g.b[1]), b2 = static_cast<T>(g.b[2]);
    const T m0 = static_cast<T>(g.m[0]), m1 = static_cast<T>(g.m[1]), m3 = static_cast<T>(g.m[3]),
            m4 = static_cast<T>(g.m[4]), m6 = static_cast<T>(g.m[6]), m7 = static_cast<T>(g.m[7]);
    const T max_x = static_cast<T>(g.width - 1), max_y = static_cast<T>(g.height - 1);
    const T th0 = static_cast<T>(theta[0]), th1 = static_cast<T>(theta[1]), th2 = static_cast<T>(theta[2]);
    const T hc0 = static_cast<T>(row3(g.m, 0, x, y, 1.0)), hc1 = static_cast<T>(row3(g.m, 1, x, y, 1.0)),
            hc2 = static_cast<T>(row3(g.m, 2, x, y, 1.0));
    // In float, pixel positions of a few thousand carry about 1e-4 px of
    // rounding. The float path therefore projects the window centre at the
    // current depth in double once and each sample as a small float offset:
    // (H + d).xy / (H + d).z = c + (d.xy - c d.z) / (H + d).z, c = H.xy / H.z.
    const bool rel = sizeof(T) == 4;
    double hz = 0.0;
    int ic0 = 0, ic1 = 0;
    T fc0 = 0, fc1 = 0, cf0 = 0, cf1 = 0, hzf = 0;
    if (rel) {
      const double H0 = row3(g.m, 0, x, y, 1.0) + g.b[0] * theta[0];
      const double H1 = row3(g.m, 1, x, y, 1.0) + g.b[1] * theta[0];
      hz = row3(g.m, 2, x, y, 1.0) + g.b[2] * theta[0];
      if (hz > 0.0) {
        const double c0 = H0 / hz, c1 = H1 / hz;
        const double f0 = floor(c0), f1 = floor(c1);
        if (fabs(f0) < 1e8 && fabs(f1) < 1e8) {
          ic0 = static_cast<int>(f0);
          ic1 = static_cast<int>(f1);
          fc0 = static_cast<T>(c0 - f0);
          fc1 = static_cast<T>(c1 - f1);
          cf0 = static_cast<T>(c0);
          cf1 = static_cast<T>(c1);
          hzf = static_cast<T>(hz);
        } else {
          hz = 0.0;
        }
      }
    }
    const bool offsets = rel && hz > 0.0;
    const double* n0s = table;
    const double* coord = table + kMaxSamples;  // offset / radius of window column c
    // Window column and row of sample s, advanced by gsize per step.
    int col = gl % p.side, row = gl / p.side;
    const int dcol = gsize % p.side, drow = gsize / p.side;
    for (int s = gl; s < p.n; s += gsize) {
      const T dx = static_cast<T>(col * p.step - p.radius), dy = static_cast<T>(row * p.step - p.radius);
      const T sx = static_cast<T>(coord[col]), sy = static_cast<T>(coord[row]);
      col += dcol;
      row += drow;
      if (col >= p.side) {
        col -= p.side;
        ++row;
      }
      T inv_z, px, py, fx, fy;
      int ix, iy;
      if (offsets) {
        const T ws = th1 * sx + th2 * sy;  // w(q) - w at the window centre
        const T d0 = (m0 * dx + m1 * dy) + b0 * ws;
        const T d1 = (m3 * dx + m4 * dy) + b1 * ws;
        const T d2 = (m6 * dx + m7 * dy) + b2 * ws;
        const T h2 = hzf + d2;
        if (!(h2 > T(0))) {
          bad = true;
          break;
        }
        inv_z = T(1) / h2;
        const T q0 = fc0 + (d0 - cf0 * d2) * inv_z, q1 = fc1 + (d1 - cf1 * d2) * inv_z;
        if (!(fabs(q0) < T(1e6) && fabs(q1) < T(1e6))) {
          bad = true;
          break;
        }
        const T fl0 = floor(q0), fl1 = floor(q1);
        ix = ic0 + static_cast<int>(fl0);
        iy = ic1 + static_cast<int>(fl1);
        fx = q0 - fl0;
        fy = q1 - fl1;
        px = static_cast<T>(ix) + fx;
        py = static_cast<T>(iy) + fy;
        // px in [0, width - 1) and py in [0, height - 1), as below.
        if (!(ix >= 0 && iy >= 0 && ix <= g.width - 2 && iy <= g.height - 2)) {
          bad = true;
          break;
        }
      } else {
        const T wq = (th0 + th1 * sx) + th2 * sy;
        const T h0 = ((hc0 + m0 * dx) + m1 * dy) + b0 * wq;
        const T h1 = ((hc1 + m3 * dx) + m4 * dy) + b1 * wq;
        const T h2 = ((hc2 + m6 * dx) + m7 * dy) + b2 * wq;
        if (!(h2 > T(0))) {
          bad = true;
          break;
        }
        inv_z = T(1) / h2;
        px = h0 * inv_z;
        py = h1 * inv_z;
        if (!(px >= T(0) && py >= T(0) && px < max_x && py < max_y)) {
          bad = true;
          break;
        }
        ix = static_cast<int>(px);
        iy = static_cast<int>(py);
        fx = px - static_cast<T>(ix);
        fy = py - static_cast<T>(iy);
      }
      const float4* r0 = g.data + static_cast<int64_t>(iy) * g.stride + ix;
      const float4 c00 = __ldg(r0), c01 = __ldg(r0 + 1), c10 = __ldg(r0 + g.stride), c11 = __ldg(r0 + g.stride + 1);
      const double fxd = fx, fyd = fy;
      const double raw = ((1.0 - fyd) * ((1.0 - fxd) * static_cast<double>(c00.x) + fxd * static_cast<double>(c01.x)) +
                          fyd * ((1.0 - fxd) * static_cast<double>(c10.x) + fxd * static_cast<double>(c11.x))) -
                         shift;
      const double n0 = n0s[s];
      ob[0] += raw;
      ob[1] += raw * raw;
      ob[2] += raw * n0;
      if (JAC) {
        const T ax = T(1) - fx, ay = T(1) - fy;
        const T gx = ay * (ax * c00.y + fx * c01.y) + fy * (ax * c10.y + fx * c11.y);
        const T gy = ay * (ax * c00.z + fx * c01.z) + fy * (ax * c10.z + fx * c11.z);
        const T dpx = (b0 - px * b2) * inv_z, dpy = (b1 - py * b2) * inv_z;
        const T dv = gx * dpx + gy * dpy;
        const T a0 = dv, a1 = dv * sx, a2 = dv * sy;
        const T rf = static_cast<T>(raw), nf = static_cast<T>(n0);
        jm[0] += a0;
        jm[1] += a1;
        jm[2] += a2;
        jm[3] += rf * a0;
        jm[4] += rf * a1;
        jm[5] += rf * a2;
        jm[6] += a0 * a0;
        jm[7] += a0 * a1;
        jm[8] += a0 * a2;
        jm[9] += a1 * a1;
        jm[10] += a1 * a2;
        jm[11] += a2 * a2;
        jm[12] += nf * a0;
        jm[13] += nf * a1;
        jm[14] += nf * a2;
      }
    }
  }
  // The group is invalid if any of its lanes left the image.
  const uint32_t lane = r3dsimt::lane_id();
  const uint32_t gmask = (gsize == 32 ? 0xFFFFFFFFu : ((1u << gsize) - 1u) << (lane & ~static_cast<uint32_t>(gsize - 1)));
  const bool group_bad = (r3dsimt::ballot(bad) & gmask) != 0;
  sums_below(ob, gsize);
  if (JAC) sums_below(jm, gsize);
  for (int i = 0; i < 6; ++i) hh[i] = 0.0;
  for (int i = 0; i < 3; ++i) gg[i] = 0.0;
  ncc_out = 0.0;
  valid = true;
  if (!active) return;
  const double nd = p.n;
  const double mean = ob[0] / nd;  // of the shifted values
  const double norm2 = ob[1] - ob[0] * mean;
  if (group_bad || !(norm2 > 1e-6 * nd)) {
    valid = false;
    return;
  }
  const double inv_norm = 1.0 / sqrt(norm2);
  const double ncc = ob[2] * inv_norm;
  ncc_out = ncc;
  if (!JAC) return;
  const T inv = static_cast<T>(inv_norm), n = static_cast<T>(p.n), meanf = static_cast<T>(mean);
  const T dm[3] = {jm[0] / n, jm[1] / n, jm[2] / n};
  const T pr[3] = {inv * (jm[3] - meanf * jm[0]), inv * (jm[4] - meanf * jm[1]), inv * (jm[5] - meanf * jm[2])};
  // sum d d^T = sum a a^T - dm (sum a)^T, then minus p p^T, times inv^2.
  const int ti[6] = {0, 0, 0, 1, 1, 2}, tj[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
  for (int e = 0; e < 6; ++e)
    hh[e] = static_cast<double>(inv * inv * ((jm[6 + e] - dm[ti[e]] * jm[tj[e]]) - pr[ti[e]] * pr[tj[e]]));
  const T nccf = static_cast<T>(ncc);
#pragma unroll
  for (int i = 0; i < 3; ++i) gg[i] = static_cast<double>(inv * (pr[i] * nccf - jm[12 + i]));
}

// refinement.cpp:155-165: pixels of motion in the view per unit of inverse depth.
R3D_DEVICE double centre_motion(const ViewGeo& g, double x, double y, double w) {
  const double h0 = row3(g.m, 0, x, y, 1.0) + g.b[0] * w;
  const double h1 = row3(g.m, 1, x, y, 1.0) + g.b[1] * w;
  const double h2 = row3(g.m, 2, x, y, 1.0) + g.b[2] * w;
  if (!(h2 > 0.0)) return 0.0;
  const double px = h0 / h2, py = h1 / h2;
  return hypot(g.b[0] - px * g.b[2], g.b[1] - py * g.b[2]) / h2;
}

// refinement.cpp:167-196: inverse-depth slope from the neighbours at +-1.
R3D_DEVICE double initial_slope(const float* depth, int w, int h, int x, int y, int ax, int ay) {
  const float z = depth[static_cast<int64_t>(y) * w + x];
  auto neighbour = [&](int k, double& wn) {
    const int nx = x + k * ax, ny = y + k * ay;
    if (nx < 0 || ny < 0 || nx >= w || ny >= h) return false;
    const float zn = depth[static_cast<int64_t>(ny) * w + nx];
    if (!(zn > 0.0F) || static_cast<double>(fabsf(zn - z)) > kDiscontinuity * static_cast<double>(fminf(z, zn)))
      return false;
    wn = 1.0 / zn;
    return true;
  };
  double wp = 0.0, wm = 0.0;
  const bool pl = neighbour(1, wp);
  const bool mi = neighbour(-1, wm);
  const double w0 = 1.0 / z;
  if (pl && mi) return 0.5 * (wp - wm);
  if (pl) return wp - w0;
  if (mi) return w0 - wm;
  return 0.0;
}

// delta = -(H (1 + 1e-6 on the diagonal) + 1e-12 I)^-1 g by LDL^T with
// symmetric diagonal pivoting (the largest remaining diagonal first).
R3D_DEVICE void solve_damped(const double* hh, const double* gg, double* delta) {
  double a[3][3] = {{hh[0], hh[1], hh[2]}, {hh[1], hh[3], hh[4]}, {hh[2], hh[4], hh[5]}};
  for (int i = 0; i < 3; ++i) a[i][i] = a[i][i] * (1.0 + 1e-6) + 1e-12;
  int perm[3] = {0, 1, 2};
  double l[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}, d[3];
  for (int k = 0; k < 3; ++k) {
    int piv = k;
    for (int i = k + 1; i < 3; ++i)
      if (fabs(a[i][i]) > fabs(a[piv][piv])) piv = i;
    if (piv != k) {
      for (int j = 0; j < 3; ++j) {
        const double t = a[k][j];
        a[k][j] = a[piv][j];
        a[piv][j] = t;
      }
      for (int i = 0; i < 3; ++i) {
        const double t = a[i][k];
        a[i][k] = a[i][piv];
        a[i][piv] = t;
      }
      for (int j = 0; j < k; ++j) {
        const double t = l[k][j];
        l[k][j] = l[piv][j];
        l[piv][j] = t;
      }
      const int t = perm[k];
      perm[k] = perm[piv];
      perm[piv] = t;
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

// One warp per depth-map pixel; per warp a table of kWarpTableDoubles
// doubles in dynamic shared memory.
template <class T>
R3D_GLOBAL void R3D_LAUNCH_BOUNDS_MIN(256, 2)
    refine_kernel(const float* R3D_RESTRICT input, float* depth, float* conf, int64_t stride,
                  const float* R3D_RESTRICT base, int64_t bstride, const ViewGeo* R3D_RESTRICT views, Params p,
                  unsigned long long* counters) {
  R3D_DYNAMIC_SMEM(smem);
  const int64_t pix = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (pix >= static_cast<int64_t>(p.width) * p.height) return;  // whole warp
  const int lane = static_cast<int>(r3dsimt::lane_id());
  const bool lead = lane == 0;
  double* table = reinterpret_cast<double*>(smem) + (threadIdx.x >> 5) * kWarpTableDoubles;
  const int y = static_cast<int>(pix / p.width), x = static_cast<int>(pix - static_cast<int64_t>(y) * p.width);
  const float z0 = input[pix];
  if (!(z0 > 0.0F)) return;
  const int64_t at = static_cast<int64_t>(y) * stride + x;
  if (lead) {
    atomicAdd(counters + kInput, 1ULL);
    conf[at] = 0.0F;
  }
  const int r = p.radius;
  if (p.num_views == 0 || x < r || y < r || x >= p.width - r || y >= p.height - r) return;

  // The normalised base window (sample s = lane + 32 k) into the table.
  double nb[kMaxSamples / 32 + 1];
  double sum = 0.0;
#pragma unroll
  for (int k = 0; k < kMaxSamples / 32 + 1; ++k) {
    const int s = lane + 32 * k;
    nb[k] = 0.0;
    if (s < p.n) {
      const int dx = (s % p.side) * p.step - r, dy = (s / p.side) * p.step - r;
      nb[k] = base[static_cast<int64_t>(y + dy) * bstride + 3 * (x + dx)];
      sum += nb[k];
    }
  }
  const double mean = warp_sum(sum) / p.n;
  double norm2 = 0.0;
#pragma unroll
  for (int k = 0; k < kMaxSamples / 32 + 1; ++k)
    if (lane + 32 * k < p.n) {
      nb[k] -= mean;
      norm2 += nb[k] * nb[k];
    }
  norm2 = warp_sum(norm2);
  if (norm2 < p.min_texture2n) return;
  const double inv_norm = 1.0 / sqrt(norm2);
#pragma unroll
  for (int k = 0; k < kMaxSamples / 32 + 1; ++k)
    if (lane + 32 * k < p.n) table[lane + 32 * k] = nb[k] * inv_norm;
  if (lane < p.side) table[kMaxSamples + lane] = static_cast<double>(lane * p.step - r) / r;
  r3dsimt::syncwarp();

  const double w0 = 1.0 / z0;
  const double theta0[3] = {w0, r * initial_slope(input, p.width, p.height, x, y, 1, 0),
                            r * initial_slope(input, p.width, p.height, x, y, 0, 1)};
  const double xd = x, yd = y;
  double hh_v[6], gg_v[3];

  // Local view selection at the initial plane: all views at once, one lane
  // group per view.
  int used[kMaxViews];
  int m = 0;
  double s0 = 0.0;
  {
    const int gsize = 32 / groups_for(p.num_views);
    const int t = lane / gsize;
    const bool active = t < p.num_views;
    bool valid;
    double ncc;
    evaluate_group<T, false>(views[active ? t : 0], active, xd, yd, theta0, p, table, mean, lane % gsize, gsize,
                             valid, ncc, hh_v, gg_v);
    const uint32_t ok = r3dsimt::ballot(active && valid && ncc >= p.min_ncc);
    for (int j = 0; j < p.num_views; ++j) {
      const double nj = shfl_t(ncc, j * gsize);  // group j's value
      if ((ok >> (j * gsize)) & 1u) {
        used[m++] = j;
        s0 += nj;
      }
    }
  }
  if (m == 0) {
    if (p.drop_unconfirmed && lead) {
      depth[at] = 0.0F;
      atomicAdd(counters + kUnconfirmed, 1ULL);
    }
    return;
  }
  s0 /= m;
  if (lead) conf[at] = static_cast<float>(s0);
  double max_motion = 0.0;
  for (int t = 0; t < m; ++t) max_motion = fmax(max_motion, centre_motion(views[used[t]], xd, yd, w0));

  // Mean NCC and Gauss-Newton terms over the used views (one lane group
  // each); -inf if a view drops out.
  const int gsize = 32 / groups_for(m);
  const int my_t = lane / gsize;
  const bool my_active = my_t < m;
  const ViewGeo& my_view = views[used[my_active ? my_t : 0]];
  auto evaluate = [&](const double* theta, double* hh, double* gg) {
    bool valid;
    double ncc;
    evaluate_group<T, true>(my_view, my_active, xd, yd, theta, p, table, mean, lane % gsize, gsize, valid, ncc,
                            hh_v, gg_v);
    if (r3dsimt::ballot(!valid) != 0) return -__builtin_huge_val();
    double tot[10] = {ncc, hh_v[0], hh_v[1], hh_v[2], hh_v[3], hh_v[4], hh_v[5], gg_v[0], gg_v[1], gg_v[2]};
    sums_from(tot, gsize);
    for (int i = 0; i < 6; ++i) hh[i] = tot[1 + i];
    for (int i = 0; i < 3; ++i) gg[i] = tot[7 + i];
    return tot[0] / m;
  };

  double hh[6], gg[3];
  double best[3] = {theta0[0], theta0[1], theta0[2]};
  double best_score = evaluate(best, hh, gg);
  if (!finite_d(best_score)) return;
  double scale = 1.0;
  for (int it = 0; it < p.iterations; ++it) {
    double delta[3];
    solve_damped(hh, gg, delta);
    if (!(finite_d(delta[0]) && finite_d(delta[1]) && finite_d(delta[2]))) break;
    // At most one pixel of motion per step at the window border.
    const double motion = max_motion * ((fabs(delta[0]) + fabs(delta[1])) + fabs(delta[2]));
    if (motion > 1.0)
      for (int i = 0; i < 3; ++i) delta[i] /= motion;
    for (int i = 0; i < 3; ++i) delta[i] *= scale;
    if (max_motion * ((fabs(delta[0]) + fabs(delta[1])) + fabs(delta[2])) < 1e-3) break;
    double h2[6], g2[3];
    const double cand[3] = {best[0] + delta[0], best[1] + delta[1], best[2] + delta[2]};
    const double score = evaluate(cand, h2, g2);
    if (score > best_score) {
      for (int i = 0; i < 3; ++i) best[i] = cand[i];
      best_score = score;
      for (int i = 0; i < 6; ++i) hh[i] = h2[i];
      for (int i = 0; i < 3; ++i) gg[i] = g2[i];
      scale = 1.0;
    } else {
      scale *= 0.25;
    }
  }
  if (best_score > s0 + p.min_gain && best[0] > 0.0 && max_motion * fabs(best[0] - w0) <= p.max_shift_px) {
    if (lead) {
      depth[at] = static_cast<float>(1.0 / best[0]);
      conf[at] = static_cast<float>(best_score);
      atomicAdd(counters + kRefined, 1ULL);
    }
  }
}

// ------------------------------------------------------------------ refinement images
// refinement.cpp:198-238: separable Gaussian, taps (normalised floats) from the host.
R3D_GLOBAL void blur_rows_kernel(const float* in, int64_t istride, int w, int h, const float* taps, int r,
                                 float* out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  const float* row = in + static_cast<int64_t>(y) * istride;
  float acc = 0.0F;
  for (int i = -r; i <= r; ++i) {
    const int xx = x + i < 0 ? 0 : (x + i > w - 1 ? w - 1 : x + i);
    acc = __fadd_rn(acc, __fmul_rn(taps[i + r], row[xx]));
  }
  out[static_cast<int64_t>(y) * w + x] = acc;
}

R3D_GLOBAL void blur_cols_kernel(const float* in, int w, int h, const float* taps, int r, float* out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  float acc = 0.0F;
  for (int i = -r; i <= r; ++i) {
    const int yy = y + i < 0 ? 0 : (y + i > h - 1 ? h - 1 : y + i);
    acc = __fadd_rn(acc, __fmul_rn(taps[i + r], in[static_cast<int64_t>(yy) * w + x]));
  }
  out[static_cast<int64_t>(y) * w + x] = acc;
}

// refinement.cpp:249-266: intensity and central-difference derivatives.
R3D_GLOBAL void gradient_kernel(const float* gray, int64_t gstride, int w, int h, float* out, int64_t ostride) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  const float* row = gray + static_cast<int64_t>(y) * gstride;
  const float* up = gray + static_cast<int64_t>(y > 0 ? y - 1 : 0) * gstride;
  const float* down = gray + static_cast<int64_t>(y < h - 1 ? y + 1 : h - 1) * gstride;
  const float sy = (y > 0 && y < h - 1) ? 0.5F : 1.0F;
  const int xl = x > 0 ? x - 1 : 0, xr = x < w - 1 ? x + 1 : w - 1;
  float* o = out + static_cast<int64_t>(y) * ostride + 3 * x;
  o[0] = row[x];
  o[1] = __fdiv_rn(__fsub_rn(row[xr], row[xl]), static_cast<float>(xr - xl > 1 ? xr - xl : 1));
  o[2] = __fmul_rn(__fsub_rn(down[x], up[x]), h > 1 ? sy : 0.0F);
}

// A view's 3-channel refinement image as one float4 per pixel (one 16-byte
// load per bilinear corner in the refinement kernel).
R3D_GLOBAL void repack_kernel(const float* in, int64_t istride, int w, int h, float4* out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  const float* p = in + static_cast<int64_t>(y) * istride + 3 * x;
  out[static_cast<int64_t>(y) * w + x] = make_float4(p[0], p[1], p[2], 0.0F);
}

// ------------------------------------------------------------------ host side
struct Scratch {
  DeviceBuffer<unsigned long long> counters;
  DeviceBuffer<float> input, blur_tmp, blur_out, taps;
  DeviceBuffer<ViewGeo> views;
  DeviceBuffer<float4> packed;  // the views' repacked images
};

Scratch& scratch() {
  thread_local Scratch s;
  s.counters.reserve(kCounters);
  s.views.reserve(kMaxViews);
  return s;
}

// Row-major 3x3 products in the reference's left-to-right order.
void mat3(const double* a, const double* b, double* out) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) out[3 * i + j] = (a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j]) + a[3 * i + 2] * b[6 + j];
}

// refinement.cpp:297-309.
ViewGeo view_geometry(const r3dgpu_pinhole_camera& c0, const r3dgpu_refinement_image& v) {
  const r3dgpu_pinhole_camera& cj = v.camera;
  const double kj[9] = {cj.intrinsics.fx, 0.0, cj.intrinsics.cx, 0.0, cj.intrinsics.fy, cj.intrinsics.cy,
                        0.0, 0.0, 1.0};
  double r0t[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r0t[3 * i + j] = c0.rotation[3 * j + i];
  double kr[9], krr[9];
  ViewGeo g{};
  mat3(kj, cj.rotation, kr);
  mat3(kr, r0t, krr);
  mat3(krr, c0.k_inv, g.m);
  const double dc[3] = {c0.center[0] - cj.center[0], c0.center[1] - cj.center[1], c0.center[2] - cj.center[2]};
  for (int i = 0; i < 3; ++i) g.b[i] = (kr[3 * i] * dc[0] + kr[3 * i + 1] * dc[1]) + kr[3 * i + 2] * dc[2];
  g.data = nullptr;  // set to the repacked image by the caller
  g.stride = cj.intrinsics.width;
  g.width = cj.intrinsics.width;
  g.height = cj.intrinsics.height;
  return g;
}

r3dgpu_refinement_options options_or_default(const r3dgpu_refinement_options* o) {
  r3dgpu_refinement_options out{};
  if (o != nullptr) return *o;
  r3dgpu_default_refinement_options(&out);
  return out;
}

template <class T>
void launch_refine(const float* input, float* depth, float* conf, int64_t stride, const float* base,
                   int64_t bstride, const ViewGeo* views, const Params& p, unsigned long long* counters,
                   cudaStream_t s) {
  const int64_t warps = static_cast<int64_t>(p.width) * p.height;
  const size_t smem = sizeof(double) * kWarpTableDoubles * 8;
  auto kernel = refine_kernel<T>;
  R3D_LAUNCH(kernel, static_cast<unsigned>(ceil_div64(warps, 8)), 256, smem, s, input, depth, conf, stride, base,
             bstride, views, p, counters);
  launched(sizeof(T) == 8 ? "refine_kernel<f64>" : "refine_kernel<f32>");
}

void refine(float* depth, float* conf, int64_t stride, const r3dgpu_pinhole_camera& cam, int w, int h,
            const r3dgpu_refinement_image& base, const r3dgpu_refinement_image* views, int num_views,
            const r3dgpu_refinement_options& o, r3dgpu_refinement_stats* stats, cudaStream_t s) {
  if (o.radius < 1 || o.step < 1 || o.iterations < 0)
    fail(R3DGPU_EINVAL, "refinement: invalid window (radius " + std::to_string(o.radius) + ", step " +
                            std::to_string(o.step) + ") or iterations " + std::to_string(o.iterations));
  if (base.camera.intrinsics.width != w || base.camera.intrinsics.height != h || base.data == nullptr ||
      base.stride < 3LL * w)
    fail(R3DGPU_EINVAL, "refinement: base image does not match the depth map");
  if (w < 0 || h < 0 || (w > 0 && h > 0 && (depth == nullptr || conf == nullptr || stride < w)))
    fail(R3DGPU_EINVAL, "refinement: bad depth map");
  const int side = 2 * o.radius / o.step + 1;
  const int n = side * side;
  if (n > kMaxSamples)
    fail(R3DGPU_EINVAL, "refinement: window of " + std::to_string(n) + " samples (at most 225)");
  if (num_views < 0 || (num_views > 0 && views == nullptr)) fail(R3DGPU_EINVAL, "refinement: null views");
  const int nv = std::min(num_views, std::min(o.max_views, kMaxViews));
  Scratch& sc = scratch();
  ViewGeo geo[kMaxViews];
  for (int j = 0; j < nv; ++j) {
    const r3dgpu_refinement_image& v = views[j];
    if (v.data == nullptr || v.camera.intrinsics.width < 2 || v.camera.intrinsics.height < 2 ||
        v.stride < 3LL * v.camera.intrinsics.width)
      fail(R3DGPU_EINVAL, "refinement: view " + std::to_string(j) + " has no image");
    geo[j] = view_geometry(cam, v);
  }
  R3D_CUDA(cudaMemsetAsync(sc.counters.get(), 0, sizeof(unsigned long long) * kCounters, s));
  if (w > 0 && h > 0) {
    // The views' images as one float4 per pixel.
    size_t total = 0;
    for (int j = 0; j < nv; ++j)
      total += static_cast<size_t>(views[j].camera.intrinsics.width) * views[j].camera.intrinsics.height;
    sc.packed.reserve(total > 0 ? total : 1);
    size_t off = 0;
    for (int j = 0; j < nv; ++j) {
      const int vw = views[j].camera.intrinsics.width, vh = views[j].camera.intrinsics.height;
      float4* dst = sc.packed.get() + off;
      const dim3 b(32, 8), g(static_cast<unsigned>(ceil_div(vw, 32)), static_cast<unsigned>(ceil_div(vh, 8)));
      R3D_LAUNCH(repack_kernel, g, b, 0, s, views[j].data, views[j].stride, vw, vh, dst);
      launched("repack_kernel");
      geo[j].data = dst;
      off += static_cast<size_t>(vw) * vh;
    }
    if (nv > 0)
      R3D_CUDA(cudaMemcpyAsync(sc.views.get(), geo, sizeof(ViewGeo) * nv, cudaMemcpyHostToDevice, s));
    sc.input.reserve(static_cast<size_t>(w) * h);
    R3D_CUDA(cudaMemcpy2DAsync(sc.input.get(), sizeof(float) * w, depth, sizeof(float) * stride, sizeof(float) * w,
                               h, cudaMemcpyDeviceToDevice, s));
    Params p{w, h, o.radius, o.step, side, n, o.iterations, nv, o.min_ncc, o.max_shift_px, o.min_gain,
             o.min_texture * o.min_texture * n, o.drop_unconfirmed};
    if (o.fp32)
      launch_refine<float>(sc.input.get(), depth, conf, stride, base.data, base.stride, sc.views.get(), p,
                           sc.counters.get(), s);
    else
      launch_refine<double>(sc.input.get(), depth, conf, stride, base.data, base.stride, sc.views.get(), p,
                            sc.counters.get(), s);
  }
  unsigned long long c[kCounters];
  R3D_CUDA(cudaMemcpyAsync(c, sc.counters.get(), sizeof(c), cudaMemcpyDeviceToHost, s));
  R3D_CUDA(cudaStreamSynchronize(s));
  if (stats != nullptr) *stats = r3dgpu_refinement_stats{c[kInput], c[kRefined], c[kInput] - c[kRefined] - c[kUnconfirmed],
                                                         c[kUnconfirmed]};
}

void make_image(const float* gray, int64_t gstride, int w, int h, double sigma, float* out, int64_t ostride,
                cudaStream_t s) {
  if (w < 0 || h < 0 || (w > 0 && h > 0 && (gray == nullptr || out == nullptr || gstride < w || ostride < 3LL * w)))
    fail(R3DGPU_EINVAL, "refinement image: bad size, stride or pointer");
  if (w == 0 || h == 0) return;
  const dim3 b(32, 8), g(static_cast<unsigned>(ceil_div(w, 32)), static_cast<unsigned>(ceil_div(h, 8)));
  const float* src = gray;
  int64_t sstride = gstride;
  if (sigma > 0.0) {
    // refinement.cpp:200-210: taps up to 3 sigma, normalised in float.
    const int r = std::max(1, static_cast<int>(std::ceil(3.0 * sigma)));
    std::vector<float> k(static_cast<size_t>(2 * r + 1));
    float ksum = 0.0F;
    for (int i = -r; i <= r; ++i) {
      k[i + r] = static_cast<float>(std::exp(-0.5 * i * i / (sigma * sigma)));
      ksum += k[i + r];
    }
    for (float& v : k) v /= ksum;
    Scratch& sc = scratch();
    sc.taps.reserve(k.size());
    sc.blur_tmp.reserve(static_cast<size_t>(w) * h);
    sc.blur_out.reserve(static_cast<size_t>(w) * h);
    float* taps = sc.taps.get();
    float* tmp = sc.blur_tmp.get();
    float* blurred = sc.blur_out.get();
    R3D_CUDA(cudaMemcpyAsync(taps, k.data(), sizeof(float) * k.size(), cudaMemcpyHostToDevice, s));
    R3D_LAUNCH(blur_rows_kernel, g, b, 0, s, gray, gstride, w, h, taps, r, tmp);
    launched("blur_rows_kernel");
    R3D_LAUNCH(blur_cols_kernel, g, b, 0, s, tmp, w, h, taps, r, blurred);
    launched("blur_cols_kernel");
    src = blurred;
    sstride = w;
  }
  R3D_LAUNCH(gradient_kernel, g, b, 0, s, src, sstride, w, h, out, ostride);
  launched("gradient_kernel");
}

}  // namespace
}  // namespace r3dgpu

using namespace r3dgpu;

extern "C" {

void r3dgpu_default_refinement_options(r3dgpu_refinement_options* out) {
  if (out == nullptr) return;
  *out = r3dgpu_refinement_options{4, 2, 6, 4, 0.3, 2.0, 0.02, 1.0, 0.0, 1, 0};
}

r3dgpu_status r3dgpu_make_refinement_image(const float* gray, int64_t gray_stride, int32_t width, int32_t height,
                                           double blur_sigma, float* out, int64_t out_stride, void* stream) {
  return guard([&] {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    make_image(gray, gray_stride, width, height, blur_sigma, out, out_stride, s);
    R3D_CUDA(cudaStreamSynchronize(s));
  });
}

r3dgpu_status r3dgpu_refine_depth_map(float* depth, float* confidence, int64_t stride,
                                      const r3dgpu_pinhole_camera* camera, int32_t width, int32_t height,
                                      const r3dgpu_refinement_image* base, const r3dgpu_refinement_image* views,
                                      int32_t num_views, const r3dgpu_refinement_options* options,
                                      r3dgpu_refinement_stats* stats, void* stream) {
  return guard([&] {
    if (camera == nullptr || base == nullptr) fail(R3DGPU_EINVAL, "refinement: null argument");
    refine(depth, confidence, stride, *camera, width, height, *base, views, num_views, options_or_default(options),
           stats, static_cast<cudaStream_t>(stream));
  });
}

r3dgpu_status r3dgpu_refine_depth_map_host(float* depth, float* confidence, int64_t stride,
                                           const r3dgpu_pinhole_camera* camera, int32_t width, int32_t height,
                                           const r3dgpu_refinement_image* base,
                                           const r3dgpu_refinement_image* views, int32_t num_views,
                                           const r3dgpu_refinement_options* options, r3dgpu_refinement_stats* stats) {
  return guard([&] {
    if (camera == nullptr || base == nullptr) fail(R3DGPU_EINVAL, "refinement: null argument");
    if (num_views < 0 || (num_views > 0 && views == nullptr)) fail(R3DGPU_EINVAL, "refinement: null views");
    if (width < 0 || height < 0 || stride < width || (width > 0 && height > 0 && (depth == nullptr || confidence == nullptr)))
      fail(R3DGPU_EINVAL, "refinement: bad depth map");
    const r3dgpu_refinement_options o = options_or_default(options);
    const int nv = std::min(num_views, std::min(o.max_views, kMaxViews));
    cudaStream_t s = nullptr;
    auto up = [](size_t n) { return (n + 255) & ~static_cast<size_t>(255); };
    auto image_bytes = [](const r3dgpu_refinement_image& v) {
      return sizeof(float) * 3 * static_cast<size_t>(v.camera.intrinsics.width) * v.camera.intrinsics.height;
    };
    const size_t px = static_cast<size_t>(width) * height;
    size_t bytes = 2 * up(4 * px) + up(image_bytes(*base));
    for (int j = 0; j < nv; ++j) bytes += up(image_bytes(views[j]));
    thread_local DeviceBuffer<unsigned char> io;
    io.reserve(bytes > 0 ? bytes : 1);
    unsigned char* p = io.get();
    auto take = [&](size_t n) {
      unsigned char* at = p;
      p += up(n);
      return at;
    };
    auto upload = [&](const r3dgpu_refinement_image& v) {
      r3dgpu_refinement_image d = v;
      const int vw = v.camera.intrinsics.width, vh = v.camera.intrinsics.height;
      float* dst = reinterpret_cast<float*>(take(image_bytes(v)));
      if (vw > 0 && vh > 0) {
        if (v.data == nullptr || v.stride < 3LL * vw) fail(R3DGPU_EINVAL, "refinement: image without data");
        R3D_CUDA(cudaMemcpy2DAsync(dst, sizeof(float) * 3 * vw, v.data, sizeof(float) * v.stride,
                                   sizeof(float) * 3 * vw, vh, cudaMemcpyHostToDevice, s));
      }
      d.data = dst;
      d.stride = 3LL * vw;
      return d;
    };
    float* dd = reinterpret_cast<float*>(take(4 * px));
    float* dc = reinterpret_cast<float*>(take(4 * px));
    if (px > 0) {
      R3D_CUDA(cudaMemcpy2DAsync(dd, 4 * static_cast<size_t>(width), depth, 4 * stride, 4 * static_cast<size_t>(width),
                                 height, cudaMemcpyHostToDevice, s));
      R3D_CUDA(cudaMemcpy2DAsync(dc, 4 * static_cast<size_t>(width), confidence, 4 * stride,
                                 4 * static_cast<size_t>(width), height, cudaMemcpyHostToDevice, s));
    }
    const r3dgpu_refinement_image dbase = upload(*base);
    std::vector<r3dgpu_refinement_image> dviews;
    for (int j = 0; j < nv; ++j) dviews.push_back(upload(views[j]));
    refine(dd, dc, width, *camera, width, height, dbase, dviews.data(), nv, o, stats, s);
    if (px > 0) {
      R3D_CUDA(cudaMemcpy2DAsync(depth, 4 * stride, dd, 4 * static_cast<size_t>(width), 4 * static_cast<size_t>(width),
                                 height, cudaMemcpyDeviceToHost, s));
      R3D_CUDA(cudaMemcpy2DAsync(confidence, 4 * stride, dc, 4 * static_cast<size_t>(width),
                                 4 * static_cast<size_t>(width), height, cudaMemcpyDeviceToHost, s));
    }
    R3D_CUDA(cudaStreamSynchronize(s));
  });
}

}  // extern "C"
