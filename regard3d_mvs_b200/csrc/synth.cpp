// Seeded synthetic rectified pairs (include/r3dgpu_synth.h), host code.
//
// Left: uniform noise in [0, 255] blurred with a Gaussian and renormalised to
// [0, 255]. Disparity: `planes` random planes d = c + a (x - sx) + b (y - sy),
// each pixel taking the plane of its nearest seed (sx, sy), clipped to
// [5, nd - 8]. Right: the texture sampled bilinearly at x + d(x, y) plus
// Gaussian noise. The texture is generated wider than the left image, so that
// right pixels whose match lies beyond the left border still see texture.
// Optional textureless patches are painted into the texture (both images see
// them); optional occlusions replace runs of right pixels with fresh noise.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "../../include/r3dgpu_synth.h"

namespace {

// Portable uniform / normal on std::mt19937 (same values on every platform).
class Rng {
 public:
  explicit Rng(uint32_t seed) : g_(seed) {}
  double uniform(double lo, double hi) { return lo + (hi - lo) * ((g_() + 0.5) / 4294967296.0); }
  double normal(double mean, double sigma) {
    const double u1 = uniform(0.0, 1.0), u2 = uniform(0.0, 1.0);
    return mean + sigma * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
  uint32_t raw() { return g_(); }

 private:
  std::mt19937 g_;
};

uint32_t mix(uint32_t a, uint32_t b) {
  uint64_t x = (static_cast<uint64_t>(a) << 32) ^ (b * 0x9E3779B97F4A7C15ull);
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdull;
  x ^= x >> 33;
  return static_cast<uint32_t>(x);
}

template <class F>
void parallel_rows(int n, F&& f) {
  const int threads = std::max(1u, std::thread::hardware_concurrency());
  std::vector<std::thread> pool;
  const int chunk = (n + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    const int a = t * chunk, b = std::min(n, a + chunk);
    if (a >= b) break;
    pool.emplace_back([&, a, b] {
      for (int y = a; y < b; ++y) f(y);
    });
  }
  for (auto& th : pool) th.join();
}

}  // namespace

extern "C" r3dgpu_status r3dgpu_synth_pair(const r3dgpu_synth_params* p, uint8_t* left, uint8_t* right, float* gt) {
  if (!p || !left || !right || p->width <= 0 || p->height <= 0 || p->num_disparities < 16 || p->planes <= 0)
    return R3DGPU_EINVAL;
  const int W = p->width, H = p->height, nd = p->num_disparities;
  const double dmax = nd - 8, dmin = 5.0;
  const int TW = W + nd + 8;  // texture width
  try {
    // 1. Noise, per row with its own stream.
    std::vector<float> tex(static_cast<size_t>(TW) * H), tmp(tex.size());
    parallel_rows(H, [&](int y) {
      Rng r(mix(p->seed, static_cast<uint32_t>(y)));
      for (int x = 0; x < TW; ++x) tex[static_cast<size_t>(y) * TW + x] = static_cast<float>(r.uniform(0.0, 255.0));
    });
    // 2. Separable Gaussian blur, clamped borders.
    const double s = p->blur_sigma > 0 ? p->blur_sigma : 1.0;
    const int rad = static_cast<int>(std::ceil(3.0 * s));
    std::vector<float> k(2 * rad + 1);
    double ks = 0;
    for (int i = -rad; i <= rad; ++i) ks += (k[i + rad] = static_cast<float>(std::exp(-0.5 * i * i / (s * s))));
    for (auto& v : k) v = static_cast<float>(v / ks);
    parallel_rows(H, [&](int y) {
      const float* in = tex.data() + static_cast<size_t>(y) * TW;
      float* out = tmp.data() + static_cast<size_t>(y) * TW;
      for (int x = 0; x < TW; ++x) {
        float a = 0;
        for (int i = -rad; i <= rad; ++i) a += k[i + rad] * in[std::clamp(x + i, 0, TW - 1)];
        out[x] = a;
      }
    });
    parallel_rows(H, [&](int y) {
      float* out = tex.data() + static_cast<size_t>(y) * TW;
      for (int x = 0; x < TW; ++x) {
        float a = 0;
        for (int i = -rad; i <= rad; ++i) a += k[i + rad] * tmp[static_cast<size_t>(std::clamp(y + i, 0, H - 1)) * TW + x];
        out[x] = a;
      }
    });
    float lo = tex[0], hi = tex[0];
    for (float v : tex) {
      lo = std::min(lo, v);
      hi = std::max(hi, v);
    }
    const float scale = hi > lo ? 255.0F / (hi - lo) : 0.0F;
    for (float& v : tex) v = (v - lo) * scale;
    Rng g(p->seed ^ 0xA5A5A5A5u);
    // 3. Textureless patches (constant intensity), painted into the texture.
    if (p->textureless_fraction > 0) {
      const double target = p->textureless_fraction * static_cast<double>(W) * H;
      std::vector<uint8_t> covered(static_cast<size_t>(W) * H, 0);
      double area = 0;
      int guard = 0;
      while (area < target && guard++ < 100000) {
        const int pw = 8 + static_cast<int>(g.uniform(0, 0.12) * W), ph = 8 + static_cast<int>(g.uniform(0, 0.12) * H);
        const int x0 = static_cast<int>(g.uniform(0, std::max(1, W - pw))), y0 = static_cast<int>(g.uniform(0, std::max(1, H - ph)));
        const float v = static_cast<float>(g.uniform(20, 235));
        for (int y = y0; y < std::min(H, y0 + ph); ++y)
          for (int x = x0; x < std::min(TW, x0 + pw); ++x) {
            tex[static_cast<size_t>(y) * TW + x] = v;
            if (x < W && !covered[static_cast<size_t>(y) * W + x]) {
              covered[static_cast<size_t>(y) * W + x] = 1;
              area += 1;
            }
          }
      }
    }
    // 4. Piecewise planar disparity.
    const int np = p->planes;
    std::vector<double> sx(np), sy(np), pc(np), pa(np), pb(np);
    const double slope = (dmax - dmin) / (2.0 * std::max(W, H));
    for (int i = 0; i < np; ++i) {
      sx[i] = g.uniform(0, W);
      sy[i] = g.uniform(0, H);
      pc[i] = g.uniform(dmin, dmax);
      pa[i] = g.uniform(-slope, slope);
      pb[i] = g.uniform(-slope, slope);
    }
    std::vector<float> disp(static_cast<size_t>(W) * H);
    parallel_rows(H, [&](int y) {
      for (int x = 0; x < W; ++x) {
        int best = 0;
        double bd = 1e300;
        for (int i = 0; i < np; ++i) {
          const double dx = x - sx[i], dy = y - sy[i], dd = dx * dx + dy * dy;
          if (dd < bd) {
            bd = dd;
            best = i;
          }
        }
        const double d = pc[best] + pa[best] * (x - sx[best]) + pb[best] * (y - sy[best]);
        disp[static_cast<size_t>(y) * W + x] = static_cast<float>(std::clamp(d, dmin, dmax));
      }
    });
    // 5. Left image, right image (bilinear inverse warp + noise).
    parallel_rows(H, [&](int y) {
      Rng r(mix(p->seed ^ 0x5EEDu, static_cast<uint32_t>(y)));
      const float* t = tex.data() + static_cast<size_t>(y) * TW;
      for (int x = 0; x < W; ++x) {
        left[static_cast<size_t>(y) * W + x] = static_cast<uint8_t>(std::lround(std::clamp(t[x], 0.0F, 255.0F)));
        const double xs = x + disp[static_cast<size_t>(y) * W + x];
        const int x0 = std::clamp(static_cast<int>(std::floor(xs)), 0, TW - 2);
        const double f = std::clamp(xs - x0, 0.0, 1.0);
        const double v = t[x0] * (1.0 - f) + t[x0 + 1] * f + r.normal(0.0, p->noise_sigma);
        right[static_cast<size_t>(y) * W + x] = static_cast<uint8_t>(std::lround(std::clamp(v, 0.0, 255.0)));
      }
    });
    // 6. Occlusions: runs of right pixels replaced by fresh noise.
    if (p->occluded_fraction > 0) {
      const double target = p->occluded_fraction * static_cast<double>(W) * H;
      double done = 0;
      while (done < target) {
        const int y = static_cast<int>(g.raw() % static_cast<uint32_t>(H));
        const int len = 4 + static_cast<int>(g.raw() % 29u);
        const int x0 = static_cast<int>(g.raw() % static_cast<uint32_t>(W));
        for (int x = x0; x < std::min(W, x0 + len); ++x) {
          right[static_cast<size_t>(y) * W + x] = static_cast<uint8_t>(g.raw() & 255u);
          done += 1;
        }
      }
    }
    if (gt) std::copy(disp.begin(), disp.end(), gt);
  } catch (...) {
    return R3DGPU_ENOMEM;
  }
  return R3DGPU_OK;
}
