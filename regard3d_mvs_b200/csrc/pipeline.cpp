// A view's depth map on the device (r3dgpu_compute_depth_map): the loop of
// the reference's compute_depth_map (src/r3d/mvs/multi_stereo.cpp:243-304)
// from the rectified pairs' geometry on, composed of the library's own entry
// points so that every intermediate stays in device memory: rectification of
// the base and partner images of each pair (with validity masks), one batch
// match of all pairs, and the combination into the grid's depth map.
#include <string>
#include <vector>

#include "api_guard.h"
#include "common.cuh"
#include "matcher_internal.h"

namespace r3dgpu {
namespace {

constexpr int kMaxPairs = 16;  // multi_stereo.cpp:23

size_t up(size_t n) { return (n + 255) & ~static_cast<size_t>(255); }

void check_pairs(const r3dgpu_view_u16* base, const r3dgpu_camera* cam, const r3dgpu_depth_grid* grid,
                 const r3dgpu_view_pair* pairs, int count) {
  if (base == nullptr || cam == nullptr || grid == nullptr || (count > 0 && pairs == nullptr))
    fail(R3DGPU_EINVAL, "compute_depth_map: null argument");
  if (count < 0 || count > kMaxPairs)
    fail(R3DGPU_EINVAL, "compute_depth_map: at most 16 pairs per view (" + std::to_string(count) + " given)");
  for (int i = 0; i < count; ++i) {
    const r3dgpu_view_pair& p = pairs[i];
    if (p.left.width <= 0 || p.left.height <= 0 || p.right.width <= 0 || p.right.height != p.left.height)
      fail(R3DGPU_EINVAL, "compute_depth_map: pair " + std::to_string(i) +
                              " needs rectified images of positive size and equal height");
  }
}

}  // namespace
}  // namespace r3dgpu

using namespace r3dgpu;

extern "C" {

r3dgpu_status r3dgpu_compute_depth_map(const r3dgpu_view_u16* base, const r3dgpu_camera* base_camera,
                                       const r3dgpu_depth_grid* grid, const r3dgpu_view_pair* pairs, int32_t count,
                                       const r3dgpu_stereo_options* stereo,
                                       const r3dgpu_multi_stereo_options* multi, float* depth, float* confidence,
                                       uint16_t* pair_mask, int64_t stride, uint64_t* cells, void* stream) {
  return guard([&] {
    check_pairs(base, base_camera, grid, pairs, count);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // Rectified images, masks, disparity and confidence of every pair in one pool.
    size_t bytes = 0;
    for (int i = 0; i < count; ++i) {
      const size_t l = static_cast<size_t>(pairs[i].left.width) * pairs[i].left.height;
      const size_t r = static_cast<size_t>(pairs[i].right.width) * pairs[i].right.height;
      bytes += up(2 * l) + up(l) + up(2 * r) + up(r) + 2 * up(4 * l);
    }
    thread_local DeviceBuffer<unsigned char> pool;
    pool.reserve(bytes > 0 ? bytes : 1);
    unsigned char* p = pool.get();
    auto take = [&](size_t n) {
      unsigned char* at = p;
      p += up(n);
      return at;
    };
    r3dgpu_stereo_options opts{};
    if (stereo != nullptr) {
      opts = *stereo;
    } else {
      r3dgpu_default_options(&opts);
    }
    std::vector<r3dgpu_pair> batch(static_cast<size_t>(count));
    for (int i = 0; i < count; ++i) {
      const r3dgpu_view_pair& vp = pairs[i];
      const int lw = vp.left.width, lh = vp.left.height, rw = vp.right.width, rh = vp.right.height;
      auto* left = reinterpret_cast<uint16_t*>(take(2 * static_cast<size_t>(lw) * lh));
      auto* lmask = take(static_cast<size_t>(lw) * lh);
      auto* right = reinterpret_cast<uint16_t*>(take(2 * static_cast<size_t>(rw) * rh));
      auto* rmask = take(static_cast<size_t>(rw) * rh);
      auto* disp = reinterpret_cast<float*>(take(4 * static_cast<size_t>(lw) * lh));
      auto* conf = reinterpret_cast<float*>(take(4 * static_cast<size_t>(lw) * lh));
      r3dgpu_status st = r3dgpu_rectify_image_u16(base, base_camera, vp.base_from_rect, &vp.left, left, lw, lmask, lw, s);
      if (st != R3DGPU_OK) fail(st, r3dgpu_last_error());
      st = r3dgpu_rectify_image_u16(&vp.partner, &vp.partner_camera, vp.partner_from_rect, &vp.right, right, rw, rmask,
                                    rw, s);
      if (st != R3DGPU_OK) fail(st, r3dgpu_last_error());
      r3dgpu_pair& q = batch[i];
      q.left = r3dgpu_view_u16{left, lw, lh, lw};
      q.right = r3dgpu_view_u16{right, rw, rh, rw};
      q.left_valid = r3dgpu_view_u8{lmask, lw, lh, lw};
      q.right_valid = r3dgpu_view_u8{rmask, rw, rh, rw};
      q.disparity_min = vp.disparity_min;
      q.num_disparities = vp.num_disparities;
      q.options = opts;
      q.out = r3dgpu_disparity_map{disp, conf, lw, 0, 0, 0, 0, 0};
    }
    if (count > 0) {
      const r3dgpu_status st = r3dgpu_match_stereo_batch(batch.data(), count, s);
      if (st != R3DGPU_OK) fail(st, r3dgpu_last_error());
    }
    std::vector<r3dgpu_pair_geometry> geo(static_cast<size_t>(count));
    uint64_t total = 0;
    for (int i = 0; i < count; ++i) {
      geo[i] = pairs[i].geometry;
      geo[i].disparity = batch[i].out.disparity;
      geo[i].confidence = batch[i].out.confidence;
      geo[i].width = pairs[i].left.width;
      geo[i].height = pairs[i].left.height;
      geo[i].stride = pairs[i].left.width;
      total += batch[i].out.cells;
    }
    const r3dgpu_status st =
        r3dgpu_combine_pairs(grid, geo.data(), count, multi, depth, confidence, pair_mask, stride, s);
    if (st != R3DGPU_OK) fail(st, r3dgpu_last_error());
    if (cells != nullptr) *cells = total;
  });
}

}  // extern "C"
