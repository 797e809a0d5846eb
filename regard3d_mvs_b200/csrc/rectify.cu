// Resampling of an image into a rotated pinhole camera with the same centre
// (r3dgpu_rectify_image_*), the reference's r3d::rectify_image
// (src/r3d/rectify/rectification.cpp:287-350) for single-channel u16 and f32
// images.
//
// One thread per target pixel: the target ray K^-1 (x, y, 1) is rotated into
// the source camera (double precision), projected through the source camera's
// distortion model (src/r3d/core/camera_model.cpp:67-100, 148-151) and, when
// it lands inside the source image, sampled with Catmull-Rom bicubic weights
// (src/r3d/core/sampling.hpp:15-55) from a pyramid level of the source when
// the target has less than 1/1.5 of its resolution. Every floating-point
// operation follows the reference's order without contraction (the library
// is built with --fmad=false), so that outputs are bit-identical to a CPU
// restatement wherever the math library agrees (all models but fisheye,
// whose atan may differ by an ulp from the host's).
//
// The kernel is a gather: each target pixel reads a 4x4 source window, which
// neighbouring threads of a warp share through L1/L2; the source of a typical
// photo (tens of MB) stays L2-resident, so DRAM traffic is about one read of
// the source plus the target writes.
#include <cmath>
#include <string>

#include "common.cuh"
#include "kernels.h"
#include "api_guard.h"
#include "matcher_internal.h"

namespace r3dgpu {
namespace {

enum : int { kPinhole = 0, kRadialK1 = 1, kRadialK3 = 2, kBrownT2 = 3, kFisheye = 4 };

// CameraIntrinsics of the camera that is sampled (a pyramid level of it).
struct Cam {
  int model;
  int width, height;
  double fx, fy, cx, cy;
  double p[5];
};

// Target intrinsics and the rotation source_from_target (row-major).
struct Target {
  int width, height;
  double fx, fy, cx, cy;
  double m[9];
};

// camera_model.cpp:67-100 (distortion in normalised coordinates).
R3D_DEVICE void distort(const Cam& c, double ux, double uy, double& dx, double& dy) {
  const double r2 = ux * ux + uy * uy;
  switch (c.model) {
    case kRadialK1: {
      const double s = 1.0 + c.p[0] * r2;
      dx = ux * s;
      dy = uy * s;
      return;
    }
    case kRadialK3: {
      const double s = 1.0 + r2 * (c.p[0] + r2 * (c.p[1] + r2 * c.p[2]));
      dx = ux * s;
      dy = uy * s;
      return;
    }
    case kBrownT2: {
      const double radial = r2 * (c.p[0] + r2 * (c.p[1] + r2 * c.p[2]));
      const double t1 = c.p[3], t2 = c.p[4];
      const double tx = t2 * (r2 + 2.0 * ux * ux) + 2.0 * t1 * ux * uy;
      const double ty = t1 * (r2 + 2.0 * uy * uy) + 2.0 * t2 * ux * uy;
      dx = ux + ux * radial + tx;
      dy = uy + uy * radial + ty;
      return;
    }
    case kFisheye: {
      const double r = sqrt(r2);
      if (r <= 1e-8) break;
      const double theta = atan(r);
      const double t2 = theta * theta;
      const double theta_d = theta * (1.0 + t2 * (c.p[0] + t2 * (c.p[1] + t2 * (c.p[2] + t2 * c.p[3]))));
      const double s = theta_d / r;
      dx = ux * s;
      dy = uy * s;
      return;
    }
    default:
      break;
  }
  dx = ux;
  dy = uy;
}

// sampling.hpp:21-26: Catmull-Rom weights of the taps -1, 0, 1, 2.
R3D_DEVICE void cubic_weights(float t, float w[4]) {
  const float t2 = __fmul_rn(t, t);
  const float t3 = __fmul_rn(t2, t);
  w[0] = __fsub_rn(__fadd_rn(__fmul_rn(-0.5F, t3), t2), __fmul_rn(0.5F, t));
  w[1] = __fadd_rn(__fsub_rn(__fmul_rn(1.5F, t3), __fmul_rn(2.5F, t2)), 1.0F);
  w[2] = __fadd_rn(__fadd_rn(__fmul_rn(-1.5F, t3), __fmul_rn(2.0F, t2)), __fmul_rn(0.5F, t));
  w[3] = __fsub_rn(__fmul_rn(0.5F, t3), __fmul_rn(0.5F, t2));
}

R3D_DEVICE int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// rectification.cpp:140-148.
R3D_DEVICE uint16_t to_pixel(float v, uint16_t*) {
  float r = roundf(v);
  r = r < 0.0F ? 0.0F : (65535.0F < r ? 65535.0F : r);
  return static_cast<uint16_t>(r);
}
R3D_DEVICE float to_pixel(float v, float*) { return v; }

template <class T>
R3D_GLOBAL void rectify_kernel(const T* R3D_RESTRICT src, int64_t sstride, Cam cam, Target k, T* R3D_RESTRICT out,
                               int64_t ostride, uint8_t* R3D_RESTRICT valid, int64_t vstride) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= k.width || y >= k.height) return;
  const double ry = (y - k.cy) / k.fy;
  const double rx = (x - k.cx) / k.fx;
  const double vx = (k.m[0] * rx + k.m[1] * ry) + k.m[2] * 1.0;
  const double vy = (k.m[3] * rx + k.m[4] * ry) + k.m[5] * 1.0;
  const double vz = (k.m[6] * rx + k.m[7] * ry) + k.m[8] * 1.0;
  bool inside = vz > 1e-9;
  double sx = 0.0, sy = 0.0;
  if (inside) {
    double dx, dy;
    distort(cam, vx / vz, vy / vz, dx, dy);
    sx = cam.fx * dx + cam.cx;
    sy = cam.fy * dy + cam.cy;
    inside = sx >= -0.5 && sy >= -0.5 && sx <= cam.width - 0.5 && sy <= cam.height - 0.5;
  }
  T value = T{};
  if (inside) {
    const double fx = floor(sx), fy = floor(sy);
    float wx[4], wy[4];
    cubic_weights(static_cast<float>(sx - fx), wx);
    cubic_weights(static_cast<float>(sy - fy), wy);
    const int x0 = static_cast<int>(fx) - 1, y0 = static_cast<int>(fy) - 1;
    int xs[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) xs[i] = clampi(x0 + i, 0, cam.width - 1);
    float acc_y = 0.0F;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const T* row = src + static_cast<int64_t>(clampi(y0 + j, 0, cam.height - 1)) * sstride;
      float acc = 0.0F;
#pragma unroll
      for (int i = 0; i < 4; ++i) acc = __fadd_rn(acc, __fmul_rn(wx[i], static_cast<float>(row[xs[i]])));
      acc_y = __fadd_rn(acc_y, __fmul_rn(wy[j], acc));
    }
    value = to_pixel(acc_y, static_cast<T*>(nullptr));
  }
  out[static_cast<int64_t>(y) * ostride + x] = value;
  if (valid != nullptr) valid[static_cast<int64_t>(y) * vstride + x] = inside ? 255 : 0;
}

// pyramid.cpp:33-83 for float images: the horizontal 1-4-6-4-1 sums of the
// five source rows, then the vertical sum of those, times 1/256.
R3D_DEVICE float pyr_row_f32(const float* row, int w, int sx) {
  const float a = row[sx - 2 > 0 ? sx - 2 : 0], b = row[sx + 2 < w - 1 ? sx + 2 : w - 1];
  const float c = row[sx - 1 > 0 ? sx - 1 : 0], d = row[sx + 1 < w - 1 ? sx + 1 : w - 1];
  return __fadd_rn(__fadd_rn(__fadd_rn(a, b), __fmul_rn(4.0F, __fadd_rn(c, d))), __fmul_rn(6.0F, row[sx]));
}

R3D_GLOBAL void pyramid_f32_kernel(const float* R3D_RESTRICT in, int64_t istride, int w, int h,
                                   float* R3D_RESTRICT out, int64_t ostride, int dw, int dh) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= dw || y >= dh) return;
  const int sx = 2 * x, sy = 2 * y;
  auto row = [&](int r) { return pyr_row_f32(in + static_cast<int64_t>(r) * istride, w, sx); };
  const float a = row(sy - 2 > 0 ? sy - 2 : 0), b = row(sy + 2 < h - 1 ? sy + 2 : h - 1);
  const float c = row(sy - 1 > 0 ? sy - 1 : 0), d = row(sy + 1 < h - 1 ? sy + 1 : h - 1);
  const float s = __fadd_rn(__fadd_rn(__fadd_rn(a, b), __fmul_rn(4.0F, __fadd_rn(c, d))), __fmul_rn(6.0F, row(sy)));
  out[static_cast<int64_t>(y) * ostride + x] = __fmul_rn(s, 1.0F / 256.0F);
}

void launch_pyramid(const float* in, int64_t istride, int w, int h, float* out, int64_t ostride, cudaStream_t s) {
  const int dw = (w + 1) / 2, dh = (h + 1) / 2;
  const dim3 b(32, 8);
  R3D_LAUNCH(pyramid_f32_kernel, dim3(ceil_div(dw, 32), ceil_div(dh, 8)), b, 0, s, in, istride, w, h, out, ostride,
             dw, dh);
  launched("pyramid_f32_kernel");
}

void launch_pyramid(const uint16_t* in, int64_t istride, int w, int h, uint16_t* out, int64_t ostride,
                    cudaStream_t s) {
  launch_pyramid_u16(in, istride, w, h, out, ostride, s);
}

// rectification.cpp:297-303: the pyramid level sampled for anti-aliasing.
int source_level(const r3dgpu_camera& cam, const r3dgpu_pinhole& k) {
  int level = 0;
  while (cam.fx / k.fx > 1.5 * std::ldexp(1.0, level) && (cam.width >> (level + 1)) >= 16 &&
         (cam.height >> (level + 1)) >= 16)
    ++level;
  return level;
}

// rectification.cpp:152-164.
Cam level_camera(const r3dgpu_camera& c, int level) {
  const double s = std::ldexp(1.0, -level);
  Cam out{c.model, c.width, c.height, c.fx * s, c.fy * s, c.cx * s, c.cy * s, {}};
  for (int i = 0; i < 5; ++i) out.p[i] = c.params[i];
  for (int i = 0; i < level; ++i) {
    out.width = (out.width + 1) / 2;
    out.height = (out.height + 1) / 2;
  }
  return out;
}

template <class T>
struct LevelPool {
  DeviceBuffer<T> a, b;
};

template <class T>
LevelPool<T>& level_pool() {
  thread_local LevelPool<T> pool;
  return pool;
}

// Rectifies the device image `src` (cam.width x cam.height, row stride
// sstride) into `out`; pyramid levels come from a per-thread pool.
template <class T>
void rectify(const T* src, int64_t sstride, const r3dgpu_camera& cam, const double* m, const r3dgpu_pinhole& k,
             T* out, int64_t ostride, uint8_t* valid, int64_t vstride, cudaStream_t s) {
  if (k.width == 0 || k.height == 0) return;
  const int level = source_level(cam, k);
  const T* level_src = src;
  int64_t level_stride = sstride;
  if (level > 0) {
    LevelPool<T>& pool = level_pool<T>();
    const size_t n1 = static_cast<size_t>((cam.width + 1) / 2) * ((cam.height + 1) / 2);
    pool.a.reserve(n1);
    if (level > 1) pool.b.reserve(static_cast<size_t>((cam.width + 3) / 4) * ((cam.height + 3) / 4));
    int w = cam.width, h = cam.height;
    T* bufs[2] = {pool.a.get(), pool.b.get()};
    for (int l = 0; l < level; ++l) {
      T* dst = bufs[l & 1];
      const int dw = (w + 1) / 2;
      launch_pyramid(level_src, level_stride, w, h, dst, dw, s);
      level_src = dst;
      level_stride = dw;
      w = dw;
      h = (h + 1) / 2;
    }
  }
  Target t{k.width, k.height, k.fx, k.fy, k.cx, k.cy, {}};
  for (int i = 0; i < 9; ++i) t.m[i] = m[i];
  const dim3 b(32, 8);
  R3D_LAUNCH(rectify_kernel<T>, dim3(ceil_div(k.width, 32), ceil_div(k.height, 8)), b, 0, s, level_src,
             level_stride, level_camera(cam, level), t, out, ostride, valid, vstride);
  launched(sizeof(T) == 2 ? "rectify_kernel<u16>" : "rectify_kernel<f32>");
}

void check(const void* src, int src_width, int src_height, int64_t src_stride, const r3dgpu_camera* cam,
           const double* m, const r3dgpu_pinhole* k, const void* out, int64_t ostride, const uint8_t* valid,
           int64_t vstride) {
  if (cam == nullptr || m == nullptr || k == nullptr) fail(R3DGPU_EINVAL, "rectify_image: null argument");
  if (cam->model < kPinhole || cam->model > kFisheye)
    fail(R3DGPU_EINVAL, "rectify_image: unknown camera model " + std::to_string(cam->model));
  if (src_width != cam->width || src_height != cam->height)
    fail(R3DGPU_EINVAL, "rectify_image: image is " + std::to_string(src_width) + "x" + std::to_string(src_height) +
                            ", camera is " + std::to_string(cam->width) + "x" + std::to_string(cam->height));
  if (src == nullptr || cam->width <= 0 || cam->height <= 0) fail(R3DGPU_EINVAL, "rectify_image: empty source image");
  if (src_stride < cam->width) fail(R3DGPU_EINVAL, "rectify_image: source stride below its width");
  if (k->width < 0 || k->height < 0) fail(R3DGPU_EINVAL, "rectify_image: negative target size");
  if (!(k->fx != 0.0 && k->fy != 0.0)) fail(R3DGPU_EINVAL, "rectify_image: target focal length is zero");
  const bool has_pixels = k->width > 0 && k->height > 0;
  if (has_pixels && (out == nullptr || ostride < k->width))
    fail(R3DGPU_EINVAL, "rectify_image: no output image or its stride is below the target width");
  if (has_pixels && valid != nullptr && vstride < k->width)
    fail(R3DGPU_EINVAL, "rectify_image: validity stride below the target width");
}

// Host images: copy in, rectify, copy out (one per-thread staging buffer).
template <class T>
void rectify_host(const T* src, int64_t sstride, const r3dgpu_camera& cam, const double* m, const r3dgpu_pinhole& k,
                  T* out, int64_t ostride, uint8_t* valid, int64_t vstride) {
  if (k.width == 0 || k.height == 0) return;
  cudaStream_t s = nullptr;
  const size_t src_bytes = sizeof(T) * static_cast<size_t>(cam.width) * cam.height;
  const size_t out_bytes = sizeof(T) * static_cast<size_t>(k.width) * k.height;
  const size_t valid_bytes = valid != nullptr ? static_cast<size_t>(k.width) * k.height : 0;
  auto round_up = [](size_t n) { return (n + 255) & ~static_cast<size_t>(255); };
  thread_local DeviceBuffer<unsigned char> io;
  io.reserve(round_up(src_bytes) + round_up(out_bytes) + valid_bytes);
  T* dsrc = reinterpret_cast<T*>(io.get());
  T* dout = reinterpret_cast<T*>(io.get() + round_up(src_bytes));
  uint8_t* dvalid = valid != nullptr ? io.get() + round_up(src_bytes) + round_up(out_bytes) : nullptr;
  R3D_CUDA(cudaMemcpy2DAsync(dsrc, sizeof(T) * cam.width, src, sizeof(T) * sstride, sizeof(T) * cam.width,
                             cam.height, cudaMemcpyHostToDevice, s));
  rectify(dsrc, cam.width, cam, m, k, dout, k.width, dvalid, k.width, s);
  R3D_CUDA(cudaMemcpy2DAsync(out, sizeof(T) * ostride, dout, sizeof(T) * k.width, sizeof(T) * k.width, k.height,
                             cudaMemcpyDeviceToHost, s));
  if (valid != nullptr)
    R3D_CUDA(cudaMemcpy2DAsync(valid, vstride, dvalid, k.width, k.width, k.height, cudaMemcpyDeviceToHost, s));
  R3D_CUDA(cudaStreamSynchronize(s));
}

}  // namespace
}  // namespace r3dgpu

using namespace r3dgpu;

extern "C" {

r3dgpu_status r3dgpu_rectify_image_u16(const r3dgpu_view_u16* src, const r3dgpu_camera* cam,
                                       const double* source_from_target, const r3dgpu_pinhole* target, uint16_t* out,
                                       int64_t out_stride, uint8_t* valid, int64_t valid_stride, void* stream) {
  return guard([&] {
    if (src == nullptr) fail(R3DGPU_EINVAL, "rectify_image: null argument");
    check(src->data, src->width, src->height, src->stride, cam, source_from_target, target, out, out_stride, valid,
          valid_stride);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    rectify(src->data, src->stride, *cam, source_from_target, *target, out, out_stride, valid, valid_stride, s);
    R3D_CUDA(cudaStreamSynchronize(s));
  });
}

r3dgpu_status r3dgpu_rectify_image_f32(const float* src, int64_t src_stride, const r3dgpu_camera* cam,
                                       const double* source_from_target, const r3dgpu_pinhole* target, float* out,
                                       int64_t out_stride, uint8_t* valid, int64_t valid_stride, void* stream) {
  return guard([&] {
    if (cam == nullptr) fail(R3DGPU_EINVAL, "rectify_image: null argument");
    check(src, cam->width, cam->height, src_stride, cam, source_from_target, target, out, out_stride, valid,
          valid_stride);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    rectify(src, src_stride, *cam, source_from_target, *target, out, out_stride, valid, valid_stride, s);
    R3D_CUDA(cudaStreamSynchronize(s));
  });
}

r3dgpu_status r3dgpu_rectify_image_u16_host(const r3dgpu_view_u16* src, const r3dgpu_camera* cam,
                                            const double* source_from_target, const r3dgpu_pinhole* target,
                                            uint16_t* out, int64_t out_stride, uint8_t* valid, int64_t valid_stride) {
  return guard([&] {
    if (src == nullptr) fail(R3DGPU_EINVAL, "rectify_image: null argument");
    check(src->data, src->width, src->height, src->stride, cam, source_from_target, target, out, out_stride, valid,
          valid_stride);
    rectify_host(src->data, src->stride, *cam, source_from_target, *target, out, out_stride, valid, valid_stride);
  });
}

r3dgpu_status r3dgpu_rectify_image_f32_host(const float* src, int64_t src_stride, const r3dgpu_camera* cam,
                                            const double* source_from_target, const r3dgpu_pinhole* target,
                                            float* out, int64_t out_stride, uint8_t* valid, int64_t valid_stride) {
  return guard([&] {
    if (cam == nullptr) fail(R3DGPU_EINVAL, "rectify_image: null argument");
    check(src, cam->width, cam->height, src_stride, cam, source_from_target, target, out, out_stride, valid,
          valid_stride);
    rectify_host(src, src_stride, *cam, source_from_target, *target, out, out_stride, valid, valid_stride);
  });
}

}  // extern "C"
