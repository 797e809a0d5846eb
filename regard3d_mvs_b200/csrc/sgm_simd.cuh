// Packed-u16 helpers shared by the SGM tile kernels that hold K label pairs
// per lane and G lanes per tile row (sgm_full.cu, sgm_ranged.cu).
#pragma once

#include "common.cuh"

namespace r3dgpu {
namespace sgm_simd {

constexpr uint32_t kSent2 = 0x7FFF7FFFu;  // two labels outside any range

// Packed minimum over the G lanes of a row group (G a power of two <= 32).
template <int G>
R3D_DEVICE uint32_t group_vmin2(uint32_t v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v = r3dsimt::vmin2(v, r3dsimt::shfl_xor(v, o));
  return v;
}
template <int G>
R3D_DEVICE uint32_t group_umin(uint32_t v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v = r3dsimt::umin(v, r3dsimt::shfl_xor(v, o));
  return v;
}

// Words base[-1 .. K] of a vector (base 16-byte aligned when K % 4 == 0,
// 8-byte aligned when K is even).
template <int K>
R3D_DEVICE void load_words(const uint32_t* base, uint32_t (&w)[K + 2]) {
  w[0] = base[-1];
  if constexpr (K % 4 == 0) {
#pragma unroll
    for (int i = 0; i < K; i += 4) {
      const uint4 v = *reinterpret_cast<const uint4*>(base + i);
      w[1 + i] = v.x;
      w[2 + i] = v.y;
      w[3 + i] = v.z;
      w[4 + i] = v.w;
    }
  } else if constexpr (K % 2 == 0) {
#pragma unroll
    for (int i = 0; i < K; i += 2) {
      const uint2 v = *reinterpret_cast<const uint2*>(base + i);
      w[1 + i] = v.x;
      w[2 + i] = v.y;
    }
  } else {
#pragma unroll
    for (int i = 0; i < K; ++i) w[1 + i] = base[i];
  }
  w[K + 1] = base[K];
}

template <int K>
R3D_DEVICE void store_words(uint32_t* base, const uint32_t (&o)[K]) {
  if constexpr (K % 4 == 0) {
#pragma unroll
    for (int i = 0; i < K; i += 4) *reinterpret_cast<uint4*>(base + i) = make_uint4(o[i], o[i + 1], o[i + 2], o[i + 3]);
  } else if constexpr (K % 2 == 0) {
#pragma unroll
    for (int i = 0; i < K; i += 2) *reinterpret_cast<uint2*>(base + i) = make_uint2(o[i], o[i + 1]);
  } else {
#pragma unroll
    for (int i = 0; i < K; ++i) base[i] = o[i];
  }
}

// Subpixel offset of the winner (stereo_matcher.cpp:426-436), clamped to +-0.5.
R3D_DEVICE float subpixel_delta(int method, float sm, float s0, float sp) {
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

}  // namespace sgm_simd
}  // namespace r3dgpu
