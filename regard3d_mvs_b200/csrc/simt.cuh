// Portability layer of the r3dgpu kernels.
//
// Under nvcc (the product build) every macro below is the plain CUDA
// construct. Under a host compiler with R3DGPU_SIMT_EMULATION defined (the
// test-only emulator build, tests/simt/) the same kernel sources run on the
// CPU: each CUDA thread is a fiber, barriers and warp shuffles switch fibers,
// cp.async copies are deferred until their wait, and buffers are plain heap
// allocations so that AddressSanitizer checks every index. The emulator is
// never part of the product library.
#pragma once

#include <cstdint>
#include <cstring>

#ifndef R3DGPU_SIMT_EMULATION
// ============================================================ CUDA build
#include <cuda_runtime.h>

#define R3D_GLOBAL __global__
#define R3D_DEVICE __device__ __forceinline__
#define R3D_DEVICE_NOINLINE __device__
#define R3D_HOSTDEV __host__ __device__ __forceinline__
#define R3D_RESTRICT __restrict__
#define R3D_LAUNCH_BOUNDS(n) __launch_bounds__(n)
#define R3D_LAUNCH_BOUNDS_MIN(n, blocks) __launch_bounds__(n, blocks)
#define R3D_DYNAMIC_SMEM(name) extern __shared__ __align__(16) unsigned char name[]
#define R3D_LAUNCH(kernel, grid, block, smem, stream, ...) kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__)

namespace r3dsimt {

R3D_DEVICE bool finitef(float v) { return isfinite(v); }
R3D_DEVICE int imin(int a, int b) { return min(a, b); }
R3D_DEVICE int imax(int a, int b) { return max(a, b); }
R3D_DEVICE uint32_t umin(uint32_t a, uint32_t b) { return min(a, b); }
R3D_DEVICE uint32_t umax(uint32_t a, uint32_t b) { return max(a, b); }
R3D_DEVICE uint32_t lane_id() { return threadIdx.x & 31u; }
R3D_DEVICE uint32_t shfl(uint32_t v, int src) { return __shfl_sync(0xffffffffu, v, src); }
R3D_DEVICE uint32_t shfl_xor(uint32_t v, int m) { return __shfl_xor_sync(0xffffffffu, v, m); }
R3D_DEVICE uint32_t ballot(bool p) { return __ballot_sync(0xffffffffu, p); }
R3D_DEVICE uint32_t match_any(uint32_t v) { return __match_any_sync(0xffffffffu, v); }  // lanes holding v
R3D_DEVICE int ffs(uint32_t v) { return __ffs(static_cast<int>(v)); }  // 1 + index of the lowest set bit, 0 if none
R3D_DEVICE void syncwarp() { __syncwarp(); }
R3D_DEVICE void syncthreads() { __syncthreads(); }
R3D_DEVICE void fence() { __threadfence(); }
// Per-halfword unsigned minimum and sum modulo 2^16: the u16x2 instructions
// of sm_90+, written as PTX so that no emulated SIMD-video form is chosen.
R3D_DEVICE uint32_t vmin2(uint32_t a, uint32_t b) {
  uint32_t r;
  asm("min.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
R3D_DEVICE uint32_t vadd2(uint32_t a, uint32_t b) {
  uint32_t r;
  asm("add.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
// Per-halfword a == b ? 0xFFFF : 0.
R3D_DEVICE uint32_t vcmpeq2(uint32_t a, uint32_t b) { return __vcmpeq2(a, b); }
// Per-halfword min(a, b, c) and min(a + b, c) (DPX instructions on sm_90+).
R3D_DEVICE uint32_t vmin3(uint32_t a, uint32_t b, uint32_t c) { return vmin2(vmin2(a, b), c); }
R3D_DEVICE uint32_t vaddmin2(uint32_t a, uint32_t b, uint32_t c) { return vmin2(vadd2(a, b), c); }
R3D_DEVICE uint32_t perm(uint32_t a, uint32_t b, uint32_t s) { return __byte_perm(a, b, s); }
// Low word of (hi:lo) >> s, s in [0, 31].
R3D_DEVICE uint32_t funnel_r(uint32_t lo, uint32_t hi, uint32_t s) { return __funnelshift_r(lo, hi, s); }
R3D_DEVICE int popc(uint32_t v) { return __popc(v); }
R3D_DEVICE int popc64(uint64_t v) { return __popcll(v); }
// Streaming (evict-first) 16-byte load and store.
R3D_DEVICE uint4 ld_stream(const uint4* p) { return __ldcs(p); }
R3D_DEVICE void st_stream(uint4* p, uint4 v) { __stcs(p, v); }
R3D_DEVICE void st_stream8(uint2* p, uint2 v) { __stcs(p, v); }

// 16-byte asynchronous global -> shared copy (L2 only). Both addresses must
// be 16-byte aligned.
R3D_DEVICE void cp_async16(void* smem_dst, const void* gmem_src) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
// 8-byte asynchronous global -> shared copy (through L1). Both addresses
// must be 8-byte aligned.
R3D_DEVICE void cp_async8(void* smem_dst, const void* gmem_src) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
// 4-byte asynchronous global -> shared copy (through L1). Both addresses
// must be 4-byte aligned.
R3D_DEVICE void cp_async4(void* smem_dst, const void* gmem_src) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
// Hint: bring the line holding p into L2 (no register, no wait).
R3D_DEVICE void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p)); }
R3D_DEVICE void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
R3D_DEVICE void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

}  // namespace r3dsimt

#else
// ============================================================ emulator build
#include <algorithm>
#include <cmath>
#include <functional>
#include <vector>

#define R3D_GLOBAL
#define R3D_DEVICE inline
#define R3D_DEVICE_NOINLINE inline
#define R3D_HOSTDEV inline
#define R3D_RESTRICT
#define R3D_LAUNCH_BOUNDS(n)
#define R3D_LAUNCH_BOUNDS_MIN(n, blocks)
#define R3D_DYNAMIC_SMEM(name) unsigned char* name = ::r3dsimt::dynamic_smem()
#define R3D_LAUNCH(kernel, grid, block, smem, stream, ...) \
  ::r3dsimt::launch((grid), (block), (smem), [=]() { kernel(__VA_ARGS__); })

struct dim3 {
  unsigned x = 1, y = 1, z = 1;
  dim3(unsigned a = 1, unsigned b = 1, unsigned c = 1) : x(a), y(b), z(c) {}
};
struct uint3 {
  unsigned x, y, z;
};
struct alignas(16) int4 {
  int x, y, z, w;
};
struct alignas(8) int2 {
  int x, y;
};
struct alignas(16) uint4 {
  unsigned x, y, z, w;
};
struct alignas(8) uint2 {
  unsigned x, y;
};
struct alignas(16) float4 {
  float x, y, z, w;
};
inline int4 make_int4(int x, int y, int z, int w) { return int4{x, y, z, w}; }
inline int2 make_int2(int x, int y) { return int2{x, y}; }
inline uint4 make_uint4(unsigned x, unsigned y, unsigned z, unsigned w) { return uint4{x, y, z, w}; }
inline uint2 make_uint2(unsigned x, unsigned y) { return uint2{x, y}; }
inline float4 make_float4(float x, float y, float z, float w) { return float4{x, y, z, w}; }

namespace r3dsimt {

// Per-fiber CUDA coordinates (set by the scheduler).
struct Coords {
  uint3 tid, bid;
  dim3 bdim, gdim;
};
const Coords& coords();
unsigned char* dynamic_smem();
void launch(dim3 grid, dim3 block, size_t smem, const std::function<void()>& body);

inline bool finitef(float v) { return std::isfinite(v); }
inline int imin(int a, int b) { return a < b ? a : b; }
inline int imax(int a, int b) { return a > b ? a : b; }
inline uint32_t umin(uint32_t a, uint32_t b) { return a < b ? a : b; }
inline uint32_t umax(uint32_t a, uint32_t b) { return a > b ? a : b; }
uint32_t lane_id();
uint32_t shfl(uint32_t v, int src);
uint32_t shfl_xor(uint32_t v, int m);
uint32_t ballot(bool p);
uint32_t match_any(uint32_t v);
inline int ffs(uint32_t v) { return __builtin_ffs(static_cast<int>(v)); }
void syncwarp();
void syncthreads();
inline void fence() {}
inline uint32_t vmin2(uint32_t a, uint32_t b) {
  const uint32_t lo = std::min(a & 0xFFFFu, b & 0xFFFFu), hi = std::min(a >> 16, b >> 16);
  return lo | (hi << 16);
}
inline uint32_t vmin3(uint32_t a, uint32_t b, uint32_t c) { return vmin2(vmin2(a, b), c); }
inline uint32_t vcmpeq2(uint32_t a, uint32_t b) {
  return (((a ^ b) & 0xFFFFu) == 0 ? 0xFFFFu : 0u) | (((a ^ b) >> 16) == 0 ? 0xFFFF0000u : 0u);
}
inline uint32_t vaddmin2(uint32_t a, uint32_t b, uint32_t c) {
  const uint32_t lo = std::min((a + b) & 0xFFFFu, c & 0xFFFFu);
  const uint32_t hi = std::min(((a >> 16) + (b >> 16)) & 0xFFFFu, c >> 16);
  return lo | (hi << 16);
}
inline uint32_t vadd2(uint32_t a, uint32_t b) {
  return ((a + b) & 0xFFFFu) | (((a >> 16) + (b >> 16)) << 16);
}
inline uint32_t perm(uint32_t a, uint32_t b, uint32_t s) {
  const uint64_t v = (static_cast<uint64_t>(b) << 32) | a;
  uint32_t r = 0;
  for (int i = 0; i < 4; ++i) {
    const unsigned sel = (s >> (4 * i)) & 7u;
    r |= static_cast<uint32_t>((v >> (8 * sel)) & 0xFFu) << (8 * i);
  }
  return r;
}
inline uint32_t funnel_r(uint32_t lo, uint32_t hi, uint32_t s) {
  return static_cast<uint32_t>(((static_cast<uint64_t>(hi) << 32) | lo) >> (s & 31u));
}
inline int popc(uint32_t v) { return __builtin_popcount(v); }
inline int popc64(uint64_t v) { return __builtin_popcountll(v); }
inline uint4 ld_stream(const uint4* p) { return *p; }
inline void st_stream(uint4* p, uint4 v) { *p = v; }
inline void st_stream8(uint2* p, uint2 v) { *p = v; }
void cp_async16(void* smem_dst, const void* gmem_src);
void cp_async8(void* smem_dst, const void* gmem_src);
void cp_async4(void* smem_dst, const void* gmem_src);
void cp_async_commit();
void cp_async_wait_n(int n);
inline void prefetch_l2(const void*) {}
template <int N>
inline void cp_async_wait() {
  cp_async_wait_n(N);
}

}  // namespace r3dsimt

#define threadIdx (::r3dsimt::coords().tid)
#define blockIdx (::r3dsimt::coords().bid)
#define blockDim (::r3dsimt::coords().bdim)
#define gridDim (::r3dsimt::coords().gdim)

// Device intrinsics used by the kernels, with their CUDA semantics.
inline float __fadd_rn(float a, float b) { return a + b; }
inline float __fsub_rn(float a, float b) { return a - b; }
inline float __fmul_rn(float a, float b) { return a * b; }
inline float __fdiv_rn(float a, float b) { return a / b; }
inline int atomicAdd(int* p, int v) { const int o = *p; *p = o + v; return o; }
inline unsigned atomicAdd(unsigned* p, unsigned v) { const unsigned o = *p; *p = o + v; return o; }
inline unsigned long long atomicAdd(unsigned long long* p, unsigned long long v) {
  const unsigned long long o = *p;
  *p = o + v;
  return o;
}
inline unsigned atomicMin(unsigned* p, unsigned v) { const unsigned o = *p; if (v < o) *p = v; return o; }
inline int atomicMax(int* p, int v) { const int o = *p; if (v > o) *p = v; return o; }
inline int atomicCAS(int* p, int cmp, int v) { const int o = *p; if (o == cmp) *p = v; return o; }
template <class T>
inline T __ldcg(const T* p) { return *p; }
template <class T>
inline T __ldg(const T* p) { return *p; }
#endif
