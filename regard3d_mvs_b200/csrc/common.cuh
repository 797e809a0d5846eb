// Shared helpers of the r3dgpu CUDA library: error propagation, launch
// counting, device buffers and small device utilities.
#pragma once

#include "runtime.h"

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>

#include "../../include/r3dgpu.h"

namespace r3dgpu {

// Library error carrying an r3dgpu_status.
struct Error : std::runtime_error {
  r3dgpu_status status;
  Error(r3dgpu_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

[[noreturn]] inline void fail(r3dgpu_status s, const std::string& m) { throw Error(s, m); }

inline void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    if (e == cudaErrorMemoryAllocation) fail(R3DGPU_ENOMEM, std::string(what) + ": " + cudaGetErrorString(e));
    fail(R3DGPU_EDEVICE, std::string(what) + ": " + cudaGetErrorString(e));
  }
}

#define R3D_CUDA(call) ::r3dgpu::cuda_check((call), #call)

// Number of kernel launches issued by the library (bench and tests read it).
std::atomic<uint64_t>& launch_counter();

// Checks the launch that just happened and counts it.
inline void launched(const char* name) {
  launch_counter().fetch_add(1, std::memory_order_relaxed);
  cuda_check(cudaGetLastError(), name);
}

// Owning device allocation.
template <class T>
class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  explicit DeviceBuffer(size_t n) { reset(n); }
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  DeviceBuffer(DeviceBuffer&& o) noexcept : p_(std::exchange(o.p_, nullptr)), n_(std::exchange(o.n_, 0)) {}
  DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
    if (this != &o) {
      release();
      p_ = std::exchange(o.p_, nullptr);
      n_ = std::exchange(o.n_, 0);
    }
    return *this;
  }
  ~DeviceBuffer() { release(); }
  void reset(size_t n) {
    release();
    if (n > 0) {
      R3D_CUDA(cudaMalloc(reinterpret_cast<void**>(&p_), n * sizeof(T)));
      n_ = n;
    }
  }
  // Grows (never shrinks) the allocation; contents are not kept.
  void reserve(size_t n) {
    if (n > n_) reset(n);
  }
  T* get() const { return p_; }
  size_t size() const { return n_; }
  size_t bytes() const { return n_ * sizeof(T); }

 private:
  void release() {
    if (p_) cudaFree(p_);
    p_ = nullptr;
    n_ = 0;
  }
  T* p_ = nullptr;
  size_t n_ = 0;
};

inline int ceil_div(int a, int b) { return (a + b - 1) / b; }
inline int64_t ceil_div64(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace r3dgpu
