// Speckle filter whose union-find scratch is a static device array instead of
// library-allocated memory (r3dgpu_remove_speckles_no_alloc).
//
// Some callers cannot let the library allocate GPU memory: a host application
// whose own pool allocator already owns the device's memory, or a pipeline
// that cannot afford the device-wide synchronisation that cudaFree brings.
// For them the scratch lives in g_speckle_scratch below. Under CUDA's lazy
// module loading (the default since CUDA 12.2) the array is reserved on a
// GPU when this file's module is first loaded there, which is the first
// call's cudaGetSymbolAddress; it is then held until the process exits.
#include <mutex>
#include <string>

#include "common.cuh"
#include "kernels.h"

namespace r3dgpu {

// Largest map the static scratch serves: 4,194,304 pixels (2048 x 2048, for
// example). The union-find keeps two ints per pixel (parent and segment
// size), so the array takes 32 MiB on every GPU that loads the library.
constexpr int64_t kStaticSpeckleMaxPixels = int64_t{1} << 22;

// In host code this name is a host-side stand-in, not a device address:
// kernels only ever receive the address that cudaGetSymbolAddress returns.
#ifdef R3DGPU_SIMT_EMULATION
alignas(256) static int g_speckle_scratch[2 * kStaticSpeckleMaxPixels];
#else
static __device__ __align__(256) int g_speckle_scratch[2 * kStaticSpeckleMaxPixels];
#endif

namespace {

constexpr int kMaxDevices = 64;

// Device address of g_speckle_scratch on `dev` (the current device), looked
// up on the first call per device and cached. The lookup loads the module on
// that device and so reserves the array there: a device that has no room for
// it answers cudaErrorMemoryAllocation, which becomes R3DGPU_ENOMEM.
int* static_speckle_scratch(int dev) {
  static std::mutex mu;
  static void* address[kMaxDevices] = {};
  std::lock_guard<std::mutex> lock(mu);
  if (!address[dev]) {
    void* p = nullptr;
    cuda_check(cudaGetSymbolAddress(&p, g_speckle_scratch), "remove_speckles_no_alloc: cudaGetSymbolAddress");
    address[dev] = p;
  }
  return static_cast<int*>(address[dev]);
}

// The map must be memory of `dev` that kernels there can use (device or
// managed memory): a host pointer or another device's memory is rejected
// before any launch.
void check_map_device(const float* d, int dev) {
#ifndef R3DGPU_SIMT_EMULATION
  cudaPointerAttributes attr{};
  if (cudaPointerGetAttributes(&attr, d) != cudaSuccess) {
    (void)cudaGetLastError();
    fail(R3DGPU_EINVAL, "remove_speckles_no_alloc: the map is not CUDA memory");
  }
  if (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged)
    fail(R3DGPU_EINVAL, "remove_speckles_no_alloc: the map is not device memory");
  if (attr.type == cudaMemoryTypeDevice && attr.device != dev)
    fail(R3DGPU_EINVAL, "remove_speckles_no_alloc: the map is memory of device " + std::to_string(attr.device) +
                            ", this thread's device is " + std::to_string(dev) + " (r3dgpu_set_device)");
#else
  (void)d;
  (void)dev;
#endif
}

}  // namespace

void remove_speckles_static_scratch(int dev, float* d, int w, int h, int min_size, float max_diff, cudaStream_t s) {
  if (!d && w > 0 && h > 0) fail(R3DGPU_EINVAL, "remove_speckles_no_alloc: null argument");
  if (w < 0 || h < 0) fail(R3DGPU_EINVAL, "remove_speckles_no_alloc: negative width or height");
  const int64_t n = static_cast<int64_t>(w) * h;
  if (n > kStaticSpeckleMaxPixels)
    fail(R3DGPU_EINVAL, "remove_speckles_no_alloc: " + std::to_string(w) + " x " + std::to_string(h) + " = " +
                            std::to_string(n) + " pixels exceeds the static scratch maximum of " +
                            std::to_string(kStaticSpeckleMaxPixels) + " pixels");
  if (dev < 0 || dev >= kMaxDevices) fail(R3DGPU_EDEVICE, "remove_speckles_no_alloc: device ordinal out of range");
  R3D_CUDA(cudaSetDevice(dev));
  if (n > 0) check_map_device(d, dev);
  // Set-up on every call, so that an empty call (width = height = 0) serves
  // as the warm-up that reserves the array.
  int* scratch = static_speckle_scratch(dev);
  if (min_size <= 1 || n == 0) return;
  // uf_tile_kernel (image_kernels.cu) writes parent and size of every pixel
  // of the map before any other kernel of the filter reads them, so the
  // previous call's contents never matter.
  launch_remove_speckles(d, w, h, min_size, max_diff, scratch, s);
}

}  // namespace r3dgpu
