// TEST INFRASTRUCTURE: the subset of the CUDA runtime API that r3dgpu's host
// code uses, implemented on host memory for the SIMT emulator build
// (simt_emu.cpp). Kernel launches run synchronously on fibers; "device"
// allocations are exact-size heap blocks so that AddressSanitizer checks every
// access the kernels make.
#pragma once

#include <cstddef>
#include <cstdint>

typedef int cudaError_t;
enum : int {
  cudaSuccess = 0,
  cudaErrorInvalidValue = 1,
  cudaErrorMemoryAllocation = 2,
  cudaErrorNoDevice = 100,
};
typedef struct FakeStream* cudaStream_t;
typedef struct FakeEvent* cudaEvent_t;
enum cudaMemcpyKind {
  cudaMemcpyHostToHost = 0,
  cudaMemcpyHostToDevice = 1,
  cudaMemcpyDeviceToHost = 2,
  cudaMemcpyDeviceToDevice = 3,
  cudaMemcpyDefault = 4
};
enum cudaDeviceAttr { cudaDevAttrMultiProcessorCount = 16, cudaDevAttrMaxSharedMemoryPerBlockOptin = 97 };
enum cudaFuncAttribute { cudaFuncAttributeMaxDynamicSharedMemorySize = 8 };
struct cudaDeviceProp {
  char name[256];
  int major, minor, multiProcessorCount;
  size_t sharedMemPerBlockOptin;
};

const char* cudaGetErrorString(cudaError_t e);
cudaError_t cudaGetLastError();
cudaError_t cudaPeekAtLastError();
cudaError_t cudaMalloc(void** p, size_t n);
cudaError_t cudaFree(void* p);
cudaError_t cudaMallocHost(void** p, size_t n);
cudaError_t cudaHostAlloc(void** p, size_t n, unsigned flags);
cudaError_t cudaHostGetDevicePointer(void** d, void* h, unsigned flags);
cudaError_t cudaFreeHost(void* p);
cudaError_t cudaMemcpy(void* d, const void* s, size_t n, cudaMemcpyKind k);
cudaError_t cudaMemcpyAsync(void* d, const void* s, size_t n, cudaMemcpyKind k, cudaStream_t st = nullptr);
cudaError_t cudaMemcpy2DAsync(void* d, size_t dpitch, const void* s, size_t spitch, size_t width, size_t height,
                              cudaMemcpyKind k, cudaStream_t st = nullptr);
cudaError_t cudaMemsetAsync(void* d, int v, size_t n, cudaStream_t st = nullptr);
cudaError_t cudaMemset(void* d, int v, size_t n);
cudaError_t cudaStreamSynchronize(cudaStream_t st);
cudaError_t cudaStreamCreateWithFlags(cudaStream_t* st, unsigned flags);
cudaError_t cudaStreamDestroy(cudaStream_t st);
cudaError_t cudaDeviceSynchronize();
cudaError_t cudaGetDevice(int* d);
cudaError_t cudaSetDevice(int d);
cudaError_t cudaGetDeviceCount(int* n);
cudaError_t cudaGetDeviceProperties(cudaDeviceProp* p, int d);
cudaError_t cudaDeviceGetAttribute(int* v, cudaDeviceAttr a, int d);
cudaError_t cudaEventCreate(cudaEvent_t* e);
cudaError_t cudaEventCreateWithFlags(cudaEvent_t* e, unsigned flags);
cudaError_t cudaEventDestroy(cudaEvent_t e);
cudaError_t cudaEventRecord(cudaEvent_t e, cudaStream_t st = nullptr);
cudaError_t cudaEventSynchronize(cudaEvent_t e);
cudaError_t cudaEventElapsedTime(float* ms, cudaEvent_t a, cudaEvent_t b);
cudaError_t cudaStreamWaitEvent(cudaStream_t st, cudaEvent_t e, unsigned flags = 0);

// Emulated device memory is host memory: a symbol's address is its own.
template <class T>
cudaError_t cudaGetSymbolAddress(void** p, const T& symbol) {
  *p = const_cast<void*>(static_cast<const void*>(&symbol));
  return cudaSuccess;
}
template <class F>
cudaError_t cudaFuncSetAttribute(F, cudaFuncAttribute, int) {
  return cudaSuccess;
}
template <class F>
cudaError_t cudaOccupancyMaxActiveBlocksPerMultiprocessor(int* n, F, int, size_t) {
  *n = 1;
  return cudaSuccess;
}

#define cudaStreamNonBlocking 1u
#define cudaEventDisableTiming 2u
#define cudaHostAllocMapped 2u
