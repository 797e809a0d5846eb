// TEST INFRASTRUCTURE: a SIMT emulator that runs r3dgpu's CUDA kernel sources
// on the CPU (see regard3d_mvs_b200/csrc/simt.cuh). Every CUDA thread is a
// ucontext fiber; __syncthreads and warp shuffles are barriers that switch
// fibers; a barrier that can never complete (divergent __syncthreads, a warp
// shuffle with missing lanes) is reported as an error instead of hanging; a
// cp.async copy reads its source when issued and lands in shared memory only
// at the cp.async.wait_group that retires it. Built with AddressSanitizer,
// out-of-range shared or global accesses are caught as well.
#include <ucontext.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../regard3d_mvs_b200/csrc/runtime.h"

#if defined(__SANITIZE_ADDRESS__)
#include <sanitizer/common_interface_defs.h>
#define R3D_ASAN 1
#endif

namespace r3dsimt {
namespace {

enum class State { runnable, block_wait, warp_wait, done };

struct Copy {
  unsigned char* dst;
  unsigned char bytes[16];
  int size;
};

struct Fiber {
  ucontext_t ctx{};
  std::unique_ptr<char[]> stack;
  Coords c{};
  State state = State::runnable;
  std::vector<Copy> pending;
  std::deque<std::vector<Copy>> groups;
};

struct WarpState {
  int arrived = 0;
  uint32_t buf[32] = {};
};

constexpr size_t kStack = 256 * 1024;

thread_local std::vector<Fiber>* t_fibers = nullptr;
thread_local Fiber* t_cur = nullptr;
thread_local ucontext_t t_sched;
thread_local int t_block_arrived = 0;
thread_local int t_nthreads = 0;
thread_local std::vector<WarpState>* t_warps = nullptr;
thread_local std::unique_ptr<unsigned char[]> t_smem;
thread_local size_t t_smem_size = 0;
thread_local const std::function<void()>* t_body = nullptr;
thread_local std::string t_error;
#ifdef R3D_ASAN
thread_local const void* t_sched_stack_bottom = nullptr;
thread_local size_t t_sched_stack_size = 0;
#endif

void switch_to_sched() {
#ifdef R3D_ASAN
  void* fake = nullptr;
  __sanitizer_start_switch_fiber(&fake, t_sched_stack_bottom, t_sched_stack_size);
#endif
  swapcontext(&t_cur->ctx, &t_sched);
#ifdef R3D_ASAN
  __sanitizer_finish_switch_fiber(fake, nullptr, nullptr);
#endif
}

void apply_group(std::vector<Copy>& g) {
  for (Copy& c : g) std::memcpy(c.dst, c.bytes, static_cast<size_t>(c.size));
}

void fiber_entry() {
#ifdef R3D_ASAN
  __sanitizer_finish_switch_fiber(nullptr, &t_sched_stack_bottom, &t_sched_stack_size);
#endif
  try {
    (*t_body)();
  } catch (const std::exception& e) {
    if (t_error.empty()) t_error = e.what();
  }
  // Copies still in flight at exit are retired (the kernels drain explicitly).
  for (auto& g : t_cur->groups) apply_group(g);
  t_cur->groups.clear();
  apply_group(t_cur->pending);
  t_cur->pending.clear();
  t_cur->state = State::done;
#ifdef R3D_ASAN
  __sanitizer_start_switch_fiber(nullptr, t_sched_stack_bottom, t_sched_stack_size);
#endif
  setcontext(&t_sched);
}

int warp_of(const Fiber* f) {
  const Coords& c = f->c;
  const unsigned linear = c.tid.x + c.bdim.x * (c.tid.y + c.bdim.y * c.tid.z);
  return static_cast<int>(linear / 32);
}

unsigned linear_tid(const Fiber* f) {
  const Coords& c = f->c;
  return c.tid.x + c.bdim.x * (c.tid.y + c.bdim.y * c.tid.z);
}

void warp_barrier() {
  const int w = warp_of(t_cur);
  WarpState& ws = (*t_warps)[w];
  const int lanes = std::min(32, t_nthreads - w * 32);
  if (lanes != 32) throw std::runtime_error("simt: warp operation in a partial warp");
  if (++ws.arrived == lanes) {
    ws.arrived = 0;
    for (Fiber& f : *t_fibers)
      if (f.state == State::warp_wait && warp_of(&f) == w) f.state = State::runnable;
    return;
  }
  t_cur->state = State::warp_wait;
  switch_to_sched();
}

}  // namespace

const Coords& coords() { return t_cur->c; }

unsigned char* dynamic_smem() { return t_smem.get(); }

uint32_t lane_id() { return linear_tid(t_cur) & 31u; }

uint32_t shfl(uint32_t v, int src) {
  WarpState& ws = (*t_warps)[warp_of(t_cur)];
  ws.buf[lane_id()] = v;
  warp_barrier();
  const uint32_t r = ws.buf[src & 31];
  warp_barrier();
  return r;
}

uint32_t shfl_xor(uint32_t v, int m) { return shfl(v, static_cast<int>(lane_id() ^ static_cast<uint32_t>(m))); }

uint32_t match_any(uint32_t v) {
  WarpState& ws = (*t_warps)[warp_of(t_cur)];
  ws.buf[lane_id()] = v;
  warp_barrier();
  uint32_t r = 0;
  for (int i = 0; i < 32; ++i)
    if (ws.buf[i] == v) r |= 1u << i;
  warp_barrier();
  return r;
}

uint32_t ballot(bool p) {
  WarpState& ws = (*t_warps)[warp_of(t_cur)];
  ws.buf[lane_id()] = p ? 1u : 0u;
  warp_barrier();
  uint32_t r = 0;
  for (int i = 0; i < 32; ++i)
    if (ws.buf[i]) r |= 1u << i;
  warp_barrier();
  return r;
}

void syncwarp() { warp_barrier(); }

void syncthreads() {
  if (++t_block_arrived == t_nthreads) {
    t_block_arrived = 0;
    for (Fiber& f : *t_fibers)
      if (f.state == State::block_wait) f.state = State::runnable;
    return;
  }
  t_cur->state = State::block_wait;
  switch_to_sched();
}

void cp_async16(void* dst, const void* src) {
  if ((reinterpret_cast<uintptr_t>(dst) & 15u) || (reinterpret_cast<uintptr_t>(src) & 15u))
    throw std::runtime_error("simt: misaligned cp.async");
  unsigned char* d = static_cast<unsigned char*>(dst);
  if (d < t_smem.get() || d + 16 > t_smem.get() + t_smem_size) throw std::runtime_error("simt: cp.async outside shared memory");
  Copy c;
  c.dst = d;
  c.size = 16;
  std::memcpy(c.bytes, src, 16);
  t_cur->pending.push_back(c);
}

void cp_async8(void* dst, const void* src) {
  if ((reinterpret_cast<uintptr_t>(dst) & 7u) || (reinterpret_cast<uintptr_t>(src) & 7u))
    throw std::runtime_error("simt: misaligned cp.async");
  unsigned char* d = static_cast<unsigned char*>(dst);
  if (d < t_smem.get() || d + 8 > t_smem.get() + t_smem_size) throw std::runtime_error("simt: cp.async outside shared memory");
  Copy c;
  c.dst = d;
  c.size = 8;
  std::memcpy(c.bytes, src, 8);
  t_cur->pending.push_back(c);
}

void cp_async4(void* dst, const void* src) {
  if ((reinterpret_cast<uintptr_t>(dst) & 3u) || (reinterpret_cast<uintptr_t>(src) & 3u))
    throw std::runtime_error("simt: misaligned cp.async");
  unsigned char* d = static_cast<unsigned char*>(dst);
  if (d < t_smem.get() || d + 4 > t_smem.get() + t_smem_size) throw std::runtime_error("simt: cp.async outside shared memory");
  Copy c;
  c.dst = d;
  c.size = 4;
  std::memcpy(c.bytes, src, 4);
  t_cur->pending.push_back(c);
}

void cp_async_commit() {
  t_cur->groups.push_back(std::move(t_cur->pending));
  t_cur->pending.clear();
}

void cp_async_wait_n(int n) {
  while (static_cast<int>(t_cur->groups.size()) > n) {
    apply_group(t_cur->groups.front());
    t_cur->groups.pop_front();
  }
}

void launch(dim3 grid, dim3 block, size_t smem, const std::function<void()>& body) {
  const int nthreads = static_cast<int>(block.x * block.y * block.z);
  std::vector<Fiber> fibers(nthreads);
  for (Fiber& f : fibers) f.stack.reset(new char[kStack]);
  std::vector<WarpState> warps((nthreads + 31) / 32);
  t_fibers = &fibers;
  t_warps = &warps;
  t_nthreads = nthreads;
  t_body = &body;
  t_error.clear();
  for (unsigned bz = 0; bz < grid.z; ++bz)
    for (unsigned by = 0; by < grid.y; ++by)
      for (unsigned bx = 0; bx < grid.x; ++bx) {
        t_smem.reset(smem > 0 ? new unsigned char[smem] : nullptr);
        t_smem_size = smem;
        if (smem > 0) std::memset(t_smem.get(), 0xA5, smem);  // garbage, as on a GPU
        t_block_arrived = 0;
        int i = 0;
        for (unsigned tz = 0; tz < block.z; ++tz)
          for (unsigned ty = 0; ty < block.y; ++ty)
            for (unsigned tx = 0; tx < block.x; ++tx, ++i) {
              Fiber& f = fibers[i];
              f.c.tid = uint3{tx, ty, tz};
              f.c.bid = uint3{bx, by, bz};
              f.c.bdim = block;
              f.c.gdim = grid;
              f.state = State::runnable;
              f.pending.clear();
              f.groups.clear();
              getcontext(&f.ctx);
              f.ctx.uc_stack.ss_sp = f.stack.get();
              f.ctx.uc_stack.ss_size = kStack;
              f.ctx.uc_link = &t_sched;
              makecontext(&f.ctx, fiber_entry, 0);
            }
        while (true) {
          bool progressed = false, all_done = true;
          for (Fiber& f : fibers) {
            if (f.state == State::done) continue;
            all_done = false;
            if (f.state != State::runnable) continue;
            t_cur = &f;
#ifdef R3D_ASAN
            void* fake = nullptr;
            __sanitizer_start_switch_fiber(&fake, f.stack.get(), kStack);
#endif
            swapcontext(&t_sched, &f.ctx);
#ifdef R3D_ASAN
            __sanitizer_finish_switch_fiber(fake, nullptr, nullptr);
#endif
            progressed = true;
            if (!t_error.empty()) break;
          }
          if (!t_error.empty()) throw std::runtime_error(t_error);
          if (all_done) break;
          if (!progressed) {
            int done = 0, bw = 0, ww = 0;
            for (Fiber& f : fibers) {
              done += f.state == State::done;
              bw += f.state == State::block_wait;
              ww += f.state == State::warp_wait;
            }
            throw std::runtime_error("simt: barrier deadlock (done " + std::to_string(done) + ", at __syncthreads " +
                                     std::to_string(bw) + ", at warp barrier " + std::to_string(ww) + ")");
          }
        }
      }
  t_fibers = nullptr;
  t_cur = nullptr;
}

}  // namespace r3dsimt

// ------------------------------------------------------------------ fake runtime
namespace {
thread_local cudaError_t t_last = cudaSuccess;
cudaError_t ok() { return cudaSuccess; }
}  // namespace

struct FakeEvent {
  std::chrono::steady_clock::time_point t;
};

const char* cudaGetErrorString(cudaError_t e) { return e == cudaSuccess ? "no error" : "emulated CUDA error"; }
cudaError_t cudaGetLastError() {
  const cudaError_t e = t_last;
  t_last = cudaSuccess;
  return e;
}
cudaError_t cudaPeekAtLastError() { return t_last; }
cudaError_t cudaMalloc(void** p, size_t n) {
  *p = n ? static_cast<void*>(new (std::nothrow) unsigned char[n]) : nullptr;
  if (n && !*p) return cudaErrorMemoryAllocation;
  if (*p) std::memset(*p, 0x5A, n);
  return ok();
}
cudaError_t cudaFree(void* p) {
  delete[] static_cast<unsigned char*>(p);
  return ok();
}
cudaError_t cudaMallocHost(void** p, size_t n) { return cudaMalloc(p, n); }
cudaError_t cudaHostAlloc(void** p, size_t n, unsigned) { return cudaMalloc(p, n); }
cudaError_t cudaHostGetDevicePointer(void** d, void* h, unsigned) {
  *d = h;
  return ok();
}
cudaError_t cudaFreeHost(void* p) { return cudaFree(p); }
cudaError_t cudaMemcpy(void* d, const void* s, size_t n, cudaMemcpyKind) {
  if (n) std::memmove(d, s, n);
  return ok();
}
cudaError_t cudaMemcpyAsync(void* d, const void* s, size_t n, cudaMemcpyKind k, cudaStream_t) {
  return cudaMemcpy(d, s, n, k);
}
cudaError_t cudaMemcpy2DAsync(void* d, size_t dp, const void* s, size_t sp, size_t w, size_t h, cudaMemcpyKind,
                              cudaStream_t) {
  for (size_t y = 0; y < h; ++y) std::memmove(static_cast<char*>(d) + y * dp, static_cast<const char*>(s) + y * sp, w);
  return ok();
}
cudaError_t cudaMemsetAsync(void* d, int v, size_t n, cudaStream_t) {
  if (n) std::memset(d, v, n);
  return ok();
}
cudaError_t cudaMemset(void* d, int v, size_t n) { return cudaMemsetAsync(d, v, n, nullptr); }
cudaError_t cudaStreamSynchronize(cudaStream_t) { return ok(); }
cudaError_t cudaStreamCreateWithFlags(cudaStream_t* st, unsigned) {
  *st = nullptr;
  return ok();
}
cudaError_t cudaStreamDestroy(cudaStream_t) { return ok(); }
cudaError_t cudaDeviceSynchronize() { return ok(); }
cudaError_t cudaGetDevice(int* d) {
  *d = 0;
  return ok();
}
cudaError_t cudaSetDevice(int) { return ok(); }
cudaError_t cudaGetDeviceCount(int* n) {
  *n = 1;
  return ok();
}
cudaError_t cudaGetDeviceProperties(cudaDeviceProp* p, int) {
  std::memset(p, 0, sizeof(*p));
  std::strcpy(p->name, "SIMT emulator");
  p->major = 10;
  p->minor = 0;
  p->multiProcessorCount = 3;
  p->sharedMemPerBlockOptin = 227 * 1024;
  return ok();
}
cudaError_t cudaDeviceGetAttribute(int* v, cudaDeviceAttr a, int) {
  *v = a == cudaDevAttrMultiProcessorCount ? 3 : 227 * 1024;
  return ok();
}
cudaError_t cudaEventCreate(cudaEvent_t* e) {
  *e = new FakeEvent;
  return ok();
}
cudaError_t cudaEventDestroy(cudaEvent_t e) {
  delete e;
  return ok();
}
cudaError_t cudaEventCreateWithFlags(cudaEvent_t* e, unsigned) { return cudaEventCreate(e); }

cudaError_t cudaEventRecord(cudaEvent_t e, cudaStream_t) {
  e->t = std::chrono::steady_clock::now();
  return ok();
}
cudaError_t cudaEventSynchronize(cudaEvent_t) { return ok(); }
cudaError_t cudaEventElapsedTime(float* ms, cudaEvent_t a, cudaEvent_t b) {
  *ms = std::chrono::duration<float, std::milli>(b->t - a->t).count();
  return ok();
}
cudaError_t cudaStreamWaitEvent(cudaStream_t, cudaEvent_t, unsigned) { return ok(); }
