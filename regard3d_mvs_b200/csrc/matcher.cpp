// Host side of r3dgpu: option checks, level pyramid, tile layout, the stage
// sequence of every level, batching of many pairs, and the C ABI.
//
// The control flow restates r3d::match_stereo (rhiestan/Regard3D_MVS,
// src/r3d/stereo/stereo_matcher.cpp:1023-1095) and match_level (:831-886):
// levels L..0, full label range at the coarsest level, per-pixel ranges from
// the coarser disparities below it, a left and (with lr_full_match) a
// mirrored right-to-left match per level, the left-right check(s), speckle
// and median filters. Every stage runs on the GPU; the host only plans
// (tile layout, job tables, buffer sizes) and launches.
#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "kernels.h"
#include "matcher_internal.h"
#include "sgm.h"
#include "sgm_full.h"
#include "sgm_path.h"
#include "sgm_ranged.h"
#include "tuning.h"

namespace r3dgpu {
namespace {

// Ranged tiles go to the ranged kernel unless R3DGPU_RANGED_KERNEL=general
// selects the general per-chunk kernel (both compute the same results).
bool general_ranged_kernel() {
  const char* e = std::getenv("R3DGPU_RANGED_KERNEL");
  return e != nullptr && std::string(e) == "general";
}

// Ranged tiles whose row shape would be at least this many labels wide go to
// the general kernel (the tuning table's ranged_general_width, or
// R3DGPU_RANGED_GENERAL_WIDTH; default: none).
int general_width() {
  if (const char* e = std::getenv("R3DGPU_RANGED_GENERAL_WIDTH")) return std::atoi(e) > 0 ? std::atoi(e) : 1 << 30;
  return tuning().ranged_general_width > 0 ? tuning().ranged_general_width : 1 << 30;
}


thread_local std::string t_error;
thread_local int t_device = 0;
thread_local r3dgpu_cancel_token* t_cancel = nullptr;
thread_local size_t t_scratch_budget = 0;  // 0: the default SGM scratch budget

// Profiling of the SGM launches (r3dgpu_profile_*).
struct ProfileState {
  bool on = false;
  r3dgpu_profile acc{};
  struct Pending {
    cudaEvent_t a, b;
    uint64_t cells, tiles, pixels;
    std::string kernel, shape;
    int grid, rows;
    bool span;  // the SGM stage of a round (fork to join), not one launch
    bool pass = false;  // one pass launch of the chain kernels (inside a group)
    uint64_t bytes = 0;  // its algorithmic HBM bytes
  };
  std::vector<Pending> pending;
  std::string launches;       // JSON objects of the launches since the last take
  std::string last_launches;  // those of the last take
};
thread_local ProfileState t_prof;

void profile_collect() {
  for (auto& p : t_prof.pending) {
    float ms = 0.0F;
    if (cudaEventElapsedTime(&ms, p.a, p.b) != cudaSuccess) ms = 0.0F;
    (void)cudaGetLastError();
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
    if (p.pass) {
      char line[256];
      std::snprintf(line, sizeof(line),
                    "{\"kernel\": \"%s\", \"pass\": true, \"shape\": \"%s\", \"cells\": %llu, \"pixels\": %llu, "
                    "\"bytes\": %llu, \"ms\": %.4f}",
                    p.kernel.c_str(), p.shape.c_str(), static_cast<unsigned long long>(p.cells),
                    static_cast<unsigned long long>(p.pixels), static_cast<unsigned long long>(p.bytes),
                    static_cast<double>(ms));
      if (!t_prof.launches.empty()) t_prof.launches += ", ";
      t_prof.launches += line;
      continue;
    }
    if (p.span) {
      // Launches of a round overlap: the stage time is the round's span.
      t_prof.acc.sgm_ms += ms;
      char line[96];
      std::snprintf(line, sizeof(line), "{\"kernel\": \"sgm_round\", \"ms\": %.4f}", static_cast<double>(ms));
      if (!t_prof.launches.empty()) t_prof.launches += ", ";
      t_prof.launches += line;
      continue;
    }
    t_prof.acc.sgm_launches += 1;
    t_prof.acc.sgm_cells += p.cells;
    t_prof.acc.sgm_tiles += p.tiles;
    t_prof.acc.sgm_pixels += p.pixels;
    char line[256];
    std::snprintf(line, sizeof(line),
                  "{\"kernel\": \"%s\", \"shape\": \"%s\", \"tiles\": %llu, \"cells\": %llu, \"pixels\": %llu, "
                  "\"ms\": %.4f, \"grid\": %d, \"rows\": %d}",
                  p.kernel.c_str(), p.shape.c_str(), static_cast<unsigned long long>(p.tiles),
                  static_cast<unsigned long long>(p.cells), static_cast<unsigned long long>(p.pixels),
                  static_cast<double>(ms), p.grid, p.rows);
    if (!t_prof.launches.empty()) t_prof.launches += ", ";
    t_prof.launches += line;
  }
  t_prof.pending.clear();
}

int align16(int n) { return (n + 15) / 16 * 16; }
// stereo_matcher.cpp:889-890
int floor_shift(int v, int k) { return v >= 0 ? v >> k : -((-v + (1 << k) - 1) >> k); }
int ceil_shift(int v, int k) { return -floor_shift(-v, k); }

// stereo_matcher.cpp:81-95 (same conditions and messages).
void check_options(const r3dgpu_stereo_options& o) {
  if (o.p1 < 0 || o.p2 < o.p1 || o.p2 > 8000)
    fail(R3DGPU_EINVAL, "stereo: invalid penalties P1 = " + std::to_string(o.p1) + ", P2 = " + std::to_string(o.p2) +
                            " (0 <= P1 <= P2 <= 8000)");
  if (o.invalid_cost < 0 || o.invalid_cost > 255)
    fail(R3DGPU_EINVAL, "stereo: invalid_cost " + std::to_string(o.invalid_cost) + " outside [0, 255]");
  if (o.tile_size < 16 || o.tile_margin < 0 || o.tile_blend < 0)
    fail(R3DGPU_EINVAL, "stereo: invalid tiling " + std::to_string(o.tile_size) + " / " + std::to_string(o.tile_margin) +
                            " / " + std::to_string(o.tile_blend));
  if (o.levels < -1 || o.levels > 12 || o.range_radius < 0 || o.range_margin < 0 || o.range_fill < 0)
    fail(R3DGPU_EINVAL, "stereo: invalid hierarchy levels " + std::to_string(o.levels) + " / radius " +
                            std::to_string(o.range_radius) + " / margin " + std::to_string(o.range_margin) + " / fill " +
                            std::to_string(o.range_fill));
  if (o.subpixel < 0 || o.subpixel > 2) fail(R3DGPU_EINVAL, "stereo: invalid subpixel method");
}

// stereo_matcher.cpp:1105-1122
int automatic_levels(int width, int height, int nd) {
  int levels = 0, w = width, h = height, n = nd;
  while (levels < 8) {
    const int nw = (w + 1) / 2, nh = (h + 1) / 2;
    if (std::min(nw, nh) < 96 || n <= 48) break;
    w = nw;
    h = nh;
    n = (n + 1) / 2;
    ++levels;
  }
  return levels;
}

// stereo_matcher.cpp:69-79
void p2_lut(const r3dgpu_stereo_options& o, uint16_t* lut) {
  for (int di = 0; di < 256; ++di) {
    int p2 = o.p2;
    if (o.p2_adapt > 0) p2 = std::max(o.p1 + 1, o.p2 * o.p2_adapt / (o.p2_adapt + di));
    lut[di] = static_cast<uint16_t>(p2);
  }
}

}  // namespace

}  // namespace r3dgpu

// A cancellation flag in page-locked host memory and its device view.
struct r3dgpu_cancel_token {
  int32_t* host = nullptr;
  const int* dev = nullptr;
};

namespace r3dgpu {
namespace {

// Throws ECANCELLED when this thread's token is set (the reference's
// CancelToken::check, src/r3d/core/cancel.hpp:36-55).
void check_cancel() {
  if (t_cancel != nullptr && *reinterpret_cast<volatile int32_t*>(t_cancel->host) != 0)
    fail(R3DGPU_ECANCELLED, "stereo: cancelled");
}

const int* cancel_device_flag() { return t_cancel != nullptr ? t_cancel->dev : nullptr; }

}  // namespace

bool profile_on() { return t_prof.on; }

cudaEvent_t profile_mark(cudaStream_t s) {
  cudaEvent_t e = nullptr;
  R3D_CUDA(cudaEventCreate(&e));
  R3D_CUDA(cudaEventRecord(e, s));
  return e;
}

void profile_pass(cudaEvent_t a, cudaEvent_t b, const char* kernel, const char* shape, uint64_t cells,
                  uint64_t pixels, uint64_t bytes) {
  ProfileState::Pending p{};
  p.a = a;
  p.b = b;
  p.kernel = kernel;
  p.shape = shape;
  p.cells = cells;
  p.pixels = pixels;
  p.pass = true;
  p.bytes = bytes;
  t_prof.pending.push_back(p);
}

namespace {

// ------------------------------------------------------------------ memory
// Bump allocator over grow-only device chunks; reset() rewinds it so that the
// next call reuses the same memory without cudaMalloc.
class Arena {
 public:
  void reset() {
    for (auto& c : chunks_) c.used = 0;
    cur_ = 0;
  }
  template <class T>
  T* alloc(size_t n) {
    size_t bytes = (n * sizeof(T) + 255) & ~static_cast<size_t>(255);
    if (bytes == 0) bytes = 256;
    while (cur_ < chunks_.size()) {
      Chunk& c = chunks_[cur_];
      if (c.used + bytes <= c.buf.size()) {
        T* p = reinterpret_cast<T*>(c.buf.get() + c.used);
        c.used += bytes;
        return p;
      }
      ++cur_;
    }
    chunks_.emplace_back();
    chunks_.back().buf.reset(std::max(bytes, kChunk));
    chunks_.back().used = bytes;
    cur_ = chunks_.size() - 1;
    return reinterpret_cast<T*>(chunks_.back().buf.get());
  }

 private:
  static constexpr size_t kChunk = size_t{256} << 20;
  struct Chunk {
    DeviceBuffer<unsigned char> buf;
    size_t used = 0;
  };
  std::vector<Chunk> chunks_;
  size_t cur_ = 0;
};

// Grow-only pinned host staging.
class Pinned {
 public:
  ~Pinned() {
    if (p_) cudaFreeHost(p_);
  }
  void reset() { used_ = 0; }
  template <class T>
  T* alloc(size_t n) {
    const size_t bytes = (n * sizeof(T) + 255) & ~static_cast<size_t>(255);
    if (used_ + bytes > cap_) {
      // Earlier allocations of this call stay valid: keep them in retired blocks.
      if (p_) retired_.push_back(p_);
      cap_ = std::max(bytes, std::max(cap_ * 2, size_t{1} << 20));
      R3D_CUDA(cudaMallocHost(reinterpret_cast<void**>(&p_), cap_));
      used_ = 0;
    }
    T* r = reinterpret_cast<T*>(p_ + used_);
    used_ += bytes;
    return r;
  }
  // Frees the blocks replaced during the last call (after the stream synced).
  void release_retired() {
    for (unsigned char* p : retired_) cudaFreeHost(p);
    retired_.clear();
  }
  // Hands the replaced blocks to a caller that still needs them (a captured
  // graph copies from them on every replay); it frees them with cudaFreeHost.
  std::vector<unsigned char*> take_retired() { return std::move(retired_); }

 private:
  unsigned char* p_ = nullptr;
  size_t cap_ = 0, used_ = 0;
  std::vector<unsigned char*> retired_;
};

struct Workspace {
  int device = -1;
  int sms = 0;
  int smem_optin = 0;
  Arena arena;
  Pinned pinned;
  DeviceBuffer<unsigned char> scratch;
  DeviceBuffer<int> counter;
  // Side streams for the concurrent SGM launches of a round, and the events
  // that fork them from and join them into the call's stream (created on
  // first use, kept for the workspace's life).
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> side_done;
  cudaEvent_t fork = nullptr;
  // Stream and events of a second track of a batch (slot 1 workspaces).
  cudaStream_t track = nullptr;
  cudaEvent_t track_start = nullptr, track_done = nullptr;
  ~Workspace() {
    if (track != nullptr) cudaStreamDestroy(track);
    if (track_start != nullptr) cudaEventDestroy(track_start);
    if (track_done != nullptr) cudaEventDestroy(track_done);
    for (cudaStream_t st : side) cudaStreamDestroy(st);
    for (cudaEvent_t ev : side_done) cudaEventDestroy(ev);
    if (fork != nullptr) cudaEventDestroy(fork);
  }
  void ensure_side(int n) {
    if (fork == nullptr) R3D_CUDA(cudaEventCreate(&fork));
    while (static_cast<int>(side.size()) < n) {
      cudaStream_t st = nullptr;
      cudaEvent_t ev = nullptr;
      R3D_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
      R3D_CUDA(cudaEventCreate(&ev));
      side.push_back(st);
      side_done.push_back(ev);
    }
  }
};

// This thread's workspaces: per device, slot 0 (every entry point) and slot
// 1 (the single-level track of a batch that also has hierarchical pairs).
constexpr int kWorkspaceSlots = 2;
thread_local std::vector<std::unique_ptr<Workspace>> t_workspaces;

Workspace& workspace(int slot = 0) {
  std::vector<std::unique_ptr<Workspace>>& per_device = t_workspaces;
  const int dev = t_device;
  const int idx = dev * kWorkspaceSlots + slot;
  if (static_cast<int>(per_device.size()) <= idx) per_device.resize(idx + 1);
  if (!per_device[idx]) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= dev) {
      (void)cudaGetLastError();
      fail(R3DGPU_EDEVICE, "r3dgpu: no CUDA device " + std::to_string(dev));
    }
    R3D_CUDA(cudaSetDevice(dev));
    cudaDeviceProp prop{};
    R3D_CUDA(cudaGetDeviceProperties(&prop, dev));
#ifndef R3DGPU_SIMT_EMULATION
    if (prop.major != 10)
      fail(R3DGPU_EDEVICE, std::string("r3dgpu: built for sm_100a, device is ") + prop.name + " (sm_" +
                               std::to_string(prop.major) + std::to_string(prop.minor) + ")");
#endif
    auto ws = std::make_unique<Workspace>();
    ws->device = dev;
    ws->sms = prop.multiProcessorCount;
    ws->smem_optin = static_cast<int>(prop.sharedMemPerBlockOptin);
    ws->counter.reset(64);
    per_device[idx] = std::move(ws);
  }
  R3D_CUDA(cudaSetDevice(dev));
  return *per_device[idx];
}

// ------------------------------------------------------------------ views
template <class T>
struct DView {
  const T* p = nullptr;
  int w = 0, h = 0;
  int64_t stride = 0;
  bool empty() const { return p == nullptr || w == 0 || h == 0; }
};

// ------------------------------------------------------------------ tiles
struct Tile {
  int x0, y0, w, h;
  int c0x, c1x, c0y, c1y;
};

// stereo_matcher.cpp:545-552
std::vector<int> split(int size, int tile) {
  const int n = std::max(1, (size + tile - 1) / tile);
  std::vector<int> b(n + 1);
  for (int i = 0; i <= n; ++i) b[i] = static_cast<int>(static_cast<long long>(size) * i / n);
  return b;
}

struct Layout {
  std::vector<Tile> tiles;
  int tiles_x = 0;
};

Layout make_layout(int W, int H, int ts, const r3dgpu_stereo_options& o) {
  const int ext = o.tile_margin + (o.tile_blend + 1) / 2;
  Layout L;
  const auto bx = split(W, ts), by = split(H, ts);
  L.tiles_x = static_cast<int>(bx.size()) - 1;
  for (size_t j = 0; j + 1 < by.size(); ++j)
    for (size_t i = 0; i + 1 < bx.size(); ++i) {
      Tile t;
      t.x0 = std::max(0, bx[i] - ext);
      const int x1 = std::min(W, bx[i + 1] + ext);
      t.y0 = std::max(0, by[j] - ext);
      const int y1 = std::min(H, by[j + 1] + ext);
      t.w = x1 - t.x0;
      t.h = y1 - t.y0;
      t.c0x = bx[i];
      t.c1x = bx[i + 1];
      t.c0y = by[j];
      t.c1y = by[j + 1];
      L.tiles.push_back(t);
    }
  return L;
}

// stereo_matcher.cpp:571-578
size_t estimated_tile_bytes(uint64_t cells_u, const Tile& t, size_t right_width) {
  const size_t cells = static_cast<size_t>(cells_u);
  const size_t w = static_cast<size_t>(t.w), h = static_cast<size_t>(t.h);
  const size_t row_cells = cells / std::max<size_t>(h, 1);
  return cells * 2 + row_cells * 2 + 6 * (row_cells + w * 2 * 8) * 2 + w * h * 32 + (w + right_width + 16) * (h + 6) * 8;
}

// ------------------------------------------------------------------ pair state
struct Match {
  SgmMatch m{};
  Layout layout;
  int tile_size = 0;
  std::vector<uint64_t> tile_cells;  // host copy (ranged: counted on the device)
  std::vector<int> tile_maxnum;
  std::vector<int> tile_width;  // ranged: label width of the kernel shape chosen for the tile
  std::vector<int> tile_over32;  // ranged: pixels with more than 32 labels
  bool ranged = false;
  // device outputs of the SGM stage
  float* tile_disp = nullptr;
  float* tile_conf = nullptr;
  std::vector<size_t> tile_off;  // per tile, offset into tile_disp / tile_conf
  unsigned long long* d_cells = nullptr;
  int first_job = 0;
  // counting buffers (ranged)
  unsigned long long* d_count = nullptr;
  int* d_stats = nullptr;  // kTileStats per tile
  unsigned long long* h_count = nullptr;
  int* h_stats = nullptr;
};

struct LevelIn {
  DView<uint16_t> left, right;
  DView<uint8_t> lmask, rmask;
  int dmin = 0, nd = 0;
};

struct PairRun {
  const r3dgpu_pair* req = nullptr;
  r3dgpu_stereo_options o{};
  int levels = 0;
  bool check_lr = false, lr_full = false;
  std::vector<LevelIn> lv;
  int cur = -1;  // level being processed
  // coarser-level results
  float* coarse_left = nullptr;
  float* coarse_right = nullptr;
  int coarse_wl = 0, coarse_wr = 0, coarse_h = 0;
  // this level
  Match left, right;
  bool has_right = false;
  RowInterval *int_l = nullptr, *int_r = nullptr;
  float *disp_l = nullptr, *conf_l = nullptr, *disp_r = nullptr;
  uint64_t cells = 0;
  std::vector<unsigned long long*> cell_arrays;  // device, summed at the end
  std::vector<int> cell_counts;
  std::vector<unsigned long long*> h_cell_arrays;
};

DView<uint16_t> view_of(const r3dgpu_view_u16& v) { return {v.data, v.width, v.height, v.stride}; }
DView<uint8_t> view_of(const r3dgpu_view_u8& v) {
  DView<uint8_t> d{v.data, v.width, v.height, v.stride};
  if (d.empty()) return {};
  return d;
}

void validate_pair(const r3dgpu_pair& p) {
  check_options(p.options);
  if (p.num_disparities <= 0) fail(R3DGPU_EINVAL, "stereo: no disparities to search");
  const auto& L = p.left;
  const auto& R = p.right;
  if (L.data == nullptr || R.data == nullptr || L.width <= 0 || L.height <= 0 || R.width <= 0 || R.height <= 0 ||
      L.height != R.height)
    fail(R3DGPU_EINVAL, "stereo: rectified images must be non-empty with equal height (" + std::to_string(L.width) +
                            "x" + std::to_string(L.height) + ", " + std::to_string(R.width) + "x" +
                            std::to_string(R.height) + ")");
  if (L.stride < L.width || R.stride < R.width) fail(R3DGPU_EINVAL, "stereo: image stride smaller than width");
  const auto lv = view_of(p.left_valid), rv = view_of(p.right_valid);
  if (!lv.empty() && (lv.w != L.width || lv.h != L.height))
    fail(R3DGPU_EINVAL, "stereo: left mask size differs from the image");
  if (!rv.empty() && (rv.w != R.width || rv.h != R.height))
    fail(R3DGPU_EINVAL, "stereo: right mask size differs from the image");
  if (p.out.disparity == nullptr || p.out.stride < L.width) fail(R3DGPU_EINVAL, "stereo: missing output buffer");
  if (L.width > 65535 || R.width > 65535) fail(R3DGPU_EUNSUPPORTED, "stereo: images wider than 65535 pixels");
}

// Level pyramid (stereo_matcher.cpp:1036-1058): u16 images, reduced masks.
void build_levels(PairRun& P, Arena& A, cudaStream_t s) {
  const r3dgpu_pair& q = *P.req;
  P.lv.assign(P.levels + 1, LevelIn{});
  P.lv[0].left = view_of(q.left);
  P.lv[0].right = view_of(q.right);
  P.lv[0].lmask = view_of(q.left_valid);
  P.lv[0].rmask = view_of(q.right_valid);
  for (int l = 1; l <= P.levels; ++l) {
    const LevelIn& a = P.lv[l - 1];
    LevelIn& b = P.lv[l];
    auto down16 = [&](const DView<uint16_t>& v) {
      DView<uint16_t> o;
      o.w = (v.w + 1) / 2;
      o.h = (v.h + 1) / 2;
      o.stride = o.w;
      uint16_t* p = A.alloc<uint16_t>(static_cast<size_t>(o.w) * o.h);
      launch_pyramid_u16(v.p, v.stride, v.w, v.h, p, o.stride, s);
      o.p = p;
      return o;
    };
    auto down8 = [&](const DView<uint8_t>& v) {
      if (v.empty()) return DView<uint8_t>{};
      DView<uint8_t> o;
      o.w = (v.w + 1) / 2;
      o.h = (v.h + 1) / 2;
      o.stride = o.w;
      uint8_t* p = A.alloc<uint8_t>(static_cast<size_t>(o.w) * o.h);
      launch_reduce_mask(v.p, v.stride, v.w, v.h, p, o.stride, s);
      o.p = p;
      return o;
    };
    b.left = down16(a.left);
    b.right = down16(a.right);
    b.lmask = down8(a.lmask);
    b.rmask = down8(a.rmask);
  }
  const int dmin = q.disparity_min, dmax = q.disparity_min + q.num_disparities - 1;
  for (int l = 0; l <= P.levels; ++l) {
    P.lv[l].dmin = floor_shift(dmin, l);
    P.lv[l].nd = align16(ceil_shift(dmax, l) - P.lv[l].dmin + 1);
  }
}

void fill_match(SgmMatch& m, const r3dgpu_stereo_options& o, const DView<uint16_t>& base, const uint64_t* cb,
                const uint64_t* cp, int wp, const RowInterval* bv, const RowInterval* pv, const uint16_t* rlo,
                const uint16_t* rnum, int dmin, int nd, bool diagonal, bool confidence) {
  m = SgmMatch{};
  m.base = base.p;
  m.base_stride = base.stride;
  m.cbase = cb;
  m.cb_stride = base.w;
  m.cpart = cp;
  m.cp_stride = wp;
  m.bv = bv;
  m.pv = pv;
  m.rlo = rlo;
  m.rnum = rnum;
  m.r_stride = base.w;
  m.wb = base.w;
  m.wp = wp;
  m.h = base.h;
  m.dmin = dmin;
  m.nd = nd;
  m.p1 = o.p1;
  m.invalid_cost = o.invalid_cost;
  m.subpixel = o.subpixel;
  m.uniqueness = o.uniqueness;
  m.lr_max_diff = o.lr_max_diff;
  m.diagonal_lr = diagonal ? 1 : 0;
  m.confidence = confidence ? 1 : 0;
  p2_lut(o, m.lut);
  // A path value is at most max(P2) + max(cost) (min_q + P2 bounds the best
  // predecessor term); 8 of them fit 16 bits unless the penalties are extreme.
  int max_p2 = 0;
  for (int i = 0; i < 256; ++i) max_p2 = std::max(max_p2, static_cast<int>(m.lut[i]));
  m.sum_no_carry = 8 * (max_p2 + std::max(o.invalid_cost, 62)) <= 65535 ? 1 : 0;
  // L_r(p, d) - C(p, d) = min(L(q, d), L(q, d -+ 1) + P1, min L(q) + P2) - min L(q)
  // lies in [0, P2]: with P2 <= 255 the chain passes keep it in one byte.
  m.term_u8 = max_p2 <= 255 ? 1 : 0;
}

// Stage 1 of a level: mirrored inputs, Census images, row intervals, label
// ranges from the coarser level, candidate tile layouts (and their device
// cell counts for ranged matches).
void prepare_level(PairRun& P, Arena& A, Pinned& H, cudaStream_t s) {
  const int l = P.cur;
  const LevelIn& in = P.lv[l];
  const r3dgpu_stereo_options& o = P.o;
  const int wl = in.left.w, wr = in.right.w, h = in.left.h;
  auto census = [&](const DView<uint16_t>& v) {
    uint64_t* c = A.alloc<uint64_t>(static_cast<size_t>(v.w) * v.h);
    launch_census(v.p, v.stride, v.w, v.h, c, v.w, s);
    return c;
  };
  auto intervals = [&](const DView<uint8_t>& m, int w) {
    RowInterval* r = A.alloc<RowInterval>(h);
    launch_intervals(m.empty() ? nullptr : m.p, m.stride, w, h, r, s);
    return r;
  };
  const uint64_t* cl = census(in.left);
  const uint64_t* cr = census(in.right);
  P.int_l = intervals(in.lmask, wl);
  P.int_r = intervals(in.rmask, wr);
  const bool ranged = l < P.levels;
  const uint16_t *llo = nullptr, *lnum = nullptr, *rlo = nullptr, *rnum = nullptr;
  if (ranged) {
    if (P.coarse_left == nullptr) fail(R3DGPU_EDEVICE, "stereo: internal error, no coarser level");
    uint16_t* lo = A.alloc<uint16_t>(static_cast<size_t>(wl) * h);
    uint16_t* nu = A.alloc<uint16_t>(static_cast<size_t>(wl) * h);
    float* scr = A.alloc<float>(static_cast<size_t>(ranges_scratch_floats(P.coarse_wl, P.coarse_h, o.range_fill)));
    RangeParams rp{o.range_radius, o.range_margin, o.range_fill, in.dmin, in.nd, -1, 0};
    launch_ranges_from_coarse(P.coarse_left, P.coarse_wl, P.coarse_h, wl, h, in.lmask.empty() ? nullptr : in.lmask.p,
                              in.lmask.stride, P.int_r, rp, scr, lo, nu, s);
    llo = lo;
    lnum = nu;
  }
  fill_match(P.left.m, o, in.left, cl, cr, wr, P.int_l, P.int_r, llo, lnum, in.dmin, in.nd,
             P.check_lr && !P.lr_full, true);
  P.has_right = P.check_lr && P.lr_full;
  if (P.has_right) {
    uint16_t* ml = A.alloc<uint16_t>(static_cast<size_t>(wl) * h);
    uint16_t* mr = A.alloc<uint16_t>(static_cast<size_t>(wr) * h);
    launch_mirror_u16(in.left.p, in.left.stride, wl, h, ml, s);
    launch_mirror_u16(in.right.p, in.right.stride, wr, h, mr, s);
    const DView<uint16_t> vml{ml, wl, h, wl}, vmr{mr, wr, h, wr};
    DView<uint8_t> mlm, mrm;
    if (!in.lmask.empty()) {
      uint8_t* p = A.alloc<uint8_t>(static_cast<size_t>(wl) * h);
      launch_mirror_u8(in.lmask.p, in.lmask.stride, wl, h, p, s);
      mlm = {p, wl, h, wl};
    }
    if (!in.rmask.empty()) {
      uint8_t* p = A.alloc<uint8_t>(static_cast<size_t>(wr) * h);
      launch_mirror_u8(in.rmask.p, in.rmask.stride, wr, h, p, s);
      mrm = {p, wr, h, wr};
    }
    const uint64_t* cml = census(vml);
    const uint64_t* cmr = census(vmr);
    RowInterval* iml = intervals(mlm, wl);
    RowInterval* imr = intervals(mrm, wr);
    if (ranged) {
      if (P.coarse_right == nullptr) fail(R3DGPU_EDEVICE, "stereo: internal error, no coarser right map");
      uint16_t* lo = A.alloc<uint16_t>(static_cast<size_t>(wr) * h);
      uint16_t* nu = A.alloc<uint16_t>(static_cast<size_t>(wr) * h);
      float* scr = A.alloc<float>(static_cast<size_t>(ranges_scratch_floats(P.coarse_wr, P.coarse_h, o.range_fill)));
      RangeParams rp{o.range_radius, o.range_margin, o.range_fill, in.dmin, in.nd, +1, 1};
      launch_ranges_from_coarse(P.coarse_right, P.coarse_wr, P.coarse_h, wr, h,
                                in.rmask.empty() ? nullptr : in.rmask.p, in.rmask.stride, P.int_l, rp, scr, lo, nu, s);
      rlo = lo;
      rnum = nu;
    }
    fill_match(P.right.m, o, vmr, cmr, cml, wl, imr, iml, rlo, rnum, in.dmin + wr - wl, in.nd, false, false);
  }
  // Candidate layouts; ranged matches count their tiles' labels on the device.
  auto plan = [&](Match& M, int W) {
    M.ranged = M.m.rlo != nullptr;
    M.tile_size = o.tile_size;
    M.layout = make_layout(W, h, M.tile_size, o);
    if (M.ranged) {
      const int n = static_cast<int>(M.layout.tiles.size());
      int4* ht = H.alloc<int4>(n);
      for (int i = 0; i < n; ++i) {
        const Tile& t = M.layout.tiles[i];
        ht[i] = make_int4(t.x0, t.y0, t.w, t.h);
      }
      int4* dt = A.alloc<int4>(n);
      R3D_CUDA(cudaMemcpyAsync(dt, ht, sizeof(int4) * n, cudaMemcpyHostToDevice, s));
      M.d_count = A.alloc<unsigned long long>(n);
      M.d_stats = A.alloc<int>(static_cast<size_t>(n) * kTileStats);
      launch_tile_cells(M.m.rnum, M.m.r_stride, dt, n, M.d_count, M.d_stats, s);
      M.h_count = H.alloc<unsigned long long>(n);
      M.h_stats = H.alloc<int>(static_cast<size_t>(n) * kTileStats);
      R3D_CUDA(cudaMemcpyAsync(M.h_count, M.d_count, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost, s));
      R3D_CUDA(cudaMemcpyAsync(M.h_stats, M.d_stats, sizeof(int) * n * kTileStats, cudaMemcpyDeviceToHost, s));
    }
  };
  plan(P.left, wl);
  if (P.has_right) plan(P.right, wr);
}

// After the counts arrived: apply the reference's tile-size halving rule
// (stereo_matcher.cpp:643-648) and fix every tile's cell count and max label
// count. Returns false when a ranged match must be recounted.
bool finalize_layout(Match& M, int W, int H_, int partner_w, const r3dgpu_stereo_options& o, Arena& A, Pinned& HP,
                     cudaStream_t s) {
  const size_t n = M.layout.tiles.size();
  M.tile_cells.resize(n);
  M.tile_maxnum.resize(n);
  M.tile_width.assign(n, 0);
  M.tile_over32.assign(n, 0);
  for (size_t i = 0; i < n; ++i) {
    const Tile& t = M.layout.tiles[i];
    if (M.ranged) {
      const int* st = M.h_stats + i * kTileStats;
      M.tile_cells[i] = M.h_count[i];
      M.tile_maxnum[i] = st[0];
      M.tile_over32[i] = st[1];
      M.tile_width[i] = sgm_ranged_width_for(st, static_cast<int64_t>(t.w) * t.h);
    } else {
      M.tile_cells[i] = static_cast<uint64_t>(t.w) * static_cast<uint64_t>(t.h) * static_cast<uint64_t>(M.m.nd);
      M.tile_maxnum[i] = M.m.nd;
    }
  }
  size_t maxb = 0;
  for (size_t i = 0; i < n; ++i)
    maxb = std::max(maxb, estimated_tile_bytes(M.tile_cells[i], M.layout.tiles[i], static_cast<size_t>(partner_w)));
  if (M.tile_size > 64 && maxb > o.memory_budget) {
    M.tile_size /= 2;
    M.layout = make_layout(W, H_, M.tile_size, o);
    if (M.ranged) {
      const int nn = static_cast<int>(M.layout.tiles.size());
      int4* ht = HP.alloc<int4>(nn);
      for (int i = 0; i < nn; ++i) {
        const Tile& t = M.layout.tiles[i];
        ht[i] = make_int4(t.x0, t.y0, t.w, t.h);
      }
      int4* dt = A.alloc<int4>(nn);
      R3D_CUDA(cudaMemcpyAsync(dt, ht, sizeof(int4) * nn, cudaMemcpyHostToDevice, s));
      M.d_count = A.alloc<unsigned long long>(nn);
      M.d_stats = A.alloc<int>(static_cast<size_t>(nn) * kTileStats);
      launch_tile_cells(M.m.rnum, M.m.r_stride, dt, nn, M.d_count, M.d_stats, s);
      M.h_count = HP.alloc<unsigned long long>(nn);
      M.h_stats = HP.alloc<int>(static_cast<size_t>(nn) * kTileStats);
      R3D_CUDA(cudaMemcpyAsync(M.h_count, M.d_count, sizeof(unsigned long long) * nn, cudaMemcpyDeviceToHost, s));
      R3D_CUDA(cudaMemcpyAsync(M.h_stats, M.d_stats, sizeof(int) * nn * kTileStats, cudaMemcpyDeviceToHost, s));
      return false;
    }
    return finalize_layout(M, W, H_, partner_w, o, A, HP, s);
  }
  for (size_t i = 0; i < n; ++i)
    if (M.tile_cells[i] >= (uint64_t{1} << 31))
      fail(R3DGPU_EUNSUPPORTED, "stereo: a tile has 2^31 or more labels; use a smaller tile_size");
  return true;
}

// Stage 3 of a level: blending, left-right check(s), filters.
void finish_level(PairRun& P, Arena& A, Pinned& H, cudaStream_t s) {
  const int l = P.cur;
  const LevelIn& in = P.lv[l];
  const r3dgpu_stereo_options& o = P.o;
  const int wl = in.left.w, wr = in.right.w, h = in.left.h;
  auto blend = [&](Match& M, int W, bool mirror_out, float offset, float* disp, float* conf) {
    const int n = static_cast<int>(M.layout.tiles.size());
    BlendTile* bt = H.alloc<BlendTile>(n);
    for (int i = 0; i < n; ++i) {
      const Tile& t = M.layout.tiles[i];
      bt[i] = BlendTile{t.x0, t.y0, t.w, t.h, t.c0x, t.c1x, t.c0y, t.c1y, M.tile_disp + M.tile_off[i],
                        M.tile_conf ? M.tile_conf + M.tile_off[i] : nullptr};
    }
    BlendTile* d = A.alloc<BlendTile>(n);
    R3D_CUDA(cudaMemcpyAsync(d, bt, sizeof(BlendTile) * n, cudaMemcpyHostToDevice, s));
    launch_blend(d, n, M.layout.tiles_x, nullptr, nullptr, W, h, o.tile_blend, mirror_out ? 1 : 0, offset, disp, conf,
                 W, s);
  };
  P.disp_l = A.alloc<float>(static_cast<size_t>(wl) * h);
  P.conf_l = A.alloc<float>(static_cast<size_t>(wl) * h);
  blend(P.left, wl, false, 0.0F, P.disp_l, P.conf_l);
  const bool need_right = P.lr_full && l > 0;
  const int speckle = o.speckle_size >> (2 * l);
  int* uf = nullptr;
  auto post_filter = [&](float*& d, int W) {
    if (speckle > 1) {
      if (!uf) uf = A.alloc<int>(2 * static_cast<size_t>(std::max(wl, wr)) * h);
      launch_remove_speckles(d, W, h, speckle, o.speckle_diff, uf, s);
    }
    if (o.median) {
      float* m = A.alloc<float>(static_cast<size_t>(W) * h);
      launch_median3x3(d, W, h, m, s);
      d = m;
    }
  };
  if (P.has_right) {
    P.disp_r = A.alloc<float>(static_cast<size_t>(wr) * h);
    blend(P.right, wr, true, static_cast<float>(wr - wl), P.disp_r, nullptr);
    uint8_t* bad_l = A.alloc<uint8_t>(static_cast<size_t>(wl) * h);
    if (need_right) {
      uint8_t* bad_r = A.alloc<uint8_t>(static_cast<size_t>(wr) * h);
      launch_lr_check(P.disp_r, P.disp_l, wr, h, wl, +1, o.lr_max_diff, bad_r, s);
      launch_lr_check(P.disp_l, P.disp_r, wl, h, wr, -1, o.lr_max_diff, bad_l, s);
      launch_apply_bad(P.disp_l, bad_l, static_cast<int64_t>(wl) * h, s);
      launch_apply_bad(P.disp_r, bad_r, static_cast<int64_t>(wr) * h, s);
      post_filter(P.disp_r, wr);
    } else {
      launch_lr_check(P.disp_l, P.disp_r, wl, h, wr, -1, o.lr_max_diff, bad_l, s);
      launch_apply_bad(P.disp_l, bad_l, static_cast<int64_t>(wl) * h, s);
    }
  }
  post_filter(P.disp_l, wl);
  P.coarse_left = P.disp_l;
  P.coarse_wl = wl;
  P.coarse_h = h;
  if (need_right) {
    P.coarse_right = P.disp_r;
    P.coarse_wr = wr;
  } else {
    P.coarse_right = nullptr;
  }
}

// Waves of the tiles of a round for the chain passes (full-range tiles, or
// with `ranged` the tiles with per-pixel ranges): tiles in order of kernel
// shape, a new wave whenever the next tile would take the wave's buffers past
// `cap_bytes` (a tile larger than that gets a wave of its own). The job
// tables are copied to the device on s; `max_bytes` receives the largest
// wave's buffer size.
void plan_path_waves(const std::vector<std::pair<int, int>>& tiles, const std::vector<Match*>& matches, bool ranged,
                     size_t cap_bytes, int sms, Arena& A, Pinned& H, cudaStream_t s,
                     std::vector<SgmPathRangedWave>& waves, std::vector<std::vector<SgmPathSegment>>& segs,
                     size_t& max_bytes, uint64_t& cells_sum, uint64_t& px_sum) {
  struct Entry {
    int i, t;
    SgmPathShape sh;
    int64_t cells, px, keys, rows;
    int maxnum;
  };
  std::vector<Entry> es;
  es.reserve(tiles.size());
  for (const auto& mt : tiles) {
    const Match& M = *matches[mt.first];
    const Tile& T = M.layout.tiles[mt.second];
    const int64_t px = static_cast<int64_t>(T.w) * T.h;
    const SgmPathShape sh = ranged ? sgm_path_ranged_shape(M.tile_over32[mt.second], px) : sgm_path_shape(M.m.nd);
    es.push_back(Entry{mt.first, mt.second, sh, static_cast<int64_t>(M.tile_cells[mt.second]), px,
                       M.m.diagonal_lr ? static_cast<int64_t>(T.h) * (T.w + M.m.nd) : 0, T.h,
                       M.tile_maxnum[mt.second]});
  }
  // Waves keep byte terms when every match of the group allows them (all
  // P2 <= 255); otherwise u16 sums only. Ranged groups take byte terms when
  // all their tiles fit one wave with them (10 bytes per cell held against
  // 3): a single hierarchical pair's level runs about twice as fast, while
  // a large batch level split into more waves measured no faster beside the
  // single-level track. R3DGPU_RANGED_TERMS=0 or 1 forces either.
  bool terms = true;
  for (const auto& mt : tiles) terms = terms && matches[mt.first]->m.term_u8 != 0;
  if (ranged && terms) {
    const char* rt = std::getenv("R3DGPU_RANGED_TERMS");
    if (rt != nullptr && *rt != '\0') {
      terms = std::atoi(rt) == 1;
    } else {
      int64_t c = 0, p = 0, k = 0, r = 0;
      int mx = 16;
      for (const Entry& e : es) {
        c += e.cells;
        p += e.px;
        k += e.keys;
        r += e.rows;
        mx = std::max(mx, e.maxnum);
      }
      terms = sgm_path_ranged_buffers(c, p, k, r, mx, sms, true).total <= cap_bytes;
    }
  }
  auto bytes = [&](int64_t cells, int64_t px, int64_t keys, int64_t rows, int maxnum) -> size_t {
    return ranged ? sgm_path_ranged_buffers(cells, px, keys, rows, maxnum, sms, terms).total
                  : sgm_path_buffers(cells, px, keys, terms).total;
  };
  std::stable_sort(es.begin(), es.end(),
                   [](const Entry& a, const Entry& b) { return a.sh.g_ * a.sh.k_ < b.sh.g_ * b.sh.k_; });
  max_bytes = 0;
  cells_sum = 0;
  px_sum = 0;
  waves.clear();
  segs.clear();
  size_t begin = 0;
  while (begin < es.size()) {
    int64_t cells = 0, px = 0, keys = 0, rows = 0;
    int maxnum = 16, span = 0;
    size_t end = begin;
    while (end < es.size()) {
      const Entry& e = es[end];
      if (end > begin &&
          bytes(cells + e.cells, px + e.px, keys + e.keys, rows + e.rows, std::max(maxnum, e.maxnum)) > cap_bytes)
        break;
      cells += e.cells;
      px += e.px;
      keys += e.keys;
      rows += e.rows;
      maxnum = std::max(maxnum, e.maxnum);
      span = std::max(span, matches[e.i]->layout.tiles[e.t].w + matches[e.i]->m.nd - 1);
      ++end;
    }
    const int n = static_cast<int>(end - begin);
    SgmPathJob* hj = H.alloc<SgmPathJob>(n);
    std::vector<SgmPathSegment> sg;
    int64_t co = 0, po = 0, ko = 0, ro = 0;
    for (int q = 0; q < n; ++q) {
      const Entry& e = es[begin + q];
      if (sg.empty() || sg.back().shape.g_ != e.sh.g_ || sg.back().shape.k_ != e.sh.k_)
        sg.push_back(SgmPathSegment{e.sh, q, 0, {0, 0, 0}, 0, 0, 1});
      SgmPathSegment& g = sg.back();
      g.cells += e.cells;
      g.pixels += e.px;
      Match& M = *matches[e.i];
      g.full = g.full != 0 && !ranged && M.m.nd == 2 * e.sh.g_ * e.sh.k_ ? 1 : 0;
      const Tile& T = M.layout.tiles[e.t];
      SgmPathJob& J = hj[q];
      J = SgmPathJob{};
      J.match = e.i;
      J.x0 = T.x0;
      J.y0 = T.y0;
      J.w = T.w;
      J.h = T.h;
      J.cell_off = co;
      J.px_off = po;
      J.rk_off = ko;
      J.row_off = ro;
      const int cpw = 32 / e.sh.g_;
      for (int c = 0; c < kPathClasses; ++c) {
        J.blk[c] = g.blocks[c];
        g.blocks[c] += (sgm_path_chains(c, T.w, T.h) + cpw - 1) / cpw;
      }
      J.disp = M.tile_disp + M.tile_off[e.t];
      J.conf = M.tile_conf ? M.tile_conf + M.tile_off[e.t] : nullptr;
      J.cells = M.d_cells + e.t;
      J.volume = nullptr;
      ++g.count;
      co += e.cells;
      po += e.px;
      ko += e.keys;
      ro += e.rows;
    }
    SgmPathJob* dj = A.alloc<SgmPathJob>(n);
    R3D_CUDA(cudaMemcpyAsync(dj, hj, sizeof(SgmPathJob) * n, cudaMemcpyHostToDevice, s));
    SgmPathRangedWave wv{};
    wv.jobs = dj;
    wv.njobs = n;
    wv.cells = co;
    wv.pixels = po;
    wv.keys = ko;
    wv.rows = ro;
    wv.maxnum = maxnum;
    wv.terms = terms ? 1 : 0;
    wv.max_span = span;
    waves.push_back(wv);
    segs.push_back(std::move(sg));
    max_bytes = std::max(max_bytes, bytes(co, po, ko, ro, maxnum));
    cells_sum += static_cast<uint64_t>(co);
    px_sum += static_cast<uint64_t>(po);
    begin = end;
  }
}

// A batch whose work is enqueued: what finish_batch completes once the
// stream has run it.
struct BatchRun {
  Workspace* W = nullptr;
  std::vector<PairRun> runs;
};

// Enqueues the whole matching of a batch of pairs on stream s, using the
// workspace `slot` of this thread. Host synchronisations happen only where
// ranged tiles need their label statistics.
BatchRun enqueue_batch(r3dgpu_pair* pairs, int count, cudaStream_t s, int slot) {
  BatchRun B;
  Workspace& W = workspace(slot);
  B.W = &W;
  W.arena.reset();
  W.pinned.reset();
  Arena& A = W.arena;
  Pinned& H = W.pinned;
  std::vector<PairRun>& runs = B.runs;
  runs.resize(count);
  int max_levels = 0;
  for (int i = 0; i < count; ++i) {
    validate_pair(pairs[i]);
    PairRun& P = runs[i];
    P.req = &pairs[i];
    P.o = pairs[i].options;
    P.levels = P.o.levels >= 0 ? P.o.levels
                               : automatic_levels(pairs[i].left.width, pairs[i].left.height, pairs[i].num_disparities);
    P.check_lr = P.o.lr_max_diff >= 0;
    P.lr_full = P.check_lr && P.o.lr_full_match != 0;
    max_levels = std::max(max_levels, P.levels);
  }
  for (auto& P : runs) build_levels(P, A, s);

  for (int round = 0; round <= max_levels; ++round) {
    check_cancel();
    std::vector<PairRun*> active;
    // Round r runs level max_levels - r of every pair that has it, so that
    // all pairs reach level 0 (the largest) in the last round, where their
    // SGM launches overlap. (Spreading single-level pairs over the earlier
    // rounds measured slower: every round costs at least its slowest tile.)
    for (auto& P : runs) {
      const int l = max_levels - round;
      if (l <= P.levels) {
        P.cur = l;
        active.push_back(&P);
      }
    }
    // Stage 1.
    bool any_ranged = false;
    for (PairRun* P : active) {
      prepare_level(*P, A, H, s);
      any_ranged = any_ranged || P->left.ranged || (P->has_right && P->right.ranged);
    }
    if (any_ranged) R3D_CUDA(cudaStreamSynchronize(s));
    // Tile sizes and counts.
    while (true) {
      bool again = false;
      for (PairRun* P : active) {
        const LevelIn& in = P->lv[P->cur];
        if (!finalize_layout(P->left, in.left.w, in.left.h, in.right.w, P->o, A, H, s)) again = true;
        if (P->has_right && !finalize_layout(P->right, in.right.w, in.right.h, in.left.w, P->o, A, H, s)) again = true;
      }
      if (!again) break;
      R3D_CUDA(cudaStreamSynchronize(s));
    }
    // Stage 2: SGM launches. Full-range matches go to the full-range kernel,
    // one launch per label-count shape; ranged matches to the general kernel.
    std::vector<Match*> matches;
    for (PairRun* P : active) {
      matches.push_back(&P->left);
      if (P->has_right) matches.push_back(&P->right);
    }
    const int nm = static_cast<int>(matches.size());
    SgmMatch* hm = H.alloc<SgmMatch>(nm);
    for (int i = 0; i < nm; ++i) {
      hm[i] = matches[i]->m;
      Match& M = *matches[i];
      const int n = static_cast<int>(M.layout.tiles.size());
      size_t px_total = 0;
      M.tile_off.resize(n);
      for (int t = 0; t < n; ++t) {
        M.tile_off[t] = px_total;
        px_total += static_cast<size_t>(M.layout.tiles[t].w) * M.layout.tiles[t].h;
      }
      M.tile_disp = A.alloc<float>(px_total);
      M.tile_conf = M.m.confidence ? A.alloc<float>(px_total) : nullptr;
      M.d_cells = A.alloc<unsigned long long>(n);
    }
    SgmMatch* dm = A.alloc<SgmMatch>(nm);
    R3D_CUDA(cudaMemcpyAsync(dm, hm, sizeof(SgmMatch) * nm, cudaMemcpyHostToDevice, s));
    // Launch groups: full-range matches by label count; ranged tiles by the
    // kernel shape chosen for each tile (or all into the general kernel).
    enum Kind { kFull, kRanged, kGeneral, kPath, kPathRanged };
    struct Group {
      Kind kind;
      SgmFullPlan plan;
      int nd;     // full: label count; ranged: shape width
      std::vector<std::pair<int, int>> tiles;  // (match, tile)
    };
    std::vector<Group> groups;
    auto group_for = [&](Kind kind, int key, SgmFullPlan plan) -> Group& {
      for (auto& q : groups)
        if (q.kind == kind && q.nd == key) return q;
      groups.push_back(Group{kind, plan, key, {}});
      return groups.back();
    };
    for (int i = 0; i < nm; ++i) {
      const Match& M = *matches[i];
      const int nt = static_cast<int>(M.layout.tiles.size());
      if (!M.ranged) {
        // Full-range tiles of every label count: the chain passes, one group.
        bool fits = true;
        for (int t = 0; t < nt; ++t) fits = fits && sgm_path_fits(M.layout.tiles[t].w, M.m.nd);
        if (sgm_path_enabled() && sgm_path_shape(M.m.nd).g_ != 0 && fits) {
          Group& g = group_for(kPath, 0, SgmFullPlan{{0, 0}, 0});
          for (int t = 0; t < nt; ++t) g.tiles.emplace_back(i, t);
          continue;
        }
        const SgmFullPlan plan = sgm_full_plan(M.m.nd, W.smem_optin);
        if (plan.shape.g_ != 0) {
          Group& g = group_for(kFull, M.m.nd, plan);
          for (int t = 0; t < nt; ++t) g.tiles.emplace_back(i, t);
          continue;
        }
      }
      if (M.ranged && sgm_path_ranged_enabled()) {
        Group& g = group_for(kPathRanged, 0, SgmFullPlan{{0, 0}, 0});
        for (int t = 0; t < nt; ++t) g.tiles.emplace_back(i, t);
        continue;
      }
      const int gw = general_width();
      for (int t = 0; t < nt; ++t) {
        if (M.ranged && !general_ranged_kernel() && M.tile_width[t] < gw)
          group_for(kRanged, M.tile_width[t], SgmFullPlan{{0, 0}, 0}).tiles.emplace_back(i, t);
        else
          group_for(kGeneral, 0, SgmFullPlan{{0, 0}, 0}).tiles.emplace_back(i, t);
      }
    }
    // Plan every group's launch: jobs (largest tiles first), scratch slot,
    // CTAs per SM, and an estimate of its slowest tile (a CTA runs a tile
    // alone: band steps x per-step cost).
    struct Launch {
      const Group* g;
      int njobs, rows, ndw, maxc, per_sm, grid, smem;
      SgmRangedPlan rplan;
      SgmJob* dj;
      size_t slot_bytes, scratch_off;
      uint64_t cells_sum, px_sum;
      double longest;
      // kPath, kPathRanged: the waves (one buffer of slot_bytes, reused wave after wave)
      std::vector<SgmPathRangedWave> waves;
      std::vector<std::vector<SgmPathSegment>> segs;
    };
    std::vector<Launch> launches;
    const size_t round_budget = t_scratch_budget != 0 ? t_scratch_budget : size_t{64} << 30;
    for (const Group& g : groups) {
      Launch L{};
      L.g = &g;
      if (g.kind == kPath || g.kind == kPathRanged) {
        // Waves up to half the budget (fewer, longer pass launches with more
        // chains in flight); a round has at most one group of each kind.
        plan_path_waves(g.tiles, matches, g.kind == kPathRanged, round_budget / 2, W.sms, A, H, s, L.waves, L.segs,
                        L.slot_bytes, L.cells_sum, L.px_sum);
        L.njobs = static_cast<int>(g.tiles.size());
        L.grid = 1;
        L.longest = 1e300;  // first: the largest share of the round's work
        launches.push_back(std::move(L));
        continue;
      }
      L.njobs = static_cast<int>(g.tiles.size());
      int max_num = 16;
      for (const auto& mt : g.tiles) max_num = std::max(max_num, matches[mt.first]->tile_maxnum[mt.second]);
      const bool full = g.kind == kFull, ranged = g.kind == kRanged;
      L.rplan = ranged ? sgm_ranged_plan(sgm_ranged_shape_for_width(g.nd), W.smem_optin) : SgmRangedPlan{{0, 0}, 0};
      L.ndw = ranged ? sgm_ranged_ndw(L.rplan.shape, max_num) : 0;
      L.maxc = g.kind == kGeneral ? sgm_maxc_for(max_num) : 0;
      L.rows = full ? g.plan.rows : (ranged ? L.rplan.rows : sgm_rows_for(L.maxc, W.smem_optin));
      const int kk = full ? g.plan.shape.k_ : (ranged ? L.rplan.shape.k_ : 2 * L.maxc);
      SgmJob* hj = H.alloc<SgmJob>(L.njobs);
      std::vector<double> work(L.njobs);
      int jb = 0;
      for (const auto& mt : g.tiles) {
        const int i = mt.first, t = mt.second;
        Match& M = *matches[i];
        const Tile& T = M.layout.tiles[t];
        SgmJob& J = hj[jb];
        J = SgmJob{};
        J.match = i;
        J.x0 = T.x0;
        J.y0 = T.y0;
        J.w = T.w;
        J.h = T.h;
        J.disp = M.tile_disp + M.tile_off[t];
        J.conf = M.tile_conf ? M.tile_conf + M.tile_off[t] : nullptr;
        J.cells = M.d_cells + t;
        // Barrier steps of both passes: the full-range and ranged kernels chain
        // a tile's bands (period max(w, 2 rows + 2)); the general kernel fills
        // and drains every band.
        const int nbands = (T.h + L.rows - 1) / L.rows;
        const double steps =
            (full || ranged)
                ? 2.0 * ((nbands - 1.0) * std::max(T.w, 2 * L.rows + 2) + T.w + 2.0 * (T.h - (nbands - 1) * L.rows - 1))
                : 2.0 * nbands * (T.w + 2.0 * (L.rows - 1));
        work[jb] = steps * (1.0 + kk / 4.0) + static_cast<double>(M.tile_cells[t]) / 256.0;
        L.longest = std::max(L.longest, work[jb]);
        L.cells_sum += M.tile_cells[t];
        L.px_sum += static_cast<uint64_t>(T.w) * T.h;
        L.slot_bytes = std::max(
            L.slot_bytes, full ? sgm_full_slot_layout(T.w, T.h, M.m.nd, 2 * g.plan.shape.g_ * g.plan.shape.k_).total
                          : ranged ? sgm_ranged_slot_layout(T.w, T.h, M.tile_cells[t], M.m.nd, L.ndw, L.rows).total
                                   : sgm_slot_layout(T.w, T.h, M.tile_cells[t], L.maxc, M.m.nd).total);
        ++jb;
      }
      {
        std::vector<int> order(L.njobs);
        for (int i = 0; i < L.njobs; ++i) order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return work[x] > work[y]; });
        std::vector<SgmJob> tmp(hj, hj + L.njobs);
        for (int i = 0; i < L.njobs; ++i) hj[i] = tmp[order[i]];
      }
      L.dj = A.alloc<SgmJob>(L.njobs);
      R3D_CUDA(cudaMemcpyAsync(L.dj, hj, sizeof(SgmJob) * L.njobs, cudaMemcpyHostToDevice, s));
      L.smem = full ? sgm_full_smem(g.plan.shape, L.rows)
               : ranged ? sgm_ranged_smem(L.rplan.shape, L.rows)
                        : sgm_smem_layout(L.maxc, L.rows).total;
      L.per_sm = std::max(1, std::min(4, (W.smem_optin + 1024) / (L.smem + 1024)));
      L.grid = std::max(1, std::min(L.njobs, W.sms * L.per_sm));
      L.slot_bytes = sgm_align16(L.slot_bytes);
      launches.push_back(L);
    }
    // Scratch for all groups at once, within the budget: grids shrink in
    // proportion when the slots would not fit.
    {
      const size_t budget = round_budget;
      size_t total = 0;
      for (const Launch& L : launches) total += static_cast<size_t>(L.grid) * L.slot_bytes;
      if (total > budget) {
        const double f = static_cast<double>(budget) / static_cast<double>(total);
        total = 0;
        for (Launch& L : launches) {
          L.grid = std::max(1, static_cast<int>(L.grid * f));
          total += static_cast<size_t>(L.grid) * L.slot_bytes;
        }
      }
      size_t off = 0;
      for (Launch& L : launches) {
        L.scratch_off = off;
        off += static_cast<size_t>(L.grid) * L.slot_bytes;
      }
      W.scratch.reserve(off);
      if (static_cast<int>(W.counter.size()) < static_cast<int>(launches.size())) W.counter.reset(launches.size());
      R3D_CUDA(cudaMemsetAsync(W.counter.get(), 0, sizeof(int) * launches.size(), s));
    }
    // Slowest tiles first: each group on its own stream, forked from and
    // joined into the call's stream, so that one group's last tiles overlap
    // the other groups' work.
    std::vector<int> lorder(launches.size());
    for (size_t i = 0; i < launches.size(); ++i) lorder[i] = static_cast<int>(i);
    std::stable_sort(lorder.begin(), lorder.end(),
                     [&](int x, int y) { return launches[x].longest > launches[y].longest; });
    const int nside = std::min<int>(static_cast<int>(launches.size()), 16);
    W.ensure_side(nside);
    ProfileState::Pending span{};
    if (t_prof.on) {
      R3D_CUDA(cudaEventCreate(&span.a));
      R3D_CUDA(cudaEventCreate(&span.b));
      R3D_CUDA(cudaEventRecord(span.a, s));
      span.span = true;
    }
    R3D_CUDA(cudaEventRecord(W.fork, s));
    for (int j = 0; j < nside; ++j) R3D_CUDA(cudaStreamWaitEvent(W.side[j], W.fork, 0));
    for (size_t q = 0; q < lorder.size(); ++q) {
      const int li = lorder[q];
      const Launch& L = launches[li];
      const Group& g = *L.g;
      cudaStream_t gs = W.side[q % nside];
      unsigned char* scratch = W.scratch.get() + L.scratch_off;
      int* counter = W.counter.get() + li;
      ProfileState::Pending ev{};
      if (t_prof.on) {
        R3D_CUDA(cudaEventCreate(&ev.a));
        R3D_CUDA(cudaEventCreate(&ev.b));
        R3D_CUDA(cudaEventRecord(ev.a, gs));
      }
      if (g.kind == kPath) {
        for (size_t k = 0; k < L.waves.size(); ++k) {
          check_cancel();
          const SgmPathRangedWave& rw = L.waves[k];
          SgmPathWave w{};
          w.cancel = cancel_device_flag();
          w.jobs = rw.jobs;
          w.njobs = rw.njobs;
          w.segs = L.segs[k].data();
          w.nsegs = static_cast<int>(L.segs[k].size());
          w.cells = rw.cells;
          w.pixels = rw.pixels;
          w.keys = rw.keys;
          w.rows = rw.rows;
          w.buffer = scratch;
          w.terms = rw.terms;
          w.max_span = rw.max_span;
          launch_sgm_path_wave(dm, w, W.sms, gs);
        }
      } else if (g.kind == kPathRanged) {
        for (size_t k = 0; k < L.waves.size(); ++k) {
          check_cancel();
          SgmPathRangedWave w = L.waves[k];
          w.cancel = cancel_device_flag();
          w.segs = L.segs[k].data();
          w.nsegs = static_cast<int>(L.segs[k].size());
          w.buffer = scratch;
          launch_sgm_path_ranged_wave(dm, w, W.sms, gs);
        }
      } else if (g.kind == kFull) {
        launch_sgm_full(g.plan.shape, g.nd, dm, L.dj, L.njobs, L.rows, L.grid, scratch, L.slot_bytes, counter, gs);
      } else if (g.kind == kRanged) {
        launch_sgm_ranged(L.rplan.shape, dm, L.dj, L.njobs, L.rows, L.ndw, L.grid, scratch, L.slot_bytes, counter, gs);
      } else {
        launch_sgm(dm, L.dj, L.njobs, L.maxc, L.rows, L.grid, scratch, L.slot_bytes, counter, gs);
      }
      if (t_prof.on) {
        R3D_CUDA(cudaEventRecord(ev.b, gs));
        ev.cells = L.cells_sum;
        ev.pixels = L.px_sum;
        ev.tiles = static_cast<uint64_t>(L.njobs);
        ev.kernel = g.kind == kPath         ? "sgm_path_kernel"
                    : g.kind == kPathRanged ? "sgm_path_ranged_kernel"
                    : g.kind == kFull       ? "sgm_full_kernel"
                                      : (g.kind == kRanged ? "sgm_ranged_kernel" : "sgm_tile_kernel");
        ev.shape = (g.kind == kPath || g.kind == kPathRanged) ? "waves" + std::to_string(L.waves.size())
                   : g.kind == kFull ? std::to_string(g.plan.shape.g_) + "x" + std::to_string(g.plan.shape.k_) + "/nd" +
                                         std::to_string(g.nd)
                   : g.kind == kRanged ? std::to_string(L.rplan.shape.g_) + "x" + std::to_string(L.rplan.shape.k_) +
                                             "/ndw" + std::to_string(L.ndw)
                                       : "maxc" + std::to_string(L.maxc);
        ev.grid = L.grid;
        ev.rows = L.rows;
        t_prof.pending.push_back(ev);
      }
    }
    for (int j = 0; j < nside; ++j) {
      R3D_CUDA(cudaEventRecord(W.side_done[j], W.side[j]));
      R3D_CUDA(cudaStreamWaitEvent(s, W.side_done[j], 0));
    }
    if (t_prof.on) {
      R3D_CUDA(cudaEventRecord(span.b, s));
      span.kernel = "sgm_round";
      t_prof.pending.push_back(span);
    }
    // Stage 3.
    for (PairRun* P : active) {
      P->cell_arrays.push_back(P->left.d_cells);
      P->cell_counts.push_back(static_cast<int>(P->left.layout.tiles.size()));
      if (P->has_right) {
        P->cell_arrays.push_back(P->right.d_cells);
        P->cell_counts.push_back(static_cast<int>(P->right.layout.tiles.size()));
      }
      finish_level(*P, A, H, s);
    }
  }
  // Outputs and cell counts.
  for (auto& P : runs) {
    r3dgpu_disparity_map& out = const_cast<r3dgpu_pair*>(P.req)->out;
    const int wl = P.lv[0].left.w, h = P.lv[0].left.h;
    launch_copy2d_f32(P.coarse_left, wl, wl, h, out.disparity, out.stride, s);
    if (out.confidence) launch_copy2d_f32(P.conf_l, wl, wl, h, out.confidence, out.stride, s);
    for (size_t k = 0; k < P.cell_arrays.size(); ++k) {
      unsigned long long* hc = H.alloc<unsigned long long>(P.cell_counts[k]);
      R3D_CUDA(cudaMemcpyAsync(hc, P.cell_arrays[k], sizeof(unsigned long long) * P.cell_counts[k],
                               cudaMemcpyDeviceToHost, s));
      P.h_cell_arrays.push_back(hc);
    }
  }
  return B;
}

// After the stream ran an enqueued batch: cell counts and output metadata.
void finish_batch(BatchRun& B) {
  B.W->pinned.release_retired();
  for (auto& P : B.runs) {
    uint64_t cells = 0;
    for (size_t k = 0; k < P.h_cell_arrays.size(); ++k)
      for (int t = 0; t < P.cell_counts[k]; ++t) cells += P.h_cell_arrays[k][t];
    r3dgpu_disparity_map& out = const_cast<r3dgpu_pair*>(P.req)->out;
    out.disparity_min = P.req->disparity_min;
    out.num_disparities = align16(P.req->num_disparities);
    out.levels = P.levels;
    out.cells = cells;
  }
}

// Whether a batch that mixes single-level and hierarchical pairs runs them
// as two concurrent tracks (default; R3DGPU_BATCH_TRACKS=1 runs one).
bool batch_tracks_enabled() {
  const char* e = std::getenv("R3DGPU_BATCH_TRACKS");
  return e == nullptr || std::atoi(e) != 1;
}

#ifndef R3DGPU_SIMT_EMULATION
// The single-level track of a two-track batch as a CUDA graph. The track
// enqueues without any host synchronisation (its layouts depend on sizes and
// options only), so its whole enqueue -- job tables copied from pinned host
// memory, every launch on the track and side streams, the cell counts copied
// back -- is captured once per batch description and replayed while the same
// description comes again: the same pairs (buffers, sizes, options; not
// their output fields), device, cancellation flag, scratch budget and kernel
// selection. Between replays nothing else uses the track's workspace (slot
// 1), so the captured pinned tables and device buffers stay as captured.
// R3DGPU_GRAPH=0 enqueues the track on every call.
struct TrackGraph {
  std::string key;
  cudaGraphExec_t exec = nullptr;
  BatchRun run;
  uint64_t launches = 0;
  std::vector<unsigned char*> pinned;  // pinned blocks the graph copies from, replaced during its capture
  void clear() {
    if (exec != nullptr) cudaGraphExecDestroy(exec);
    exec = nullptr;
    for (unsigned char* p : pinned) cudaFreeHost(p);
    pinned.clear();
    key.clear();
  }
  ~TrackGraph() { clear(); }
};
thread_local std::vector<std::unique_ptr<TrackGraph>> t_track_graphs;

bool track_graph_enabled() {
  const char* e = std::getenv("R3DGPU_GRAPH");
  return !t_prof.on && (e == nullptr || std::atoi(e) != 0);
}

std::string track_key(const std::vector<r3dgpu_pair>& fp) {
  std::string k;
  for (r3dgpu_pair p : fp) {
    p.out.disparity_min = 0;
    p.out.num_disparities = 0;
    p.out.levels = 0;
    p.out.reserved = 0;
    p.out.cells = 0;
    k.append(reinterpret_cast<const char*>(&p), sizeof(p));
  }
  const int* c = cancel_device_flag();
  k.append(reinterpret_cast<const char*>(&c), sizeof(c));
  k.append(reinterpret_cast<const char*>(&t_device), sizeof(t_device));
  k.append(reinterpret_cast<const char*>(&t_scratch_budget), sizeof(t_scratch_budget));
  // Every environment setting that selects kernels or launch shapes (a
  // captured graph replays the launches it was captured with).
  for (const char* name :
       {"R3DGPU_FULL_KERNEL", "R3DGPU_RANGED_KERNEL", "R3DGPU_RANGED_GENERAL_WIDTH", "R3DGPU_TUNING",
        "R3DGPU_TUNING_FILE", "R3DGPU_PATH_SHAPE", "R3DGPU_RANGED_TERMS", "R3DGPU_FULL_ROWS", "R3DGPU_FULL_SHAPE",
        "R3DGPU_RANGED_ROWS", "R3DGPU_RANGED_SHAPE", "R3DGPU_RANGED_WIDE_FRAC"}) {
    const char* v = std::getenv(name);
    k += v != nullptr ? v : "";
    k += '\n';
  }
  return k;
}

TrackGraph& track_graph() {
  const int idx = t_device;
  if (static_cast<int>(t_track_graphs.size()) <= idx) t_track_graphs.resize(idx + 1);
  if (!t_track_graphs[idx]) t_track_graphs[idx] = std::make_unique<TrackGraph>();
  return *t_track_graphs[idx];
}

// Enqueues the single-level track on `track`: the captured graph of the same
// description, or a fresh capture of enqueue_batch.
BatchRun enqueue_track(std::vector<r3dgpu_pair>& fp, cudaStream_t track) {
  TrackGraph& g = track_graph();
  std::string key = track_key(fp);
  if (g.exec == nullptr || g.key != key) {
    R3D_CUDA(cudaStreamSynchronize(track));  // a previous replay may still read the blocks freed here
    g.clear();
    const uint64_t l0 = launch_counter().load();
    R3D_CUDA(cudaStreamBeginCapture(track, cudaStreamCaptureModeRelaxed));
    BatchRun run;
    cudaGraph_t graph = nullptr;
    try {
      run = enqueue_batch(fp.data(), static_cast<int>(fp.size()), track, 1);
    } catch (...) {
      (void)cudaStreamEndCapture(track, &graph);
      if (graph != nullptr) (void)cudaGraphDestroy(graph);
      (void)cudaGetLastError();
      throw;
    }
    R3D_CUDA(cudaStreamEndCapture(track, &graph));
    g.pinned = run.W->pinned.take_retired();
    const cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
    (void)cudaGraphDestroy(graph);
    R3D_CUDA(e);
    g.launches = launch_counter().load() - l0;
    g.run = run;
    g.key = std::move(key);
  } else {
    launch_counter().fetch_add(g.launches, std::memory_order_relaxed);
  }
  R3D_CUDA(cudaGraphLaunch(g.exec, track));
  BatchRun run = g.run;
  for (size_t i = 0; i < run.runs.size(); ++i) run.runs[i].req = &fp[i];
  return run;
}
#endif

// Runs a batch of pairs to completion on stream s. The levels of a batch run
// in rounds (every pair's coarsest level first); when single-level pairs
// share the batch with hierarchical ones, the single-level pairs form a
// second track on their own stream and workspace, so that their matching
// overlaps the hierarchy's rounds instead of waiting for its last one.
void run_batch(r3dgpu_pair* pairs, int count, cudaStream_t s) {
  std::vector<int> flat, hier;
  for (int i = 0; i < count; ++i) {
    validate_pair(pairs[i]);
    const int lv = pairs[i].options.levels >= 0
                       ? pairs[i].options.levels
                       : automatic_levels(pairs[i].left.width, pairs[i].left.height, pairs[i].num_disparities);
    (lv == 0 ? flat : hier).push_back(i);
  }
  // On any error (a cancellation included) the work already enqueued ends
  // before the call returns: the call's stream, the second track's, and the
  // side streams of both workspaces (a round's SGM groups are forked onto
  // them, and an error between the fork and the join leaves them running;
  // the next call would reuse their buffers).
  auto drain = [&](cudaStream_t other) {
    (void)cudaStreamSynchronize(s);
    if (other != nullptr) (void)cudaStreamSynchronize(other);
    for (int slot = 0; slot < kWorkspaceSlots; ++slot) {
      const int idx = t_device * kWorkspaceSlots + slot;
      if (idx < static_cast<int>(t_workspaces.size()) && t_workspaces[idx])
        for (cudaStream_t side : t_workspaces[idx]->side) (void)cudaStreamSynchronize(side);
    }
    (void)cudaGetLastError();
    profile_collect();
  };
  if (flat.empty() || hier.empty() || !batch_tracks_enabled()) {
    BatchRun B;
    try {
      B = enqueue_batch(pairs, count, s, 0);
    } catch (...) {
      drain(nullptr);
      throw;
    }
    R3D_CUDA(cudaStreamSynchronize(s));
    profile_collect();
    check_cancel();
    finish_batch(B);
    return;
  }
  std::vector<r3dgpu_pair> fp, hp;
  for (int i : flat) fp.push_back(pairs[i]);
  for (int i : hier) hp.push_back(pairs[i]);
  // A scratch budget set for this thread (a server worker's) bounds both
  // tracks together: each track gets half of it.
  struct HalfBudget {
    size_t saved;
    HalfBudget() : saved(t_scratch_budget) { t_scratch_budget /= 2; }
    ~HalfBudget() { t_scratch_budget = saved; }
  } half_budget;
  Workspace& W1 = workspace(1);
  if (W1.track == nullptr) {
    R3D_CUDA(cudaStreamCreateWithFlags(&W1.track, cudaStreamNonBlocking));
    R3D_CUDA(cudaEventCreateWithFlags(&W1.track_start, cudaEventDisableTiming));
    R3D_CUDA(cudaEventCreateWithFlags(&W1.track_done, cudaEventDisableTiming));
  }
  R3D_CUDA(cudaEventRecord(W1.track_start, s));
  R3D_CUDA(cudaStreamWaitEvent(W1.track, W1.track_start, 0));
  BatchRun a, b;
  try {
#ifndef R3DGPU_SIMT_EMULATION
    if (track_graph_enabled())
      a = enqueue_track(fp, W1.track);
    else
#endif
      a = enqueue_batch(fp.data(), static_cast<int>(fp.size()), W1.track, 1);
    R3D_CUDA(cudaEventRecord(W1.track_done, W1.track));
    b = enqueue_batch(hp.data(), static_cast<int>(hp.size()), s, 0);
  } catch (...) {
    drain(W1.track);
    throw;
  }
  R3D_CUDA(cudaStreamWaitEvent(s, W1.track_done, 0));
  R3D_CUDA(cudaStreamSynchronize(s));
  profile_collect();
  check_cancel();
  finish_batch(a);
  finish_batch(b);
  for (size_t k = 0; k < flat.size(); ++k) pairs[flat[k]].out = fp[k].out;
  for (size_t k = 0; k < hier.size(); ++k) pairs[hier[k]].out = hp[k].out;
}

template <class F>
r3dgpu_status guarded(F&& f) {
  try {
    t_error.clear();
    f();
    return R3DGPU_OK;
  } catch (const Error& e) {
    t_error = e.what();
    return e.status;
  } catch (const std::bad_alloc&) {
    t_error = "r3dgpu: out of host memory";
    return R3DGPU_ENOMEM;
  } catch (const std::exception& e) {
    t_error = e.what();
    return R3DGPU_EDEVICE;
  }
}

// Host image -> device copy in the arena.
template <class T>
T* upload(Arena& A, const T* p, int w, int h, int64_t stride, cudaStream_t s) {
  T* d = A.alloc<T>(static_cast<size_t>(w) * h);
  R3D_CUDA(cudaMemcpy2DAsync(d, sizeof(T) * w, p, sizeof(T) * stride, sizeof(T) * w, h, cudaMemcpyHostToDevice, s));
  return d;
}

}  // namespace

void validate_request(const r3dgpu_pair& p) { validate_pair(p); }
void set_thread_scratch_budget(size_t bytes) { t_scratch_budget = bytes; }
void set_thread_error(const std::string& message) { t_error = message; }

}  // namespace r3dgpu

using namespace r3dgpu;

extern "C" {

const char* r3dgpu_last_error(void) { return t_error.c_str(); }

void r3dgpu_default_options(r3dgpu_stereo_options* o) {
  *o = r3dgpu_stereo_options{};
  o->p1 = 28;
  o->p2 = 200;
  o->p2_adapt = 4;
  o->invalid_cost = 31;
  o->subpixel = R3DGPU_SUBPIXEL_EQUIANGULAR;
  o->uniqueness = 0.0F;
  o->lr_max_diff = 1;
  o->lr_full_match = 1;
  o->speckle_size = 100;
  o->speckle_diff = 1.0F;
  o->median = 1;
  o->levels = -1;
  o->range_radius = 3;
  o->range_margin = 4;
  o->range_fill = 64;
  o->tile_size = 512;
  o->tile_margin = 32;
  o->tile_blend = 32;
  o->memory_budget = uint64_t{2} << 30;
  o->scalar_kernels = 0;
}

int32_t r3dgpu_automatic_levels(int32_t width, int32_t height, int32_t nd) { return automatic_levels(width, height, nd); }

r3dgpu_status r3dgpu_set_device(int32_t device) {
  return guarded([&] {
    if (device < 0) fail(R3DGPU_EINVAL, "r3dgpu: negative device index");
    t_device = device;
    (void)workspace();
  });
}

r3dgpu_status r3dgpu_cancel_token_create(r3dgpu_cancel_token** out) {
  return guarded([&] {
    if (out == nullptr) fail(R3DGPU_EINVAL, "cancel_token_create: null argument");
    (void)workspace();  // the thread's device, current
    auto* t = new r3dgpu_cancel_token();
    void* h = nullptr;
    void* d = nullptr;
    const cudaError_t e = cudaHostAlloc(&h, sizeof(int32_t), cudaHostAllocMapped);
    if (e != cudaSuccess) {
      delete t;
      cuda_check(e, "cancel_token_create: cudaHostAlloc");
    }
    *static_cast<int32_t*>(h) = 0;
    const cudaError_t e2 = cudaHostGetDevicePointer(&d, h, 0);
    if (e2 != cudaSuccess) {
      cudaFreeHost(h);
      delete t;
      cuda_check(e2, "cancel_token_create: cudaHostGetDevicePointer");
    }
    t->host = static_cast<int32_t*>(h);
    t->dev = static_cast<const int*>(d);
    *out = t;
  });
}

void r3dgpu_cancel_token_destroy(r3dgpu_cancel_token* token) {
  if (token == nullptr) return;
  if (t_cancel == token) t_cancel = nullptr;
  cudaFreeHost(token->host);
  delete token;
}

void r3dgpu_cancel(r3dgpu_cancel_token* token) {
  if (token != nullptr) __atomic_store_n(token->host, 1, __ATOMIC_SEQ_CST);
}

void r3dgpu_cancel_token_reset(r3dgpu_cancel_token* token) {
  if (token != nullptr) __atomic_store_n(token->host, 0, __ATOMIC_SEQ_CST);
}

int32_t r3dgpu_cancel_requested(const r3dgpu_cancel_token* token) {
  return token != nullptr ? __atomic_load_n(token->host, __ATOMIC_SEQ_CST) : 0;
}

void r3dgpu_set_cancel_token(r3dgpu_cancel_token* token) { t_cancel = token; }

r3dgpu_status r3dgpu_release_workspace(void) {
  return guarded([&] {
#ifndef R3DGPU_SIMT_EMULATION
    if (t_device < static_cast<int>(t_track_graphs.size())) t_track_graphs[t_device].reset();
#endif
    for (int slot = 0; slot < kWorkspaceSlots; ++slot) {
      const int idx = t_device * kWorkspaceSlots + slot;
      if (idx < static_cast<int>(t_workspaces.size()) && t_workspaces[idx]) {
        R3D_CUDA(cudaSetDevice(t_device));
        R3D_CUDA(cudaDeviceSynchronize());
        t_workspaces[idx].reset();
      }
    }
  });
}

uint64_t r3dgpu_launch_count(void) { return launch_counter().load(); }

void r3dgpu_profile_enable(int32_t on) { t_prof.on = on != 0; }

void r3dgpu_profile_take(r3dgpu_profile* out) {
  if (out) *out = t_prof.acc;
  t_prof.acc = r3dgpu_profile{};
  t_prof.last_launches = "[" + t_prof.launches + "]";
  t_prof.launches.clear();
}

uint64_t r3dgpu_profile_launches(char* buf, uint64_t len) {
  const std::string& s = t_prof.last_launches;
  if (buf && len > 0) {
    const size_t n = std::min<size_t>(s.size(), static_cast<size_t>(len - 1));
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
  }
  return s.size();
}

r3dgpu_status r3dgpu_match_stereo_batch(r3dgpu_pair* pairs, int32_t count, void* stream) {
  return guarded([&] {
    if (count < 0 || (count > 0 && pairs == nullptr)) fail(R3DGPU_EINVAL, "stereo: bad batch");
    if (count == 0) return;
    run_batch(pairs, count, static_cast<cudaStream_t>(stream));
  });
}

r3dgpu_status r3dgpu_match_stereo(const r3dgpu_view_u16* left, const r3dgpu_view_u16* right,
                                  const r3dgpu_view_u8* left_valid, const r3dgpu_view_u8* right_valid,
                                  int32_t disparity_min, int32_t num_disparities, const r3dgpu_stereo_options* options,
                                  r3dgpu_disparity_map* out, void* stream) {
  return guarded([&] {
    if (!left || !right || !out) fail(R3DGPU_EINVAL, "stereo: null argument");
    r3dgpu_pair p{};
    p.left = *left;
    p.right = *right;
    if (left_valid) p.left_valid = *left_valid;
    if (right_valid) p.right_valid = *right_valid;
    p.disparity_min = disparity_min;
    p.num_disparities = num_disparities;
    if (options) {
      p.options = *options;
    } else {
      r3dgpu_default_options(&p.options);
    }
    p.out = *out;
    run_batch(&p, 1, static_cast<cudaStream_t>(stream));
    *out = p.out;
  });
}

r3dgpu_status r3dgpu_match_stereo_host(const r3dgpu_view_u16* left, const r3dgpu_view_u16* right,
                                       const r3dgpu_view_u8* left_valid, const r3dgpu_view_u8* right_valid,
                                       int32_t disparity_min, int32_t num_disparities,
                                       const r3dgpu_stereo_options* options, r3dgpu_disparity_map* out) {
  return guarded([&] {
    if (!left || !right || !out || !left->data || !right->data) fail(R3DGPU_EINVAL, "stereo: null argument");
    if (!out->disparity) fail(R3DGPU_EINVAL, "stereo: missing output buffer");
    Workspace& W = workspace();
    cudaStream_t s = nullptr;
    // Inputs go into a dedicated allocation: run_batch rewinds the arena.
    const int wl = left->width, wr = right->width, h = left->height;
    if (wl <= 0 || wr <= 0 || h <= 0 || right->height != h)
      fail(R3DGPU_EINVAL, "stereo: rectified images must be non-empty with equal height");
    const bool lm = left_valid && left_valid->data && left_valid->width > 0;
    const bool rm = right_valid && right_valid->data && right_valid->width > 0;
    const size_t bytes = sizeof(uint16_t) * (static_cast<size_t>(wl) + wr) * h + (lm ? static_cast<size_t>(wl) * h : 0) +
                         (rm ? static_cast<size_t>(wr) * h : 0) + 2 * sizeof(float) * static_cast<size_t>(wl) * h + 1024;
    static thread_local DeviceBuffer<unsigned char> io;
    io.reserve(bytes);
    unsigned char* p = io.get();
    auto take = [&](size_t n) {
      unsigned char* r = p;
      p += (n + 255) & ~static_cast<size_t>(255);
      return r;
    };
    uint16_t* dl = reinterpret_cast<uint16_t*>(take(sizeof(uint16_t) * static_cast<size_t>(wl) * h));
    uint16_t* dr = reinterpret_cast<uint16_t*>(take(sizeof(uint16_t) * static_cast<size_t>(wr) * h));
    R3D_CUDA(cudaMemcpy2DAsync(dl, 2 * wl, left->data, 2 * left->stride, 2 * wl, h, cudaMemcpyHostToDevice, s));
    R3D_CUDA(cudaMemcpy2DAsync(dr, 2 * wr, right->data, 2 * right->stride, 2 * wr, h, cudaMemcpyHostToDevice, s));
    r3dgpu_pair q{};
    q.left = r3dgpu_view_u16{dl, wl, h, wl};
    q.right = r3dgpu_view_u16{dr, wr, h, wr};
    if (lm) {
      if (left_valid->width != wl || left_valid->height != h)
        fail(R3DGPU_EINVAL, "stereo: left mask size differs from the image");
      uint8_t* d = take(static_cast<size_t>(wl) * h);
      R3D_CUDA(cudaMemcpy2DAsync(d, wl, left_valid->data, left_valid->stride, wl, h, cudaMemcpyHostToDevice, s));
      q.left_valid = r3dgpu_view_u8{d, wl, h, wl};
    }
    if (rm) {
      if (right_valid->width != wr || right_valid->height != h)
        fail(R3DGPU_EINVAL, "stereo: right mask size differs from the image");
      uint8_t* d = take(static_cast<size_t>(wr) * h);
      R3D_CUDA(cudaMemcpy2DAsync(d, wr, right_valid->data, right_valid->stride, wr, h, cudaMemcpyHostToDevice, s));
      q.right_valid = r3dgpu_view_u8{d, wr, h, wr};
    }
    float* dd = reinterpret_cast<float*>(take(sizeof(float) * static_cast<size_t>(wl) * h));
    float* dc = reinterpret_cast<float*>(take(sizeof(float) * static_cast<size_t>(wl) * h));
    q.disparity_min = disparity_min;
    q.num_disparities = num_disparities;
    if (options) {
      q.options = *options;
    } else {
      r3dgpu_default_options(&q.options);
    }
    q.out.disparity = dd;
    q.out.confidence = dc;
    q.out.stride = wl;
    (void)W;
    run_batch(&q, 1, s);
    R3D_CUDA(cudaMemcpy2DAsync(out->disparity, sizeof(float) * out->stride, dd, sizeof(float) * wl, sizeof(float) * wl,
                               h, cudaMemcpyDeviceToHost, s));
    if (out->confidence)
      R3D_CUDA(cudaMemcpy2DAsync(out->confidence, sizeof(float) * out->stride, dc, sizeof(float) * wl,
                                 sizeof(float) * wl, h, cudaMemcpyDeviceToHost, s));
    R3D_CUDA(cudaStreamSynchronize(s));
    out->disparity_min = q.out.disparity_min;
    out->num_disparities = q.out.num_disparities;
    out->levels = q.out.levels;
    out->cells = q.out.cells;
  });
}

r3dgpu_status r3dgpu_census_transform(const r3dgpu_view_u16* image, uint64_t* out, int64_t out_stride, void* stream) {
  return guarded([&] {
    if (!image || !out) fail(R3DGPU_EINVAL, "census_transform: null argument");
    (void)workspace();
    if (image->width <= 0 || image->height <= 0) return;
    launch_census(image->data, image->stride, image->width, image->height, out, out_stride,
                  static_cast<cudaStream_t>(stream));
    R3D_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  });
}

r3dgpu_status r3dgpu_pyramid_down_u16(const r3dgpu_view_u16* image, uint16_t* out, int64_t out_stride, void* stream) {
  return guarded([&] {
    if (!image || !out) fail(R3DGPU_EINVAL, "pyramid_down: null argument");
    if (image->width <= 0 || image->height <= 0) fail(R3DGPU_EINVAL, "pyramid_down: empty image");
    (void)workspace();
    launch_pyramid_u16(image->data, image->stride, image->width, image->height, out, out_stride,
                       static_cast<cudaStream_t>(stream));
    R3D_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  });
}

r3dgpu_status r3dgpu_sgm_cost_volume_host(const r3dgpu_view_u16* left, const r3dgpu_view_u16* right,
                                          int32_t disparity_min, int32_t num_disparities,
                                          const r3dgpu_stereo_options* options, const uint16_t* ranges_lo,
                                          const uint16_t* ranges_num, uint16_t* out, uint64_t out_capacity,
                                          uint64_t* out_count) {
  return guarded([&] {
    if (!left || !right || !out_count) fail(R3DGPU_EINVAL, "sgm_cost_volume: null argument");
    r3dgpu_stereo_options o;
    if (options) {
      o = *options;
    } else {
      r3dgpu_default_options(&o);
    }
    check_options(o);
    const int wl = left->width, wr = right->width, h = left->height;
    if (wl <= 0 || wr <= 0 || h <= 0 || right->height != h)
      fail(R3DGPU_EINVAL, "stereo: rectified images must be non-empty with equal height");
    if (num_disparities <= 0) fail(R3DGPU_EINVAL, "stereo: no disparities to search");
    const int nd = align16(num_disparities);
    uint64_t cells = 0;
    int max_num = nd;
    if (ranges_lo && ranges_num) {
      max_num = 0;
      for (int64_t i = 0; i < static_cast<int64_t>(wl) * h; ++i) {
        const int lo = ranges_lo[i], n = ranges_num[i];
        if (n <= 0 || n % 16 != 0 || lo + n > nd)
          fail(R3DGPU_EINVAL, "stereo: invalid label range " + std::to_string(lo) + " + " + std::to_string(n) +
                                  " at (" + std::to_string(i % wl) + ", " + std::to_string(i / wl) + ") for " +
                                  std::to_string(nd) + " labels");
        cells += static_cast<uint64_t>(n);
        max_num = std::max(max_num, n);
      }
    } else {
      cells = static_cast<uint64_t>(wl) * h * nd;
    }
    *out_count = cells;
    if (out == nullptr) return;
    if (out_capacity < cells) fail(R3DGPU_EINVAL, "sgm_cost_volume: output too small");
    if (cells >= (uint64_t{1} << 31)) fail(R3DGPU_EUNSUPPORTED, "sgm_cost_volume: 2^31 or more labels");
    Workspace& W = workspace();
    W.arena.reset();
    W.pinned.reset();
    Arena& A = W.arena;
    cudaStream_t s = nullptr;
    const uint16_t* dl = upload(A, left->data, wl, h, left->stride, s);
    const uint16_t* dr = upload(A, right->data, wr, h, right->stride, s);
    uint64_t* cl = A.alloc<uint64_t>(static_cast<size_t>(wl) * h);
    uint64_t* cr = A.alloc<uint64_t>(static_cast<size_t>(wr) * h);
    launch_census(dl, wl, wl, h, cl, wl, s);
    launch_census(dr, wr, wr, h, cr, wr, s);
    RowInterval* il = A.alloc<RowInterval>(h);
    RowInterval* ir = A.alloc<RowInterval>(h);
    launch_intervals(nullptr, 0, wl, h, il, s);
    launch_intervals(nullptr, 0, wr, h, ir, s);
    uint16_t *rlo = nullptr, *rnum = nullptr;
    if (ranges_lo && ranges_num) {
      rlo = upload(A, ranges_lo, wl, h, wl, s);
      rnum = upload(A, ranges_num, wl, h, wl, s);
    }
    SgmMatch* hm = W.pinned.alloc<SgmMatch>(1);
    fill_match(*hm, o, DView<uint16_t>{dl, wl, h, wl}, cl, cr, wr, il, ir, rlo, rnum, disparity_min, nd, false, false);
    if (!(ranges_lo && ranges_num) && sgm_path_enabled() && sgm_path_shape(nd).g_ != 0 && sgm_path_fits(wl, nd)) {
      // The whole image as one full-range tile through the chain passes.
      SgmMatch* dm = A.alloc<SgmMatch>(1);
      R3D_CUDA(cudaMemcpyAsync(dm, hm, sizeof(SgmMatch), cudaMemcpyHostToDevice, s));
      const int64_t px = static_cast<int64_t>(wl) * h;
      SgmPathJob* hj = W.pinned.alloc<SgmPathJob>(1);
      *hj = SgmPathJob{};
      hj->w = wl;
      hj->h = h;
      const SgmPathShape sh = sgm_path_shape(nd);
      SgmPathSegment seg{sh, 0, 1, {0, 0, 0}, static_cast<int64_t>(cells), px};
      for (int c = 0; c < kPathClasses; ++c) seg.blocks[c] = (sgm_path_chains(c, wl, h) + 32 / sh.g_ - 1) / (32 / sh.g_);
      hj->disp = A.alloc<float>(static_cast<size_t>(px));
      hj->cells = A.alloc<unsigned long long>(1);
      uint16_t* vol = A.alloc<uint16_t>(cells);
      hj->volume = vol;
      SgmPathJob* dj = A.alloc<SgmPathJob>(1);
      R3D_CUDA(cudaMemcpyAsync(dj, hj, sizeof(SgmPathJob), cudaMemcpyHostToDevice, s));
      SgmPathWave wv{};
      wv.jobs = dj;
      wv.njobs = 1;
      wv.segs = &seg;
      wv.nsegs = 1;
      wv.cells = static_cast<int64_t>(cells);
      wv.pixels = px;
      wv.keys = 0;
      wv.rows = h;
      wv.terms = hm->term_u8;
      W.scratch.reserve(sgm_path_buffers(wv.cells, px, 0, wv.terms != 0).total);
      wv.buffer = W.scratch.get();
      launch_sgm_path_wave(dm, wv, W.sms, s);
      R3D_CUDA(cudaMemcpyAsync(out, vol, sizeof(uint16_t) * cells, cudaMemcpyDeviceToHost, s));
      R3D_CUDA(cudaStreamSynchronize(s));
      return;
    }
    if (ranges_lo && ranges_num && sgm_path_ranged_enabled()) {
      // The whole image as one ranged tile through the chain passes.
      SgmMatch* dm = A.alloc<SgmMatch>(1);
      R3D_CUDA(cudaMemcpyAsync(dm, hm, sizeof(SgmMatch), cudaMemcpyHostToDevice, s));
      const int64_t px = static_cast<int64_t>(wl) * h;
      int over32 = 0;
      for (int64_t i = 0; i < px; ++i) over32 += ranges_num[i] > 32 ? 1 : 0;
      const SgmPathShape sh = sgm_path_ranged_shape(over32, px);
      SgmPathJob* hj = W.pinned.alloc<SgmPathJob>(1);
      *hj = SgmPathJob{};
      hj->w = wl;
      hj->h = h;
      SgmPathSegment seg{sh, 0, 1, {0, 0, 0}, static_cast<int64_t>(cells), px};
      for (int c = 0; c < kPathClasses; ++c) seg.blocks[c] = (sgm_path_chains(c, wl, h) + 32 / sh.g_ - 1) / (32 / sh.g_);
      hj->disp = A.alloc<float>(static_cast<size_t>(px));
      hj->cells = A.alloc<unsigned long long>(1);
      uint16_t* vol = A.alloc<uint16_t>(cells);
      hj->volume = vol;
      SgmPathJob* dj = A.alloc<SgmPathJob>(1);
      R3D_CUDA(cudaMemcpyAsync(dj, hj, sizeof(SgmPathJob), cudaMemcpyHostToDevice, s));
      SgmPathRangedWave wv{};
      wv.jobs = dj;
      wv.njobs = 1;
      wv.segs = &seg;
      wv.nsegs = 1;
      wv.cells = static_cast<int64_t>(cells);
      wv.pixels = px;
      wv.keys = 0;
      wv.rows = h;
      wv.maxnum = max_num;
      wv.terms = hm->term_u8;
      W.scratch.reserve(sgm_path_ranged_buffers(wv.cells, px, 0, h, max_num, W.sms, wv.terms != 0).total);
      wv.buffer = W.scratch.get();
      launch_sgm_path_ranged_wave(dm, wv, W.sms, s);
      R3D_CUDA(cudaMemcpyAsync(out, vol, sizeof(uint16_t) * cells, cudaMemcpyDeviceToHost, s));
      R3D_CUDA(cudaStreamSynchronize(s));
      return;
    }
    const SgmFullPlan plan = (ranges_lo && ranges_num) ? SgmFullPlan{{0, 0}, 0} : sgm_full_plan(nd, W.smem_optin);
    const SgmFullShape sh = plan.shape;
    const bool ranged = !sh.g_ && !general_ranged_kernel();
    SgmRangedPlan rplan{{0, 0}, 0};
    if (ranged) {
      // The whole image is one tile: its label statistics from the host ranges.
      int st[kTileStats] = {};
      for (int64_t i = 0; i < static_cast<int64_t>(wl) * h; ++i) {
        const int n = ranges_num[i];
        st[0] = std::max(st[0], n);
        for (int k = 1; k < kTileStats; ++k) st[k] += n > tile_stat_width(k - 1) ? 1 : 0;
      }
      rplan = sgm_ranged_plan(sgm_ranged_shape_for_width(sgm_ranged_width_for(st, static_cast<int64_t>(wl) * h)),
                              W.smem_optin);
    }
    const int ndw = ranged ? sgm_ranged_ndw(rplan.shape, max_num) : 0;
    const int maxc = (sh.g_ || ranged) ? 0 : sgm_maxc_for(max_num);
    const int rows = sh.g_ ? plan.rows : (ranged ? rplan.rows : sgm_rows_for(maxc, W.smem_optin));
    float* disp = A.alloc<float>(static_cast<size_t>(wl) * h);
    unsigned long long* dcells = A.alloc<unsigned long long>(1);
    uint16_t* vol = A.alloc<uint16_t>(cells);
    SgmJob* hj = W.pinned.alloc<SgmJob>(1);
    *hj = SgmJob{};
    hj->match = 0;
    hj->w = wl;
    hj->h = h;
    hj->disp = disp;
    hj->cells = dcells;
    hj->volume = vol;
    SgmMatch* dm = A.alloc<SgmMatch>(1);
    SgmJob* dj = A.alloc<SgmJob>(1);
    R3D_CUDA(cudaMemcpyAsync(dm, hm, sizeof(SgmMatch), cudaMemcpyHostToDevice, s));
    R3D_CUDA(cudaMemcpyAsync(dj, hj, sizeof(SgmJob), cudaMemcpyHostToDevice, s));
    const size_t slot = sh.g_    ? sgm_full_slot_layout(wl, h, nd, 2 * sh.g_ * sh.k_).total
                        : ranged ? sgm_ranged_slot_layout(wl, h, cells, nd, ndw, rows).total
                                 : sgm_slot_layout(wl, h, cells, maxc, nd).total;
    W.scratch.reserve(slot);
    R3D_CUDA(cudaMemsetAsync(W.counter.get(), 0, sizeof(int), s));
    if (sh.g_) {
      launch_sgm_full(sh, nd, dm, dj, 1, rows, 1, W.scratch.get(), slot, W.counter.get(), s);
    } else if (ranged) {
      launch_sgm_ranged(rplan.shape, dm, dj, 1, rows, ndw, 1, W.scratch.get(), slot, W.counter.get(), s);
    } else {
      launch_sgm(dm, dj, 1, maxc, rows, 1, W.scratch.get(), slot, W.counter.get(), s);
    }
    R3D_CUDA(cudaMemcpyAsync(out, vol, sizeof(uint16_t) * cells, cudaMemcpyDeviceToHost, s));
    R3D_CUDA(cudaStreamSynchronize(s));
  });
}

r3dgpu_status r3dgpu_ranges_from_coarse_host(const float* coarse, int32_t wc, int32_t hc, int32_t width,
                                             int32_t height, const uint8_t* fine_valid, const uint8_t* partner_valid,
                                             int32_t partner_width, int32_t partner_sign, int32_t disparity_min,
                                             int32_t num_disparities, const r3dgpu_stereo_options* options,
                                             int32_t mirrored, uint16_t* lo_out, uint16_t* num_out) {
  return guarded([&] {
    if (!coarse || !lo_out || !num_out) fail(R3DGPU_EINVAL, "ranges_from_coarse: null argument");
    if (wc != (width + 1) / 2 || hc != (height + 1) / 2)
      fail(R3DGPU_EINVAL, "stereo: coarse map of " + std::to_string(wc) + "x" + std::to_string(hc) + " for a level of " +
                              std::to_string(width) + "x" + std::to_string(height));
    r3dgpu_stereo_options o;
    if (options) {
      o = *options;
    } else {
      r3dgpu_default_options(&o);
    }
    Workspace& W = workspace();
    W.arena.reset();
    Arena& A = W.arena;
    cudaStream_t s = nullptr;
    const float* dc = upload(A, coarse, wc, hc, wc, s);
    const uint8_t* dfv = fine_valid ? upload(A, fine_valid, width, height, width, s) : nullptr;
    const uint8_t* dpv = partner_valid ? upload(A, partner_valid, partner_width, height, partner_width, s) : nullptr;
    RowInterval* pr = A.alloc<RowInterval>(height);
    launch_intervals(dpv, partner_width, partner_width, height, pr, s);
    float* scr = A.alloc<float>(static_cast<size_t>(ranges_scratch_floats(wc, hc, o.range_fill)));
    uint16_t* lo = A.alloc<uint16_t>(static_cast<size_t>(width) * height);
    uint16_t* nu = A.alloc<uint16_t>(static_cast<size_t>(width) * height);
    RangeParams rp{o.range_radius, o.range_margin, o.range_fill, disparity_min, align16(num_disparities), partner_sign,
                   mirrored ? 1 : 0};
    launch_ranges_from_coarse(dc, wc, hc, width, height, dfv, width, pr, rp, scr, lo, nu, s);
    R3D_CUDA(cudaMemcpyAsync(lo_out, lo, sizeof(uint16_t) * width * height, cudaMemcpyDeviceToHost, s));
    R3D_CUDA(cudaMemcpyAsync(num_out, nu, sizeof(uint16_t) * width * height, cudaMemcpyDeviceToHost, s));
    R3D_CUDA(cudaStreamSynchronize(s));
  });
}

r3dgpu_status r3dgpu_remove_speckles_host(float* disparity, int32_t width, int32_t height, int32_t min_size,
                                          float max_diff) {
  return guarded([&] {
    if (!disparity && width > 0 && height > 0) fail(R3DGPU_EINVAL, "remove_speckles: null argument");
    if (min_size <= 1 || width <= 0 || height <= 0) return;
    Workspace& W = workspace();
    W.arena.reset();
    Arena& A = W.arena;
    cudaStream_t s = nullptr;
    float* d = upload(A, static_cast<const float*>(disparity), width, height, width, s);
    int* uf = A.alloc<int>(2 * static_cast<size_t>(width) * height);
    launch_remove_speckles(d, width, height, min_size, max_diff, uf, s);
    R3D_CUDA(cudaMemcpyAsync(disparity, d, sizeof(float) * width * height, cudaMemcpyDeviceToHost, s));
    R3D_CUDA(cudaStreamSynchronize(s));
  });
}

r3dgpu_status r3dgpu_remove_speckles_no_alloc(float* disparity, int32_t width, int32_t height, int32_t min_size,
                                              float max_diff, void* stream) {
  return guarded([&] {
    // The device this thread chose with r3dgpu_set_device, as for every other
    // entry point, but without workspace(): that would allocate.
    remove_speckles_static_scratch(t_device, disparity, width, height, min_size, max_diff,
                                   static_cast<cudaStream_t>(stream));
  });
}

r3dgpu_status r3dgpu_median_filter_3x3_host(const float* disparity, int32_t width, int32_t height, float* out) {
  return guarded([&] {
    if ((!disparity || !out) && width > 0 && height > 0) fail(R3DGPU_EINVAL, "median_filter_3x3: null argument");
    if (width <= 0 || height <= 0) return;
    Workspace& W = workspace();
    W.arena.reset();
    Arena& A = W.arena;
    cudaStream_t s = nullptr;
    const float* d = upload(A, disparity, width, height, width, s);
    float* m = A.alloc<float>(static_cast<size_t>(width) * height);
    launch_median3x3(d, width, height, m, s);
    R3D_CUDA(cudaMemcpyAsync(out, m, sizeof(float) * width * height, cudaMemcpyDeviceToHost, s));
    R3D_CUDA(cudaStreamSynchronize(s));
  });
}

}  // extern "C"
