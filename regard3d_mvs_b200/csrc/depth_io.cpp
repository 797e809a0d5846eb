// Depth-map files (.r3dd, format version 2): r3dgpu_write_depth_map,
// r3dgpu_read_depth_map_info, r3dgpu_read_depth_map. The layout is the
// reference's write_depth_map / read_depth_map
// (src/r3d/mvs/depth_map.cpp:135-239), so that maps served by this library
// feed the reference pipeline's --reuse and the other way round: the magic
// "R3DD", u32 version 2, u32 view, i32 camera width and height, f64 fx, fy,
// cx, cy, f64 rotation (row-major), f64 centre, u32 partner count (at most
// 16) and the partners (u32), i32 map width and height, then the rows of
// depth (f32), confidence (f32), pair mask (u16), support (u8) and colour
// (3 x u8), all little-endian without padding.
#include <array>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "api_guard.h"
#include "matcher_internal.h"

namespace r3dgpu {
namespace {

constexpr char kMagic[4] = {'R', '3', 'D', 'D'};
constexpr uint32_t kVersion = 2;

struct File {
  std::FILE* f = nullptr;
  ~File() {
    if (f != nullptr) std::fclose(f);
  }
};

template <class T>
void put(std::FILE* f, const T& v, const std::string& path) {
  if (std::fwrite(&v, sizeof(T), 1, f) != 1) fail(R3DGPU_EINVAL, "error writing depth map " + path);
}

template <class T>
void get(std::FILE* f, T& v, const std::string& path) {
  if (std::fread(&v, sizeof(T), 1, f) != 1) fail(R3DGPU_EINVAL, "corrupt depth map " + path);
}

// Rows of one image: `elem` bytes per pixel, `stride` bytes between rows in
// `src` (host memory), or zeros when src is NULL.
void put_rows(std::FILE* f, const void* src, int64_t stride, int w, int h, size_t elem, const std::string& path) {
  const size_t row = elem * static_cast<size_t>(w);
  std::vector<unsigned char> zeros(src == nullptr ? row : 0, 0);
  for (int y = 0; y < h; ++y) {
    const void* p = src != nullptr ? static_cast<const unsigned char*>(src) + static_cast<int64_t>(y) * stride
                                   : zeros.data();
    if (row > 0 && std::fwrite(p, 1, row, f) != row) fail(R3DGPU_EINVAL, "error writing depth map " + path);
  }
}

void get_rows(std::FILE* f, void* dst, int64_t stride, int w, int h, size_t elem, const std::string& path) {
  const size_t row = elem * static_cast<size_t>(w);
  std::vector<unsigned char> skip(dst == nullptr ? row : 0);
  for (int y = 0; y < h; ++y) {
    void* p = dst != nullptr ? static_cast<unsigned char*>(dst) + static_cast<int64_t>(y) * stride : skip.data();
    if (row > 0 && std::fread(p, 1, row, f) != row) fail(R3DGPU_EINVAL, "corrupt depth map " + path);
  }
}

// Host copy of a device image (dense rows), or NULL for a NULL image.
std::vector<unsigned char> host_copy(const void* src, int64_t stride, int w, int h, size_t elem, cudaStream_t s) {
  std::vector<unsigned char> out;
  if (src == nullptr) return out;
  out.resize(elem * static_cast<size_t>(w) * h);
  if (!out.empty())
    R3D_CUDA(cudaMemcpy2DAsync(out.data(), elem * w, src, stride, elem * w, h, cudaMemcpyDeviceToHost, s));
  return out;
}

void check_map(const r3dgpu_depth_map* m) {
  if (m == nullptr) fail(R3DGPU_EINVAL, "depth map: null argument");
  if (m->width < 0 || m->height < 0 || (m->width > 0 && m->height > 0 && m->stride < m->width))
    fail(R3DGPU_EINVAL, "depth map: bad size or stride");
  if (m->num_partners > R3DGPU_MAX_PARTNERS) fail(R3DGPU_EINVAL, "depth map: more than 16 partners");
  if (m->color != nullptr && m->color_stride < 3LL * m->width)
    fail(R3DGPU_EINVAL, "depth map: colour stride below 3 x width");
}

// Header fields up to the images (sets the camera, K^-1, view, partners, width and height).
void read_header(std::FILE* f, const std::string& path, r3dgpu_depth_map& m) {
  char magic[4];
  uint32_t version = 0;
  if (std::fread(magic, 1, 4, f) != 4 || std::fread(&version, sizeof(version), 1, f) != 1 ||
      std::memcmp(magic, kMagic, 4) != 0 || version != kVersion)
    fail(R3DGPU_EINVAL, path + " is not an r3d depth map (version 2)");
  get(f, m.view, path);
  int32_t cw = 0, ch = 0;
  get(f, cw, path);
  get(f, ch, path);
  r3dgpu_pinhole& k = m.camera.intrinsics;
  k.width = cw;
  k.height = ch;
  get(f, k.fx, path);
  get(f, k.fy, path);
  get(f, k.cx, path);
  get(f, k.cy, path);
  for (double& v : m.camera.rotation) get(f, v, path);
  for (double& v : m.camera.center) get(f, v, path);
  uint32_t np = 0;
  get(f, np, path);
  if (np > R3DGPU_MAX_PARTNERS) fail(R3DGPU_EINVAL, "corrupt depth map " + path);
  m.num_partners = np;
  for (uint32_t i = 0; i < np; ++i) get(f, m.partners[i], path);
  int32_t w = 0, h = 0;
  get(f, w, path);
  get(f, h, path);
  if (w <= 0 || h <= 0 || w > (1 << 16) || h > (1 << 16)) fail(R3DGPU_EINVAL, "corrupt depth map " + path);
  m.width = w;
  m.height = h;
  // K^-1 of the pinhole intrinsics (callers that need Eigen's rounding of it
  // replace it).
  const double ki[9] = {1.0 / k.fx, 0.0, -k.cx / k.fx, 0.0, 1.0 / k.fy, -k.cy / k.fy, 0.0, 0.0, 1.0};
  std::memcpy(m.camera.k_inv, ki, sizeof(ki));
}

}  // namespace
}  // namespace r3dgpu

using namespace r3dgpu;

extern "C" {

r3dgpu_status r3dgpu_write_depth_map(const char* path, const r3dgpu_depth_map* map, int32_t device, void* stream) {
  return guard([&] {
    if (path == nullptr) fail(R3DGPU_EINVAL, "depth map: null path");
    check_map(map);
    const std::string p(path);
    const int w = map->width, h = map->height;
    const void *depth = map->depth, *conf = map->confidence, *mask = map->pair_mask, *sup = map->support,
               *color = map->color;
    int64_t s4 = 4 * map->stride, s2 = 2 * map->stride, s1 = map->stride, s3 = map->color_stride;
    std::vector<unsigned char> hd, hc, hm, hs, hcol;
    if (device != 0) {
      cudaStream_t s = static_cast<cudaStream_t>(stream);
      hd = host_copy(depth, s4, w, h, 4, s);
      hc = host_copy(conf, s4, w, h, 4, s);
      hm = host_copy(mask, s2, w, h, 2, s);
      hs = host_copy(sup, s1, w, h, 1, s);
      hcol = host_copy(color, s3, w, h, 3, s);
      R3D_CUDA(cudaStreamSynchronize(s));
      auto pick = [](const void* d, std::vector<unsigned char>& v) -> const void* { return d ? v.data() : nullptr; };
      depth = pick(depth, hd);
      conf = pick(conf, hc);
      mask = pick(mask, hm);
      sup = pick(sup, hs);
      color = pick(color, hcol);
      s4 = 4LL * w;
      s2 = 2LL * w;
      s1 = w;
      s3 = 3LL * w;
    }
    File file;
    file.f = std::fopen(path, "wb");
    if (file.f == nullptr) fail(R3DGPU_EINVAL, "cannot write depth map " + p);
    std::FILE* f = file.f;
    if (std::fwrite(kMagic, 1, 4, f) != 4) fail(R3DGPU_EINVAL, "error writing depth map " + p);
    put(f, kVersion, p);
    put(f, map->view, p);
    const r3dgpu_pinhole& k = map->camera.intrinsics;
    put(f, static_cast<int32_t>(k.width), p);
    put(f, static_cast<int32_t>(k.height), p);
    for (const double v : {k.fx, k.fy, k.cx, k.cy}) put(f, v, p);
    for (const double v : map->camera.rotation) put(f, v, p);
    for (const double v : map->camera.center) put(f, v, p);
    put(f, map->num_partners, p);
    for (uint32_t i = 0; i < map->num_partners; ++i) put(f, map->partners[i], p);
    put(f, static_cast<int32_t>(w), p);
    put(f, static_cast<int32_t>(h), p);
    put_rows(f, depth, s4, w, h, 4, p);
    put_rows(f, conf, s4, w, h, 4, p);
    put_rows(f, mask, s2, w, h, 2, p);
    put_rows(f, sup, s1, w, h, 1, p);
    put_rows(f, color, s3, w, h, 3, p);
    if (std::fflush(f) != 0) fail(R3DGPU_EINVAL, "error writing depth map " + p);
  });
}

r3dgpu_status r3dgpu_read_depth_map_info(const char* path, r3dgpu_depth_map* map) {
  return guard([&] {
    if (path == nullptr || map == nullptr) fail(R3DGPU_EINVAL, "depth map: null argument");
    File file;
    file.f = std::fopen(path, "rb");
    if (file.f == nullptr) fail(R3DGPU_EINVAL, std::string("cannot open depth map ") + path);
    r3dgpu_depth_map m = *map;
    read_header(file.f, path, m);
    *map = m;
  });
}

r3dgpu_status r3dgpu_read_depth_map(const char* path, r3dgpu_depth_map* map) {
  return guard([&] {
    if (path == nullptr || map == nullptr) fail(R3DGPU_EINVAL, "depth map: null argument");
    File file;
    file.f = std::fopen(path, "rb");
    if (file.f == nullptr) fail(R3DGPU_EINVAL, std::string("cannot open depth map ") + path);
    r3dgpu_depth_map m = *map;
    read_header(file.f, path, m);
    if (map->width != m.width || map->height != m.height)
      fail(R3DGPU_EINVAL, "read_depth_map: the buffers are " + std::to_string(map->width) + "x" +
                              std::to_string(map->height) + ", the file's map is " + std::to_string(m.width) + "x" +
                              std::to_string(m.height));
    check_map(&m);
    std::FILE* f = file.f;
    const int w = m.width, h = m.height;
    get_rows(f, m.depth, 4 * m.stride, w, h, 4, path);
    get_rows(f, m.confidence, 4 * m.stride, w, h, 4, path);
    get_rows(f, m.pair_mask, 2 * m.stride, w, h, 2, path);
    get_rows(f, m.support, m.stride, w, h, 1, path);
    get_rows(f, const_cast<uint8_t*>(m.color), m.color_stride, w, h, 3, path);
    *map = m;
  });
}

}  // extern "C"
