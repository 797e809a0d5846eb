// Launch wrappers of the r3dgpu image kernels (image_kernels.cu) and the SGM
// tile kernel (sgm.cu). All pointers are device pointers; strides are in
// elements; every wrapper launches on `s` and counts its launches.
#pragma once

#include "runtime.h"

#include <cstdint>

namespace r3dgpu {

// Valid column interval [first, last] of a row (first > last: none).
struct RowInterval {
  int first;
  int last;
};

// ---- image_kernels.cu
void launch_census(const uint16_t* img, int64_t stride, int w, int h, uint64_t* out, int64_t ostride, cudaStream_t s);
void launch_pyramid_u16(const uint16_t* in, int64_t istride, int w, int h, uint16_t* out, int64_t ostride,
                        cudaStream_t s);
// pyramid_down<uint8_t> followed by the >= 128 threshold (reduce_mask).
void launch_reduce_mask(const uint8_t* in, int64_t istride, int w, int h, uint8_t* out, int64_t ostride,
                        cudaStream_t s);
void launch_mirror_u16(const uint16_t* in, int64_t istride, int w, int h, uint16_t* out, cudaStream_t s);
void launch_mirror_u8(const uint8_t* in, int64_t istride, int w, int h, uint8_t* out, cudaStream_t s);
// mask == nullptr: every row is [0, w - 1].
void launch_intervals(const uint8_t* mask, int64_t stride, int w, int h, RowInterval* out, cudaStream_t s);
// map[i] = +inf where bad[i] != 0.
void launch_lr_check(const float* map, const float* other, int w, int h, int wo, int sign, int max_diff,
                     uint8_t* bad, cudaStream_t s);
void launch_apply_bad(float* map, const uint8_t* bad, int64_t n, cudaStream_t s);
// Segments of 4-neighbours of the contiguous map d (w x h, invalid = +inf)
// whose values differ by at most max_diff: afterwards parent[i] is the root
// (smallest index) of valid pixel i's segment and size[root] its pixel count.
void launch_segments(const float* d, int w, int h, float max_diff, int* parent, int* size, cudaStream_t s);
// In place; scratch: 2 * w * h ints.
void launch_remove_speckles(float* d, int w, int h, int min_size, float max_diff, int* scratch, cudaStream_t s);
// Same filter with the scratch in a static device array (noalloc.cu); the
// map is device memory of `device`, contiguous, and the work is enqueued on `s`.
void remove_speckles_static_scratch(int device, float* d, int w, int h, int min_size, float max_diff, cudaStream_t s);
void launch_median3x3(const float* in, int w, int h, float* out, cudaStream_t s);
// out[y][x] = in[y][w - 1 - x] - offset.
void launch_unmirror_offset(const float* in, int w, int h, float offset, float* out, cudaStream_t s);
void launch_copy2d_f32(const float* in, int64_t istride, int w, int h, float* out, int64_t ostride, cudaStream_t s);

struct RangeParams {
  int radius, margin, fill;
  int dmin, n_all;       // n_all: aligned label count of the fine level
  int partner_sign;      // -1: left base image, +1: right base image
  int mirrored;
};

// Scratch needed by launch_ranges_from_coarse, in floats.
int64_t ranges_scratch_floats(int wc, int hc, int fill);
void launch_ranges_from_coarse(const float* coarse, int wc, int hc, int w, int h, const uint8_t* fine_valid,
                               int64_t fv_stride, const RowInterval* partner_rows, const RangeParams& p,
                               float* scratch, uint16_t* lo, uint16_t* num, cudaStream_t s);

// ---- blend (image_kernels.cu)
struct BlendTile {
  int x0, y0, w, h;        // tile in the base image
  int c0x, c1x, c0y, c1y;  // core
  const float* disp;       // w x h, tile-local
  const float* conf;       // may be null
};

// Blends the tiles of one match (stereo_matcher.cpp:700-766). Output at
// (x, y) goes to out_disp[y * ostride + (mirror_out ? w - 1 - x : x)] minus
// `offset`; conf_out may be null.
void launch_blend(const BlendTile* tiles, int ntiles, int tiles_x, const int* bx, const int* by, int w, int h,
                  int blend, int mirror_out, float offset, float* out_disp, float* out_conf, int64_t ostride,
                  cudaStream_t s);

// Per-tile label statistics: stats[0] = largest num, stats[1 + i] = pixels
// with num above tile_stat_width(i) (32, 64, 128, 192, 256, 384, 512).
constexpr int kTileStats = 8;
R3D_HOSTDEV constexpr int tile_stat_width(int i) {
  return i < 3 ? 32 << i : (i < 5 ? 192 + 64 * (i - 3) : (i == 5 ? 384 : 512));
}

// Per tile: number of labels (sum of num over its pixels) and the label
// statistics (kTileStats ints). tiles: (x0, y0, w, h) per tile; one block per tile.
void launch_tile_cells(const uint16_t* rnum, int64_t stride, const int4* tiles, int ntiles,
                       unsigned long long* cells, int* stats, cudaStream_t s);

}  // namespace r3dgpu
