// Full-range SGM as eight chain passes (sgm_path.cu): the tiles of a wave are
// aggregated one path direction at a time, every path split into its
// independent 1-D chains (tile rows, columns or diagonals), many chains in
// flight per SM. Costs (u8) are computed once per wave; each pass adds its
// path to the wave's sum volume (u16 per cell), and the last pass also runs
// the winner-takes-all. The acceptance rules follow in a per-pixel kernel.
#pragma once

#include <cstddef>
#include <cstdint>

#include "sgm.h"

namespace r3dgpu {

// Chain classes: tile rows (horizontal paths), tile columns (vertical
// paths) and diagonals (both diagonal directions: w + h - 1 chains).
constexpr int kPathClasses = 3;

// One tile of a wave. Jobs of a wave are ordered by kernel shape; cell_off
// and px_off run over the whole wave, blk restarts at 0 with every shape.
struct SgmPathJob {
  int match;
  int x0, y0, w, h;
  int pad_;
  int64_t cell_off;           // first cell of the tile in the wave's cost and sum volumes
  int64_t px_off;             // first pixel of the tile in the wave's WTA records
  int64_t rk_off;             // first right-WTA key of the tile (diagonal LR only)
  int64_t blk[kPathClasses];  // first chain block (32 / G chains) of the tile, per chain class
  int64_t row_off;            // ranged waves: first row of the tile in the wave's per-row arrays
  float* disp;
  float* conf;
  unsigned long long* cells;
  uint16_t* volume;
};

// G lanes per chain, K label pairs per lane (2 G K >= nd).
struct SgmPathShape {
  int g_;
  int k_;
};

// Narrowest compiled shape for nd labels ({0, 0}: more labels than the path
// kernels take, or a tile too wide for the cost kernel's staged partner row:
// tile width + nd - 1 must stay within 2048).
SgmPathShape sgm_path_shape(int nd);
// Whether a full-range tile of width w with nd labels fits the cost kernel.
inline bool sgm_path_fits(int w, int nd) { return w + nd - 1 <= 2048; }
inline int64_t sgm_path_chains(int cls, int w, int h) { return cls == 0 ? h : (cls == 1 ? w : w + h - 1); }

// Device buffers of a wave (bytes, 256-byte aligned pieces). Byte terms:
// seven arrays of term_stride bytes from `terms` on (full-range waves keep
// them in place of the u16 sum volume, ranged waves beside it).
struct SgmPathBuffers {
  size_t cost, sum, terms, info, rkeys, ints, total;  // ints: full-range waves, the tiles' intensities
  int64_t term_stride;
  size_t rec, rowsum, rowstart, rowshift, overflow;  // ranged waves only
  int64_t overflow_words;                            // per chain buffer
};
SgmPathBuffers sgm_path_buffers(int64_t cells, int64_t pixels, int64_t keys, bool terms);

// A wave on the device: all jobs (device pointer), and per shape the range
// of jobs with its chain-block counts.
struct SgmPathSegment {
  SgmPathShape shape;
  int first, count;
  int64_t blocks[kPathClasses];
  int64_t cells, pixels;  // of the segment's tiles (per-launch profiling)
  int full = 0;           // every match of the segment has exactly 2 G K labels (no unit past nd)
};

// Per-launch timing of the pass kernels while the library's profiling is on
// (defined with the rest of the profiling in matcher.cpp): `bytes` is the
// launch's algorithmic HBM traffic.
bool profile_on();
cudaEvent_t profile_mark(cudaStream_t s);
void profile_pass(cudaEvent_t a, cudaEvent_t b, const char* kernel, const char* shape, uint64_t cells,
                  uint64_t pixels, uint64_t bytes);
struct SgmPathWave {
  const SgmPathJob* jobs;
  int njobs;
  const SgmPathSegment* segs;  // host array
  int nsegs;
  int64_t cells, pixels, keys, rows;
  unsigned char* buffer;  // sgm_path_buffers(cells, pixels, keys, terms).total bytes
  const int* cancel;      // device view of the caller's cancellation flag, or null
  int terms;              // 1: byte terms (every match of the wave has term_u8)
  int max_span;           // largest tile width + labels - 1 of the wave (0: unknown)
};

// Costs, the 8 passes and the acceptance rules of one wave, on stream s.
void launch_sgm_path_wave(const SgmMatch* dm, const SgmPathWave& wave, int sms, cudaStream_t s);

// Whether full-range tiles go to the path kernels (default) or to the
// one-CTA-per-tile wavefront kernel (R3DGPU_FULL_KERNEL=wavefront).
bool sgm_path_enabled();

// ---- Ranged tiles (per-pixel label ranges lo, num) through the chain passes.
// Sums and costs are packed per tile (each pixel's num labels, row-major);
// chunk 0 of a chain's predecessor vector (64 labels) stays in shared memory,
// labels beyond it of the rare wide pixels in a per-chain overflow in global
// memory. Shapes: (2, 8) = 32 labels per chunk, (4, 8) = 64.
SgmPathShape sgm_path_ranged_shape(int over32, int64_t pixels);
struct SgmPathRangedWave {
  const SgmPathJob* jobs;
  int njobs;
  const SgmPathSegment* segs;
  int nsegs;
  int64_t cells, pixels, keys, rows;
  int maxnum;  // largest label count of a pixel of the wave
  unsigned char* buffer;
  const int* cancel;  // device view of the caller's cancellation flag, or null
  int terms;          // byte terms (every match of the wave has term_u8)
  int max_span;       // largest tile width + labels - 1 of the wave (0: unknown)
};
SgmPathBuffers sgm_path_ranged_buffers(int64_t cells, int64_t pixels, int64_t keys, int64_t rows, int maxnum,
                                       int sms, bool terms);
void launch_sgm_path_ranged_wave(const SgmMatch* dm, const SgmPathRangedWave& wave, int sms, cudaStream_t s);
bool sgm_path_ranged_enabled();

}  // namespace r3dgpu
