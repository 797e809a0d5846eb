/*
 * r3dgpu — seeded synthetic rectified pairs for benchmarks and tests.
 *
 * No reference counterpart: the reference's bench generates multi-scale
 * noise (bench/bench_stereo.cpp:31-65); this generator produces the pairs of
 * the benchmark configurations instead: blurred uniform noise, a piecewise
 * planar disparity field, a bilinear inverse warp with Gaussian noise, and
 * optionally textureless patches and occluded (re-noised) right pixels.
 * Deterministic for a given seed on every platform (std::mt19937 with a
 * portable uniform and Box-Muller normal).
 */
#ifndef R3DGPU_SYNTH_H
#define R3DGPU_SYNTH_H

#include <stdint.h>

#include "r3dgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct r3dgpu_synth_params {
  int32_t width;
  int32_t height;
  int32_t num_disparities;    /* disparities are clipped to [5, num_disparities - 8] */
  uint32_t seed;
  float blur_sigma;           /* Gaussian blur of the noise, pixels (1.5) */
  float noise_sigma;          /* noise added to the right image, grey levels (2) */
  int32_t planes;             /* disparity planes (8) */
  float textureless_fraction; /* area covered by constant patches (0 or 0.15) */
  float occluded_fraction;    /* right pixels replaced by fresh noise (0 or 0.10) */
} r3dgpu_synth_params;

/* Writes width x height 8-bit left and right images (row stride = width) and,
 * if gt is not NULL, the true disparity x_left - x_right of every left pixel.
 * Uses all host threads. */
r3dgpu_status r3dgpu_synth_pair(const r3dgpu_synth_params* params, uint8_t* left, uint8_t* right, float* gt);

#ifdef __cplusplus
}
#endif

#endif /* R3DGPU_SYNTH_H */
