/*
 * r3dgpu — B200-native Census+SGM stereo matcher, C ABI.
 *
 * Drop-in replacement for the matcher of R3DMVS (rhiestan/Regard3D_MVS):
 * every entry point below names the reference interface it replaces
 * (path within the reference project, file:line). The library computes on
 * the GPU only; there is no CPU fallback. Every call returns an r3dgpu_status
 * and leaves a thread-local message for r3dgpu_last_error().
 *
 * Images are non-owning strided views (the reference's ImageView,
 * src/r3d/core/image.hpp:15-60): `stride` is in elements. Entry points whose
 * name ends in _host take host pointers and copy inside the call; the others
 * take device pointers.
 */
#ifndef R3DGPU_H
#define R3DGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (the reference throws r3d::Error / r3d::Cancelled /
 * std::bad_alloc at the same points, src/r3d/core/error.hpp:10-30,
 * src/r3d/core/cancel.hpp:9-13). */
typedef enum r3dgpu_status {
  R3DGPU_OK = 0,
  R3DGPU_EINVAL = 1,     /* invalid options, sizes or ranges (r3d::Error) */
  R3DGPU_ECANCELLED = 2, /* cancellation requested (r3d::Cancelled) */
  R3DGPU_ENOMEM = 3,     /* device or host allocation failed (std::bad_alloc) */
  R3DGPU_EDEVICE = 4,    /* CUDA error, or no usable sm_100 device */
  R3DGPU_ETIMEOUT = 5,   /* a bounded device-side wait gave up */
  R3DGPU_EUNSUPPORTED = 6 /* valid input beyond this build's limits (e.g. labels per pixel) */
} r3dgpu_status;

/* SubpixelMethod, src/r3d/stereo/stereo_matcher.hpp:23-27 (same order). */
enum { R3DGPU_SUBPIXEL_NONE = 0, R3DGPU_SUBPIXEL_PARABOLA = 1, R3DGPU_SUBPIXEL_EQUIANGULAR = 2 };

/* StereoOptions, src/r3d/stereo/stereo_matcher.hpp:30-57: same fields, same
 * meaning, same defaults (r3dgpu_default_options). `scalar_kernels` is kept
 * for layout parity and ignored. */
typedef struct r3dgpu_stereo_options {
  int32_t p1;
  int32_t p2;
  int32_t p2_adapt;
  int32_t invalid_cost;
  int32_t subpixel;
  float uniqueness;
  int32_t lr_max_diff;
  int32_t lr_full_match;
  int32_t speckle_size;
  float speckle_diff;
  int32_t median;
  int32_t levels;
  int32_t range_radius;
  int32_t range_margin;
  int32_t range_fill;
  int32_t tile_size;
  int32_t tile_margin;
  int32_t tile_blend;
  uint64_t memory_budget;
  int32_t scalar_kernels;
  int32_t reserved;
} r3dgpu_stereo_options;

/* ImageView<const T> (src/r3d/core/image.hpp:15-60), single channel. A view
 * with data == NULL or a zero size is "empty" (masks: all pixels valid). */
typedef struct r3dgpu_view_u16 {
  const uint16_t* data;
  int32_t width;
  int32_t height;
  int64_t stride;
} r3dgpu_view_u16;

typedef struct r3dgpu_view_u8 {
  const uint8_t* data;
  int32_t width;
  int32_t height;
  int64_t stride;
} r3dgpu_view_u8;

/* DisparityMap, src/r3d/stereo/stereo_matcher.hpp:61-68. The caller owns
 * `disparity` and `confidence` (width x height floats, row stride `stride`
 * elements, host memory for _host calls, device memory otherwise);
 * confidence may be NULL. Invalid disparities are +inf. */
typedef struct r3dgpu_disparity_map {
  float* disparity;
  float* confidence;
  int64_t stride;
  int32_t disparity_min;   /* out */
  int32_t num_disparities; /* out: rounded up to 16 */
  int32_t levels;          /* out: coarser pyramid levels used */
  int32_t reserved;
  uint64_t cells;          /* out: aggregated (pixel, label) cells, all levels, both directions */
} r3dgpu_disparity_map;

/* Message of the last failed call on this thread ("" after success). */
const char* r3dgpu_last_error(void);

/* Reference defaults (StereoOptions{}). */
void r3dgpu_default_options(r3dgpu_stereo_options* out);

/* Number of coarser levels chosen by levels = -1.
 * Replaces r3d::detail::automatic_levels, src/r3d/stereo/stereo_matcher.cpp:1105-1122. */
int32_t r3dgpu_automatic_levels(int32_t width, int32_t height, int32_t num_disparities);

/* Selects the CUDA device used by this thread's later calls (default 0). */
r3dgpu_status r3dgpu_set_device(int32_t device);

/* Cancellation token, the counterpart of the reference's per-thread
 * CancelToken (src/r3d/core/cancel.hpp:36-55, polled before every tile chunk
 * at src/r3d/core/thread_pool.cpp:53-55). A token is a flag in page-locked
 * host memory mapped into the device's address space. r3dgpu_cancel sets it
 * (from any thread); the matcher entry points of a thread that attached it
 * with r3dgpu_set_cancel_token poll it on the host between hierarchy rounds
 * and waves of tiles, and the SGM chain kernels read it once per chain block
 * (a plain read, never a wait), so work already enqueued drains within one
 * block. A call that sees the flag returns R3DGPU_ECANCELLED after its
 * enqueued work has finished; its outputs are then unspecified, and the
 * device and the library stay usable. r3dgpu_cancel_token_reset clears the
 * flag for the next call. */
typedef struct r3dgpu_cancel_token r3dgpu_cancel_token;
r3dgpu_status r3dgpu_cancel_token_create(r3dgpu_cancel_token** out);
void r3dgpu_cancel_token_destroy(r3dgpu_cancel_token* token);
void r3dgpu_cancel(r3dgpu_cancel_token* token);
void r3dgpu_cancel_token_reset(r3dgpu_cancel_token* token);
int32_t r3dgpu_cancel_requested(const r3dgpu_cancel_token* token);
/* Attaches a token to this thread's later calls (NULL detaches). */
void r3dgpu_set_cancel_token(r3dgpu_cancel_token* token);

/* Matches a rectified pair (host images, host outputs; copies inside).
 * Replaces r3d::match_stereo, src/r3d/stereo/stereo_matcher.hpp:82-85
 * (implementation src/r3d/stereo/stereo_matcher.cpp:1023-1095). */
r3dgpu_status r3dgpu_match_stereo_host(const r3dgpu_view_u16* left, const r3dgpu_view_u16* right,
                                       const r3dgpu_view_u8* left_valid, const r3dgpu_view_u8* right_valid,
                                       int32_t disparity_min, int32_t num_disparities,
                                       const r3dgpu_stereo_options* options, r3dgpu_disparity_map* out);

/* Same with device-resident images and outputs; runs on `stream`
 * (cudaStream_t, NULL = legacy default stream) and synchronises it. */
r3dgpu_status r3dgpu_match_stereo(const r3dgpu_view_u16* left, const r3dgpu_view_u16* right,
                                  const r3dgpu_view_u8* left_valid, const r3dgpu_view_u8* right_valid,
                                  int32_t disparity_min, int32_t num_disparities,
                                  const r3dgpu_stereo_options* options, r3dgpu_disparity_map* out, void* stream);

/* One pair of a batch (device pointers). */
typedef struct r3dgpu_pair {
  r3dgpu_view_u16 left;
  r3dgpu_view_u16 right;
  r3dgpu_view_u8 left_valid;
  r3dgpu_view_u8 right_valid;
  int32_t disparity_min;
  int32_t num_disparities;
  r3dgpu_stereo_options options;
  r3dgpu_disparity_map out;
} r3dgpu_pair;

/* Matches many pairs of uneven size, range and hierarchy depth together:
 * every stage runs once for all pairs (one launch per stage, tiles of all
 * pairs in one persistent work queue). Results equal r3dgpu_match_stereo per
 * pair. No reference counterpart: the reference matches pairs one at a time
 * (src/r3d/mvs/multi_stereo.cpp:264-293). */
r3dgpu_status r3dgpu_match_stereo_batch(r3dgpu_pair* pairs, int32_t count, void* stream);

/* Census image, 62 bits per pixel (device pointers; out stride in elements).
 * Replaces r3d::census_transform, src/r3d/stereo/census.hpp:20. */
r3dgpu_status r3dgpu_census_transform(const r3dgpu_view_u16* image, uint64_t* out, int64_t out_stride,
                                      void* stream);

/* One 2x binomial pyramid reduction of a 16-bit image (device pointers).
 * Replaces r3d::pyramid_down<uint16_t>, src/r3d/core/pyramid.hpp:21-22. */
r3dgpu_status r3dgpu_pyramid_down_u16(const r3dgpu_view_u16* image, uint16_t* out, int64_t out_stride,
                                      void* stream);

/* Aggregated volume of the whole image as one tile (host images; out holds
 * the labels of every pixel in row-major pixel order; `out_capacity` is its
 * length in elements; `out_count` receives the cell count). ranges_lo /
 * ranges_num: per-pixel label ranges (width x height, contiguous) or NULL.
 * Replaces r3d::detail::sgm_cost_volume, src/r3d/stereo/stereo_matcher.hpp:98-101. */
r3dgpu_status r3dgpu_sgm_cost_volume_host(const r3dgpu_view_u16* left, const r3dgpu_view_u16* right,
                                          int32_t disparity_min, int32_t num_disparities,
                                          const r3dgpu_stereo_options* options, const uint16_t* ranges_lo,
                                          const uint16_t* ranges_num, uint16_t* out, uint64_t out_capacity,
                                          uint64_t* out_count);

/* Label ranges from the next coarser level (host arrays, contiguous).
 * Replaces r3d::detail::ranges_from_coarse, src/r3d/stereo/stereo_matcher.hpp:121-125. */
r3dgpu_status r3dgpu_ranges_from_coarse_host(const float* coarse, int32_t coarse_width, int32_t coarse_height,
                                             int32_t width, int32_t height, const uint8_t* fine_valid,
                                             const uint8_t* partner_valid, int32_t partner_width,
                                             int32_t partner_sign, int32_t disparity_min,
                                             int32_t num_disparities, const r3dgpu_stereo_options* options,
                                             int32_t mirrored, uint16_t* lo_out, uint16_t* num_out);

/* Speckle filter in place (host array, contiguous).
 * Replaces r3d::remove_speckles, src/r3d/stereo/stereo_matcher.hpp:89. */
r3dgpu_status r3dgpu_remove_speckles_host(float* disparity, int32_t width, int32_t height, int32_t min_size,
                                          float max_diff);

/* Speckle filter in place on a DEVICE map (contiguous, width * height floats)
 * that allocates no GPU memory: no reference counterpart. It is for callers
 * that cannot let the library call cudaMalloc -- an application whose own
 * pool allocator owns the device's memory, or a pipeline that cannot take the
 * device-wide synchronisation of cudaFree. The union-find scratch is a static
 * device array of 32 MiB that every GPU using this entry point holds until the
 * process exits; maps above 4,194,304 pixels (2048 x 2048) are rejected with
 * R3DGPU_EINVAL. Like every other entry point it runs on the device this
 * thread chose with r3dgpu_set_device (device 0 by default) and makes that
 * device current; the map must be device (or managed) memory of that device,
 * otherwise R3DGPU_EINVAL before any launch. The work is enqueued on `stream`
 * (cudaStream_t of that device, NULL = legacy default stream) without
 * synchronising it; launch errors are returned, errors during execution
 * surface at the caller's next synchronisation. Set-up: the first call on a
 * device looks up the array's device address there, which (under CUDA's lazy
 * module loading, the default) loads the module and reserves the 32 MiB at
 * that moment; a device without room answers R3DGPU_ENOMEM. Make that first
 * call -- a call with width = height = 0 does only the set-up -- before the
 * caller's pool takes the device's memory and before any stream capture on
 * the device. All calls share the one array, so calls whose work overlaps on
 * the GPU (different streams or host threads without ordering between them)
 * race: order them on one stream or synchronise between them. Results equal
 * r3dgpu_remove_speckles_host's. */
r3dgpu_status r3dgpu_remove_speckles_no_alloc(float* disparity, int32_t width, int32_t height, int32_t min_size,
                                              float max_diff, void* stream);

/* 3x3 median of the valid disparities (host arrays, contiguous).
 * Replaces r3d::median_filter_3x3, src/r3d/stereo/stereo_matcher.hpp:91. */
r3dgpu_status r3dgpu_median_filter_3x3_host(const float* disparity, int32_t width, int32_t height, float* out);

/* ------------------------------------------------------------------ rectification
 * Resampling of a source image into a rectified (or any rotated pinhole)
 * camera with the same centre: Catmull-Rom bicubic sampling of the source
 * (of a pyramid level of it when the target has less than 1/1.5 of its
 * resolution), pixels without a source 0, an optional validity mask (255 /
 * 0). Replaces r3d::rectify_image, src/r3d/rectify/rectification.hpp:75-88
 * (implementation src/r3d/rectify/rectification.cpp:287-350), for single
 * channel u16 and f32 images. */

/* CameraIntrinsics, src/r3d/core/camera_model.hpp:32-41; model: 0 pinhole,
 * 1 radial_k1, 2 radial_k3, 3 brown_t2, 4 fisheye (params as there). */
typedef struct r3dgpu_camera {
  int32_t model;
  int32_t width;
  int32_t height;
  int32_t reserved;
  double fx, fy, cx, cy;
  double params[5];
} r3dgpu_camera;

/* PinholeIntrinsics of the target camera. */
typedef struct r3dgpu_pinhole {
  int32_t width;
  int32_t height;
  double fx, fy, cx, cy;
} r3dgpu_pinhole;

/* source_from_target: R_source R_target^T (row-major), the rotation that
 * takes target camera rays to source camera rays. Device images; `valid` may
 * be NULL; runs on `stream` and synchronises it. */
r3dgpu_status r3dgpu_rectify_image_u16(const r3dgpu_view_u16* src, const r3dgpu_camera* cam,
                                       const double* source_from_target, const r3dgpu_pinhole* target, uint16_t* out,
                                       int64_t out_stride, uint8_t* valid, int64_t valid_stride, void* stream);
r3dgpu_status r3dgpu_rectify_image_f32(const float* src, int64_t src_stride, const r3dgpu_camera* cam,
                                       const double* source_from_target, const r3dgpu_pinhole* target, float* out,
                                       int64_t out_stride, uint8_t* valid, int64_t valid_stride, void* stream);
/* Same with host images (copies inside). */
r3dgpu_status r3dgpu_rectify_image_u16_host(const r3dgpu_view_u16* src, const r3dgpu_camera* cam,
                                            const double* source_from_target, const r3dgpu_pinhole* target,
                                            uint16_t* out, int64_t out_stride, uint8_t* valid, int64_t valid_stride);
r3dgpu_status r3dgpu_rectify_image_f32_host(const float* src, int64_t src_stride, const r3dgpu_camera* cam,
                                            const double* source_from_target, const r3dgpu_pinhole* target,
                                            float* out, int64_t out_stride, uint8_t* valid, int64_t valid_stride);

/* ------------------------------------------------------------------ multi-view
 * Combination of up to 16 matched pairs that share a base camera into one
 * depth map (the consumer of the matcher in the multi-view stage).
 * Replaces r3d::combine_pairs, src/r3d/mvs/multi_stereo.hpp:43-44
 * (implementation src/r3d/mvs/multi_stereo.cpp:74-216). The caller passes
 * the geometry the reference derives with Eigen from the cameras. */

/* The depth map's grid camera (r3d::PinholeCamera): K^-1 and R^T (row-major)
 * and the centre. */
typedef struct r3dgpu_depth_grid {
  double k_inv[9];
  double rot_t[9];
  double center[3];
  int32_t width;
  int32_t height;
} r3dgpu_depth_grid;

/* One pair (multi_stereo.cpp:24-33 PairGeometry): grid pixel -> rectified
 * left pixel homography K_r R_r R_g^T K_g^-1 (row-major), focal * baseline,
 * disparity offset (cx_left - cx_right), the partner camera's centre, and the
 * pair's disparity map (and confidence, or NULL) in the rectified left image. */
typedef struct r3dgpu_pair_geometry {
  double grid_to_rect[9];
  double fb;
  double offset;
  double partner_center[3];
  const float* disparity;
  const float* confidence;
  int32_t width;
  int32_t height;
  int64_t stride;
} r3dgpu_pair_geometry;

/* MultiStereoOptions, src/r3d/mvs/multi_stereo.hpp:25-30 (same defaults). */
typedef struct r3dgpu_multi_stereo_options {
  double inlier_px;
  double max_reprojection_px;
  double min_angle_deg;
  int32_t min_pairs;
  int32_t reserved;
} r3dgpu_multi_stereo_options;

void r3dgpu_default_multi_stereo_options(r3dgpu_multi_stereo_options* out);

/* Depth (0 = none), confidence and pair mask (bit i: pair i was used) of
 * every grid pixel; maps and outputs in device memory, row stride `stride`
 * elements; runs on `stream` and synchronises it. */
r3dgpu_status r3dgpu_combine_pairs(const r3dgpu_depth_grid* grid, const r3dgpu_pair_geometry* pairs, int32_t count,
                                   const r3dgpu_multi_stereo_options* options, float* depth, float* confidence,
                                   uint16_t* pair_mask, int64_t stride, void* stream);

/* Same with the pairs' maps and the outputs in host memory (copies inside). */
r3dgpu_status r3dgpu_combine_pairs_host(const r3dgpu_depth_grid* grid, const r3dgpu_pair_geometry* pairs,
                                        int32_t count, const r3dgpu_multi_stereo_options* options, float* depth,
                                        float* confidence, uint16_t* pair_mask, int64_t stride);

/* ------------------------------------------------------------------ a view's depth map
 * The multi-view stage for one view on the device: every partner pair is
 * rectified (r3dgpu_rectify_image_u16 of the base and the partner image),
 * all pairs are matched in one batch (r3dgpu_match_stereo_batch) and the
 * matched pairs are combined into the grid's depth map (r3dgpu_combine_pairs);
 * rectified images and disparity maps never leave the device. Replaces the
 * loop of r3d::compute_depth_map, src/r3d/mvs/multi_stereo.hpp:76-79
 * (implementation src/r3d/mvs/multi_stereo.cpp:243-304), from the rectified
 * pairs' geometry (which the caller's compute_rectification provides) on. */
typedef struct r3dgpu_view_pair {
  r3dgpu_view_u16 partner;           /* the partner's image (device memory) */
  r3dgpu_camera partner_camera;
  double base_from_rect[9];          /* R_base R_rect^T, row-major */
  double partner_from_rect[9];       /* R_partner R_rect^T */
  r3dgpu_pinhole left;               /* rectified base camera */
  r3dgpu_pinhole right;              /* rectified partner camera (same height) */
  int32_t disparity_min;
  int32_t num_disparities;
  r3dgpu_pair_geometry geometry;     /* grid_to_rect, fb, offset, partner_center (map pointers ignored) */
} r3dgpu_view_pair;

/* Depth, confidence and pair mask of the grid (device memory, `stride`
 * elements per row) from the base image (device) and up to 16 pairs;
 * *cells (may be NULL) receives the matched cells of all pairs. Runs on
 * `stream` and synchronises it. */
r3dgpu_status r3dgpu_compute_depth_map(const r3dgpu_view_u16* base, const r3dgpu_camera* base_camera,
                                       const r3dgpu_depth_grid* grid, const r3dgpu_view_pair* pairs, int32_t count,
                                       const r3dgpu_stereo_options* stereo,
                                       const r3dgpu_multi_stereo_options* multi, float* depth, float* confidence,
                                       uint16_t* pair_mask, int64_t stride, uint64_t* cells, void* stream);

/* ------------------------------------------------------------------ depth maps
 * Multi-view geometric consistency of depth maps (the step after the
 * combination). Replaces prepare_depth_map, check_consistency,
 * filter_depth_maps, erode_depth_edges, remove_weak_depths,
 * remove_depth_halos and remove_depth_speckles,
 * src/r3d/mvs/consistency.hpp:97-125 (implementation
 * src/r3d/mvs/consistency.cpp:57-487). */

/* PinholeCamera (src/r3d/core/camera.hpp:26-80): intrinsics, pose (R maps
 * world to camera axes, C is the centre; row-major), and K^-1 as the caller
 * computes it (the reference takes Eigen's K().inverse()). */
typedef struct r3dgpu_pinhole_camera {
  r3dgpu_pinhole intrinsics;
  double rotation[9];
  double center[3];
  double k_inv[9];
} r3dgpu_pinhole_camera;

/* DepthMap (src/r3d/mvs/depth_map.hpp:17-41) in device memory (host memory
 * for _host calls). depth 0 = invalid; `support` is written by the check;
 * `color` is RGB interleaved (or NULL: weak-texture and halo removal then do
 * nothing); `stride` is the row stride of depth, confidence, pair_mask and
 * support in elements, `color_stride` that of color in bytes. */
#define R3DGPU_MAX_PARTNERS 16
typedef struct r3dgpu_depth_map {
  r3dgpu_pinhole_camera camera;
  float* depth;
  float* confidence;
  uint16_t* pair_mask;
  uint8_t* support;
  const uint8_t* color;
  int64_t stride;
  int64_t color_stride;
  int32_t width;
  int32_t height;
  uint32_t view;
  uint32_t num_partners;
  uint32_t partners[R3DGPU_MAX_PARTNERS];
} r3dgpu_depth_map;

/* ConsistencyOptions, src/r3d/mvs/consistency.hpp:59-78: same fields, same
 * defaults (r3dgpu_default_consistency_options). max_neighbours belongs to
 * the caller's neighbour selection and is not read here. */
typedef struct r3dgpu_consistency_options {
  double max_relative_depth_error;
  double max_reprojection_px;
  int32_t min_views;
  int32_t min_evidence;
  float min_confidence;
  int32_t edge_erosion;
  double discontinuity;
  int32_t erode_holes;
  int32_t max_neighbours;
  int32_t independent_support;
  int32_t average_depths;
  double weak_texture;
  double weak_segment;
  int32_t reject_weak;
  int32_t halo_px;
  int32_t halo_colour;
  int32_t speckle_size;
  double speckle_step;
} r3dgpu_consistency_options;

/* ConsistencyStats, src/r3d/mvs/consistency.hpp:80-89. */
typedef struct r3dgpu_consistency_stats {
  uint64_t input, unconfident, eroded, rejected, weak, halo, speckles, output;
} r3dgpu_consistency_stats;

void r3dgpu_default_consistency_options(r3dgpu_consistency_options* out);

/* At most this many neighbours per map in one check. */
#define R3DGPU_MAX_NEIGHBOURS 64

/* prepare_depth_map: removes unconfident depths and depth edges in place;
 * counts are added to *stats (may be NULL). Runs on `stream`, synchronises it. */
r3dgpu_status r3dgpu_prepare_depth_map(r3dgpu_depth_map* map, const r3dgpu_consistency_options* options,
                                       r3dgpu_consistency_stats* stats, void* stream);

/* check_consistency: checks `map` against its prepared neighbours (read
 * only), fills map->support, removes unconfirmed depths, weak depths, halos
 * and speckles; counts are added to *stats. */
r3dgpu_status r3dgpu_check_consistency(r3dgpu_depth_map* map, const r3dgpu_depth_map* neighbours, int32_t count,
                                       const r3dgpu_consistency_options* options, r3dgpu_consistency_stats* stats,
                                       void* stream);

/* filter_depth_maps: both steps for all maps in place; the neighbours of
 * map i are maps[neighbour_index[neighbour_offset[i] .. neighbour_offset[i+1])]
 * (count + 1 offsets). All checks read the prepared, unfiltered maps. *stats
 * (may be NULL) is set, not added to. */
r3dgpu_status r3dgpu_filter_depth_maps(r3dgpu_depth_map* maps, int32_t count, const int32_t* neighbour_offset,
                                       const int32_t* neighbour_index, const r3dgpu_consistency_options* options,
                                       r3dgpu_consistency_stats* stats, void* stream);
/* Same with the maps in host memory (copies inside). */
r3dgpu_status r3dgpu_filter_depth_maps_host(r3dgpu_depth_map* maps, int32_t count, const int32_t* neighbour_offset,
                                            const int32_t* neighbour_index,
                                            const r3dgpu_consistency_options* options,
                                            r3dgpu_consistency_stats* stats);

/* The single filters (device maps); *removed receives the pixels removed. */
r3dgpu_status r3dgpu_erode_depth_edges(r3dgpu_depth_map* map, int32_t radius, double discontinuity, int32_t holes,
                                       uint64_t* removed, void* stream);
r3dgpu_status r3dgpu_remove_weak_depths(r3dgpu_depth_map* map, const r3dgpu_consistency_options* options,
                                        uint64_t* removed, void* stream);
r3dgpu_status r3dgpu_remove_depth_halos(r3dgpu_depth_map* map, int32_t max_px, int32_t colour_step,
                                        uint64_t* removed, void* stream);
r3dgpu_status r3dgpu_remove_depth_speckles(r3dgpu_depth_map* map, int32_t min_size, double max_relative_step,
                                           uint64_t* removed, void* stream);

/* Depth-map files (.r3dd, format version 2). Replace write_depth_map and
 * read_depth_map, src/r3d/mvs/depth_map.hpp:57-59 (implementation
 * src/r3d/mvs/depth_map.cpp:135-239): the same bytes, so served maps feed the
 * reference pipeline's --reuse. The map's images are host memory, or device
 * memory when `device` != 0 (copied on `stream` first); NULL images are
 * written as zeros. */
r3dgpu_status r3dgpu_write_depth_map(const char* path, const r3dgpu_depth_map* map, int32_t device, void* stream);
/* Reading takes two calls: _info fills the camera (and K^-1 of its
 * intrinsics), width, height, view and partners without touching the image
 * pointers; the caller allocates host images of that size and
 * r3dgpu_read_depth_map fills the non-NULL ones (at map->stride and
 * map->color_stride). */
r3dgpu_status r3dgpu_read_depth_map_info(const char* path, r3dgpu_depth_map* map);
r3dgpu_status r3dgpu_read_depth_map(const char* path, r3dgpu_depth_map* map);

/* ------------------------------------------------------------------ refinement
 * Patch-based depth refinement: per valid pixel an inverse-depth plane
 * (w, a, b) fitted by Gauss-Newton on 2 - 2 NCC of the window warped into the
 * neighbouring views. Replaces make_refinement_image and refine_depth_map,
 * src/r3d/mvs/refinement.hpp:33-68 (implementation
 * src/r3d/mvs/refinement.cpp:1-451). */

/* RefinementOptions (refinement.hpp:33-44, same defaults), plus `fp32`:
 * 0 computes the window terms in double precision as the reference does;
 * 1 computes them in float (the 3x3 solve stays double). */
typedef struct r3dgpu_refinement_options {
  int32_t radius;
  int32_t step;
  int32_t iterations;
  int32_t max_views;
  double min_ncc;
  double max_shift_px;
  double min_gain;
  double min_texture;
  double blur_sigma;
  int32_t drop_unconfirmed;
  int32_t fp32;
} r3dgpu_refinement_options;

/* RefinementStats (refinement.hpp:46-51). */
typedef struct r3dgpu_refinement_stats {
  uint64_t input, refined, kept, unconfirmed;
} r3dgpu_refinement_stats;

/* RefinementImage (refinement.hpp:53-58): a view's intensity (0..255) and its
 * x / y derivatives, three interleaved floats per pixel on the camera's grid
 * (camera.intrinsics.width x height); `stride` in floats per row. */
typedef struct r3dgpu_refinement_image {
  r3dgpu_pinhole_camera camera;
  const float* data;
  int64_t stride;
} r3dgpu_refinement_image;

void r3dgpu_default_refinement_options(r3dgpu_refinement_options* out);

/* make_refinement_image (refinement.hpp:60-63): gray (width x height,
 * `gray_stride` floats per row), optionally Gaussian-smoothed by blur_sigma
 * pixels, into out (3 floats per pixel, `out_stride` floats per row).
 * Device pointers; runs on `stream` and synchronises it. */
r3dgpu_status r3dgpu_make_refinement_image(const float* gray, int64_t gray_stride, int32_t width, int32_t height,
                                           double blur_sigma, float* out, int64_t out_stride, void* stream);

/* refine_depth_map (refinement.hpp:65-68): refines the depth map (depth and
 * confidence, width x height at `stride` floats per row, on `camera`'s grid)
 * in place; `base` is on the same grid, `views` are the neighbouring images
 * (at most options->max_views, and at most 8, are used). *stats may be NULL.
 * Device pointers; runs on `stream` and synchronises it. */
r3dgpu_status r3dgpu_refine_depth_map(float* depth, float* confidence, int64_t stride,
                                      const r3dgpu_pinhole_camera* camera, int32_t width, int32_t height,
                                      const r3dgpu_refinement_image* base, const r3dgpu_refinement_image* views,
                                      int32_t num_views, const r3dgpu_refinement_options* options,
                                      r3dgpu_refinement_stats* stats, void* stream);
/* Same with host maps and images (copies inside). */
r3dgpu_status r3dgpu_refine_depth_map_host(float* depth, float* confidence, int64_t stride,
                                           const r3dgpu_pinhole_camera* camera, int32_t width, int32_t height,
                                           const r3dgpu_refinement_image* base,
                                           const r3dgpu_refinement_image* views, int32_t num_views,
                                           const r3dgpu_refinement_options* options, r3dgpu_refinement_stats* stats);

/* The depth stage of a set of views in one call (host maps and images):
 * every view refined against its neighbours' refinement images
 * (r3dgpu_refine_depth_map with views = its neighbour list, in order), then
 * r3dgpu_filter_depth_maps of all maps over the same neighbour lists; each
 * image is copied to the device once, and depth, confidence and support come
 * back. The reference runs the two stages view by view
 * (src/r3d/mvs/refinement.hpp:65-68, src/r3d/mvs/consistency.hpp:110-115). */
r3dgpu_status r3dgpu_depth_stage_host(r3dgpu_depth_map* maps, const r3dgpu_refinement_image* images, int32_t count,
                                      const int32_t* neighbour_offset, const int32_t* neighbour_index,
                                      const r3dgpu_refinement_options* refine,
                                      const r3dgpu_consistency_options* consistency,
                                      r3dgpu_refinement_stats* refine_stats,
                                      r3dgpu_consistency_stats* consistency_stats);

/* Frees the device and pinned host buffers that this thread's calls keep on
 * its current device for reuse (they grow to the largest call made so far);
 * the next call allocates them again. No reference counterpart. */
r3dgpu_status r3dgpu_release_workspace(void);

/* Kernel launches issued by this process so far (the library counts its own
 * launches; bench.py reads the difference around a timed region). */
uint64_t r3dgpu_launch_count(void);

/* Device time of the SGM tile kernel, measured with CUDA events on the
 * launching stream around every launch and read after each call's final
 * synchronisation (profiling adds no synchronisation of its own). No
 * reference counterpart (the reference logs wall-clock stage times,
 * src/r3d/stereo/stereo_matcher.cpp:663-677). */
typedef struct r3dgpu_profile {
  double sgm_ms;         /* summed device time of the SGM launches */
  uint64_t sgm_launches; /* SGM launches */
  uint64_t sgm_cells;    /* aggregated (pixel, label) cells of their tiles */
  uint64_t sgm_tiles;    /* tiles processed */
  uint64_t sgm_pixels;   /* tile pixels processed */
} r3dgpu_profile;

/* Enables (1) or disables (0) the accounting on this thread. */
void r3dgpu_profile_enable(int32_t on);
/* Returns the totals accumulated on this thread since the last call and resets them. */
void r3dgpu_profile_take(r3dgpu_profile* out);

/* The launches behind the last r3dgpu_profile_take, one JSON object per
 * launch ({"kernel", "shape", "tiles", "cells", "pixels", "ms", "grid", "rows"}),
 * as a JSON array written into buf (truncated to len - 1 bytes). Returns the
 * full length. */
uint64_t r3dgpu_profile_launches(char* buf, uint64_t len);

#ifdef __cplusplus
}
#endif

#endif /* R3DGPU_H */
