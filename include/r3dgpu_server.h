/* r3dgpu serving loop: a request queue in front of the batch matcher.
 *
 * No reference counterpart: the reference matches the partner pairs of a
 * view one call at a time on the calling thread
 * (src/r3d/mvs/multi_stereo.cpp:264-293). The server accepts pair requests
 * from any thread at any time and runs them in continuous batches: each of
 * `workers` threads owns a CUDA stream and a workspace, takes the oldest
 * queued requests that fit the device-memory budget, matches them with one
 * r3dgpu_match_stereo_batch call and completes them; requests that arrive
 * while batches are on the GPU are admitted by the next free worker, so
 * their work overlaps the running batches on the device. Results equal
 * r3dgpu_match_stereo_host per request, whatever the mix.
 *
 * Residency across requests: a request may name its images by content key
 * (left_key, right_key; 0 = none). The server keeps device copies of keyed
 * images in a cache of cache_budget bytes (least recently used first out,
 * never while a running batch reads them) and uploads a keyed image only
 * when its key is not cached, so the partner pairs of one view, which share
 * the view's image, send it to the device once.
 */
#ifndef R3DGPU_SERVER_H
#define R3DGPU_SERVER_H

#include "r3dgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct r3dgpu_server r3dgpu_server;

typedef struct r3dgpu_server_config {
  int32_t device;            /* CUDA device of every worker */
  int32_t workers;           /* concurrent batches (threads, streams, workspaces), >= 1 */
  int32_t max_batch;         /* requests per batch, >= 1 */
  int32_t reserved;
  uint64_t hbm_budget;       /* bytes of device memory the admitted requests may hold together */
  uint64_t scratch_budget;   /* bytes of SGM scratch per worker, both tracks of a batch together (0: 16 GiB) */
  uint64_t cache_budget;     /* bytes of device memory for keyed input images (0: no cache) */
} r3dgpu_server_config;

/* A request: host images and host outputs, kept alive by the caller until
 * r3dgpu_server_wait returns for its ticket. Fields as in r3dgpu_pair, then
 * the content keys: a nonzero key promises that every request carrying it
 * has the same image (same size and pixels); the server may then use a
 * cached device copy instead of this request's host image. */
typedef struct r3dgpu_request {
  r3dgpu_view_u16 left;
  r3dgpu_view_u16 right;
  r3dgpu_view_u8 left_valid;
  r3dgpu_view_u8 right_valid;
  int32_t disparity_min;
  int32_t num_disparities;
  r3dgpu_stereo_options options;
  r3dgpu_disparity_map out;
  uint64_t left_key;
  uint64_t right_key;
} r3dgpu_request;

/* What happened to a request (milliseconds on the host's steady clock). */
typedef struct r3dgpu_request_times {
  double queued_ms;       /* submit -> admitted into a batch */
  double run_ms;          /* admitted -> completed */
  double total_ms;        /* submit -> completed */
  uint64_t device_bytes;  /* admission estimate of the request's device memory */
  int32_t batch_size;     /* requests in its batch */
  int32_t worker;
  int32_t cache_hits;     /* images of the request served from the cache (0..2) */
  int32_t reserved;
  uint64_t uploaded_bytes; /* host -> device bytes of the request's images */
} r3dgpu_request_times;

/* Starts the workers. hbm_budget must hold the largest single request's
 * estimate for that request to run without others beside it; a request
 * larger than the budget still runs, alone. */
r3dgpu_status r3dgpu_server_create(const r3dgpu_server_config* config, r3dgpu_server** out);

/* Queues a request (copied; its buffers are not). `ticket` receives the id
 * to wait on. Invalid requests are rejected here with R3DGPU_EINVAL. */
r3dgpu_status r3dgpu_server_submit(r3dgpu_server* server, const r3dgpu_request* request, uint64_t* ticket);

/* Waits up to timeout_ms (< 0: forever) for the request, fills `times` (may
 * be NULL) and the request's out fields (disparity_min, num_disparities,
 * levels, cells), and returns the request's own status (its message through
 * r3dgpu_last_error on this thread). R3DGPU_ETIMEOUT leaves the ticket
 * valid; any other status consumes it. */
r3dgpu_status r3dgpu_server_wait(r3dgpu_server* server, uint64_t ticket, double timeout_ms, r3dgpu_request* request,
                                 r3dgpu_request_times* times);

/* Requests queued or running. */
int32_t r3dgpu_server_pending(r3dgpu_server* server);

/* Finishes every queued request, stops the workers and frees the server. */
r3dgpu_status r3dgpu_server_destroy(r3dgpu_server* server);

#ifdef __cplusplus
}
#endif

#endif /* R3DGPU_SERVER_H */
