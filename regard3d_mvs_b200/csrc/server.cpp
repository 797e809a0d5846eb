// Serving loop (include/r3dgpu_server.h): a FIFO of pair requests with host
// buffers, drained by worker threads that each own a CUDA stream, a device
// staging buffer and (through the matcher's per-thread workspace) their own
// level data and SGM scratch. A worker admits the oldest queued requests
// whose estimated device memory fits beside the requests already running,
// stages their inputs, matches them with one batch call on its stream and
// copies the maps back; another worker can meanwhile admit the requests that
// arrived later, so batches overlap on the device (continuous batching).
// Requests are admitted in arrival order: a request that does not fit waits
// until running ones complete, and later ones wait behind it. Images that a
// request names by content key are kept on the device in an LRU cache and
// uploaded once while they stay cached.
#include <chrono>
#include <condition_variable>
#include <deque>
#include <list>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/r3dgpu_server.h"
#include "common.cuh"
#include "matcher_internal.h"

namespace r3dgpu {
namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// Device memory a request holds while it runs: its staged images, masks and
// maps, and the matcher's level data (pyramids, Census images of both
// directions, ranges, tile maps, blended maps), about 160 bytes per pixel of
// the wider image summed over the pyramid.
uint64_t request_bytes(const r3dgpu_request& r) {
  const uint64_t w = static_cast<uint64_t>(std::max(r.left.width, r.right.width));
  const uint64_t h = static_cast<uint64_t>(std::max(r.left.height, 0));
  return 160 * w * h + (uint64_t{1} << 20);
}

struct Request {
  uint64_t ticket = 0;
  r3dgpu_request req{};
  uint64_t bytes = 0;
  Clock::time_point submitted, admitted, done;
  r3dgpu_status status = R3DGPU_OK;
  std::string error;
  bool finished = false;
  int batch_size = 0;
  int worker = -1;
  int cache_hits = 0;
  uint64_t uploaded = 0;
};

// A device copy of a keyed input image.
struct CacheEntry {
  uint16_t* data = nullptr;  // width x height, dense rows
  int width = 0, height = 0;
  size_t bytes = 0;
  int users = 0;                // batches reading it now
  cudaEvent_t ready = nullptr;  // recorded after its upload
  std::list<uint64_t>::iterator lru;
};

using RequestPtr = std::shared_ptr<Request>;

r3dgpu_pair as_pair(const r3dgpu_request& r) {
  r3dgpu_pair p{};
  p.left = r.left;
  p.right = r.right;
  p.left_valid = r.left_valid;
  p.right_valid = r.right_valid;
  p.disparity_min = r.disparity_min;
  p.num_disparities = r.num_disparities;
  p.options = r.options;
  p.out = r.out;
  return p;
}

bool has_mask(const r3dgpu_view_u8& v) { return v.data != nullptr && v.width > 0 && v.height > 0; }

}  // namespace
}  // namespace r3dgpu

using namespace r3dgpu;

struct r3dgpu_server {
  r3dgpu_server_config cfg{};
  std::mutex mu;
  std::condition_variable work_cv;  // queue grew, memory freed, or stop
  std::condition_variable done_cv;  // a request finished
  std::deque<RequestPtr> queue;
  std::unordered_map<uint64_t, RequestPtr> tickets;
  uint64_t next_ticket = 1;
  uint64_t inflight = 0;  // bytes of the admitted, unfinished requests
  int running = 0;
  bool stop = false;
  std::vector<std::thread> threads;
  // Keyed image cache (its own lock: workers stage while others admit).
  std::mutex cache_mu;
  std::unordered_map<uint64_t, CacheEntry> cache;
  std::list<uint64_t> lru;  // least recently used first
  uint64_t cache_bytes = 0;

  // The device copy of a keyed image for a batch on stream st, uploaded on
  // st if it is not cached; `hit` tells which. Null when the image is not
  // cached and cannot be (no key, no cache, a key seen with another size, or
  // no room beside the images in use): the caller stages it itself.
  const uint16_t* cache_acquire(uint64_t key, const r3dgpu_view_u16& v, cudaStream_t st, bool& hit) {
    hit = false;
    if (key == 0 || cfg.cache_budget == 0) return nullptr;
    std::lock_guard<std::mutex> lk(cache_mu);
    auto it = cache.find(key);
    if (it != cache.end()) {
      CacheEntry& e = it->second;
      if (e.width != v.width || e.height != v.height) return nullptr;
      if (cudaStreamWaitEvent(st, e.ready, 0) != cudaSuccess) {
        (void)cudaGetLastError();
        return nullptr;
      }
      ++e.users;
      lru.splice(lru.end(), lru, e.lru);
      hit = true;
      return e.data;
    }
    const size_t bytes = 2 * static_cast<size_t>(v.width) * static_cast<size_t>(v.height);
    if (bytes > cfg.cache_budget) return nullptr;
    for (auto li = lru.begin(); cache_bytes + bytes > cfg.cache_budget && li != lru.end();) {
      auto ci = cache.find(*li);
      if (ci->second.users == 0) {
        // cudaFree waits for the device; entries in use are never freed.
        (void)cudaFree(ci->second.data);
        (void)cudaEventDestroy(ci->second.ready);
        cache_bytes -= ci->second.bytes;
        cache.erase(ci);
        li = lru.erase(li);
      } else {
        ++li;
      }
    }
    if (cache_bytes + bytes > cfg.cache_budget) return nullptr;
    CacheEntry e;
    if (cudaMalloc(reinterpret_cast<void**>(&e.data), bytes) != cudaSuccess) {
      (void)cudaGetLastError();
      return nullptr;
    }
    if (cudaEventCreateWithFlags(&e.ready, cudaEventDisableTiming) != cudaSuccess ||
        cudaMemcpy2DAsync(e.data, 2 * static_cast<size_t>(v.width), v.data, 2 * static_cast<size_t>(v.stride),
                          2 * static_cast<size_t>(v.width), v.height, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaEventRecord(e.ready, st) != cudaSuccess) {
      (void)cudaGetLastError();
      (void)cudaStreamSynchronize(st);
      (void)cudaFree(e.data);
      if (e.ready != nullptr) (void)cudaEventDestroy(e.ready);
      return nullptr;
    }
    e.width = v.width;
    e.height = v.height;
    e.bytes = bytes;
    e.users = 1;
    e.lru = lru.insert(lru.end(), key);
    cache_bytes += bytes;
    const uint16_t* data = e.data;
    cache.emplace(key, e);
    return data;
  }

  void cache_release(const std::vector<uint64_t>& keys) {
    std::lock_guard<std::mutex> lk(cache_mu);
    for (uint64_t k : keys) {
      auto it = cache.find(k);
      if (it != cache.end() && it->second.users > 0) --it->second.users;
    }
  }

  void cache_clear() {
    std::lock_guard<std::mutex> lk(cache_mu);
    for (auto& kv : cache) {
      (void)cudaFree(kv.second.data);
      (void)cudaEventDestroy(kv.second.ready);
    }
    cache.clear();
    lru.clear();
    cache_bytes = 0;
  }

  bool can_admit() const {
    return !queue.empty() && (inflight == 0 || inflight + queue.front()->bytes <= cfg.hbm_budget);
  }

  // Stages the batch's inputs in `io`, matches, copies the maps back.
  // Returns the batch call's status; the message is on this thread.
  r3dgpu_status run(std::vector<RequestPtr>& batch, cudaStream_t st, DeviceBuffer<unsigned char>& io) {
    std::vector<uint64_t> used;  // cache entries this batch reads, released once it ran
    struct Release {
      r3dgpu_server* s;
      std::vector<uint64_t>& keys;
      ~Release() { s->cache_release(keys); }
    } release{this, used};
    size_t total = 0;
    auto room = [](size_t n) { return (n + 255) & ~static_cast<size_t>(255); };
    for (const RequestPtr& r : batch) {
      const r3dgpu_request& q = r->req;
      const size_t wl = static_cast<size_t>(q.left.width), wr = static_cast<size_t>(q.right.width),
                   h = static_cast<size_t>(q.left.height);
      total += room(2 * wl * h) + room(2 * wr * h) + room(has_mask(q.left_valid) ? wl * h : 0) +
               room(has_mask(q.right_valid) ? wr * h : 0) + 2 * room(4 * wl * h);
    }
    try {
      io.reserve(total);
    } catch (const Error& e) {
      set_thread_error(e.what());
      return e.status;
    }
    unsigned char* p = io.get();
    auto take = [&](size_t n) {
      unsigned char* at = p;
      p += room(n);
      return at;
    };
    std::vector<r3dgpu_pair> pairs(batch.size());
    for (size_t i = 0; i < batch.size(); ++i) {
      const r3dgpu_request& q = batch[i]->req;
      const int wl = q.left.width, wr = q.right.width, h = q.left.height;
      r3dgpu_pair& d = pairs[i];
      d = as_pair(q);
      Request& rq = *batch[i];
      rq.cache_hits = 0;
      rq.uploaded = 0;
      // Each image: the cached device copy of its key, or a staged copy.
      auto image = [&](uint64_t key, const r3dgpu_view_u16& v) -> const uint16_t* {
        bool hit = false;
        const uint16_t* c = cache_acquire(key, v, st, hit);
        if (c != nullptr) {
          used.push_back(key);
          if (hit) ++rq.cache_hits;
          else rq.uploaded += 2 * static_cast<uint64_t>(v.width) * v.height;
          return c;
        }
        auto* dv = reinterpret_cast<uint16_t*>(take(2 * static_cast<size_t>(v.width) * v.height));
        if (cudaMemcpy2DAsync(dv, 2 * static_cast<size_t>(v.width), v.data, 2 * static_cast<size_t>(v.stride),
                              2 * static_cast<size_t>(v.width), v.height, cudaMemcpyHostToDevice, st) != cudaSuccess)
          return nullptr;
        rq.uploaded += 2 * static_cast<uint64_t>(v.width) * v.height;
        return dv;
      };
      const uint16_t* dl = image(q.left_key, q.left);
      const uint16_t* dr = dl != nullptr ? image(q.right_key, q.right) : nullptr;
      if (dl == nullptr || dr == nullptr) {
        set_thread_error(std::string("server: image upload: ") + cudaGetErrorString(cudaGetLastError()));
        return R3DGPU_EDEVICE;
      }
      d.left = r3dgpu_view_u16{dl, wl, h, wl};
      d.right = r3dgpu_view_u16{dr, wr, h, wr};
      if (has_mask(q.left_valid)) {
        uint8_t* m = take(static_cast<size_t>(wl) * h);
        if (cudaMemcpy2DAsync(m, wl, q.left_valid.data, q.left_valid.stride, wl, h, cudaMemcpyHostToDevice, st) !=
            cudaSuccess) {
          set_thread_error(std::string("server: mask upload: ") + cudaGetErrorString(cudaGetLastError()));
          return R3DGPU_EDEVICE;
        }
        d.left_valid = r3dgpu_view_u8{m, wl, h, wl};
      }
      if (has_mask(q.right_valid)) {
        uint8_t* m = take(static_cast<size_t>(wr) * h);
        if (cudaMemcpy2DAsync(m, wr, q.right_valid.data, q.right_valid.stride, wr, h, cudaMemcpyHostToDevice, st) !=
            cudaSuccess) {
          set_thread_error(std::string("server: mask upload: ") + cudaGetErrorString(cudaGetLastError()));
          return R3DGPU_EDEVICE;
        }
        d.right_valid = r3dgpu_view_u8{m, wr, h, wr};
      }
      d.out.disparity = reinterpret_cast<float*>(take(4 * static_cast<size_t>(wl) * h));
      d.out.confidence = q.out.confidence ? reinterpret_cast<float*>(take(4 * static_cast<size_t>(wl) * h)) : nullptr;
      d.out.stride = wl;
    }
    const r3dgpu_status st_batch = r3dgpu_match_stereo_batch(pairs.data(), static_cast<int32_t>(pairs.size()), st);
    if (st_batch != R3DGPU_OK) return st_batch;
    for (size_t i = 0; i < batch.size(); ++i) {
      r3dgpu_request& q = batch[i]->req;
      const int wl = q.left.width, h = q.left.height;
      if (cudaMemcpy2DAsync(q.out.disparity, 4 * q.out.stride, pairs[i].out.disparity, 4 * wl, 4 * wl, h,
                            cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          (q.out.confidence && cudaMemcpy2DAsync(q.out.confidence, 4 * q.out.stride, pairs[i].out.confidence, 4 * wl,
                                                 4 * wl, h, cudaMemcpyDeviceToHost, st) != cudaSuccess)) {
        set_thread_error(std::string("server: map download: ") + cudaGetErrorString(cudaGetLastError()));
        return R3DGPU_EDEVICE;
      }
      q.out.disparity_min = pairs[i].out.disparity_min;
      q.out.num_disparities = pairs[i].out.num_disparities;
      q.out.levels = pairs[i].out.levels;
      q.out.cells = pairs[i].out.cells;
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) {
      set_thread_error(std::string("server: ") + cudaGetErrorString(cudaGetLastError()));
      return R3DGPU_EDEVICE;
    }
    return R3DGPU_OK;
  }

  void worker(int index, cudaStream_t st) {
    DeviceBuffer<unsigned char> io;
    while (true) {
      std::vector<RequestPtr> batch;
      {
        std::unique_lock<std::mutex> lk(mu);
        work_cv.wait(lk, [&] { return can_admit() || (stop && queue.empty()); });
        if (!can_admit()) break;  // stopping with an empty queue
        const auto now = Clock::now();
        // A worker's level data live in its own grow-only workspace, which
        // keeps the memory of the largest batch it ran; a batch is therefore
        // also held to the worker's share of the budget, so that what all
        // workers keep stays within it (a larger single request runs alone).
        const uint64_t share = cfg.hbm_budget / static_cast<uint64_t>(cfg.workers);
        uint64_t mine = 0;
        while (!queue.empty() && static_cast<int>(batch.size()) < cfg.max_batch) {
          const RequestPtr& r = queue.front();
          if ((inflight > 0 || !batch.empty()) && inflight + r->bytes > cfg.hbm_budget) break;
          if (!batch.empty() && mine + r->bytes > share) break;
          mine += r->bytes;
          inflight += r->bytes;
          r->admitted = now;
          r->worker = index;
          batch.push_back(r);
          queue.pop_front();
        }
        running += static_cast<int>(batch.size());
      }
      for (RequestPtr& r : batch) r->batch_size = static_cast<int>(batch.size());
      r3dgpu_status status = run(batch, st, io);
      if (status != R3DGPU_OK && batch.size() > 1) {
        // One request's failure must not fail the others: run each alone.
        for (RequestPtr& r : batch) {
          std::vector<RequestPtr> one{r};
          r->status = run(one, st, io);
          r->error = r->status == R3DGPU_OK ? std::string() : std::string(r3dgpu_last_error());
        }
      } else {
        for (RequestPtr& r : batch) {
          r->status = status;
          r->error = status == R3DGPU_OK ? std::string() : std::string(r3dgpu_last_error());
        }
      }
      {
        std::lock_guard<std::mutex> lk(mu);
        const auto now = Clock::now();
        for (RequestPtr& r : batch) {
          r->done = now;
          r->finished = true;
          inflight -= r->bytes;
        }
        running -= static_cast<int>(batch.size());
      }
      done_cv.notify_all();
      work_cv.notify_all();
    }
  }
};

extern "C" {

r3dgpu_status r3dgpu_server_create(const r3dgpu_server_config* config, r3dgpu_server** out) {
  if (config == nullptr || out == nullptr) {
    set_thread_error("server: null argument");
    return R3DGPU_EINVAL;
  }
  if (config->workers < 1 || config->max_batch < 1 || config->hbm_budget == 0) {
    set_thread_error("server: workers and max_batch must be >= 1 and hbm_budget > 0");
    return R3DGPU_EINVAL;
  }
  auto srv = std::make_unique<r3dgpu_server>();
  srv->cfg = *config;
  const size_t scratch = config->scratch_budget != 0 ? config->scratch_budget : size_t{16} << 30;
  // Every worker selects the device and creates its stream before the
  // server is handed out; a worker that cannot reports here.
  std::mutex init_mu;
  std::condition_variable init_cv;
  int ready = 0;
  r3dgpu_status init_status = R3DGPU_OK;
  std::string init_error;
  for (int i = 0; i < config->workers; ++i) {
    srv->threads.emplace_back([&, i, scratch, s = srv.get()] {
      cudaStream_t st = nullptr;
      r3dgpu_status status = r3dgpu_set_device(s->cfg.device);
      std::string err = status == R3DGPU_OK ? "" : r3dgpu_last_error();
      if (status == R3DGPU_OK && cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
        status = R3DGPU_EDEVICE;
        err = std::string("server: stream: ") + cudaGetErrorString(cudaGetLastError());
      }
      set_thread_scratch_budget(scratch);
      {
        std::lock_guard<std::mutex> lk(init_mu);
        if (status != R3DGPU_OK && init_status == R3DGPU_OK) {
          init_status = status;
          init_error = err;
        }
        ++ready;
        init_cv.notify_all();  // under the lock: the creator's locals die once it sees `ready`
      }
      if (status == R3DGPU_OK) s->worker(i, st);
      if (st != nullptr) cudaStreamDestroy(st);
    });
  }
  {
    std::unique_lock<std::mutex> lk(init_mu);
    init_cv.wait(lk, [&] { return ready == config->workers; });
  }
  if (init_status != R3DGPU_OK) {
    {
      std::lock_guard<std::mutex> lk(srv->mu);
      srv->stop = true;
    }
    srv->work_cv.notify_all();
    for (auto& t : srv->threads) t.join();
    set_thread_error(init_error);
    return init_status;
  }
  set_thread_error("");
  *out = srv.release();
  return R3DGPU_OK;
}

r3dgpu_status r3dgpu_server_submit(r3dgpu_server* server, const r3dgpu_request* request, uint64_t* ticket) {
  if (server == nullptr || request == nullptr || ticket == nullptr) {
    set_thread_error("server: null argument");
    return R3DGPU_EINVAL;
  }
  try {
    validate_request(as_pair(*request));
  } catch (const Error& e) {
    set_thread_error(e.what());
    return e.status;
  }
  auto r = std::make_shared<Request>();
  r->req = *request;
  r->bytes = request_bytes(*request);
  r->submitted = Clock::now();
  {
    std::lock_guard<std::mutex> lk(server->mu);
    if (server->stop) {
      set_thread_error("server: stopping");
      return R3DGPU_ECANCELLED;
    }
    r->ticket = server->next_ticket++;
    server->tickets[r->ticket] = r;
    server->queue.push_back(r);
    *ticket = r->ticket;
  }
  server->work_cv.notify_one();
  set_thread_error("");
  return R3DGPU_OK;
}

r3dgpu_status r3dgpu_server_wait(r3dgpu_server* server, uint64_t ticket, double timeout_ms, r3dgpu_request* request,
                                 r3dgpu_request_times* times) {
  if (server == nullptr) {
    set_thread_error("server: null argument");
    return R3DGPU_EINVAL;
  }
  RequestPtr r;
  {
    std::unique_lock<std::mutex> lk(server->mu);
    auto it = server->tickets.find(ticket);
    if (it == server->tickets.end()) {
      set_thread_error("server: unknown ticket " + std::to_string(ticket));
      return R3DGPU_EINVAL;
    }
    r = it->second;
    auto done = [&] { return r->finished; };
    if (timeout_ms < 0) {
      server->done_cv.wait(lk, done);
    } else if (!server->done_cv.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), done)) {
      set_thread_error("server: request " + std::to_string(ticket) + " still running");
      return R3DGPU_ETIMEOUT;
    }
    server->tickets.erase(it);
  }
  if (request != nullptr) {
    request->out.disparity_min = r->req.out.disparity_min;
    request->out.num_disparities = r->req.out.num_disparities;
    request->out.levels = r->req.out.levels;
    request->out.cells = r->req.out.cells;
  }
  if (times != nullptr) {
    times->queued_ms = ms_between(r->submitted, r->admitted);
    times->run_ms = ms_between(r->admitted, r->done);
    times->total_ms = ms_between(r->submitted, r->done);
    times->device_bytes = r->bytes;
    times->batch_size = r->batch_size;
    times->worker = r->worker;
    times->cache_hits = r->cache_hits;
    times->reserved = 0;
    times->uploaded_bytes = r->uploaded;
  }
  set_thread_error(r->error);
  return r->status;
}

int32_t r3dgpu_server_pending(r3dgpu_server* server) {
  if (server == nullptr) return 0;
  std::lock_guard<std::mutex> lk(server->mu);
  return static_cast<int32_t>(server->queue.size()) + server->running;
}

r3dgpu_status r3dgpu_server_destroy(r3dgpu_server* server) {
  if (server == nullptr) return R3DGPU_OK;
  {
    std::lock_guard<std::mutex> lk(server->mu);
    server->stop = true;
  }
  server->work_cv.notify_all();
  for (auto& t : server->threads) t.join();
  if (server->cfg.cache_budget != 0 && r3dgpu_set_device(server->cfg.device) == R3DGPU_OK) server->cache_clear();
  delete server;
  set_thread_error("");
  return R3DGPU_OK;
}

}  // extern "C"
