// Serving: continuous batching of render requests over one path pool.
//
// The reference renders one viewport per WebGL context and frame loop
// (renderer.ts:512-565).  A server keeps up to kMaxJobs requests -- each a
// viewport of a resident scene with its own resolution, spp and settings --
// in the job table of one Engine, so their paths share every extend /
// connect / shade launch.  A driver thread owns the engine's stream and runs:
//   admit    queued requests in arrival order (later ones may pass one that
//            does not fit yet) while job slots and the HBM budget allow;
//            request buffers come from a stream-ordered memory pool,
//   iterate  the captured two-iteration graph, kept a few steps ahead,
//   retire   requests whose job reports done: mean + device-to-host copy on a
//            second stream (overlapping the next iterations), then the
//            caller's buffer is filled and the request marked done.
// A request's paths depend only on its own job record, so its image is the
// one it renders alone; only the order of the FP64 pixel sums differs.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <set>
#include <thread>
#include <vector>

#include "objects.h"

using namespace dspbr;

namespace {

struct ReqRec {
  uint64_t id = 0;
  dspbr_request req{};
  int state = DSPBR_REQ_QUEUED;
  double submit_ms = 0, admit_ms = 0, done_ms = 0;
  int slot = -1;
  uint64_t bytes = 0;
  double4* accum = nullptr;
  float4* mean = nullptr;
  bool out_pinned = false;
  float* stage = nullptr;      // pinned staging when out_rgba is pageable
  cudaEvent_t copied = nullptr;
  bool cancel = false;
  bool cancel_sent = false;
  bool retiring = false;
  long admit_seq = 0;  // loop events recorded before the job's table write
};

struct Staging {
  float* p = nullptr;
  size_t bytes = 0;
  bool busy = false;
};

constexpr uint64_t kDefaultBudget = 120ull << 30;

}  // namespace

struct dspbr_server {
  dspbr_ctx* ctx = nullptr;
  int device = 0;
  dspbr_server_config cfg{};
  std::string err;
  cudaStream_t stream = nullptr, copy_stream = nullptr;
  cudaMemPool_t mempool = nullptr;
  std::unique_ptr<Engine> eng;
  std::mutex mu;
  std::condition_variable cv;       // driver: new work; waiters: request finished
  std::thread driver;
  bool stop = false, running = false;
  uint64_t next_id = 1;
  std::map<uint64_t, ReqRec> reqs;
  std::deque<uint64_t> queue;        // submitted, not yet admitted
  std::vector<uint64_t> order;       // admitted and running, in admission order
  std::vector<uint64_t> slot_owner = std::vector<uint64_t>(kMaxJobs, 0);
  std::vector<uint64_t> retiring;    // result copies in flight
  std::vector<Staging> staging;
  std::vector<double> latencies;
  uint64_t submitted = 0, admitted = 0, completed = 0, cancelled = 0, failed = 0;
  uint64_t bytes_in_use = 0, bytes_peak = 0;
  bool active_dirty = false;
  long events_recorded = 0;  // driver loop events so far
  Status st() { return Status{&err}; }
};

namespace {

uint64_t request_bytes(const dspbr_request& r) { return uint64_t(r.width) * uint64_t(r.height) * (32 + 16); }

uint64_t scenes_in_use(dspbr_server* s, const dspbr_scene* extra) {
  std::set<const dspbr_scene*> sc;
  for (uint64_t id : s->order) sc.insert(s->reqs[id].req.scene);
  if (extra) sc.insert(extra);
  uint64_t b = 0;
  for (auto* p : sc) b += p->bytes();
  return b;
}

float* acquire_staging(dspbr_server* s, size_t bytes) {
  for (auto& b : s->staging)
    if (!b.busy && b.bytes >= bytes) {
      b.busy = true;
      return b.p;
    }
  Staging n;
  if (cudaHostAlloc(reinterpret_cast<void**>(&n.p), bytes, cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  n.bytes = bytes;
  n.busy = true;
  s->staging.push_back(n);
  return n.p;
}

void release_staging(dspbr_server* s, float* p) {
  for (auto& b : s->staging)
    if (b.p == p) b.busy = false;
}

Job job_of(const dspbr_request& r, double4* accum) {
  Job j{};
  j.p = make_job_params(r.params, r.camera, r.fov_deg, r.near_plane, r.width, r.height, r.ibl != nullptr, 1);
  j.s = r.scene->view();
  j.s.wide = r.params.traversal == DSPBR_TRAVERSAL_WIDE;
  if (r.ibl) j.e = r.ibl->view();
  j.accum = reinterpret_cast<double*>(accum);
  return j;
}

// Under the lock: admit queued requests while slots and budget allow.
int admit(dspbr_server* s) {
  Status st = s->st();
  for (auto it = s->queue.begin(); it != s->queue.end() && int(s->order.size()) < s->cfg.max_active;) {
    ReqRec& r = s->reqs[*it];
    if (r.cancel) {
      r.state = DSPBR_REQ_CANCELLED;
      r.done_ms = now_ms();
      ++s->cancelled;
      it = s->queue.erase(it);
      s->cv.notify_all();
      continue;
    }
    uint64_t need = r.bytes;
    uint64_t total = s->eng->pool_bytes() + scenes_in_use(s, r.req.scene) + s->bytes_in_use + need;
    if (total > s->cfg.hbm_budget_bytes) {
      ++it;  // a later, smaller request may still fit
      continue;
    }
    int slot = -1;
    for (int k = 0; k < kMaxJobs; ++k)
      if (!s->slot_owner[k]) {
        slot = k;
        break;
      }
    if (slot < 0) break;
    const size_t npix = size_t(r.req.width) * r.req.height;
    int rc;
    if ((rc = st.cuda(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&r.accum), npix * 32, s->mempool, s->stream),
                      "request buffer")) ||
        (rc = st.cuda(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&r.mean), npix * 16, s->mempool, s->stream),
                      "request buffer")) ||
        (rc = st.cuda(cudaMemsetAsync(r.accum, 0, npix * 32, s->stream), "request buffer")) ||
        (rc = st.cuda(cudaEventCreateWithFlags(&r.copied, cudaEventDisableTiming), "event")) ||
        (rc = s->eng->set_job(slot, job_of(r.req, r.accum), uint64_t(npix) * uint64_t(r.req.spp)))) {
      r.state = DSPBR_REQ_FAILED;
      r.done_ms = now_ms();
      ++s->failed;
      it = s->queue.erase(it);
      s->cv.notify_all();
      return rc;
    }
    r.slot = slot;
    r.admit_seq = s->events_recorded;
    s->slot_owner[slot] = r.id;
    r.state = DSPBR_REQ_RUNNING;
    r.admit_ms = now_ms();
    s->bytes_in_use += need;
    s->bytes_peak = std::max(s->bytes_peak, s->bytes_in_use);
    ++s->admitted;
    s->order.push_back(r.id);
    s->active_dirty = true;
    it = s->queue.erase(it);
  }
  return DSPBR_OK;
}

// Under the lock: the request's job is done; copy its mean out on the copy
// stream after everything queued so far on the render stream.
int start_retire(dspbr_server* s, ReqRec& r, cudaEvent_t after) {
  Status st = s->st();
  const size_t npix = size_t(r.req.width) * r.req.height;
  TRY_CUDA(st, cudaEventRecord(after, s->stream), "retire event");
  TRY_CUDA(st, cudaStreamWaitEvent(s->copy_stream, after, 0), "retire wait");
  if (!r.cancel) {
    launch_mean(r.accum, 1.0 / double(r.req.spp), r.mean, int(npix), s->copy_stream);
    float* dst = r.req.out_rgba;
    if (!r.out_pinned) {
      r.stage = acquire_staging(s, npix * 16);
      if (!r.stage) return st.fail(DSPBR_ERR_OOM, "server: no page-locked staging memory");
      dst = r.stage;
    }
    TRY_CUDA(st, cudaMemcpyAsync(dst, r.mean, npix * 16, cudaMemcpyDeviceToHost, s->copy_stream), "result copy");
  }
  TRY_CUDA(st, cudaFreeAsync(r.accum, s->copy_stream), "free request buffer");
  TRY_CUDA(st, cudaFreeAsync(r.mean, s->copy_stream), "free request buffer");
  r.accum = nullptr;
  r.mean = nullptr;
  TRY_CUDA(st, cudaEventRecord(r.copied, s->copy_stream), "retire event");
  r.retiring = true;
  s->retiring.push_back(r.id);
  s->slot_owner[r.slot] = 0;
  s->order.erase(std::find(s->order.begin(), s->order.end(), r.id));
  s->active_dirty = true;
  return DSPBR_OK;
}

// Under the lock: requests whose copy finished become done.
void finish_retired(dspbr_server* s) {
  for (size_t k = 0; k < s->retiring.size();) {
    ReqRec& r = s->reqs[s->retiring[k]];
    cudaError_t e = cudaEventQuery(r.copied);
    if (e == cudaErrorNotReady) {
      cudaGetLastError();
      ++k;
      continue;
    }
    s->retiring.erase(s->retiring.begin() + long(k));
    r.retiring = false;
    const size_t bytes = size_t(r.req.width) * r.req.height * 16;
    if (e != cudaSuccess) {
      s->st().cuda(e, "result copy");
      r.state = DSPBR_REQ_FAILED;
      ++s->failed;
    } else if (r.cancel) {
      r.state = DSPBR_REQ_CANCELLED;
      ++s->cancelled;
    } else {
      if (r.stage) std::memcpy(r.req.out_rgba, r.stage, bytes);
      r.state = DSPBR_REQ_DONE;
      ++s->completed;
    }
    if (r.stage) release_staging(s, r.stage);
    r.stage = nullptr;
    cudaEventDestroy(r.copied);
    r.copied = nullptr;
    r.done_ms = now_ms();
    if (r.state == DSPBR_REQ_DONE) s->latencies.push_back(r.done_ms - r.submit_ms);
    s->bytes_in_use -= r.bytes;
    s->cv.notify_all();
  }
}

bool any_retiring(dspbr_server* s) { return !s->retiring.empty(); }

void driver_loop(dspbr_server* s) {
  cudaSetDevice(s->device);
  constexpr int kRing = 8, kLookahead = 3;
  cudaEvent_t ring[kRing];
  for (auto& e : ring) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  cudaEvent_t after;
  cudaEventCreateWithFlags(&after, cudaEventDisableTiming);
  long k = 0;
  long drained = -1;  // events up to this index were recorded before the last drain
  int rc = DSPBR_OK;
  for (;;) {
    bool have_jobs;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      finish_retired(s);
      if (rc == DSPBR_OK) rc = admit(s);
      if (s->active_dirty && rc == DSPBR_OK) {
        std::vector<int> slots;
        for (uint64_t id : s->order) slots.push_back(s->reqs[id].slot);
        rc = s->eng->set_active(slots);
        s->active_dirty = false;
      }
      have_jobs = !s->order.empty();
      if (!have_jobs) {
        if (s->stop && s->queue.empty() && !any_retiring(s)) break;
        // idle: wait for a submission (or a copy to finish)
        s->cv.wait_for(lk, std::chrono::milliseconds(any_retiring(s) ? 1 : 20));
        continue;
      }
    }
    if (rc != DSPBR_OK) {
      std::lock_guard<std::mutex> lk(s->mu);
      for (uint64_t id : s->order) {
        ReqRec& r = s->reqs[id];
        r.state = DSPBR_REQ_FAILED;
        r.done_ms = now_ms();
        ++s->failed;
        s->slot_owner[r.slot] = 0;
      }
      s->order.clear();
      for (uint64_t id : s->queue) {
        s->reqs[id].state = DSPBR_REQ_FAILED;
        ++s->failed;
      }
      s->queue.clear();
      s->cv.notify_all();
      if (s->stop) break;
      continue;
    }
    int d = 0;
    rc = s->eng->iterate(1, false, &d);
    if (rc) continue;
    cudaEventRecord(ring[k % kRing], s->stream);
    ++k;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->events_recorded = k;
    }
    if (k > kLookahead) {
      const long synced = k - 1 - kLookahead;  // index of the event waited for
      cudaError_t e = cudaEventSynchronize(ring[synced % kRing]);
      if (e != cudaSuccess) {
        rc = s->st().cuda(e, "server iteration");
        continue;
      }
      std::lock_guard<std::mutex> lk(s->mu);
      std::vector<uint64_t> done;
      // a job's status record is its own only after an event that follows
      // its table write (a reused slot still shows the previous job before)
      for (uint64_t id : s->order)
        if (s->reqs[id].admit_seq <= synced && s->eng->job_done(s->reqs[id].slot)) done.push_back(id);
      for (uint64_t id : done) {
        rc = start_retire(s, s->reqs[id], after);
        if (rc) break;
      }
      // cancellations: no further samples of cancelled requests start; the
      // job then reports done once its paths in flight have finished
      for (uint64_t id : s->order) {
        ReqRec& r = s->reqs[id];
        if (r.cancel && !r.cancel_sent && r.slot >= 0) {
          s->eng->cancel_job(r.slot);
          r.cancel_sent = true;
        }
      }
      // the tail: nothing waits for admission, every active request's work
      // items have started and few paths are left: finish them in one drain
      // launch instead of iterations bound by the latency of the longest path
      if (rc == DSPBR_OK && synced > drained && s->queue.empty() && !s->order.empty() &&
          done.size() < s->order.size()) {
        const volatile HostStatus* hs = s->eng->status();
        bool started = hs->live_paths < s->eng->drain_below();
        for (uint64_t id : s->order) {
          const ReqRec& r = s->reqs[id];
          const volatile JobStatus& js = hs->job[r.slot];
          if (r.admit_seq > synced || js.items_next < js.items_total) started = false;
        }
        if (started) {
          rc = s->eng->drain();
          drained = k;  // the statuses of later events include the drain
        }
      }
    }
  }
  cudaStreamSynchronize(s->stream);
  cudaStreamSynchronize(s->copy_stream);
  for (auto& e : ring) cudaEventDestroy(e);
  cudaEventDestroy(after);
}

void fill_info(const ReqRec& r, dspbr_request_info* info) {
  info->state = r.state;
  info->tag = r.req.tag;
  info->submit_ms = r.submit_ms;
  info->admit_ms = r.admit_ms;
  info->done_ms = r.done_ms;
  info->device_bytes = r.bytes;
}

bool finished(int state) {
  return state == DSPBR_REQ_DONE || state == DSPBR_REQ_CANCELLED || state == DSPBR_REQ_FAILED;
}

}  // namespace

extern "C" {

int dspbr_server_create(dspbr_ctx* ctx, const dspbr_server_config* cfg, dspbr_server** out) {
  if (!ctx || !out) return DSPBR_ERR_INVALID;
  *out = nullptr;
  auto* s = new dspbr_server();
  s->ctx = ctx;
  s->device = ctx->device;
  if (cfg) s->cfg = *cfg;
  if (s->cfg.path_pool == 0) s->cfg.path_pool = 1u << 23;
  if (s->cfg.max_active <= 0 || s->cfg.max_active > kMaxJobs) s->cfg.max_active = kMaxJobs;
  if (s->cfg.hbm_budget_bytes == 0) s->cfg.hbm_budget_bytes = kDefaultBudget;
  Status st = ctx->st();
  int rc = DSPBR_OK;
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = s->device;
  if ((rc = st.cuda(cudaSetDevice(s->device), "cudaSetDevice")) ||
      (rc = st.cuda(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "stream")) ||
      (rc = st.cuda(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking), "stream")) ||
      (rc = st.cuda(cudaMemPoolCreate(&s->mempool, &props), "memory pool"))) {
    dspbr_server_destroy(s);
    return rc;
  }
  uint64_t keep = ~0ull;  // keep freed request buffers in the pool for the next requests
  cudaMemPoolSetAttribute(s->mempool, cudaMemPoolAttrReleaseThreshold, &keep);
  s->eng.reset(new Engine(s->device, s->stream, &s->err));
  if ((rc = s->eng->ensure_pool(s->cfg.path_pool))) {
    ctx->err = s->err;
    dspbr_server_destroy(s);
    return rc;
  }
  *out = s;
  return DSPBR_OK;
}

int dspbr_server_submit(dspbr_server* s, const dspbr_request* req, uint64_t* id) {
  if (!s || !req || !id) return DSPBR_ERR_INVALID;
  Status st = s->st();
  if (!req->scene || req->scene->ctx != s->ctx || (req->ibl && req->ibl->ctx != s->ctx))
    return st.fail(DSPBR_ERR_INVALID, "submit: scene / IBL of another context");
  if (int64_t(req->scene->max_tex_id) >= int64_t(req->scene->num_texinfo))
    return st.fail(DSPBR_ERR_STATE, "submit: the scene's materials use textures; call dspbr_scene_set_textures");
  if (req->width <= 0 || req->height <= 0 || int64_t(req->width) * req->height > (int64_t(1) << 28) ||
      req->spp <= 0 || !req->out_rgba || !(req->fov_deg > 0.f && req->fov_deg < 180.f) || !(req->near_plane > 0.f) ||
      req->params.max_bounces < 0 || req->params.max_bounces > 4096)
    return st.fail(DSPBR_ERR_INVALID, "submit: invalid request");
  ReqRec r;
  r.req = *req;
  r.bytes = request_bytes(*req);
  if (s->eng->pool_bytes() + req->scene->bytes() + r.bytes > s->cfg.hbm_budget_bytes)
    return st.fail(DSPBR_ERR_ADMISSION, "submit: request needs %llu bytes, above the HBM budget",
                   (unsigned long long)r.bytes);
  cudaPointerAttributes attr{};
  r.out_pinned = cudaPointerGetAttributes(&attr, req->out_rgba) == cudaSuccess && attr.type == cudaMemoryTypeHost;
  cudaGetLastError();
  r.submit_ms = now_ms();
  std::lock_guard<std::mutex> lk(s->mu);
  r.id = s->next_id++;
  *id = r.id;
  s->reqs[r.id] = r;
  s->queue.push_back(r.id);
  ++s->submitted;
  if (!s->running) {
    s->running = true;
    s->driver = std::thread(driver_loop, s);
  }
  s->cv.notify_all();
  return DSPBR_OK;
}

int dspbr_server_poll(dspbr_server* s, uint64_t id, dspbr_request_info* info) {
  if (!s || !info) return DSPBR_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return DSPBR_ERR_NOT_FOUND;
  fill_info(it->second, info);
  return DSPBR_OK;
}

int dspbr_server_wait(dspbr_server* s, uint64_t id, int timeout_ms, dspbr_request_info* info) {
  if (!s) return DSPBR_ERR_INVALID;
  std::unique_lock<std::mutex> lk(s->mu);
  auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms < 0 ? 0 : timeout_ms);
  for (;;) {
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return DSPBR_ERR_NOT_FOUND;
    if (finished(it->second.state)) {
      if (info) fill_info(it->second, info);
      return it->second.state == DSPBR_REQ_FAILED ? DSPBR_ERR_CUDA : DSPBR_OK;
    }
    if (timeout_ms < 0) s->cv.wait_for(lk, std::chrono::milliseconds(50));
    else if (s->cv.wait_until(lk, deadline) == std::cv_status::timeout) {
      auto it2 = s->reqs.find(id);
      if (it2 != s->reqs.end() && finished(it2->second.state)) continue;
      if (info && it2 != s->reqs.end()) fill_info(it2->second, info);
      return DSPBR_ERR_STATE;
    }
  }
}

int dspbr_server_cancel(dspbr_server* s, uint64_t id) {
  if (!s) return DSPBR_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return DSPBR_ERR_NOT_FOUND;
  if (!finished(it->second.state)) it->second.cancel = true;
  s->cv.notify_all();
  return DSPBR_OK;
}

int dspbr_server_release(dspbr_server* s, uint64_t id) {
  if (!s) return DSPBR_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return DSPBR_ERR_NOT_FOUND;
  if (!finished(it->second.state)) return s->st().fail(DSPBR_ERR_STATE, "release: request %llu not finished",
                                                        (unsigned long long)id);
  s->reqs.erase(it);
  return DSPBR_OK;
}

int dspbr_server_get_stats(dspbr_server* s, dspbr_server_stats* out) {
  if (!s || !out) return DSPBR_ERR_INVALID;
  std::memset(out, 0, sizeof *out);
  unsigned long long st[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  cudaSetDevice(s->device);
  // counters are read without stopping the render (a snapshot)
  if (cudaMemcpy(st, s->eng->stats(), sizeof st, cudaMemcpyDeviceToHost) != cudaSuccess) cudaGetLastError();
  std::lock_guard<std::mutex> lk(s->mu);
  out->submitted = s->submitted;
  out->admitted = s->admitted;
  out->completed = s->completed;
  out->cancelled = s->cancelled;
  out->failed = s->failed;
  out->queued = s->queue.size();
  out->running = s->order.size();
  out->iterations = s->eng->status() ? s->eng->status()->iteration : 0;
  out->rays_closest = st[0];
  out->rays_shadow = st[1];
  out->bytes_in_use = s->bytes_in_use + s->eng->pool_bytes();
  out->bytes_peak = s->bytes_peak + s->eng->pool_bytes();
  if (!s->latencies.empty()) {
    std::vector<double> v = s->latencies;
    std::sort(v.begin(), v.end());
    auto pct = [&](double q) { return v[std::min(v.size() - 1, size_t(q * double(v.size() - 1) + 0.5))]; };
    out->p50_ms = pct(0.50);
    out->p99_ms = pct(0.99);
  }
  out->path_pool = s->eng->capacity();
  const LaunchCfg& lc = s->eng->launch();
  out->trace_threads = 128;
  out->trace_blocks = lc.dyn_blocks;
  out->shade_threads = 128;
  out->shade_blocks = lc.shade_dyn_blocks[0];
  out->connect_blocks = lc.connect_dyn_blocks;
  return DSPBR_OK;
}

int dspbr_server_destroy(dspbr_server* s) {
  if (!s) return DSPBR_ERR_INVALID;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    for (auto& kv : s->reqs)
      if (!finished(kv.second.state)) kv.second.cancel = true;
    s->cv.notify_all();
  }
  if (s->driver.joinable()) s->driver.join();
  cudaSetDevice(s->device);
  s->eng.reset();
  for (auto& b : s->staging)
    if (b.p) cudaFreeHost(b.p);
  for (auto& kv : s->reqs)
    if (kv.second.copied) cudaEventDestroy(kv.second.copied);
  if (s->mempool) cudaMemPoolDestroy(s->mempool);
  if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return DSPBR_OK;
}

// ---- autotuner -----------------------------------------------------------------------------------
// Coordinate search over the path-pool size, then the extend/connect grid
// (threads x blocks per SM), then the shade grid.  Each candidate is timed in
// steady state (full pool) on the sample requests with CUDA events over a
// fixed number of graph-launched iterations; the score is traced rays per
// second from the device counters.
int dspbr_server_get_launch(dspbr_server* s, dspbr_launch* out) {
  if (!s || !out) return DSPBR_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  *out = dspbr_launch{};
  out->path_pool = s->eng->capacity();
  const LaunchCfg& lc = s->eng->launch();
  out->extend_blocks = lc.dyn_blocks;
  out->connect_blocks = lc.connect_dyn_blocks;
  out->shade_blocks = lc.shade_dyn_blocks[0];
  return DSPBR_OK;
}

int dspbr_server_set_launch(dspbr_server* s, const dspbr_launch* l) {
  if (!s || !l) return DSPBR_ERR_INVALID;
  Status st = s->st();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->running) return st.fail(DSPBR_ERR_STATE, "set_launch: call while the server is idle");
  }
  TRY_CUDA(st, cudaSetDevice(s->device), "cudaSetDevice");
  const LaunchLimits L = launch_limits();
  auto ok = [&](int blocks, int per_sm) { return blocks >= L.sms && blocks % L.sms == 0 && blocks <= per_sm * L.sms; };
  if (!ok(l->extend_blocks, L.trace_per_sm) || !ok(l->connect_blocks, L.connect_per_sm) ||
      !ok(l->shade_blocks, L.shade_per_sm[0]))
    return st.fail(DSPBR_ERR_INVALID, "set_launch: grids must be 1..%d / %d / %d x %d SMs", L.trace_per_sm,
                   L.connect_per_sm, L.shade_per_sm[0], L.sms);
  if (l->path_pool < 1024 || l->path_pool > (1u << 26))
    return st.fail(DSPBR_ERR_INVALID, "set_launch: path pool %u outside 1024..2^26", l->path_pool);
  Engine& E = *s->eng;
  int rc = E.set_active({});
  if (!rc) rc = l->path_pool != E.capacity() ? E.ensure_pool(l->path_pool) : E.reset_pool();
  if (rc) return rc;
  LaunchCfg lc = E.launch();
  lc.dyn_blocks = l->extend_blocks;
  lc.connect_dyn_blocks = l->connect_blocks;
  lc.shade_dyn_blocks[0] = l->shade_blocks;
  lc.shade_dyn_blocks[1] = std::min(l->shade_blocks / L.sms, L.shade_per_sm[1]) * L.sms;
  E.set_launch(lc);
  s->cfg.path_pool = l->path_pool;
  return st.cuda(cudaStreamSynchronize(s->stream), "set_launch");
}

// the gain a tuning candidate needs over the best so far
constexpr double kTuneMargin = 1.02;

int dspbr_server_autotune(dspbr_server* s, const dspbr_request* samples, int n, double seconds) {
  if (!s || !samples || n <= 0 || n > kMaxJobs) return DSPBR_ERR_INVALID;
  Status st = s->st();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->running) return st.fail(DSPBR_ERR_STATE, "autotune: call before the first submit");
  }
  TRY_CUDA(st, cudaSetDevice(s->device), "cudaSetDevice");
  Engine& E = *s->eng;
  const double t_end = now_ms() + 1e3 * (seconds > 0 ? seconds : 10.0);
  std::vector<DevBuf<double4>> accum(n);
  for (int i = 0; i < n; ++i) {
    const dspbr_request& r = samples[i];
    if (!r.scene || r.width <= 0 || r.height <= 0) return st.fail(DSPBR_ERR_INVALID, "autotune: invalid sample");
    TRY_CUDA(st, accum[i].alloc(size_t(r.width) * r.height), "autotune buffers");
  }
  unsigned long long ev_st[2] = {0, 0};
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // (re)starts the sample jobs with effectively unbounded work
  auto load = [&]() -> int {
    std::vector<int> slots;
    for (int i = 0; i < n; ++i) {
      const dspbr_request& r = samples[i];
      int rc = E.set_job(i, job_of(r, accum[i].p), uint64_t(r.width) * r.height * 100000ull);
      if (rc) return rc;
      slots.push_back(i);
    }
    return E.set_active(slots);
  };
  auto measure = [&](uint32_t pool, const LaunchCfg& lc, double* score) -> int {
    int rc;
    if ((rc = E.set_active({}))) return rc;
    if (pool != E.capacity()) {
      if ((rc = E.ensure_pool(pool))) return rc;
    } else if ((rc = E.reset_pool())) {
      return rc;
    }
    E.set_launch(lc);
    if ((rc = load())) return rc;
    int d;
    if ((rc = E.iterate(8, false, &d))) return rc;  // fill the pool, capture the graph
    TRY_CUDA(st, cudaMemcpyAsync(&ev_st[0], E.stats(), 8, cudaMemcpyDeviceToHost, s->stream), "stats");
    unsigned long long sh0 = 0;
    TRY_CUDA(st, cudaMemcpyAsync(&sh0, E.stats() + 1, 8, cudaMemcpyDeviceToHost, s->stream), "stats");
    TRY_CUDA(st, cudaEventRecord(e0, s->stream), "event");
    if ((rc = E.iterate(12, false, &d))) return rc;
    TRY_CUDA(st, cudaEventRecord(e1, s->stream), "event");
    unsigned long long sh1 = 0;
    TRY_CUDA(st, cudaMemcpyAsync(&ev_st[1], E.stats(), 8, cudaMemcpyDeviceToHost, s->stream), "stats");
    TRY_CUDA(st, cudaMemcpyAsync(&sh1, E.stats() + 1, 8, cudaMemcpyDeviceToHost, s->stream), "stats");
    TRY_CUDA(st, cudaStreamSynchronize(s->stream), "autotune");
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    *score = ms > 0 ? double((ev_st[1] - ev_st[0]) + (sh1 - sh0)) / double(ms) : 0.0;
    return DSPBR_OK;
  };
  uint32_t best_pool = E.capacity();
  LaunchCfg best = E.launch();
  double best_score = -1;
  int rc = measure(best_pool, best, &best_score);
  auto consider = [&](uint32_t pool, const LaunchCfg& lc) -> int {
    if (now_ms() > t_end) return DSPBR_OK;
    uint64_t pool_mem = uint64_t(pool) * (E.capacity() ? E.pool_bytes() / E.capacity() : 300);
    if (pool_mem > s->cfg.hbm_budget_bytes / 2) return DSPBR_OK;
    double sc = 0;
    int r = measure(pool, lc, &sc);
    if (r) return r;
    // a candidate replaces the best only by a clear margin: one short
    // measurement each, so the largest of many scores is partly noise (a
    // sweep without the margin once settled on 2 shading blocks per SM, and
    // the batched mix then ran 16% below the occupancy limits' rate)
    if (sc > kTuneMargin * best_score) {
      best_score = sc;
      best_pool = pool;
      best = lc;
    }
    return DSPBR_OK;
  };
  for (uint32_t pool : {1u << 20, 1u << 21, 1u << 22, 1u << 23, 1u << 24})
    if (!rc && pool != best_pool) rc = consider(pool, best);
  // then the grids of the persistent kernels: resident blocks per SM from the
  // occupancy limit down (fewer blocks: more L1 per block, less contention on
  // the queue cursors; the limit: more warps to hide memory latency)
  const LaunchLimits L = launch_limits();
  for (int k = L.trace_per_sm - 1; k >= std::max(2, L.trace_per_sm - 4) && !rc; --k) {
    LaunchCfg lc = best;
    lc.dyn_blocks = k * L.sms;
    rc = consider(best_pool, lc);
  }
  for (int k = L.connect_per_sm - 1; k >= std::max(2, L.connect_per_sm - 4) && !rc; --k) {
    LaunchCfg lc = best;
    lc.connect_dyn_blocks = k * L.sms;
    rc = consider(best_pool, lc);
  }
  for (int k = L.shade_per_sm[0] - 1; k >= std::max(2, L.shade_per_sm[0] - 3) && !rc; --k) {
    LaunchCfg lc = best;
    lc.shade_dyn_blocks[0] = k * L.sms;
    lc.shade_dyn_blocks[1] = std::min(k, L.shade_per_sm[1]) * L.sms;
    rc = consider(best_pool, lc);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // leave an empty pool of the chosen size with the chosen launch sizes
  int rc2 = E.set_active({});
  if (!rc2) rc2 = best_pool != E.capacity() ? E.ensure_pool(best_pool) : E.reset_pool();
  if (!rc2) {
    E.set_launch(best);
    rc2 = st.cuda(cudaStreamSynchronize(s->stream), "autotune");
  }
  return rc ? rc : rc2;
}

}  // extern "C"
