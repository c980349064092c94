// Render engine: path pool, job table, iteration loop (see engine.h).
#include "engine.h"

#include <algorithm>
#include <cstring>

namespace dspbr {

namespace {

// Table writes travel as kernel arguments, ordered on the engine's stream.
__global__ void k_set_job(Job job, unsigned long long items_total, int slot, Job* jobs, JobState* js,
                          HostStatus* hs) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  jobs[slot] = job;
  JobState s;
  s.items_next = 0;
  s.items_total = items_total;
  s.live = 0;
  s.pad = 0;
  js[slot] = s;
  volatile JobStatus* st = &hs->job[slot];
  st->items_next = 0;
  st->items_total = items_total;
  st->live = 0;
  st->done = 0;
}

__global__ void k_set_active(ActiveList list, int* active) {
  int t = threadIdx.x;
  if (t < kMaxJobs) active[t] = t < list.n ? list.slot[t] : -1;
  if (t == 0) active[kMaxJobs] = list.n;
}

// Cancel: no further work items start; paths in flight finish normally.
__global__ void k_cancel_job(int slot, JobState* js) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  if (js[slot].items_total > js[slot].items_next) js[slot].items_total = js[slot].items_next;
}

}  // namespace

Engine::~Engine() {
  cudaSetDevice(device_);
  if (stream_) cudaStreamSynchronize(stream_);
  drop_graph();
  for (auto e : ring_)
    if (e) cudaEventDestroy(e);
  for (auto e : ev_pool_) cudaEventDestroy(e);
  if (h_status_) cudaFreeHost(h_status_);
}

int Engine::init() {
  if (ready_) return DSPBR_OK;
  Status s{err_};
  TRY_CUDA(s, cudaSetDevice(device_), "cudaSetDevice");
  TRY_CUDA(s, jobs_.alloc(kMaxJobs), "job table");
  TRY_CUDA(s, js_.alloc(kMaxJobs), "job table");
  TRY_CUDA(s, active_.alloc(kMaxJobs + 1), "job table");
  TRY_CUDA(s, counts_.alloc(kCntNum), "counters");
  TRY_CUDA(s, cursors_.alloc(3), "counters");
  TRY_CUDA(s, stats_.alloc(8), "stats");
  TRY_CUDA(s, cudaMemsetAsync(js_.p, 0, js_.bytes(), stream_), "job table");
  TRY_CUDA(s, cudaMemsetAsync(active_.p, 0, active_.bytes(), stream_), "job table");
  TRY_CUDA(s, cudaMemsetAsync(counts_.p, 0, counts_.bytes(), stream_), "counters");
  TRY_CUDA(s, cudaMemsetAsync(cursors_.p, 0, cursors_.bytes(), stream_), "counters");
  TRY_CUDA(s, cudaMemsetAsync(stats_.p, 0, stats_.bytes(), stream_), "stats");
  TRY_CUDA(s, cudaHostAlloc(reinterpret_cast<void**>(&h_status_), sizeof(HostStatus), cudaHostAllocMapped),
           "mapped status");
  std::memset(h_status_, 0, sizeof(HostStatus));
  TRY_CUDA(s, cudaHostGetDevicePointer(reinterpret_cast<void**>(&d_status_), h_status_, 0), "mapped status");
  for (auto& e : ring_) TRY_CUDA(s, cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
  TRY_CUDA(s, cudaStreamSynchronize(stream_), "engine init");
  ready_ = true;
  return DSPBR_OK;
}

size_t Engine::pool_bytes() const {
  return org_.bytes() * 9 + rng_.bytes() + sh_flags_.bytes() + bounce_.bytes() + pixel_.bytes() + frame_.bytes() +
         job_.bytes() + q0_.bytes() * 6 + qh_.bytes();
}

int Engine::ensure_pool(uint32_t cap) {
  int rc = init();
  if (rc) return rc;
  if (cap == capacity_) return DSPBR_OK;
  Status s{err_};
  if (cap == 0) return s.fail(DSPBR_ERR_INVALID, "path pool: capacity 0");
  TRY_CUDA(s, cudaStreamSynchronize(stream_), "sync");
  drop_graph();
  capacity_ = 0;
  if ((rc = s.cuda(org_.alloc(cap), "paths")) || (rc = s.cuda(dir_.alloc(cap), "paths")) ||
      (rc = s.cuda(weight_.alloc(cap), "paths")) || (rc = s.cuda(rad_.alloc(cap), "paths")) ||
      (rc = s.cuda(hit_.alloc(cap), "paths")) || (rc = s.cuda(sh_dir_.alloc(cap), "paths")) ||
      (rc = s.cuda(sh_c_.alloc(cap), "paths")) || (rc = s.cuda(pl_dir_.alloc(cap), "paths")) ||
      (rc = s.cuda(pl_c_.alloc(cap), "paths")) || (rc = s.cuda(rng_.alloc(cap), "paths")) ||
      (rc = s.cuda(sh_flags_.alloc(cap), "paths")) || (rc = s.cuda(bounce_.alloc(cap), "paths")) ||
      (rc = s.cuda(pixel_.alloc(cap), "paths")) || (rc = s.cuda(frame_.alloc(cap), "paths")) ||
      (rc = s.cuda(job_.alloc(cap), "paths")) || (rc = s.cuda(q0_.alloc(cap), "queues")) ||
      (rc = s.cuda(q1_.alloc(cap), "queues")) || (rc = s.cuda(qs0_.alloc(cap), "queues")) ||
      (rc = s.cuda(qs1_.alloc(cap), "queues")) || (rc = s.cuda(qh_.alloc(size_t(cap) * kNumClasses), "queues")) ||
      (rc = s.cuda(qm_.alloc(cap), "queues")) || (rc = s.cuda(qfree_.alloc(cap), "queues")))
    return rc;
  capacity_ = cap;
  cur_ = 0;
  launch_init_pool(paths(), stream_);
  TRY_CUDA(s, cudaGetLastError(), "init pool");
  return DSPBR_OK;
}

int Engine::reset_pool() {
  Status s{err_};
  if (!capacity_) return DSPBR_OK;
  cur_ = 0;
  launch_init_pool(paths(), stream_);
  return s.cuda(cudaGetLastError(), "init pool");
}

void Engine::set_launch(const LaunchCfg& lc) {
  if (lc.trace_blocks == lc_.trace_blocks && lc.trace_threads == lc_.trace_threads &&
      lc.shade_blocks == lc_.shade_blocks && lc.shade_threads == lc_.shade_threads)
    return;
  cudaStreamSynchronize(stream_);
  drop_graph();
  const int trav = lc_.traversal;
  const bool tex = lc_.textured;
  lc_ = lc;
  lc_.traversal = trav;
  lc_.textured = tex;
}

Sched Engine::sched() const {
  Sched sc;
  sc.jobs = jobs_.p;
  sc.js = js_.p;
  sc.active = active_.p;
  sc.nactive = active_.p + kMaxJobs;
  sc.status = d_status_;
  sc.iteration = cursors_.p + 2;
  return sc;
}

PathBuf Engine::paths() const {
  PathBuf b{};
  b.org = org_.p; b.dir = dir_.p; b.weight = weight_.p; b.rad = rad_.p; b.rng = rng_.p; b.hit = hit_.p;
  b.sh_dir = sh_dir_.p; b.sh_c = sh_c_.p; b.pl_dir = pl_dir_.p; b.pl_c = pl_c_.p; b.sh_flags = sh_flags_.p;
  b.pixel = pixel_.p; b.frame = frame_.p; b.bounce = bounce_.p; b.job = job_.p;
  b.q[0] = q0_.p; b.q[1] = q1_.p; b.qs[0] = qs0_.p; b.qs[1] = qs1_.p; b.qh = qh_.p; b.qm = qm_.p;
  b.qfree = qfree_.p; b.free_head = cursors_.p; b.free_tail = cursors_.p + 1;
  b.counts = counts_.p; b.stats = stats_.p;
  b.capacity = capacity_;
  return b;
}

int Engine::set_job(int slot, const Job& job, unsigned long long items_total) {
  Status s{err_};
  if (slot < 0 || slot >= kMaxJobs) return s.fail(DSPBR_ERR_INVALID, "job slot %d out of range", slot);
  k_set_job<<<1, 32, 0, stream_>>>(job, items_total, slot, jobs_.p, js_.p, d_status_);
  slot_traversal_[slot] = job.s.wide ? kTravWide : kTravReference;
  slot_textured_[slot] = job.s.num_texinfo > 0;
  ++kind_launches[3];
  return s.cuda(cudaGetLastError(), "set job");
}

int Engine::cancel_job(int slot) {
  Status s{err_};
  if (slot < 0 || slot >= kMaxJobs) return s.fail(DSPBR_ERR_INVALID, "job slot %d out of range", slot);
  k_cancel_job<<<1, 32, 0, stream_>>>(slot, js_.p);
  ++kind_launches[3];
  return s.cuda(cudaGetLastError(), "cancel job");
}

int Engine::set_active(const std::vector<int>& order) {
  Status s{err_};
  if (order.size() > size_t(kMaxJobs)) return s.fail(DSPBR_ERR_INVALID, "too many active jobs");
  ActiveList list;
  list.n = int(order.size());
  for (int i = 0; i < kMaxJobs; ++i) list.slot[i] = i < list.n ? order[i] : -1;
  k_set_active<<<1, kMaxJobs, 0, stream_>>>(list, active_.p);
  ++kind_launches[3];
  // one traversal kind for all active jobs: launch the kernels specialised for it
  int trav = order.empty() ? lc_.traversal : slot_traversal_[order[0]];
  for (int k : order)
    if (slot_traversal_[k] != trav) trav = kTravPerPath;
  // the shade kernels without the texture code when no active job samples textures
  bool tex = false;
  for (int k : order) tex = tex || slot_textured_[k];
  if (trav != lc_.traversal || tex != lc_.textured) {
    TRY_CUDA(s, cudaStreamSynchronize(stream_), "sync");
    drop_graph();
    lc_.traversal = trav;
    lc_.textured = tex;
  }
  return s.cuda(cudaGetLastError(), "set active jobs");
}

cudaEvent_t Engine::next_event() {
  if (ev_used_ == ev_pool_.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    ev_pool_.push_back(e);
  }
  return ev_pool_[ev_used_++];
}
void Engine::mark_begin(int kind) {
  if (!profiling) return;
  ev_marks_.push_back({kind, int(ev_used_)});
  cudaEventRecord(next_event(), stream_);
}
void Engine::mark_end() {
  if (profiling) cudaEventRecord(next_event(), stream_);
}
void Engine::resolve_marks() {
  for (auto& m : ev_marks_) {
    if (size_t(m.second) + 1 >= ev_used_) break;
    float ms = 0;
    if (cudaEventElapsedTime(&ms, ev_pool_[m.second], ev_pool_[m.second + 1]) == cudaSuccess) kind_ms[m.first] += ms;
    else cudaGetLastError();
  }
  clear_marks();
}
void Engine::clear_marks() {
  ev_marks_.clear();
  ev_used_ = 0;
}

int Engine::one_iteration(bool counting) {
  const Sched sc = sched();
  const PathBuf b = paths();
  const int cur = cur_;
  mark_begin(0);
  launch_extend(sc, b, cur, counting, lc_, stream_);
  mark_end();
  mark_begin(1);
  launch_connect(sc, b, cur, counting, lc_, stream_);
  mark_end();
  mark_begin(2);
  launch_shade_miss(sc, b, lc_, stream_);
  launch_shade(sc, b, cur ^ 1, lc_, stream_);
  launch_regen(sc, b, cur ^ 1, stream_);
  launch_commit(sc, b, cur, stream_);
  mark_end();
  kind_launches[0] += 1;
  kind_launches[1] += 1;
  kind_launches[2] += 4;
  cur_ ^= 1;
  return Status{err_}.cuda(cudaGetLastError(), "render launch");
}

void Engine::drop_graph() {
  if (graph_) cudaGraphExecDestroy(graph_);
  graph_ = nullptr;
}

// Two iterations (parity 0, then 1) captured from the stream.  Every argument
// is a device pointer or a constant of the pool, so the graph stays valid
// until the pool or the launch configuration changes.
int Engine::capture_graph() {
  Status s{err_};
  const Sched sc = sched();
  const PathBuf b = paths();
  cudaGraph_t g = nullptr;
  TRY_CUDA(s, cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "graph capture");
  for (int cur = 0; cur < 2; ++cur) {
    launch_extend(sc, b, cur, false, lc_, stream_);
    launch_connect(sc, b, cur, false, lc_, stream_);
    launch_shade_miss(sc, b, lc_, stream_);
    launch_shade(sc, b, cur ^ 1, lc_, stream_);
    launch_regen(sc, b, cur ^ 1, stream_);
    launch_commit(sc, b, cur, stream_);
  }
  cudaError_t e = cudaStreamEndCapture(stream_, &g);
  if (e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return s.cuda(e, "graph capture");
  }
  e = cudaGraphInstantiate(&graph_, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    graph_ = nullptr;
    return s.cuda(e, "graph instantiate");
  }
  return DSPBR_OK;
}

int Engine::iterate(int n, bool counting, int* done) {
  Status s{err_};
  int k = 0;
  const bool use_graph = !profiling && !counting;
  while (k < n) {
    if (use_graph && cur_ == 0) {
      if (!graph_) {
        int rc = capture_graph();
        if (rc) return rc;
      }
      TRY_CUDA(s, cudaGraphLaunch(graph_, stream_), "graph launch");
      kind_launches[0] += 2;
      kind_launches[1] += 2;
      kind_launches[2] += 8;
      k += 2;
    } else {
      int rc = one_iteration(counting);
      if (rc) return rc;
      k += 1;
    }
  }
  if (done) *done = k;
  return DSPBR_OK;
}

bool Engine::job_done(int slot) const { return h_status_ && h_status_->job[slot].done != 0u; }

int Engine::drain() {
  const Sched sc = sched();
  const PathBuf b = paths();
  const int cur = cur_;
  mark_begin(2);
  launch_connect(sc, b, cur, false, lc_, stream_);
  launch_drain(sc, b, cur, lc_, stream_);
  launch_commit(sc, b, cur, stream_, false);
  mark_end();
  kind_launches[1] += 1;
  kind_launches[3] += 2;
  cur_ ^= 1;
  return Status{err_}.cuda(cudaGetLastError(), "drain");
}

int Engine::run_until_done(int slot, unsigned long long max_iter, bool counting) {
  Status s{err_};
  unsigned long long it = 0;
  long k = 0;
  while (it < max_iter) {
    int d = 0;
    int rc = iterate(1, counting, &d);
    if (rc) return rc;
    it += unsigned(d);
    TRY_CUDA(s, cudaEventRecord(ring_[k % kRing], stream_), "loop event");
    ++k;
    if (k > kLookahead) {
      TRY_CUDA(s, cudaEventSynchronize(ring_[(k - 1 - kLookahead) % kRing]), "render");
      if (job_done(slot)) return DSPBR_OK;
      // the tail: every work item started and few paths left
      const volatile JobStatus& js = h_status_->job[slot];
      if (!counting && js.items_next >= js.items_total && h_status_->live_paths < kDrainBelow) {
        int rc2 = drain();
        if (rc2) return rc2;
        TRY_CUDA(s, cudaStreamSynchronize(stream_), "render");
        if (job_done(slot)) return DSPBR_OK;
      }
    }
  }
  TRY_CUDA(s, cudaStreamSynchronize(stream_), "render");
  if (job_done(slot)) return DSPBR_OK;
  return s.fail(DSPBR_ERR_DEVICE_FAULT, "render: job not finished after %llu iterations", max_iter);
}

}  // namespace dspbr
