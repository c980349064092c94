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
// The ray counters into mapped host memory by one warp: a copy-engine
// transfer would queue behind a pending device-to-host copy of an image.
__global__ void k_read_stats(const unsigned long long* stats, HostStatus* out) {
  if (threadIdx.x < 8) out->stats[threadIdx.x] = stats[threadIdx.x];
}

__global__ void k_add_items(int slot, unsigned long long items, JobState* js, HostStatus* hs) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  js[slot].items_total += items;
  volatile JobStatus* st = &hs->job[slot];
  st->items_total = js[slot].items_total;
  st->done = 0;
}

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
  if (fork_) cudaEventDestroy(fork_);
  if (join_) cudaEventDestroy(join_);
  if (side_) cudaStreamDestroy(side_);
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
  TRY_CUDA(s, timeline_.alloc(kTimeline), "timeline");
  TRY_CUDA(s, cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking), "stream");
  init_launch_sizes(lc_);
  TRY_CUDA(s, cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming), "event");
  TRY_CUDA(s, cudaEventCreateWithFlags(&join_, cudaEventDisableTiming), "event");
  TRY_CUDA(s, cudaMemsetAsync(timeline_.p, 0, timeline_.bytes(), stream_), "timeline");
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
  return st_.bytes() + hits_.bytes() + sh_.bytes() + q0_.bytes() * 6 + qh_.bytes() + fmap_.bytes() + fblock_.bytes();
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
  if ((rc = s.cuda(st_.alloc(cap), "paths")) || (rc = s.cuda(hits_.alloc(cap), "paths")) ||
      (rc = s.cuda(sh_.alloc(cap), "paths")) || (rc = s.cuda(q0_.alloc(cap), "queues")) ||
      (rc = s.cuda(q1_.alloc(cap), "queues")) || (rc = s.cuda(qs0_.alloc(cap), "queues")) ||
      (rc = s.cuda(qs1_.alloc(cap), "queues")) || (rc = s.cuda(qh_.alloc(size_t(cap) * kNumClasses), "queues")) ||
      (rc = s.cuda(qm_.alloc(cap), "queues")) || (rc = s.cuda(qfree_.alloc(cap), "queues")) ||
      (rc = s.cuda(fmap_.alloc((size_t(cap) + 31) / 32), "free map")) ||
      (rc = s.cuda(fblock_.alloc(((size_t(cap) + 31) / 32 + kFreeMapBlock - 1) / kFreeMapBlock + 1), "free map")))
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
      lc.shade_blocks == lc_.shade_blocks && lc.shade_threads == lc_.shade_threads &&
      lc.dyn_blocks == lc_.dyn_blocks && lc.connect_dyn_blocks == lc_.connect_dyn_blocks &&
      lc.shade_dyn_blocks[0] == lc_.shade_dyn_blocks[0] &&
      lc.shade_dyn_blocks[1] == lc_.shade_dyn_blocks[1])
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
  sc.timeline = timeline_.p;
  return sc;
}

PathBuf Engine::paths() const {
  PathBuf b{};
  b.st = st_.p; b.hits = hits_.p; b.sh = sh_.p;
  b.q[0] = q0_.p; b.q[1] = q1_.p; b.qs[0] = qs0_.p; b.qs[1] = qs1_.p; b.qh = qh_.p; b.qm = qm_.p;
  b.qfree = qfree_.p; b.fmap = fmap_.p; b.fblock = fblock_.p;
  b.free_head = cursors_.p; b.free_tail = cursors_.p + 1;
  b.counts = counts_.p; b.stats = stats_.p;
  b.capacity = capacity_;
  return b;
}

int Engine::set_job(int slot, const Job& job, unsigned long long items_total) {
  Status s{err_};
  if (slot < 0 || slot >= kMaxJobs) return s.fail(DSPBR_ERR_INVALID, "job slot %d out of range", slot);
  k_set_job<<<1, 32, 0, stream_>>>(job, items_total, slot, jobs_.p, js_.p, d_status_);
  slot_traversal_[slot] = job.s.wide ? (job.s.cnodes ? kTravWide8 : kTravWide) : kTravReference;
  slot_textured_[slot] = job.s.num_texinfo > 0;
  ++kind_launches[3];
  return s.cuda(cudaGetLastError(), "set job");
}

int Engine::add_items(int slot, unsigned long long items) {
  Status s{err_};
  if (slot < 0 || slot >= kMaxJobs) return s.fail(DSPBR_ERR_INVALID, "job slot %d out of range", slot);
  k_add_items<<<1, 32, 0, stream_>>>(slot, items, js_.p, d_status_);
  ++kind_launches[3];
  return s.cuda(cudaGetLastError(), "add work items");
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
  for (int k : order) {
    const int t = slot_traversal_[k];
    if (t == trav) continue;
    // 4-wide and 8-wide jobs together: the 4-wide tree, which every scene keeps
    const bool wide_mix = (t == kTravWide || t == kTravWide8) && (trav == kTravWide || trav == kTravWide8);
    trav = wide_mix ? kTravWide : kTravPerPath;
  }
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
  launch_shade(sc, b, cur ^ 1, lc_, stream_);
  launch_free_list(sc, b, stream_);
  launch_regen(sc, b, cur ^ 1, stream_);
  launch_commit(sc, b, cur, stream_);
  mark_end();
  kind_launches[0] += 1;
  kind_launches[1] += 1;
  kind_launches[2] += 5;  // shade, free list (2), regen, commit
  cur_ ^= 1;
  return Status{err_}.cuda(cudaGetLastError(), "render launch");
}

// In a captured iteration the closest-hit launch (q[cur]) and the shadow-ray
// launch (qs[cur]) run as parallel branches: extend writes the hit records,
// hit / miss queues and their counters, connect adds to the path radiance;
// neither reads what the other writes.  When few paths are left, each is
// bound by the latency of its slowest ray, and the two overlap.
void Engine::extend_and_connect(const Sched& sc, const PathBuf& b, int cur) {
  cudaEventRecord(fork_, stream_);
  cudaStreamWaitEvent(side_, fork_, 0);
  launch_connect(sc, b, cur, false, lc_, side_);
  launch_extend(sc, b, cur, false, lc_, stream_);
  cudaEventRecord(join_, side_);
  cudaStreamWaitEvent(stream_, join_, 0);
}

void Engine::drop_graph() {
  if (graph_) cudaGraphExecDestroy(graph_);
  graph_ = nullptr;
  for (auto& g : loop_graph_) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
}

// Nodes of `g` that no other node depends on.
static cudaError_t graph_sinks(cudaGraph_t g, std::vector<cudaGraphNode_t>& out) {
  size_t n = 0;
  cudaError_t e = cudaGraphGetNodes(g, nullptr, &n);
  if (e != cudaSuccess) return e;
  std::vector<cudaGraphNode_t> nodes(n);
  if ((e = cudaGraphGetNodes(g, nodes.data(), &n)) != cudaSuccess) return e;
  for (size_t i = 0; i < n; ++i) {
    size_t k = 0;
    if ((e = cudaGraphNodeGetDependentNodes(nodes[i], nullptr, &k)) != cudaSuccess) return e;
    if (k == 0) out.push_back(nodes[i]);
  }
  return cudaSuccess;
}

// while (loop) { iteration(p0); if (second) iteration(p0 ^ 1) }; if (tail[0])
// { connect(0); drain(0); commit(0) }; if (tail[1]) { connect(1); drain(1);
// commit(1) }.  The loop condition starts at 1 on every launch; each
// iteration's commit (kernels.cu, k_commit) decides whether the next one
// runs, so the tail starts after the first iteration that leaves fewer than
// the drain threshold of paths, at either parity.  LoopCtl::iters_left
// bounds the number of iterations.
int Engine::capture_loop_graph(int p0) {
  Status s{err_};
  const Sched sc = sched();
  const PathBuf b = paths();
  if (!loop_ctl_.p) TRY_CUDA(s, loop_ctl_.alloc(1), "loop control");
  cudaGraph_t g = nullptr;
  TRY_CUDA(s, cudaGraphCreate(&g, 0), "loop graph");
  auto fail = [&](cudaError_t e, const char* what) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return s.cuda(e, what);
  };
  // handles: the while loop (entered), iteration B's IF (set by A), one IF
  // per tail parity (set by the commit that stops the loop)
  cudaGraphConditionalHandle h_loop, h_second, h_tail[2];
  cudaError_t e = cudaGraphConditionalHandleCreate(&h_loop, g, 1u, cudaGraphCondAssignDefault);
  for (int k = 0; k < 2 && e == cudaSuccess; ++k)
    e = cudaGraphConditionalHandleCreate(&h_tail[k], g, 0u, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) return fail(e, "loop graph condition");
  auto add_cond = [&](cudaGraph_t parent, const cudaGraphNode_t* deps, size_t ndeps, cudaGraphConditionalHandle h,
                      cudaGraphConditionalNodeType type, cudaGraphNode_t& node, cudaGraph_t& body) {
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = type;
    cp.conditional.size = 1;
    cudaError_t r = cudaGraphAddNode(&node, parent, deps, ndeps, &cp);
    if (r == cudaSuccess) body = cp.conditional.phGraph_out[0];
    return r;
  };
  auto iteration = [&](int cur, const LoopHandles& lh) {
    extend_and_connect(sc, b, cur);
    launch_shade(sc, b, cur ^ 1, lc_, stream_);
    launch_free_list(sc, b, stream_);
    launch_regen(sc, b, cur ^ 1, stream_);
    launch_commit_loop(sc, b, cur, lh, loop_ctl_.p, stream_);
  };
  cudaGraphNode_t loop_node, second_node, tail_node[2];
  cudaGraph_t body = nullptr, body_b = nullptr, tail_body[2] = {nullptr, nullptr};
  cudaGraph_t captured = nullptr;
  e = add_cond(g, nullptr, 0, h_loop, cudaGraphCondTypeWhile, loop_node, body);
  if (e != cudaSuccess) return fail(e, "loop graph node");
  e = cudaGraphConditionalHandleCreate(&h_second, body, 0u, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) return fail(e, "loop graph condition");
  // iteration A (parity p0); the tail after an iteration drains the other parity's queue
  e = cudaStreamBeginCaptureToGraph(stream_, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return fail(e, "loop body capture");
  iteration(p0, LoopHandles{h_loop, h_second, h_tail[p0 ^ 1], 1});
  e = cudaStreamEndCapture(stream_, &captured);
  if (e != cudaSuccess) return fail(e, "loop body capture");
  // iteration B (parity p0 ^ 1) after A's commit, the only node of the body without dependents
  std::vector<cudaGraphNode_t> sinks;
  if ((e = graph_sinks(body, sinks)) != cudaSuccess) return fail(e, "loop body");
  e = add_cond(body, sinks.data(), sinks.size(), h_second, cudaGraphCondTypeIf, second_node, body_b);
  if (e != cudaSuccess) return fail(e, "loop graph node");
  e = cudaStreamBeginCaptureToGraph(stream_, body_b, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return fail(e, "loop body capture");
  iteration(p0 ^ 1, LoopHandles{h_loop, cudaGraphConditionalHandle(0), h_tail[p0], 0});
  e = cudaStreamEndCapture(stream_, &captured);
  if (e != cudaSuccess) return fail(e, "loop body capture");
  // the tails: connect, drain and commit of the parity the loop stopped at
  for (int k = 0; k < 2; ++k) {
    const cudaGraphNode_t dep = k == 0 ? loop_node : tail_node[0];
    e = add_cond(g, &dep, 1, h_tail[k], cudaGraphCondTypeIf, tail_node[k], tail_body[k]);
    if (e != cudaSuccess) return fail(e, "loop graph node");
    e = cudaStreamBeginCaptureToGraph(stream_, tail_body[k], nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return fail(e, "loop tail capture");
    launch_connect(sc, b, k, false, lc_, stream_);
    launch_drain(sc, b, k, lc_, stream_);
    launch_commit(sc, b, k, stream_, false);
    e = cudaStreamEndCapture(stream_, &captured);
    if (e != cudaSuccess) return fail(e, "loop tail capture");
  }
  e = cudaGraphInstantiate(&loop_graph_[p0], g, 0);
  cudaGraphDestroy(g);
  g = nullptr;
  if (e != cudaSuccess) {
    loop_graph_[p0] = nullptr;
    return fail(e, "loop graph instantiate");
  }
  return DSPBR_OK;
}

int Engine::timeline(uint32_t max_entries, std::vector<TimelineEntry>& out) {
  Status s{err_};
  out.clear();
  if (!timeline_.p) return DSPBR_OK;
  std::vector<TimelineEntry> all(kTimeline);
  TRY_CUDA(s, cudaStreamSynchronize(stream_), "timeline");
  TRY_CUDA(s, cudaMemcpy(all.data(), timeline_.p, timeline_.bytes(), cudaMemcpyDeviceToHost), "timeline");
  const unsigned long long last = h_status_->iteration;
  const unsigned long long n = std::min<unsigned long long>({max_entries, last, kTimeline});
  for (unsigned long long it = last + 1 - n; it <= last && n; ++it) {
    const TimelineEntry& e = all[it % kTimeline];
    if (e.iteration == it) out.push_back(e);
  }
  return DSPBR_OK;
}

int Engine::run_loop(int slot, unsigned long long max_iter) {
  Status s{err_};
  const volatile HostStatus* hs = h_status_;
  const unsigned long long it0 = hs->iteration;  // every earlier launch has completed
  const int p0 = cur_;
  if (!loop_graph_[p0]) {
    int rc = capture_loop_graph(p0);
    if (rc) return rc;
  }
  launch_set_loop(loop_ctl_.p, max_iter, drain_below_, kLoopDrain, -1, stream_);
  TRY_CUDA(s, cudaGetLastError(), "loop control");
  TRY_CUDA(s, cudaGraphLaunch(loop_graph_[p0], stream_), "loop graph launch");
  TRY_CUDA(s, cudaStreamSynchronize(stream_), "render");
  // the tail's commit counts as one more iteration
  const unsigned long long body = hs->iteration - it0 - 1;
  kind_launches[0] += body;
  kind_launches[1] += body + 1;
  kind_launches[2] += 5 * body;
  kind_launches[3] += 3;
  cur_ = 0;  // the tail drained every path: both queues are empty
  if (job_done(slot)) return DSPBR_OK;
  return s.fail(DSPBR_ERR_DEVICE_FAULT, "render: job not finished after %llu iterations", max_iter);
}

int Engine::launch_pipelined(int wait_slot, unsigned long long max_iter, cudaEvent_t between,
                             unsigned long long* it0, int* loops) {
  Status s{err_};
  // the caller has waited for every earlier loop launch (a pipelined call is
  // completed before the next one): the status below is current
  *it0 = h_status_->iteration;
  *loops = 0;
  // the loop starts at the parity the last iteration left: kLoopUntilDone
  // ends at the parity it started at (or empties the pool), so the same
  // graph serves the kLoopUntilStarted launch after it
  const int p0 = cur_;
  if (!loop_graph_[p0]) {
    int rc = capture_loop_graph(p0);
    if (rc) return rc;
  }
  if (wait_slot >= 0 && !job_done(wait_slot)) {
    // the previous epoch's paths were all started: each ends within
    // max_bounces + 1 more iterations; the bound only guards the loop
    launch_set_loop(loop_ctl_.p, max_iter, drain_below_, kLoopUntilDone, wait_slot, stream_);
    TRY_CUDA(s, cudaGetLastError(), "loop control");
    TRY_CUDA(s, cudaGraphLaunch(loop_graph_[p0], stream_), "loop graph launch");
    ++*loops;
  }
  if (between) TRY_CUDA(s, cudaEventRecord(between, stream_), "event");
  launch_set_loop(loop_ctl_.p, max_iter, drain_below_, kLoopUntilStarted, -1, stream_);
  TRY_CUDA(s, cudaGetLastError(), "loop control");
  TRY_CUDA(s, cudaGraphLaunch(loop_graph_[p0], stream_), "loop graph launch");
  ++*loops;
  return DSPBR_OK;
}

void Engine::finish_pipelined(unsigned long long it0, int loops) {
  const unsigned long long body = h_status_->iteration - it0;
  kind_launches[0] += body;
  kind_launches[1] += body;
  kind_launches[2] += 5 * body;
  kind_launches[3] += unsigned(loops);
  cur_ = int(h_status_->next_cur & 1u);  // the queues of this parity hold the paths still alive
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
    extend_and_connect(sc, b, cur);
    launch_shade(sc, b, cur ^ 1, lc_, stream_);
    launch_free_list(sc, b, stream_);
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
      kind_launches[2] += 10;
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

int Engine::read_stats(unsigned long long out[8]) {
  Status s{err_};
  k_read_stats<<<1, 32, 0, stream_>>>(stats_.p, d_status_);
  ++kind_launches[3];
  TRY_CUDA(s, cudaGetLastError(), "read stats");
  TRY_CUDA(s, cudaStreamSynchronize(stream_), "read stats");
  for (int i = 0; i < 8; ++i) out[i] = h_status_->stats[i];
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
  if (!counting && !profiling) return run_loop(slot, max_iter);
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
      if (!counting && js.items_next >= js.items_total && h_status_->live_paths < drain_below_) {
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
