// Render engine: one path pool, a device job table and the iteration loop
// over them.  A context's progressive render is one job run to completion; the
// server keeps many jobs active in one engine.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

#include "host.h"
#include "kernels.h"

namespace dspbr {

// The active list travels to the device as a kernel argument: table updates
// need no staging memory and stay ordered on the engine's stream.
struct ActiveList {
  int n;
  int slot[kMaxJobs];
};

class Engine {
 public:
  Engine(int device, cudaStream_t stream, std::string* err) : device_(device), stream_(stream), err_(err) {}
  ~Engine();
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;

  // Job table, counters and the mapped status record (first use).
  int init();
  // Grows the path pool to `capacity` slots.  Only while no job is active.
  int ensure_pool(uint32_t capacity);
  // Drops every path: all slots free, queues empty.  Only while no job is active.
  int reset_pool();
  uint32_t capacity() const { return capacity_; }
  size_t pool_bytes() const;
  void set_launch(const LaunchCfg& lc);
  const LaunchCfg& launch() const { return lc_; }

  // Table updates, enqueued on the stream (ordered before later iterations).
  int set_job(int slot, const Job& job, unsigned long long items_total);
  int cancel_job(int slot);
  int set_active(const std::vector<int>& order);

  // Enqueues at least `n` iterations (two per graph launch when the graph is
  // usable) and returns how many were enqueued in `done`.
  int iterate(int n, bool counting, int* done);
  // Runs iterations until job `slot` has started all items and has no live
  // path, keeping `lookahead` steps queued; `max_iter` bounds the loop.
  int run_until_done(int slot, unsigned long long max_iter, bool counting);
  // The same as one graph launch: a device-side while loop over pairs of
  // iterations (the commit kernel decides whether another pair runs), then
  // the tail drain; the host waits once.  Not while profiling or counting.
  int run_loop(int slot, unsigned long long max_iter);
  // Pipelined frames (the renders of consecutive accumulation epochs overlap):
  // enqueues the loop graph until job `wait_slot` has finished (skipped when
  // wait_slot < 0 or the job has already finished), records `between` (if not
  // null), then the loop graph until every work item of the active jobs has
  // started; no tail, no host wait.  The paths still alive stay in the pool.
  // Returns the iteration counter before the launches in *it0 and the number
  // of loop launches in *loops, for finish_pipelined() once the stream has
  // passed them.
  int launch_pipelined(int wait_slot, unsigned long long max_iter, cudaEvent_t between, unsigned long long* it0,
                       int* loops);
  void finish_pipelined(unsigned long long it0, int loops);
  // More work items for a job already in the table (a progressive render that
  // continues the same accumulation while its earlier paths are in flight).
  int add_items(int slot, unsigned long long items);
  // Any path of any job in the pool (from the last completed iteration).
  bool pool_live() const { return h_status_ && h_status_->live_paths != 0u; }
  void set_drain_below(uint32_t paths) { drain_below_ = paths ? paths : kDrainBelow; }
  unsigned drain_below() const { return drain_below_; }
  // The last (up to max_entries, at most kTimeline) iterations' records, oldest first.
  int timeline(uint32_t max_entries, std::vector<TimelineEntry>& out);
  // Finishes every path in the pool in one launch (connect of the pending
  // shadow rays, then each path run to its end).  Only when no active job has
  // unstarted work items.
  int drain();
  bool job_done(int slot) const;
  const volatile HostStatus* status() const { return h_status_; }

  // Per-kind device time (extend / connect / shade+regen+commit) with events
  // around every launch, and launch counts.
  bool profiling = false;
  double kind_ms[3] = {0, 0, 0};
  unsigned long long kind_launches[4] = {0, 0, 0, 0};  // extend, connect, shade-side, other
  void resolve_marks();
  void clear_marks();

  unsigned long long* stats() const { return stats_.p; }
  // the eight ray counters, read through the mapped status record (no copy engine)
  int read_stats(unsigned long long out[8]);
  Sched sched() const;
  PathBuf paths() const;
  cudaStream_t stream() const { return stream_; }

 private:
  int one_iteration(bool counting);
  int capture_graph();
  int capture_loop_graph(int p0);
  void extend_and_connect(const Sched& sc, const PathBuf& b, int cur);
  void drop_graph();
  cudaEvent_t next_event();
  void mark_begin(int kind);
  void mark_end();

  int device_;
  cudaStream_t stream_;
  std::string* err_;
  bool ready_ = false;
  uint32_t capacity_ = 0;
  int cur_ = 0;  // parity of the next iteration
  int slot_traversal_[kMaxJobs] = {};  // kTravWide / kTravReference of each job slot
  bool slot_textured_[kMaxJobs] = {};  // the job's scene samples material textures
  LaunchCfg lc_;
  // pool
  DevBuf<PathState> st_;
  DevBuf<PathHit> hits_;
  DevBuf<PathShadow> sh_;
  DevBuf<uint32_t> q0_, q1_, qs0_, qs1_, qh_, qm_, qfree_, fmap_, fblock_;
  // job table and counters
  DevBuf<Job> jobs_;
  DevBuf<JobState> js_;
  DevBuf<int> active_;  // kMaxJobs + 1: list, then its length
  DevBuf<uint32_t> counts_;
  DevBuf<unsigned long long> cursors_;  // free head, free tail, iteration
  DevBuf<unsigned long long> stats_;
  DevBuf<TimelineEntry> timeline_;
  HostStatus* h_status_ = nullptr;
  HostStatus* d_status_ = nullptr;
  // two iterations (parity 0 then 1) captured once
  cudaGraphExec_t graph_ = nullptr;
  // a render call: while (device condition) { two iterations }, then the tail;
  // one graph per parity of the loop's first iteration
  cudaGraphExec_t loop_graph_[2] = {nullptr, nullptr};
  // fork / join of the parallel extend and connect branches during capture
  cudaStream_t side_ = nullptr;
  cudaEvent_t fork_ = nullptr, join_ = nullptr;
  DevBuf<LoopCtl> loop_ctl_;
  // loop events and profiling events
  static constexpr int kRing = 8, kLookahead = 4;
  // default: live paths below which a render call drains, checked after every
  // iteration (single-frame 1080p calls of the large workload: 2^14 fastest
  // of 2^11..2^15; at 2^15 the drain starts from 19.5K paths and is 0.2 ms
  // slower than one more iteration and a drain from 6.9K)
  static constexpr unsigned kDrainBelow = 1u << 14;
  unsigned drain_below_ = kDrainBelow;
  cudaEvent_t ring_[kRing] = {};
  std::vector<cudaEvent_t> ev_pool_;
  std::vector<std::pair<int, int>> ev_marks_;
  size_t ev_used_ = 0;
};

}  // namespace dspbr
