// Host-visible interface of the wavefront kernels (kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "device.cuh"

namespace dspbr {

// Per-job constants of the reference's uniform block (renderer.frag:10-31)
// plus the job's image layout.
struct WaveParams {
  Camera cam;
  int npix;              // width * height
  uint32_t frame_base;   // 1-based progressive frame number of work item 0
  int max_bounces;
  int rng_pcg;           // 0: MWC of rng.glsl, 1: PCG32
  uint64_t seed;
  int use_ibl, bg_from_ibl, env_mode, lean, has_ibl;
  float ibl_rot;         // radians
  float4 bg_color;
  float ray_eps, clamp_threshold;
  float rr_prob, rr_factor;
  int rr_start;
  float4 pl_pos, pl_emis;
};

// One render job: a viewport of one scene, rendered for a number of
// progressive frames.  Work item k of a job is pixel k % npix of frame
// frame_base + k / npix.  Jobs live in a device table; paths refer to their
// job by slot index, so jobs of different scenes, sizes and settings share
// one path pool and one set of launches.
struct Job {
  WaveParams p;
  DevScene s;
  DevIbl e;
  double* accum;         // RGBA sums per pixel (FP64)
};

// Device-updated progress of a job.
struct JobState {
  unsigned long long items_next;   // next work item to start
  unsigned long long items_total;  // frames * npix (lowered to items_next to cancel)
  unsigned int live;               // paths of this job in the pool
  unsigned int pad;
};

constexpr int kMaxJobs = 256;  // job table slots = most jobs active at once

// Progress record the commit kernel writes to mapped host memory after every
// iteration; the host reads it after an event that follows the iteration.
struct JobStatus {
  unsigned long long items_next, items_total;
  unsigned int live;
  unsigned int done;  // set once every item has started and no path is live (single 32-bit store)
};
struct HostStatus {
  unsigned long long iteration;     // iterations committed so far
  unsigned int live_paths;          // paths queued for the next extend
  unsigned int nactive;
  unsigned int next_cur;            // parity of the next iteration (0 after a tail drain: both queues empty)
  unsigned int pad;
  JobStatus job[kMaxJobs];          // by job slot
  unsigned long long stats[8];      // ray counters, stored on request (Engine::read_stats)
};

// Queue counters (uint32 slots of PathBuf::counts).  Iteration i works on
// parity cur = i & 1: extend reads q[cur], connect reads qs[cur], shade and
// regen fill q[cur ^ 1] and qs[cur ^ 1]; commit resets what was consumed.
enum : int {
  kCntExt0 = 0,     // extension queues (ping-pong)
  kCntExt1 = 1,
  kCntShadow0 = 2,  // NEE shadow queues (ping-pong)
  kCntShadow1 = 3,
  kCntMiss = 4,     // paths whose extension ray left the scene
  kCntFetchExt = 5,     // next q[cur] entry a k_extend warp starts (dynamic fetch)
  kCntFetchShadow = 6,  // next qs[cur] entry a k_connect warp starts
  kCntHit0 = 8,     // paths whose extension ray hit a triangle, one queue per shading class
  kCntFetchShade = 24,  // next hit-queue entry a k_shade warp starts
  kCntNum = 32
};
constexpr int kNumClasses = 16;
static_assert(kCntHit0 + kNumClasses <= kCntNum, "counter block too small");

// Structure-of-arrays state of a pool of path slots.  Jobs stream their work
// items through the pool: a path that terminates accumulates its sample into
// its job's image and frees its slot, and the next work item takes it.
// Path state of one slot, 96 B: three 32 B sectors that every kernel reads
// and writes whole.  Slots are visited through queues in no particular
// order, so a record per slot (not one array per field) keeps each access to
// whole sectors: a partly written sector costs the memory system a read of
// the rest.
struct __align__(32) PathState {
  float4 org;     // ray origin (the shadow rays of the vertex share it); w: bounces so far (int bits)
  float4 dir;     // xyz; w: job slot (uint bits)
  float4 weight;  // path_weight.xyz, last_bounce_pdf
  float4 rad;     // L.xyz; w: shadow rays pending (int bits: 1 IBL, 2 point light)
  uint64_t rng;
  uint32_t pixel;  // pixel index of the slot's sample
  uint32_t frame;  // progressive frame number of the slot's sample
  uint32_t pad[4];
};
static_assert(sizeof(PathState) == 96, "PathState is three sectors");
// closest hit of the slot's extension ray: t, u, v, triangle id bits (+ pad to a sector)
struct __align__(32) PathHit {
  float4 h;
  float4 pad;
};
// NEE shadow rays of the slot's last vertex, 64 B
struct __align__(32) PathShadow {
  float4 sh_dir;  // IBL shadow ray dir.xyz, tfar
  float4 sh_c;    // IBL NEE contribution * path weight
  float4 pl_dir;  // point-light shadow ray dir.xyz, tfar
  float4 pl_c;
};

__device__ __forceinline__ int path_bounce(const PathState& s) { return __float_as_int(s.org.w); }
__device__ __forceinline__ uint32_t path_job(const PathState& s) { return __float_as_uint(s.dir.w); }
__device__ __forceinline__ int path_flags(const PathState& s) { return __float_as_int(s.rad.w); }

struct PathBuf {
  PathState* st;
  PathHit* hits;
  PathShadow* sh;
  uint32_t* q[2];   // extension queues (slot ids)
  uint32_t* qs[2];  // shadow queues
  uint32_t* qh;     // hit queues: class k at qh + k * capacity
  uint32_t* qm;     // miss queue
  // Free slots.  fmap holds one bit per slot, set while it is free; before
  // each regen k_free_count / k_free_emit write the free slots into qfree in
  // ascending order, and the regen takes the lowest ones, so that new paths
  // sit close together in the path arrays however the old ones ended.
  uint32_t* qfree;
  uint32_t* fmap;    // (capacity + 31) / 32 words
  uint32_t* fblock;  // free slots per kFreeMapBlock words of fmap; last entry: the slots the regen takes
  unsigned long long* free_head;  // slots taken by regens so far
  unsigned long long* free_tail;  // slots freed so far (free_tail - free_head = bits set in fmap)
  uint32_t* counts; // kCnt*
  // [0] closest-hit rays, [1] shadow rays, [2] aborted traversals,
  // [3]/[4] nodes visited / triangles tested by closest-hit rays, [5]/[6] by shadow rays
  unsigned long long* stats;
  uint32_t capacity;
};

// The job table as the kernels see it.
// Per-iteration record written by k_commit (a ring of kTimeline entries,
// indexed by iteration number): device clock and paths queued afterwards.
constexpr int kTimeline = 1024;
struct TimelineEntry {
  unsigned long long iteration, t_ns;
  unsigned int live, pad;
};

struct Sched {
  const Job* jobs;        // kMaxJobs slots
  JobState* js;           // kMaxJobs slots
  const int* active;      // job slots in priority order
  const int* nactive;
  HostStatus* status;     // mapped host memory (device pointer)
  unsigned long long* iteration;
  TimelineEntry* timeline;  // kTimeline entries
};

// Traversal of the path kernels: per path (the job's DevScene::wide), or one
// kind for every path when all active jobs use the same (smaller kernels).
// kTravWide: the 4-wide tree; kTravWide8: the compressed 8-wide tree (every
// active job's scene has one); kTravPerPath: each job's own choice (wide
// jobs take the 4-wide tree, which every scene keeps)
enum : int { kTravPerPath = 0, kTravWide = 1, kTravReference = 2, kTravWide8 = 3 };

struct LaunchCfg {
  int trace_blocks = 148 * 16, trace_threads = 128;
  int shade_blocks = 148 * 8, shade_threads = 128;
  int traversal = kTravPerPath;
  bool textured = false;  // some active job samples material textures
  int dyn_blocks = 148 * 8;          // k_extend_dyn: resident blocks of 128 threads (64 registers)
  int connect_dyn_blocks = 148 * 8;  // k_connect_dyn: the same
  // resident blocks of the persistent shading kernels (set by init_launch_sizes)
  int shade_dyn_blocks[2] = {148 * 5, 148 * 5};  // k_shade<false>, k_shade<true>, 128 threads
};

void launch_init_pool(const PathBuf& b, cudaStream_t st);
// resident-block counts of the persistent kernels on this device (occupancy API)
void init_launch_sizes(LaunchCfg& lc);
// the most blocks per SM each persistent kernel can keep resident, and the SM count
struct LaunchLimits {
  int sms, trace_per_sm, connect_per_sm, shade_per_sm[2];
};
LaunchLimits launch_limits();
constexpr int kFreeMapBlock = 1024;  // fmap words per block of the free-list kernels
// the free slots the next regen takes, in ascending order (qfree), from fmap:
// call right before launch_regen
void launch_free_list(const Sched& sc, const PathBuf& b, cudaStream_t st);
void launch_regen(const Sched& sc, const PathBuf& b, int next, cudaStream_t st);
void launch_extend(const Sched& sc, const PathBuf& b, int cur, bool count, const LaunchCfg& lc, cudaStream_t st);
void launch_connect(const Sched& sc, const PathBuf& b, int cur, bool count, const LaunchCfg& lc, cudaStream_t st);
void launch_shade(const Sched& sc, const PathBuf& b, int next, const LaunchCfg& lc, cudaStream_t st);
void launch_commit(const Sched& sc, const PathBuf& b, int cur, cudaStream_t st, bool regen_ran = true);

// Device-side loop control of a render call run as one graph.  The loop body
// is iteration A, then iteration B of the other parity under an IF node; the
// loop graph is captured once per parity of A.
// kLoopDrain: after each iteration k_commit keeps going while iterations
// remain and either a work item has not started or at least drain_below paths
// are alive; the commit that stops selects the tail of its parity (an IF node
// each), which runs every remaining path to its end.
// kLoopUntilStarted (pipelined frames): stops after the first iteration whose
// regen placed every work item of the active jobs, at either parity; the paths
// still alive stay in the pool, and the next launch takes the loop graph that
// starts at HostStatus::next_cur.
// kLoopUntilDone (pipelined frames): whole pairs (A always continues to B, so
// the launch ends at the parity it started at) until job wait_job has finished
// (every item started, no live path); it ends in the tail instead, like
// kLoopDrain, once every work item has started and fewer than drain_below
// paths are alive: the pool is then empty.
enum { kLoopDrain = 0, kLoopUntilDone = 1, kLoopUntilStarted = 2 };
struct LoopCtl {
  unsigned long long iters_left;
  unsigned long long drain_below;
  int mode;      // kLoop*
  int wait_job;  // kLoopUntilDone: the job slot to finish
};
struct LoopHandles {
  cudaGraphConditionalHandle loop;    // the while node
  cudaGraphConditionalHandle second;  // iteration B's IF node (set by A)
  cudaGraphConditionalHandle tail;    // the IF node of the tail that follows this iteration
  int first;                          // 1: iteration A
};
void launch_commit_loop(const Sched& sc, const PathBuf& b, int cur, const LoopHandles& h, LoopCtl* ctl,
                        cudaStream_t st);
void launch_set_loop(LoopCtl* ctl, unsigned long long iterations, unsigned long long drain_below, int mode,
                     int wait_job, cudaStream_t st);
// runs every path queued in q[cur] to its end (call after connect(cur), when no work item is left)
void launch_drain(const Sched& sc, const PathBuf& b, int cur, const LaunchCfg& lc, cudaStream_t st);
void launch_mean(const double4* accum, double inv_count, float4* out, int npix, cudaStream_t st);

// kernel-level queries (device buffers)
void launch_trace_rays(const DevScene& s, const float4* rays, uint32_t n, int any, int32_t* tri, float* t, float2* uv,
                       int32_t* occ, cudaStream_t st);
void launch_bsdf_query(const DevScene& s, uint32_t n, const float* hit20, const float* wo3, const float* rnd4,
                       int lean, float* eval4, float* sample10, int32_t* flags, cudaStream_t st);
void launch_ibl_query(const DevIbl& e, float rot, int mode, uint32_t n, const float* r2, const float* dirs,
                      float* sdp4, float* pdf, float* rgb, cudaStream_t st);
void launch_camera_rays(const Camera& c, uint32_t n, const int32_t* xy, const float* r2, float* rays6,
                        cudaStream_t st);

// environment tables (ibl.cu)
void launch_ibl_tables(const float4* rgba, int w, int h, float* lum, float* pdf, float* cdf, float* rowsum,
                       float* ypdf, float* ycdf, double* total, cudaStream_t st);

// scene preparation (kernels.cu)
void launch_gather_tris(const float4* verts, const uint32_t* indices, const int32_t* remap, uint32_t nslots,
                        uint32_t ntris, float4* tris, cudaStream_t st);

}  // namespace dspbr
