// Wavefront path tracer with path regeneration over a table of jobs.
//
// The reference evaluates a whole path per fragment (renderer.frag:146-157 ->
// integrator/misptdl.glsl:34-93).  Here the pixel samples of one or many
// render jobs stream through a fixed pool of path slots; every iteration runs
//   extend      closest hit for every live path (bvh.glsl:149-216); misses go
//               to one queue, hits to the queue of their material class,
//   connect     any-hit test of the NEE shadow rays emitted by the previous
//               shade; visible contributions are added to the path radiance,
//   shade       surface hits by material class: RR, absorption, emission, BSDF
//               sampling, NEE sample generation (misptdl.glsl:54-90,
//               renderer.frag:94-123); then, in the same launch, the misses:
//               background / MIS-weighted environment (misptdl.glsl:41-46, 84-88),
//   regen       new samples (rng_init + calcuateViewRay) of the active jobs,
//               in priority order, into the slots freed by terminated paths,
//   commit      job progress, free-list head, queue counter resets and the
//               status record for the host,
// so every launch works on a full pool instead of a shrinking per-bounce
// queue, and an iteration is a fixed launch sequence whose arguments never
// change (it can be captured in a CUDA graph).  Queues are compacted with one
// atomic per warp (__ballot_sync / __popc, __match_any_sync for keyed
// queues); a finished path adds its sample to its job's FP64 pixel sums.  The
// per-path arithmetic and RNG consumption order follow the reference exactly.
#include <cuda_runtime.h>

#include "kernels.h"

namespace dspbr {

namespace {

DEV void enqueue(uint32_t* q, uint32_t* counter, bool pred, uint32_t value) {
  unsigned m = __ballot_sync(0xffffffffu, pred);
  if (!m) return;
  int lane = threadIdx.x & 31;
  int leader = __ffs(m) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(counter, uint32_t(__popc(m)));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (pred) q[base + __popc(m & ((1u << lane) - 1u))] = value;
}

// Append to one of several queues (queue `key` starts at q + key * stride):
// lanes with the same key share one atomic.
DEV void enqueue_keyed(uint32_t* q, uint32_t* counters, uint32_t stride, bool pred, int key, uint32_t value) {
  if (!__ballot_sync(0xffffffffu, pred)) return;
  int k = pred ? key : -1;
  unsigned peers = __match_any_sync(0xffffffffu, k);
  int lane = threadIdx.x & 31;
  int leader = __ffs(peers) - 1;
  uint32_t base = 0;
  if (pred && lane == leader) base = atomicAdd(counters + key, uint32_t(__popc(peers)));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (pred) q[size_t(key) * stride + base + __popc(peers & ((1u << lane) - 1u))] = value;
}

DEV void count_warp(unsigned long long* ctr, bool pred) {
  unsigned m = __ballot_sync(0xffffffffu, pred);
  if ((threadIdx.x & 31) == 0 && m) atomicAdd(ctr, (unsigned long long)__popc(m));
}

DEV void add_warp(unsigned long long* ctr, uint32_t v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(ctr, (unsigned long long)v);
}

DEV float4 f4(v3 a, float w) { return make_float4(a.x, a.y, a.z, w); }

// A terminated path adds its sample to its job's pixel sums; the caller
// frees the slot (free_slots).
DEV void finish_path(const Job& J, uint32_t pixel, float4 c) {
  double* a = J.accum + 4 * size_t(pixel);
  atomicAdd(a + 0, double(c.x));
  atomicAdd(a + 1, double(c.y));
  atomicAdd(a + 2, double(c.z));
  atomicAdd(a + 3, double(c.w));
}

// Frees the slots of terminated paths: their bits in the free map, the count
// of freed slots and the live-path count of each job (one atomic per job per warp).
DEV void free_slots(const Sched& sc, const PathBuf& b, bool pred, uint32_t slot, uint32_t job) {
  unsigned m = __ballot_sync(0xffffffffu, pred);
  if (!m) return;
  int lane = threadIdx.x & 31;
  int leader = __ffs(m) - 1;
  if (lane == leader) atomicAdd(b.free_tail, (unsigned long long)__popc(m));
  if (pred) atomicOr(b.fmap + (slot >> 5), 1u << (slot & 31u));
  unsigned peers = __match_any_sync(0xffffffffu, pred ? int(job) : -1);
  if (pred && lane == __ffs(peers) - 1) atomicSub(&sc.js[job].live, uint32_t(__popc(peers)));
}

// The same for persistent warps, batched: freed slots collect in a per-warp
// shared-memory buffer and go to the free list with one atomic on its tail
// per kFreeBuf slots; live-path decrements collect per job in a register.
// Per batch of 32 paths, free_slots costs an atomic on a counter that every
// warp of the kernel updates; here a warp flushes a few times per launch.
// flush() must run before the warp exits.
constexpr int kFreeBuf = 256;
struct WarpFree {
  uint32_t* buf;  // this warp's kFreeBuf entries (shared memory)
  uint32_t n;     // entries held (warp-uniform)
  int job;        // job of the pending live decrement (warp-uniform), -1: none
  uint32_t dec;
  DEV void init(uint32_t* warp_buf) {
    buf = warp_buf;
    n = 0;
    job = -1;
    dec = 0;
  }
  DEV void flush_slots(const PathBuf& b) {
    if (!n) return;
    const int lane = threadIdx.x & 31;
    if (lane == 0) atomicAdd(b.free_tail, (unsigned long long)n);
    __syncwarp();
    for (uint32_t k = uint32_t(lane); k < n; k += 32u) {
      const uint32_t slot = buf[k];
      atomicOr(b.fmap + (slot >> 5), 1u << (slot & 31u));
    }
    __syncwarp();
    n = 0;
  }
  DEV void flush_live(const Sched& sc) {
    if (job >= 0 && dec && (threadIdx.x & 31) == 0) atomicSub(&sc.js[job].live, dec);
    job = -1;
    dec = 0;
  }
  DEV void flush(const Sched& sc, const PathBuf& b) {
    flush_slots(b);
    flush_live(sc);
  }
  DEV void add(const Sched& sc, const PathBuf& b, bool pred, uint32_t slot, uint32_t jb) {
    const unsigned m = __ballot_sync(0xffffffffu, pred);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    if (n + uint32_t(__popc(m)) > uint32_t(kFreeBuf)) flush_slots(b);
    if (pred) buf[n + uint32_t(__popc(m & ((1u << lane) - 1u)))] = slot;
    n += uint32_t(__popc(m));
    __syncwarp();
    // live counts: one job for every freed path of the batch (the usual case) or several
    const int first_job = __shfl_sync(0xffffffffu, int(jb), __ffs(m) - 1);
    const bool one_job = __all_sync(0xffffffffu, !pred || int(jb) == first_job);
    if (one_job) {
      if (first_job != job) {
        flush_live(sc);
        job = first_job;
      }
      dec += uint32_t(__popc(m));
    } else {
      const unsigned peers = __match_any_sync(0xffffffffu, pred ? int(jb) : -1);
      if (pred && lane == __ffs(peers) - 1) atomicSub(&sc.js[jb].live, uint32_t(__popc(peers)));
    }
  }
};

// Exclusive prefix sum over the block (blockDim.x == kMaxJobs threads); `n`
// values are non-zero at most (a single active job needs no scan).
DEV unsigned long long block_scan(unsigned long long v, unsigned long long* sh, unsigned long long& total, int n) {
  const int t = threadIdx.x;
  if (n <= 1) {
    if (t == 0) sh[0] = v;
    __syncthreads();
    total = sh[0];
    __syncthreads();
    return 0ull;
  }
  sh[t] = v;
  __syncthreads();
  for (int off = 1; off < kMaxJobs; off <<= 1) {
    unsigned long long add = t >= off ? sh[t - off] : 0ull;
    __syncthreads();
    sh[t] += add;
    __syncthreads();
  }
  unsigned long long inc = sh[t];
  total = sh[kMaxJobs - 1];
  __syncthreads();
  return inc - v;
}

// Work items not yet started of active job number `a` (0 beyond the list).
DEV unsigned long long remaining(const Sched& sc, int a, int n, int& j) {
  j = -1;
  if (a >= n) return 0ull;
  j = sc.active[a];
  unsigned long long next = sc.js[j].items_next, total = sc.js[j].items_total;
  return total > next ? total - next : 0ull;
}

}  // namespace

// ---- pool set-up -----------------------------------------------------------------------------
__global__ void k_init_pool(PathBuf b) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < b.capacity; i += gridDim.x * blockDim.x)
    b.qfree[i] = i;
  const uint32_t words = (b.capacity + 31u) / 32u;
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < words; w += gridDim.x * blockDim.x) {
    const uint32_t left = b.capacity - w * 32u;  // every slot starts free
    b.fmap[w] = left >= 32u ? 0xffffffffu : (1u << left) - 1u;
  }
  if (blockIdx.x == 0 && threadIdx.x < kCntNum) {
    b.counts[threadIdx.x] = 0u;
    if (threadIdx.x == 0) {
      *b.free_head = 0ull;
      *b.free_tail = b.capacity;
    }
  }
}

// ---- the free list: fmap -> qfree in ascending order ------------------------------------------
DEV uint32_t block_sum_1024(uint32_t v, uint32_t* warp_sums) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (lane == 0) warp_sums[warp] = v;
  __syncthreads();
  uint32_t t = threadIdx.x < (blockDim.x >> 5) ? warp_sums[threadIdx.x] : 0u;
  if (warp == 0)
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  __syncthreads();
  return t;  // the total in thread 0
}

// Free slots per block of kFreeMapBlock map words, and (block 0) how many
// the regen will take: min(free slots, work items the active jobs have left),
// in fblock[nblocks].
__global__ void __launch_bounds__(kFreeMapBlock) k_free_count(Sched sc, PathBuf b) {
  __shared__ uint32_t warp_sums[32];
  __shared__ unsigned long long scan[kMaxJobs];
  const uint32_t words = (b.capacity + 31u) / 32u;
  const uint32_t w = blockIdx.x * kFreeMapBlock + threadIdx.x;
  const uint32_t total = block_sum_1024(w < words ? uint32_t(__popc(b.fmap[w])) : 0u, warp_sums);
  if (threadIdx.x == 0) b.fblock[blockIdx.x] = total;
  if (blockIdx.x == 0) {
    const int n = min(*sc.nactive, kMaxJobs);
    int j;
    unsigned long long rem = threadIdx.x < kMaxJobs ? remaining(sc, threadIdx.x, n, j) : 0ull;
    if (threadIdx.x < kMaxJobs) scan[threadIdx.x] = rem;
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long sum = 0;
      for (int k = 0; k < n; ++k) sum += scan[k];
      const unsigned long long nfree = *b.free_tail - *b.free_head;
      b.fblock[gridDim.x] = uint32_t(min(sum, nfree));
    }
  }
}

// The first `need` free slots in ascending order: each block starts at the
// count of the blocks before it; a warp writes its 32 words' slots
// cooperatively (lane k of a round takes the warp's k-th free slot), so that
// consecutive lanes store consecutive entries.
__global__ void __launch_bounds__(kFreeMapBlock) k_free_emit(PathBuf b) {
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t block_base;
  const uint32_t words = (b.capacity + 31u) / 32u;
  const uint32_t need = b.fblock[gridDim.x];
  uint32_t before = 0;
  for (uint32_t k = threadIdx.x; k < blockIdx.x; k += blockDim.x) before += b.fblock[k];
  before = block_sum_1024(before, warp_sums);
  if (threadIdx.x == 0) block_base = before;
  __syncthreads();
  if (block_base >= need) return;  // every slot the regen takes lies before this block
  const uint32_t w = blockIdx.x * kFreeMapBlock + threadIdx.x;
  const uint32_t bits = w < words ? b.fmap[w] : 0u;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t c = uint32_t(__popc(bits));
  uint32_t incl = c;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t n = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += n;
  }
  const uint32_t warp_total = __shfl_sync(0xffffffffu, incl, 31);
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t t = lane < int(blockDim.x >> 5) ? warp_sums[lane] : 0u, ti = t;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t n = __shfl_up_sync(0xffffffffu, ti, o);
      if (lane >= o) ti += n;
    }
    warp_sums[lane] = ti - t;  // exclusive prefix of the warps
  }
  __syncthreads();
  const uint32_t pos0 = block_base + warp_sums[warp];
  const uint32_t word0 = blockIdx.x * kFreeMapBlock + uint32_t(warp) * 32u;
  for (uint32_t k0 = 0; k0 < warp_total && pos0 + k0 < need; k0 += 32u) {
    const uint32_t k = k0 + uint32_t(lane);
    // the lane j whose word holds the warp's k-th free slot: the first with incl > k
    int lo = 0, hi = 31;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      const uint32_t v = __shfl_sync(0xffffffffu, incl, mid);
      if (v > k) hi = mid;
      else lo = mid + 1;
    }
    const uint32_t jb = __shfl_sync(0xffffffffu, bits, lo);
    const uint32_t jc = __shfl_sync(0xffffffffu, c, lo), ji = __shfl_sync(0xffffffffu, incl, lo);
    if (k < warp_total && pos0 + k < need) {
      const uint32_t bit = __fns(jb, 0u, int(k - (ji - jc)) + 1);
      b.qfree[pos0 + k] = (word0 + uint32_t(lo)) * 32u + bit;
    }
  }
}

// ---- regen: new samples in free slots (renderer.frag:146-150) ----------------------------
// The k-th pixel of a frame in the order its samples start: 8 x 4 tiles (the
// 32 consecutive work items a warp takes), tile rows top to bottom; then the
// columns right of the last whole tile of each band of 4 rows, and the rows
// below the last whole band, in row order.  A bijection of [0, width*height):
// only the order changes, not a pixel's index, random stream or sums; the rays
// of a warp start from a compact patch instead of a 32 x 1 strip.
DEV void tile_pixel(uint32_t k, uint32_t w, uint32_t h, int& px, int& py) {
  const uint32_t w8 = w & ~7u, h4 = h & ~3u;
  if (k < h4 * w) {
    const uint32_t band = k / (4u * w), r = k - band * 4u * w;
    if (r < 4u * w8) {
      const uint32_t t = r >> 5, j = r & 31u;
      px = int(t * 8u + (j & 7u));
      py = int(band * 4u + (j >> 3));
    } else {
      const uint32_t r2 = r - 4u * w8, wr = w - w8;
      px = int(w8 + r2 % wr);
      py = int(band * 4u + r2 / wr);
    }
  } else {
    const uint32_t r = k - h4 * w;
    px = int(r % w);
    py = int(h4 + r / w);
  }
}

// Free slot i (in free-list order) takes the i-th unstarted work item of the
// active jobs in priority order and entry base + i of q[next], where base is
// the queue's length after this iteration's shade (no atomic: k_commit adds
// the number of new paths to the queue counter).
__global__ void __launch_bounds__(kMaxJobs) k_regen(Sched sc, PathBuf b, int next) {
  __shared__ unsigned long long scan[kMaxJobs];
  __shared__ unsigned long long pre[kMaxJobs];
  __shared__ int act[kMaxJobs];
  const int n = min(*sc.nactive, kMaxJobs);
  int j;
  unsigned long long rem = remaining(sc, threadIdx.x, n, j), total;
  pre[threadIdx.x] = block_scan(rem, scan, total, n);
  act[threadIdx.x] = j;
  __syncthreads();
  const unsigned long long head = *b.free_head;
  const unsigned long long nfree = *b.free_tail - head;
  const uint32_t avail = uint32_t(min(nfree, total));
  uint32_t* q = b.q[next] + b.counts[next];
  for (uint32_t base = blockIdx.x * blockDim.x; base < avail; base += gridDim.x * blockDim.x) {
    uint32_t i = base + threadIdx.x;
    {
      // the slots taken leave the free map: one atomic per map word and warp
      // (consecutive entries of the ascending list share words)
      const bool take = i < avail;
      const uint32_t s = take ? b.qfree[i] : 0u;
      const unsigned peers = __match_any_sync(0xffffffffu, take ? int(s >> 5) : -1);
      const uint32_t bits = __reduce_or_sync(peers, take ? 1u << (s & 31u) : 0u);
      if (take && (threadIdx.x & 31) == __ffs(peers) - 1) atomicAnd(b.fmap + (s >> 5), ~bits);
    }
    if (i < avail) {
      uint32_t slot = 0;
      int lo = 0, hi = n - 1;  // last active job whose range starts at or before i
      while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= i) lo = mid;
        else hi = mid - 1;
      }
      const int jj = act[lo];
      const WaveParams& p = sc.jobs[jj].p;
      unsigned long long item = sc.js[jj].items_next + (i - pre[lo]);
      slot = b.qfree[i];
      uint32_t k, frame;
      if (item <= 0xffffffffull) {
        k = uint32_t(item) % uint32_t(p.npix);
        frame = p.frame_base + uint32_t(item) / uint32_t(p.npix);
      } else {
        k = uint32_t(item % uint64_t(p.npix));
        frame = p.frame_base + uint32_t(item / uint64_t(p.npix));
      }
      int px, py;
      tile_pixel(k, uint32_t(p.cam.width), uint32_t(p.cam.height), px, py);
      const uint32_t pixel = uint32_t(py) * uint32_t(p.cam.width) + uint32_t(px);
      Rng r;
      if (p.rng_pcg) {
        uint64_t stream = uint64_t(frame) * uint64_t(p.npix) + pixel;
        r.inc = pcg_inc(stream);
        r.state = pcg_init(p.seed, stream);
      } else {
        Mwc m = mwc_init(int(frame) * p.max_bounces, px, py);
        r.state = uint64_t(m.x) | (uint64_t(m.y) << 32);
        r.inc = 0;
      }
      float r0 = r.next();
      float r1 = r.next();
      v3 org, dir;
      camera_ray(p.cam, px, py, r0, r1, org, dir);
      PathState ps;
      ps.org = f4(org, __int_as_float(0));
      ps.dir = f4(dir, __uint_as_float(uint32_t(jj)));
      ps.weight = make_float4(1.f, 1.f, 1.f, 0.f);
      ps.rad = make_float4(0.f, 0.f, 0.f, __int_as_float(0));
      ps.rng = r.state;
      ps.pixel = pixel;
      ps.frame = frame;
      ps.pad[0] = ps.pad[1] = ps.pad[2] = ps.pad[3] = 0u;
      b.st[slot] = ps;
      q[i] = slot;
    }
  }
}

// ---- commit: book-keeping of one iteration (one block of kMaxJobs threads) -----------------
// regen_ran = false (after a drain): no work item was handed out, only the
// counters and the status are updated.
__global__ void __launch_bounds__(kMaxJobs) k_commit(Sched sc, PathBuf b, int cur, int regen_ran, LoopHandles lh,
                                                     LoopCtl* ctl) {
  __shared__ unsigned long long scan[kMaxJobs];
  const int n = min(*sc.nactive, kMaxJobs);
  int j;
  unsigned long long rem = remaining(sc, threadIdx.x, n, j), total;
  unsigned long long pre = block_scan(rem, scan, total, n);
  const unsigned long long head = *b.free_head;
  const unsigned long long avail = regen_ran ? min(*b.free_tail - head, total) : 0ull;
  // the regen that just ran gave job a the items [pre, pre + rem) clipped to avail
  if (j >= 0 && avail > pre) {
    unsigned long long took = min(avail - pre, rem);
    sc.js[j].items_next += took;
    sc.js[j].live += uint32_t(took);
  }
  __syncthreads();
  const int t = threadIdx.x;
  if (t == 0) {
    *b.free_head = head + avail;
    b.counts[cur ^ 1] += uint32_t(avail);  // q[next]: the paths the regen that just ran appended
    b.counts[cur] = 0;                 // q[cur]: consumed by this iteration's extend
    b.counts[kCntShadow0 + cur] = 0;   // qs[cur]: consumed by this iteration's connect
    b.counts[kCntMiss] = 0;
    b.counts[kCntFetchExt] = 0;
    b.counts[kCntFetchShadow] = 0;
    b.counts[kCntFetchShade] = 0;
  }
  if (t < kNumClasses) b.counts[kCntHit0 + t] = 0;
  // status for the host (mapped memory)
  if (j >= 0) {
    volatile JobStatus* s = &sc.status->job[j];
    const unsigned long long nx = sc.js[j].items_next, tot = sc.js[j].items_total;
    const unsigned int live = sc.js[j].live;
    s->items_next = nx;
    s->items_total = tot;
    s->live = live;
    if (nx >= tot && live == 0u) s->done = 1u;
  }
  __syncthreads();
  if (t == 0) {
    unsigned long long it = *sc.iteration + 1;
    *sc.iteration = it;
    volatile HostStatus* hs = sc.status;
    const unsigned int live = b.counts[cur ^ 1];
    hs->live_paths = live;
    hs->nactive = uint32_t(n);
    hs->next_cur = regen_ran ? uint32_t(cur ^ 1) : 0u;
    __threadfence_system();
    hs->iteration = it;
    unsigned long long now;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
    TimelineEntry te;
    te.iteration = it;
    te.t_ns = now;
    te.live = live;
    te.pad = 0;
    sc.timeline[it % kTimeline] = te;
    if (ctl) {  // the render loop's next iteration, or the tail
      const bool started = total <= avail;  // the regen that just ran placed every remaining work item
      const unsigned long long left = ctl->iters_left;
      const int mode = ctl->mode;
      bool stop, tail = false;
      if (mode == kLoopDrain) {
        stop = started && live < ctl->drain_below;
      } else if (mode == kLoopUntilDone) {
        const int w = ctl->wait_job;
        stop = w < 0 || w >= kMaxJobs || (sc.js[w].items_next >= sc.js[w].items_total && sc.js[w].live == 0u);
        // every work item of every active job has started and few paths are
        // left: the tail drain finishes them all (the iterations it replaces
        // would each cost a path's latency, whatever they hold)
        if (!stop && started && live < ctl->drain_below) stop = tail = true;
      } else {
        stop = started;
      }
      const bool go = left > 1 && !stop;
      ctl->iters_left = left ? left - 1 : 0;
      if (mode == kLoopUntilDone && !tail) {  // whole pairs, no tail
        if (lh.first) cudaGraphSetConditional(lh.second, 1u);
        else cudaGraphSetConditional(lh.loop, go ? 1u : 0u);
      } else {
        if (lh.first) {
          cudaGraphSetConditional(lh.second, go ? 1u : 0u);
          if (!go) cudaGraphSetConditional(lh.loop, 0u);
        } else {
          cudaGraphSetConditional(lh.loop, go ? 1u : 0u);
        }
        if (!go && mode != kLoopUntilStarted) cudaGraphSetConditional(lh.tail, 1u);
      }
    }
  }
}

__global__ void k_set_loop(LoopCtl* ctl, unsigned long long iterations, unsigned long long drain_below, int mode,
                           int wait_job) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ctl->iters_left = iterations;
    ctl->drain_below = drain_below;
    ctl->mode = mode;
    ctl->wait_job = wait_job;
  }
}

// ---- extend: closest hit ------------------------------------------------------------------------
// Closest hit / any hit of one path ray with the traversal the variant names:
// counting frames take the reference's binary traversal, whose node and
// triangle counts define the algorithmic bytes of the roofline.
template <bool kAny, bool kCount, int kTrav>
DEV bool trace_path_ray(const DevScene& s, v3 org, v3 dir, float tfar, Hit& h, bool& aborted, uint32_t* nodes,
                        uint32_t* tris) {
  if (!kCount && kTrav == kTravWide8) return traverse_cw8_rt(s, org, dir, tfar, kAny, h, aborted);
  if (!kCount && (kTrav == kTravWide || (kTrav == kTravPerPath && s.wide)))
    return traverse_wide4<kAny>(s, org, dir, tfar, h, aborted);
  return traverse<kAny>(s, org, dir, tfar, h, aborted, kCount ? nodes : nullptr, kCount ? tris : nullptr);
}

// 256 threads x 4 blocks per SM: at most 64 registers, 32 warps resident
template <bool kCount, int kTrav>
__global__ void __launch_bounds__(256, 4) k_extend(Sched sc, PathBuf b, int cur) {
  const uint32_t count = b.counts[cur];
  const uint32_t* q = b.q[cur];
  for (uint32_t base = blockIdx.x * blockDim.x; base < count; base += gridDim.x * blockDim.x) {
    uint32_t i = base + threadIdx.x;
    bool aborted = false, is_hit = false, is_miss = false;
    uint32_t nodes = 0, tris = 0, slot = 0;
    int cls = 0;
    if (i < count) {
      slot = q[i];
      const float4 o = b.st[slot].org, d = b.st[slot].dir;
      const DevScene& s = sc.jobs[__float_as_uint(d.w)].s;
      Hit h;
      trace_path_ray<false, kCount, kTrav>(s, mk(o), mk(d), kTfarMax, h, aborted, &nodes, &tris);
      b.hits[slot] = PathHit{make_float4(h.t, h.u, h.v, __int_as_float(h.tri)), make_float4(0.f, 0.f, 0.f, 0.f)};
      is_hit = h.tri >= 0;
      is_miss = !is_hit;
      if (is_hit) cls = __ldg(s.tri_class + h.tri);
    }
    // misses go to the environment kernel, hits to the queue of their
    // material's shading class
    enqueue_keyed(b.qh, b.counts + kCntHit0, b.capacity, is_hit, cls, slot);
    enqueue(b.qm, b.counts + kCntMiss, is_miss, slot);
    count_warp(b.stats + 0, i < count);
    count_warp(b.stats + 2, aborted);
    if (kCount) {
      add_warp(b.stats + 3, nodes);
      add_warp(b.stats + 4, tris);
    }
  }
}

// Persistent warps (one grid of resident blocks) that take batches of 32
// consecutive queue entries: the first batch of a warp is its own index, the
// later ones come from a cursor (one atomic per batch), so a warp that drew
// short work takes more and a short queue costs no atomic at all.  Starting
// rays one lane at a time as lanes finish balanced the lanes better but was
// slower (each start pays the latency of a ray's first loads) and lost the
// queue order the shading kernels' memory accesses benefit from.
DEV bool next_warp_batch(uint32_t* cursor, uint32_t count, uint32_t& i, bool& first) {
  const int lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  uint32_t batch;
  if (first) {
    batch = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    first = false;
  } else {
    uint32_t c = 0;
    if (lane == 0) c = atomicAdd(cursor, 1u);
    batch = warps + __shfl_sync(0xffffffffu, c, 0);
  }
  if (batch >= (count + 31u) / 32u) return false;
  i = batch * 32u + uint32_t(lane);
  return true;
}

DEV void shade_miss_path(const Sched& sc, const PathBuf& b, uint32_t slot);

// closest hits of q[cur], 4-wide traversal (kTrav kTravWide) or compressed 8-wide (kTravWide8).  A camera ray that leaves the
// scene ends its path here: its sample is the background (misptdl.glsl:41-46),
// added to the job's sums before the slot is freed, instead of a trip through
// the miss queue and the shading kernel.  Only camera rays: a later vertex's
// path may still receive its shadow rays' contribution from k_connect, which
// runs beside this kernel; its misses are shaded after both.
template <int kTrav>
__global__ void __launch_bounds__(128, 8) k_extend_dyn(Sched sc, PathBuf b, int cur) {
  const uint32_t count = b.counts[cur];
  const uint32_t* q = b.q[cur];
  uint32_t rays = 0, aborted_n = 0;
  uint32_t i;
  bool first = true;
  while (next_warp_batch(b.counts + kCntFetchExt, count, i, first)) {
    bool is_hit = false, is_miss = false, sky = false;
    uint32_t slot = 0, job = 0;
    int cls = 0;
    if (i < count) {
      slot = q[i];
      const float4 o = b.st[slot].org, d = b.st[slot].dir;
      job = __float_as_uint(d.w);
      const DevScene& s = sc.jobs[job].s;
      Hit h;
      bool aborted = false;
      trace_path_ray<false, false, kTrav>(s, mk(o), mk(d), kTfarMax, h, aborted, nullptr, nullptr);
      is_hit = h.tri >= 0;
      is_miss = !is_hit;
      sky = is_miss && __float_as_int(o.w) == 0;
      if (!sky)
        b.hits[slot] = PathHit{make_float4(h.t, h.u, h.v, __int_as_float(h.tri)), make_float4(0.f, 0.f, 0.f, 0.f)};
      if (is_hit) cls = __ldg(s.tri_class + h.tri);
      ++rays;
      aborted_n += aborted ? 1u : 0u;
    }
    if (sky) shade_miss_path(sc, b, slot);
    free_slots(sc, b, sky, slot, job);
    enqueue_keyed(b.qh, b.counts + kCntHit0, b.capacity, is_hit, cls, slot);
    enqueue(b.qm, b.counts + kCntMiss, is_miss && !sky, slot);
  }
  add_warp(b.stats + 0, rays);
  add_warp(b.stats + 2, aborted_n);
}

// ---- connect: NEE shadow rays (bvh.glsl:218-229) ---------------------------------------------
// The NEE shadow rays of one path vertex (IBL and point light): visible
// contributions are added to the path radiance.
template <bool kCount, int kTrav>
DEV void connect_slot(const Sched& sc, const PathBuf& b, uint32_t slot, bool& aborted, int& nrays, uint32_t* nodes,
                      uint32_t* tris) {
  const float4 o4 = b.st[slot].org, d4 = b.st[slot].dir;
  const DevScene& s = sc.jobs[__float_as_uint(d4.w)].s;
  const float4 w4 = b.st[slot].weight, L = b.st[slot].rad;
  const int flags = __float_as_int(L.w);
  v3 org = mk(o4);
  v3 add = mk(0.f);
  if (flags & 1) {
    float4 d = b.sh[slot].sh_dir;
    Hit h;
    bool ab = false;
    // isOccluded normalises the light direction (bvh.glsl:225-229)
    if (!trace_path_ray<true, kCount, kTrav>(s, org, normalize_rn(mk(d)), d.w, h, ab, nodes, tris))
      add = mk(b.sh[slot].sh_c);
    aborted |= ab;
    ++nrays;
  }
  if (flags & 2) {
    float4 d = b.sh[slot].pl_dir;
    Hit h;
    bool ab = false;
    if (!trace_path_ray<true, kCount, kTrav>(s, org, normalize_rn(mk(d)), d.w, h, ab, nodes, tris))
      add = add + mk(b.sh[slot].pl_c);
    aborted |= ab;
    ++nrays;
  }
  // the whole sector (weight, radiance) written back
  b.st[slot].weight = w4;
  b.st[slot].rad = make_float4(L.x + add.x, L.y + add.y, L.z + add.z, L.w);
}

template <bool kCount, int kTrav>
__global__ void __launch_bounds__(256, 4) k_connect(Sched sc, PathBuf b, int cur) {
  const uint32_t count = b.counts[kCntShadow0 + cur];
  const uint32_t* qs = b.qs[cur];
  for (uint32_t base = blockIdx.x * blockDim.x; base < count; base += gridDim.x * blockDim.x) {
    uint32_t i = base + threadIdx.x;
    bool aborted = false;
    int nrays = 0;
    uint32_t nodes = 0, tris = 0;
    if (i < count) connect_slot<kCount, kTrav>(sc, b, qs[i], aborted, nrays, &nodes, &tris);
    unsigned m1 = __ballot_sync(0xffffffffu, nrays >= 1), m2 = __ballot_sync(0xffffffffu, nrays >= 2);
    if ((threadIdx.x & 31) == 0 && (m1 | m2)) atomicAdd(b.stats + 1, (unsigned long long)(__popc(m1) + __popc(m2)));
    count_warp(b.stats + 2, aborted);
    if (kCount) {
      add_warp(b.stats + 5, nodes);
      add_warp(b.stats + 6, tris);
    }
  }
}

// the shadow rays of qs[cur] by persistent warps (see next_warp_batch), 4-wide or 8-wide traversal
template <int kTrav>
__global__ void __launch_bounds__(128, 8) k_connect_dyn(Sched sc, PathBuf b, int cur) {
  const uint32_t count = b.counts[kCntShadow0 + cur];
  const uint32_t* qs = b.qs[cur];
  uint32_t rays = 0, aborted_n = 0;
  uint32_t i;
  bool first = true;
  while (next_warp_batch(b.counts + kCntFetchShadow, count, i, first)) {
    if (i < count) {
      bool aborted = false;
      int nrays = 0;
      connect_slot<false, kTrav>(sc, b, qs[i], aborted, nrays, nullptr, nullptr);
      rays += uint32_t(nrays);
      aborted_n += aborted ? 1u : 0u;
    }
  }
  add_warp(b.stats + 1, rays);
  add_warp(b.stats + 2, aborted_n);
}

// ---- shade ------------------------------------------------------------------------------------
DEV float mis_balance(float a, float c) { return a / (a + c); }

DEV float4 clamp_result(const WaveParams& p, v3 L) {
  if (p.clamp_threshold > 0.f)
    return make_float4(clampf(L.x, 0.f, p.clamp_threshold), clampf(L.y, 0.f, p.clamp_threshold),
                       clampf(L.z, 0.f, p.clamp_threshold), 1.f);
  return f4(L, 1.f);
}

// A path whose ray left the scene: background for camera rays
// (misptdl.glsl:41-46), MIS-weighted environment otherwise (misptdl.glsl:84-88).
DEV void shade_miss_path(const Sched& sc, const PathBuf& b, uint32_t slot) {
  const PathState ps = b.st[slot];
  const Job& J = sc.jobs[path_job(ps)];
  // read in place (the job table does not change during an iteration): fewer
  // registers held across the outlined material calls than a local copy
  const WaveParams& p = J.p;
  v3 dir = mk(ps.dir);
  v3 w = mk(ps.weight);
  float last_pdf = ps.weight.w;
  v3 L = mk(ps.rad);
  if (path_bounce(ps) == 0) {
    if (p.bg_from_ibl > 0) {
      v3 env = p.has_ibl ? ibl_eval(J.e, p.ibl_rot, dir) : mk(0.f);
      finish_path(J, ps.pixel, f4(env * w, 1.f));
    } else {
      finish_path(J, ps.pixel,
                  make_float4(powf(p.bg_color.x, 2.2f), powf(p.bg_color.y, 2.2f), powf(p.bg_color.z, 2.2f),
                              p.bg_color.w));
    }
    return;
  }
  if (p.has_ibl) {
    float ipdf = ibl_pdf(J.e, p.ibl_rot, dir);
    float mis = mis_balance(last_pdf, ipdf);
    L = L + ibl_eval(J.e, p.ibl_rot, dir) * w * mis * float(p.use_ibl);
  }
  finish_path(J, ps.pixel, clamp_result(p, L));
}


// Surface hit.  Returns true if the path continues with an extension ray and
// sets `shadow` when NEE shadow rays were emitted; otherwise the path's sample
// has been accumulated.
template <bool kTextured>
DEV bool shade_path(const Sched& sc, const PathBuf& b, uint32_t slot, bool& shadow) {
  shadow = false;
  PathState& ps = b.st[slot];
  const float4 o4 = ps.org, d4 = ps.dir, w4 = ps.weight, l4 = ps.rad;
  const Job& J = sc.jobs[__float_as_uint(d4.w)];
  // read in place (the job table does not change during an iteration): fewer
  // registers held across the outlined material calls than a local copy
  const WaveParams& p = J.p;
  float4 hit = b.hits[slot].h;
  int tri = __float_as_int(hit.w);
  v3 dir = mk(d4);
  v3 w = mk(w4);
  v3 L = mk(l4);
  const int bounce = __float_as_int(o4.w);
  if (!(bounce < p.max_bounces)) {  // loop condition (misptdl.glsl:54)
    finish_path(J, ps.pixel, clamp_result(p, L));
    return false;
  }
  Rng rng;
  {
    const uint4 aux = *reinterpret_cast<const uint4*>(&ps.rng);  // rng (2 words), pixel, frame
    rng.state = uint64_t(aux.x) | (uint64_t(aux.y) << 32);
    rng.inc = p.rng_pcg ? pcg_inc(uint64_t(aux.w) * uint64_t(p.npix) + aux.z) : 0;
  }
  // Russian roulette (renderer.frag:119-123): weight boost every bounce
  w = w * p.rr_factor;
  if (bounce > p.rr_start && rng.next() <= p.rr_prob) {
    finish_path(J, ps.pixel, clamp_result(p, L));
    return false;
  }
  v3 org = mk(o4);
  v3 wi = -dir;
  v3 pos = org + dir * hit.x;
  Surface S = make_surface_t<kTextured>(J.s, tri, hit.y, hit.z, pos, wi, p.lean != 0);
  if (S.backside && !S.thin_walled) {  // Beer-Lambert absorption (misptdl.glsl:60-63)
    v3 sigma = -vlog(S.att_color) / S.att_dist;
    w = w * vexp(-sigma * hit.x);
  }
  L = L + S.emissive * 1.0f * w;

  // sample_bsdf_bounce (renderer.frag:94-116)
  v3 wo;
  v3 bw = mk(1.f);
  float pdf = 1.f;
  if (rng.next() > S.cutout) {
    wo = -wi;
  } else {
    float u0 = rng.next(), u1 = rng.next(), u2 = rng.next();
    float comp = rng.next();
    BsdfSample bs = bsdf_sample(S.c, S.n, wi, comp, u0, u1, u2);
    wo = bs.dir;
    pdf = bs.pdf;
    bw = bs.weight;
    if (pdf < kEpsPdf) {  // absorbed: returns L without the clamp
      finish_path(J, ps.pixel, f4(L, 1.f));
      return false;
    }
  }
  pos = pos + (dot(S.ng, wo) < 0.f ? -S.ng : S.ng) * p.ray_eps;

  // next-event estimation (misptdl.glsl:2-32, lighting.glsl:2-22)
  float r0 = rng.next(), r1 = rng.next();
  v3 n_nee = S.backside ? -S.n : S.n;
  int flags = 0;
  if (p.use_ibl > 0 && p.has_ibl) {
    float ipdf;
    v3 ld = ibl_sample(J.e, p.ibl_rot, p.env_mode, r0, r1, ipdf);
    float cosnl = sat(dot(ld, n_nee));
    if (cosnl > kEpsCos && ipdf > kEpsPdf) {
      float bpdf;
      v3 f = bsdf_eval_pdf(S.c, S.n, wi, ld, bpdf) / fmaxf(fabsf(dot(S.n, ld)), kEps);
      v3 c = ibl_eval(J.e, p.ibl_rot, ld) * f * cosnl / ipdf;
      if (bpdf > kEpsPdf) c = c * mis_balance(ipdf, bpdf);
      b.sh[slot].sh_dir = f4(ld, kTfarMax);  // one whole sector
      b.sh[slot].sh_c = f4(c * w, 0.f);
      flags |= 1;
    }
  }
  if (p.pl_pos.w > 0.5f) {
    v3 lp = mk(p.pl_pos.x, p.pl_pos.y, p.pl_pos.z);
    v3 ld = lp - pos;
    float dist2 = dot(ld, ld);
    v3 ldn = normalize(ld);
    float cosnl = sat(dot(ldn, n_nee));
    if (cosnl > kEpsCos) {
      v3 f = bsdf_eval(S.c, S.n, wi, ldn) / fmaxf(fabsf(dot(S.n, ldn)), kEps);
      v3 c = f * (mk(p.pl_emis.x, p.pl_emis.y, p.pl_emis.z) / dist2) * cosnl;
      b.sh[slot].pl_dir = f4(ldn, sqrtf(dist2));  // one whole sector
      b.sh[slot].pl_c = f4(c * w, 0.f);
      flags |= 2;
    }
  }
  shadow = flags != 0;

  w = w * bw;
  // the whole record: three sectors (job, pixel and frame read back, not kept live)
  const float job_bits = ps.dir.w;
  const uint2 pf = *reinterpret_cast<const uint2*>(&ps.pixel);
  ps.org = f4(pos, __int_as_float(bounce + 1));
  ps.dir = f4(wo, job_bits);
  ps.weight = f4(w, pdf);
  ps.rad = f4(L, __int_as_float(flags));
  *reinterpret_cast<uint4*>(&ps.rng) = make_uint4(uint32_t(rng.state), uint32_t(rng.state >> 32), pf.x, pf.y);
  *reinterpret_cast<uint4*>(ps.pad) = make_uint4(0u, 0u, 0u, 0u);
  return true;
}

// kTextured = false: no active job's scene has textures (their texture ids are all unset)
template <bool kTextured>
// 5 blocks of 128 threads per SM (96 registers, some spilled): of 3..8 blocks
// per SM the fastest frames (3: 168 registers, no spills; 4 and 6..8 slower)
__global__ void __launch_bounds__(128, 5) k_shade(Sched sc, PathBuf b, int next) {
  // the class queues, then the miss queue, read as one sequence: the misses
  // (environment, background) are shaded by the same persistent warps after
  // the surface hits, with no launch of their own
  __shared__ uint32_t start[kNumClasses + 2];
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (int k = 0; k < kNumClasses; ++k) {
      start[k] = acc;
      acc += b.counts[kCntHit0 + k];
    }
    start[kNumClasses] = acc;
    start[kNumClasses + 1] = acc + b.counts[kCntMiss];
  }
  __syncthreads();
  const uint32_t hits = start[kNumClasses];
  const uint32_t count = start[kNumClasses + 1];
  uint32_t* qn = b.q[next];
  uint32_t* cn = b.counts + next;
  __shared__ uint32_t freed[128 / 32][kFreeBuf];
  WarpFree wf;
  wf.init(freed[threadIdx.x >> 5]);
  uint32_t i;
  bool first = true;
  while (next_warp_batch(b.counts + kCntFetchShade, count, i, first)) {
    bool cont = false, shadow = false;
    uint32_t slot = 0, job = 0;
    if (i < hits) {
      int k = 0;
#pragma unroll
      for (int jk = 1; jk < kNumClasses; ++jk) k += i >= start[jk] ? 1 : 0;
      slot = b.qh[size_t(k) * b.capacity + (i - start[k])];
      job = __float_as_uint(b.st[slot].dir.w);
      cont = shade_path<kTextured>(sc, b, slot, shadow);
    } else if (i < count) {
      slot = b.qm[i - hits];
      job = __float_as_uint(b.st[slot].dir.w);
      shade_miss_path(sc, b, slot);
    }
    enqueue(qn, cn, cont, slot);
    enqueue(b.qs[next], b.counts + kCntShadow0 + next, shadow, slot);
    wf.add(sc, b, i < count && !cont, slot, job);
  }
  wf.flush(sc, b);
}

// ---- drain: the last paths of a render call, each run to completion ---------------------
// Once every work item has started and few paths are left, the remaining
// bounces are latency-bound: each wavefront iteration costs about the latency
// of its slowest ray whatever the number of paths.  This kernel takes the
// paths queued for the next extend (their pending shadow rays were connected
// by the k_connect launched before it) and runs every path through extend ->
// shade_miss / shade -> connect until it ends: the same device functions in
// the same order per path, so each path's result is unchanged.
template <bool kTextured>
__global__ void __launch_bounds__(128) k_drain(Sched sc, PathBuf b, int cur) {
  // two lanes per path: the even lane runs the path (extension ray, shading),
  // the odd lane the NEE shadow rays of the path's last vertex.  The shadow
  // rays of vertex k and the extension ray of vertex k + 1 start at the same
  // point and are independent, so the two lanes trace them side by side
  // (one traversal routine, any-hit chosen at run time); the shadow
  // contribution reaches the path radiance before the next shading reads it,
  // the order of the one-lane loop, so each path's result is unchanged.
  const uint32_t count = b.counts[cur];
  const uint32_t* q = b.q[cur];
  const int lane = threadIdx.x & 31;
  const bool helper = (lane & 1) != 0;
  const unsigned pair = 3u << (lane & ~1);
  const uint32_t per_round = (gridDim.x * blockDim.x) >> 1;
  for (uint32_t base = (blockIdx.x * blockDim.x) >> 1; base < count; base += per_round) {
    const uint32_t i = base + (threadIdx.x >> 1);
    uint32_t slot = 0, job = 0, closest = 0, shadow_rays = 0;
    bool aborted = false;
    if (i < count) {
      slot = q[i];
      job = __float_as_uint(b.st[slot].dir.w);
      bool pending = false;  // shadow rays of the last vertex not yet traced (pair-uniform)
      for (int guard = 0; guard < 4 * kMaxSteps; ++guard) {
        const DevScene& s = sc.jobs[job].s;
        Hit h;
        h.tri = -1;
        h.t = h.u = h.v = 0.f;
        if (s.wide) {
          // extension ray (even lane) and IBL shadow ray (odd lane) in one pass
          const float4 o = b.st[slot].org;
          float4 d = b.st[slot].dir;
          float tfar = kTfarMax;
          bool trace = !helper;
          int flags = 0;
          if (helper && pending) {
            flags = __float_as_int(b.st[slot].rad.w);
            if (flags & 1) {
              const float4 sd = b.sh[slot].sh_dir;
              d = make_float4(sd.x, sd.y, sd.z, 0.f);
              tfar = sd.w;
              trace = true;
            }
          }
          bool ab = false, occluded = false;
          if (trace) {
            // isOccluded normalises the light direction (bvh.glsl:225-229)
            const v3 dir = helper ? normalize_rn(mk(d)) : mk(d);
            occluded = traverse_wide_rt(s, mk(o), dir, tfar, helper, h, ab);
            aborted |= ab;
          }
          if (helper && pending) {
            v3 add = mk(0.f);
            if (flags & 1) {
              if (!occluded) add = mk(b.sh[slot].sh_c);
              ++shadow_rays;
            }
            if (flags & 2) {  // the point-light ray, after
              const float4 pd = b.sh[slot].pl_dir;
              Hit hp;
              bool abp = false;
              if (!traverse_wide_rt(s, mk(o), normalize_rn(mk(pd)), pd.w, true, hp, abp))
                add = add + mk(b.sh[slot].pl_c);
              aborted |= abp;
              ++shadow_rays;
            }
            const float4 w4 = b.st[slot].weight, L = b.st[slot].rad;
            b.st[slot].weight = w4;
            b.st[slot].rad = make_float4(L.x + add.x, L.y + add.y, L.z + add.z, L.w);
          }
        } else {
          // the reference's binary traversal: shadow rays, then the extension ray
          if (helper && pending) {
            int nrays = 0;
            connect_slot<false, kTravPerPath>(sc, b, slot, aborted, nrays, nullptr, nullptr);
            shadow_rays += uint32_t(nrays);
          }
          __syncwarp(pair);
          if (!helper) {
            const float4 o = b.st[slot].org, d = b.st[slot].dir;
            bool ab = false;
            trace_path_ray<false, false, kTravPerPath>(s, mk(o), mk(d), kTfarMax, h, ab, nullptr, nullptr);
            aborted |= ab;
          }
        }
        __syncwarp(pair);  // the shadow contribution is in the record before the shading reads it
        bool cont = false, shadow = false;
        if (!helper) {
          ++closest;
          b.hits[slot] = PathHit{make_float4(h.t, h.u, h.v, __int_as_float(h.tri)), make_float4(0.f, 0.f, 0.f, 0.f)};
          if (h.tri < 0) shade_miss_path(sc, b, slot);
          else cont = shade_path<kTextured>(sc, b, slot, shadow);
        }
        cont = __shfl_sync(pair, cont, lane & ~1);
        pending = __shfl_sync(pair, shadow, lane & ~1);
        __syncwarp(pair);  // the shading's records are written before the helper reads them
        if (!cont) break;  // a path that ends emits no shadow ray
      }
    }
    // one free per path (even lanes)
    free_slots(sc, b, i < count && !helper, slot, job);
    add_warp(b.stats + 0, closest);
    add_warp(b.stats + 1, shadow_rays);
    count_warp(b.stats + 2, aborted);
  }
}

// Streaming (evict-first) loads and stores: the 48 bytes per pixel it moves
// would otherwise push the scene's BVH out of L2 before the next frame.
__global__ void k_mean(const double4* accum, double inv, float4* out, int npix) {
  const double2* a2 = reinterpret_cast<const double2*>(accum);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
    const double2 lo = __ldcs(a2 + 2 * size_t(i)), hi = __ldcs(a2 + 2 * size_t(i) + 1);
    __stcs(out + i, make_float4(float(lo.x * inv), float(lo.y * inv), float(hi.x * inv), float(hi.y * inv)));
  }
}

// ---- scene preparation: leaf-ordered triangle records ------------------------------------
__global__ void k_gather_tris(const float4* verts, const uint32_t* indices, const int32_t* remap, uint32_t nslots,
                              uint32_t ntris, float4* tris) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nslots; i += gridDim.x * blockDim.x) {
    int32_t t = remap[i];
    if (t < 0 || uint32_t(t) >= ntris) {
      tris[3 * size_t(i)] = make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
      tris[3 * size_t(i) + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
      tris[3 * size_t(i) + 2] = make_float4(0.f, 0.f, 0.f, 0.f);
      continue;
    }
    float4 a = verts[5 * size_t(indices[3 * size_t(t)])];
    float4 b = verts[5 * size_t(indices[3 * size_t(t) + 1])];
    float4 c = verts[5 * size_t(indices[3 * size_t(t) + 2])];
    tris[3 * size_t(i)] = make_float4(a.x, a.y, a.z, __int_as_float(t));
    tris[3 * size_t(i) + 1] = make_float4(__fsub_rn(b.x, a.x), __fsub_rn(b.y, a.y), __fsub_rn(b.z, a.z), 0.f);
    tris[3 * size_t(i) + 2] = make_float4(__fsub_rn(c.x, a.x), __fsub_rn(c.y, a.y), __fsub_rn(c.z, a.z), 0.f);
  }
}

// ---- kernel-level queries ----------------------------------------------------------------
__global__ void __launch_bounds__(128) k_trace_rays(DevScene s, const float4* rays, uint32_t n, int any, int32_t* tri,
                                                    float* t, float2* uv, int32_t* occ) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 a = rays[2 * i], c = rays[2 * i + 1];
    v3 org = mk(a.x, a.y, a.z), dir = mk(a.w, c.x, c.y);
    Hit h;
    bool ab = false;
    if (any) {
      // isOccluded (bvh.glsl:225-229) normalises the direction first
      const v3 nd = normalize_rn(dir);
      occ[i] = (s.wide ? traverse_wide<true>(s, org, nd, c.z, h, ab) : traverse<true>(s, org, nd, c.z, h, ab)) ? 1 : 0;
    } else {
      if (s.wide) traverse_wide<false>(s, org, dir, c.z, h, ab);
      else traverse<false>(s, org, dir, c.z, h, ab);
      tri[i] = h.tri;
      t[i] = h.t;
      uv[i] = make_float2(h.u, h.v);
    }
  }
}

__global__ void k_bsdf_query(DevScene s, uint32_t n, const float* hit20, const float* wo3, const float* rnd4, int lean,
                             float* eval4, float* sample10, int32_t* flags) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float* h = hit20 + 20 * size_t(i);
    // Build the surface the way fillRenderState + configure_gltf_material do,
    // from explicit shading inputs instead of a triangle fetch.
    v3 n0 = mk(h[0], h[1], h[2]), ng = mk(h[3], h[4], h[5]);
    float4 tangent = make_float4(h[6], h[7], h[8], h[9]);
    v3 wi = mk(h[10], h[11], h[12]);
    float4 vcol = make_float4(h[15], h[16], h[17], h[18]);
    const int mat = int(uint32_t(h[19]));
    Surface S = s.num_texinfo > 0 ? configure_gltf<true>(s, mat, n0, ng, tangent, wi, h[13], h[14], vcol, lean != 0)
                                  : configure_gltf<false>(s, mat, n0, ng, tangent, wi, h[13], h[14], vcol, lean != 0);
    const Closure& c = S.c;
    n0 = S.n;
    const bool back = S.backside;
    v3 wo = mk(wo3[3 * i], wo3[3 * i + 1], wo3[3 * i + 2]);
    v3 ev = bsdf_eval(c, n0, wi, wo);
    float pd = bsdf_pdf(c, n0, wi, wo);
    eval4[4 * i] = ev.x; eval4[4 * i + 1] = ev.y; eval4[4 * i + 2] = ev.z; eval4[4 * i + 3] = pd;
    const float* r = rnd4 + 4 * size_t(i);
    BsdfSample bs = bsdf_sample(c, n0, wi, r[0], r[1], r[2], r[3]);
    float* o = sample10 + 10 * size_t(i);
    o[0] = bs.dir.x; o[1] = bs.dir.y; o[2] = bs.dir.z; o[3] = bs.pdf;
    o[4] = bs.weight.x; o[5] = bs.weight.y; o[6] = bs.weight.z;
    o[7] = bs.specular; o[8] = bs.crossed; o[9] = bs.next_ior;
    flags[i] = back ? 1 : 0;
  }
}

__global__ void k_ibl_query(DevIbl e, float rot, int mode, uint32_t n, const float* r2, const float* dirs, float* sdp4,
                            float* pdf, float* rgb) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float sp;
    v3 d = ibl_sample(e, rot, mode, r2[2 * i], r2[2 * i + 1], sp);
    sdp4[4 * i] = d.x; sdp4[4 * i + 1] = d.y; sdp4[4 * i + 2] = d.z; sdp4[4 * i + 3] = sp;
    v3 q = mk(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]);
    pdf[i] = ibl_pdf(e, rot, q);
    v3 c = ibl_eval(e, rot, q);
    rgb[3 * i] = c.x; rgb[3 * i + 1] = c.y; rgb[3 * i + 2] = c.z;
  }
}

__global__ void k_camera_rays(Camera c, uint32_t n, const int32_t* xy, const float* r2, float* rays6) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    v3 o, d;
    camera_ray(c, xy[2 * i], xy[2 * i + 1], r2[2 * i], r2[2 * i + 1], o, d);
    float* r = rays6 + 6 * size_t(i);
    r[0] = o.x; r[1] = o.y; r[2] = o.z; r[3] = d.x; r[4] = d.y; r[5] = d.z;
  }
}

// ---- launchers --------------------------------------------------------------------------------
static int grid_for(uint64_t n, int threads, int cap) {
  uint64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  return int(b < uint64_t(cap) ? b : uint64_t(cap));
}

LaunchLimits launch_limits() {
  LaunchLimits l{148, 8, 8, {5, 5}};
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&l.sms, cudaDevAttrMultiProcessorCount, dev);
  auto resident = [&](const void* fn, int threads, int fallback) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, 0) != cudaSuccess || n <= 0) {
      cudaGetLastError();
      n = fallback;
    }
    return n;
  };
  l.trace_per_sm = resident(reinterpret_cast<const void*>(k_extend_dyn<kTravWide>), 128, 8);
  l.connect_per_sm = resident(reinterpret_cast<const void*>(k_connect_dyn<kTravWide>), 128, 8);
  l.shade_per_sm[0] = resident(reinterpret_cast<const void*>(k_shade<false>), 128, 5);
  l.shade_per_sm[1] = resident(reinterpret_cast<const void*>(k_shade<true>), 128, 5);
  return l;
}

void init_launch_sizes(LaunchCfg& lc) {
  const LaunchLimits l = launch_limits();
  lc.dyn_blocks = l.trace_per_sm * l.sms;
  lc.connect_dyn_blocks = l.connect_per_sm * l.sms;
  lc.shade_dyn_blocks[0] = l.shade_per_sm[0] * l.sms;
  lc.shade_dyn_blocks[1] = l.shade_per_sm[1] * l.sms;
}

void launch_init_pool(const PathBuf& b, cudaStream_t st) {
  k_init_pool<<<grid_for(b.capacity, 256, 148 * 8), 256, 0, st>>>(b);
}
void launch_free_list(const Sched& sc, const PathBuf& b, cudaStream_t st) {
  const uint32_t words = (b.capacity + 31u) / 32u;
  const int blocks = int((words + kFreeMapBlock - 1) / kFreeMapBlock);
  k_free_count<<<blocks, kFreeMapBlock, 0, st>>>(sc, b);
  k_free_emit<<<blocks, kFreeMapBlock, 0, st>>>(b);
}
void launch_regen(const Sched& sc, const PathBuf& b, int next, cudaStream_t st) {
  k_regen<<<grid_for(b.capacity, kMaxJobs, 148 * 8), kMaxJobs, 0, st>>>(sc, b, next);
}
void launch_commit(const Sched& sc, const PathBuf& b, int cur, cudaStream_t st, bool regen_ran) {
  k_commit<<<1, kMaxJobs, 0, st>>>(sc, b, cur, regen_ran ? 1 : 0, LoopHandles{}, nullptr);
}
void launch_commit_loop(const Sched& sc, const PathBuf& b, int cur, const LoopHandles& h, LoopCtl* ctl,
                        cudaStream_t st) {
  k_commit<<<1, kMaxJobs, 0, st>>>(sc, b, cur, 1, h, ctl);
}
void launch_set_loop(LoopCtl* ctl, unsigned long long iterations, unsigned long long drain_below, int mode,
                     int wait_job, cudaStream_t st) {
  k_set_loop<<<1, 32, 0, st>>>(ctl, iterations, drain_below, mode, wait_job);
}
void launch_extend(const Sched& sc, const PathBuf& b, int cur, bool count, const LaunchCfg& lc, cudaStream_t st) {
  const dim3 g(lc.trace_blocks), t(lc.trace_threads);
  if (count) k_extend<true, kTravReference><<<g, t, 0, st>>>(sc, b, cur);
  else if (lc.traversal == kTravWide) k_extend_dyn<kTravWide><<<lc.dyn_blocks, 128, 0, st>>>(sc, b, cur);
  else if (lc.traversal == kTravWide8) k_extend_dyn<kTravWide8><<<lc.dyn_blocks, 128, 0, st>>>(sc, b, cur);
  else if (lc.traversal == kTravReference) k_extend<false, kTravReference><<<g, t, 0, st>>>(sc, b, cur);
  else k_extend<false, kTravPerPath><<<g, t, 0, st>>>(sc, b, cur);
}
void launch_connect(const Sched& sc, const PathBuf& b, int cur, bool count, const LaunchCfg& lc, cudaStream_t st) {
  const dim3 g(lc.trace_blocks), t(lc.trace_threads);
  if (count) k_connect<true, kTravReference><<<g, t, 0, st>>>(sc, b, cur);
  else if (lc.traversal == kTravWide) k_connect_dyn<kTravWide><<<lc.connect_dyn_blocks, 128, 0, st>>>(sc, b, cur);
  else if (lc.traversal == kTravWide8)
    k_connect_dyn<kTravWide8><<<lc.connect_dyn_blocks, 128, 0, st>>>(sc, b, cur);
  else if (lc.traversal == kTravReference) k_connect<false, kTravReference><<<g, t, 0, st>>>(sc, b, cur);
  else k_connect<false, kTravPerPath><<<g, t, 0, st>>>(sc, b, cur);
}
void launch_shade(const Sched& sc, const PathBuf& b, int next, const LaunchCfg& lc, cudaStream_t st) {
  if (lc.textured) k_shade<true><<<lc.shade_dyn_blocks[1], 128, 0, st>>>(sc, b, next);
  else k_shade<false><<<lc.shade_dyn_blocks[0], 128, 0, st>>>(sc, b, next);
}
void launch_drain(const Sched& sc, const PathBuf& b, int cur, const LaunchCfg& lc, cudaStream_t st) {
  if (lc.textured) k_drain<true><<<148 * 4, 128, 0, st>>>(sc, b, cur);
  else k_drain<false><<<148 * 4, 128, 0, st>>>(sc, b, cur);
}
void launch_mean(const double4* accum, double inv_count, float4* out, int npix, cudaStream_t st) {
  k_mean<<<grid_for(npix, 256, 148 * 8), 256, 0, st>>>(accum, inv_count, out, npix);
}
void launch_gather_tris(const float4* verts, const uint32_t* indices, const int32_t* remap, uint32_t nslots,
                        uint32_t ntris, float4* tris, cudaStream_t st) {
  k_gather_tris<<<grid_for(nslots, 256, 148 * 16), 256, 0, st>>>(verts, indices, remap, nslots, ntris, tris);
}
void launch_trace_rays(const DevScene& s, const float4* rays, uint32_t n, int any, int32_t* tri, float* t, float2* uv,
                       int32_t* occ, cudaStream_t st) {
  k_trace_rays<<<grid_for(n, 128, 148 * 16), 128, 0, st>>>(s, rays, n, any, tri, t, uv, occ);
}
void launch_bsdf_query(const DevScene& s, uint32_t n, const float* hit20, const float* wo3, const float* rnd4,
                       int lean, float* eval4, float* sample10, int32_t* flags, cudaStream_t st) {
  k_bsdf_query<<<grid_for(n, 128, 148 * 16), 128, 0, st>>>(s, n, hit20, wo3, rnd4, lean, eval4, sample10, flags);
}
void launch_ibl_query(const DevIbl& e, float rot, int mode, uint32_t n, const float* r2, const float* dirs,
                      float* sdp4, float* pdf, float* rgb, cudaStream_t st) {
  k_ibl_query<<<grid_for(n, 128, 148 * 16), 128, 0, st>>>(e, rot, mode, n, r2, dirs, sdp4, pdf, rgb);
}
void launch_camera_rays(const Camera& c, uint32_t n, const int32_t* xy, const float* r2, float* rays6,
                        cudaStream_t st) {
  k_camera_rays<<<grid_for(n, 128, 148 * 16), 128, 0, st>>>(c, n, xy, r2, rays6);
}

}  // namespace dspbr
