// C ABI of libdspbr_cuda.so (include/dspbr.h): contexts, scenes, IBLs, the
// progressive render loop and the kernel-level query entry points.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "bvh_gpu.h"
#include "bvh_wide.h"
#include "display.h"
#include "dspbr.h"
#include "engine.h"
#include "host.h"
#include "kernels.h"
#include "objects.h"

using namespace dspbr;

namespace dspbr {
WaveParams make_job_params(const dspbr_params& q, const float matrix[16], float fov, float near_plane, int width,
                           int height, bool has_ibl, uint32_t frame_base) {
  WaveParams p{};
  double film = std::tan(double(fov) * 0.5 * M_PI / 180.0) * double(near_plane);
  for (int col = 0; col < 3; ++col)
    for (int r = 0; r < 3; ++r) p.cam.m[col * 3 + r] = matrix[col * 4 + r];
  p.cam.pos[0] = matrix[12]; p.cam.pos[1] = matrix[13]; p.cam.pos[2] = matrix[14];
  p.cam.film_height = float(film);
  p.cam.focal = near_plane;
  p.cam.inv_res[0] = float(1.0 / width);
  p.cam.inv_res[1] = float(1.0 / height);
  p.cam.width = width;
  p.cam.height = height;
  p.npix = width * height;
  p.frame_base = frame_base;
  p.max_bounces = q.max_bounces;
  p.rng_pcg = q.rng == DSPBR_RNG_PCG;
  p.seed = q.seed;
  p.use_ibl = q.use_ibl ? 1 : 0;
  p.bg_from_ibl = q.background_from_ibl ? 1 : 0;
  p.env_mode = q.env_sampling == DSPBR_ENV_CDF ? 1 : 0;
  p.lean = q.profile == DSPBR_PROFILE_LEAN;
  p.has_ibl = has_ibl;
  p.ibl_rot = float(double(q.ibl_rotation_deg) / 180.0 * M_PI);
  p.bg_color = make_float4(q.background_color[0], q.background_color[1], q.background_color[2], q.background_color[3]);
  p.ray_eps = q.ray_eps;
  p.clamp_threshold = q.clamp_threshold;
  p.rr_prob = q.rr_termination_prob;
  p.rr_factor = 1.0f / (1.0f - q.rr_termination_prob);
  p.rr_start = q.rr_start_depth;
  p.pl_pos = make_float4(q.point_light_position[0], q.point_light_position[1], q.point_light_position[2],
                         q.point_light_position[3]);
  p.pl_emis = make_float4(q.point_light_emission[0], q.point_light_emission[1], q.point_light_emission[2],
                          q.point_light_emission[3]);
  return p;
}

}  // namespace dspbr


// Joins the worker of a render_async call, so that the caller's next stream
// operation is ordered after all of that render's launches.  Returns the
// worker's status.
// A copy of read_accum_async may still be reading the mean buffer: the
// stream's next writes to it wait for that copy.
static cudaError_t after_pending_copy(dspbr_ctx* c) {
  return c->copy_pending ? cudaStreamWaitEvent(c->stream, c->ev_copied, 0) : cudaSuccess;
}

// the context's stream waits for the copy stream's pending mean (the sums it
// reads may be written next), not for the device-to-host copy behind it
static cudaError_t after_pending_mean(dspbr_ctx* c) {
  if (!c->mean_pending) return cudaSuccess;
  c->mean_pending = false;
  return cudaStreamWaitEvent(c->stream, c->ev_meaned, 0);
}

// Joins the render_async worker; returns its status.
static int settle_worker(dspbr_ctx* c) {
  if (c->worker.joinable()) c->worker.join();
  int rc = c->worker_rc;
  c->worker_rc = 0;
  return rc;
}

// Mean and device-to-host copy of an epoch's sums, after `after` (recorded
// on the context's stream) when given: the mean on the mean stream into the
// next read buffer, the copy on the copy stream.
static int issue_read(dspbr_ctx* c, const double4* accum, uint64_t count, float* dst, cudaEvent_t after) {
  Status s = c->st();
  const size_t npix = size_t(c->width) * c->height;
  const double inv = count ? 1.0 / double(count) : 0.0;
  const int r = c->read_next;
  c->read_next = (r + 1) % dspbr_ctx::kReadRing;
  if (c->read_mean[r].n < npix) {
    // the buffer is replaced: its last copy has to be done first
    if (c->read_used[r]) TRY_CUDA(s, cudaEventSynchronize(c->ev_read_copied[r]), "read accumulation");
    TRY_CUDA(s, c->read_mean[r].alloc(npix), "alloc readback");
  }
  if (!after) {
    TRY_CUDA(s, cudaEventRecord(c->ev_mean, c->stream), "event");
    after = c->ev_mean;
  }
  TRY_CUDA(s, cudaStreamWaitEvent(c->mean_stream, after, 0), "read accumulation");
  if (c->read_used[r]) TRY_CUDA(s, cudaStreamWaitEvent(c->mean_stream, c->ev_read_copied[r], 0), "read accumulation");
  launch_mean(accum, inv, c->read_mean[r].p, int(npix), c->mean_stream);
  TRY_CUDA(s, cudaGetLastError(), "read accumulation");
  TRY_CUDA(s, cudaEventRecord(c->ev_meaned, c->mean_stream), "event");
  c->mean_pending = true;
  TRY_CUDA(s, cudaStreamWaitEvent(c->copy_stream, c->ev_meaned, 0), "read accumulation");
  TRY_CUDA(s, cudaMemcpyAsync(dst, c->read_mean[r].p, npix * 16, cudaMemcpyDeviceToHost, c->copy_stream),
           "read accumulation");
  TRY_CUDA(s, cudaEventRecord(c->ev_read_copied[r], c->copy_stream), "event");
  c->read_used[r] = true;
  TRY_CUDA(s, cudaEventRecord(c->ev_copied, c->copy_stream), "event");
  c->copy_pending = true;
  return DSPBR_OK;
}

// A sum buffer of at least npix pixels for a new epoch: a finished epoch's,
// or a new allocation.  The caller orders its first write after the pending
// copy (after_pending_copy): a read of the epoch that left it may still run.
static cudaError_t take_spare(dspbr_ctx* c, size_t npix, std::unique_ptr<DevBuf<double4>>& out) {
  if (!c->spare.empty()) {
    out = std::move(c->spare.back());
    c->spare.pop_back();
  } else {
    out.reset(new DevBuf<double4>());
  }
  return out->n < npix ? out->alloc(npix) : cudaSuccess;
}

// a job slot no epoch in flight uses
static int free_slot(const dspbr_ctx* c) {
  for (int k = 0;; ++k) {
    bool used = k == c->slot;
    for (const auto& o : c->older) used = used || o.slot == k;
    if (!used) return k;
  }
}

// A deferred read of a finished epoch, enqueued after the next loop launch.
struct LateRead {
  const double4* sums;
  uint64_t samples;
  float* dst;
};

// The older epochs that have finished leave the flight list, oldest first:
// their deferred reads are enqueued (after `after` when given; with `late`,
// collected there for the caller to enqueue) and their sum buffers become
// spares (taken again only by a reset, after the caller's reads).
static int retire_finished(dspbr_ctx* c, cudaEvent_t after, std::vector<LateRead>* late = nullptr) {
  Engine& E = *c->eng;
  for (size_t i = 0; i < c->older.size();) {
    auto& o = c->older[i];
    if (!E.job_done(o.slot)) {
      ++i;
      continue;
    }
    if (o.deferred && late) {
      late->push_back(LateRead{o.sums->p, o.samples, o.deferred});
    } else if (o.deferred) {
      int rc = issue_read(c, o.sums->p, o.samples, o.deferred, after);
      if (rc) return rc;
    }
    c->spare.push_back(std::move(o.sums));
    c->older.erase(c->older.begin() + long(i));
  }
  return DSPBR_OK;
}

// Waits for the loop launches of the last pipelined render call and takes
// over its results: the parity the pool's queues are at, the epochs that
// finished (their deferred reads enqueued, their sums spare), whether the
// call's epoch still has paths in the pool, and the call's device time.
static int complete_call(dspbr_ctx* c, std::vector<LateRead>* late = nullptr) {
  if (!c->call_inflight) return DSPBR_OK;
  c->call_inflight = false;
  Status s = c->st();
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  TRY_CUDA(s, cudaStreamSynchronize(c->stream), "render");
  Engine& E = *c->eng;
  E.finish_pipelined(c->call_it0, c->call_loops);
  if (c->call_wait >= 0 && !E.job_done(c->call_wait))
    return s.fail(DSPBR_ERR_DEVICE_FAULT, "render: earlier frame not finished by the render loop");
  int rc = retire_finished(c, nullptr, late);
  if (rc) return rc;
  // a reset since the call has moved its epoch to the older ones
  if (c->slot == c->call_slot && c->tail_live) c->tail_live = !E.job_done(c->slot);
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  c->last_render_ms = ms;
  return DSPBR_OK;
}

// Pipelined frames: finishes every path of the context's epochs in the pool
// (the render loop with its tail drain) and enqueues the deferred reads, oldest
// epoch first.
static int flush_pipeline(dspbr_ctx* c) {
  if (int rc = complete_call(c)) return rc;
  if (!c->tail_live && c->older.empty() && !c->deferred) return DSPBR_OK;
  Status s = c->st();
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  Engine& E = *c->eng;
  if (c->tail_live || !c->older.empty()) {
    std::vector<int> act;
    for (const auto& o : c->older) act.push_back(o.slot);
    if (c->tail_live) act.push_back(c->slot);
    int rc = E.set_active(act);
    // every work item has started: iterations until fewer than the drain
    // threshold of paths are alive, then the tail drain (the bound only
    // guards the loop: a path lives at most max_bounces + 1 iterations)
    if (!rc) rc = E.run_loop(act.back(), 4096 + 8);
    if (rc) return rc;
    for (const auto& o : c->older)
      if (!E.job_done(o.slot)) return s.fail(DSPBR_ERR_DEVICE_FAULT, "render: earlier frame not finished by the drain");
    c->tail_live = false;
    if ((rc = retire_finished(c, nullptr))) return rc;
  }
  if (c->deferred) {
    float* dst = c->deferred;
    c->deferred = nullptr;
    int rc = issue_read(c, c->accum.p, c->sample_count, dst, nullptr);
    if (rc) return rc;
    // the copy stream's mean reads these sums: later renders and resets,
    // which write them on the context's stream, wait for it
    TRY_CUDA(s, after_pending_mean(c), "read accumulation");
  }
  return DSPBR_OK;
}

// Joins the render_async worker and finishes pipelined frames: the state every
// call that is not pipeline-aware starts from.
static int settle(dspbr_ctx* c) {
  int rc = settle_worker(c);
  if (rc) return rc;
  return c->pipelined ? flush_pipeline(c) : DSPBR_OK;
}

// Texture slots of the material record (material.ts layout): 39, 44-59, 63.
static const int kTexSlots[] = {39, 44, 45, 46, 47, 48, 49, 50, 51, 52, 53, 54, 55, 56, 57, 58, 59, 63};
static int32_t max_texture_id(const float* materials, uint32_t num_materials) {
  int32_t mx = -1;
  for (uint32_t m = 0; m < num_materials; ++m)
    for (int k : kTexSlots) {
      float id = materials[size_t(m) * 68 + k];
      if (id >= 0.f) mx = std::max(mx, id < 2147483520.f ? int32_t(id) : INT32_MAX);
    }
  return mx;
}

// Reference-layout nodes for the device: child index / count / first become
// the shader's int() of the stored floats (int bits in lanes 3, 7, 11, 15).
// Returns whether every box bound is finite.
static bool convert_bvh_nodes(const float* nodes, uint32_t num_nodes, std::vector<float>& conv) {
  bool finite = true;
  conv.resize(size_t(num_nodes) * 16);
  for (size_t i = 0; i < size_t(num_nodes); ++i) {
    const float* src = nodes + i * 16;
    float* dst = conv.data() + i * 16;
    std::memcpy(dst, src, 16 * sizeof(float));
    for (int k = 0; k < 16; ++k)
      if (k % 4 != 3 && !std::isfinite(src[k])) finite = false;
    for (int k = 3; k < 16; k += 4) {
      float f = src[k];
      int32_t v = (std::isfinite(f) && f > -2147483648.f && f < 2147483648.f) ? int32_t(f) : -1;
      std::memcpy(dst + k, &v, 4);
    }
  }
  return finite;
}

// Shading classes.  Surface hits are queued per class so that a warp of the
// shading kernel runs one material code path (the DSPBR closure branches on
// these features).  The class only orders the work; results do not depend on it.
static uint32_t material_signature(const float* m) {
  // record offsets: material.ts MaterialData layout (68 floats)
  uint32_t sig = 0;
  if (m[7] > 0.f) sig |= 1u;                                   // transmission
  if (m[7] > 0.f && m[35] > 0.5f) sig |= 2u;                   // thin-walled transmission
  if (m[40] > 0.f) sig |= 4u;                                  // iridescence
  if (m[16] > 0.f || m[17] > 0.f || m[18] > 0.f) sig |= 8u;    // sheen
  if (m[24] > 0.f) sig |= 16u;                                 // clearcoat
  if (m[3] >= 1.f) sig |= 32u;                                 // pure metal
  if (m[64] > 0.f) sig |= 64u;                                 // dispersion
  if (m[26] > 0.f) sig |= 128u;                                // diffuse transmission
  if (m[5] != 0.f) sig |= 256u;                                // anisotropy
  if (m[8] < 1.f || m[27] > 0.f) sig |= 512u;                  // cutout
  for (int k : kTexSlots)
    if (m[k] >= 0.f) sig |= 1024u;                             // textured
  return sig;
}

static int classify_triangles(Status& s, dspbr_scene* sc, cudaStream_t st) {
  std::vector<uint32_t> sigs;
  std::vector<uint8_t> mat_class(sc->num_materials);
  for (uint32_t m = 0; m < sc->num_materials; ++m) {
    uint32_t sig = material_signature(sc->host_materials.data() + size_t(m) * 68);
    size_t k = std::find(sigs.begin(), sigs.end(), sig) - sigs.begin();
    if (k == sigs.size()) sigs.push_back(sig);
    mat_class[m] = uint8_t(k % kNumClasses);
  }
  sc->num_classes = uint32_t(std::min<size_t>(sigs.size(), kNumClasses));
  std::vector<uint8_t> cls(std::max<size_t>(sc->tri_material.size(), 1), 0);
  for (size_t t = 0; t < sc->tri_material.size(); ++t) cls[t] = mat_class[sc->tri_material[t]];
  if (!sc->tri_class.p) {
    int rc = s.cuda(sc->tri_class.alloc(cls.size()), "alloc triangle classes");
    if (rc) return rc;
  }
  int rc = s.cuda(cudaMemcpyAsync(sc->tri_class.p, cls.data(), cls.size(), cudaMemcpyHostToDevice, st), "upload classes");
  if (rc) return rc;
  return s.cuda(cudaStreamSynchronize(st), "upload classes");
}

// The compressed 8-wide BVH of a scene whose binary tree and leaf-ordered
// triangle records are on the device (context option dspbr_set_wide_bvh).
// Rays of scenes with non-finite boxes take the binary traversal anyway.
static int attach_cw8(dspbr_ctx* c, dspbr_scene* sc, Status& s) {
  DeviceCw8 cw;
  if (c->wide_bvh == 8 && sc->boxes_finite && sc->num_nodes) {
    int rc = build_cw8_device(sc->nodes.p, sc->num_nodes, sc->num_slots, sc->tris.p, c->stream, &cw, s);
    if (rc) return rc;
  }
  sc->cnodes.swap(cw.nodes);
  sc->ctris.swap(cw.recs);
  sc->num_cnodes = cw.num_nodes;
  sc->num_crecs = cw.num_recs;
  sc->cw8_levels = cw.levels;
  return DSPBR_OK;
}

// Scene creation with the BVH built and collapsed on the device.
static int scene_create_device_bvh(dspbr_ctx* c, const float* vertices, uint32_t num_vertices,
                                   const uint32_t* indices, uint32_t num_indices, const float* materials,
                                   uint32_t num_materials, dspbr_scene** out) {
  Status s = c->st();
  std::unique_ptr<dspbr_scene> sc(new dspbr_scene());
  sc->ctx = c;
  sc->num_tris = num_indices / 3;
  sc->num_verts = num_vertices;
  sc->num_materials = num_materials;
  double t0 = now_ms();
  int rc;
  if ((rc = s.cuda(sc->verts.alloc(size_t(num_vertices) * 5), "alloc vertices")) ||
      (rc = s.cuda(sc->indices.alloc(num_indices), "alloc indices")) ||
      (rc = s.cuda(sc->materials.alloc(size_t(num_materials) * 17), "alloc materials")) ||
      (rc = s.cuda(cudaMemcpyAsync(sc->verts.p, vertices, size_t(num_vertices) * 80, cudaMemcpyHostToDevice, c->stream), "upload vertices")) ||
      (rc = s.cuda(cudaMemcpyAsync(sc->indices.p, indices, size_t(num_indices) * 4, cudaMemcpyHostToDevice, c->stream), "upload indices")) ||
      (rc = s.cuda(cudaMemcpyAsync(sc->materials.p, materials, size_t(num_materials) * 272, cudaMemcpyHostToDevice, c->stream), "upload materials")))
    return rc;
  DeviceBvh bin;
  rc = c->bvh_builder == DSPBR_BVH_BUILD_DEVICE_LBVH
           ? build_bvh_device(sc->verts.p, sc->indices.p, sc->num_tris, c->stream, &bin, s)
           : build_bvh_device_sah(sc->verts.p, sc->indices.p, sc->num_tris, c->stream, &bin, s);
  if (rc) return rc;
  DeviceWideBvh wide;
  if ((rc = collapse_bvh4_device(bin, c->stream, &wide, s))) return rc;
  sc->bvh_build_ms = now_ms() - t0;
  t0 = now_ms();
  sc->nodes.swap(bin.nodes);
  sc->num_nodes = bin.num_nodes;
  sc->num_slots = bin.num_slots;
  sc->wnodes.swap(wide.nodes);
  sc->wleaves.swap(wide.leaves);
  sc->wroot = wide.root;
  sc->num_wnodes = wide.num_nodes;
  // the builder's boxes are unions of vertex positions: finite iff they are
  for (uint32_t v = 0; v < num_vertices && sc->boxes_finite; ++v)
    for (int k = 0; k < 3; ++k)
      if (!std::isfinite(vertices[size_t(v) * 20 + k])) sc->boxes_finite = false;
  sc->host_materials.assign(materials, materials + size_t(num_materials) * 68);
  sc->max_tex_id = max_texture_id(materials, num_materials);
  sc->tri_material.resize(sc->num_tris);
  for (uint32_t t = 0; t < sc->num_tris; ++t)
    sc->tri_material[t] = uint32_t(vertices[size_t(indices[3 * size_t(t)]) * 20 + 3]);
  if ((rc = classify_triangles(s, sc.get(), c->stream))) return rc;
  if ((rc = s.cuda(sc->tris.alloc(size_t(sc->num_slots) * 3), "alloc tris"))) return rc;
  launch_gather_tris(sc->verts.p, sc->indices.p, bin.remap.p, sc->num_slots, sc->num_tris, sc->tris.p, c->stream);
  if ((rc = s.cuda(cudaGetLastError(), "gather triangles")) ||
      (rc = s.cuda(cudaStreamSynchronize(c->stream), "scene upload")))
    return rc;
  sc->device_remap.swap(bin.remap);
  if ((rc = attach_cw8(c, sc.get(), s))) return rc;
  sc->upload_ms = now_ms() - t0;
  *out = sc.release();
  return DSPBR_OK;
}

extern "C" {

void dspbr_params_default(dspbr_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->max_bounces = 8;
  p->use_ibl = 1;
  p->ibl_rotation_deg = 0.f;
  p->background_from_ibl = 1;
  p->background_color[0] = 0.f; p->background_color[1] = 0.f; p->background_color[2] = 0.f;
  p->background_color[3] = 1.f;
  p->ray_eps = 0.0001f;
  p->clamp_threshold = 3.0f;
  p->rr_start_depth = 2;
  p->rr_termination_prob = 0.1f;
  p->profile = DSPBR_PROFILE_FULL;
  p->rng = DSPBR_RNG_MWC;
  p->seed = 0;
  p->env_sampling = DSPBR_ENV_ALIAS;
}

int dspbr_device_count(int* count) {
  if (!count) return DSPBR_ERR_INVALID;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) { cudaGetLastError(); *count = 0; return DSPBR_ERR_CUDA; }
  *count = n;
  return DSPBR_OK;
}

int dspbr_create(int device, dspbr_ctx** out) {
  if (!out) return DSPBR_ERR_INVALID;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
    cudaGetLastError();
    return DSPBR_ERR_CUDA;
  }
  auto* c = new dspbr_ctx();
  c->device = device;
  dspbr_params_default(&c->params);
  Status s = c->st();
  if (s.cuda(cudaSetDevice(device), "cudaSetDevice") || s.cuda(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream") ||
      s.cuda(cudaEventCreate(&c->ev0), "event") || s.cuda(cudaEventCreate(&c->ev1), "event") ||
      s.cuda(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking), "stream") ||
      s.cuda(cudaEventCreateWithFlags(&c->ev_mean, cudaEventDisableTiming), "event") ||
      s.cuda(cudaEventCreateWithFlags(&c->ev_meaned, cudaEventDisableTiming), "event") ||
      s.cuda(cudaStreamCreateWithFlags(&c->mean_stream, cudaStreamNonBlocking), "stream") ||
      s.cuda(cudaEventCreateWithFlags(&c->ev_copied, cudaEventDisableTiming), "event")) {
    dspbr_destroy(c);
    return DSPBR_ERR_CUDA;
  }
  for (int r = 0; r < dspbr_ctx::kReadRing; ++r)
    if (s.cuda(cudaEventCreateWithFlags(&c->ev_read_copied[r], cudaEventDisableTiming), "event")) {
      dspbr_destroy(c);
      return DSPBR_ERR_CUDA;
    }
  c->eng.reset(new Engine(device, c->stream, &c->err));
  if (int rc = c->eng->init()) {
    dspbr_destroy(c);
    return rc;
  }
  *out = c;
  return DSPBR_OK;
}

int dspbr_destroy(dspbr_ctx* c) {
  if (!c) return DSPBR_ERR_INVALID;
  settle(c);
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->ev_mean) cudaEventDestroy(c->ev_mean);
  if (c->ev_meaned) cudaEventDestroy(c->ev_meaned);
  if (c->mean_stream) cudaStreamSynchronize(c->mean_stream);
  for (int r = 0; r < dspbr_ctx::kReadRing; ++r)
    if (c->ev_read_copied[r]) cudaEventDestroy(c->ev_read_copied[r]);
  if (c->mean_stream) cudaStreamDestroy(c->mean_stream);
  if (c->ev_copied) cudaEventDestroy(c->ev_copied);
  if (c->ev_between) cudaEventDestroy(c->ev_between);
  if (c->ev_retired) cudaEventDestroy(c->ev_retired);
  c->eng.reset();
  if (c->stage) cudaFreeHost(c->stage);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return DSPBR_OK;
}

int dspbr_last_error(const dspbr_ctx* c, char* buf, size_t size) {
  if (!c || !buf || size == 0) return DSPBR_ERR_INVALID;
  std::snprintf(buf, size, "%s", c->err.c_str());
  return DSPBR_OK;
}

// ---- scene -------------------------------------------------------------------------------------
int dspbr_scene_create(dspbr_ctx* c, const float* vertices, uint32_t num_vertices, const uint32_t* indices,
                       uint32_t num_indices, const float* materials, uint32_t num_materials, const float* bvh_nodes,
                       uint32_t num_bvh_nodes, const int32_t* bvh_indices, uint32_t num_bvh_indices,
                       dspbr_scene** out) {
  if (!c || !out) return DSPBR_ERR_INVALID;
  { int rc_ = settle(c); if (rc_) return rc_; }
  Status s = c->st();
  *out = nullptr;
  if (!vertices || num_vertices == 0) return s.fail(DSPBR_ERR_INVALID, "scene: empty vertex buffer");
  if (!indices || num_indices == 0 || num_indices % 3)
    return s.fail(DSPBR_ERR_INVALID, "scene: index buffer does not describe whole triangles");
  if (!materials || num_materials == 0) return s.fail(DSPBR_ERR_INVALID, "scene: no materials");
  for (uint32_t i = 0; i < num_indices; ++i)
    if (indices[i] >= num_vertices) return s.fail(DSPBR_ERR_INVALID, "scene: index %u out of range", i);
  for (uint32_t v = 0; v < num_vertices; ++v) {
    float m = vertices[size_t(v) * 20 + 3];
    if (!(m >= 0.f) || uint32_t(m) >= num_materials)
      return s.fail(DSPBR_ERR_INVALID, "scene: vertex %u references material %g of %u", v, m, num_materials);
  }
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  if ((!bvh_nodes || !bvh_indices) &&
      (c->bvh_builder == DSPBR_BVH_BUILD_DEVICE || c->bvh_builder == DSPBR_BVH_BUILD_DEVICE_LBVH))
    return scene_create_device_bvh(c, vertices, num_vertices, indices, num_indices, materials, num_materials, out);
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  auto* sc = new dspbr_scene();
  sc->ctx = c;
  std::vector<float> host_nodes;
  std::vector<int32_t> host_remap;
  double t0 = now_ms();
  if (!bvh_nodes || !bvh_indices) {
    dspbr_bvh* bvh = nullptr;
    int rc = dspbr_bvh_build(vertices, num_vertices, 20, indices, num_indices, &bvh);
    if (rc != DSPBR_OK) {
      char msg[256] = {0};
      if (bvh) dspbr_bvh_error(bvh, msg, sizeof msg);
      dspbr_bvh_free(bvh);
      delete sc;
      return s.fail(DSPBR_ERR_INVALID, "bvh build failed: %s", msg);
    }
    uint32_t nn = 0, ni = 0;
    dspbr_bvh_info(bvh, &nn, &ni, nullptr, nullptr);
    host_nodes.resize(size_t(nn) * 16);
    host_remap.resize(ni);
    dspbr_bvh_copy(bvh, host_nodes.data(), host_remap.data());
    dspbr_bvh_free(bvh);
    bvh_nodes = host_nodes.data();
    num_bvh_nodes = nn;
    bvh_indices = host_remap.data();
    num_bvh_indices = ni;
  }
  sc->bvh_build_ms = now_ms() - t0;
  if (num_bvh_nodes == 0) { delete sc; return s.fail(DSPBR_ERR_INVALID, "scene: empty BVH"); }
  t0 = now_ms();
  std::vector<float> conv;
  sc->boxes_finite = convert_bvh_nodes(bvh_nodes, num_bvh_nodes, conv);
  sc->num_nodes = num_bvh_nodes;
  sc->num_slots = num_bvh_indices;
  sc->num_tris = num_indices / 3;
  sc->num_verts = num_vertices;
  sc->num_materials = num_materials;
  DevBuf<int32_t> remap;
  int rc = DSPBR_OK;
  if ((rc = s.cuda(sc->nodes.alloc(size_t(num_bvh_nodes) * 4), "alloc nodes")) ||
      (rc = s.cuda(sc->tris.alloc(size_t(std::max<uint32_t>(num_bvh_indices, 1)) * 3), "alloc tris")) ||
      (rc = s.cuda(sc->verts.alloc(size_t(num_vertices) * 5), "alloc vertices")) ||
      (rc = s.cuda(sc->indices.alloc(num_indices), "alloc indices")) ||
      (rc = s.cuda(sc->materials.alloc(size_t(num_materials) * 17), "alloc materials")) ||
      (rc = s.cuda(remap.alloc(std::max<uint32_t>(num_bvh_indices, 1)), "alloc remap")) ||
      (rc = s.cuda(cudaMemcpyAsync(sc->nodes.p, conv.data(), conv.size() * 4, cudaMemcpyHostToDevice, c->stream), "upload nodes")) ||
      (rc = s.cuda(cudaMemcpyAsync(sc->verts.p, vertices, size_t(num_vertices) * 80, cudaMemcpyHostToDevice, c->stream), "upload vertices")) ||
      (rc = s.cuda(cudaMemcpyAsync(sc->indices.p, indices, size_t(num_indices) * 4, cudaMemcpyHostToDevice, c->stream), "upload indices")) ||
      (rc = s.cuda(cudaMemcpyAsync(sc->materials.p, materials, size_t(num_materials) * 272, cudaMemcpyHostToDevice, c->stream), "upload materials")) ||
      (rc = s.cuda(cudaMemcpyAsync(remap.p, bvh_indices, size_t(num_bvh_indices) * 4, cudaMemcpyHostToDevice, c->stream), "upload remap"))) {
    delete sc;
    return rc;
  }
  {
    // the 4-wide BVH for the path kernels, collapsed from the same binary tree
    WideBvh wb = collapse_bvh4(conv.data(), num_bvh_nodes, num_bvh_indices);
    sc->wroot = wb.root;
    sc->num_wnodes = uint32_t(wb.nodes.size());
    if ((rc = s.cuda(sc->wnodes.alloc(std::max<size_t>(wb.nodes.size(), 1) * 8), "alloc wide nodes")) ||
        (rc = s.cuda(sc->wleaves.alloc(std::max<size_t>(wb.leaves.size(), 1)), "alloc wide leaves")) ||
        (rc = s.cuda(cudaMemcpyAsync(sc->wnodes.p, wb.nodes.data(), wb.nodes.size() * sizeof(WideNode4),
                                     cudaMemcpyHostToDevice, c->stream), "upload wide nodes")) ||
        (rc = s.cuda(cudaMemcpyAsync(sc->wleaves.p, wb.leaves.data(), wb.leaves.size() * sizeof(WideLeaf),
                                     cudaMemcpyHostToDevice, c->stream), "upload wide leaves")) ||
        (rc = s.cuda(cudaStreamSynchronize(c->stream), "upload wide BVH"))) {
      delete sc;
      return rc;
    }
  }
  sc->host_materials.assign(materials, materials + size_t(num_materials) * 68);
  sc->max_tex_id = max_texture_id(materials, num_materials);
  sc->tri_material.resize(sc->num_tris);
  for (uint32_t t = 0; t < sc->num_tris; ++t)
    sc->tri_material[t] = uint32_t(vertices[size_t(indices[3 * size_t(t)]) * 20 + 3]);
  if ((rc = classify_triangles(s, sc, c->stream))) {
    delete sc;
    return rc;
  }
  if (num_bvh_indices)
    launch_gather_tris(sc->verts.p, sc->indices.p, remap.p, num_bvh_indices, sc->num_tris, sc->tris.p, c->stream);
  if ((rc = s.cuda(cudaGetLastError(), "gather triangles")) || (rc = s.cuda(cudaStreamSynchronize(c->stream), "scene upload")) ||
      (rc = attach_cw8(c, sc, s))) {
    delete sc;
    return rc;
  }
  sc->upload_ms = now_ms() - t0;
  *out = sc;
  return DSPBR_OK;
}

int dspbr_set_wide_bvh(dspbr_ctx* c, int width) {
  if (!c || (width != 4 && width != 8)) return DSPBR_ERR_INVALID;
  c->wide_bvh = width;
  return DSPBR_OK;
}

int dspbr_scene_wide_bvh(const dspbr_scene* sc, int* width, uint32_t* nodes, uint32_t* levels) {
  if (!sc) return DSPBR_ERR_INVALID;
  if (width) *width = sc->num_cnodes ? 8 : 4;
  if (nodes) *nodes = sc->num_cnodes ? sc->num_cnodes : sc->num_wnodes;
  if (levels) *levels = sc->cw8_levels;
  return DSPBR_OK;
}

int dspbr_set_bvh_builder(dspbr_ctx* c, int builder) {
  if (!c || (builder != DSPBR_BVH_BUILD_HOST && builder != DSPBR_BVH_BUILD_DEVICE &&
             builder != DSPBR_BVH_BUILD_DEVICE_LBVH))
    return DSPBR_ERR_INVALID;
  c->bvh_builder = builder;
  return DSPBR_OK;
}

int dspbr_scene_bvh(const dspbr_scene* sc, float* nodes, int32_t* remap, uint32_t* num_nodes, uint32_t* num_indices) {
  if (!sc) return DSPBR_ERR_INVALID;
  if (num_nodes) *num_nodes = sc->num_nodes;
  if (num_indices) *num_indices = sc->num_slots;
  Status s = sc->ctx->st();
  TRY_CUDA(s, cudaSetDevice(sc->ctx->device), "cudaSetDevice");
  if (nodes) {
    TRY_CUDA(s, cudaMemcpy(nodes, sc->nodes.p, size_t(sc->num_nodes) * 64, cudaMemcpyDeviceToHost), "read BVH");
    for (size_t i = 0; i < size_t(sc->num_nodes) * 16; i += 4) {  // int bits back to the reference's floats
      int32_t v;
      std::memcpy(&v, nodes + i + 3, 4);
      nodes[i + 3] = float(v);
    }
  }
  if (remap) {
    if (sc->device_remap.p) {
      TRY_CUDA(s, cudaMemcpy(remap, sc->device_remap.p, size_t(sc->num_slots) * 4, cudaMemcpyDeviceToHost), "read remap");
    } else {
      std::vector<float4> t(size_t(sc->num_slots) * 3);
      TRY_CUDA(s, cudaMemcpy(t.data(), sc->tris.p, t.size() * 16, cudaMemcpyDeviceToHost), "read remap");
      for (size_t i = 0; i < sc->num_slots; ++i) std::memcpy(remap + i, &t[3 * i].w, 4);
    }
  }
  return DSPBR_OK;
}

int dspbr_scene_set_textures(dspbr_scene* sc, const float* tex_infos, uint32_t num_tex_infos,
                             const dspbr_texture_array* arrays, uint32_t num_arrays) {
  if (!sc || (num_tex_infos && !tex_infos) || (num_arrays && !arrays)) return DSPBR_ERR_INVALID;
  { int rc_ = settle(sc->ctx); if (rc_) return rc_; }
  Status s = sc->ctx->st();
  if (int64_t(sc->max_tex_id) >= int64_t(num_tex_infos))
    return s.fail(DSPBR_ERR_INVALID, "set_textures: the materials use texture id %d, %u texture infos given",
                  sc->max_tex_id, num_tex_infos);
  for (uint32_t a = 0; a < num_arrays; ++a) {
    const dspbr_texture_array& t = arrays[a];
    if (t.width <= 0 || t.height <= 0 || t.layers <= 0 || !t.rgba8 || int64_t(t.width) * t.height * t.layers > (int64_t(1) << 31))
      return s.fail(DSPBR_ERR_INVALID, "set_textures: texture array %u is malformed", a);
  }
  TRY_CUDA(s, cudaSetDevice(sc->ctx->device), "cudaSetDevice");
  cudaStream_t st = sc->ctx->stream;
  TRY_CUDA(s, cudaStreamSynchronize(st), "set textures");
  std::vector<std::unique_ptr<DevBuf<uchar4>>> data;
  std::vector<DevTexArray> desc(num_arrays);
  for (uint32_t a = 0; a < num_arrays; ++a) {
    const dspbr_texture_array& t = arrays[a];
    const size_t n = size_t(t.width) * t.height * t.layers;
    data.emplace_back(new DevBuf<uchar4>());
    TRY_CUDA(s, data.back()->alloc(n), "alloc texture array");
    TRY_CUDA(s, cudaMemcpyAsync(data.back()->p, t.rgba8, n * 4, cudaMemcpyHostToDevice, st), "upload texture array");
    desc[a] = DevTexArray{data.back()->p, t.width, t.height, t.layers};
  }
  DevBuf<DevTexArray> dt;
  DevBuf<float4> di;
  if (num_arrays) {
    TRY_CUDA(s, dt.alloc(num_arrays), "alloc texture arrays");
    TRY_CUDA(s, cudaMemcpyAsync(dt.p, desc.data(), desc.size() * sizeof(DevTexArray), cudaMemcpyHostToDevice, st),
             "upload texture arrays");
  }
  if (num_tex_infos) {
    TRY_CUDA(s, di.alloc(size_t(num_tex_infos) * 2), "alloc texture infos");
    TRY_CUDA(s, cudaMemcpyAsync(di.p, tex_infos, size_t(num_tex_infos) * 32, cudaMemcpyHostToDevice, st),
             "upload texture infos");
  }
  TRY_CUDA(s, cudaStreamSynchronize(st), "set textures");
  sc->tex_data.swap(data);
  sc->tex_arrays.swap(dt);
  sc->texinfo.swap(di);
  sc->num_texinfo = num_tex_infos;
  sc->num_tex_arrays = num_arrays;
  return dspbr_reset(sc->ctx);
}

int dspbr_scene_update_materials(dspbr_scene* sc, const float* materials, uint32_t first, uint32_t count) {
  if (!sc || !materials || first + count > sc->num_materials) return DSPBR_ERR_INVALID;
  { int rc_ = settle(sc->ctx); if (rc_) return rc_; }
  Status s = sc->ctx->st();
  TRY_CUDA(s, cudaSetDevice(sc->ctx->device), "cudaSetDevice");
  TRY_CUDA(s, cudaMemcpyAsync(sc->materials.p + size_t(first) * 17, materials, size_t(count) * 272,
                              cudaMemcpyHostToDevice, sc->ctx->stream), "update materials");
  TRY_CUDA(s, cudaStreamSynchronize(sc->ctx->stream), "update materials");
  std::copy(materials, materials + size_t(count) * 68, sc->host_materials.begin() + size_t(first) * 68);
  sc->max_tex_id = max_texture_id(sc->host_materials.data(), sc->num_materials);
  { int rc_ = classify_triangles(s, sc, sc->ctx->stream); if (rc_) return rc_; }
  dspbr_reset(sc->ctx);
  return DSPBR_OK;
}

int dspbr_scene_update_vertices(dspbr_scene* sc, const float* vertices, uint32_t first, uint32_t count) {
  if (!sc || (count && !vertices) || uint64_t(first) + count > sc->num_verts) return DSPBR_ERR_INVALID;
  { int rc_ = settle(sc->ctx); if (rc_) return rc_; }
  Status s = sc->ctx->st();
  for (uint32_t v = 0; v < count; ++v) {
    const float m = vertices[size_t(v) * 20 + 3];
    if (!(m >= 0.f) || m >= float(sc->num_materials))
      return s.fail(DSPBR_ERR_INVALID, "update vertices: vertex %u references material %g of %u", first + v, m,
                    sc->num_materials);
  }
  TRY_CUDA(s, cudaSetDevice(sc->ctx->device), "cudaSetDevice");
  cudaStream_t st = sc->ctx->stream;
  TRY_CUDA(s, cudaStreamSynchronize(st), "update vertices");
  TRY_CUDA(s, cudaMemcpyAsync(sc->verts.p + size_t(first) * 5, vertices, size_t(count) * 80, cudaMemcpyHostToDevice, st),
           "update vertices");
  const double t0 = now_ms();
  int rc = refit_scene_device(sc->nodes.p, sc->num_nodes, sc->num_slots, sc->wnodes.p, sc->num_wnodes, sc->wleaves.p,
                              sc->tris.p, sc->device_remap.p, sc->verts.p, sc->indices.p, sc->num_tris, st, s);
  if (rc) return rc;
  for (uint32_t v = 0; v < count && sc->boxes_finite; ++v)
    for (int k = 0; k < 3; ++k)
      if (!std::isfinite(vertices[size_t(v) * 20 + k])) sc->boxes_finite = false;
  // the 8-wide tree is rebuilt from the refitted binary tree (its grouping follows the new boxes)
  if ((rc = attach_cw8(sc->ctx, sc, s))) return rc;
  sc->refit_ms = now_ms() - t0;
  dspbr_reset(sc->ctx);
  return DSPBR_OK;
}

int dspbr_scene_device_bytes(const dspbr_scene* sc, uint64_t* bytes) {
  if (!sc || !bytes) return DSPBR_ERR_INVALID;
  *bytes = sc->bytes();
  return DSPBR_OK;
}

int dspbr_scene_destroy(dspbr_scene* sc) {
  if (!sc) return DSPBR_ERR_INVALID;
  { int rc_ = settle(sc->ctx); if (rc_) return rc_; }
  cudaSetDevice(sc->ctx->device);
  cudaStreamSynchronize(sc->ctx->stream);
  if (sc->ctx->scene == sc) sc->ctx->scene = nullptr;
  delete sc;
  return DSPBR_OK;
}

// ---- IBL ---------------------------------------------------------------------------------------------
// Vose's alias method in FP64 over p(x,y) = yPdf[y] * pdf[y][x], the pmf the
// reference's two-level CDF inversion realises.
static void build_alias(const std::vector<float>& pdf, const std::vector<float>& ypdf, int w, int h,
                        std::vector<float>& prob, std::vector<int>& alias) {
  size_t n = size_t(w) * h;
  std::vector<double> q(n);
  double tot = 0;
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      double v = double(ypdf[y]) * double(pdf[size_t(y) * w + x]);
      q[size_t(y) * w + x] = v;
      tot += v;
    }
  prob.assign(n, 1.f);
  alias.resize(n);
  for (size_t i = 0; i < n; ++i) alias[i] = int(i);
  if (!(tot > 0)) return;
  std::vector<size_t> small, large;
  for (size_t i = 0; i < n; ++i) {
    q[i] = q[i] * double(n) / tot;
    (q[i] < 1.0 ? small : large).push_back(i);
  }
  while (!small.empty() && !large.empty()) {
    size_t l = small.back(); small.pop_back();
    size_t g = large.back();
    prob[l] = float(q[l]);
    alias[l] = int(g);
    q[g] = (q[g] + q[l]) - 1.0;
    if (q[g] < 1.0) { large.pop_back(); small.push_back(g); }
  }
  for (size_t g : large) prob[g] = 1.f;
  for (size_t l : small) prob[l] = 1.f;
}

int dspbr_ibl_create(dspbr_ctx* c, const float* rgba, int w, int h, dspbr_ibl** out) {
  if (!c || !out) return DSPBR_ERR_INVALID;
  { int rc_ = settle(c); if (rc_) return rc_; }
  Status s = c->st();
  *out = nullptr;
  if (!rgba || w <= 0 || h <= 0) return s.fail(DSPBR_ERR_INVALID, "ibl: empty image");
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  auto* e = new dspbr_ibl();
  e->ctx = c;
  e->w = w;
  e->h = h;
  size_t n = size_t(w) * h;
  int rc;
  if ((rc = s.cuda(e->rgba.alloc(n), "alloc env")) || (rc = s.cuda(e->pdf.alloc(n), "alloc pdf")) ||
      (rc = s.cuda(e->cdf.alloc(n), "alloc cdf")) || (rc = s.cuda(e->lum.alloc(n), "alloc lum")) ||
      (rc = s.cuda(e->ypdf.alloc(h), "alloc ypdf")) || (rc = s.cuda(e->ycdf.alloc(h), "alloc ycdf")) ||
      (rc = s.cuda(e->rowsum.alloc(h), "alloc rowsum")) || (rc = s.cuda(e->total.alloc(1), "alloc total")) ||
      (rc = s.cuda(e->alias_prob.alloc(n), "alloc alias")) || (rc = s.cuda(e->alias_idx.alloc(n), "alloc alias")) ||
      (rc = s.cuda(cudaMemcpyAsync(e->rgba.p, rgba, n * 16, cudaMemcpyHostToDevice, c->stream), "upload env"))) {
    delete e;
    return rc;
  }
  launch_ibl_tables(e->rgba.p, w, h, e->lum.p, e->pdf.p, e->cdf.p, e->rowsum.p, e->ypdf.p, e->ycdf.p, e->total.p,
                    c->stream);
  std::vector<float> pdf(n), ypdf(h);
  if ((rc = s.cuda(cudaGetLastError(), "ibl tables")) ||
      (rc = s.cuda(cudaMemcpyAsync(pdf.data(), e->pdf.p, n * 4, cudaMemcpyDeviceToHost, c->stream), "read pdf")) ||
      (rc = s.cuda(cudaMemcpyAsync(ypdf.data(), e->ypdf.p, size_t(h) * 4, cudaMemcpyDeviceToHost, c->stream), "read ypdf")) ||
      (rc = s.cuda(cudaMemcpyAsync(&e->total_sum, e->total.p, 8, cudaMemcpyDeviceToHost, c->stream), "read total")) ||
      (rc = s.cuda(cudaStreamSynchronize(c->stream), "ibl tables"))) {
    delete e;
    return rc;
  }
  e->lum.reset();
  e->rowsum.reset();
  std::vector<float> prob;
  std::vector<int> alias;
  build_alias(pdf, ypdf, w, h, prob, alias);
  if ((rc = s.cuda(cudaMemcpyAsync(e->alias_prob.p, prob.data(), n * 4, cudaMemcpyHostToDevice, c->stream), "upload alias")) ||
      (rc = s.cuda(cudaMemcpyAsync(e->alias_idx.p, alias.data(), n * 4, cudaMemcpyHostToDevice, c->stream), "upload alias")) ||
      (rc = s.cuda(cudaStreamSynchronize(c->stream), "upload alias"))) {
    delete e;
    return rc;
  }
  *out = e;
  return DSPBR_OK;
}

int dspbr_ibl_tables(const dspbr_ibl* e, float* pdf, float* cdf, float* ypdf, float* ycdf, double* total) {
  if (!e) return DSPBR_ERR_INVALID;
  Status s = e->ctx->st();
  size_t n = size_t(e->w) * e->h;
  TRY_CUDA(s, cudaSetDevice(e->ctx->device), "cudaSetDevice");
  if (pdf) TRY_CUDA(s, cudaMemcpy(pdf, e->pdf.p, n * 4, cudaMemcpyDeviceToHost), "read pdf");
  if (cdf) TRY_CUDA(s, cudaMemcpy(cdf, e->cdf.p, n * 4, cudaMemcpyDeviceToHost), "read cdf");
  if (ypdf) TRY_CUDA(s, cudaMemcpy(ypdf, e->ypdf.p, size_t(e->h) * 4, cudaMemcpyDeviceToHost), "read ypdf");
  if (ycdf) TRY_CUDA(s, cudaMemcpy(ycdf, e->ycdf.p, size_t(e->h) * 4, cudaMemcpyDeviceToHost), "read ycdf");
  if (total) *total = e->total_sum;
  return DSPBR_OK;
}

int dspbr_ibl_alias_table(const dspbr_ibl* e, float* prob, int32_t* alias) {
  if (!e) return DSPBR_ERR_INVALID;
  Status s = e->ctx->st();
  size_t n = size_t(e->w) * e->h;
  TRY_CUDA(s, cudaSetDevice(e->ctx->device), "cudaSetDevice");
  if (prob) TRY_CUDA(s, cudaMemcpy(prob, e->alias_prob.p, n * 4, cudaMemcpyDeviceToHost), "read alias prob");
  if (alias) TRY_CUDA(s, cudaMemcpy(alias, e->alias_idx.p, n * 4, cudaMemcpyDeviceToHost), "read alias");
  return DSPBR_OK;
}

int dspbr_ibl_destroy(dspbr_ibl* e) {
  if (!e) return DSPBR_ERR_INVALID;
  { int rc_ = settle(e->ctx); if (rc_) return rc_; }
  cudaSetDevice(e->ctx->device);
  cudaStreamSynchronize(e->ctx->stream);
  if (e->ctx->ibl == e) e->ctx->ibl = nullptr;
  delete e;
  return DSPBR_OK;
}

// ---- viewport state -------------------------------------------------------------------------------
int dspbr_set_scene(dspbr_ctx* c, dspbr_scene* sc) {
  if (!c || (sc && sc->ctx != c)) return DSPBR_ERR_INVALID;
  c->scene = sc;
  return dspbr_reset(c);
}
int dspbr_set_ibl(dspbr_ctx* c, dspbr_ibl* e) {
  if (!c || (e && e->ctx != c)) return DSPBR_ERR_INVALID;
  c->ibl = e;
  return dspbr_reset(c);
}
int dspbr_set_camera(dspbr_ctx* c, const float m[16], float fov_deg, float near_plane) {
  if (!c || !m || !(fov_deg > 0.f && fov_deg < 180.f) || !(near_plane > 0.f)) return DSPBR_ERR_INVALID;
  std::memcpy(c->matrix, m, sizeof c->matrix);
  c->fov = fov_deg;
  c->near_plane = near_plane;
  c->has_camera = true;
  return dspbr_reset(c);
}
int dspbr_set_params(dspbr_ctx* c, const dspbr_params* p) {
  if (!c || !p || p->max_bounces < 0 || p->max_bounces > 4096) return DSPBR_ERR_INVALID;
  c->params = *p;
  return dspbr_reset(c);
}
int dspbr_get_params(const dspbr_ctx* c, dspbr_params* p) {
  if (!c || !p) return DSPBR_ERR_INVALID;
  *p = c->params;
  return DSPBR_OK;
}
int dspbr_set_wave_paths(dspbr_ctx* c, uint32_t paths) {
  if (!c) return DSPBR_ERR_INVALID;
  { int rc_ = settle(c); if (rc_) return rc_; }
  c->wave_paths = paths ? paths : (1u << 24);
  return DSPBR_OK;
}

int dspbr_set_drain_threshold(dspbr_ctx* c, uint32_t paths) {
  if (!c) return DSPBR_ERR_INVALID;
  { int rc_ = settle(c); if (rc_) return rc_; }
  c->eng->set_drain_below(paths);
  return DSPBR_OK;
}

int dspbr_resize(dspbr_ctx* c, int w, int h) {
  if (!c || w <= 0 || h <= 0 || int64_t(w) * h > (int64_t(1) << 28)) return DSPBR_ERR_INVALID;
  { int rc_ = settle(c); if (rc_) return rc_; }
  Status s = c->st();
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  TRY_CUDA(s, cudaStreamSynchronize(c->stream), "resize");
  { int rc_ = dspbr_read_wait(c); if (rc_) return rc_; }  // a pending copy reads the mean buffer
  // the image buffers only grow: a viewport that changes size request by
  // request keeps its allocations (a fresh cudaMalloc of tens of MB after
  // other allocations were freed costs milliseconds)
  size_t npix = size_t(w) * h;
  if (c->accum.n < npix) TRY_CUDA(s, c->accum.alloc(npix), "alloc accumulation");
  if (c->mean.n < npix) TRY_CUDA(s, c->mean.alloc(npix), "alloc readback");
  c->width = w;
  c->height = h;
  return dspbr_reset(c);
}

int dspbr_reset(dspbr_ctx* c) {
  if (!c) return DSPBR_ERR_INVALID;
  { int rc_ = settle_worker(c); if (rc_) return rc_; }
  Status s = c->st();
  if (c->pipelined && c->tail_live) {
    // with a render call in flight, its epochs that finish leave the older
    // ones when it completes (at the latest in the next render call, before
    // its launches): until then one more epoch than depth - 1 may wait there
    if (int(c->older.size()) + 1 >= c->depth && !c->call_inflight) {
      int rc = flush_pipeline(c);
      if (rc) return rc;
    } else {
      // a new epoch in a free slot and sum buffer; the old one finishes
      // during the next render calls
      TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
      const size_t npix = size_t(c->width) * c->height;
      dspbr_ctx::Older o;
      TRY_CUDA(s, take_spare(c, npix, o.sums), "alloc accumulation");
      o.sums->swap(c->accum);
      o.samples = c->sample_count;
      o.slot = c->slot;
      o.deferred = c->deferred;
      c->deferred = nullptr;
      c->older.push_back(std::move(o));
      c->slot = free_slot(c);
      c->tail_live = false;
      // the buffer taken over may still be read by the mean of an earlier
      // epoch's read (the device-to-host copy behind it reads the mean buffer)
      TRY_CUDA(s, after_pending_mean(c), "reset");
    }
  }
  c->sample_count = 0;
  if (c->accum.p) {
    TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
    TRY_CUDA(s, after_pending_mean(c), "reset");  // a read's mean may still read these sums
    TRY_CUDA(s, cudaMemsetAsync(c->accum.p, 0, size_t(c->width) * c->height * sizeof(double4), c->stream),
             "clear accumulation");
  }
  return DSPBR_OK;
}

static WaveParams make_wave(const dspbr_ctx* c, uint32_t frame_base) {
  return make_job_params(c->params, c->matrix, c->fov, c->near_plane, c->width, c->height, c->ibl != nullptr,
                         frame_base);
}

static int enqueue_frames(dspbr_ctx* c, int frames, bool async) {
  Status s = c->st();
  int rc = settle(c);
  if (rc) return rc;
  if (frames <= 0) return s.fail(DSPBR_ERR_INVALID, "render: frames must be positive");
  if (!c->scene) return s.fail(DSPBR_ERR_STATE, "render: no scene set");
  if (int64_t(c->scene->max_tex_id) >= int64_t(c->scene->num_texinfo))
    return s.fail(DSPBR_ERR_STATE, "render: the scene's materials use textures; call dspbr_scene_set_textures");
  if (!c->has_camera) return s.fail(DSPBR_ERR_STATE, "render: no camera set");
  if (c->width <= 0 || !c->accum.p) return s.fail(DSPBR_ERR_STATE, "render: resize() was not called");
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  Engine& E = *c->eng;
  Job job{};
  job.p = make_wave(c, uint32_t(c->sample_count + 1));
  job.s = c->scene->view();
  job.s.wide = c->params.traversal == DSPBR_TRAVERSAL_WIDE;
  if (c->ibl) job.e = c->ibl->view();
  job.accum = reinterpret_cast<double*>(c->accum.p);
  const unsigned long long items = uint64_t(job.p.npix) * uint64_t(frames);
  // pool: up to wave_paths slots, no more than the work needs; it is kept
  // between renders unless the limit drops below it
  uint32_t want = uint32_t(std::min<uint64_t>(c->wave_paths, items));
  if (E.capacity() < want || E.capacity() > c->wave_paths) {
    if ((rc = E.ensure_pool(want))) return rc;
  }
  const uint64_t pool = E.capacity();
  // every slot runs paths back to back: while work items remain all slots are
  // busy, and a path lives at most max_bounces + 1 iterations
  const uint64_t per_path = uint64_t(job.p.max_bounces) + 1;
  const unsigned long long max_iter = (items * per_path + pool - 1) / pool + per_path + 4;
  if ((rc = E.set_job(0, job, items)) || (rc = E.set_active({0}))) return rc;
  c->sample_count += uint64_t(frames);
  c->rays_primary += items;
  TRY_CUDA(s, cudaEventRecord(c->ev0, c->stream), "event");
  c->pending = true;
  const bool counting = c->counting;
  if (!async) {
    rc = E.run_until_done(0, max_iter, counting);
    if (rc) {
      c->pending = false;
      E.clear_marks();
      return rc;
    }
    TRY_CUDA(s, cudaEventRecord(c->ev1, c->stream), "event");
    return DSPBR_OK;
  }
  c->worker_done.store(false);
  c->worker = std::thread([c, max_iter, counting]() {
    int r = c->st().cuda(cudaSetDevice(c->device), "cudaSetDevice");
    if (!r) r = c->eng->run_until_done(0, max_iter, counting);
    if (!r) r = c->st().cuda(cudaEventRecord(c->ev1, c->stream), "event");
    c->worker_rc = r;
    c->worker_done.store(true);
  });
  return DSPBR_OK;
}

// Pipelined frames: the render loop until the previous epoch (if it still
// has paths in the pool) has finished, its deferred read enqueued on the copy
// stream right then, and on until every sample of these frames has started.
// The call returns once the loop launches are enqueued, with this epoch's
// last paths possibly still in the pool; the next call that needs the pool's
// state waits for them (complete_call).
static int render_pipelined_launch(dspbr_ctx* c, int frames, std::vector<LateRead>& late);

static int render_pipelined(dspbr_ctx* c, int frames) {
  Status s = c->st();
  int rc = settle_worker(c);
  if (rc) return rc;
  if (frames <= 0) return s.fail(DSPBR_ERR_INVALID, "render: frames must be positive");
  if (!c->scene) return s.fail(DSPBR_ERR_STATE, "render: no scene set");
  if (int64_t(c->scene->max_tex_id) >= int64_t(c->scene->num_texinfo))
    return s.fail(DSPBR_ERR_STATE, "render: the scene's materials use textures; call dspbr_scene_set_textures");
  if (!c->has_camera) return s.fail(DSPBR_ERR_STATE, "render: no camera set");
  if (c->width <= 0 || !c->accum.p) return s.fail(DSPBR_ERR_STATE, "render: resize() was not called");
  // the reads of the epochs the last call finished are enqueued after this
  // call's loop launches (their means wait for ev_retired, recorded before
  // them): the device goes on to the loop first
  std::vector<LateRead> late;
  rc = complete_call(c, &late);
  if (!rc && !late.empty()) rc = s.cuda(cudaEventRecord(c->ev_retired, c->stream), "event");
  if (!rc) rc = render_pipelined_launch(c, frames, late);
  // the reads the launch did not enqueue (an error, or a flush before it)
  for (const LateRead& r : late) {
    int rc2 = issue_read(c, r.sums, r.samples, r.dst, c->ev_retired);
    if (!rc) rc = rc2;
  }
  return rc;
}

static int render_pipelined_launch(dspbr_ctx* c, int frames, std::vector<LateRead>& late) {
  Status s = c->st();
  int rc = DSPBR_OK;
  // a read of this epoch waits for the samples rendered so far, not these
  if (c->deferred && (rc = flush_pipeline(c))) return rc;
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  Engine& E = *c->eng;
  const unsigned long long npix = uint64_t(c->width) * uint64_t(c->height);
  const unsigned long long items = npix * uint64_t(frames);
  // room for this epoch's samples and the last paths of the epochs in flight;
  // the pool changes size only when empty
  const uint32_t want = uint32_t(std::min<uint64_t>(c->wave_paths, uint64_t(c->depth) * items));
  if (E.capacity() < want || E.capacity() > c->wave_paths) {
    if ((rc = flush_pipeline(c)) || (rc = E.ensure_pool(want))) return rc;
  }
  if (c->tail_live) {
    // the epoch goes on: its job takes more work items (frame numbers continue)
    if ((rc = E.add_items(c->slot, items))) return rc;
  } else {
    Job job{};
    job.p = make_wave(c, uint32_t(c->sample_count + 1));
    job.s = c->scene->view();
    job.s.wide = c->params.traversal == DSPBR_TRAVERSAL_WIDE;
    if (c->ibl) job.e = c->ibl->view();
    job.accum = reinterpret_cast<double*>(c->accum.p);
    if ((rc = E.set_job(c->slot, job, items))) return rc;
  }
  std::vector<int> act;
  for (const auto& o : c->older) act.push_back(o.slot);
  act.push_back(c->slot);
  // with depth - 1 older epochs in flight the oldest is waited for
  const int wait = int(c->older.size()) + 1 >= c->depth ? c->older.front().slot : -1;
  if ((rc = E.set_active(act))) return rc;
  c->sample_count += uint64_t(frames);
  c->rays_primary += items;
  const uint64_t pool = E.capacity();
  const uint64_t per_path = uint64_t(std::max(c->params.max_bounces, 0)) + 1;
  const unsigned long long max_iter = (items * per_path + pool - 1) / pool + uint64_t(c->depth) * per_path + 8;
  TRY_CUDA(s, cudaEventRecord(c->ev0, c->stream), "event");
  const bool read_oldest = wait >= 0 && c->older.front().deferred;
  unsigned long long it0 = 0;
  int loops = 0;
  rc = E.launch_pipelined(wait, max_iter, read_oldest ? c->ev_between : nullptr, &it0, &loops);
  for (const LateRead& r : late)
    if (!rc) rc = issue_read(c, r.sums, r.samples, r.dst, c->ev_retired);
  late.clear();
  if (!rc && read_oldest) {
    // the oldest epoch is complete at ev_between: its image is copied while
    // this epoch's iterations run
    auto& o = c->older.front();
    float* dst = o.deferred;
    o.deferred = nullptr;
    rc = issue_read(c, o.sums->p, o.samples, dst, c->ev_between);
  }
  if (!rc) rc = s.cuda(cudaEventRecord(c->ev1, c->stream), "event");
  if (rc) return rc;
  // the host goes on (the caller's next camera, reads and render call) while
  // the loop runs; complete_call takes over its results
  c->call_inflight = true;
  c->call_it0 = it0;
  c->call_loops = loops;
  c->call_wait = wait;
  c->call_slot = c->slot;
  c->tail_live = true;
  return DSPBR_OK;
}

int dspbr_set_pipelining(dspbr_ctx* c, int enable) {
  if (!c) return DSPBR_ERR_INVALID;
  int rc = settle(c);
  if (rc) return rc;
  Status s = c->st();
  if (enable && !c->ev_between)
    TRY_CUDA(s, cudaEventCreateWithFlags(&c->ev_between, cudaEventDisableTiming), "event");
  if (enable && !c->ev_retired)
    TRY_CUDA(s, cudaEventCreateWithFlags(&c->ev_retired, cudaEventDisableTiming), "event");
  c->pipelined = enable != 0;
  return DSPBR_OK;
}

int dspbr_set_pipeline_depth(dspbr_ctx* c, int depth) {
  if (!c || depth < 2 || depth > dspbr_ctx::kMaxDepth) return DSPBR_ERR_INVALID;
  int rc = settle(c);
  if (rc) return rc;
  c->depth = depth;
  return DSPBR_OK;
}

int dspbr_read_wait_ready(dspbr_ctx* c, int* in_flight) {
  if (!c) return DSPBR_ERR_INVALID;
  { int rc_ = settle_worker(c); if (rc_) return rc_; }
  int n = c->deferred ? 1 : 0;
  for (const auto& o : c->older) n += o.deferred ? 1 : 0;
  if (in_flight) *in_flight = n;
  if (!c->copy_pending) return DSPBR_OK;
  Status s = c->st();
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  c->copy_pending = false;
  TRY_CUDA(s, cudaEventSynchronize(c->ev_copied), "read accumulation");
  return DSPBR_OK;
}

int dspbr_wait(dspbr_ctx* c) {
  if (!c) return DSPBR_ERR_INVALID;
  Status s = c->st();
  int rc = settle(c);
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  TRY_CUDA(s, cudaStreamSynchronize(c->stream), "render");
  if (rc) {
    c->pending = false;
    c->eng->clear_marks();
    return rc;
  }
  if (c->pending) {
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->last_render_ms = ms;
    c->pending = false;
  }
  c->eng->resolve_marks();
  return DSPBR_OK;
}

int dspbr_set_counting(dspbr_ctx* c, int enable) {
  if (!c) return DSPBR_ERR_INVALID;
  Status s = c->st();
  int rc = settle(c);
  if (rc) return rc;
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  TRY_CUDA(s, cudaMemsetAsync(c->eng->stats() + 3, 0, 4 * sizeof(unsigned long long), c->stream), "counters");
  c->counting = enable != 0;
  return DSPBR_OK;
}

int dspbr_set_profiling(dspbr_ctx* c, int enable) {
  if (!c) return DSPBR_ERR_INVALID;
  int rc = dspbr_wait(c);
  if (rc) return rc;
  c->eng->profiling = enable != 0;
  for (double& v : c->eng->kind_ms) v = 0;
  for (auto& v : c->eng->kind_launches) v = 0;
  return DSPBR_OK;
}

int dspbr_render(dspbr_ctx* c, int frames) {
  if (!c) return DSPBR_ERR_INVALID;
  if (c->pipelined && !c->counting && !c->eng->profiling) return render_pipelined(c, frames);
  int rc = enqueue_frames(c, frames, false);
  if (rc) {
    dspbr_wait(c);
    return rc;
  }
  return dspbr_wait(c);
}

int dspbr_render_async(dspbr_ctx* c, int frames) {
  if (!c) return DSPBR_ERR_INVALID;
  return enqueue_frames(c, frames, true);
}

int dspbr_poll(dspbr_ctx* c, int* done) {
  if (!c || !done) return DSPBR_ERR_INVALID;
  if (!c->worker_done.load()) { *done = 0; return DSPBR_OK; }
  if (c->worker.joinable()) c->worker.join();
  cudaSetDevice(c->device);
  cudaError_t e = cudaStreamQuery(c->stream);
  if (e == cudaErrorNotReady) { cudaGetLastError(); *done = 0; return DSPBR_OK; }
  *done = 1;
  if (e != cudaSuccess) return c->st().cuda(e, "render");
  return dspbr_wait(c);
}

// Host copy with several threads: a single thread copies well below the
// host memory bandwidth.
static void parallel_copy(void* dst, const void* src, size_t bytes) {
  const size_t kChunk = size_t(4) << 20;
  unsigned nt = std::min<unsigned>(std::max(1u, std::thread::hardware_concurrency()), 8u);
  if (bytes < 2 * kChunk || nt < 2) {
    std::memcpy(dst, src, bytes);
    return;
  }
  size_t per = (bytes + nt - 1) / nt;
  std::vector<std::thread> th;
  for (unsigned i = 1; i < nt; ++i) {
    size_t o = size_t(i) * per;
    if (o >= bytes) break;
    th.emplace_back([=] { std::memcpy(static_cast<char*>(dst) + o, static_cast<const char*>(src) + o, std::min(per, bytes - o)); });
  }
  std::memcpy(dst, src, std::min(per, bytes));
  for (auto& t : th) t.join();
}

// Device-to-host copy of a result: one DMA into page-locked memory, else
// through the context's page-locked staging buffer and a parallel host copy.
static int copy_out(dspbr_ctx* c, void* dst, const void* src, size_t bytes, const char* what) {
  Status s = c->st();
  cudaPointerAttributes attr{};
  bool pinned = cudaPointerGetAttributes(&attr, dst) == cudaSuccess && attr.type == cudaMemoryTypeHost;
  cudaGetLastError();
  if (pinned) {
    TRY_CUDA(s, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream), what);
    TRY_CUDA(s, cudaStreamSynchronize(c->stream), what);
    return DSPBR_OK;
  }
  if (c->stage_bytes < bytes) {
    if (c->stage) cudaFreeHost(c->stage);
    c->stage = nullptr;
    c->stage_bytes = 0;
    TRY_CUDA(s, cudaHostAlloc(reinterpret_cast<void**>(&c->stage), bytes, cudaHostAllocDefault), "alloc staging");
    c->stage_bytes = bytes;
  }
  TRY_CUDA(s, cudaMemcpyAsync(c->stage, src, bytes, cudaMemcpyDeviceToHost, c->stream), what);
  TRY_CUDA(s, cudaStreamSynchronize(c->stream), what);
  parallel_copy(dst, c->stage, bytes);
  return DSPBR_OK;
}

int dspbr_read_accum(dspbr_ctx* c, float* rgba, size_t num_floats) {
  if (!c || !rgba) return DSPBR_ERR_INVALID;
  { int rc_ = settle(c); if (rc_) return rc_; }
  Status s = c->st();
  size_t npix = size_t(c->width) * c->height;
  if (num_floats < npix * 4) return s.fail(DSPBR_ERR_INVALID, "read_accum: buffer holds %zu floats, need %zu", num_floats, npix * 4);
  if (!c->accum.p) return s.fail(DSPBR_ERR_STATE, "read_accum: no image");
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  double inv = c->sample_count ? 1.0 / double(c->sample_count) : 0.0;
  TRY_CUDA(s, after_pending_copy(c), "read accumulation");
  launch_mean(c->accum.p, inv, c->mean.p, int(npix), c->stream);
  return copy_out(c, rgba, c->mean.p, npix * 16, "read accumulation");
}

int dspbr_read_accum_async(dspbr_ctx* c, float* rgba, size_t num_floats) {
  if (!c || !rgba) return DSPBR_ERR_INVALID;
  { int rc_ = settle_worker(c); if (rc_) return rc_; }
  if (c->pipelined && c->deferred) {  // one deferred read per epoch
    int rc = flush_pipeline(c);
    if (rc) return rc;
  }
  Status s = c->st();
  size_t npix = size_t(c->width) * c->height;
  if (num_floats < npix * 4)
    return s.fail(DSPBR_ERR_INVALID, "read_accum_async: buffer holds %zu floats, need %zu", num_floats, npix * 4);
  if (!c->accum.p) return s.fail(DSPBR_ERR_STATE, "read_accum_async: no image");
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  cudaPointerAttributes attr{};
  const bool pinned = cudaPointerGetAttributes(&attr, rgba) == cudaSuccess && attr.type == cudaMemoryTypeHost;
  cudaGetLastError();
  if (!pinned) return s.fail(DSPBR_ERR_INVALID, "read_accum_async: the buffer is not page-locked (dspbr_host_alloc)");
  if (c->pipelined) {
    // this epoch's last paths are in the pool: the mean and copy follow when
    // they finish (in a later render call, or dspbr_read_wait)
    if (c->tail_live) {
      c->deferred = rgba;
      return DSPBR_OK;
    }
    // its sums are complete: mean and copy on the copy stream, so that the
    // context's stream (the next renders) never waits for a copy
    return issue_read(c, c->accum.p, c->sample_count, rgba, nullptr);
  }
  double inv = c->sample_count ? 1.0 / double(c->sample_count) : 0.0;
  TRY_CUDA(s, after_pending_copy(c), "read accumulation");
  launch_mean(c->accum.p, inv, c->mean.p, int(npix), c->stream);
  TRY_CUDA(s, cudaGetLastError(), "read accumulation");
  TRY_CUDA(s, cudaEventRecord(c->ev_mean, c->stream), "event");
  TRY_CUDA(s, cudaStreamWaitEvent(c->copy_stream, c->ev_mean, 0), "read accumulation");
  TRY_CUDA(s, cudaMemcpyAsync(rgba, c->mean.p, npix * 16, cudaMemcpyDeviceToHost, c->copy_stream), "read accumulation");
  TRY_CUDA(s, cudaEventRecord(c->ev_copied, c->copy_stream), "event");
  c->copy_pending = true;
  return DSPBR_OK;
}

int dspbr_read_wait(dspbr_ctx* c) {
  if (!c) return DSPBR_ERR_INVALID;
  bool deferred = c->deferred != nullptr;
  for (const auto& o : c->older) deferred = deferred || o.deferred;
  if (deferred) {
    int rc = settle(c);  // finishes the epoch and enqueues the read
    if (rc) return rc;
  }
  if (!c->copy_pending) return DSPBR_OK;
  Status s = c->st();
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  c->copy_pending = false;
  TRY_CUDA(s, cudaEventSynchronize(c->ev_copied), "read accumulation");
  return DSPBR_OK;
}

// tonemap (+ FXAA) of the running mean into `out` (float4 or uchar4 per pixel)
// The canvas the display pass draws: true (and its size) when it differs from
// the render resolution.
static bool canvas_size(const dspbr_ctx* c, const dspbr_display* d, int* w, int* h) {
  if (d->canvas_width <= 0 || d->canvas_height <= 0) return false;
  if (d->canvas_width == c->width && d->canvas_height == c->height) return false;
  *w = d->canvas_width;
  *h = d->canvas_height;
  return true;
}

static size_t display_pixels(const dspbr_ctx* c, const dspbr_display* d) {
  int w = 0, h = 0;
  return canvas_size(c, d, &w, &h) ? size_t(w) * h : size_t(c->width) * c->height;
}

static int display_pass(dspbr_ctx* c, const dspbr_display* d, bool bytes8, void** out) {
  Status s = c->st();
  size_t npix = size_t(c->width) * c->height;
  if (!c->accum.p) return s.fail(DSPBR_ERR_STATE, "read_display: no image");
  if (!(d->exposure == d->exposure)) return s.fail(DSPBR_ERR_INVALID, "read_display: exposure is NaN");
  if (d->canvas_width < 0 || d->canvas_height < 0 || (d->canvas_width == 0) != (d->canvas_height == 0) ||
      int64_t(d->canvas_width) * d->canvas_height > (int64_t(1) << 28))
    return s.fail(DSPBR_ERR_INVALID, "read_display: canvas %d x %d", d->canvas_width, d->canvas_height);
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  if (c->display.n < npix) TRY_CUDA(s, c->display.alloc(npix), "alloc display buffer");
  TRY_CUDA(s, after_pending_copy(c), "read display");  // the mean buffer is the epilogue's scratch
  DisplayParams p;
  p.exposure = d->exposure;
  p.mode = d->tonemapping;
  p.gamma = d->gamma != 0;
  const double inv = c->sample_count ? 1.0 / double(c->sample_count) : 0.0;
  float4* f = c->display.p;
  uchar4* b = reinterpret_cast<uchar4*>(c->mean.p);  // the mean buffer holds 16 B per pixel
  if (d->fxaa) {
    launch_tonemap(c->accum.p, inv, p, c->mean.p, int(npix), c->stream);
    if (bytes8) launch_fxaa8(c->mean.p, c->width, c->height, reinterpret_cast<uchar4*>(f), c->stream);
    else launch_fxaa(c->mean.p, c->width, c->height, f, c->stream);
    *out = f;
  } else if (bytes8) {
    launch_tonemap8(c->accum.p, inv, p, b, int(npix), c->stream);
    *out = b;
  } else {
    launch_tonemap(c->accum.p, inv, p, f, int(npix), c->stream);
    *out = f;
  }
  int dw = 0, dh = 0;
  if (canvas_size(c, d, &dw, &dh)) {
    const size_t n = size_t(dw) * dh;
    if (c->present.n < n) TRY_CUDA(s, c->present.alloc(n), "alloc canvas buffer");
    if (bytes8)
      launch_present8(static_cast<const uchar4*>(*out), c->width, c->height,
                      reinterpret_cast<uchar4*>(c->present.p), dw, dh, c->stream);
    else
      launch_present(static_cast<const float4*>(*out), c->width, c->height, c->present.p, dw, dh, c->stream);
    *out = c->present.p;
  }
  return s.cuda(cudaGetLastError(), "display pass");
}

int dspbr_read_display(dspbr_ctx* c, const dspbr_display* d, float* rgba, size_t num_floats) {
  if (!c || !d || !rgba) return DSPBR_ERR_INVALID;
  { int rc_ = settle(c); if (rc_) return rc_; }
  size_t npix = display_pixels(c, d);
  if (num_floats < npix * 4)
    return c->st().fail(DSPBR_ERR_INVALID, "read_display: buffer holds %zu floats, need %zu", num_floats, npix * 4);
  void* src = nullptr;
  int rc = display_pass(c, d, false, &src);
  if (rc) return rc;
  return copy_out(c, rgba, src, npix * 16, "read display");
}

int dspbr_read_display_rgba8(dspbr_ctx* c, const dspbr_display* d, uint8_t* rgba8, size_t num_bytes) {
  if (!c || !d || !rgba8) return DSPBR_ERR_INVALID;
  { int rc_ = settle(c); if (rc_) return rc_; }
  size_t npix = display_pixels(c, d);
  if (num_bytes < npix * 4)
    return c->st().fail(DSPBR_ERR_INVALID, "read_display_rgba8: buffer holds %zu bytes, need %zu", num_bytes, npix * 4);
  void* src = nullptr;
  int rc = display_pass(c, d, true, &src);
  if (rc) return rc;
  return copy_out(c, rgba8, src, npix * 4, "read display");
}

int dspbr_bvh_wide(const float* nodes, uint32_t num_nodes, uint32_t num_indices, uint32_t* num_wide_nodes,
                   uint32_t* num_wide_leaves, int32_t* root, float* wide_nodes, int32_t* wide_leaves) {
  if (!nodes || num_nodes == 0) return DSPBR_ERR_INVALID;
  std::vector<float> conv;
  convert_bvh_nodes(nodes, num_nodes, conv);
  WideBvh wb = collapse_bvh4(conv.data(), num_nodes, num_indices);
  if (num_wide_nodes) *num_wide_nodes = uint32_t(wb.nodes.size());
  if (num_wide_leaves) *num_wide_leaves = uint32_t(wb.leaves.size());
  if (root) *root = wb.root;
  if (wide_nodes && !wb.nodes.empty()) std::memcpy(wide_nodes, wb.nodes.data(), wb.nodes.size() * sizeof(WideNode4));
  if (wide_leaves && !wb.leaves.empty()) std::memcpy(wide_leaves, wb.leaves.data(), wb.leaves.size() * sizeof(WideLeaf));
  return DSPBR_OK;
}

int dspbr_display_image(dspbr_ctx* c, const float* rgba, int w, int h, const dspbr_display* d, float* out_rgba,
                        uint8_t* out_rgba8) {
  if (!c || !rgba || !d || w <= 0 || h <= 0 || int64_t(w) * h > (int64_t(1) << 28)) return DSPBR_ERR_INVALID;
  { int rc_ = settle(c); if (rc_) return rc_; }
  Status s = c->st();
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  const size_t npix = size_t(w) * h;
  // the image as one-sample sums: exactly the floats given (double holds them)
  std::vector<double> sums(npix * 4);
  for (size_t i = 0; i < npix * 4; ++i) sums[i] = double(rgba[i]);
  DevBuf<double4> acc;
  DevBuf<float4> tm, out;
  DevBuf<uchar4> out8;
  TRY_CUDA(s, acc.alloc(npix), "alloc");
  TRY_CUDA(s, tm.alloc(npix), "alloc");
  TRY_CUDA(s, out.alloc(npix), "alloc");
  TRY_CUDA(s, out8.alloc(npix), "alloc");
  TRY_CUDA(s, cudaMemcpyAsync(acc.p, sums.data(), npix * 32, cudaMemcpyHostToDevice, c->stream), "upload");
  DisplayParams p;
  p.exposure = d->exposure;
  p.mode = d->tonemapping;
  p.gamma = d->gamma != 0;
  if (d->fxaa) {
    launch_tonemap(acc.p, 1.0, p, tm.p, int(npix), c->stream);
    if (out_rgba) launch_fxaa(tm.p, w, h, out.p, c->stream);
    if (out_rgba8) launch_fxaa8(tm.p, w, h, out8.p, c->stream);
  } else {
    if (out_rgba) launch_tonemap(acc.p, 1.0, p, out.p, int(npix), c->stream);
    if (out_rgba8) launch_tonemap8(acc.p, 1.0, p, out8.p, int(npix), c->stream);
  }
  TRY_CUDA(s, cudaGetLastError(), "display pass");
  if (out_rgba) TRY_CUDA(s, cudaMemcpyAsync(out_rgba, out.p, npix * 16, cudaMemcpyDeviceToHost, c->stream), "download");
  if (out_rgba8) TRY_CUDA(s, cudaMemcpyAsync(out_rgba8, out8.p, npix * 4, cudaMemcpyDeviceToHost, c->stream), "download");
  return s.cuda(cudaStreamSynchronize(c->stream), "display image");
}

int dspbr_host_alloc(dspbr_ctx* c, size_t bytes, void** out) {
  if (!c || !out || bytes == 0) return DSPBR_ERR_INVALID;
  *out = nullptr;
  Status s = c->st();
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  TRY_CUDA(s, cudaHostAlloc(out, bytes, cudaHostAllocDefault), "host alloc");
  return DSPBR_OK;
}

int dspbr_host_free(dspbr_ctx* c, void* ptr) {
  if (!ptr) return DSPBR_ERR_INVALID;
  cudaError_t e = cudaFreeHost(ptr);
  if (e == cudaSuccess) return DSPBR_OK;
  if (c) return c->st().cuda(e, "host free");
  cudaGetLastError();
  return DSPBR_ERR_CUDA;
}

int dspbr_get_timeline(dspbr_ctx* c, uint32_t max_entries, uint64_t* iteration, uint64_t* t_ns, uint32_t* live,
                       uint32_t* count) {
  if (!c || !count) return DSPBR_ERR_INVALID;
  { int rc_ = settle(c); if (rc_) return rc_; }
  Status s = c->st();
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  std::vector<TimelineEntry> tl;
  int rc = c->eng->timeline(max_entries, tl);
  if (rc) return rc;
  for (size_t k = 0; k < tl.size(); ++k) {
    if (iteration) iteration[k] = tl[k].iteration;
    if (t_ns) t_ns[k] = tl[k].t_ns;
    if (live) live[k] = tl[k].live;
  }
  *count = uint32_t(tl.size());
  return DSPBR_OK;
}

int dspbr_get_device_info(dspbr_ctx* c, dspbr_device_info* info) {
  if (!c || !info) return DSPBR_ERR_INVALID;
  Status s = c->st();
  cudaDeviceProp prop{};
  TRY_CUDA(s, cudaGetDeviceProperties(&prop, c->device), "device properties");
  std::memset(info, 0, sizeof *info);
  std::snprintf(info->name, sizeof info->name, "%s", prop.name);
  info->sm_count = prop.multiProcessorCount;
  info->cc_major = prop.major;
  info->cc_minor = prop.minor;
  info->total_bytes = uint64_t(prop.totalGlobalMem);
  return DSPBR_OK;
}

int dspbr_get_sample_count(dspbr_ctx* c, unsigned long long* count) {
  if (!c || !count) return DSPBR_ERR_INVALID;
  *count = c->sample_count;
  return DSPBR_OK;
}

int dspbr_get_diagnostics(dspbr_ctx* c, dspbr_diag* d) {
  if (!c || !d) return DSPBR_ERR_INVALID;
  // pipelined frames stay in flight: the ray counters cover the iterations run so far
  { int rc_ = settle_worker(c); if (rc_) return rc_; }
  { int rc_ = complete_call(c); if (rc_) return rc_; }
  Status s = c->st();
  std::memset(d, 0, sizeof *d);
  unsigned long long st[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  if (int rc = c->eng->read_stats(st)) return rc;
  d->sample_count = c->sample_count;
  d->width = c->width;
  d->height = c->height;
  d->rays_primary = c->rays_primary;
  d->rays_extension = st[0] >= c->rays_primary ? st[0] - c->rays_primary : 0;
  d->rays_shadow = st[1];
  d->traversal_aborted = st[2];
  if (c->scene) {
    d->scene_triangles = c->scene->num_tris;
    d->bvh_nodes = c->scene->num_nodes;
    d->bvh_indices = c->scene->num_slots;
    d->bvh_build_ms = c->scene->bvh_build_ms;
    d->upload_ms = c->scene->upload_ms;
  }
  d->device_bytes = c->eng->pool_bytes() + c->accum.bytes() + c->mean.bytes();
  for (const auto& m : c->read_mean) d->device_bytes += m.bytes();
  for (const auto& o : c->older) d->device_bytes += o.sums->bytes();
  for (const auto& b : c->spare) d->device_bytes += b->bytes();
  d->last_render_ms = c->last_render_ms;
  d->nodes_closest = st[3];
  d->tris_closest = st[4];
  d->nodes_shadow = st[5];
  d->tris_shadow = st[6];
  d->extend_ms = c->eng->kind_ms[0];
  d->connect_ms = c->eng->kind_ms[1];
  d->shade_ms = c->eng->kind_ms[2];
  d->extend_launches = c->eng->kind_launches[0];
  d->connect_launches = c->eng->kind_launches[1];
  d->shade_launches = c->eng->kind_launches[2];
  d->other_launches = c->eng->kind_launches[3];
  return DSPBR_OK;
}

}  // extern "C"

// ---- kernel-level queries -------------------------------------------------------------------------
template <class T>
static int up(Status& s, DevBuf<T>& d, const T* h, size_t n, cudaStream_t st) {
  int rc = s.cuda(d.alloc(std::max<size_t>(n, 1)), "alloc");
  if (rc) return rc;
  return s.cuda(cudaMemcpyAsync(d.p, h, n * sizeof(T), cudaMemcpyHostToDevice, st), "upload");
}
template <class T>
static int down(Status& s, T* h, const DevBuf<T>& d, size_t n, cudaStream_t st) {
  return s.cuda(cudaMemcpyAsync(h, d.p, n * sizeof(T), cudaMemcpyDeviceToHost, st), "download");
}

extern "C" {

int dspbr_trace_closest(dspbr_ctx* c, const dspbr_scene* sc, const float* rays, uint32_t n, int32_t* tri, float* t,
                        float* uv) {
  if (!c || !sc || !rays || !tri || !t || !uv) return DSPBR_ERR_INVALID;
  { int rc_ = settle(c); if (rc_) return rc_; }
  Status s = c->st();
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  DevBuf<float> r;
  DevBuf<int32_t> dt;
  DevBuf<float> dtt, duv;
  int rc;
  if ((rc = up(s, r, rays, size_t(n) * 8, c->stream)) || (rc = s.cuda(dt.alloc(std::max(n, 1u)), "alloc")) ||
      (rc = s.cuda(dtt.alloc(std::max(n, 1u)), "alloc")) || (rc = s.cuda(duv.alloc(2 * size_t(std::max(n, 1u))), "alloc")))
    return rc;
  DevScene sv = sc->view();
  sv.wide = c->params.traversal == DSPBR_TRAVERSAL_WIDE;
  launch_trace_rays(sv, reinterpret_cast<const float4*>(r.p), n, 0, dt.p, dtt.p,
                    reinterpret_cast<float2*>(duv.p), nullptr, c->stream);
  if ((rc = s.cuda(cudaGetLastError(), "trace")) || (rc = down(s, tri, dt, n, c->stream)) ||
      (rc = down(s, t, dtt, n, c->stream)) || (rc = down(s, uv, duv, 2 * size_t(n), c->stream)))
    return rc;
  return s.cuda(cudaStreamSynchronize(c->stream), "trace");
}

int dspbr_trace_occluded(dspbr_ctx* c, const dspbr_scene* sc, const float* rays, uint32_t n, int32_t* occ) {
  if (!c || !sc || !rays || !occ) return DSPBR_ERR_INVALID;
  { int rc_ = settle(c); if (rc_) return rc_; }
  Status s = c->st();
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  DevBuf<float> r;
  DevBuf<int32_t> o;
  int rc;
  if ((rc = up(s, r, rays, size_t(n) * 8, c->stream)) || (rc = s.cuda(o.alloc(std::max(n, 1u)), "alloc"))) return rc;
  DevScene sv = sc->view();
  sv.wide = c->params.traversal == DSPBR_TRAVERSAL_WIDE;
  launch_trace_rays(sv, reinterpret_cast<const float4*>(r.p), n, 1, nullptr, nullptr, nullptr, o.p,
                    c->stream);
  if ((rc = s.cuda(cudaGetLastError(), "occluded")) || (rc = down(s, occ, o, n, c->stream))) return rc;
  return s.cuda(cudaStreamSynchronize(c->stream), "occluded");
}

int dspbr_bsdf_query(dspbr_ctx* c, const dspbr_scene* sc, uint32_t n, const float* hit, const float* wo,
                     const float* rnd, float* eval4, float* sample10, int32_t* flags) {
  if (!c || !sc || !hit || !wo || !rnd || !eval4 || !sample10 || !flags) return DSPBR_ERR_INVALID;
  { int rc_ = settle(c); if (rc_) return rc_; }
  Status s = c->st();
  if (int64_t(sc->max_tex_id) >= int64_t(sc->num_texinfo))
    return s.fail(DSPBR_ERR_STATE, "bsdf_query: the scene's materials use textures; call dspbr_scene_set_textures");
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  DevBuf<float> dh, dw, dr, de, ds;
  DevBuf<int32_t> df;
  int rc;
  size_t m = std::max(n, 1u);
  if ((rc = up(s, dh, hit, size_t(n) * 20, c->stream)) || (rc = up(s, dw, wo, size_t(n) * 3, c->stream)) ||
      (rc = up(s, dr, rnd, size_t(n) * 4, c->stream)) || (rc = s.cuda(de.alloc(m * 4), "alloc")) ||
      (rc = s.cuda(ds.alloc(m * 10), "alloc")) || (rc = s.cuda(df.alloc(m), "alloc")))
    return rc;
  launch_bsdf_query(sc->view(), n, dh.p, dw.p, dr.p, c->params.profile == DSPBR_PROFILE_LEAN, de.p, ds.p, df.p,
                    c->stream);
  if ((rc = s.cuda(cudaGetLastError(), "bsdf")) || (rc = down(s, eval4, de, size_t(n) * 4, c->stream)) ||
      (rc = down(s, sample10, ds, size_t(n) * 10, c->stream)) || (rc = down(s, flags, df, n, c->stream)))
    return rc;
  return s.cuda(cudaStreamSynchronize(c->stream), "bsdf");
}

int dspbr_ibl_query(dspbr_ctx* c, const dspbr_ibl* e, uint32_t n, const float* r2, const float* dirs, float* sdp4,
                    float* pdf, float* rgb) {
  if (!c || !e || !r2 || !dirs || !sdp4 || !pdf || !rgb) return DSPBR_ERR_INVALID;
  { int rc_ = settle(c); if (rc_) return rc_; }
  Status s = c->st();
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  DevBuf<float> dr, dd, ds, dp, dc;
  size_t m = std::max(n, 1u);
  int rc;
  if ((rc = up(s, dr, r2, size_t(n) * 2, c->stream)) || (rc = up(s, dd, dirs, size_t(n) * 3, c->stream)) ||
      (rc = s.cuda(ds.alloc(m * 4), "alloc")) || (rc = s.cuda(dp.alloc(m), "alloc")) ||
      (rc = s.cuda(dc.alloc(m * 3), "alloc")))
    return rc;
  float rot = float(double(c->params.ibl_rotation_deg) / 180.0 * M_PI);
  launch_ibl_query(e->view(), rot, c->params.env_sampling == DSPBR_ENV_CDF ? 1 : 0, n, dr.p, dd.p, ds.p, dp.p, dc.p,
                   c->stream);
  if ((rc = s.cuda(cudaGetLastError(), "ibl query")) || (rc = down(s, sdp4, ds, size_t(n) * 4, c->stream)) ||
      (rc = down(s, pdf, dp, n, c->stream)) || (rc = down(s, rgb, dc, size_t(n) * 3, c->stream)))
    return rc;
  return s.cuda(cudaStreamSynchronize(c->stream), "ibl query");
}

int dspbr_camera_rays(dspbr_ctx* c, uint32_t n, const int32_t* xy, const float* r2, float* rays6) {
  if (!c || !xy || !r2 || !rays6) return DSPBR_ERR_INVALID;
  { int rc_ = settle(c); if (rc_) return rc_; }
  Status s = c->st();
  if (!c->has_camera || c->width <= 0) return s.fail(DSPBR_ERR_STATE, "camera_rays: camera and size required");
  TRY_CUDA(s, cudaSetDevice(c->device), "cudaSetDevice");
  DevBuf<int32_t> dxy;
  DevBuf<float> dr, dout;
  int rc;
  if ((rc = up(s, dxy, xy, size_t(n) * 2, c->stream)) || (rc = up(s, dr, r2, size_t(n) * 2, c->stream)) ||
      (rc = s.cuda(dout.alloc(std::max(n, 1u) * size_t(6)), "alloc")))
    return rc;
  WaveParams p = make_wave(c, 1);
  launch_camera_rays(p.cam, n, dxy.p, dr.p, dout.p, c->stream);
  if ((rc = s.cuda(cudaGetLastError(), "camera rays")) || (rc = down(s, rays6, dout, size_t(n) * 6, c->stream)))
    return rc;
  return s.cuda(cudaStreamSynchronize(c->stream), "camera rays");
}

}  // extern "C"
