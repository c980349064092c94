// Internal definitions of the C ABI's opaque handles, shared by the context
// API (api.cu) and the server (server.cu).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "dspbr.h"
#include "engine.h"
#include "host.h"
#include "kernels.h"

struct dspbr_scene {
  dspbr_ctx* ctx = nullptr;
  dspbr::DevBuf<float4> nodes, tris, verts, materials;
  dspbr::DevBuf<uint32_t> indices;
  dspbr::DevBuf<uint8_t> tri_class;
  dspbr::DevBuf<float4> wnodes;  // 4-wide BVH (8 float4 per node)
  dspbr::DevBuf<int2> wleaves;
  int wroot = 0;
  uint32_t num_wnodes = 0;  // wide nodes in use
  // compressed 8-wide BVH (bvh_gpu.h DeviceCw8), empty when the 4-wide one serves
  dspbr::DevBuf<uint4> cnodes;
  dspbr::DevBuf<float4> ctris;
  uint32_t num_cnodes = 0, num_crecs = 0, cw8_levels = 0;
  double refit_ms = 0.0;    // the last dspbr_scene_update_vertices
  dspbr::DevBuf<int32_t> device_remap;  // leaf-slot remap of a device-built BVH
  // material textures
  std::vector<std::unique_ptr<dspbr::DevBuf<uchar4>>> tex_data;
  dspbr::DevBuf<dspbr::DevTexArray> tex_arrays;
  dspbr::DevBuf<float4> texinfo;
  uint32_t num_texinfo = 0, num_tex_arrays = 0;
  int32_t max_tex_id = -1;  // largest texture id the materials use
  uint32_t num_nodes = 0, num_slots = 0, num_tris = 0, num_verts = 0, num_materials = 0;
  std::vector<uint32_t> tri_material;  // host copy, for re-classing after material edits
  std::vector<float> host_materials;
  uint32_t num_classes = 0;
  bool boxes_finite = true;
  double bvh_build_ms = 0, upload_ms = 0;
  dspbr::DevScene view() const {
    dspbr::DevScene s;
    s.nodes = nodes.p; s.tris = tris.p; s.verts = verts.p; s.indices = indices.p; s.materials = materials.p;
    s.num_nodes = int(num_nodes); s.num_slots = int(num_slots); s.num_tris = int(num_tris);
    s.num_materials = int(num_materials);
    s.tri_class = tri_class.p;
    s.wnodes = wnodes.p;
    s.wleaves = wleaves.p;
    s.wroot = wroot;
    s.cnodes = num_cnodes ? cnodes.p : nullptr;
    s.ctris = num_cnodes ? ctris.p : nullptr;
    s.wide = 1;
    s.texinfo = texinfo.p;
    s.tex_arrays = tex_arrays.p;
    s.num_texinfo = int(num_texinfo);
    s.num_tex_arrays = int(num_tex_arrays);
    s.boxes_finite = boxes_finite ? 1 : 0;
    return s;
  }
  uint64_t bytes() const {
    return nodes.bytes() + tris.bytes() + verts.bytes() + materials.bytes() + indices.bytes() + tri_class.bytes() +
           wnodes.bytes() + wleaves.bytes() + cnodes.bytes() + ctris.bytes() + device_remap.bytes() + texinfo.bytes() + tex_arrays.bytes() +
           tex_bytes();
  }
  uint64_t tex_bytes() const {
    uint64_t b = 0;
    for (auto& t : tex_data) b += t->bytes();
    return b;
  }
};

struct dspbr_ibl {
  dspbr_ctx* ctx = nullptr;
  dspbr::DevBuf<float4> rgba;
  dspbr::DevBuf<float> pdf, cdf, ypdf, ycdf, alias_prob, lum, rowsum;
  dspbr::DevBuf<int> alias_idx;
  dspbr::DevBuf<double> total;
  double total_sum = 0;
  int w = 0, h = 0;
  dspbr::DevIbl view() const {
    dspbr::DevIbl e;
    e.rgba = rgba.p; e.pdf = pdf.p; e.cdf = cdf.p; e.ypdf = ypdf.p; e.ycdf = ycdf.p;
    e.alias_prob = alias_prob.p; e.alias_idx = alias_idx.p; e.w = w; e.h = h;
    return e;
  }
};

struct dspbr_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::string err;
  dspbr_params params{};
  float matrix[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
  float fov = 45.f, near_plane = 0.01f;
  bool has_camera = false;
  int width = 0, height = 0;
  dspbr_scene* scene = nullptr;
  dspbr_ibl* ibl = nullptr;
  // paths per wave: of 2^22..2^24 the large workload's frames per second over
  // long calls rise with the pool (2^22: -5%, 2^23: -2% against 2^24; ~4.4 GB)
  uint32_t wave_paths = 1u << 24;
  // for scenes created without a BVH: the binned SAH on the device, which
  // builds the host builder's tree (47-132 ms against ~430 ms on the host for
  // 1.15M triangles)
  int bvh_builder = DSPBR_BVH_BUILD_DEVICE;
  // width of the wide BVH the path kernels trace: 4 (float boxes) or 8 (quantised boxes)
  int wide_bvh = 4;
  std::unique_ptr<dspbr::Engine> eng;  // path pool + job table; this context's render is job slot 0
  // render_async: the iteration loop runs on a worker thread
  std::thread worker;
  std::atomic<bool> worker_done{true};
  int worker_rc = 0;
  dspbr::DevBuf<double4> accum;
  dspbr::DevBuf<float4> mean;
  dspbr::DevBuf<float4> display;  // display epilogue output (allocated on first use)
  dspbr::DevBuf<float4> present;  // canvas-size output of the display pass (allocated on first use)
  float* stage = nullptr;  // page-locked staging for readback into pageable memory
  size_t stage_bytes = 0;
  // read_accum_async: the mean is computed on `stream`, copied on `copy_stream`
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_mean = nullptr, ev_copied = nullptr;
  bool copy_pending = false;
  // issue_read: the mean of an accumulation runs on mean_stream into one of
  // kReadRing buffers in turn, its device-to-host copy on copy_stream; a mean
  // waits only for its own inputs and for the copy that last used its buffer,
  // never behind other copies.  ev_meaned: the latest such mean (what next
  // writes the sums it read waits for that, not for the copy).
  static constexpr int kReadRing = 3;
  cudaStream_t mean_stream = nullptr;
  dspbr::DevBuf<float4> read_mean[kReadRing];
  cudaEvent_t ev_read_copied[kReadRing] = {};
  bool read_used[kReadRing] = {};
  int read_next = 0;
  cudaEvent_t ev_meaned = nullptr;
  bool mean_pending = false;
  uint64_t sample_count = 0;
  uint64_t rays_primary = 0;
  double last_render_ms = 0;
  bool pending = false;
  bool counting = false;
  // Pipelined frames (dspbr_set_pipelining).  The frames since the last reset
  // (an accumulation epoch) render as job `slot` into `accum`; a render call
  // returns once every sample has started, so the epoch's last paths may still
  // be in the pool (tail_live).  A reset then moves the epoch to `older` (its
  // sums, job slot and any deferred read) and starts a new one in a free job
  // slot and sum buffer.  At most `depth` epochs are in flight: a render call
  // that finds depth - 1 older epochs waits for the oldest before it returns.
  bool pipelined = false;
  static constexpr int kMaxDepth = 16;
  int depth = 2;
  int slot = 0;
  bool tail_live = false;
  struct Older {
    std::unique_ptr<dspbr::DevBuf<double4>> sums;
    uint64_t samples = 0;
    int slot = 0;
    float* deferred = nullptr;  // a read_accum_async requested while it was in flight
  };
  std::vector<Older> older;                                    // oldest first, each with paths in the pool
  std::vector<std::unique_ptr<dspbr::DevBuf<double4>>> spare;  // sum buffers of finished epochs
  // a read_accum_async of the current epoch while it has paths in the pool:
  // its mean and copy are enqueued once the epoch has finished
  float* deferred = nullptr;
  cudaEvent_t ev_between = nullptr;
  cudaEvent_t ev_retired = nullptr;  // a render call's start: the epochs retired before it are complete
  // A pipelined render call returns once its loop launches are enqueued; the
  // next call that needs the pool's state waits for them (complete_call):
  // the iteration counter before them, the loop launches, the job slot the
  // call waited for (-1: none) and its epoch's slot.  Until then tail_live
  // is assumed.
  bool call_inflight = false;
  unsigned long long call_it0 = 0;
  int call_loops = 0, call_wait = -1, call_slot = 0;
  dspbr::Status st() { return dspbr::Status{&err}; }
};


namespace dspbr {
// Uniform block values of one job from the renderer settings and camera
// (renderer.ts:399-431 updatePathracingUniforms).
WaveParams make_job_params(const dspbr_params& q, const float matrix[16], float fov, float near_plane, int width,
                           int height, bool has_ibl, uint32_t frame_base);
}  // namespace dspbr
