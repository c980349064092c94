/*
 * dspbr.h — C ABI of the B200 path-tracing library (libdspbr_cuda.so).
 *
 * Drop-in boundary for the hot path of dspbr-pt's PathtracingViewport /
 * PathtracingRenderer (packages/lib/pathtracing_viewport.ts:100-342,
 * packages/lib/renderer.ts:116-1109).  Each entry point names the reference
 * interface it replaces.  Conventions:
 *   - every call returns an int status: DSPBR_OK (0) or a negative DSPBR_ERR_*;
 *     dspbr_last_error() gives the message of the last failure on a context;
 *   - handles are opaque; all host buffers passed in are copied (the caller
 *     keeps ownership, like the reference's typed arrays -> GL textures);
 *   - one context per host thread (a context is not internally locked);
 *   - data formats are the reference's: 20-float vertex records
 *     (scene_data.ts:21, scene_loader.ts:296-344), uint32 triangle indices,
 *     68-float material records (material.ts:2-481), the binary BVH node
 *     layout of bvh.glsl:1-6 (16 floats per node) and RGBA32F environment maps.
 */
#ifndef DSPBR_H
#define DSPBR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  DSPBR_OK = 0,
  DSPBR_ERR_INVALID = -1,     /* bad argument or malformed input data */
  DSPBR_ERR_CUDA = -2,        /* CUDA runtime error (message in dspbr_last_error) */
  DSPBR_ERR_OOM = -3,         /* device allocation failed */
  DSPBR_ERR_STATE = -4,       /* missing scene/IBL/camera, or a render in flight */
  DSPBR_ERR_ADMISSION = -5,   /* serving: request refused by the HBM budget */
  DSPBR_ERR_NOT_FOUND = -6,   /* serving: unknown request id */
  DSPBR_ERR_DEVICE_FAULT = -7 /* a kernel reported a bounded-wait / traversal abort status */
};

enum { DSPBR_PROFILE_FULL = 0, DSPBR_PROFILE_LEAN = 1 };
enum { DSPBR_RNG_MWC = 0, DSPBR_RNG_PCG = 1 };
enum { DSPBR_TRAVERSAL_WIDE = 0, DSPBR_TRAVERSAL_REFERENCE = 1 };
enum { DSPBR_BVH_BUILD_HOST = 0, DSPBR_BVH_BUILD_DEVICE = 1, DSPBR_BVH_BUILD_DEVICE_LBVH = 2 };
enum { DSPBR_ENV_ALIAS = 0, DSPBR_ENV_CDF = 1 };

typedef struct dspbr_ctx dspbr_ctx;
typedef struct dspbr_scene dspbr_scene;
typedef struct dspbr_ibl dspbr_ibl;
typedef struct dspbr_bvh dspbr_bvh;
typedef struct dspbr_server dspbr_server;

/* Renderer settings: the uniform block of renderer.frag:10-31 plus the setters
 * of renderer.ts:172-306 (defaults in dspbr_params_default). */
typedef struct dspbr_params {
  int32_t max_bounces;            /* u_max_bounces, renderer.ts:229 (8) */
  int32_t use_ibl;                /* u_use_ibl, renderer.ts:238 (1) */
  float ibl_rotation_deg;         /* iblRotation, renderer.ts:265-271 (0) */
  int32_t background_from_ibl;    /* showBackground -> u_background_from_ibl (1) */
  float background_color[4];      /* u_background_color, renderer.ts:282 (0,0,0,1) */
  float ray_eps;                  /* u_ray_eps, renderer.ts:290 (1e-4) */
  float clamp_threshold;          /* u_clamp_threshold, renderer.ts:299 (3.0) */
  float point_light_position[4];  /* u_point_light_position, w>0.5 enables (renderer.ts:422-424) */
  float point_light_emission[4];  /* u_point_light_emission */
  int32_t rr_start_depth;         /* RR_START_DEPTH, constants.glsl:19 (2) */
  float rr_termination_prob;      /* RR_TERMINATION_PROB, constants.glsl:20 (0.1) */
  int32_t profile;                /* DSPBR_PROFILE_*: material kernel profile (renderer.ts:154, 1078-1080) */
  int32_t rng;                    /* DSPBR_RNG_MWC = rng.glsl sequence; DSPBR_RNG_PCG = PCG32 per pixel/sample */
  uint64_t seed;                  /* PCG seed */
  int32_t env_sampling;           /* DSPBR_ENV_ALIAS (O(1), same pmf) or DSPBR_ENV_CDF (reference's binary search) */
  int32_t traversal;              /* DSPBR_TRAVERSAL_WIDE (4-wide BVH collapsed from the binary one) or
                                     DSPBR_TRAVERSAL_REFERENCE (the binary traversal of bvh.glsl:149-229, bit for bit) */
  int32_t reserved[6];
} dspbr_params;

/* PathtracingRendererDiagnostics (renderer.ts:79-110) plus throughput counters. */
typedef struct dspbr_diag {
  uint64_t sample_count;          /* frames accumulated since the last reset */
  int32_t width, height;
  uint64_t rays_primary, rays_extension, rays_shadow; /* since context creation */
  uint64_t traversal_aborted;     /* rays that hit MAX_BVH_TRAVERSAL_STEPS (bvh.glsl:9) */
  uint64_t scene_triangles, bvh_nodes, bvh_indices;
  uint64_t device_bytes;          /* device memory held by the context's own buffers */
  double last_render_ms;          /* device time of the last dspbr_render call */
  double bvh_build_ms, upload_ms; /* set-up profiling, renderer.ts:930-958 */
  /* with dspbr_set_counting(ctx, 1): traversal work since counting was enabled */
  uint64_t nodes_closest, tris_closest, nodes_shadow, tris_shadow;
  /* with dspbr_set_profiling(ctx, 1): device time per kernel kind (CUDA events
   * on the render stream) and launch counts since profiling was enabled */
  double extend_ms, connect_ms, shade_ms;
  uint64_t extend_launches, connect_launches, shade_launches, other_launches;
} dspbr_diag;

void dspbr_params_default(dspbr_params* p);

/* ---- context: replaces new PathtracingRenderer (renderer.ts:309-325) ----- */
int dspbr_create(int device, dspbr_ctx** out);
int dspbr_destroy(dspbr_ctx* ctx);
int dspbr_last_error(const dspbr_ctx* ctx, char* buf, size_t size);
int dspbr_device_count(int* count);

/* ---- BVH: replaces the TinyBVH module ABI (tinybvh_builder.ts:7-24) ------ */
/* _build_bvh_indexed: positions = float records with `vertex_stride_floats`
 * stride (3 for a packed float3 buffer, 20 for the reference vertex record). */
int dspbr_bvh_build(const float* positions, uint32_t num_vertices, uint32_t vertex_stride_floats,
                    const uint32_t* indices, uint32_t num_indices, dspbr_bvh** out);
/* _get_bvh_node_count / _get_bvh_indices_len / _get_bvh_depth / _get_bvh_triangle_count */
int dspbr_bvh_info(const dspbr_bvh* bvh, uint32_t* num_nodes, uint32_t* num_indices, uint32_t* depth,
                   uint32_t* num_triangles);
/* _get_bvh_nodes_ptr / _get_bvh_indices_ptr: copies 16*num_nodes floats and num_indices ints. */
int dspbr_bvh_copy(const dspbr_bvh* bvh, float* nodes, int32_t* indices);
/* _get_last_error_ptr / _get_last_error_len */
int dspbr_bvh_error(const dspbr_bvh* bvh, char* buf, size_t size);
/* The 4-wide BVH the path kernels traverse (DSPBR_TRAVERSAL_WIDE), collapsed
 * from a reference-layout BVH (16 floats per node): 32 words per wide node
 * (float lo_x[4], lo_y[4], lo_z[4], hi_x[4], hi_y[4], hi_z[4]; int child[4];
 * int count, pad[3]; child >= 0 wide node, < 0 ~leaf) and 2 ints per leaf
 * (leaf-slot range [begin, end)).  root >= 0: wide node; < 0: ~leaf.  Call
 * with NULL outputs for the sizes.  No context needed (host only). */
int dspbr_bvh_wide(const float* nodes, uint32_t num_nodes, uint32_t num_indices, uint32_t* num_wide_nodes,
                   uint32_t* num_wide_leaves, int32_t* root, float* wide_nodes, int32_t* wide_leaves);
void dspbr_bvh_free(dspbr_bvh* bvh);

/* ---- scene: replaces PathtracingSceneDataWebGL2.init + initBvh
 *      (scene_data_webgl2.ts:74-100, renderer.ts:872-912) ----------------- */
/* bvh_nodes/bvh_indices may be NULL: the BVH is then built here, by the
 * builder dspbr_set_bvh_builder selects:
 *   DSPBR_BVH_BUILD_HOST         binned SAH on the host (TinyBVH's role);
 *   DSPBR_BVH_BUILD_DEVICE       binned SAH on the device with the host
 *                                builder's rules, level by level, and the
 *                                4-wide collapse on the device (default: the
 *                                host builder's tree, built faster);
 *   DSPBR_BVH_BUILD_DEVICE_LBVH  linear BVH on the device (Morton order, radix
 *                                tree, leaves of <= 4 triangles): the fastest
 *                                build, somewhat slower to trace. */
int dspbr_scene_create(dspbr_ctx* ctx, const float* vertices, uint32_t num_vertices, const uint32_t* indices,
                       uint32_t num_indices, const float* materials, uint32_t num_materials,
                       const float* bvh_nodes, uint32_t num_bvh_nodes, const int32_t* bvh_indices,
                       uint32_t num_bvh_indices, dspbr_scene** out);
/* material edits (dirty materials re-uploaded, renderer.ts:440-448) */
int dspbr_set_bvh_builder(dspbr_ctx* ctx, int builder);
/* The wide BVH that the path kernels (and dspbr_trace_* with the wide
 * traversal) use for scenes created after the call; 4 or 8:
 *   4  4-wide nodes of 128 B with the binary tree's float boxes (default);
 *   8  compressed 8-wide nodes of 80 B: per axis a float origin and a
 *      power-of-two step, per child six 8-bit planes chosen on or outside its
 *      exact box, and each leaf's exact box in a record ahead of its
 *      triangles (published as compressed wide BVHs, Ylitie, Karras and Laine,
 *      HPG 2017; the reference's TinyBVH offers such a layout as BVH8_CWBVH).
 * The closest t equals the binary traversal's except for ties within
 * rounding between coplanar faces (t differing by an ulp), where the face
 * found first is kept.  Scenes whose tree cannot be compressed (a leaf root,
 * non-finite boxes) keep the 4-wide tree. */
int dspbr_set_wide_bvh(dspbr_ctx* ctx, int width);
/* The wide BVH a scene's path kernels use: width 4 or 8, its node count and,
 * for the 8-wide tree, its depth in levels (0 otherwise). */
int dspbr_scene_wide_bvh(const dspbr_scene* scene, int* width, uint32_t* nodes, uint32_t* levels);
/* Material textures (scene_data.ts:71-100, scene_data_webgl2.ts:233-363):
 * textures of one resolution form an RGBA8 texture array sampled LINEAR +
 * REPEAT; tex_infos holds 8 floats per texture reference (TexInfo,
 * material.ts:483-523: offset.xy, array index, layer, scale.xy, uv set, pad),
 * the ids the material records' texture slots name.  Every id a material uses
 * must be below num_tex_infos; a scene whose materials use textures renders
 * only once this was called.  The data is copied. */
typedef struct dspbr_texture_array {
  int32_t width, height, layers;
  const uint8_t* rgba8;       /* layers x height x width x 4 bytes, row 0 first */
} dspbr_texture_array;
int dspbr_scene_set_textures(dspbr_scene* scene, const float* tex_infos, uint32_t num_tex_infos,
                             const dspbr_texture_array* arrays, uint32_t num_arrays);
/* The scene's binary BVH in the reference layout (16 floats per node, child /
 * count / first as floats) and its leaf-slot remap; NULL arrays query the sizes. */
int dspbr_scene_bvh(const dspbr_scene* scene, float* nodes, int32_t* remap, uint32_t* num_nodes,
                    uint32_t* num_indices);
int dspbr_scene_update_materials(dspbr_scene* scene, const float* materials, uint32_t first, uint32_t count);
/* Moves vertices [first, first + count) to new 20-float records (same
 * triangles): the BVH keeps its topology and its boxes are refitted on the
 * device, bottom-up from the leaves' triangles (the binary tree of
 * dspbr_scene_bvh and the 4-wide tree of the path kernels), then the
 * leaf-ordered triangle records are gathered again; a compressed 8-wide tree
 * (dspbr_set_wide_bvh) is built again from the refitted binary tree.  New: the reference
 * rebuilds its BVH on every setScene (tinybvh_builder.ts:43-256); a refit is
 * the animated-geometry step of a device BVH.  Resets the accumulation of the
 * scene's context; not while a server request renders the scene.  Shading
 * classes stay those of the creation (they only group hits for speed). */
int dspbr_scene_update_vertices(dspbr_scene* scene, const float* vertices, uint32_t first, uint32_t count);
int dspbr_scene_device_bytes(const dspbr_scene* scene, uint64_t* bytes);
int dspbr_scene_destroy(dspbr_scene* scene);

/* ---- IBL: replaces setIBL + precomputeIBLImportanceSamplingData
 *      (renderer.ts:777-865).  Tables are built on the device: FP64 prefix
 *      sums stored as float32 (the reference's Float32Array), plus an alias
 *      table over the same pmf. ------------------------------------------- */
int dspbr_ibl_create(dspbr_ctx* ctx, const float* rgba32f, int width, int height, dspbr_ibl** out);
/* copies back pdf (w*h), cdf (w*h), yPdf (h), yCdf (h), totalSum */
int dspbr_ibl_tables(const dspbr_ibl* ibl, float* pdf, float* cdf, float* ypdf, float* ycdf, double* total_sum);
/* alias table: prob (w*h float) and alias (w*h int32) */
int dspbr_ibl_alias_table(const dspbr_ibl* ibl, float* prob, int32_t* alias);
int dspbr_ibl_destroy(dspbr_ibl* ibl);
/* Allocation-free table build.  No counterpart in the reference: it exists for
 * hosts that cannot let a library call cudaMalloc (an engine that owns all
 * device memory through its own pool, or a frame loop that must not take the
 * implicit device synchronisation of cudaMalloc / cudaFree).  It writes the
 * same pdf, cdf, yPdf, yCdf and totalSum as dspbr_ibl_create into buffers the
 * caller allocated: every pointer is device memory of the current device
 * (rgba32f w*h*4 floats, pdf and cdf w*h floats, ypdf and ycdf h floats, one
 * double), and the work is enqueued on `stream` (a cudaStream_t, NULL for the
 * default stream) without synchronising.  Scratch is a fixed 64 KiB device
 * array inside the library, so height is limited to 16384 rows; larger maps
 * are refused with DSPBR_ERR_INVALID.  rgba32f must be 16-byte aligned,
 * total_sum 8-byte aligned and the four tables 4-byte aligned (else
 * DSPBR_ERR_INVALID).  The first call on a device looks up that array's
 * address and keeps it, so make it before any stream capture, and do not call
 * this entry point after a cudaDeviceReset of that device in the same process.
 * All calls share the array: calls that overlap on the GPU race on it.  With
 * no context to hold a message, errors are reported on stderr, not through
 * dspbr_last_error. */
int dspbr_ibl_tables_noalloc(const float* rgba32f, int width, int height, float* pdf, float* cdf, float* ypdf,
                             float* ycdf, double* total_sum, void* stream);

/* ---- viewport state (pathtracing_viewport.ts:147-291) -------------------- */
int dspbr_set_scene(dspbr_ctx* ctx, dspbr_scene* scene);          /* setScene */
int dspbr_set_ibl(dspbr_ctx* ctx, dspbr_ibl* ibl);                /* setIBL */
/* setCamera: matrixWorld column-major 16 floats (camera-to-world), vertical fov
 * in degrees, near plane (renderer.ts:399-404) */
int dspbr_set_camera(dspbr_ctx* ctx, const float matrix_world[16], float fov_deg, float near_plane);
int dspbr_set_params(dspbr_ctx* ctx, const dspbr_params* params); /* setSettings */
int dspbr_get_params(const dspbr_ctx* ctx, dspbr_params* params);
int dspbr_resize(dspbr_ctx* ctx, int width, int height);          /* resize */
int dspbr_reset(dspbr_ctx* ctx);                                  /* resetAccumulation */
/* start(sampleLimit) driven synchronously: renders `frames` progressive frames
 * (1 sample per pixel each) and returns when they are on the device. */
int dspbr_render(dspbr_ctx* ctx, int frames);
/* asynchronous variant: enqueue and return; dspbr_poll reports completion */
int dspbr_render_async(dspbr_ctx* ctx, int frames);
int dspbr_poll(dspbr_ctx* ctx, int* done);
int dspbr_wait(dspbr_ctx* ctx);
/* readAccumulation (absent in the reference, which only displays): running
 * mean RGBA32F, width*height*4 floats, row 0 = bottom row (gl_FragCoord.y 0.5). */
int dspbr_read_accum(dspbr_ctx* ctx, float* rgba, size_t num_floats);
/* Pipelined readAccumulation: enqueues the running mean of the frames rendered
 * so far and its device-to-host copy (on a copy stream of the context), and
 * returns.  The next render can start at once and overlaps the copy.  `rgba`
 * is page-locked (dspbr_host_alloc; else DSPBR_ERR_INVALID) and is complete
 * when dspbr_read_wait returns.  Later calls that write the mean (another
 * read, a display read, a resize) are ordered after the pending copy. */
int dspbr_read_accum_async(dspbr_ctx* ctx, float* rgba, size_t num_floats);
int dspbr_read_wait(dspbr_ctx* ctx);
/* Pipelined frames (off by default).  The reference renders one frame per
 * requestAnimationFrame and presents it (renderer.ts:512-565, 595-714); here
 * the frames of consecutive accumulations overlap on the device.  With it on,
 * dspbr_render enqueues the render loop until every sample of its frames has
 * started and returns without waiting for it: the host prepares the next
 * frame while the device runs, the last paths stay in the path pool and
 * finish during the next dspbr_render, which first completes the previous
 * accumulation.  A device error of the loop is reported by the next call
 * that waits for it (render, reads, diagnostics).  A reset (setCamera, setSettings,
 * resetAccumulation) starts the new accumulation in a second sum buffer while
 * the old one finishes.  dspbr_read_accum_async of an accumulation still in
 * flight is enqueued when its paths finish (during the next render, or in
 * dspbr_read_wait); dspbr_read_accum, the display reads and every other call
 * finish all paths first.  Images are the same as with it off. */
int dspbr_set_pipelining(dspbr_ctx* ctx, int enable);
/* Accumulations in flight with pipelined frames: 2 (default) to 16.  A
 * render call that finds depth - 1 earlier accumulations with paths in the
 * pool waits only for the oldest: a caller that takes frame k's image while
 * frame k + depth - 1 renders (a render-ahead queue, dspbr_read_wait_ready)
 * keeps the pool fuller, and each call runs fewer, fuller iterations.  Each
 * accumulation in flight holds a sum buffer (32 bytes per pixel).  Images are
 * the same. */
int dspbr_set_pipeline_depth(dspbr_ctx* ctx, int depth);
/* Waits for the device-to-host copies enqueued so far (reads of
 * accumulations that have finished) and returns in *in_flight the number of
 * reads still deferred because their accumulation has paths in the pool; it
 * renders nothing, unlike dspbr_read_wait, which finishes them all. */
int dspbr_read_wait_ready(dspbr_ctx* ctx, int* in_flight);
/* Display epilogue (renderer.ts:666-700): the accumulation mean through
 * tonemap.frag (exposure, operator, gamma) and optionally fxaa.frag -- the
 * reference's "postprocess" buffer, at the render resolution -- as RGBA32F,
 * or converted to the 8-bit canvas bytes.  With a canvas size set, the output
 * is the canvas instead: display.frag's nearest-neighbour draw of the
 * postprocess buffer at that size (renderer.ts:689-697), which is how the
 * reference presents a render resolution scaled by pixelRatio
 * (renderer.ts:365-372); the output buffer then holds canvas_width *
 * canvas_height pixels. */
typedef struct dspbr_display {
  float exposure;             /* renderer.ts `exposure` (1.0) */
  int tonemapping;            /* DSPBR_TONEMAP_*: renderer.ts tonemappingModes index */
  int gamma;                  /* enableGamma: pow(c, 1/2.2) */
  int fxaa;                   /* enableFxaa */
  int canvas_width;           /* displayRes; 0 (or both equal to the render size): no resampling */
  int canvas_height;
  int reserved[2];
} dspbr_display;
enum {
  DSPBR_TONEMAP_OFF = -1,     /* a mode name not in tonemappingModes: no operator, no exposure */
  DSPBR_TONEMAP_NONE = 0,     /* "None": exposure only */
  DSPBR_TONEMAP_REINHARD = 1,
  DSPBR_TONEMAP_CINEON = 2,
  DSPBR_TONEMAP_ACES = 3,     /* "AcesFilm" */
  DSPBR_TONEMAP_UNCHARTED2 = 4
};
int dspbr_read_display(dspbr_ctx* ctx, const dspbr_display* display, float* rgba, size_t num_floats);
int dspbr_read_display_rgba8(dspbr_ctx* ctx, const dspbr_display* display, uint8_t* rgba8, size_t num_bytes);
/* The same epilogue on a caller's RGBA32F image (width*height*4 floats), for
 * hosts that accumulate elsewhere; either output may be NULL. */
int dspbr_display_image(dspbr_ctx* ctx, const float* rgba, int width, int height, const dspbr_display* display,
                        float* out_rgba, uint8_t* out_rgba8);
/* Page-locked host memory for readback buffers.  dspbr_read_accum into such
 * a buffer is one device-to-host DMA; into ordinary memory it goes through an
 * internal page-locked staging buffer.  dspbr_host_free accepts ctx == NULL
 * (for buffers that outlive their context). */
int dspbr_host_alloc(dspbr_ctx* ctx, size_t bytes, void** out);
int dspbr_host_free(dspbr_ctx* ctx, void* ptr);
int dspbr_get_diagnostics(dspbr_ctx* ctx, dspbr_diag* diag);
/* Samples per pixel of the current accumulation handed to render calls so
 * far (diag.sample_count), read without waiting for the device: the
 * progressive loop's counter (renderer.ts frameCount), which lets a
 * pipelined render call's loop run while the caller prepares the next one. */
int dspbr_get_sample_count(dspbr_ctx* ctx, unsigned long long* count);
/* The context's GPU (diagnostics.backend's counterpart, renderer.ts:79-110):
 * name, SM count, compute capability, device memory; keys per-GPU caches
 * such as the autotuner's. */
typedef struct dspbr_device_info {
  char name[256];
  int sm_count, cc_major, cc_minor;
  uint64_t total_bytes;
} dspbr_device_info;
int dspbr_get_device_info(dspbr_ctx* ctx, dspbr_device_info* info);
/* The last iterations of the path engine (at most max_entries, at most 1024),
 * oldest first: iteration number, device clock (ns) at its end and the paths
 * queued for the next one.  New: the reference renders one full-screen pass
 * per frame and has no iterations to report (renderer.ts:512-565). */
int dspbr_get_timeline(dspbr_ctx* ctx, uint32_t max_entries, uint64_t* iteration, uint64_t* t_ns, uint32_t* live,
                       uint32_t* count);
/* paths per wave (0 = default 2^24); the wave covers min(frames, paths/pixels)
 * samples of every pixel.  Set by the autotuner. */
int dspbr_set_wave_paths(dspbr_ctx* ctx, uint32_t paths);
/* live paths below which a render call, once every sample has started,
 * finishes the remaining paths in one launch (each path run to its end by
 * one thread) instead of more wavefront iterations.  0 = the default. */
int dspbr_set_drain_threshold(dspbr_ctx* ctx, uint32_t paths);
/* count BVH node visits and triangle tests of every traced ray (diagnostics) */
int dspbr_set_counting(dspbr_ctx* ctx, int enable);
/* time every extend / connect / shade launch with CUDA events (diagnostics) */
int dspbr_set_profiling(dspbr_ctx* ctx, int enable);

/* ---- kernel-level entry points used by parity tests and embedders -------- */
/* closest hit (bvh.glsl:149-216): rays n x 8 floats (org.xyz, dir.xyz, tfar, 0);
 * outputs mesh triangle index (-1 = miss), t, barycentric u,v. */
int dspbr_trace_closest(dspbr_ctx* ctx, const dspbr_scene* scene, const float* rays, uint32_t n, int32_t* tri,
                        float* t, float* uv);
/* isOccluded (bvh.glsl:225-229) with an any-hit traversal: rays n x 8 floats. */
int dspbr_trace_occluded(dspbr_ctx* ctx, const dspbr_scene* scene, const float* rays, uint32_t n, int32_t* occluded);
/* BSDF through configure_gltf_material + pbrEval/Pdf/SampleGltfState
 * (material.glsl:5-110, material_kernel.glsl:4390-4425).  hit: n x 20 floats
 * (n.xyz, ng.xyz, tangent.xyzw, wi.xyz, uv0.xy, vertex colour rgba, material
 * index); wo: n x 3; rnd: n x 4 (component, lobe.x, lobe.y, boundary).
 * eval4: bsdf*cos rgb + pdf; sample10: dir.xyz, pdf, bsdfOverPdf.rgb, specular,
 * crossedBoundary, nextMediumIor; flags: bit0 = backside. */
int dspbr_bsdf_query(dspbr_ctx* ctx, const dspbr_scene* scene, uint32_t n, const float* hit, const float* wo,
                     const float* rnd, float* eval4, float* sample10, int32_t* flags);
/* IBL (lighting.glsl:24-98): sample (r0,r1) -> dir.xyz + pdf with the
 * context's env_sampling mode; pdf and radiance at given directions. */
int dspbr_ibl_query(dspbr_ctx* ctx, const dspbr_ibl* ibl, uint32_t n, const float* r2, const float* dirs,
                    float* sample_dir_pdf4, float* pdf, float* rgb);
/* camera rays (renderer.frag:129-142) for pixels xy with jitter r2: n x 6 (org, dir) */
int dspbr_camera_rays(dspbr_ctx* ctx, uint32_t n, const int32_t* xy, const float* r2, float* rays6);

/* ---- serving: continuous batching of render requests --------------------
 * The reference renders one viewport per WebGL context, one frame per
 * animation frame (renderer.ts:512-565).  A server renders many requests --
 * each a viewport of a resident scene at its own resolution, spp and
 * settings -- in one path pool: requests are admitted while the GPU works on
 * others (as pool slots and the HBM budget allow), their paths share every
 * launch, and each result is the image the same request renders alone.  A
 * driver thread owns the server's CUDA stream; the calls below are
 * thread-safe. */
typedef struct dspbr_server_config {
  uint32_t path_pool;         /* path slots (0: 2^23) */
  int max_active;             /* requests in flight at once, 1..256 (0: 256) */
  uint64_t hbm_budget_bytes;  /* path pool + scenes in use + request buffers (0: 120 GB) */
  int reserved[8];
} dspbr_server_config;

typedef struct dspbr_request {
  const dspbr_scene* scene;   /* created on the server's context */
  const dspbr_ibl* ibl;       /* NULL: no environment */
  float camera[16];           /* camera-to-world, column-major (setCamera) */
  float fov_deg, near_plane;
  int width, height;
  int spp;                    /* progressive frames, 1 sample per pixel each */
  dspbr_params params;
  float* out_rgba;            /* caller's buffer of width*height*4 floats; holds the mean once the request is done */
  uint64_t tag;               /* returned in dspbr_request_info */
} dspbr_request;

enum {
  DSPBR_REQ_QUEUED = 0,
  DSPBR_REQ_RUNNING = 1,
  DSPBR_REQ_DONE = 2,
  DSPBR_REQ_CANCELLED = 3,
  DSPBR_REQ_FAILED = 4
};

typedef struct dspbr_request_info {
  int state;                  /* DSPBR_REQ_* */
  uint64_t tag;
  double submit_ms, admit_ms, done_ms;  /* steady clock, milliseconds */
  uint64_t device_bytes;      /* request buffers charged to the budget */
} dspbr_request_info;

typedef struct dspbr_server_stats {
  uint64_t submitted, admitted, completed, cancelled, failed, queued, running;
  uint64_t iterations;        /* wavefront iterations run */
  uint64_t rays_closest, rays_shadow;
  uint64_t bytes_in_use, bytes_peak;
  double p50_ms, p99_ms;      /* submit -> done latency of completed requests */
  uint32_t path_pool;
  /* launch sizes in use: threads per block and grid (resident blocks) of the
   * persistent extend (trace_*), shade and connect kernels */
  int trace_threads, trace_blocks, shade_threads, shade_blocks;
  int connect_blocks;
} dspbr_server_stats;

/* Launch sizes of the path kernels, as the autotuner chooses them: the path
 * pool and the grids (resident blocks of 128 threads) of the persistent
 * extend, connect and shade kernels.  A grid is a multiple of the SM count, at
 * least one and at most the kernel's occupancy limit per SM. */
typedef struct dspbr_launch {
  uint32_t path_pool;
  int extend_blocks, connect_blocks, shade_blocks;
  int reserved[4];
} dspbr_launch;

int dspbr_server_create(dspbr_ctx* ctx, const dspbr_server_config* cfg, dspbr_server** out);
/* queue a request; DSPBR_ERR_ADMISSION if it can never fit the budget */
int dspbr_server_submit(dspbr_server* srv, const dspbr_request* req, uint64_t* id);
int dspbr_server_poll(dspbr_server* srv, uint64_t id, dspbr_request_info* info);
/* blocks until the request is done, cancelled or failed, or timeout_ms passes
 * (timeout_ms < 0: no limit); returns DSPBR_ERR_STATE on timeout */
int dspbr_server_wait(dspbr_server* srv, uint64_t id, int timeout_ms, dspbr_request_info* info);
/* no further samples start; the request ends as DSPBR_REQ_CANCELLED and its
 * buffer is not written */
int dspbr_server_cancel(dspbr_server* srv, uint64_t id);
/* forgets a finished request (its info is no longer available) */
int dspbr_server_release(dspbr_server* srv, uint64_t id);
int dspbr_server_get_stats(dspbr_server* srv, dspbr_server_stats* stats);
/* Autotuner: renders the sample requests (results discarded) in steady state
 * under candidate launch sizes and keeps the fastest in rays per second, one
 * coordinate at a time: the path pool (2^20..2^23, within half the HBM
 * budget), then the resident blocks per SM of the extend, connect and shade
 * kernels (from the occupancy limit down).  Call while the server is idle.
 * seconds bounds the time.  New: the reference has one fixed fragment-shader
 * pass (renderer.ts:512-565) and nothing to tune. */
int dspbr_server_autotune(dspbr_server* srv, const dspbr_request* samples, int n, double seconds);
/* The launch sizes in use, and setting them (an idle server only; e.g. the
 * autotuner's choice cached from an earlier run on the same GPU). */
int dspbr_server_get_launch(dspbr_server* srv, dspbr_launch* launch);
int dspbr_server_set_launch(dspbr_server* srv, const dspbr_launch* launch);
int dspbr_server_destroy(dspbr_server* srv);

#ifdef __cplusplus
}
#endif

#endif /* DSPBR_H */
