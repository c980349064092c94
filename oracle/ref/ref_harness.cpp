// ORACLE TEST INFRASTRUCTURE — not part of the product.
//
// Host harness around the reference's own fragment shader, compiled as C++
// (see glsl2cpp.py).  It plays the role WebGL2 plays in the reference: it owns
// the data "textures", the std140 uniform block (renderer.frag:10-31) and the
// per-fragment built-ins, and it runs `main()` once per pixel per frame.
// Entry points expose the shader's functions at every level the parity tests
// need: closest hit, camera ray, RNG, BSDF eval/pdf/sample, IBL, whole frames.
//
// Build: oracle/ref/build_ref.sh (writes only to oracle/_ref/).
#include "glsl_shim.h"

#include <algorithm>
#include <thread>
#include <vector>

#ifndef REF_PREFIX
#define REF_PREFIX ref_f32_
#endif
#define REF_CAT2(a, b) a##b
#define REF_CAT(a, b) REF_CAT2(a, b)
#define REF(name) REF_CAT(REF_PREFIX, name)

namespace glsl {
thread_local vec4 gl_FragCoord;
thread_local vec2 v_uv;
thread_local vec4 out_FragColor;
thread_local uint64_t glsl_rays_traced = 0;

// ---- the uniform block of renderer.frag:10-31, in its std140 order -------
mat4 u_u_view_mat;
vec4 u_background_color;
vec4 u_camera_pos;
vec2 u_inv_render_res;
vec2 u_ibl_resolution;
real u_frame_count, u_debug_mode, u_uniform_pad1, u_use_ibl, u_ibl_rotation, u_background_from_ibl,
    u_max_bounces, u_focal_length, u_ibl_pdf_total_sum, u_ray_eps, u_clamp_threshold, u_uniform_pad0;
vec4 u_scene_counts;
vec4 u_point_light_position;
vec4 u_point_light_emission;

// ---- samplers ---------------------------------------------------------------
sampler2D u_sampler2D_PreviousTexture;
sampler2D u_sampler_triangle_data;
isampler2D u_sampler_triangle_indices;
sampler2D u_sampler_bvh;
isampler2D u_sampler_bvh_index;
sampler2D u_sampler_env_map, u_sampler_env_map_pdf, u_sampler_env_map_cdf, u_sampler_env_map_yPdf,
    u_sampler_env_map_yCdf;
const f32* glsl_material_table = nullptr;

#include REF_SOURCE
#ifdef REF_POST_SOURCE
// display epilogue (tonemap.frag, fxaa.frag), renderer.ts:668-690
#include REF_POST_SOURCE
#endif
}  // namespace glsl
using namespace glsl;

namespace {
const int kTexW = 16384;  // MAX_TEXTURE_SIZE of buffer_accessor.inc

struct HostScene {
  std::vector<float> vertex_tex;    // RGBA32F, 5 texels per vertex
  std::vector<int32_t> index_tex;   // R32I
  std::vector<float> bvh_tex;       // RGBA32F, 4 texels per node
  std::vector<int32_t> bvh_idx_tex; // R32I
  std::vector<float> materials;     // 68 floats per material
  int num_tris = 0, num_nodes = 0, num_bvh_idx = 0;
} g_scene;

struct HostIbl {
  std::vector<float> rgba, pdf, cdf, ypdf, ycdf;
  double total_sum = 0.0;
  int w = 0, h = 0;
} g_ibl;

template <class T>
void pad_texture(std::vector<T>& dst, const T* src, size_t count, int per_texel) {
  size_t texels = (count + per_texel - 1) / per_texel;
  size_t rows = std::max<size_t>(1, (texels + kTexW - 1) / kTexW);
  dst.assign(rows * kTexW * per_texel, T(0));
  if (count) std::memcpy(dst.data(), src, count * sizeof(T));
}

// renderer.ts:777-800, with the host's JS number semantics: the row sum and
// every quotient/prefix step are evaluated in double and stored to Float32Array.
double pdf_cdf_row(const float* data, float* pdf, float* cdf, int num) {
  double sum = 0.0;
  for (int i = 0; i < num; ++i) sum += double(data[i]);
  if (sum == 0.0) sum = 1.0;
  for (int i = 0; i < num; ++i) pdf[i] = float(double(data[i]) / sum);
  cdf[0] = pdf[0];
  for (int i = 1; i < num; ++i) cdf[i] = float(double(cdf[i - 1]) + double(pdf[i]));
  cdf[num - 1] = 1.0f;
  return sum;
}
}  // namespace

extern "C" {

int REF(set_scene)(const float* vertices, int nverts, const uint32_t* indices, int nidx, const float* materials,
                   int nmat, const float* nodes, int nnodes, const int32_t* bvh_index, int nbvh_index) {
  if (nverts <= 0 || nidx <= 0 || nidx % 3 || nmat <= 0 || nnodes <= 0) return -1;
  pad_texture(g_scene.vertex_tex, vertices, size_t(nverts) * 20, 4);
  pad_texture(g_scene.index_tex, reinterpret_cast<const int32_t*>(indices), size_t(nidx), 1);
  pad_texture(g_scene.bvh_tex, nodes, size_t(nnodes) * 16, 4);
  pad_texture(g_scene.bvh_idx_tex, bvh_index, size_t(nbvh_index), 1);
  g_scene.materials.assign(materials, materials + size_t(nmat) * 68);
  g_scene.num_tris = nidx / 3;
  g_scene.num_nodes = nnodes;
  g_scene.num_bvh_idx = nbvh_index;
  auto rows = [](size_t n) { return int(n / kTexW); };
  u_sampler_triangle_data = {g_scene.vertex_tex.data(), kTexW, rows(g_scene.vertex_tex.size() / 4), 4};
  u_sampler_triangle_indices = {g_scene.index_tex.data(), kTexW, rows(g_scene.index_tex.size())};
  u_sampler_bvh = {g_scene.bvh_tex.data(), kTexW, rows(g_scene.bvh_tex.size() / 4), 4};
  u_sampler_bvh_index = {g_scene.bvh_idx_tex.data(), kTexW, rows(g_scene.bvh_idx_tex.size())};
  glsl_material_table = g_scene.materials.data();
  u_scene_counts = vec4(g_scene.num_tris, g_scene.num_nodes, g_scene.num_bvh_idx, 0);
  return 0;
}

// renderer.ts:802-838 (luminance 0.299/0.587/0.114, per-row then marginal).
// Material textures (scene_data_webgl2.ts:233-363): `infos` holds 8 floats per
// TexInfo, `data[i]` the RGBA8 layers of texture array i, whl[3 i..3 i+2] its
// width, height and layer count.  The harness keeps copies.
int REF(set_textures)(const float* infos, int ninfos, int narrays, const uint8_t* const* data, const int* whl) {
  if (ninfos < 0 || narrays < 0 || narrays > kGlslMaxTexArrays) return -1;
  static std::vector<float> info_copy;
  static std::vector<std::vector<uint8_t>> array_copy;
  info_copy.assign(infos, infos + 8 * size_t(ninfos));
  array_copy.assign(size_t(narrays), {});
  for (int i = 0; i < narrays; ++i) {
    size_t bytes = size_t(whl[3 * i]) * whl[3 * i + 1] * whl[3 * i + 2] * 4;
    array_copy[i].assign(data[i], data[i] + bytes);
    glsl_tex_arrays[i] = sampler2DArray{array_copy[i].data(), whl[3 * i], whl[3 * i + 1], whl[3 * i + 2]};
  }
  glsl_tex_infos = info_copy.data();
  glsl_num_tex_infos = ninfos;
  glsl_num_tex_arrays = narrays;
  return 0;
}

int REF(set_ibl)(const float* rgba, int w, int h) {
  if (w <= 0 || h <= 0) return -1;
  HostIbl& I = g_ibl;
  I.w = w;
  I.h = h;
  I.rgba.assign(rgba, rgba + size_t(w) * h * 4);
  std::vector<float> f(size_t(w) * h), sumx(h);
  for (size_t k = 0; k < f.size(); ++k)
    f[k] = float(double(rgba[4 * k]) * 0.299 + double(rgba[4 * k + 1]) * 0.587 + double(rgba[4 * k + 2]) * 0.114);
  I.pdf.assign(f.size(), 0.f);
  I.cdf.assign(f.size(), 0.f);
  I.ypdf.assign(h, 0.f);
  I.ycdf.assign(h, 0.f);
  for (int y = 0; y < h; ++y)
    sumx[y] = float(pdf_cdf_row(&f[size_t(y) * w], &I.pdf[size_t(y) * w], &I.cdf[size_t(y) * w], w));
  I.total_sum = pdf_cdf_row(sumx.data(), I.ypdf.data(), I.ycdf.data(), h);
  u_sampler_env_map = {I.rgba.data(), w, h, 4};
  u_sampler_env_map_pdf = {I.pdf.data(), w, h, 1};
  u_sampler_env_map_cdf = {I.cdf.data(), w, h, 1};
  u_sampler_env_map_yPdf = {I.ypdf.data(), h, 1, 1};
  u_sampler_env_map_yCdf = {I.ycdf.data(), h, 1, 1};
  u_ibl_resolution = vec2(w, h);
  u_ibl_pdf_total_sum = real(float(I.total_sum));
  return 0;
}

void REF(get_ibl_tables)(float* pdf, float* cdf, float* ypdf, float* ycdf, double* total) {
  std::copy(g_ibl.pdf.begin(), g_ibl.pdf.end(), pdf);
  std::copy(g_ibl.cdf.begin(), g_ibl.cdf.end(), cdf);
  std::copy(g_ibl.ypdf.begin(), g_ibl.ypdf.end(), ypdf);
  std::copy(g_ibl.ycdf.begin(), g_ibl.ycdf.end(), ycdf);
  *total = g_ibl.total_sum;
}

// 52 floats in the order renderer.ts:376-397 flattens them.
void REF(set_uniforms)(const float* b) {
  for (int c = 0; c < 4; ++c) u_u_view_mat.c[c] = vec4(b[4 * c], b[4 * c + 1], b[4 * c + 2], b[4 * c + 3]);
  u_background_color = vec4(b[16], b[17], b[18], b[19]);
  u_camera_pos = vec4(b[20], b[21], b[22], b[23]);
  u_inv_render_res = vec2(b[24], b[25]);
  // b[26..27] = u_ibl_resolution: owned by set_ibl
  u_frame_count = b[28];
  u_debug_mode = b[29];
  u_uniform_pad1 = b[30];
  u_use_ibl = b[31];
  u_ibl_rotation = b[32];
  u_background_from_ibl = b[33];
  u_max_bounces = b[34];
  u_focal_length = b[35];
  // b[36] = u_ibl_pdf_total_sum: owned by set_ibl
  u_ray_eps = b[37];
  u_clamp_threshold = b[38];
  u_uniform_pad0 = b[39];
  // b[40..43] = u_scene_counts: owned by set_scene
  u_point_light_position = vec4(b[44], b[45], b[46], b[47]);
  u_point_light_emission = vec4(b[48], b[49], b[50], b[51]);
}

static void set_fragment(int x, int y, int W, int H) {
  gl_FragCoord = vec4(real(x) + real(0.5), real(y) + real(0.5), real(0.5), real(1));
  v_uv = vec2(real(2 * x + 1) / real(W) - real(1), real(2 * y + 1) / real(H) - real(1));
}

// One progressive frame (renderer.frag:146-157) over the whole image; `accum`
// is RGBA W*H, row 0 = gl_FragCoord.y 0.5, read as the previous frame and
// overwritten with the new running mean.
int REF(render)(int W, int H, float* accum, int nthreads) {
  std::vector<float> prev(accum, accum + size_t(W) * H * 4);
  u_sampler2D_PreviousTexture = {prev.data(), W, H, 4};
  nthreads = std::max(1, nthreads);
  std::vector<std::thread> pool;
  int bad = 0;
  for (int t = 0; t < nthreads; ++t) {
    pool.emplace_back([&, t] {
      for (int y = t; y < H; y += nthreads)
        for (int x = 0; x < W; ++x) {
          set_fragment(x, y, W, H);
          glsl_main();
          float* o = accum + (size_t(y) * W + x) * 4;
          o[0] = float(out_FragColor.x);
          o[1] = float(out_FragColor.y);
          o[2] = float(out_FragColor.z);
          o[3] = float(out_FragColor.w);
        }
      if (glsl_texture_requested) bad = 1;
    });
  }
  for (auto& th : pool) th.join();
  return bad ? -2 : 0;
}

// One frame of the listed pixels only (a bounded sample of a frame): out is
// n x 4 RGBA of the running mean with an all-zero previous frame.  Returns the
// number of rays traced (closest-hit + shadow) through *rays.
int REF(render_pixels)(int n, const int32_t* xy, int W, int H, float* out, int nthreads, uint64_t* rays) {
  std::vector<float> prev(4, 0.f);
  u_sampler2D_PreviousTexture = {nullptr, 0, 0, 4};  // texelFetch outside -> 0 (first frame)
  nthreads = std::max(1, nthreads);
  std::vector<std::thread> pool;
  std::vector<uint64_t> counts(nthreads, 0);
  for (int t = 0; t < nthreads; ++t) {
    pool.emplace_back([&, t] {
      glsl_rays_traced = 0;
      for (int i = t; i < n; i += nthreads) {
        set_fragment(xy[2 * i], xy[2 * i + 1], W, H);
        glsl_main();
        float* o = out + size_t(i) * 4;
        o[0] = float(out_FragColor.x); o[1] = float(out_FragColor.y);
        o[2] = float(out_FragColor.z); o[3] = float(out_FragColor.w);
      }
      counts[t] = glsl_rays_traced;
    });
  }
  for (auto& th : pool) th.join();
  uint64_t tot = 0;
  for (auto c : counts) tot += c;
  if (rays) *rays = tot;
  return 0;
}

// rays: n x 8 floats (org.xyz, dir.xyz, tfar, unused) -> bvh_intersect_nearest
void REF(trace)(int n, const float* rays, int32_t* tri, float* t, float* uv) {
  for (int i = 0; i < n; ++i) {
    const float* r = rays + 8 * size_t(i);
    bvh_ray ray = bvh_create_ray(vec3(r[3], r[4], r[5]), vec3(r[0], r[1], r[2]), real(r[6]));
    bvh_hit hit;
    bool h = bvh_intersect_nearest(ray, hit);
    tri[i] = h ? hit.triIndex : -1;
    t[i] = float(hit.tfar);
    uv[2 * i] = h ? float(hit.uv.x) : 0.f;
    uv[2 * i + 1] = h ? float(hit.uv.y) : 0.f;
  }
}

// isOccluded (bvh.glsl:225-229) for origins/directions: n x 8 floats as above.
void REF(occluded)(int n, const float* rays, int32_t* occ) {
  for (int i = 0; i < n; ++i) {
    const float* r = rays + 8 * size_t(i);
    occ[i] = isOccluded(vec3(r[0], r[1], r[2]), vec3(r[3], r[4], r[5])) ? 1 : 0;
  }
}

// Camera ray of renderer.frag:129-142 for pixel (x,y) with jitter (r0,r1).
void REF(camera_ray)(int n, const int32_t* xy, const float* r2, int W, int H, float* ray6) {
  for (int i = 0; i < n; ++i) {
    set_fragment(xy[2 * i], xy[2 * i + 1], W, H);
    bvh_ray r = calcuateViewRay(real(r2[2 * i]), real(r2[2 * i + 1]));
    float* o = ray6 + 6 * size_t(i);
    o[0] = float(r.org.x); o[1] = float(r.org.y); o[2] = float(r.org.z);
    o[3] = float(r.dir.x); o[4] = float(r.dir.y); o[5] = float(r.dir.z);
  }
}

// rng_init(seed) at pixel (x,y), then n draws of rng_float (rng.glsl:5-29).
void REF(rng)(int x, int y, int seed, int n, float* out) {
  gl_FragCoord = vec4(real(x) + real(0.5), real(y) + real(0.5), real(0.5), real(1));
  rng_init(seed);
  for (int i = 0; i < n; ++i) out[i] = float(rng_float());
}

// BSDF queries through the integrator's own call chain:
// configure_gltf_material (material.glsl:5-110) -> make_pbr_gltf_state
// (pbr_material_adapter.glsl:13-24) -> pbrEval/Pdf/SampleGltfState.
// hit: n x 20 floats = n.xyz, ng.xyz, tangent.xyzw, wi.xyz, uv0.xy,
//      vertex colour.rgba, material index.
// wo: n x 3. rnd: n x 4 = component, lobe.x, lobe.y, boundary.
// eval4: bsdf*cos rgb + pdf.  sample10: dir.xyz, pdf, bsdfOverPdf.rgb,
//      specular, crossedBoundary, nextMediumIor.  flags: bit0 backside.
void REF(bsdf)(int n, const float* hit, const float* wo3, const float* rnd, float* eval4, float* sample10,
               int32_t* flags) {
  for (int i = 0; i < n; ++i) {
    const float* h = hit + 20 * size_t(i);
    RenderState rs;
    rs.n = vec3(h[0], h[1], h[2]);
    rs.ng = vec3(h[3], h[4], h[5]);
    rs.tangent = vec4(h[6], h[7], h[8], h[9]);
    rs.wi = vec3(h[10], h[11], h[12]);
    rs.uv0 = vec2(h[13], h[14]);
    rs.uv1 = vec2(0, 0);
    vec4 vcol(h[15], h[16], h[17], h[18]);
    uint mat = uint(h[19]);
    configure_gltf_material(mat, rs, rs.closure, vcol);
    PbrGltfState st = make_pbr_gltf_state(rs.closure);
    PbrNormals nn = make_pbr_normals(rs.closure);
    vec3 wo(wo3[3 * i], wo3[3 * i + 1], wo3[3 * i + 2]);
    PbrDirections d = make_pbr_directions(rs.wi, wo);
    vec3 e = pbrEvalGltfState(st, d, nn);
    real p = pbrPdfGltfState(st, d, nn);
    eval4[4 * i] = float(e.x); eval4[4 * i + 1] = float(e.y); eval4[4 * i + 2] = float(e.z);
    eval4[4 * i + 3] = float(p);
    PbrRandoms R;
    R.component = rnd[4 * i];
    R.lobe = vec2(rnd[4 * i + 1], rnd[4 * i + 2]);
    R.boundary = rnd[4 * i + 3];
    PbrSample s = pbrSampleGltfState(st, make_pbr_directions(rs.wi, vec3(0)), nn, R);
    float* o = sample10 + 10 * size_t(i);
    o[0] = float(s.direction.x); o[1] = float(s.direction.y); o[2] = float(s.direction.z);
    o[3] = float(s.pdf);
    o[4] = float(s.bsdfOverPdf.x); o[5] = float(s.bsdfOverPdf.y); o[6] = float(s.bsdfOverPdf.z);
    o[7] = float(s.specular); o[8] = float(s.crossedBoundary); o[9] = float(s.nextMediumIor);
    flags[i] = rs.closure.backside ? 1 : 0;
  }
}

// IBL: ibl_sample_direction(r0,r1) -> dir+pdf; ibl_pdf(dir); ibl_eval(dir)
// (lighting.glsl:24-98).
void REF(ibl)(int n, const float* r2, const float* dirs, float* sdirpdf4, float* pdf1, float* rgb3) {
  for (int i = 0; i < n; ++i) {
    real pdf;
    vec3 s = ibl_sample_direction(real(r2[2 * i]), real(r2[2 * i + 1]), pdf);
    sdirpdf4[4 * i] = float(s.x); sdirpdf4[4 * i + 1] = float(s.y); sdirpdf4[4 * i + 2] = float(s.z);
    sdirpdf4[4 * i + 3] = float(pdf);
    vec3 d(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]);
    pdf1[i] = float(ibl_pdf(d));
    vec3 c = ibl_eval(d);
    rgb3[3 * i] = float(c.x); rgb3[3 * i + 1] = float(c.y); rgb3[3 * i + 2] = float(c.z);
  }
}

#ifdef REF_POST_SOURCE
// Tone-mapping pass over an RGBA32F image (the accumulation mean), as the
// reference draws it into the "postprocess" buffer: one fragment per pixel,
// v_uv at the pixel centre, NEAREST sampling (gl_utils.ts:22-30).
void REF(tonemap)(const float* rgba, int W, int H, float exposure, int gamma, int mode, float* out) {
  post_tonemap::tex = sampler2D{rgba, W, H, 4, true};
  post_tonemap::exposure = real(exposure);
  post_tonemap::gamma = gamma != 0;
  post_tonemap::tonemappingMode = mode;
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      v_uv = vec2(real(2 * x + 1) / real(W) - real(1), real(2 * y + 1) / real(H) - real(1));
      gl_FragCoord = vec4(real(x) + real(0.5), real(y) + real(0.5), real(0.5), real(1));
      post_tonemap::glsl_main();
      float* o = out + 4 * (size_t(y) * W + x);
      o[0] = float(out_FragColor.x); o[1] = float(out_FragColor.y); o[2] = float(out_FragColor.z);
      o[3] = float(out_FragColor.w);
    }
}

// FXAA pass (fxaa.frag) over the tone-mapped RGBA32F image.
void REF(fxaa)(const float* rgba, int W, int H, float* out) {
  post_fxaa::tex = sampler2D{rgba, W, H, 4, true};
  post_fxaa::u_inv_res = vec2(real(1) / real(W), real(1) / real(H));
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      gl_FragCoord = vec4(real(x) + real(0.5), real(y) + real(0.5), real(0.5), real(1));
      post_fxaa::glsl_main();
      float* o = out + 4 * (size_t(y) * W + x);
      o[0] = float(out_FragColor.x); o[1] = float(out_FragColor.y); o[2] = float(out_FragColor.z);
      o[3] = float(out_FragColor.w);
    }
}
#endif

}  // extern "C"
