// ORACLE TEST INFRASTRUCTURE — not part of the product.
//
// CPU restatement of dspbr-pt's path-tracing hot path, used only by tests/,
// the smoke check and bench.py's CPU-baseline leg as the checker.  Scalar C++,
// templated on the arithmetic type: `float` performs the shaders' FP32
// arithmetic with every operation separately rounded (built with
// -ffp-contract=off), `double` is the FP64 port.  Each function cites the
// reference file:line it restates (paths relative to the reference checkout):
//   shader/bvh.glsl              traversal, Moller-Trumbore, attribute fetch
//   shader/utils.glsl            frames, env mapping, lower_bound, MIS
//   shader/lighting.glsl         IBL sampling / pdf / eval, point light
//   shader/material.glsl         configure_gltf_material
//   shader/pbr_material_adapter.glsl + generated/slang_materials/webgl-full/
//       material_kernel.glsl     DSPBR closure, eval, pdf, sample
//   shader/integrator/misptdl.glsl, shader/renderer.frag   integrator
//   shader/rng.glsl              MWC random numbers
//   renderer.ts:777-838          environment pdf / cdf tables
//   packages/app/index.ts:561-596  brute-force closest hit (CPU picking)
// Exposed through a C ABI mirroring the reference harness (oracle/_ref), with
// prefixes orc_f32_ / orc_f64_.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace orc {

template <class R>
struct V {
  R x, y, z;
};
template <class R> inline V<R> v3(R x, R y, R z) { return V<R>{x, y, z}; }
template <class R> inline V<R> vs(R s) { return V<R>{s, s, s}; }
template <class R> inline V<R> operator+(V<R> a, V<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V<R> operator-(V<R> a, V<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V<R> operator*(V<R> a, V<R> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class R> inline V<R> operator/(V<R> a, V<R> b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
template <class R> inline V<R> operator*(V<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <class R> inline V<R> operator*(R s, V<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class R> inline V<R> operator/(V<R> a, R s) { return {a.x / s, a.y / s, a.z / s}; }
template <class R> inline V<R> operator+(V<R> a, R s) { return {a.x + s, a.y + s, a.z + s}; }
template <class R> inline V<R> operator+(R s, V<R> a) { return {s + a.x, s + a.y, s + a.z}; }
template <class R> inline V<R> operator-(V<R> a, R s) { return {a.x - s, a.y - s, a.z - s}; }
template <class R> inline V<R> operator-(R s, V<R> a) { return {s - a.x, s - a.y, s - a.z}; }
template <class R> inline V<R> operator-(V<R> a) { return {-a.x, -a.y, -a.z}; }

// GLSL ES 3.00 8.3 built-ins
template <class R> inline R gmin(R x, R y) { return y < x ? y : x; }
template <class R> inline R gmax(R x, R y) { return x < y ? y : x; }
template <class R> inline R gclamp(R x, R a, R b) { return gmin(gmax(x, a), b); }
template <class R> inline R sat(R x) { return gclamp(x, R(0), R(1)); }
template <class R> inline R mix(R x, R y, R a) { return x * (R(1) - a) + y * a; }
template <class R> inline V<R> vmax(V<R> a, V<R> b) { return {gmax(a.x, b.x), gmax(a.y, b.y), gmax(a.z, b.z)}; }
template <class R> inline V<R> vmin(V<R> a, V<R> b) { return {gmin(a.x, b.x), gmin(a.y, b.y), gmin(a.z, b.z)}; }
template <class R> inline V<R> vclamp(V<R> a, R lo, R hi) {
  return {gclamp(a.x, lo, hi), gclamp(a.y, lo, hi), gclamp(a.z, lo, hi)};
}
template <class R> inline V<R> vsat(V<R> a) { return vclamp(a, R(0), R(1)); }
template <class R> inline V<R> vmix(V<R> x, V<R> y, R a) { return x * (R(1) - a) + y * a; }
template <class R> inline R max3(V<R> a) { return gmax(a.x, gmax(a.y, a.z)); }
template <class R> inline R dot(V<R> a, V<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline V<R> cross(V<R> a, V<R> b) {
  return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
template <class R> inline R len(V<R> a) { return std::sqrt(dot(a, a)); }
template <class R> inline V<R> nrm(V<R> a) { return a / len(a); }
template <class R> inline V<R> reflect(V<R> i, V<R> n) { return i - R(2) * dot(n, i) * n; }
template <class R> inline V<R> vexp(V<R> a) { return {std::exp(a.x), std::exp(a.y), std::exp(a.z)}; }
template <class R> inline V<R> vlog(V<R> a) { return {std::log(a.x), std::log(a.y), std::log(a.z)}; }
template <class R> inline V<R> vsqrt(V<R> a) { return {std::sqrt(a.x), std::sqrt(a.y), std::sqrt(a.z)}; }
template <class R> inline V<R> vcos(V<R> a) { return {std::cos(a.x), std::cos(a.y), std::cos(a.z)}; }
template <class R> inline R pw(R x, R y) { return std::pow(x, y); }

// constants.glsl:12-21
template <class R> struct K {
  static constexpr R PI = R(3.14159265358979323);
  static constexpr R TWO_PI = R(6.28318530717958648);
  static constexpr R EPS = R(1e-8);
  static constexpr R EPS_COS = R(0.001);
  static constexpr R EPS_PDF = R(0.001);
  static constexpr R TFAR_MAX = R(100000.0);
  static constexpr R BVH_FAR = R(1e30);
  // generated kernel literals
  static constexpr R kPi = R(3.14159274101257324);
  static constexpr R kTwoPi = R(6.28318548202514648);
  static constexpr R kInvPi = R(0.31830987334251404);
  static constexpr R kAvg = R(0.0476190485060215);
  static constexpr R e5 = R(0.00000999999974738);
  static constexpr R e4 = R(0.00009999999747379);
  static constexpr R e6 = R(9.99999997475242708e-07);
  static constexpr R e8 = R(9.99999993922529029e-09);
  static constexpr R e12 = R(9.999999960041972e-13);
};

// ---------------------------------------------------------------------------------
// scene (formats of scene_data.ts:21, material.ts, bvh.glsl:1-6)
struct Scene {
  const float* verts = nullptr;   // 20 floats per vertex
  const uint32_t* idx = nullptr;  // 3 per triangle
  const float* mats = nullptr;    // 68 floats per material
  const float* nodes = nullptr;   // 16 floats per node
  const int32_t* remap = nullptr;
  int nverts = 0, ntris = 0, nmats = 0, nnodes = 0, nremap = 0;
};

struct Ibl {
  const float* rgba = nullptr;
  int w = 0, h = 0;
  std::vector<float> pdf, cdf, ypdf, ycdf;
  std::vector<float> alias_prob;
  std::vector<int> alias_idx;
  double total = 0;
};

// precompute1DPdfAndCdf (renderer.ts:777-800) with JavaScript number semantics:
// double arithmetic, Float32Array storage.
inline double pdf_cdf(const float* d, float* pdf, float* cdf, int num) {
  double sum = 0;
  for (int i = 0; i < num; ++i) sum += double(d[i]);
  if (sum == 0) sum = 1;
  for (int i = 0; i < num; ++i) pdf[i] = float(double(d[i]) / sum);
  cdf[0] = pdf[0];
  for (int i = 1; i < num; ++i) cdf[i] = float(double(cdf[i - 1]) + double(pdf[i]));
  cdf[num - 1] = 1.0f;
  return sum;
}

// precomputeIBLImportanceSamplingData (renderer.ts:802-838)
inline void build_ibl(Ibl& I, const float* rgba, int w, int h) {
  I.rgba = rgba;
  I.w = w;
  I.h = h;
  size_t n = size_t(w) * h;
  std::vector<float> f(n), sumx(h);
  for (size_t k = 0; k < n; ++k)
    f[k] = float(double(rgba[4 * k]) * 0.299 + double(rgba[4 * k + 1]) * 0.587 + double(rgba[4 * k + 2]) * 0.114);
  I.pdf.assign(n, 0.f);
  I.cdf.assign(n, 0.f);
  I.ypdf.assign(h, 0.f);
  I.ycdf.assign(h, 0.f);
  for (int y = 0; y < h; ++y)
    sumx[y] = float(pdf_cdf(&f[size_t(y) * w], &I.pdf[size_t(y) * w], &I.cdf[size_t(y) * w], w));
  I.total = pdf_cdf(sumx.data(), I.ypdf.data(), I.ycdf.data(), h);
  // alias table over p(x,y) = yPdf[y] pdf[y][x] (Vose), for the alias mode
  std::vector<double> q(n);
  double tot = 0;
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) tot += (q[size_t(y) * w + x] = double(I.ypdf[y]) * double(I.pdf[size_t(y) * w + x]));
  I.alias_prob.assign(n, 1.f);
  I.alias_idx.resize(n);
  for (size_t i = 0; i < n; ++i) I.alias_idx[i] = int(i);
  if (!(tot > 0)) return;
  std::vector<size_t> sm, lg;
  for (size_t i = 0; i < n; ++i) {
    q[i] = q[i] * double(n) / tot;
    (q[i] < 1.0 ? sm : lg).push_back(i);
  }
  while (!sm.empty() && !lg.empty()) {
    size_t l = sm.back();
    sm.pop_back();
    size_t g = lg.back();
    I.alias_prob[l] = float(q[l]);
    I.alias_idx[l] = int(g);
    q[g] = (q[g] + q[l]) - 1.0;
    if (q[g] < 1.0) { lg.pop_back(); sm.push_back(g); }
  }
}

// ---------------------------------------------------------------------------------
// RNG: rng.glsl:5-29 (MWC seeded from gl_FragCoord) and PCG32 streams
template <class R>
struct Rng {
  bool pcg = false;
  uint32_t x = 0, y = 0;
  uint64_t st = 0, inc = 0;
  void mwc_init(int seed, int px, int py) {
    R off = R(seed * 17);
    R fx = R(px) + R(0.5), fy = R(py) + R(0.5);
    x = uint32_t(R(397.6432) * (fx + off));
    y = uint32_t(R(397.6432) * (fy + R(0)));
    x ^= uint32_t(R(32.9875) * (fy + off));
    y ^= uint32_t(R(32.9875) * (fx + R(0)));
  }
  uint32_t pcg_next() {
    uint64_t old = st;
    st = old * 6364136223846793005ull + inc;
    uint32_t xs = uint32_t(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = uint32_t(old >> 59u);
    return (xs >> rot) | (xs << ((32u - rot) & 31u));
  }
  void pcg_init(uint64_t seed, uint64_t stream) {
    pcg = true;
    inc = (stream << 1u) | 1u;
    st = 0;
    pcg_next();
    st += seed;
    pcg_next();
  }
  R next() {
    if (pcg) return R(float(pcg_next() >> 8) * (1.0f / 16777216.0f));
    x = 36969u * (x & 65535u) + (x >> 16u);
    y = 18000u * (y & 65535u) + (y >> 16u);
    return R((x << 16u) + y) / R(0xFFFFFFFFu);
  }
};

// ---------------------------------------------------------------------------------
// traversal: bvh.glsl:31-62 (slab, Moller-Trumbore), 149-229 (stack traversal)
template <class R>
struct Hit {
  int tri = -1;
  R t = 0, u = 0, v = 0;
};
struct TraversalStats {
  uint64_t nodes = 0, tris = 0, rays = 0, aborted = 0;
};

template <class R>
R slab(const float* lo, const float* hi, V<R> o, V<R> inv, R tfar) {
  V<R> t0 = (v3<R>(lo[0], lo[1], lo[2]) - o) * inv;
  V<R> t1 = (v3<R>(hi[0], hi[1], hi[2]) - o) * inv;
  V<R> mn = vmin(t0, t1), mx = vmax(t0, t1);
  R tmin = gmax(gmax(mn.x, mn.y), mn.z);
  R tmax = gmin(gmin(mx.x, mx.y), mx.z);
  if (std::isnan(tmin) || std::isnan(tmax) || tmin > tmax || tmax < R(0) || tmin >= tfar) return K<R>::BVH_FAR;
  return tmin;
}

template <class R>
V<R> vpos(const Scene& s, uint32_t vi) {
  const float* p = s.verts + size_t(vi) * 20;
  return v3<R>(p[0], p[1], p[2]);
}

template <class R>
bool moller_trumbore(V<R> o, V<R> d, V<R> p0, V<R> p1, V<R> p2, R tfar, R& t, R& u, R& v) {
  V<R> e0 = p1 - p0, e1 = p2 - p0;
  V<R> pv = cross(d, e1);
  R det = dot(e0, pv);
  if (std::fabs(det) < K<R>::EPS) return false;
  R f = R(1) / det;
  V<R> sv = o - p0;
  u = f * dot(sv, pv);
  if (u < R(0) || u > R(1)) return false;
  V<R> q = cross(sv, e0);
  v = f * dot(d, q);
  if (v < R(0) || u + v > R(1)) return false;
  t = f * dot(e1, q);
  if (t < K<R>::EPS || t >= tfar) return false;
  return true;
}

template <class R>
bool closest_hit(const Scene& s, V<R> o, V<R> d, R tfar, Hit<R>& hit, TraversalStats* ts = nullptr,
                 bool any = false) {
  V<R> inv = v3<R>(R(1) / d.x, R(1) / d.y, R(1) / d.z);
  hit = Hit<R>();
  hit.t = tfar;
  int stack[64];
  int top = 1;
  stack[0] = 0;
  int step = 0;
  if (ts) ts->rays++;
  for (; step < 4096 && top > 0; ++step) {
    int ni = stack[--top];
    if (ni < 0 || ni >= s.nnodes) continue;
    if (ts) ts->nodes++;
    const float* nd = s.nodes + size_t(ni) * 16;
    int cnt = int(nd[11]), first = int(nd[15]);
    if (cnt > 0) {
      int end = std::min(first + std::min(cnt, 64), s.nremap);
      for (int i = first; i < end; ++i) {
        int idx = (i < 0 || i >= s.nremap) ? -1 : s.remap[i];
        if (idx < 0 || idx >= s.ntris) continue;
        if (ts) ts->tris++;
        R t, u, v;
        V<R> p0 = vpos<R>(s, s.idx[3 * idx]), p1 = vpos<R>(s, s.idx[3 * idx + 1]), p2 = vpos<R>(s, s.idx[3 * idx + 2]);
        if (moller_trumbore(o, d, p0, p1, p2, hit.t, t, u, v)) {
          hit.t = t; hit.tri = idx; hit.u = u; hit.v = v;
          if (any) return true;
        }
      }
    } else {
      int left = int(nd[3]), right = int(nd[7]);
      R d0 = slab(nd + 0, nd + 4, o, inv, hit.t);
      R d1 = slab(nd + 8, nd + 12, o, inv, hit.t);
      auto push = [&](int c) {
        if (top < 64 && c >= 0 && c < s.nnodes && c != ni) stack[top++] = c;
      };
      if (d0 < K<R>::BVH_FAR && d1 < K<R>::BVH_FAR) {
        if (d0 < d1) { push(right); push(left); }
        else { push(left); push(right); }
      } else if (d0 < K<R>::BVH_FAR) {
        push(left);
      } else if (d1 < K<R>::BVH_FAR) {
        push(right);
      }
    }
  }
  if (ts && top > 0 && step >= 4096) ts->aborted++;
  return hit.tri >= 0;
}

// packages/app/index.ts:561-596, all-triangle brute force with the shader's
// rejection tests (EPS 1e-8) instead of the app's 1e-7.
template <class R>
bool brute_force(const Scene& s, V<R> o, V<R> d, R tfar, Hit<R>& hit) {
  hit = Hit<R>();
  hit.t = tfar;
  for (int i = 0; i < s.ntris; ++i) {
    R t, u, v;
    V<R> p0 = vpos<R>(s, s.idx[3 * i]), p1 = vpos<R>(s, s.idx[3 * i + 1]), p2 = vpos<R>(s, s.idx[3 * i + 2]);
    if (moller_trumbore(o, d, p0, p1, p2, hit.t, t, u, v)) { hit.t = t; hit.tri = i; hit.u = u; hit.v = v; }
  }
  return hit.tri >= 0;
}

// ---------------------------------------------------------------------------------
// DSPBR material (material_kernel.glsl, webgl-full profile)
template <class R>
struct GMat {  // PbrGltfMaterial fields after configure_gltf_material
  V<R> base;
  R metallic, roughness, specular;
  V<R> spec_color;
  R transmission, dt;
  V<R> dt_color;
  R ior, clearcoat, cc_rough;
  V<R> sheen;
  R sheen_rough, aniso, irid, irid_ior, irid_thick, dispersion, thickness;
};

template <class R>
struct Cl {  // SurfaceClosure_0 (kernel:316-354)
  V<R> drc, albedo;
  R dw, sw, aniso;
  V<R> at;
  V<R> f0;
  R f90, diel_w, spec_w, cc_w, rough;
  V<R> sheen;
  R sheen_rough, transp, cc, cc_rough, metallic, specular, ior, irid, irid_ior, irid_thick, disp, thin, tw;
  V<R> dtc;
  R dtw;
};

template <class R> R avg_alb(R a) {  // kernel:5-10
  R r = std::sqrt(gmax(a, R(0)));
  return sat(R(1) - R(0.57999998331069946) * r + R(0.07999999821186066) * r * r);
}
template <class R> R dir_alb(R a, R c) {  // kernel:34-40
  return sat(R(1) - std::sqrt(gmax(a, R(0))) * (R(0.5) + R(0.5) * pw(R(1) - sat(c), R(5))));
}
template <class R> R avg_alb_ms(R a, R e0) {  // kernel:13-16
  return sat(sat(e0 + (R(1) - e0) * K<R>::kAvg) * avg_alb(a));
}
template <class R> R dir_alb_ms(R th, R a, R e0) {  // kernel:43-49
  R nv = sat(th);
  return sat(sat(e0 + (R(1) - e0) * pw(R(1) - nv, R(5))) * mix(R(1), dir_alb(a, nv), R(0.64999997615814209)));
}
template <class R> V<R> schlick_avg(V<R> f0, V<R> f90) { return f0 + (f90 - f0) * K<R>::kAvg; }
template <class R> V<R> schlick(V<R> f0, V<R> f90, R c) {  // kernel:709-716
  R m = sat(R(1) - c);
  R m2 = m * m;
  return f0 + (f90 - f0) * (m2 * m2 * m);
}

// buildEnterpriseSurfaceFromGltf_0 + buildSurfaceClosure_0 (kernel:209-261, 357-422)
template <class R>
Cl<R> closure(const GMat<R>& m, V<R> at, bool lean) {
  V<R> albedo = vsat(m.base);
  R metallic = sat(m.metallic), roughness = sat(m.roughness), transp = sat(m.transmission);
  R ior = gmax(m.ior, R(1));
  V<R> sc = vsat(m.spec_color);
  R spec = sat(m.specular);
  R thin = m.thickness > R(0) ? R(0) : R(1);
  R tl = sat(m.dt);
  V<R> tlc = vsat(m.dt_color);
  R irid = sat(m.irid), irid_ior = gclamp(m.irid_ior, R(1), R(2.5)), irid_thick = gmax(m.irid_thick, R(0));
  R disp = gmax(m.dispersion, R(0));
  R cc = sat(m.clearcoat), ccr = sat(m.cc_rough);
  V<R> sheen = vsat(m.sheen);
  R sr = sat(m.sheen_rough), an = sat(m.aniso);
  if (lean) { irid = R(0); disp = R(0); }
  Cl<R> c;
  R dw = R(1) - metallic;
  R op = R(1) - transp;
  R odw = dw * op, tdw = dw * transp;
  V<R> drc = albedo * odw * (R(1) - tl);
  V<R> dtc = odw * tlc * tl;
  R ratio = (R(1) - ior) / (R(1) + ior);
  V<R> f0 = vsat(vs(ratio * ratio * spec) * sc);
  V<R> metal = schlick_avg(albedo, vs(R(1)));
  c.drc = drc; c.albedo = albedo; c.dw = max3(drc); c.sw = max3(sheen) * op; c.aniso = an; c.at = at;
  c.f0 = f0; c.f90 = spec; c.diel_w = dw;
  R fi = gmax(irid_ior, R(1));
  R fr = (fi - R(1)) / gmax(fi + R(1), K<R>::e5);
  R film_w = sat(irid) * pw(fr, R(2));
  c.spec_w = gmax(max3(metal), film_w) * metallic;
  R ccrb = sat(gmax(ccr, R(0.0020000000949949)));
  c.cc_w = cc * mix(R(0.20000000298023224), R(1), R(1) - ccrb);
  c.rough = sat(gmax(roughness, R(0.0020000000949949)));
  c.sheen = sheen; c.sheen_rough = sr; c.transp = transp; c.cc = cc; c.cc_rough = ccrb;
  c.metallic = metallic; c.specular = spec; c.ior = ior; c.irid = irid; c.irid_ior = irid_ior;
  c.irid_thick = irid_thick; c.disp = disp; c.thin = thin; c.tw = max3(albedo) * tdw; c.dtc = dtc; c.dtw = max3(dtc);
  return c;
}

// fresnelSchlickDielectric_0 (kernel:681-707) for n_i = 1 (adapter:18)
template <class R> V<R> fresnel_d(R c, V<R> f0, R f90, R nt) {
  if (std::fabs(R(1) - nt) <= K<R>::e4) return vs(R(0));
  return schlick(f0, vs(f90), sat(c));
}
template <class R> V<R> sensitivity(R opd, V<R> shift) {  // kernel:764-790
  R ph = R(6.28318548202514648) * opd * R(9.99999971718068537e-10);
  R ph2 = ph * ph;
  V<R> var = v3<R>(R(4.327799808e+09), R(9.304599552e+09), R(6.612100096e+09));
  V<R> xyz = v3<R>(R(5.48560003844900113e-13), R(4.42010008238832852e-13), R(5.24810013155518895e-13)) *
             vsqrt(R(6.28318548202514648) * var) *
             vcos(v3<R>(R(1.681e+06), R(1.7953e+06), R(2.2084e+06)) * ph + shift) * vexp(-ph2 * var);
  xyz.x = xyz.x + R(9.74699989231449238e-14) * std::sqrt(R(2.845152256e+10)) *
                      std::cos(R(2.2399e+06) * ph + shift.x) * std::exp(R(-4.528200192e+09) * ph2);
  xyz = xyz / R(1.06850002623559703e-07);
  return v3<R>(R(3.24045419692993164) * xyz.x - R(1.53713846206665039) * xyz.y - R(0.49853140115737915) * xyz.z,
               R(-0.96926599740982056) * xyz.x + R(1.87601077556610107) * xyz.y + R(0.04155600070953369) * xyz.z,
               R(0.05564339831471443) * xyz.x - R(0.20402589440345764) * xyz.y + R(1.05722522735595703) * xyz.z);
}
template <class R> R ior_f0(R t, R i) {
  R r = (t - i) / gmax(t + i, K<R>::e5);
  return r * r;
}
template <class R> V<R> film_refl(R outside, R film, V<R> base_f0, R thick, R cos1) {  // kernel:796-924
  R fi = gclamp(film, R(1), R(2.5));
  R c1 = sat(cos1);
  R c2sq = R(1) - outside / fi * (outside / fi) * (R(1) - c1 * c1);
  if (c2sq < R(0)) return vs(R(1));
  R c2 = std::sqrt(c2sq);
  R r12 = schlick(vs(ior_f0(fi, outside)), vs(R(1)), c1).x;
  R t121 = R(1) - r12;
  V<R> sf = vsqrt(vclamp(base_f0, R(0), R(0.99989998340606689)));
  V<R> bior = (vs(R(1)) + sf) / vmax(vs(R(1)) - sf, vs(K<R>::e5));
  V<R> r1 = (bior - vs(fi)) / vmax(bior + vs(fi), vs(K<R>::e5));
  V<R> r23 = schlick(r1 * r1, vs(R(1)), c2);
  R opd = R(2) * fi * gmax(thick, R(0)) * c2;
  R phi12 = fi < outside ? K<R>::kPi : R(0);
  R phi21 = K<R>::kPi - phi12;
  V<R> phi = vs(phi21) + v3<R>(bior.x < fi ? K<R>::kPi : R(0), bior.y < fi ? K<R>::kPi : R(0),
                                bior.z < fi ? K<R>::kPi : R(0));
  V<R> r123 = vclamp(vs(r12) * r23, K<R>::e5, R(0.99989998340606689));
  V<R> s123 = vsqrt(r123);
  V<R> rs = t121 * t121 * r23 / vmax(vs(R(1)) - r123, vs(K<R>::e5));
  V<R> refl = vs(r12) + rs;
  V<R> cm = rs - vs(t121);
  for (int m = 1; m <= 2; ++m) {
    cm = cm * s123;
    R fm = R(m);
    refl = refl + cm * R(2) * sensitivity(fm * opd, fm * phi);
  }
  return vmax(refl, vs(R(0)));
}
template <class R> V<R> film_fresnel(const Cl<R>& c, R cos_t, V<R> reg) {  // kernel:932-941
  if (c.irid <= K<R>::e5) return reg;
  R fi = gmax(c.ior, R(1));
  return vmix(reg, film_refl(R(1), c.irid_ior, vs(ior_f0(fi, R(1))), c.irid_thick, cos_t), sat(c.irid));
}

template <class R> struct Fr {
  V<R> t, b, n;
};
template <class R> Fr<R> frame(V<R> n, V<R> t) {  // projectToAnisotropicFrame_0 (kernel:448-454)
  V<R> st = nrm(t - n * dot(t, n));
  return Fr<R>{st, nrm(cross(n, st)), n};
}
template <class R> V<R> loc(const Fr<R>& f, V<R> d) { return v3<R>(dot(d, f.t), dot(d, f.b), dot(d, f.n)); }
template <class R> void alpha(R rough, R an, R& ax, R& ay) {  // kernel:457-465
  R a = sat(an);
  R r2 = gmax(rough * rough, R(0));
  ax = mix(r2, R(1), a * a);
  ay = r2;
}
template <class R> R d_an(R ax, R ay, V<R> h) {  // kernel:468-479
  R hx = h.x / ax, hy = h.y / ay;
  R den = hx * hx + hy * hy + h.z * h.z;
  return R(1) / gmax(K<R>::kPi * ax * ay * den * den, K<R>::e12);
}
template <class R> R lam_an(R ax, R ay, V<R> d) {  // kernel:482-507
  R c2 = d.z * d.z;
  if (c2 <= K<R>::e8) return R(0);
  if (gmax(R(1) - c2, R(0)) <= K<R>::e8) return R(0);
  return R(0.5) * (R(-1) + std::sqrt(R(1) + (d.x * d.x * ax * ax + d.y * d.y * ay * ay) / gmax(c2, K<R>::e8)));
}
template <class R> R micro(const Cl<R>& c, const Fr<R>& f, V<R> v, V<R> l) {  // kernel:515-586
  V<R> h = nrm(v + l);
  V<R> lv = loc(f, v), ll = loc(f, l), lh = loc(f, h);
  R nv = std::fabs(lv.z), nl = std::fabs(ll.z), nh = std::fabs(lh.z);
  R vh = gmax(dot(v, h), R(0));
  if (nv <= R(0) || nl <= R(0) || nh <= R(0) || vh <= R(0)) return R(0);
  R ax, ay;
  alpha(c.rough, c.aniso, ax, ay);
  return d_an(ax, ay, lh) * (R(1) / (R(1) + lam_an(ax, ay, lv) + lam_an(ax, ay, ll))) / gmax(R(4) * nv * nl, K<R>::e5);
}
template <class R> R d_iso(R a, R nh) {  // kernel:1893-1898
  R a2 = a * a;
  R d = nh * nh * (a2 - R(1)) + R(1);
  return a2 / gmax(K<R>::kPi * d * d, K<R>::e12);
}
template <class R> R lam_iso(R a, R nx) {  // kernel:1901-1926
  R ct = std::fabs(nx);
  R c2 = ct * ct;
  R s2 = gmax(R(1) - c2, R(0));
  if (s2 <= K<R>::e8 || ct <= K<R>::e8) return R(0);
  return R(0.5) * (R(-1) + std::sqrt(R(1) + a * a * (s2 / gmax(c2, K<R>::e8))));
}
template <class R> void ms(R rough, R cl, R cv, R& eavg, R& m) {
  R a = gmax(rough * rough, R(0));
  eavg = avg_alb(a);
  m = (R(1) - dir_alb(a, cl)) * (R(1) - dir_alb(a, cv)) / gmax(K<R>::kPi * (R(1) - eavg), K<R>::e6);
}
template <class R> V<R> ms_e(V<R> favg, R eavg, R m) {
  return m * (favg * favg * eavg / vmax(vs(R(1)) - favg * (R(1) - eavg), vs(K<R>::e5)));
}
template <class R> R tdw(const Cl<R>& c) { return c.diel_w * c.transp; }
template <class R> V<R> wtc(const Cl<R>& c) { return c.albedo * tdw(c); }

template <class R> V<R> diel_spec(const Cl<R>& c, const Fr<R>& f, V<R> n, V<R> v, V<R> l) {  // kernel:953-1033
  R nl = gmax(dot(n, l), R(0));
  R t = tdw(c);
  if (nl <= R(0) || t <= R(0)) return vs(R(0));
  R mr = micro(c, f, v, l);
  R vh = gmax(dot(v, nrm(v + l)), R(0));
  R eavg, m;
  ms(c.rough, nl, std::fabs(dot(n, v)), eavg, m);
  V<R> F = film_fresnel(c, vh, fresnel_d(vh, c.f0, c.f90, c.ior));
  V<R> favg = std::fabs(R(1) - c.ior) <= K<R>::e4 ? vs(R(0)) : schlick_avg(c.f0, vs(c.f90));
  return t * (mr * F + ms_e(favg, eavg, m)) * nl;
}
template <class R> struct TC {
  V<R> refl, trans;
  R pr, pt;
};
template <class R> TC<R> tcoef(const Cl<R>& c, V<R> n, V<R> v) {  // kernel:1065-1108
  R cv = gmax(dot(n, v), K<R>::e5);
  V<R> film = film_fresnel(c, cv, fresnel_d(cv, c.f0, c.f90, c.ior));
  TC<R> k;
  k.refl = film * tdw(c);
  k.trans = (vs(R(1)) - film) * wtc(c);
  R rw = max3(vmax(vs(R(1)), vs(R(0))) * vmax(k.refl, vs(R(0))));
  R tw = max3(vmax(vs(R(1)), vs(R(0))) * vmax(k.trans, vs(R(0))));
  R tot = rw + tw;
  if (tot <= K<R>::e5) { k.pr = R(1); k.pt = R(0); }
  else { k.pr = rw / tot; k.pt = tw / tot; }
  return k;
}
template <class R> V<R> flip(V<R> v, V<R> n) { return nrm(v - R(2) * n * dot(v, n)); }
template <class R> V<R> thin_trans(const Cl<R>& c, const Fr<R>& f, V<R> n, V<R> v, V<R> l) {  // kernel:1118-1148
  R nl = dot(n, l);
  if (dot(n, v) * nl >= R(0)) return vs(R(0));
  V<R> ml = flip(l, n);
  R vh = gmax(dot(v, nrm(v + ml)), K<R>::e5);
  V<R> film = film_fresnel(c, vh, fresnel_d(vh, c.f0, c.f90, c.ior));
  return wtc(c) * (vs(R(1)) - film) * micro(c, f, v, ml) * std::fabs(nl);
}
template <class R> V<R> thick_trans(const Cl<R>& c, const Fr<R>& f, V<R> coeff, V<R> n, V<R> v, V<R> l, R io) {
  // kernel:1151-1241
  V<R> lv = loc(f, v), ll = loc(f, l);
  R nv = std::fabs(lv.z), nl = std::fabs(ll.z);
  if (nv <= K<R>::e5 || nl <= K<R>::e5 || dot(n, v) * dot(n, l) >= R(0)) return vs(R(0));
  R eta = io / gmax(R(1), K<R>::e5);
  V<R> h = -nrm(v + l * eta);
  V<R> lh = loc(f, h);
  R vh = dot(v, h), lhh = dot(l, h);
  if (std::fabs(lh.z) <= K<R>::e5 || vh * lhh >= R(0)) return vs(R(0));
  R ax, ay;
  alpha(c.rough, c.aniso, ax, ay);
  R dd = d_an(ax, ay, lh);
  R g = R(1) / (R(1) + lam_an(ax, ay, lv) + lam_an(ax, ay, ll));
  R factor = eta * eta * std::fabs(vh) * std::fabs(lhh) / gmax(pw(vh + eta * lhh, R(2)) * nv, K<R>::e5);
  V<R> eff = coeff;
  if (c.irid > K<R>::e5) eff = (vs(R(1)) - film_fresnel(c, std::fabs(vh), fresnel_d(std::fabs(vh), c.f0, c.f90, io))) * wtc(c);
  return eff * dd * g * factor;
}
template <class R> V<R> disp_iors(const Cl<R>& c) {  // kernel:1289-1299
  R i = gmax(c.ior, R(1));
  R s = (i - R(1)) * gmax(c.disp, R(0)) * R(0.05000000074505806);
  return vmax(v3<R>(i + s * R(-0.30094969272613525), i, i + s * R(0.69905030727386475)), vs(R(1)));
}
template <class R> V<R> thick_disp(const Cl<R>& c, const Fr<R>& f, V<R> k, V<R> n, V<R> v, V<R> l) {  // kernel:1302-1425
  if (c.disp <= K<R>::e5 || c.thin > R(0.5)) return thick_trans(c, f, k, n, v, l, c.ior);
  V<R> io = disp_iors(c);
  V<R> r = thick_trans(c, f, v3<R>(k.x, R(0), R(0)), n, v, l, io.x);
  V<R> g = thick_trans(c, f, v3<R>(R(0), k.y, R(0)), n, v, l, io.y);
  V<R> b = thick_trans(c, f, v3<R>(R(0), R(0), k.z), n, v, l, io.z);
  return v3<R>(r.x, g.y, b.z);
}
template <class R> V<R> diel_trans(const Cl<R>& c, const Fr<R>& f, V<R> n, V<R> v, V<R> l) {  // kernel:1427-1497
  if (dot(n, v) * dot(n, l) > R(0)) return diel_spec(c, f, n, v, l);
  if (c.thin > R(0.5)) return thin_trans(c, f, n, v, l);
  return thick_disp(c, f, tcoef(c, n, v).trans, n, v, l);
}
template <class R> R coupled(const Cl<R>& c, R nv, R nl) {  // kernel:1510-1517
  R a = gmax(c.rough * c.rough, R(0));
  R e0 = max3(c.f0 * c.diel_w);
  return mix(K<R>::kInvPi,
             (R(1) - dir_alb_ms(nl, a, e0)) * (R(1) - dir_alb_ms(nv, a, e0)) /
                 gmax(K<R>::kPi * (R(1) - avg_alb_ms(a, e0)), K<R>::e6),
             c.specular);
}
template <class R> V<R> tsc(const Cl<R>& c) { return c.f0 * c.diel_w + c.albedo * c.metallic; }
template <class R> V<R> tsf(const Cl<R>& c) { return vs(c.f90) * c.diel_w + vs(c.metallic); }
template <class R> R tdcf(const Cl<R>& c, R nv, R nl) {  // kernel:1541-1587
  R cp = coupled(c, nv, nl);
  bool thin = c.thin > R(0.5);
  V<R> sc = thin ? tsc(c) : c.f0;
  V<R> sf = thin ? tsf(c) : vs(c.f90);
  R F0 = max3(sc);
  R dF = max3(sf) - F0;
  V<R> de = vsat(vs(R(1)) - (schlick_avg(c.albedo, vs(R(1))) * c.metallic + schlick_avg(c.f0, vs(c.f90)) * c.diel_w));
  return cp * mix(R(1), R(1) / gmax(max3(de), K<R>::e4),
                  std::sqrt(R(0.5) * (sat(F0 + dF * pw(R(1) - sat(nv), R(5))) + sat(F0 + dF * pw(R(1) - sat(nl), R(5))))));
}
template <class R> V<R> diffuse(const Cl<R>& c, V<R> n, V<R> v, V<R> l) {  // kernel:1589-1631
  R nl = gmax(dot(n, l), R(0));
  if (c.specular <= K<R>::e5 && c.transp <= R(0)) return c.drc * K<R>::kInvPi * nl;
  R nv = gmax(std::fabs(dot(v, n)), R(0));
  R fac = c.transp > R(0) ? tdcf(c, nv, nl) : coupled(c, nv, nl);
  return c.drc * fac * nl;
}
template <class R> bool thin_td(const Cl<R>& c) {  // kernel:1633-1660
  return c.thin > R(0.5) && (c.transp > R(0) || c.dtw > R(0)) && c.metallic < R(1);
}
template <class R> V<R> thin_shared(const Cl<R>& c, const Fr<R>& f, V<R> n, V<R> v, V<R> l) {  // kernel:1662-1721
  R nl = gmax(dot(n, l), R(0));
  if (nl <= R(0)) return vs(R(0));
  R mr = micro(c, f, v, l);
  R vh = gmax(dot(v, nrm(v + l)), R(0));
  R eavg, m;
  ms(c.rough, nl, std::fabs(dot(n, v)), eavg, m);
  V<R> f0 = tsc(c), f90 = tsf(c);
  V<R> F = schlick(f0, f90, vh);
  if (c.irid > K<R>::e5)
    F = vmix(F, film_refl(R(1), c.irid_ior, vs(ior_f0(gmax(c.ior, R(1)), R(1))), c.irid_thick, vh), sat(c.irid));
  return (mr * F + ms_e(schlick_avg(f0, f90), eavg, m)) * nl;
}
template <class R> V<R> base_spec_ggx(const Cl<R>& c, const Fr<R>& f, V<R> n, V<R> v, V<R> l) {  // kernel:1723-1786
  R mr = micro(c, f, v, l);
  R vh = gmax(dot(v, nrm(v + l)), R(0));
  R eavg, m;
  ms(c.rough, std::fabs(dot(n, l)), std::fabs(dot(n, v)), eavg, m);
  bool film = c.irid > K<R>::e5;
  V<R> mf = schlick(c.albedo, vs(R(1)), vh);
  if (film) mf = vmix(mf, film_refl(R(1), c.irid_ior, c.albedo, c.irid_thick, vh), sat(c.irid));
  V<R> df = schlick(c.f0, vs(c.f90), vh);
  if (film) df = vmix(df, film_refl(R(1), c.irid_ior, vs(ior_f0(gmax(c.ior, R(1)), R(1))), c.irid_thick, vh), sat(c.irid));
  return c.metallic * (mr * mf + ms_e(schlick_avg(c.albedo, vs(R(1))), eavg, m)) +
         c.diel_w * (R(1) - c.transp) * (mr * df + ms_e(schlick_avg(c.f0, vs(c.f90)), eavg, m));
}
template <class R> V<R> base_spec(const Cl<R>& c, const Fr<R>& f, V<R> n, V<R> v, V<R> l) {  // kernel:1788-1796
  R nl = gmax(dot(n, l), R(0));
  if (thin_td(c)) return thin_shared(c, f, n, v, l);
  return base_spec_ggx(c, f, n, v, l) * nl;
}
template <class R> R sheen_l(R x, R a) {  // kernel:1804-1810
  R o = R(1) - a;
  R o2 = o * o;
  return mix(R(21.54730033874511719), R(25.32449913024902344), o2) /
             (R(1) + mix(R(3.82986998558044434), R(3.32435011863708496), o2) *
                         pw(std::fabs(x), mix(R(0.19822999835014343), R(0.16800999641418457), o2))) +
         mix(R(-1.97759997844696045), R(-1.27392995357513428), o2) * x +
         mix(R(-4.32053995132446289), R(-4.85967016220092773), o2);
}
template <class R> R sheen_lam(R c, R a) {  // kernel:1813-1827
  if (std::fabs(c) >= R(0.5)) return std::exp(R(2) * sheen_l(R(0.5), a) - sheen_l(R(1) - c, a));
  return std::exp(sheen_l(c, a));
}
template <class R> V<R> sheen(const Cl<R>& c, V<R> n, V<R> v, V<R> l) {  // kernel:1830-1890
  if (max3(c.sheen) <= R(0)) return vs(R(0));
  R nv = gmax(dot(n, v), R(0)), nl = gmax(dot(n, l), R(0)), nh = gmax(dot(n, nrm(v + l)), R(0));
  if (nv <= R(0) || nl <= R(0) || nh <= R(0)) return vs(R(0));
  R a = gmax(c.sheen_rough * c.sheen_rough, R(0));
  R inv = R(1) / gmax(a, K<R>::e5);
  return c.sheen * (R(1) / (R(1) + sheen_lam(nv, a) + sheen_lam(nl, a)) *
                    ((R(2) + inv) * pw(std::fabs(gmax(R(1) - nh * nh, R(0.00100000004749745))), R(0.5) * inv) /
                     R(6.28318548202514648)) /
                    gmax(R(4) * nv * nl, K<R>::e5)) *
         nl;
}
template <class R> V<R> clearcoat(const Cl<R>& c, V<R> n, V<R> v, V<R> l) {  // kernel:1956-2043
  if (c.cc <= R(0)) return vs(R(0)) * gmax(dot(n, l), R(0));
  V<R> h = nrm(v + l);
  R nv = gmax(dot(n, v), R(0)), nl = gmax(dot(n, l), R(0)), nh = gmax(dot(n, h), R(0)), vh = gmax(dot(v, h), R(0));
  V<R> g = vs(R(0));
  if (!(nv <= R(0) || nl <= R(0) || nh <= R(0) || vh <= R(0))) {
    R a = gmax(c.cc_rough * c.cc_rough, R(0));
    g = schlick(vs(R(0.03999999910593033)), vs(R(1)), vh) * d_iso(a, nh) * (R(1) / (R(1) + lam_iso(a, nv) + lam_iso(a, nl))) /
        gmax(R(4) * nv * nl, K<R>::e5);
  }
  return c.cc * g * gmax(dot(n, l), R(0));
}
template <class R> R cc_base(const Cl<R>& c, V<R> n, V<R> v, V<R> l) {  // kernel:2035-2043
  if (c.cc <= R(0)) return R(1);
  V<R> a = schlick(vs(R(0.03999999910593033)), vs(R(1)), std::fabs(dot(n, v)));
  V<R> b = schlick(vs(R(0.03999999910593033)), vs(R(1)), std::fabs(dot(n, l)));
  return sat(R(1) - c.cc * gmax(max3(a), max3(b)));
}
template <class R> V<R> dtrans(const Cl<R>& c, V<R> n, V<R> l) {  // kernel:440-443
  return c.dtc * K<R>::kInvPi * gmax(std::fabs(dot(n, l)), R(0));
}
template <class R> V<R> refl_base(const Cl<R>& c, const Fr<R>& f, V<R> n, V<R> v, V<R> l) {
  return diffuse(c, n, v, l) + base_spec(c, f, n, v, l) + sheen(c, n, v, l);
}
// evalMaterialBsdfMixture_0 (kernel:2045-2089)
template <class R> V<R> eval(const Cl<R>& c, V<R> n, V<R> v, V<R> l) {
  Fr<R> f = frame(n, c.at);
  if (!(dot(n, v) * dot(n, l) > R(0))) return dtrans(c, n, l) + diel_trans(c, f, n, v, l);
  V<R> b = refl_base(c, f, n, v, l);
  if (c.thin < R(0.5) && c.transp > R(0)) b = b + diel_trans(c, f, n, v, l);
  return clearcoat(c, n, v, l) + b * cc_base(c, n, v, l);
}

// pdfMaterialBsdfMixture_0 and helpers (kernel:2113-2617)
template <class R> R slobe(const Cl<R>& c, const Fr<R>& f, V<R> v, V<R> d) {
  V<R> h = nrm(v + d);
  V<R> lh = loc(f, h);
  R nh = std::fabs(lh.z), vh = gmax(dot(v, h), R(0));
  if (nh <= R(0) || vh <= R(0)) return R(0);
  R ax, ay;
  alpha(c.rough, c.aniso, ax, ay);
  return d_an(ax, ay, lh) * nh / gmax(R(4) * vh, K<R>::e5);
}
template <class R> R slobe_iso(V<R> n, V<R> v, R rough, V<R> d) {
  V<R> h = nrm(v + d);
  R nh = gmax(dot(n, h), R(0)), vh = gmax(dot(v, h), R(0));
  if (nh <= R(0) || vh <= R(0)) return R(0);
  return d_iso(gmax(rough * rough, R(0)), nh) * nh / gmax(R(4) * vh, K<R>::e5);
}
template <class R> R pdf_cc(const Cl<R>& c, V<R> n, V<R> v, V<R> l) {
  return gmax(dot(n, l), R(0)) > R(0) ? slobe_iso(n, v, c.cc_rough, l) : R(0);
}
template <class R> R thick_pdf(const Cl<R>& c, const Fr<R>& f, V<R> n, V<R> v, V<R> l, R io) {
  V<R> lv = loc(f, v);
  R nv = std::fabs(lv.z), nl = std::fabs(loc(f, l).z);
  if (nv <= K<R>::e5 || nl <= K<R>::e5 || dot(n, v) * dot(n, l) >= R(0)) return R(0);
  R eta = io / gmax(R(1), K<R>::e5);
  V<R> h = -nrm(v + l * eta);
  V<R> lh = loc(f, h);
  R vh = dot(v, h), lhh = dot(l, h);
  if (std::fabs(lh.z) <= K<R>::e5 || vh * lhh >= R(0)) return R(0);
  R ax, ay;
  alpha(c.rough, c.aniso, ax, ay);
  return d_an(ax, ay, lh) * (R(1) / (R(1) + lam_an(ax, ay, lv))) *
         (eta * eta * std::fabs(vh) * std::fabs(lhh) / gmax(pw(vh + eta * lhh, R(2)) * nv, K<R>::e5));
}
template <class R> R pdf_dt(const Cl<R>& c, const Fr<R>& f, V<R> n, V<R> v, V<R> l) {  // kernel:2210-2272
  TC<R> k = tcoef(c, n, v);
  if (dot(n, v) * dot(n, l) < R(0)) {
    R pt = gmax(k.pt, K<R>::e5);
    R lobe = c.thin > R(0.5) ? slobe(c, f, v, flip(l, n)) : thick_pdf(c, f, n, v, l, c.ior);
    return gmax(pt * lobe, K<R>::e5);
  }
  return gmax(sat(k.pr) * slobe(c, f, v, l), K<R>::e5);
}
template <class R> R thin_base_p(const Cl<R>& c, V<R> n, V<R> v) {
  return sat(R(1) - max3(schlick(tsc(c), tsf(c), gmax(std::fabs(dot(n, v)), K<R>::e5))));
}
template <class R> R tblw(const Cl<R>& c) { return gmax(c.dw + c.sw + c.dtw + c.tw, K<R>::e5); }
template <class R> R vfm(const Cl<R>& c, V<R> n, V<R> v) {
  return max3(schlick(c.f0, vs(c.f90), gmax(dot(n, v), R(0))));
}
template <class R> R pdf_f(const Cl<R>& c, const Fr<R>& f, V<R> n, V<R> v, V<R> d) {
  R nd = dot(n, d);
  R nl = gmax(nd, R(0)), cnl = gmax(dot(n, d), R(0));
  bool ts = dot(n, v) * nd < R(0);
  bool thin = thin_td(c);
  R tb = thin ? thin_base_p(c, n, v) : R(0);
  R tsp = thin ? R(1) - tb : R(0);
  R pdt = gmax(dot(-n, d), R(0)) * K<R>::kInvPi;
  if (ts) {
    R p;
    if (thin) {
      R b = tblw(c);
      p = c.dtw > R(0) ? tb * (c.dtw / b) * pdt : R(0);
      if (c.tw > R(0)) p = p + tb * (c.tw / b) * slobe(c, f, v, flip(d, n));
      return p > R(0) ? gmax(p, K<R>::e5) : R(0);
    }
    R t = gmax(c.dtw + c.tw, K<R>::e5);
    p = c.dtw > R(0) ? c.dtw / t * pdt : R(0);
    if (c.tw > R(0)) p = p + c.tw / t * pdf_dt(c, f, n, v, d);
    return p > R(0) ? gmax(p, K<R>::e5) : R(0);
  }
  if (nl <= R(0)) return R(0);
  R pd = nl * K<R>::kInvPi;
  if (thin) {
    R b = tblw(c);
    R tot = gmax(tb + tsp + c.cc_w, K<R>::e5);
    R a = tb * c.dw / b / tot * pd, s = tb * c.sw / b / tot * pd;
    R sp = tsp / tot * slobe(c, f, v, d);
    R cw = c.cc_w / tot;
    R cc = cnl > R(0) ? pdf_cc(c, n, v, d) : R(0);
    return gmax(a + s + sp + cw * cc, K<R>::e5);
  }
  R vf = vfm(c, n, v);
  R om = R(1) - vf;
  R dw = c.dw * om, sw = c.sw * om;
  R spw = c.spec_w + c.diel_w * (R(1) - c.transp) * vf;
  R tot = gmax(dw + sw + c.dtw + spw + c.tw + c.cc_w, K<R>::e5);
  R a = dw / tot * pd, s = sw / tot * pd, sp = spw / tot * slobe(c, f, v, d);
  R tr = c.tw > R(0) ? c.tw / tot * pdf_dt(c, f, n, v, d) : R(0);
  R cw = c.cc_w / tot;
  R cc = cnl > R(0) ? pdf_cc(c, n, v, d) : R(0);
  return gmax(a + s + sp + tr + cw * cc, K<R>::e5);
}
template <class R> R pdf(const Cl<R>& c, V<R> n, V<R> v, V<R> d) { return pdf_f(c, frame(n, c.at), n, v, d); }

// sampling (kernel:2625-3567)
template <class R> struct Smp {
  V<R> dir;
  R pdf = 0;
  V<R> w;
  R spec = 0, crossed = 0, next = 1;
};
template <class R> void onb(V<R> n, V<R>& t, V<R>& b) {  // kernel:2625-2650
  R sg = n.z >= R(0) ? R(1) : R(-1);
  R a = R(-1) / (sg + n.z);
  R bb = n.x * n.y * a;
  t = nrm(v3<R>(R(1) + sg * n.x * n.x * a, sg * bb, -sg * n.x));
  b = nrm(v3<R>(bb, sg + n.y * n.y * a, -n.y));
}
template <class R> V<R> cosine(V<R> n, R u0, R u1) {  // kernel:2662-2676
  R r = std::sqrt(u0), phi = R(6.28318548202514648) * u1;
  R x = r * std::cos(phi), y = r * std::sin(phi), z = std::sqrt(gmax(R(0), R(1) - u0));
  V<R> t, b;
  onb(n, t, b);
  return nrm(t * x + b * y + n * z);
}
template <class R> V<R> ggx_h(const Cl<R>& c, const Fr<R>& f, R u0, R u1) {  // kernel:2806-2826
  R ax, ay;
  alpha(c.rough, c.aniso, ax, ay);
  R phi = R(6.28318548202514648) * u1;
  R sp = std::sin(phi), cp = std::cos(phi);
  R ct = R(1) / std::sqrt(R(1) + u0 / gmax(R(1) - u0, K<R>::e6) /
                                     gmax(cp * cp / gmax(ax * ax, K<R>::e12) + sp * sp / gmax(ay * ay, K<R>::e12), K<R>::e6));
  R st = std::sqrt(gmax(R(0), R(1) - ct * ct));
  return nrm(f.t * (st * cp) + f.b * (st * sp) + f.n * ct);
}
template <class R> V<R> ggx_h_iso(V<R> n, R rough, R u0, R u1) {  // kernel:3165-3182
  R a = gmax(rough * rough, R(0));
  R phi = R(6.28318548202514648) * u1;
  R ct = std::sqrt((R(1) - u0) / gmax(R(1) + (a * a - R(1)) * u0, K<R>::e6));
  R st = std::sqrt(gmax(R(0), R(1) - ct * ct));
  V<R> t, b;
  onb(n, t, b);
  return nrm(t * (st * std::cos(phi)) + b * (st * std::sin(phi)) + n * ct);
}
template <class R> R hpdf(const Cl<R>& c, const Fr<R>& f, V<R> h) {
  V<R> lh = loc(f, h);
  R nh = std::fabs(lh.z);
  if (nh <= K<R>::e5) return R(0);
  R ax, ay;
  alpha(c.rough, c.aniso, ax, ay);
  return d_an(ax, ay, lh) * nh;
}
template <class R> V<R> srefract(V<R> i, V<R> n, R eta) {
  R ni = dot(n, i);
  R k = R(1) - eta * eta * (R(1) - ni * ni);
  if (k <= R(0)) return vs(R(0));
  return eta * i - (eta * ni + std::sqrt(k)) * n;
}
template <class R> Smp<R> sample_dt(const Cl<R>& c, const Fr<R>& f, V<R> n, V<R> v, R u0, R u1, R ev) {  // kernel:2881-3145
  Smp<R> s;
  if (c.thin < R(0.5) && std::fabs(R(1) - c.ior) <= K<R>::e4) {
    s.dir = -v; s.pdf = R(1); s.w = wtc(c); s.spec = R(2); s.crossed = R(1); s.next = c.ior;
    return s;
  }
  V<R> h = ggx_h(c, f, u0, u1);
  TC<R> k = tcoef(c, n, v);
  R hp = hpdf(c, f, h);
  R pr = sat(k.pr), pt = gmax(k.pt, K<R>::e5);
  s.crossed = R(0);
  s.next = R(1);
  if (ev <= pr) {
    V<R> d = reflect(-v, h);
    R lobe = hp / gmax(R(4) * std::fabs(dot(d, h)), K<R>::e5);
    s.dir = d; s.pdf = gmax(pr * lobe, K<R>::e5); s.w = diel_spec(c, f, n, v, d) / s.pdf; s.spec = R(1);
    return s;
  }
  if (c.thin > R(0.5)) {
    V<R> d = flip(reflect(-v, h), n);
    R lobe = hp / gmax(R(4) * std::fabs(dot(d, h)), K<R>::e5);
    s.dir = d; s.pdf = gmax(pt * lobe, K<R>::e5); s.w = thin_trans(c, f, n, v, d) / s.pdf; s.spec = R(1);
    return s;
  }
  bool disp = c.disp > K<R>::e5;
  R cu = gclamp((ev - pr) / gmax(pt, K<R>::e5), R(0), R(0.99999898672103882));
  V<R> mask = vs(R(1));
  if (disp) mask = cu < R(0.3333333432674408) ? v3<R>(1, 0, 0) : (cu < R(0.66666668653488159) ? v3<R>(0, 1, 0) : v3<R>(0, 0, 1));
  R ti = disp ? dot(disp_iors(c), mask) : c.ior;
  R cp = disp ? R(0.3333333432674408) : R(1);
  V<R> rf = srefract(-v, h, R(1) / gmax(ti, K<R>::e5));
  if (len(rf) <= K<R>::e5) {
    V<R> d = reflect(-v, h);
    s.dir = d; s.pdf = gmax(pdf_dt(c, f, n, v, d), K<R>::e5); s.w = diel_spec(c, f, n, v, d) / s.pdf; s.spec = R(3);
    return s;
  }
  R vh = dot(v, h), rh = dot(rf, h);
  R lobe = hp * (ti * ti) * std::fabs(rh) / gmax(pw(R(1) * vh + ti * rh, R(2)), K<R>::e5);
  R ax, ay;
  alpha(c.rough, c.aniso, ax, ay);
  R g1 = R(1) / (R(1) + lam_an(ax, ay, loc(f, rf)));
  V<R> eff = k.trans;
  if (c.irid > K<R>::e5) eff = (vs(R(1)) - film_fresnel(c, std::fabs(vh), fresnel_d(std::fabs(vh), c.f0, c.f90, ti))) * wtc(c);
  R pc = pt * cp;
  s.dir = rf; s.pdf = gmax(pc * lobe, K<R>::e5); s.w = eff * mask / gmax(pc, K<R>::e5) * g1;
  s.spec = R(1); s.crossed = R(1); s.next = c.ior;
  return s;
}
template <class R> Smp<R> finish(const Cl<R>& c, const Fr<R>& f, V<R> n, V<R> v, V<R> d, R spec, R u0, R u1, bool thin,
                                 R crossed, R next) {
  Smp<R> s;
  s.crossed = crossed;
  s.next = next;
  R nd = dot(n, d);
  R nl = gmax(nd, R(0)), cnl = gmax(dot(n, d), R(0));
  if (nl <= R(0)) {
    if (nd < R(0)) {
      R mp = pdf_f(c, f, n, v, d);
      s.dir = d; s.pdf = gmax(mp, K<R>::e5); s.w = dtrans(c, n, d) / gmax(s.pdf, K<R>::e5); s.spec = R(0);
      return s;
    }
    V<R> fd = cosine(n, u0, u1);
    s.dir = fd; s.pdf = gmax(gmax(dot(n, fd), R(0)) * K<R>::kInvPi, K<R>::e5); s.w = vs(R(0)); s.spec = R(0);
    s.next = R(1);
    return s;
  }
  s.next = R(1);
  R mp = pdf_f(c, f, n, v, d);
  V<R> b = refl_base(c, f, n, v, d) / gmax(nl, K<R>::e5);
  V<R> cc = cnl > R(0) ? clearcoat(c, n, v, d) / gmax(cnl, K<R>::e5) : vs(R(0));
  R bw = cc_base(c, n, v, d);
  s.dir = d;
  s.pdf = mp;
  s.w = thin ? (b * bw + cc) * nl / gmax(mp, K<R>::e5) : (b * bw + cc) * std::fabs(nd) / mp;
  s.spec = spec;
  return s;
}
template <class R> Smp<R> sample(const Cl<R>& c, V<R> n, V<R> v, R ch, R u0, R u1, R ev) {  // kernel:3200-3567
  Fr<R> f = frame(n, c.at);
  if (thin_td(c)) {
    R tb = thin_base_p(c, n, v), ts = R(1) - tb, b = tblw(c);
    R tot = gmax(tb + ts + c.cc_w, K<R>::e5);
    R pd = tb * (c.dw / b) / tot, ps = tb * (c.sw / b) / tot, pdt = tb * (c.dtw / b) / tot;
    R ptt = tb * (c.tw / b) / tot, psp = ts / tot;
    V<R> d;
    R sp;
    if (ch < pd) { d = cosine(n, u0, u1); sp = R(0); }
    else if (ch < pd + ps) { d = cosine(n, u0, u1); sp = R(0); }
    else if (ch < pd + ps + pdt) { d = cosine(-n, u0, u1); sp = R(0); }
    else if (ch < pd + ps + pdt + ptt) {
      Smp<R> s = sample_dt(c, f, n, v, u0, u1, R(1));
      R mp = pdf_f(c, f, n, v, s.dir);
      s.pdf = mp;
      s.w = diel_trans(c, f, n, v, s.dir) / gmax(mp, K<R>::e5);
      s.crossed = R(0);
      s.next = R(1);
      return s;
    } else if (ch < pd + ps + pdt + ptt + psp) { d = reflect(-v, ggx_h(c, f, u0, u1)); sp = R(1); }
    else { d = reflect(-v, ggx_h_iso(n, c.cc_rough, u0, u1)); sp = R(1); }
    return finish(c, f, n, v, d, sp, u0, u1, true, R(0), R(1));
  }
  R vf = vfm(c, n, v);
  R om = R(1) - vf;
  R dw = c.dw * om, sw = c.sw * om;
  R spw = c.spec_w + c.diel_w * (R(1) - c.transp) * vf;
  R bw = dw + sw + c.dtw;
  R tot = gmax(bw + spw + c.tw + c.cc_w, K<R>::e5);
  R pb = bw / tot, psp = spw / tot, ptr = c.tw / tot;
  V<R> d;
  R sp;
  R crossed = R(0), next = R(1);
  if (ch < pb) {
    R bu = ch / gmax(pb, K<R>::e5);
    R pdr = bw > R(0) ? dw / bw : R(0);
    R psr = bw > R(0) ? sw / bw : R(0);
    if (bu < pdr) { d = cosine(n, u0, u1); sp = R(0); }
    else if (bu < pdr + psr) { d = cosine(n, u0, u1); sp = R(0); }
    else {
      d = cosine(-n, u0, u1); sp = R(0);
      bool thick = c.thin < R(0.5);
      crossed = thick ? R(1) : R(0);
      next = thick ? c.ior : R(1);
    }
  } else if (ch < pb + psp) {
    d = reflect(-v, ggx_h(c, f, u0, u1)); sp = R(1);
  } else if (ch < pb + psp + ptr) {
    Smp<R> s = sample_dt(c, f, n, v, u0, u1, ev);
    s.w = s.w / gmax(ptr, K<R>::e5);
    if (s.pdf < R(1)) s.pdf = s.pdf * ptr;
    return s;
  } else {
    d = reflect(-v, ggx_h_iso(n, c.cc_rough, u0, u1)); sp = R(1);
  }
  return finish(c, f, n, v, d, sp, u0, u1, false, crossed, next);
}

// ---------------------------------------------------------------------------------
// hit set-up: fillRenderState (renderer.frag:72-91) + configure_gltf_material
// (material.glsl:5-110) for untextured materials (texture values are vec4(1))
template <class R>
struct Surf {
  Cl<R> c;
  V<R> n, ng, emissive, att_color;
  R att_dist, cutout;
  bool back, thin;
};

template <class R>
Surf<R> configure(const float* m, V<R> n, V<R> ng, R t[4], V<R> wi, R vc[4], bool lean) {
  GMat<R> g;
  g.base = v3<R>(m[0], m[1], m[2]);
  R opacity = R(1);
  if (std::sqrt(vc[0] * vc[0] + vc[1] * vc[1] + vc[2] * vc[2] + vc[3] * vc[3]) > R(0)) {
    g.base = g.base * v3<R>(vc[0], vc[1], vc[2]);
    opacity = opacity * vc[3];
  }
  Surf<R> S;
  R cut = R(m[8]) * opacity;
  if (R(m[27]) > R(0)) cut = cut < R(m[27]) ? R(0) : R(1);
  if (R(m[27]) == R(1)) cut = R(1);
  g.metallic = m[3]; g.roughness = m[4]; g.aniso = m[5]; g.transmission = m[7]; g.ior = m[11];
  g.spec_color = v3<R>(m[12], m[13], m[14]); g.specular = m[15];
  g.sheen = v3<R>(m[16], m[17], m[18]); g.sheen_rough = m[19];
  g.clearcoat = m[24]; g.cc_rough = m[25]; g.dt = m[26];
  g.dt_color = v3<R>(m[60], m[61], m[62]);
  bool thin = m[35] > 0.5f;
  g.thickness = thin ? R(0) : R(1);
  g.irid = m[40]; g.irid_ior = m[41]; g.irid_thick = mix(R(m[42]), R(m[43]), R(1));
  g.dispersion = m[64];
  bool back = false;  // fix_normals (utils.glsl:79-89)
  if (dot(wi, ng) < R(0)) { ng = -ng; back = true; }
  if (dot(ng, n) < R(0)) n = -n;
  R rot = std::atan2(R(m[37]), R(m[36])) + K<R>::PI;  // material.glsl:84-93
  V<R> t3 = v3<R>(t[0], t[1], t[2]);
  if (rot > R(0)) t3 = t3 * std::cos(rot) + (cross(n, t3) * t[3]) * std::sin(rot);  // utils.glsl:179-186
  S.c = closure(g, t3, lean);
  S.n = n; S.ng = ng; S.emissive = v3<R>(m[20], m[21], m[22]); S.att_color = v3<R>(m[28], m[29], m[30]);
  S.att_dist = m[31]; S.cutout = cut; S.back = back; S.thin = thin;
  return S;
}

template <class R>
Surf<R> fill_state(const Scene& s, int tri, R bu, R bv, V<R> wi, bool lean) {
  const uint32_t* ix = s.idx + 3 * size_t(tri);
  const float* v0 = s.verts + size_t(ix[0]) * 20;
  const float* v1 = s.verts + size_t(ix[1]) * 20;
  const float* v2 = s.verts + size_t(ix[2]) * 20;
  auto at = [](const float* v, int o) { return v3<R>(v[o], v[o + 1], v[o + 2]); };
  V<R> p0 = at(v0, 0), p1 = at(v1, 0), p2 = at(v2, 0);
  V<R> ng = nrm(cross(p1 - p0, p2 - p0));  // utils.glsl:172-176
  R w0 = R(1) - bu - bv;
  V<R> n = nrm(w0 * at(v0, 4) + bu * at(v1, 4) + bv * at(v2, 4));
  R hand = (v0[15] == v1[15] && v0[15] == v2[15]) ? R(v0[15]) : R(0);  // bvh.glsl:125-134
  V<R> tg = nrm(w0 * at(v0, 12) + bu * at(v1, 12) + bv * at(v2, 12));
  R t[4];
  if (len(tg) > R(0.99) && std::fabs(hand) > R(0.99)) { t[0] = tg.x; t[1] = tg.y; t[2] = tg.z; t[3] = -hand; }
  else {
    V<R> o = nrm(cross(n, v3<R>(-n.z, n.x, -n.y)));  // get_onb (utils.glsl:97-102)
    t[0] = o.x; t[1] = o.y; t[2] = o.z; t[3] = R(1);
  }
  R vc[4];
  for (int k = 0; k < 4; ++k) vc[k] = w0 * R(v0[16 + k]) + bu * R(v1[16 + k]) + bv * R(v2[16 + k]);
  uint32_t mat = uint32_t(v0[3]);
  return configure<R>(s.mats + size_t(mat) * 68, n, ng, t, wi, vc, lean);
}

// ---------------------------------------------------------------------------------
// environment (lighting.glsl:24-98, utils.glsl:125-154)
struct Params {
  float view[16];
  float fov, near_plane;
  int width, height;
  int max_bounces, use_ibl, bg_from_ibl, rr_start, env_mode, lean, pcg;
  float ibl_rot_deg, bg[4], ray_eps, clamp, rr_prob;
  uint64_t seed;
  float pl_pos[4], pl_emis[4];  // u_point_light_position / _emission; w > 0.5 enables
};

template <class R> V<R> rot_phi(V<R> d, R a) {
  return v3<R>(std::cos(a) * d.x - std::sin(a) * d.z, d.y, std::sin(a) * d.x + std::cos(a) * d.z);
}
template <class R> R theta_pdf(R th) { return R(1) / (R(2) * K<R>::PI * K<R>::PI * gmax(K<R>::EPS_COS, std::sin(th))); }
template <class R> void dir_uv(V<R> d, R& u, R& v, R& p) {
  R th = std::acos(gmax(R(-1), gmin(R(1), d.y)));
  R ph = std::atan2(d.z, d.x);
  if (ph < R(0)) ph = K<R>::TWO_PI + ph;
  u = ph / K<R>::TWO_PI;
  v = th / K<R>::PI;
  p = theta_pdf(th);
}
template <class R> V<R> uv_dir(R u, R v, R& p) {
  R th = v * K<R>::PI, ph = u * K<R>::TWO_PI;
  p = theta_pdf(th);
  return v3<R>(std::sin(th) * std::cos(ph), std::cos(th), std::sin(th) * std::sin(ph));
}
template <class R> V<R> texel(const Ibl& I, int x, int y) {
  const float* t = I.rgba + (size_t(y) * I.w + x) * 4;
  return v3<R>(t[0], t[1], t[2]);
}
inline int wrapi(int i, int n) { int m = i % n; return m < 0 ? m + n : m; }
template <class R> V<R> bilinear(const Ibl& I, R u, R v) {  // texture(), LINEAR + REPEAT
  R fu = u * R(I.w) - R(0.5), fv = v * R(I.h) - R(0.5);
  R u0 = std::floor(fu), v0 = std::floor(fv);
  R a = fu - u0, b = fv - v0;
  int i0 = wrapi(int(u0), I.w), j0 = wrapi(int(v0), I.h), i1 = wrapi(int(u0) + 1, I.w), j1 = wrapi(int(v0) + 1, I.h);
  return (R(1) - a) * (R(1) - b) * texel<R>(I, i0, j0) + a * (R(1) - b) * texel<R>(I, i1, j0) +
         (R(1) - a) * b * texel<R>(I, i0, j1) + a * b * texel<R>(I, i1, j1);
}
template <class R> V<R> ibl_eval(const Ibl& I, R rot, V<R> d) {
  R u, v, p;
  dir_uv(rot_phi(d, rot), u, v, p);
  return bilinear(I, u, v);
}
inline int lbound(const float* data, int size, double value) {
  int count = size, first = 0;
  while (count > 0) {
    int step = count / 2, idx = first + step;
    if (double(data[idx]) < value) { first = idx + 1; count -= step + 1; }
    else count = step;
  }
  return first;
}
template <class R> V<R> ibl_sample(const Ibl& I, R rot, int mode, R r0, R r1, R& pdf_out) {
  int x, y;
  R py, px;
  if (mode == 1) {  // sampleRow1D x2 (lighting.glsl:24-42)
    int yi = lbound(I.ycdf.data(), I.h, double(r1));
    py = yi < I.h ? R(I.ypdf[yi]) : R(0);
    y = yi >= I.h ? I.h - 1 : yi;
    int xi = lbound(I.cdf.data() + size_t(y) * I.w, I.w, double(r0));
    px = xi < I.w ? R(I.pdf[size_t(y) * I.w + xi]) : R(0);
    x = xi >= I.w ? I.w - 1 : xi;
  } else {  // alias table over the same pmf
    int n = I.w * I.h;
    int i = std::min(int(float(r1) * float(n)), n - 1);
    if (float(r0) >= I.alias_prob[i]) i = I.alias_idx[i];
    y = i / I.w;
    x = i - y * I.w;
    py = R(I.ypdf[y]);
    px = R(I.pdf[i]);
  }
  R sp = R(I.w) * R(I.h) * py * px;
  R pw_;
  V<R> d = uv_dir(R(x) / R(I.w), R(y) / R(I.h), pw_);
  pdf_out = sp * pw_;
  return rot_phi(d, -rot);
}
template <class R> R ibl_pdf(const Ibl& I, R rot, V<R> d) {
  R u, v, pw_;
  dir_uv(rot_phi(d, rot), u, v, pw_);
  R w = R(I.w), h = R(I.h);
  R x = gmin(u * w, w - R(1)), y = gmin(v * h, h - R(1));
  int xi = int(x), yi = int(y);
  R py = (yi >= 0 && yi < I.h) ? R(I.ypdf[yi]) : R(0);
  R px = (xi >= 0 && yi >= 0 && xi < I.w && yi < I.h) ? R(I.pdf[size_t(yi) * I.w + xi]) : R(0);
  return w * h * py * px * pw_;
}

// ---------------------------------------------------------------------------------
// camera (renderer.frag:129-142) and integrator (misptdl.glsl:2-93)
template <class R>
void camera_ray(const Params& P, int px, int py, R r0, R r1, V<R>& o, V<R>& d) {
  R vx = R(2 * px + 1) / R(P.width) - R(1), vy = R(2 * py + 1) / R(P.height) - R(1);
  R irx = R(float(1.0 / P.width)), iry = R(float(1.0 / P.height));
  R film = R(float(std::tan(double(P.fov) * 0.5 * M_PI / 180.0) * double(P.near_plane)));
  R ox = r0 * irx, oy = r1 * iry;
  R aspect = iry / irx;
  R ux = (vx * aspect + ox) * film, uy = (vy * R(1) + oy) * film;
  V<R> dv = nrm(v3<R>(ux, uy, -R(P.near_plane)));
  const float* m = P.view;
  d = v3<R>(m[0], m[1], m[2]) * dv.x + v3<R>(m[4], m[5], m[6]) * dv.y + v3<R>(m[8], m[9], m[10]) * dv.z;
  o = v3<R>(m[12], m[13], m[14]);
}

template <class R>
void trace_path(const Scene& s, const Ibl* I, const Params& P, int px, int py, uint32_t frame, R out[4],
                TraversalStats* ts) {
  Rng<R> rng;
  if (P.pcg) rng.pcg_init(P.seed, uint64_t(frame) * uint64_t(P.width) * uint64_t(P.height) + uint64_t(py) * P.width + px);
  else rng.mwc_init(int(frame) * P.max_bounces, px, py);
  R rot = R(float(double(P.ibl_rot_deg) / 180.0 * M_PI));
  R r0 = rng.next(), r1 = rng.next();
  V<R> o, d;
  camera_ray(P, px, py, r0, r1, o, d);
  V<R> w = vs(R(1)), L = vs(R(0));
  R last_pdf = R(0);
  Hit<R> h;
  if (!closest_hit(s, o, d, K<R>::TFAR_MAX, h, ts)) {
    if (P.bg_from_ibl) {
      V<R> c = I ? ibl_eval(*I, rot, d) * w : vs(R(0));
      out[0] = c.x; out[1] = c.y; out[2] = c.z; out[3] = R(1);
    } else {
      out[0] = pw(R(P.bg[0]), R(2.2)); out[1] = pw(R(P.bg[1]), R(2.2)); out[2] = pw(R(P.bg[2]), R(2.2)); out[3] = P.bg[3];
    }
    return;
  }
  R rr_factor = R(1) / (R(1) - R(P.rr_prob));
  int bounce = 0;
  auto finish = [&](bool clampit) {
    if (clampit && R(P.clamp) > R(0)) {
      out[0] = gclamp(L.x, R(0), R(P.clamp)); out[1] = gclamp(L.y, R(0), R(P.clamp)); out[2] = gclamp(L.z, R(0), R(P.clamp));
    } else {
      out[0] = L.x; out[1] = L.y; out[2] = L.z;
    }
    out[3] = R(1);
  };
  // last_bounce_specular reads the event_type that configure_gltf_material
  // leaves zero-initialised (material.glsl never assigns it, and WebGL
  // zero-initialises locals), so it is false at every bounce: NEE runs on
  // every bounce and the env MIS weight always applies (misptdl.glsl:68-86).
  while (bounce < P.max_bounces) {
    w = w * rr_factor;
    if (bounce > P.rr_start && rng.next() <= R(P.rr_prob)) break;
    V<R> wi = -d;
    V<R> pos = o + d * h.t;
    Surf<R> S = fill_state<R>(s, h.tri, h.u, h.v, wi, P.lean != 0);
    if (S.back && !S.thin) w = w * vexp(-(-vlog(S.att_color) / S.att_dist) * h.t);
    L = L + S.emissive * R(1) * w;
    V<R> wo = -wi, bw = vs(R(1));
    R p = R(1);
    if (rng.next() > S.cutout) {
      wo = -wi;
    } else {
      R u0 = rng.next(), u1 = rng.next(), u2 = rng.next(), comp = rng.next();
      Smp<R> sm = sample(S.c, S.n, wi, comp, u0, u1, u2);
      wo = sm.dir; p = sm.pdf; bw = sm.w;
      if (p < K<R>::EPS_PDF) { finish(false); return; }
    }
    pos = pos + (dot(S.ng, wo) < R(0) ? -S.ng : S.ng) * R(P.ray_eps);
    R q0 = rng.next(), q1 = rng.next();
    V<R> Ld = vs(R(0));
    V<R> nn = S.back ? -S.n : S.n;
    if (P.use_ibl > 0 && I) {
      R ip;
      V<R> ld = ibl_sample(*I, rot, P.env_mode, q0, q1, ip);
      R cnl = sat(dot(ld, nn));
      if (cnl > K<R>::EPS_COS && ip > K<R>::EPS_PDF) {
        Hit<R> sh;
        if (!closest_hit(s, pos, nrm(ld), K<R>::TFAR_MAX, sh, ts, true)) {
          V<R> f = eval(S.c, S.n, wi, ld) / gmax(std::fabs(dot(S.n, ld)), K<R>::EPS);
          R bp = pdf(S.c, S.n, wi, ld);
          Ld = ibl_eval(*I, rot, ld) * f * cnl / ip;
          if (bp > K<R>::EPS_PDF) Ld = Ld * (ip / (ip + bp));
        }
      }
    }
    // sampleAndEvaluatePointLight (lighting.glsl:2-22): visibility by a
    // nearest-hit ray bounded by the light distance (bvh.glsl:218-223)
    if (P.pl_pos[3] > 0.5f) {
      V<R> lp = v3<R>(R(P.pl_pos[0]), R(P.pl_pos[1]), R(P.pl_pos[2]));
      V<R> ld = lp - pos;
      R dist2 = dot(ld, ld);
      V<R> ldn = nrm(ld);
      R cnl = sat(dot(ldn, nn));
      Hit<R> sh;
      bool visible = !closest_hit(s, pos, ldn, std::sqrt(dist2), sh, ts, true);
      if (cnl > K<R>::EPS_COS && visible) {
        V<R> f = eval(S.c, S.n, wi, ldn) / gmax(std::fabs(dot(S.n, ldn)), K<R>::EPS);
        V<R> e = v3<R>(R(P.pl_emis[0]), R(P.pl_emis[1]), R(P.pl_emis[2]));
        Ld = Ld + f * (e / dist2) * cnl;
      }
    }
    L = L + Ld * w;
    w = w * bw;
    last_pdf = p;
    o = pos;
    d = wo;
    if (closest_hit(s, o, d, K<R>::TFAR_MAX, h, ts)) {
      ++bounce;
    } else {
      if (I) {
        R ip = ibl_pdf(*I, rot, d);
        R mis = last_pdf / (last_pdf + ip);
        L = L + ibl_eval(*I, rot, d) * w * mis * R(P.use_ibl);
      }
      break;
    }
  }
  finish(true);
}

}  // namespace orc

// ---------------------------------------------------------------------------------
// C ABI for the test harness
namespace {
orc::Scene g_scene;
orc::Ibl g_ibl;
bool g_has_ibl = false;
std::vector<float> g_rgba;

template <class R>
void render_impl(const orc::Params& P, int n, const int32_t* xy, uint32_t frame, float* out, int threads,
                 uint64_t* counters) {
  threads = std::max(1, threads);
  std::vector<std::thread> pool;
  std::vector<orc::TraversalStats> st(threads);
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([&, t] {
      for (int i = t; i < n; i += threads) {
        R o[4];
        orc::trace_path<R>(g_scene, g_has_ibl ? &g_ibl : nullptr, P, xy[2 * i], xy[2 * i + 1], frame, o,
                           counters ? &st[t] : nullptr);
        for (int k = 0; k < 4; ++k) out[4 * size_t(i) + k] = float(o[k]);
      }
    });
  for (auto& th : pool) th.join();
  if (counters) {
    for (auto& s : st) { counters[0] += s.rays; counters[1] += s.nodes; counters[2] += s.tris; counters[3] += s.aborted; }
  }
}

template <class R>
void bsdf_impl(int n, const float* hit, const float* wo3, const float* rnd, int lean, float* eval4, float* sample10,
               int32_t* flags) {
  for (int i = 0; i < n; ++i) {
    const float* h = hit + 20 * size_t(i);
    using V = orc::V<R>;
    V nn = orc::v3<R>(h[0], h[1], h[2]), ng = orc::v3<R>(h[3], h[4], h[5]), wi = orc::v3<R>(h[10], h[11], h[12]);
    R t[4] = {h[6], h[7], h[8], h[9]};
    R vc[4] = {h[15], h[16], h[17], h[18]};
    uint32_t m = uint32_t(h[19]);
    orc::Surf<R> S = orc::configure<R>(g_scene.mats + size_t(m) * 68, nn, ng, t, wi, vc, lean != 0);
    V wo = orc::v3<R>(wo3[3 * i], wo3[3 * i + 1], wo3[3 * i + 2]);
    V e = orc::eval(S.c, S.n, wi, wo);
    R p = orc::pdf(S.c, S.n, wi, wo);
    eval4[4 * i] = float(e.x); eval4[4 * i + 1] = float(e.y); eval4[4 * i + 2] = float(e.z); eval4[4 * i + 3] = float(p);
    const float* r = rnd + 4 * size_t(i);
    orc::Smp<R> s = orc::sample(S.c, S.n, wi, R(r[0]), R(r[1]), R(r[2]), R(r[3]));
    float* o = sample10 + 10 * size_t(i);
    o[0] = float(s.dir.x); o[1] = float(s.dir.y); o[2] = float(s.dir.z); o[3] = float(s.pdf);
    o[4] = float(s.w.x); o[5] = float(s.w.y); o[6] = float(s.w.z);
    o[7] = float(s.spec); o[8] = float(s.crossed); o[9] = float(s.next);
    flags[i] = S.back ? 1 : 0;
  }
}
}  // namespace

extern "C" {

int orc_set_scene(const float* vertices, int nverts, const uint32_t* indices, int nidx, const float* materials,
                  int nmat, const float* nodes, int nnodes, const int32_t* remap, int nremap) {
  if (nverts <= 0 || nidx <= 0 || nidx % 3 || nmat <= 0) return -1;
  g_scene = orc::Scene{vertices, indices, materials, nodes, remap, nverts, nidx / 3, nmat, nnodes, nremap};
  return 0;
}

int orc_set_ibl(const float* rgba, int w, int h) {
  if (w <= 0 || h <= 0) return -1;
  g_rgba.assign(rgba, rgba + size_t(w) * h * 4);
  orc::build_ibl(g_ibl, g_rgba.data(), w, h);
  g_has_ibl = true;
  return 0;
}

void orc_get_ibl_tables(float* pdf, float* cdf, float* ypdf, float* ycdf, double* total, float* alias_prob,
                        int32_t* alias_idx) {
  std::copy(g_ibl.pdf.begin(), g_ibl.pdf.end(), pdf);
  std::copy(g_ibl.cdf.begin(), g_ibl.cdf.end(), cdf);
  std::copy(g_ibl.ypdf.begin(), g_ibl.ypdf.end(), ypdf);
  std::copy(g_ibl.ycdf.begin(), g_ibl.ycdf.end(), ycdf);
  *total = g_ibl.total;
  if (alias_prob) std::copy(g_ibl.alias_prob.begin(), g_ibl.alias_prob.end(), alias_prob);
  if (alias_idx) std::copy(g_ibl.alias_idx.begin(), g_ibl.alias_idx.end(), alias_idx);
}

// rays n x 8 (org, dir, tfar, 0).  mode 0: BVH closest hit, 1: brute force,
// 2: isOccluded (normalised direction).  counters: rays, nodes, tris, aborted.
void orc_f32_trace(int n, const float* rays, int mode, int32_t* tri, float* t, float* uv, uint64_t* counters) {
  orc::TraversalStats ts;
  for (int i = 0; i < n; ++i) {
    const float* r = rays + 8 * size_t(i);
    orc::V<float> o = orc::v3<float>(r[0], r[1], r[2]), d = orc::v3<float>(r[3], r[4], r[5]);
    orc::Hit<float> h;
    bool hit;
    if (mode == 1) hit = orc::brute_force(g_scene, o, d, r[6], h);
    else if (mode == 2) hit = orc::closest_hit(g_scene, o, orc::nrm(d), r[6], h, &ts, true);
    else hit = orc::closest_hit(g_scene, o, d, r[6], h, &ts);
    tri[i] = hit ? h.tri : -1;
    t[i] = h.t;
    uv[2 * i] = hit ? h.u : 0.f;
    uv[2 * i + 1] = hit ? h.v : 0.f;
  }
  if (counters) { counters[0] = ts.rays; counters[1] = ts.nodes; counters[2] = ts.tris; counters[3] = ts.aborted; }
}

void orc_f64_brute_force(int n, const float* rays, int32_t* tri, double* t) {
  for (int i = 0; i < n; ++i) {
    const float* r = rays + 8 * size_t(i);
    orc::Hit<double> h;
    bool hit = orc::brute_force(g_scene, orc::v3<double>(r[0], r[1], r[2]), orc::v3<double>(r[3], r[4], r[5]),
                                double(r[6]), h);
    tri[i] = hit ? h.tri : -1;
    t[i] = h.t;
  }
}

void orc_f32_bsdf(int n, const float* hit, const float* wo, const float* rnd, int lean, float* e, float* s, int32_t* f) {
  bsdf_impl<float>(n, hit, wo, rnd, lean, e, s, f);
}
void orc_f64_bsdf(int n, const float* hit, const float* wo, const float* rnd, int lean, float* e, float* s, int32_t* f) {
  bsdf_impl<double>(n, hit, wo, rnd, lean, e, s, f);
}

void orc_f32_ibl(int n, const float* r2, const float* dirs, float rot_deg, int mode, float* sdp4, float* pdf, float* rgb) {
  float rot = float(double(rot_deg) / 180.0 * M_PI);
  for (int i = 0; i < n; ++i) {
    float p;
    orc::V<float> d = orc::ibl_sample<float>(g_ibl, rot, mode, r2[2 * i], r2[2 * i + 1], p);
    sdp4[4 * i] = d.x; sdp4[4 * i + 1] = d.y; sdp4[4 * i + 2] = d.z; sdp4[4 * i + 3] = p;
    orc::V<float> q = orc::v3<float>(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]);
    pdf[i] = orc::ibl_pdf<float>(g_ibl, rot, q);
    orc::V<float> c = orc::ibl_eval<float>(g_ibl, rot, q);
    rgb[3 * i] = c.x; rgb[3 * i + 1] = c.y; rgb[3 * i + 2] = c.z;
  }
}

void orc_f32_camera_rays(const orc::Params* P, int n, const int32_t* xy, const float* r2, float* rays6) {
  for (int i = 0; i < n; ++i) {
    orc::V<float> o, d;
    orc::camera_ray<float>(*P, xy[2 * i], xy[2 * i + 1], r2[2 * i], r2[2 * i + 1], o, d);
    float* r = rays6 + 6 * size_t(i);
    r[0] = o.x; r[1] = o.y; r[2] = o.z; r[3] = d.x; r[4] = d.y; r[5] = d.z;
  }
}

void orc_rng(int mode_pcg, uint64_t seed, uint64_t stream, int x, int y, int mwc_seed, int n, float* out) {
  orc::Rng<float> r;
  if (mode_pcg) r.pcg_init(seed, stream);
  else r.mwc_init(mwc_seed, x, y);
  for (int i = 0; i < n; ++i) out[i] = r.next();
}

// One sample of the listed pixels at progressive frame `frame` (1-based).
void orc_f32_render(const orc::Params* P, int n, const int32_t* xy, uint32_t frame, float* out, int threads,
                    uint64_t* counters) {
  render_impl<float>(*P, n, xy, frame, out, threads, counters);
}
void orc_f64_render(const orc::Params* P, int n, const int32_t* xy, uint32_t frame, float* out, int threads,
                    uint64_t* counters) {
  render_impl<double>(*P, n, xy, frame, out, threads, counters);
}

}  // extern "C"
