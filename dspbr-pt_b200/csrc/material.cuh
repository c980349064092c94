// DSPBR (Enterprise PBR, "webgl-full" profile) material model on the device.
//
// Behaviour follows the reference's generated kernel
// packages/lib/shader/generated/slang_materials/webgl-full/material_kernel.glsl
// (slang-pbr 0.1.0, analytic energy compensation, absorption-only media) as
// called by the reference's adapter (pbr_material_adapter.glsl:13-71):
//   closure build   kernel:209-261 (surface clamps), :357-422 (lobe weights)
//   eval            kernel:2045-2089 and the lobes it calls
//   pdf             kernel:2413-2617
//   sample          kernel:3200-3567 (+ sampleDielectricTransmission :2881-3145)
// Arithmetic follows the reference term by term so that results stay within
// FP32 rounding of the host oracle.  Device-specific choices:
//   * the closure is built once per hit and held in registers;
//   * the adapter always passes currentMediumIor = 1 (adapter:18), so the
//     "inside medium" branches are folded (ior_i = 1, ior_o = closure ior);
//   * sub-lobe samplers return only the direction / specular flag the mixture
//     sampler keeps (it recomputes pdf and value of the mixture itself);
//   * the shading frame of the anisotropic projection is built once per call.
#pragma once
#include "vecmath.cuh"

namespace dspbr {

constexpr float kPi = 3.14159274101257324f;
constexpr float kTwoPi = 6.28318548202514648f;
constexpr float kInvPi = 0.31830987334251404f;
constexpr float kSchlickAvg = 0.0476190485060215f;  // 1/21
constexpr float kEps5 = 0.00000999999974738f;
constexpr float kEps4 = 0.00009999999747379f;

// PbrGltfMaterial after configure_gltf_material (material.glsl:5-110).
struct GltfMaterial {
  v3 base_color;        // baseColorFactor.rgb
  float metallic, roughness;
  float specular;       // specularFactor
  v3 specular_color;
  float transmission, diffuse_transmission;
  v3 diffuse_transmission_color;
  float ior;
  float clearcoat, clearcoat_roughness;
  v3 sheen_color;
  float sheen_roughness;
  float anisotropy;     // anisotropyStrength
  float iridescence, iridescence_ior, iridescence_thickness;
  float dispersion;
  float thickness;      // thicknessFactor: thin ? 0 : 1
};

// SurfaceClosure_0 (kernel:316-354), fields the eval/pdf/sample paths read.
struct Closure {
  v3 diffuse_reflection_color;
  v3 albedo;                    // transmissionColor = specularColor = albedo
  float diffuse_weight, sheen_weight;
  float anisotropy;
  v3 aniso_tangent;
  v3 dielectric_f0;             // dielectricSpecularColor
  float dielectric_f90;         // dielectricSpecularF90 = vec3(specular)
  float dielectric_weight, specular_weight, clearcoat_weight;
  float roughness;
  v3 sheen_color;
  float sheen_roughness;
  float transparency, clearcoat, clearcoat_roughness;
  float metallic, specular, ior;
  float iridescence, iridescence_ior, iridescence_thickness;
  float dispersion;
  float thin;                   // thinWalled: 1 or 0
  float transmission_weight;
  v3 diffuse_transmission_color;
  float diffuse_transmission_weight;
};

struct BsdfSample {
  v3 dir;
  float pdf;
  v3 weight;                    // bsdfOverPdf
  float specular;
  float crossed;
  float next_ior;
};

// ---- energy approximations (kernel:5-90) -----------------------------------
DEV float avg_albedo_ggx(float alpha) {
  float r = sqrtf(fmaxf(alpha, 0.f));
  return sat(1.f - 0.57999998331069946f * r + 0.07999999821186066f * r * r);
}
DEV float dir_albedo_ggx(float alpha, float cos_t) {
  return sat(1.f - sqrtf(fmaxf(alpha, 0.f)) * (0.5f + 0.5f * pow5(1.f - sat(cos_t))));
}
DEV float avg_albedo_ggx_ms(float alpha, float e0) {
  return sat(sat(e0 + (1.f - e0) * kSchlickAvg) * avg_albedo_ggx(alpha));
}
DEV float dir_albedo_ggx_ms(float theta, float alpha, float e0) {
  float nov = sat(theta);
  return sat(sat(e0 + (1.f - e0) * pow5(1.f - nov)) * mixf(1.f, dir_albedo_ggx(alpha, nov), 0.64999997615814209f));
}

// ---- closure build (kernel:209-261, 357-422) -------------------------------
DEV float iridescence_interface_weight(float irid, float film_ior) {
  float f = fmaxf(film_ior, 1.f);
  float r = (f - 1.f) / fmaxf(f + 1.f, kEps5);
  return sat(irid) * (r * r);
}
DEV v3 schlick_avg(v3 f0, v3 f90) { return f0 + (f90 - f0) * kSchlickAvg; }

DEV Closure build_closure(const GltfMaterial& m, v3 aniso_tangent, bool lean) {
  // buildEnterpriseSurfaceFromGltf_0
  v3 albedo = sat(m.base_color);
  float metallic = sat(m.metallic);
  float roughness = sat(m.roughness);
  float transparency = sat(m.transmission);
  float ior = fmaxf(m.ior, 1.f);
  v3 spec_color = sat(m.specular_color);
  float specular = sat(m.specular);
  float thin = m.thickness > 0.f ? 0.f : 1.f;
  float translucency = sat(m.diffuse_transmission);
  v3 translucency_color = sat(m.diffuse_transmission_color);
  float irid = sat(m.iridescence);
  float irid_ior = clampf(m.iridescence_ior, 1.f, 2.5f);
  float irid_thick = fmaxf(m.iridescence_thickness, 0.f);
  float dispersion = fmaxf(m.dispersion, 0.f);
  float clearcoat = sat(m.clearcoat);
  float cc_rough = sat(m.clearcoat_roughness);
  v3 sheen = sat(m.sheen_color);
  float sheen_rough = sat(m.sheen_roughness);
  float aniso = sat(m.anisotropy);
  if (lean) { irid = 0.f; dispersion = 0.f; }  // webgl-lean profile zeroes both

  // buildSurfaceClosure_0
  Closure c;
  float diel_w = 1.f - metallic;
  float opaque = 1.f - transparency;
  float opaque_diel = diel_w * opaque;
  float transp_diel = diel_w * transparency;
  v3 drc = albedo * opaque_diel * (1.f - translucency);
  v3 dtc = opaque_diel * translucency_color * translucency;
  float ratio = (1.f - ior) / (1.f + ior);
  v3 f0 = sat(mk(ratio * ratio * specular) * spec_color);
  v3 metal_energy = schlick_avg(albedo, mk(1.f));
  float mat_rough = sat(fmaxf(roughness, 0.0020000000949949f));
  float cc_rough_bsdf = sat(fmaxf(cc_rough, 0.0020000000949949f));
  c.diffuse_reflection_color = drc;
  c.albedo = albedo;
  c.diffuse_weight = max3(drc);
  c.sheen_weight = max3(sheen) * opaque;
  c.anisotropy = aniso;
  c.aniso_tangent = aniso_tangent;
  c.dielectric_f0 = f0;
  c.dielectric_f90 = specular;
  c.dielectric_weight = diel_w;
  float film_w = iridescence_interface_weight(irid, irid_ior);
  c.specular_weight = fmaxf(max3(metal_energy), film_w) * metallic;
  c.clearcoat_weight = clearcoat * mixf(0.20000000298023224f, 1.f, 1.f - cc_rough_bsdf);
  c.roughness = mat_rough;
  c.sheen_color = sheen;
  c.sheen_roughness = sheen_rough;
  c.transparency = transparency;
  c.clearcoat = clearcoat;
  c.clearcoat_roughness = cc_rough_bsdf;
  c.metallic = metallic;
  c.specular = specular;
  c.ior = ior;
  c.iridescence = irid;
  c.iridescence_ior = irid_ior;
  c.iridescence_thickness = irid_thick;
  c.dispersion = dispersion;
  c.thin = thin;
  c.transmission_weight = max3(albedo) * transp_diel;
  c.diffuse_transmission_color = dtc;
  c.diffuse_transmission_weight = max3(dtc);
  return c;
}

// ---- Fresnel ----------------------------------------------------------------
DEV v3 schlick(v3 f0, v3 f90, float cos_t) {
  float m = sat(1.f - cos_t);
  float m2 = m * m;
  return f0 + (f90 - f0) * (m2 * m2 * m);
}
DEV float schlick1(float f0, float f90, float cos_t) {
  float m = sat(1.f - cos_t);
  float m2 = m * m;
  return f0 + (f90 - f0) * (m2 * m2 * m);
}
// fresnelSchlickDielectric_0 (kernel:681-707) with n_i = 1 <= n_t: never TIR,
// Schlick at the incident cosine; index-matched interfaces reflect nothing.
DEV v3 fresnel_dielectric(float cos_t, v3 f0, float f90, float nt) {
  if (fabsf(1.f - nt) <= kEps4) return mk(0.f);
  return schlick(f0, mk(f90), sat(cos_t));
}

// ---- thin-film interference (kernel:741-937) --------------------------------
DEV v3 film_sensitivity(float opd_nm, v3 shift) {
  float phase = 6.28318548202514648f * opd_nm * 9.99999971718068537e-10f;
  float phase2 = phase * phase;
  const v3 var = mk(4.327799808e+09f, 9.304599552e+09f, 6.612100096e+09f);
  v3 xyz = mk(5.48560003844900113e-13f, 4.42010008238832852e-13f, 5.24810013155518895e-13f) *
           vsqrt(6.28318548202514648f * var) *
           vcos(mk(1.681e+06f, 1.7953e+06f, 2.2084e+06f) * phase + shift) * vexp(-phase2 * var);
  xyz.x = xyz.x + 9.74699989231449238e-14f * sqrtf(2.845152256e+10f) * cosf(2.2399e+06f * phase + shift.x) *
                      expf(-4.528200192e+09f * phase2);
  xyz = xyz / 1.06850002623559703e-07f;
  return mk(3.24045419692993164f * xyz.x - 1.53713846206665039f * xyz.y - 0.49853140115737915f * xyz.z,
            -0.96926599740982056f * xyz.x + 1.87601077556610107f * xyz.y + 0.04155600070953369f * xyz.z,
            0.05564339831471443f * xyz.x - 0.20402589440345764f * xyz.y + 1.05722522735595703f * xyz.z);
}

DEV float ior_to_f0(float t, float i) {
  float r = (t - i) / fmaxf(t + i, kEps5);
  return r * r;
}
DEV v3 substrate_f0(float ior) { return mk(ior_to_f0(fmaxf(ior, 1.f), 1.f)); }

NOINL v3 film_reflectance(float outside, float film_ior, v3 base_f0, float thick_nm, float cos1) {
  float fi = clampf(film_ior, 1.f, 2.5f);
  float c1 = sat(cos1);
  float c2sq = 1.f - outside / fi * (outside / fi) * (1.f - c1 * c1);
  if (c2sq < 0.f) return mk(1.f);
  float c2 = sqrtf(c2sq);
  float r12 = schlick1(ior_to_f0(fi, outside), 1.f, c1);
  float t121 = 1.f - r12;
  v3 sf0 = vsqrt(vclamp(base_f0, 0.f, 0.99989998340606689f));
  v3 base_ior = (1.f + sf0) / vmax(1.f - sf0, mk(kEps5));
  v3 r1 = (base_ior - fi) / vmax(base_ior + fi, mk(kEps5));
  v3 r23 = schlick(r1 * r1, mk(1.f), c2);
  float opd = 2.f * fi * fmaxf(thick_nm, 0.f) * c2;
  float phi12 = fi < outside ? kPi : 0.f;
  float phi21 = kPi - phi12;
  v3 phi = mk(phi21) + mk(base_ior.x < fi ? kPi : 0.f, base_ior.y < fi ? kPi : 0.f, base_ior.z < fi ? kPi : 0.f);
  v3 r123 = vmin(vmax(r12 * r23, mk(kEps5)), mk(0.99989998340606689f));
  v3 sr123 = vsqrt(r123);
  v3 rs = t121 * t121 * r23 / vmax(1.f - r123, mk(kEps5));
  v3 refl = mk(r12) + rs;
  v3 cm = rs - t121;
#pragma unroll
  for (int m = 1; m <= 2; ++m) {
    cm = cm * sr123;
    float fm = float(m);
    refl = refl + cm * 2.f * film_sensitivity(fm * opd, fm * phi);
  }
  return vmax(refl, mk(0.f));
}

// thinFilmDielectricFresnel_0 with incident ior 1
DEV v3 film_dielectric_fresnel(const Closure& c, float cos_t, v3 regular) {
  if (c.iridescence <= kEps5) return regular;
  v3 film = film_reflectance(1.f, c.iridescence_ior, substrate_f0(c.ior), c.iridescence_thickness, cos_t);
  return vmix(regular, film, sat(c.iridescence));
}

// ---- GGX ---------------------------------------------------------------------
struct Frame {  // projectToAnisotropicFrame_0 basis (kernel:448-454)
  v3 t, b, n;
};
DEV Frame aniso_frame(v3 n, v3 tangent) {
  v3 st = normalize(tangent - n * dot(tangent, n));
  return Frame{st, normalize(cross(n, st)), n};
}
DEV v3 to_local(const Frame& f, v3 d) { return mk(dot(d, f.t), dot(d, f.b), dot(d, f.n)); }

struct Alpha {
  float x, y;
};
DEV Alpha aniso_alpha(float rough, float aniso) {
  float a = sat(aniso);
  float r2 = fmaxf(rough * rough, 0.f);
  return Alpha{mixf(r2, 1.f, a * a), r2};
}
DEV float ggx_d_aniso(Alpha a, v3 h) {
  float hx = h.x / a.x, hy = h.y / a.y;
  float den = hx * hx + hy * hy + h.z * h.z;
  return 1.f / fmaxf(kPi * a.x * a.y * den * den, 9.999999960041972e-13f);
}
DEV float ggx_lambda_aniso(Alpha a, v3 d) {
  float c2 = d.z * d.z;
  if (c2 <= 9.99999993922529029e-09f) return 0.f;
  if (fmaxf(1.f - c2, 0.f) <= 9.99999993922529029e-09f) return 0.f;
  return 0.5f * (-1.f + sqrtf(1.f + (d.x * d.x * a.x * a.x + d.y * d.y * a.y * a.y) /
                                       fmaxf(c2, 9.99999993922529029e-09f)));
}
DEV float ggx_g2_aniso(Alpha a, v3 v, v3 l) { return 1.f / (1.f + ggx_lambda_aniso(a, v) + ggx_lambda_aniso(a, l)); }
DEV float ggx_g1_aniso(Alpha a, v3 d) { return 1.f / (1.f + ggx_lambda_aniso(a, d)); }

// evaluateMicrofacetResponseAnisotropic_0 (kernel:515-586), scalar result
DEV float microfacet_aniso(const Closure& c, const Frame& f, v3 v, v3 l) {
  v3 h = normalize(v + l);
  v3 lv = to_local(f, v), ll = to_local(f, l), lh = to_local(f, h);
  float nov = fabsf(lv.z), nol = fabsf(ll.z), noh = fabsf(lh.z);
  float voh = fmaxf(dot(v, h), 0.f);
  if (nov <= 0.f || nol <= 0.f || noh <= 0.f || voh <= 0.f) return 0.f;
  Alpha a = aniso_alpha(c.roughness, c.anisotropy);
  return ggx_d_aniso(a, lh) * ggx_g2_aniso(a, lv, ll) / fmaxf(4.f * nov * nol, kEps5);
}

DEV float ggx_d(float alpha, float noh) {
  float a2 = alpha * alpha;
  float d = noh * noh * (a2 - 1.f) + 1.f;
  return a2 / fmaxf(kPi * d * d, 9.999999960041972e-13f);
}
DEV float ggx_lambda(float alpha, float nox) {
  float ct = fabsf(nox);
  float c2 = ct * ct;
  float s2 = fmaxf(1.f - c2, 0.f);
  if (s2 <= 9.99999993922529029e-09f || ct <= 9.99999993922529029e-09f) return 0.f;
  return 0.5f * (-1.f + sqrtf(1.f + alpha * alpha * (s2 / fmaxf(c2, 9.99999993922529029e-09f))));
}

// multiple-scattering term shared by the GGX lobes
struct MsTerm {
  float e_avg, ms;
};
DEV MsTerm ms_term(float roughness, float cos_l, float cos_v) {
  float a = fmaxf(roughness * roughness, 0.f);
  float e_avg = avg_albedo_ggx(a);
  float ms = (1.f - dir_albedo_ggx(a, cos_l)) * (1.f - dir_albedo_ggx(a, cos_v)) /
             fmaxf(kPi * (1.f - e_avg), 9.99999997475242708e-07f);
  return MsTerm{e_avg, ms};
}
DEV v3 ms_energy(v3 favg, MsTerm t) {
  return t.ms * (favg * favg * t.e_avg / vmax(1.f - favg * (1.f - t.e_avg), mk(kEps5)));
}

// ---- lobes ---------------------------------------------------------------------
DEV float transparent_dielectric_weight(const Closure& c) { return c.dielectric_weight * c.transparency; }
DEV v3 weighted_transmission_color(const Closure& c) { return c.albedo * transparent_dielectric_weight(c); }

// evaluateDielectricSpecularGGX_0 (kernel:953-1033), ior_i = 1, ior_o = c.ior
DEV v3 eval_dielectric_specular(const Closure& c, const Frame& f, v3 n, v3 v, v3 l) {
  float nol = fmaxf(dot(n, l), 0.f);
  float tw = transparent_dielectric_weight(c);
  if (nol <= 0.f || tw <= 0.f) return mk(0.f);
  float micro = microfacet_aniso(c, f, v, l);
  float voh = fmaxf(dot(v, normalize(v + l)), 0.f);
  MsTerm t = ms_term(c.roughness, nol, fabsf(dot(n, v)));
  v3 reg = fresnel_dielectric(voh, c.dielectric_f0, c.dielectric_f90, c.ior);
  v3 F = film_dielectric_fresnel(c, voh, reg);
  v3 favg = fabsf(1.f - c.ior) <= kEps4 ? mk(0.f) : schlick_avg(c.dielectric_f0, mk(c.dielectric_f90));
  return tw * (micro * F + ms_energy(favg, t)) * nol;
}

struct TransCoeffs {
  v3 refl, trans;
  float p_refl, p_trans;
};
// computeDielectricTransmissionCoefficients_0 (kernel:1065-1108) with
// currentMediumIor = 1: the probability weight max(throughput, 1) is 1.
DEV TransCoeffs transmission_coeffs(const Closure& c, v3 n, v3 v) {
  float cos_v = fmaxf(dot(n, v), kEps5);
  v3 fr = fresnel_dielectric(cos_v, c.dielectric_f0, c.dielectric_f90, c.ior);
  v3 film = film_dielectric_fresnel(c, cos_v, fr);
  TransCoeffs k;
  k.refl = film * transparent_dielectric_weight(c);
  k.trans = (1.f - film) * weighted_transmission_color(c);
  float rw = max3(vmax(k.refl, mk(0.f)));
  float tw = max3(vmax(k.trans, mk(0.f)));
  float tot = rw + tw;
  if (tot <= kEps5) { k.p_refl = 1.f; k.p_trans = 0.f; }
  else { k.p_refl = rw / tot; k.p_trans = tw / tot; }
  return k;
}

DEV v3 flip_across(v3 v, v3 n) { return normalize(v - 2.f * n * dot(v, n)); }

// evaluateThinTransmissionScattering_0 (kernel:1118-1148)
DEV v3 eval_thin_transmission(const Closure& c, const Frame& f, v3 n, v3 v, v3 l) {
  float nl = dot(n, l);
  if (dot(n, v) * nl >= 0.f) return mk(0.f);
  v3 ml = flip_across(l, n);
  float voh = fmaxf(dot(v, normalize(v + ml)), kEps5);
  v3 reg = fresnel_dielectric(voh, c.dielectric_f0, c.dielectric_f90, c.ior);
  v3 film = film_dielectric_fresnel(c, voh, reg);
  return weighted_transmission_color(c) * (1.f - film) * microfacet_aniso(c, f, v, ml) * fabsf(nl);
}

// evaluateThickTransmissionScattering_0 (kernel:1151-1241), ior_i = 1
NOINL v3 eval_thick_transmission(const Closure& c, const Frame& f, v3 coeff, v3 n, v3 v, v3 l, float ior_o) {
  v3 lv = to_local(f, v), ll = to_local(f, l);
  float nov = fabsf(lv.z), nol = fabsf(ll.z);
  if (nov <= kEps5 || nol <= kEps5 || dot(n, v) * dot(n, l) >= 0.f) return mk(0.f);
  float eta = ior_o / fmaxf(1.f, kEps5);
  v3 h = -normalize(v + l * eta);
  v3 lh = to_local(f, h);
  float voh = dot(v, h), loh = dot(l, h);
  if (fabsf(lh.z) <= kEps5 || voh * loh >= 0.f) return mk(0.f);
  Alpha a = aniso_alpha(c.roughness, c.anisotropy);
  float d = ggx_d_aniso(a, lh);
  float g = ggx_g2_aniso(a, lv, ll);
  float s = voh + eta * loh;
  float factor = eta * eta * fabsf(voh) * fabsf(loh) / fmaxf(s * s * nov, kEps5);
  v3 eff = coeff;
  if (c.iridescence > kEps5) {
    v3 reg = fresnel_dielectric(fabsf(voh), c.dielectric_f0, c.dielectric_f90, ior_o);
    eff = (1.f - film_dielectric_fresnel(c, fabsf(voh), reg)) * weighted_transmission_color(c);
  }
  return eff * d * g * factor;
}

DEV v3 dispersion_iors(const Closure& c) {
  float i = fmaxf(c.ior, 1.f);
  float s = (i - 1.f) * fmaxf(c.dispersion, 0.f) * 0.05000000074505806f;
  return vmax(mk(i + s * -0.30094969272613525f, i, i + s * 0.69905030727386475f), mk(1.f));
}

// evaluateThickTransmissionScatteringDispersed_0 (kernel:1302-1425)
DEV v3 eval_thick_dispersed(const Closure& c, const Frame& f, v3 coeff, v3 n, v3 v, v3 l) {
  if (c.dispersion <= kEps5 || c.thin > 0.5f) return eval_thick_transmission(c, f, coeff, n, v, l, c.ior);
  v3 iors = dispersion_iors(c);
  v3 r = eval_thick_transmission(c, f, mk(coeff.x, 0.f, 0.f), n, v, l, iors.x);
  v3 g = eval_thick_transmission(c, f, mk(0.f, coeff.y, 0.f), n, v, l, iors.y);
  v3 b = eval_thick_transmission(c, f, mk(0.f, 0.f, coeff.z), n, v, l, iors.z);
  return mk(r.x, g.y, b.z);
}

// evalDielectricTransmission_0 (kernel:1427-1497)
NOINL v3 eval_dielectric_transmission(const Closure& c, const Frame& f, v3 n, v3 v, v3 l) {
  if (dot(n, v) * dot(n, l) > 0.f) return eval_dielectric_specular(c, f, n, v, l);
  if (c.thin > 0.5f) return eval_thin_transmission(c, f, n, v, l);
  TransCoeffs k = transmission_coeffs(c, n, v);
  return eval_thick_dispersed(c, f, k.trans, n, v, l);
}

DEV float coupled_diffuse_factor(const Closure& c, float nov, float nol) {
  float a = fmaxf(c.roughness * c.roughness, 0.f);
  float e0 = max3(c.dielectric_f0 * c.dielectric_weight);
  return mixf(kInvPi,
              (1.f - dir_albedo_ggx_ms(nol, a, e0)) * (1.f - dir_albedo_ggx_ms(nov, a, e0)) /
                  fmaxf(kPi * (1.f - avg_albedo_ggx_ms(a, e0)), 9.99999997475242708e-07f),
              c.specular);
}
DEV v3 thin_shared_f0(const Closure& c) { return c.dielectric_f0 * c.dielectric_weight + c.albedo * c.metallic; }
DEV v3 thin_shared_f90(const Closure& c) { return mk(c.dielectric_f90) * c.dielectric_weight + mk(c.metallic); }
DEV v3 diffuse_energy(const Closure& c) {
  return sat(1.f - (schlick_avg(c.albedo, mk(1.f)) * c.metallic +
                    schlick_avg(c.dielectric_f0, mk(c.dielectric_f90)) * c.dielectric_weight));
}
DEV float transmissive_diffuse_compensation(const Closure& c, float nov, float nol) {
  float coupled = coupled_diffuse_factor(c, nov, nol);
  bool thin = c.thin > 0.5f;
  v3 sc = thin ? thin_shared_f0(c) : c.dielectric_f0;
  v3 sf = thin ? thin_shared_f90(c) : mk(c.dielectric_f90);
  float F0 = max3(sc);
  float dF = max3(sf) - F0;
  return coupled * mixf(1.f, 1.f / fmaxf(max3(diffuse_energy(c)), kEps4),
                        sqrtf(0.5f * (sat(F0 + dF * pow5(1.f - sat(nov))) + sat(F0 + dF * pow5(1.f - sat(nol))))));
}
// evalDiffuseReflection_0 (kernel:1589-1631)
DEV v3 eval_diffuse(const Closure& c, v3 n, v3 v, v3 l) {
  float nol = fmaxf(dot(n, l), 0.f);
  if (c.specular <= kEps5 && c.transparency <= 0.f) return c.diffuse_reflection_color * kInvPi * nol;
  float nov = fmaxf(fabsf(dot(v, n)), 0.f);
  float factor = c.transparency > 0.f ? transmissive_diffuse_compensation(c, nov, nol)
                                      : coupled_diffuse_factor(c, nov, nol);
  return c.diffuse_reflection_color * factor * nol;
}

DEV bool is_thin_transmissive(const Closure& c) {
  return c.thin > 0.5f && (c.transparency > 0.f || c.diffuse_transmission_weight > 0.f) && c.metallic < 1.f;
}

// evaluateThinSharedSpecularGGX_0 (kernel:1662-1721)
DEV v3 eval_thin_shared_specular(const Closure& c, const Frame& f, v3 n, v3 v, v3 l) {
  float nol = fmaxf(dot(n, l), 0.f);
  if (nol <= 0.f) return mk(0.f);
  float micro = microfacet_aniso(c, f, v, l);
  float voh = fmaxf(dot(v, normalize(v + l)), 0.f);
  MsTerm t = ms_term(c.roughness, nol, fabsf(dot(n, v)));
  v3 f0 = thin_shared_f0(c), f90 = thin_shared_f90(c);
  v3 F = schlick(f0, f90, voh);
  if (c.iridescence > kEps5)
    F = vmix(F, film_reflectance(1.f, c.iridescence_ior, substrate_f0(c.ior), c.iridescence_thickness, voh),
             sat(c.iridescence));
  v3 favg = schlick_avg(f0, f90);
  return (micro * F + ms_energy(favg, t)) * nol;
}

// evaluateBaseSpecularGGX_0 (kernel:1723-1786)
DEV v3 eval_base_specular_ggx(const Closure& c, const Frame& f, v3 n, v3 v, v3 l) {
  float micro = microfacet_aniso(c, f, v, l);
  float voh = fmaxf(dot(v, normalize(v + l)), 0.f);
  MsTerm t = ms_term(c.roughness, fabsf(dot(n, l)), fabsf(dot(n, v)));
  bool film = c.iridescence > kEps5;
  v3 metal_f = schlick(c.albedo, mk(1.f), voh);
  if (film)
    metal_f = vmix(metal_f, film_reflectance(1.f, c.iridescence_ior, c.albedo, c.iridescence_thickness, voh),
                   sat(c.iridescence));
  v3 metal_ss = micro * metal_f;
  v3 metal_ms = ms_energy(schlick_avg(c.albedo, mk(1.f)), t);
  v3 diel_f = schlick(c.dielectric_f0, mk(c.dielectric_f90), voh);
  if (film)
    diel_f = vmix(diel_f, film_reflectance(1.f, c.iridescence_ior, substrate_f0(c.ior), c.iridescence_thickness, voh),
                  sat(c.iridescence));
  v3 diel_favg = schlick_avg(c.dielectric_f0, mk(c.dielectric_f90));
  return c.metallic * (metal_ss + metal_ms) +
         c.dielectric_weight * (1.f - c.transparency) * (micro * diel_f + ms_energy(diel_favg, t));
}

DEV v3 eval_base_specular(const Closure& c, const Frame& f, v3 n, v3 v, v3 l) {
  float nol = fmaxf(dot(n, l), 0.f);
  if (is_thin_transmissive(c)) return eval_thin_shared_specular(c, f, n, v, l);
  return eval_base_specular_ggx(c, f, n, v, l) * nol;
}

// sheen (kernel:1798-1890)
DEV float sheen_log(float x, float alpha) {
  float o = 1.f - alpha;
  float o2 = o * o;
  return mixf(21.54730033874511719f, 25.32449913024902344f, o2) /
             (1.f + mixf(3.82986998558044434f, 3.32435011863708496f, o2) *
                        powf(fabsf(x), mixf(0.19822999835014343f, 0.16800999641418457f, o2))) +
         mixf(-1.97759997844696045f, -1.27392995357513428f, o2) * x +
         mixf(-4.32053995132446289f, -4.85967016220092773f, o2);
}
DEV float sheen_lambda(float cos_t, float alpha) {
  if (fabsf(cos_t) >= 0.5f) return expf(2.f * sheen_log(0.5f, alpha) - sheen_log(1.f - cos_t, alpha));
  return expf(sheen_log(cos_t, alpha));
}
DEV v3 eval_sheen(const Closure& c, v3 n, v3 v, v3 l) {
  if (max3(c.sheen_color) <= 0.f) return mk(0.f);
  float nov = fmaxf(dot(n, v), 0.f), nol = fmaxf(dot(n, l), 0.f);
  float noh = fmaxf(dot(n, normalize(v + l)), 0.f);
  if (nov <= 0.f || nol <= 0.f || noh <= 0.f) return mk(0.f);
  float alpha = fmaxf(c.sheen_roughness * c.sheen_roughness, 0.f);
  float inv = 1.f / fmaxf(alpha, kEps5);
  float d = (2.f + inv) * powf(fabsf(fmaxf(1.f - noh * noh, 0.00100000004749745f)), 0.5f * inv) / kTwoPi;
  return c.sheen_color * (1.f / (1.f + sheen_lambda(nov, alpha) + sheen_lambda(nol, alpha)) * d /
                          fmaxf(4.f * nov * nol, kEps5)) *
         nol;
}

// clearcoat (kernel:1956-2043)
DEV v3 eval_clearcoat(const Closure& c, v3 n, v3 v, v3 l) {
  if (c.clearcoat <= 0.f) return mk(0.f);
  v3 h = normalize(v + l);
  float nov = fmaxf(dot(n, v), 0.f), nol = fmaxf(dot(n, l), 0.f);
  float noh = fmaxf(dot(n, h), 0.f), voh = fmaxf(dot(v, h), 0.f);
  if (nov <= 0.f || nol <= 0.f || noh <= 0.f || voh <= 0.f) return mk(0.f);
  float a = fmaxf(c.clearcoat_roughness * c.clearcoat_roughness, 0.f);
  float F = schlick1(0.03999999910593033f, 1.f, voh);
  float g2 = 1.f / (1.f + ggx_lambda(a, nov) + ggx_lambda(a, nol));
  float ggx = F * ggx_d(a, noh) * g2 / fmaxf(4.f * nov * nol, kEps5);
  return mk(c.clearcoat * ggx) * fmaxf(dot(n, l), 0.f);
}
DEV float clearcoat_base_weight(const Closure& c, v3 n, v3 v, v3 l) {
  if (c.clearcoat <= 0.f) return 1.f;
  float fv = schlick1(0.03999999910593033f, 1.f, fabsf(dot(n, v)));
  float fl = schlick1(0.03999999910593033f, 1.f, fabsf(dot(n, l)));
  return sat(1.f - c.clearcoat * fmaxf(fv, fl));
}

DEV v3 eval_diffuse_transmission(const Closure& c, v3 n, v3 l) {
  return c.diffuse_transmission_color * kInvPi * fmaxf(fabsf(dot(n, l)), 0.f);
}

NOINL v3 eval_reflected_base(const Closure& c, const Frame& f, v3 n, v3 v, v3 l) {
  return eval_diffuse(c, n, v, l) + eval_base_specular(c, f, n, v, l) + eval_sheen(c, n, v, l);
}

// evalMaterialBsdfMixture_0 (kernel:2045-2089): returns BSDF * |cos|.  The
// adapter passes the same shading normal as base and clearcoat normal.
NOINL v3 bsdf_eval(const Closure& c, v3 n, v3 v, v3 l) {
  Frame f = aniso_frame(n, c.aniso_tangent);
  if (!(dot(n, v) * dot(n, l) > 0.f))
    return eval_diffuse_transmission(c, n, l) + eval_dielectric_transmission(c, f, n, v, l);
  v3 base = eval_reflected_base(c, f, n, v, l);
  if (c.thin < 0.5f && c.transparency > 0.f) base = base + eval_dielectric_transmission(c, f, n, v, l);
  return eval_clearcoat(c, n, v, l) + base * clearcoat_base_weight(c, n, v, l);
}

// ---- pdf (kernel:2113-2617) ------------------------------------------------------
DEV float spec_lobe_pdf(const Closure& c, const Frame& f, v3 v, v3 d) {
  v3 h = normalize(v + d);
  v3 lh = to_local(f, h);
  float noh = fabsf(lh.z);
  float voh = fmaxf(dot(v, h), 0.f);
  if (noh <= 0.f || voh <= 0.f) return 0.f;
  return ggx_d_aniso(aniso_alpha(c.roughness, c.anisotropy), lh) * noh / fmaxf(4.f * voh, kEps5);
}
DEV float spec_lobe_pdf_iso(v3 n, v3 v, float rough, v3 d) {
  v3 h = normalize(v + d);
  float noh = fmaxf(dot(n, h), 0.f), voh = fmaxf(dot(v, h), 0.f);
  if (noh <= 0.f || voh <= 0.f) return 0.f;
  return ggx_d(fmaxf(rough * rough, 0.f), noh) * noh / fmaxf(4.f * voh, kEps5);
}
DEV float pdf_clearcoat(const Closure& c, v3 n, v3 v, v3 l) {
  return fmaxf(dot(n, l), 0.f) > 0.f ? spec_lobe_pdf_iso(n, v, c.clearcoat_roughness, l) : 0.f;
}
DEV float thick_transmission_pdf(const Closure& c, const Frame& f, v3 n, v3 v, v3 l, float ior_o) {
  v3 lv = to_local(f, v);
  float nov = fabsf(lv.z);
  float nol = fabsf(to_local(f, l).z);
  if (nov <= kEps5 || nol <= kEps5 || dot(n, v) * dot(n, l) >= 0.f) return 0.f;
  float eta = ior_o / fmaxf(1.f, kEps5);
  v3 h = -normalize(v + l * eta);
  v3 lh = to_local(f, h);
  float voh = dot(v, h), loh = dot(l, h);
  if (fabsf(lh.z) <= kEps5 || voh * loh >= 0.f) return 0.f;
  Alpha a = aniso_alpha(c.roughness, c.anisotropy);
  float s = voh + eta * loh;
  return ggx_d_aniso(a, lh) * ggx_g1_aniso(a, lv) *
         (eta * eta * fabsf(voh) * fabsf(loh) / fmaxf(s * s * nov, kEps5));
}
DEV float pdf_dielectric_transmission(const Closure& c, const Frame& f, v3 n, v3 v, v3 l) {
  TransCoeffs k = transmission_coeffs(c, n, v);
  if (dot(n, v) * dot(n, l) < 0.f) {
    float pt = fmaxf(k.p_trans, kEps5);
    float lobe = c.thin > 0.5f ? spec_lobe_pdf(c, f, v, flip_across(l, n)) : thick_transmission_pdf(c, f, n, v, l, c.ior);
    return fmaxf(pt * lobe, kEps5);
  }
  return fmaxf(sat(k.p_refl) * spec_lobe_pdf(c, f, v, l), kEps5);
}
DEV float thin_base_probability(const Closure& c, v3 n, v3 v) {
  return sat(1.f - max3(schlick(thin_shared_f0(c), thin_shared_f90(c), fmaxf(fabsf(dot(n, v)), kEps5))));
}
DEV float transmissive_base_layer_weight(const Closure& c) {
  return fmaxf(c.diffuse_weight + c.sheen_weight + c.diffuse_transmission_weight + c.transmission_weight, kEps5);
}
DEV float dielectric_view_fresnel_max(const Closure& c, v3 n, v3 v) {
  return max3(schlick(c.dielectric_f0, mk(c.dielectric_f90), fmaxf(dot(n, v), 0.f)));
}

NOINL float bsdf_pdf_f(const Closure& c, const Frame& f, v3 n, v3 v, v3 d) {
  float nd = dot(n, d);
  float nol = fmaxf(nd, 0.f);
  float ccnol = fmaxf(dot(n, d), 0.f);
  bool trans_side = dot(n, v) * nd < 0.f;
  bool thin = is_thin_transmissive(c);
  float thin_base = thin ? thin_base_probability(c, n, v) : 0.f;
  float thin_spec = thin ? 1.f - thin_base : 0.f;
  const float pdt = fmaxf(dot(-n, d), 0.f) * kInvPi;
  if (trans_side) {
    float pdf;
    if (thin) {
      float blw = transmissive_base_layer_weight(c);
      pdf = c.diffuse_transmission_weight > 0.f ? thin_base * (c.diffuse_transmission_weight / blw) * pdt : 0.f;
      if (c.transmission_weight > 0.f)
        pdf = pdf + thin_base * (c.transmission_weight / blw) * spec_lobe_pdf(c, f, v, flip_across(d, n));
      return pdf > 0.f ? fmaxf(pdf, kEps5) : 0.f;
    }
    float tw = fmaxf(c.diffuse_transmission_weight + c.transmission_weight, kEps5);
    pdf = c.diffuse_transmission_weight > 0.f ? c.diffuse_transmission_weight / tw * pdt : 0.f;
    if (c.transmission_weight > 0.f) pdf = pdf + c.transmission_weight / tw * pdf_dielectric_transmission(c, f, n, v, d);
    return pdf > 0.f ? fmaxf(pdf, kEps5) : 0.f;
  }
  if (nol <= 0.f) return 0.f;
  const float pdiff = nol * kInvPi;  // pdfDiffuseReflection_0 == pdfSheen_0
  if (thin) {
    float blw = transmissive_base_layer_weight(c);
    float tot = fmaxf(thin_base + thin_spec + c.clearcoat_weight, kEps5);
    float diffuse = thin_base * c.diffuse_weight / blw / tot * pdiff;
    float sheen = thin_base * c.sheen_weight / blw / tot * pdiff;
    float spec = thin_spec / tot * spec_lobe_pdf(c, f, v, d);
    float ccw = c.clearcoat_weight / tot;
    float cc = ccnol > 0.f ? pdf_clearcoat(c, n, v, d) : 0.f;
    return fmaxf(diffuse + sheen + spec + ccw * cc, kEps5);
  }
  float vf = dielectric_view_fresnel_max(c, n, v);
  float one_m = 1.f - vf;
  float dw = c.diffuse_weight * one_m;
  float sw = c.sheen_weight * one_m;
  float spw = c.specular_weight + c.dielectric_weight * (1.f - c.transparency) * vf;
  float tot = fmaxf(dw + sw + c.diffuse_transmission_weight + spw + c.transmission_weight + c.clearcoat_weight, kEps5);
  float diffuse = dw / tot * pdiff;
  float sheen = sw / tot * pdiff;
  float spec = spw / tot * spec_lobe_pdf(c, f, v, d);
  float trans = c.transmission_weight > 0.f ? c.transmission_weight / tot * pdf_dielectric_transmission(c, f, n, v, d) : 0.f;
  float ccw = c.clearcoat_weight / tot;
  float cc = ccnol > 0.f ? pdf_clearcoat(c, n, v, d) : 0.f;
  return fmaxf(diffuse + sheen + spec + trans + ccw * cc, kEps5);
}
DEV float bsdf_pdf(const Closure& c, v3 n, v3 v, v3 d) {
  Frame f = aniso_frame(n, c.aniso_tangent);
  return bsdf_pdf_f(c, f, n, v, d);
}

// bsdf_eval and bsdf_pdf of one direction in one call: the anisotropy frame is
// built once and the caller saves its registers around one call, not two;
// the values are those of the two separate calls.
NOINL v3 bsdf_eval_pdf(const Closure& c, v3 n, v3 v, v3 l, float& pdf) {
  Frame f = aniso_frame(n, c.aniso_tangent);
  pdf = bsdf_pdf_f(c, f, n, v, l);
  if (!(dot(n, v) * dot(n, l) > 0.f))
    return eval_diffuse_transmission(c, n, l) + eval_dielectric_transmission(c, f, n, v, l);
  v3 base = eval_reflected_base(c, f, n, v, l);
  if (c.thin < 0.5f && c.transparency > 0.f) base = base + eval_dielectric_transmission(c, f, n, v, l);
  return eval_clearcoat(c, n, v, l) + base * clearcoat_base_weight(c, n, v, l);
}

// ---- sampling (kernel:2625-3567) ----------------------------------------------
DEV void orthonormal_basis(v3 n, v3& t, v3& b) {
  float sign = n.z >= 0.f ? 1.f : -1.f;
  float a = -1.f / (sign + n.z);
  float bb = n.x * n.y * a;
  t = normalize(mk(1.f + sign * n.x * n.x * a, sign * bb, -sign * n.x));
  b = normalize(mk(bb, sign + n.y * n.y * a, -n.y));
}
DEV v3 sample_cosine(v3 n, float u0, float u1) {
  float r = sqrtf(u0);
  float phi = kTwoPi * u1;
  float s, co;
  sincosf(phi, &s, &co);
  float x = r * co, y = r * s, z = sqrtf(fmaxf(0.f, 1.f - u0));
  v3 t, b;
  orthonormal_basis(n, t, b);
  return normalize(t * x + b * y + n * z);
}
DEV v3 sample_ggx_half(const Closure& c, const Frame& f, float u0, float u1) {
  Alpha a = aniso_alpha(c.roughness, c.anisotropy);
  float phi = kTwoPi * u1;
  float sp, cp;
  sincosf(phi, &sp, &cp);
  float ct = 1.f / sqrtf(1.f + u0 / fmaxf(1.f - u0, 9.99999997475242708e-07f) /
                                   fmaxf(cp * cp / fmaxf(a.x * a.x, 9.999999960041972e-13f) +
                                             sp * sp / fmaxf(a.y * a.y, 9.999999960041972e-13f),
                                         9.99999997475242708e-07f));
  float st = sqrtf(fmaxf(0.f, 1.f - ct * ct));
  // anisotropicBasis_0 (kernel:2792-2798) is the same basis as the frame
  return normalize(f.t * (st * cp) + f.b * (st * sp) + f.n * ct);
}
DEV v3 sample_ggx_half_iso(v3 n, float rough, float u0, float u1) {
  float a = fmaxf(rough * rough, 0.f);
  float phi = kTwoPi * u1;
  float ct = sqrtf((1.f - u0) / fmaxf(1.f + (a * a - 1.f) * u0, 9.99999997475242708e-07f));
  float st = sqrtf(fmaxf(0.f, 1.f - ct * ct));
  float sp, cp;
  sincosf(phi, &sp, &cp);
  v3 t, b;
  orthonormal_basis(n, t, b);
  return normalize(t * (st * cp) + b * (st * sp) + n * ct);
}
DEV float half_vector_pdf(const Closure& c, const Frame& f, v3 h) {
  v3 lh = to_local(f, h);
  float noh = fabsf(lh.z);
  if (noh <= kEps5) return 0.f;
  return ggx_d_aniso(aniso_alpha(c.roughness, c.anisotropy), lh) * noh;
}
DEV v3 safe_refract(v3 i, v3 n, float eta) {
  float noi = dot(n, i);
  float k = 1.f - eta * eta * (1.f - noi * noi);
  if (k <= 0.f) return mk(0.f);
  return eta * i - (eta * noi + sqrtf(k)) * n;
}

// sampleDielectricTransmission_0 (kernel:2881-3145), currentMediumIor = 1
NOINL BsdfSample sample_dielectric_transmission(const Closure& c, const Frame& f, v3 n, v3 v, float u0, float u1,
                                              float event_u) {
  BsdfSample s;
  if (c.thin < 0.5f && fabsf(1.f - c.ior) <= kEps4) {
    s.dir = -v; s.pdf = 1.f; s.weight = weighted_transmission_color(c);
    s.specular = 2.f; s.crossed = 1.f; s.next_ior = c.ior;
    return s;
  }
  v3 h = sample_ggx_half(c, f, u0, u1);
  TransCoeffs k = transmission_coeffs(c, n, v);
  float half_pdf = half_vector_pdf(c, f, h);
  float pr = sat(k.p_refl);
  float pt = fmaxf(k.p_trans, kEps5);
  s.crossed = 0.f;
  s.next_ior = 1.f;
  if (event_u <= pr) {
    v3 d = reflect(-v, h);
    float lobe = half_pdf / fmaxf(4.f * fabsf(dot(d, h)), kEps5);
    s.dir = d;
    s.pdf = fmaxf(pr * lobe, kEps5);
    s.weight = eval_dielectric_specular(c, f, n, v, d) / s.pdf;
    s.specular = 1.f;
    return s;
  }
  if (c.thin > 0.5f) {
    v3 d = flip_across(reflect(-v, h), n);
    float lobe = half_pdf / fmaxf(4.f * fabsf(dot(d, h)), kEps5);
    s.dir = d;
    s.pdf = fmaxf(pt * lobe, kEps5);
    s.weight = eval_thin_transmission(c, f, n, v, d) / s.pdf;
    s.specular = 1.f;
    return s;
  }
  bool disp = c.dispersion > kEps5;
  float chan_u = clampf((event_u - pr) / fmaxf(pt, kEps5), 0.f, 0.99999898672103882f);
  v3 mask = mk(1.f);
  if (disp) mask = chan_u < 0.3333333432674408f ? mk(1.f, 0.f, 0.f)
                   : (chan_u < 0.66666668653488159f ? mk(0.f, 1.f, 0.f) : mk(0.f, 0.f, 1.f));
  float t_ior = disp ? dot(dispersion_iors(c), mask) : c.ior;
  float chan_p = disp ? 0.3333333432674408f : 1.f;
  v3 refr = safe_refract(-v, h, 1.f / fmaxf(t_ior, kEps5));
  if (length(refr) <= kEps5) {
    v3 d = reflect(-v, h);
    s.dir = d;
    s.pdf = fmaxf(pdf_dielectric_transmission(c, f, n, v, d), kEps5);
    s.weight = eval_dielectric_specular(c, f, n, v, d) / s.pdf;
    s.specular = 3.f;
    return s;
  }
  float voh = dot(v, h), roh = dot(refr, h);
  float den = 1.f * voh + t_ior * roh;
  float lobe = half_pdf * (t_ior * t_ior) * fabsf(roh) / fmaxf(den * den, kEps5);
  float g1 = ggx_g1_aniso(aniso_alpha(c.roughness, c.anisotropy), to_local(f, refr));
  v3 eff = k.trans;
  if (c.iridescence > kEps5) {
    v3 reg = fresnel_dielectric(fabsf(voh), c.dielectric_f0, c.dielectric_f90, t_ior);
    eff = (1.f - film_dielectric_fresnel(c, fabsf(voh), reg)) * weighted_transmission_color(c);
  }
  s.dir = refr;
  float pc = pt * chan_p;
  s.pdf = fmaxf(pc * lobe, kEps5);
  s.weight = eff * mask / fmaxf(pc, kEps5) * g1;
  s.specular = 1.f;
  s.crossed = 1.f;
  s.next_ior = c.ior;
  return s;
}

// Finishes a sample whose direction came from a reflection-side lobe
// (kernel:3480-3567 / 3284-3364): value and pdf of the whole mixture.
NOINL BsdfSample finish_reflection_sample(const Closure& c, const Frame& f, v3 n, v3 v, v3 d, float spec, float u0,
                                        float u1, bool thin_path, float crossed, float next_ior) {
  BsdfSample s;
  s.crossed = crossed;
  s.next_ior = next_ior;
  float nd = dot(n, d);
  float nol = fmaxf(nd, 0.f);
  float ccnol = fmaxf(dot(n, d), 0.f);
  if (nol <= 0.f) {
    if (nd < 0.f) {
      float mix_pdf = bsdf_pdf_f(c, f, n, v, d);
      v3 dt = eval_diffuse_transmission(c, n, d);
      s.dir = d;
      s.pdf = fmaxf(mix_pdf, kEps5);
      s.weight = dt / fmaxf(s.pdf, kEps5);
      s.specular = 0.f;
      return s;
    }
    v3 fd = sample_cosine(n, u0, u1);
    s.dir = fd;
    s.pdf = fmaxf(fmaxf(dot(n, fd), 0.f) * kInvPi, kEps5);
    s.weight = mk(0.f);
    s.specular = 0.f;
    s.next_ior = 1.f;
    return s;
  }
  s.next_ior = 1.f;
  float mix_pdf = bsdf_pdf_f(c, f, n, v, d);
  v3 base = eval_reflected_base(c, f, n, v, d) / fmaxf(nol, kEps5);
  v3 cc = ccnol > 0.f ? eval_clearcoat(c, n, v, d) / fmaxf(ccnol, kEps5) : mk(0.f);
  float bw = clearcoat_base_weight(c, n, v, d);
  s.dir = d;
  s.pdf = mix_pdf;
  v3 num = (base * bw + cc);
  s.weight = thin_path ? num * nol / fmaxf(mix_pdf, kEps5) : num * fabsf(nd) / mix_pdf;
  s.specular = spec;
  return s;
}

// sampleMaterialBsdfMixture_0 (kernel:3200-3567).  rnd = (component, lobe.x,
// lobe.y, boundary) as PbrRandoms (kernel:3570-3575).
NOINL BsdfSample bsdf_sample(const Closure& c, v3 n, v3 v, float choice, float u0, float u1, float event_u) {
  Frame f = aniso_frame(n, c.aniso_tangent);
  if (is_thin_transmissive(c)) {
    float tb = thin_base_probability(c, n, v);
    float ts = 1.f - tb;
    float blw = transmissive_base_layer_weight(c);
    float tot = fmaxf(tb + ts + c.clearcoat_weight, kEps5);
    float p_diff = tb * (c.diffuse_weight / blw) / tot;
    float p_sheen = tb * (c.sheen_weight / blw) / tot;
    float p_dt = tb * (c.diffuse_transmission_weight / blw) / tot;
    float p_tt = tb * (c.transmission_weight / blw) / tot;
    float p_spec = ts / tot;
    v3 d;
    float spec;
    if (choice < p_diff) { d = sample_cosine(n, u0, u1); spec = 0.f; }
    else if (choice < p_diff + p_sheen) { d = sample_cosine(n, u0, u1); spec = 0.f; }
    else if (choice < p_diff + p_sheen + p_dt) { d = sample_cosine(-n, u0, u1); spec = 0.f; }
    else if (choice < p_diff + p_sheen + p_dt + p_tt) {
      BsdfSample s = sample_dielectric_transmission(c, f, n, v, u0, u1, 1.f);
      float mp = bsdf_pdf_f(c, f, n, v, s.dir);
      s.pdf = mp;
      s.weight = eval_dielectric_transmission(c, f, n, v, s.dir) / fmaxf(mp, kEps5);
      s.crossed = 0.f;
      s.next_ior = 1.f;
      return s;
    } else if (choice < p_diff + p_sheen + p_dt + p_tt + p_spec) {
      d = reflect(-v, sample_ggx_half(c, f, u0, u1)); spec = 1.f;
    } else {
      d = reflect(-v, sample_ggx_half_iso(n, c.clearcoat_roughness, u0, u1)); spec = 1.f;
    }
    return finish_reflection_sample(c, f, n, v, d, spec, u0, u1, true, 0.f, 1.f);
  }
  float vf = dielectric_view_fresnel_max(c, n, v);
  float one_m = 1.f - vf;
  float dw = c.diffuse_weight * one_m;
  float sw = c.sheen_weight * one_m;
  float spw = c.specular_weight + c.dielectric_weight * (1.f - c.transparency) * vf;
  float bw = dw + sw + c.diffuse_transmission_weight;
  float tot = fmaxf(bw + spw + c.transmission_weight + c.clearcoat_weight, kEps5);
  float p_base = bw / tot;
  float p_spec = spw / tot;
  float p_trans = c.transmission_weight / tot;
  v3 d;
  float spec;
  float crossed = 0.f, next_ior = 1.f;
  if (choice < p_base) {
    float bu = choice / fmaxf(p_base, kEps5);
    float pd = bw > 0.f ? dw / bw : 0.f;
    float ps = bw > 0.f ? sw / bw : 0.f;
    if (bu < pd) { d = sample_cosine(n, u0, u1); spec = 0.f; }
    else if (bu < pd + ps) { d = sample_cosine(n, u0, u1); spec = 0.f; }
    else {
      // sampleDiffuseTransmission_0 (kernel:2729-2790): crosses into thick media
      d = sample_cosine(-n, u0, u1); spec = 0.f;
      bool thick = c.thin < 0.5f;
      crossed = thick ? 1.f : 0.f;
      next_ior = thick ? c.ior : 1.f;
    }
  } else if (choice < p_base + p_spec) {
    d = reflect(-v, sample_ggx_half(c, f, u0, u1)); spec = 1.f;
  } else if (choice < p_base + p_spec + p_trans) {
    BsdfSample s = sample_dielectric_transmission(c, f, n, v, u0, u1, event_u);
    s.weight = s.weight / fmaxf(p_trans, kEps5);
    if (s.pdf < 1.f) s.pdf = s.pdf * p_trans;
    return s;
  } else {
    d = reflect(-v, sample_ggx_half_iso(n, c.clearcoat_roughness, u0, u1)); spec = 1.f;
  }
  return finish_reflection_sample(c, f, n, v, d, spec, u0, u1, false, crossed, next_ior);
}

}  // namespace dspbr
