// dev_bsdf.cuh — the principled BSDF on the device: six lobes, GGX (anisotropic) with VNDF
// sampling, height-correlated Smith G2, exact dielectric / Schlick Fresnel and the
// multiple-scattering factor, restated from the CPU backend's src/material/bsdf.h (not from
// the reference's GPU copy, which differs): helpers :31-249, diffuse :256-279, microfacet
// reflection :288-356, microfacet transmission :364-460, delta reflection :468-505, delta
// transmission :513-548, subsurface :557-590, eval/pdf for NEE :601-657, sampling :666-708.
// All vectors are in the local frame (z = normal). Operand order as in the reference.
#pragma once

#include "dev_math.cuh"
#include "dev_scene.cuh"

namespace xbd {

constexpr int kMatConductor = 1, kMatTransmissive = 2, kMatSubsurface = 4, kMatDelta = 8;

struct BsdfSample {
  V3 wi, f;
  float pdf;
  bool delta;
};

__device__ __forceinline__ float cos2_theta(V3 w) { return w.z * w.z; }
__device__ __forceinline__ float sin2_theta(V3 w) { return smax(0.f, 1.f - cos2_theta(w)); }
__device__ __forceinline__ float sin_theta(V3 w) { return sqrtf(sin2_theta(w)); }
__device__ __forceinline__ float tan2_theta(V3 w) {
  float c2 = cos2_theta(w);
  return (c2 < 1e-8f) ? 0.f : sin2_theta(w) / c2;
}
__device__ __forceinline__ float cos_phi(V3 w) {
  float s = sin_theta(w);
  return (s == 0.f) ? 1.f : sclamp(w.x / s, -1.f, 1.f);
}
__device__ __forceinline__ float sin_phi(V3 w) {
  float s = sin_theta(w);
  return (s == 0.f) ? 0.f : sclamp(w.y / s, -1.f, 1.f);
}
__device__ __forceinline__ bool same_hemisphere(V3 a, V3 b) { return a.z * b.z > 0.f; }

__device__ __forceinline__ float mis_power2(float a, float b) {
  float a2 = a * a, b2 = b * b, sum = a2 + b2;
  return (sum > 0.f) ? a2 / sum : 0.f;
}

__device__ __forceinline__ float ggx_d_aniso(V3 wh, float ax, float ay) {
  float c2 = cos2_theta(wh);
  if (c2 <= 0.f) return 0.f;
  float ex = cos_phi(wh) / ax;
  float ey = sin_phi(wh) / ay;
  float tan2 = (ex * ex + ey * ey) * tan2_theta(wh);
  float d = c2 * c2 * (1.f + tan2);
  return 1.f / (kPi * ax * ay * d * d);
}

__device__ __forceinline__ float ggx_lambda_aniso(V3 w, float ax, float ay) {
  float t2 = tan2_theta(w);
  if (t2 == 0.f) return 0.f;
  float cp = cos_phi(w), sp = sin_phi(w);
  float a2 = (cp * ax) * (cp * ax) + (sp * ay) * (sp * ay);
  return (-1.f + sqrtf(1.f + a2 * t2)) * 0.5f;
}
__device__ __forceinline__ float ggx_g1_aniso(V3 w, float ax, float ay) {
  return 1.f / (1.f + ggx_lambda_aniso(w, ax, ay));
}
__device__ __forceinline__ float ggx_g2_aniso(V3 wo, V3 wi, float ax, float ay) {
  return 1.f / (1.f + ggx_lambda_aniso(wo, ax, ay) + ggx_lambda_aniso(wi, ax, ay));
}

__device__ __forceinline__ float fresnel_dielectric(float ci, float ior) {
  ci = sclamp(ci, -1.f, 1.f);
  float eta_i = 1.f, eta_t = ior;
  if (ci < 0.f) { float tmp = eta_i; eta_i = eta_t; eta_t = tmp; ci = -ci; }
  float sin2_i = 1.f - ci * ci;
  float sin2_t = (eta_i / eta_t) * (eta_i / eta_t) * sin2_i;
  if (sin2_t >= 1.f) return 1.f;
  float cos_t = sqrtf(smax(0.f, 1.f - sin2_t));
  float r_parl = ((eta_t * ci) - (eta_i * cos_t)) / ((eta_t * ci) + (eta_i * cos_t));
  float r_perp = ((eta_i * ci) - (eta_t * cos_t)) / ((eta_i * ci) + (eta_t * cos_t));
  return (r_parl * r_parl + r_perp * r_perp) * 0.5f;
}

__device__ __forceinline__ V3 fresnel_schlick(float c, V3 f0) {
  float m = sclamp(1.f - c, 0.f, 1.f);
  float m2 = m * m;
  return f0 + (v3s(1.f) - f0) * (m2 * m2 * m);
}

__device__ __forceinline__ V3 sample_cosine_hemisphere(float u1, float u2) {
  float r = sqrtf(u1);
  float phi = 2.0f * kPi * u2;
  return v3(r * cosf(phi), r * sinf(phi), sqrtf(smax(0.0f, 1.0f - u1)));
}

// VNDF sampling, Heitz 2018 (bsdf.h:164-190)
__device__ __forceinline__ V3 sample_vndf(V3 wo, float ax, float ay, float u1, float u2) {
  V3 vh = normalize(v3(ax * wo.x, ay * wo.y, wo.z));
  float len2 = vh.x * vh.x + vh.y * vh.y;
  V3 t1v = (len2 > 1e-7f) ? v3(-vh.y, vh.x, 0.f) * (1.f / sqrtf(len2)) : v3(1.f, 0.f, 0.f);
  V3 t2v = cross(vh, t1v);
  float r = sqrtf(u1);
  float phi = 2.0f * kPi * u2;
  float t1 = r * cosf(phi);
  float t2 = r * sinf(phi);
  float s = 0.5f * (1.0f + vh.z);
  t2 = (1.0f - s) * sqrtf(smax(0.f, 1.0f - t1 * t1)) + s * t2;
  V3 nh = t1 * t1v + t2 * t2v + sqrtf(smax(0.f, 1.0f - t1 * t1 - t2 * t2)) * vh;
  return normalize(v3(ax * nh.x, ay * nh.y, smax(0.f, nh.z)));
}

__device__ __forceinline__ float vndf_pdf(V3 wo, V3 wh, float ax, float ay) {
  float d = ggx_d_aniso(wh, ax, ay);
  float g1 = ggx_g1_aniso(wo, ax, ay);
  float co = fabsf(wo.z);
  if (co < 1e-8f) return 0.f;
  return d * g1 * smax(0.f, dot(wo, wh)) / co;
}

// Multiple-scattering compensation (bsdf.h:212-249). The direction-free terms (5 exp(-2.69 a),
// 1 + 22.7 a^1.5 and F_avg^2 E_avg / denom) are per-material constants computed on the host.
__device__ __forceinline__ float ggx_dir_albedo(float c, float k1, float k2) {
  float e = 1.0f - powf(1.0f - c, k1) / k2;
  return sclamp(e, 0.f, 1.f);
}
__device__ __forceinline__ V3 multiscatter(const DevMaterial& m, float co, float ci) {
  float eo = ggx_dir_albedo(fabsf(co), m.ms_k1, m.ms_k2);
  float ei = ggx_dir_albedo(fabsf(ci), m.ms_k1, m.ms_k2);
  V3 fms = v3(m.ms_fms[0], m.ms_fms[1], m.ms_fms[2]);
  float comp_ = (1.f - eo) * (1.f - ei);
  return v3s(1.f) + fms * comp_ / v3s(smax(eo * ei, 1e-4f));
}

__device__ __forceinline__ V3 mat_base(const DevMaterial& m) { return v3(m.base[0], m.base[1], m.base[2]); }
__device__ __forceinline__ V3 mat_f0(const DevMaterial& m) { return v3(m.f0[0], m.f0[1], m.f0[2]); }

// ── diffuse ─────────────────────────────────────────────────────────────────────
__device__ __forceinline__ V3 diffuse_eval(V3 wi, const DevMaterial& m) {
  if (wi.z <= 0.f) return v3s(0.f);
  return mat_base(m) * (1.f - m.metallic) * kInvPi;
}
__device__ __forceinline__ float diffuse_pdf(V3 wi) {
  if (wi.z <= 0.f) return 0.f;
  return wi.z * kInvPi;
}

// ── microfacet reflection ──────────────────────────────────────────────────────
__device__ __forceinline__ V3 mf_fresnel(float cth, const DevMaterial& m) {
  if (m.flags & kMatConductor) return fresnel_schlick(fabsf(cth), mat_f0(m));
  return v3s(fresnel_dielectric(cth, m.ior));
}
__device__ __forceinline__ V3 mfr_eval(V3 wo, V3 wi, const DevMaterial& m) {
  if (wo.z <= 0.f || wi.z <= 0.f) return v3s(0.f);
  V3 wh = normalize(wo + wi);
  if (wh.z <= 0.f) return v3s(0.f);
  float d = ggx_d_aniso(wh, m.alpha_x, m.alpha_y);
  float g = ggx_g2_aniso(wo, wi, m.alpha_x, m.alpha_y);
  V3 f = mf_fresnel(dot(wo, wh), m);
  float denom = 4.f * wo.z * wi.z;
  if (denom < 1e-8f) return v3s(0.f);
  V3 res = f * d * g / denom;
  if (!(m.flags & kMatTransmissive)) res = res * multiscatter(m, wo.z, wi.z);
  return res;
}
__device__ __forceinline__ float mfr_pdf(V3 wo, V3 wi, const DevMaterial& m) {
  if (wo.z <= 0.f || wi.z <= 0.f) return 0.f;
  V3 wh = normalize(wo + wi);
  if (wh.z <= 0.f) return 0.f;
  float dv = vndf_pdf(wo, wh, m.alpha_x, m.alpha_y);
  float jac = 1.f / (4.f * fabsf(dot(wo, wh)));
  return dv * jac;
}
__device__ __forceinline__ bool mfr_sample(V3 wo, const DevMaterial& m, Pcg& rng, BsdfSample& s) {
  if (wo.z <= 0.f) return false;
  // The reference passes rng.next_float() twice as call arguments; GCC evaluates them right
  // to left, so the first draw is the second parameter (u2). Kept for sample-exact parity.
  float u2 = rng.next_float();
  float u1 = rng.next_float();
  V3 wh = sample_vndf(wo, m.alpha_x, m.alpha_y, u1, u2);
  if (wh.z <= 0.f) return false;
  s.wi = reflect(-wo, wh);
  if (s.wi.z <= 0.f) return false;
  s.pdf = mfr_pdf(wo, s.wi, m);
  if (s.pdf < 1e-8f) return false;
  s.f = mfr_eval(wo, s.wi, m);
  s.delta = false;
  return true;
}

// ── microfacet transmission (Walter 2007) ──────────────────────────────────────
__device__ __forceinline__ V3 mft_eval(V3 wo, V3 wi, const DevMaterial& m) {
  if (wo.z == 0.f || wi.z == 0.f) return v3s(0.f);
  if (same_hemisphere(wo, wi)) return v3s(0.f);
  const float eta = (wo.z > 0.f) ? (1.f / m.ior) : m.ior;
  V3 wh = normalize(wo + eta * wi);
  if (wh.z < 0.f) wh = -wh;
  float dwo = dot(wo, wh), dwi = dot(wi, wh);
  if (dwo * dwi >= 0.f) return v3s(0.f);
  float d = ggx_d_aniso(wh, m.alpha_x, m.alpha_y);
  float g = ggx_g2_aniso(wo, wi, m.alpha_x, m.alpha_y);
  float f = fresnel_dielectric(dwo, m.ior);
  float co = fabsf(wo.z), ci = fabsf(wi.z);
  if (co < 1e-8f || ci < 1e-8f) return v3s(0.f);
  float denom = dwo + eta * dwi;
  float denom2 = denom * denom;
  if (fabsf(denom) < 1e-8f) return v3s(0.f);
  float factor = fabsf(dwo * dwi) * (eta * eta) / (co * ci * denom2);
  return mat_base(m) * ((1.f - f) * d * g * factor);
}
__device__ __forceinline__ float mft_pdf(V3 wo, V3 wi, const DevMaterial& m) {
  if (wo.z == 0.f || wi.z == 0.f) return 0.f;
  if (same_hemisphere(wo, wi)) return 0.f;
  const float eta = (wo.z > 0.f) ? (1.f / m.ior) : m.ior;
  V3 wh = normalize(wo + eta * wi);
  if (wh.z < 0.f) wh = -wh;
  float dwo = dot(wo, wh), dwi = dot(wi, wh);
  if (dwo * dwi >= 0.f) return 0.f;
  float pwh = vndf_pdf(wo, wh, m.alpha_x, m.alpha_y);
  float denom = dwo + eta * dwi;
  if (fabsf(denom) < 1e-8f) return 0.f;
  float dwh = fabsf((eta * eta * dwi) / (denom * denom));
  return pwh * dwh;
}
__device__ __forceinline__ bool mft_sample(V3 wo, const DevMaterial& m, Pcg& rng, BsdfSample& s) {
  if (fabsf(wo.z) < 1e-8f) return false;
  // The reference passes rng.next_float() twice as call arguments; GCC evaluates them right
  // to left, so the first draw is the second parameter (u2). Kept for sample-exact parity.
  float u2 = rng.next_float();
  float u1 = rng.next_float();
  V3 wh = sample_vndf(wo, m.alpha_x, m.alpha_y, u1, u2);
  if (wh.z < 0.f) wh = -wh;
  const float eta = (wo.z > 0.f) ? (1.f / m.ior) : m.ior;
  float dwo = dot(wo, wh);
  float s2o = smax(0.f, 1.f - dwo * dwo);
  float s2i = eta * eta * s2o;
  if (s2i >= 1.f) return false;
  float cti = sqrtf(smax(0.f, 1.f - s2i));
  float sg = (dwo > 0.f) ? 1.f : -1.f;
  s.wi = normalize((-eta * wo) + (eta * dwo - sg * cti) * wh);
  if (same_hemisphere(wo, s.wi)) return false;
  s.pdf = mft_pdf(wo, s.wi, m);
  if (s.pdf < 1e-8f) return false;
  s.f = mft_eval(wo, s.wi, m);
  s.delta = false;
  return true;
}

// ── delta lobes ────────────────────────────────────────────────────────────────
__device__ __forceinline__ bool delta_refl_sample(V3 wo, const DevMaterial& m, BsdfSample& s) {
  if (fabsf(wo.z) < 1e-8f) return false;
  V3 n = v3(0.f, 0.f, (wo.z > 0.f) ? 1.f : -1.f);
  s.wi = reflect(-wo, n);
  V3 fv = (m.flags & kMatConductor) ? fresnel_schlick(fabsf(wo.z), mat_f0(m))
                                    : v3s(fresnel_dielectric(fabsf(wo.z), m.ior));
  float ci = fabsf(s.wi.z);
  if (ci < 1e-8f) return false;
  s.f = fv / ci;
  s.pdf = 1.f;
  s.delta = true;
  return true;
}

// refract (src/math/vec3.h:62-69)
__device__ __forceinline__ bool refract(V3 v, V3 n, float eta, V3& out) {
  float ci = -dot(normalize(v), n);
  float s2t = eta * eta * (1.f - ci * ci);
  if (s2t >= 1.f) return false;
  out = eta * v + (eta * ci - sqrtf(1.f - s2t)) * n;
  return true;
}

__device__ __forceinline__ bool delta_trans_sample(V3 wo, const DevMaterial& m, BsdfSample& s) {
  if (fabsf(wo.z) < 1e-8f) return false;
  float eta = (wo.z > 0.f) ? (1.f / m.ior) : m.ior;
  V3 n = v3(0.f, 0.f, (wo.z > 0.f) ? 1.f : -1.f);
  if (!refract(-wo, n, eta, s.wi)) return false;
  s.wi = normalize(s.wi);
  float f = fresnel_dielectric(fabsf(wo.z), m.ior);
  float ci = fabsf(s.wi.z);
  if (ci < 1e-8f) return false;
  s.f = mat_base(m) * ((1.f - f) * eta * eta / ci);
  s.pdf = 1.f;
  s.delta = true;
  return true;
}

// ── subsurface (diffuse-like) ──────────────────────────────────────────────────
__device__ __forceinline__ V3 ss_color(const DevMaterial& m) {
  return lerp(mat_base(m), v3(m.ss_color[0], m.ss_color[1], m.ss_color[2]), m.subsurface);
}

__device__ __forceinline__ bool cosine_sample(V3 wo, V3 color, const DevMaterial& m, Pcg& rng,
                                              BsdfSample& s) {
  // The reference passes rng.next_float() twice as call arguments; GCC evaluates them right
  // to left, so the first draw is the second parameter (u2). Kept for sample-exact parity.
  float u2 = rng.next_float();
  float u1 = rng.next_float();
  s.wi = sample_cosine_hemisphere(u1, u2);
  if (wo.z < 0.f) s.wi.z = -s.wi.z;
  s.pdf = fabsf(s.wi.z) * kInvPi;
  if (s.pdf < 1e-8f) return false;
  s.f = color * (1.f - m.metallic) * kInvPi;
  s.delta = false;
  return true;
}

// ── combined eval / pdf for NEE (bsdf.h:601-657) ───────────────────────────────
// The three entry points the bounce kernels call: inlined (the default build) or, built with
// XB_BSDF_CALLS, kept as calls so that a bounce kernel holds one copy of each body (its two NEE
// sites evaluate the BSDF) — less code for the instruction cache, more register traffic at the calls.
#ifdef XB_BSDF_CALLS
#define XB_BSDF_ENTRY __device__ __noinline__
#else
#define XB_BSDF_ENTRY __device__ __forceinline__
#endif

// kOpaque: the scene has no delta, transmissive or subsurface material (the renderer checks at
// upload), so those branches are left out of the bounce kernel's code; the same arithmetic runs
// for every material it does have.
template <bool kOpaque>
__device__ __forceinline__ uint32_t lobe_flags(const DevMaterial& m) {
  return kOpaque ? (m.flags & kMatConductor) : m.flags;
}

template <bool kOpaque = false>
XB_BSDF_ENTRY V3 bsdf_eval(V3 wo, V3 wi, const DevMaterial& m) {
  const uint32_t fl = lobe_flags<kOpaque>(m);
  if (fl & kMatDelta) return v3s(0.f);
  if (fl & kMatConductor) return mfr_eval(wo, wi, m);
  if (fl & kMatTransmissive) return (wi.z > 0.f) ? mfr_eval(wo, wi, m) : mft_eval(wo, wi, m);
  if (fl & kMatSubsurface) {
    if (wi.z <= 0.f) return v3s(0.f);
    return ss_color(m) * (1.f - m.metallic) * kInvPi;
  }
  float spec = m.f0[0];
  float diff = 1.f - spec;
  if (wi.z > 0.f) return diffuse_eval(wi, m) * diff + mfr_eval(wo, wi, m) * spec;
  return v3s(0.f);
}

template <bool kOpaque = false>
XB_BSDF_ENTRY float bsdf_pdf(V3 wo, V3 wi, const DevMaterial& m) {
  const uint32_t fl = lobe_flags<kOpaque>(m);
  if (fl & kMatDelta) return 0.f;
  if (fl & kMatConductor) return mfr_pdf(wo, wi, m);
  if (fl & kMatTransmissive) {
    float f = fresnel_dielectric(fabsf(wo.z), m.ior);
    if (wi.z > 0.f) return f * mfr_pdf(wo, wi, m);
    return (1.f - f) * mft_pdf(wo, wi, m);
  }
  if (fl & kMatSubsurface) return diffuse_pdf(wi);
  float spec = m.f0[0];
  float diff = 1.f - spec;
  if (wi.z > 0.f) return diffuse_pdf(wi) * diff + mfr_pdf(wo, wi, m) * spec;
  return 0.f;
}

// ── lobe selection and sampling (bsdf.h:666-708) ───────────────────────────────
template <bool kOpaque = false>
XB_BSDF_ENTRY bool bsdf_sample(V3 wo, const DevMaterial& m, Pcg& rng, BsdfSample& s) {
  s.delta = false;
  s.pdf = 0.f;
  s.f = v3s(0.f);
  s.wi = v3s(0.f);
  const uint32_t fl = lobe_flags<kOpaque>(m);
  if (fl & kMatDelta) {
    if (fl & kMatTransmissive) {
      float f = fresnel_dielectric(wo.z, m.ior);
      if (rng.next_float() < f) return delta_refl_sample(wo, m, s);
      return delta_trans_sample(wo, m, s);
    }
    return delta_refl_sample(wo, m, s);
  }
  if (fl & kMatConductor) return mfr_sample(wo, m, rng, s);
  if (fl & kMatSubsurface) return cosine_sample(wo, ss_color(m), m, rng, s);
  if (fl & kMatTransmissive) {
    float f = fresnel_dielectric(fabsf(wo.z), m.ior);
    if (rng.next_float() < f) {
      if (!mfr_sample(wo, m, rng, s)) return false;
      s.pdf *= f;
      return true;
    }
    if (!mft_sample(wo, m, rng, s)) return false;
    s.pdf *= (1.f - f);
    return true;
  }
  float spec = sclamp(m.f0[0], 0.f, 1.f);
  float diff = 1.f - spec;
  if (rng.next_float() < spec) {
    if (!mfr_sample(wo, m, rng, s)) return false;
    s.pdf *= spec;
    return true;
  }
  if (!cosine_sample(wo, mat_base(m), m, rng, s)) return false;
  s.pdf *= diff;
  return true;
}

// ── the sampler's true densities (guided sampling; no reference counterpart) ──────
// The reference's anisotropic GGX distribution (ggx_d_aniso, bsdf.h:67-76) squares
// cos^4(theta_h) (1 + tan^2 ...) in its denominator, so every pdf built on it is the density of
// the standard GGX visible normals divided by cos^4(theta_h). Its sampler (sample_vndf, Heitz
// 2018) draws the standard visible normals, so the density of what mfr_sample actually returns
// is the stated pdf times cos^4(theta_h). The plain tracer never needs the difference (it divides
// f by the pdf of its own sample, where D cancels), but guided sampling weighs directions drawn
// elsewhere by the sampler's density, which must be the true one.
__device__ __forceinline__ float cos4(float c) { const float c2 = c * c; return c2 * c2; }

__device__ __forceinline__ float mfr_density(V3 wo, V3 wi, const DevMaterial& m) {
  const float p = mfr_pdf(wo, wi, m);
  if (!(p > 0.f)) return 0.f;
  return p * cos4(normalize(wo + wi).z);
}

// For a non-delta, non-transmissive material seen from its front side (wo.z > 0), bsdf_sample
// draws a lobe l with probability P_l and a direction from that lobe, returning f_l and its
// stated P_l pdf_l. Given a direction wi drawn by another proposal, this returns what the sampler
// would have returned had it produced wi — a lobe chosen with its posterior P_l d_l(wi) /
// sum_k P_k d_k(wi) (d: true densities; u selects it), that lobe's f and stated P_l pdf_l — and
// the sampler's true marginal density sum_k P_k d_k(wi). Returns false where the sampler cannot
// produce wi.
__device__ __forceinline__ bool bsdf_lobe_for_direction(V3 wo, V3 wi, const DevMaterial& m, float u, V3& f,
                                                        float& pdf_sel, float& density) {
  if (m.flags & kMatConductor) {
    pdf_sel = mfr_pdf(wo, wi, m);
    density = mfr_density(wo, wi, m);
    f = mfr_eval(wo, wi, m);
  } else if (m.flags & kMatSubsurface) {
    pdf_sel = density = diffuse_pdf(wi);
    f = (wi.z > 0.f) ? ss_color(m) * (1.f - m.metallic) * kInvPi : v3s(0.f);
  } else {
    const float spec = sclamp(m.f0[0], 0.f, 1.f), diff = 1.f - spec;
    const float ds = spec * mfr_density(wo, wi, m), dd = diff * diffuse_pdf(wi);
    density = ds + dd;
    if (!(density > 0.f)) return false;
    if (u * density < ds) {
      pdf_sel = spec * mfr_pdf(wo, wi, m);
      f = mfr_eval(wo, wi, m);
    } else {
      pdf_sel = dd;
      f = diffuse_eval(wi, m);
    }
  }
  return pdf_sel >= 1e-8f && density > 0.f;
}

// The true density with which bsdf_sample (front side; non-delta, non-transmissive material)
// returns wi, over all lobes.
__device__ __forceinline__ float bsdf_density(V3 wo, V3 wi, const DevMaterial& m) {
  if (m.flags & kMatConductor) return mfr_density(wo, wi, m);
  if (m.flags & kMatSubsurface) return diffuse_pdf(wi);
  const float spec = sclamp(m.f0[0], 0.f, 1.f);
  return spec * mfr_density(wo, wi, m) + (1.f - spec) * diffuse_pdf(wi);
}

}  // namespace xbd

