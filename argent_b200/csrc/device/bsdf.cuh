// bsdf.cuh — per-hit scattering (crates/argent-core/src/bsdf.rs) and the
// material -> BSDF mapping (material.rs:96-138, 157-237) on the device.
#pragma once
#include "../../../include/argent_gpu.h"
#include "sampler.cuh"
#include "spectral.cuh"

namespace dev {

enum BsdfKind { B_CONDUCTOR = 0, B_COATED = 1, B_DIFFUSE = 2, B_DIELECTRIC = 3, B_BLACK = 4, B_OPAL = 5 };

struct Bsdf {
  int kind;
  Ggx ggx;
  Spec eta, k;  // conductor eta/k; dielectric eta
  // Conductor: F(1) per wavelength and E(wo.z), which argent recomputes on
  // every eval (bsdf.rs:62-64); both depend only on the hit, so they are
  // evaluated once per hit (same values).
  Spec f0;
  float e_wo;
  float eta1;   // coated eta
  Spec base;    // coated base, diffuse albedo, opal body
  V3 n;         // opal lattice normal (local)
  float spacing_nm, strength, w;
  Spec lambda;
};

struct BsdfSample {
  V3 wi;
  Spec f;
  float pdf;
  bool delta, transmit, terminate_secondary;
};

__device__ __forceinline__ bool bsdf_is_delta(const Bsdf& b) {
  if (b.kind == B_DIELECTRIC) return true;
  if (b.kind == B_CONDUCTOR) return is_smooth(b.ggx);
  return false;
}

// bsdf.rs:257-264
__device__ __forceinline__ float coat_spec_prob(float cos_o, float eta, const Spec& base) {
  float f = fresnel_dielectric(cos_o, eta);
  float d = average(base) * (1.0f - f);
  return rclamp(f / fmaxf(f + d, 1e-6f), 0.15f, 0.95f);
}

// Coated lobe eval/pdf (bsdf.rs:67-78, 105-113), shared by plastic, patina
// and the opal body.
__device__ __forceinline__ Spec coated_eval(Ggx ggx, float eta, const Spec& base, V3 wo, V3 wi) {
  if (wo.z <= 0.0f || wi.z <= 0.0f) return spec(0.0f);
  V3 h = normalize(wo + wi);
  float fs = fresnel_dielectric(dot(wo, h), eta);
  float sp = ggx_d(ggx, h) * ggx_g2(ggx, wo, wi) * fs / (4.0f * wo.z * wi.z);
  float fo = fresnel_dielectric(wo.z, eta);
  float fi = fresnel_dielectric(wi.z, eta);
  return base * ((1.0f - fo) * (1.0f - fi) * ARGENT_FRAC_1_PI_F) + spec(sp);
}
__device__ __forceinline__ float coated_pdf(Ggx ggx, float eta, const Spec& base, V3 wo, V3 wi) {
  if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f;
  float ps = coat_spec_prob(wo.z, eta, base);
  V3 h = normalize(wo + wi);
  float p_spec = ggx_d_visible(ggx, wo, h) / (4.0f * fmaxf(dot(wo, h), 1e-8f));
  return ps * p_spec + (1.0f - ps) * wi.z * ARGENT_FRAC_1_PI_F;
}

// coated_eval and coated_pdf of the same directions, sharing the half
// vector and the Fresnel term of wo: the same values as the two calls.
__device__ __forceinline__ void coated_eval_pdf(Ggx ggx, float eta, const Spec& base, V3 wo, V3 wi, Spec* f,
                                                float* pdf) {
  if (wo.z <= 0.0f || wi.z <= 0.0f) {
    *f = spec(0.0f);
    *pdf = 0.0f;
    return;
  }
  V3 h = normalize(wo + wi);
  float fo = fresnel_dielectric(wo.z, eta);
  float fs = fresnel_dielectric(dot(wo, h), eta);
  float sp = ggx_d(ggx, h) * ggx_g2(ggx, wo, wi) * fs / (4.0f * wo.z * wi.z);
  float fi = fresnel_dielectric(wi.z, eta);
  *f = base * ((1.0f - fo) * (1.0f - fi) * ARGENT_FRAC_1_PI_F) + spec(sp);
  // coat_spec_prob(wo.z, eta, base) from the same Fresnel value
  float d = average(base) * (1.0f - fo);
  float ps = rclamp(fo / fmaxf(fo + d, 1e-6f), 0.15f, 0.95f);
  float p_spec = ggx_d_visible(ggx, wo, h) / (4.0f * fmaxf(dot(wo, h), 1e-8f));
  *pdf = ps * p_spec + (1.0f - ps) * wi.z * ARGENT_FRAC_1_PI_F;
}

// bsdf.rs:219-254
__device__ __forceinline__ float bragg(float spacing_nm, float cos_t, float l) {
  float peak = 2.0f * spacing_nm * 1.37f * rclamp(cos_t, 0.0f, 1.0f);
  float sigma = 0.045f * fmaxf(peak, 1.0f);
  float x = (l - peak) / sigma;
  return expf(-0.5f * x * x);
}
__device__ Spec opal_flake_eval(V3 n, Ggx ggx, float spacing, float strength, const Spec& lambda, V3 wo, V3 wi) {
  Frame fr = make_frame(n);
  V3 a = to_local(fr, wo), b = to_local(fr, wi);
  if (a.z <= 0.0f || b.z <= 0.0f) return spec(0.0f);
  V3 h = normalize(a + b);
  float g = ggx_d(ggx, h) * ggx_g2(ggx, a, b) / (4.0f * a.z * b.z);
  float cos_t = dot(a, h);
  Spec r;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.v[i] = strength * bragg(spacing, cos_t, lambda.v[i]);
  return r * (g * b.z / fmaxf(wi.z, 1e-6f));
}
__device__ float opal_flake_pdf(V3 n, Ggx ggx, V3 wo, V3 wi) {
  Frame fr = make_frame(n);
  V3 a = to_local(fr, wo), b = to_local(fr, wi);
  if (a.z <= 0.0f || b.z <= 0.0f) return 0.0f;
  V3 h = normalize(a + b);
  return ggx_d_visible(ggx, a, h) / (4.0f * fmaxf(dot(a, h), 1e-8f));
}

// Shading kernels are specialised per material class; KM is the set of BSDF
// kinds (bit per BsdfKind) a class can produce, so the other kinds' code is
// left out of that kernel.
#define KM_ALL 0x3Fu
#define KM_HAS(KM, K) (((KM) >> (K)) & 1u)

// bsdf.rs:53-95
template <unsigned KM = KM_ALL>
__device__ Spec bsdf_eval(const Bsdf& b, V3 wo, V3 wi) {
  switch (b.kind) {
    case B_CONDUCTOR: {
      if constexpr (!KM_HAS(KM, B_CONDUCTOR)) return spec(0.0f);
      if (wo.z <= 0.0f || wi.z <= 0.0f || is_smooth(b.ggx)) return spec(0.0f);
      V3 h = normalize(wo + wi);
      Spec f = fresnel_conductor(dot(wo, h), b.eta, b.k);
      float base = ggx_d(b.ggx, h) * ggx_g2(b.ggx, wo, wi) / (4.0f * wo.z * wi.z);
      float e = b.e_wo;
      return f * base * (spec(1.0f) + b.f0 * ((1.0f - e) / e));
    }
    case B_COATED:
      if constexpr (!KM_HAS(KM, B_COATED)) return spec(0.0f);
      return coated_eval(b.ggx, b.eta1, b.base, wo, wi);
    case B_DIFFUSE:
      if constexpr (!KM_HAS(KM, B_DIFFUSE)) return spec(0.0f);
      if (wo.z <= 0.0f || wi.z <= 0.0f) return spec(0.0f);
      return b.base * ARGENT_FRAC_1_PI_F;
    case B_OPAL: {
      if constexpr (!KM_HAS(KM, B_OPAL)) return spec(0.0f);
      if (wo.z <= 0.0f || wi.z <= 0.0f) return spec(0.0f);
      Spec bb = coated_eval(ggx_from_roughness(0.12f), 1.45f, b.base, wo, wi);
      Spec flake = opal_flake_eval(b.n, b.ggx, b.spacing_nm, b.strength, b.lambda, wo, wi);
      return bb * (1.0f - b.w) + flake * b.w;
    }
    default:
      return spec(0.0f);
  }
}

// bsdf.rs:97-131
template <unsigned KM = KM_ALL>
__device__ float bsdf_pdf(const Bsdf& b, V3 wo, V3 wi) {
  switch (b.kind) {
    case B_CONDUCTOR: {
      if constexpr (!KM_HAS(KM, B_CONDUCTOR)) return 0.0f;
      if (wo.z <= 0.0f || wi.z <= 0.0f || is_smooth(b.ggx)) return 0.0f;
      V3 h = normalize(wo + wi);
      return ggx_d_visible(b.ggx, wo, h) / (4.0f * fmaxf(dot(wo, h), 1e-8f));
    }
    case B_COATED:
      if constexpr (!KM_HAS(KM, B_COATED)) return 0.0f;
      return coated_pdf(b.ggx, b.eta1, b.base, wo, wi);
    case B_DIFFUSE:
      if constexpr (!KM_HAS(KM, B_DIFFUSE)) return 0.0f;
      if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f;
      return wi.z * ARGENT_FRAC_1_PI_F;
    case B_OPAL: {
      if constexpr (!KM_HAS(KM, B_OPAL)) return 0.0f;
      if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f;
      float pb = coated_pdf(ggx_from_roughness(0.12f), 1.45f, b.base, wo, wi);
      return pb * (1.0f - b.w) + opal_flake_pdf(b.n, b.ggx, wo, wi) * b.w;
    }
    default:
      return 0.0f;
  }
}

// bsdf_eval and bsdf_pdf of the same directions; conductor and coated lobes
// share their half vector (and the coat its Fresnel term of wo).
template <unsigned KM = KM_ALL>
__device__ __forceinline__ void bsdf_eval_pdf(const Bsdf& b, V3 wo, V3 wi, Spec* f, float* pdf) {
  if (KM_HAS(KM, B_COATED) && b.kind == B_COATED) {
    coated_eval_pdf(b.ggx, b.eta1, b.base, wo, wi, f, pdf);
    return;
  }
  if (KM_HAS(KM, B_CONDUCTOR) && b.kind == B_CONDUCTOR) {
    if (wo.z <= 0.0f || wi.z <= 0.0f || is_smooth(b.ggx)) {
      *f = spec(0.0f);
      *pdf = 0.0f;
      return;
    }
    V3 h = normalize(wo + wi);
    Spec fr = fresnel_conductor(dot(wo, h), b.eta, b.k);
    float base = ggx_d(b.ggx, h) * ggx_g2(b.ggx, wo, wi) / (4.0f * wo.z * wi.z);
    float e = b.e_wo;
    *f = fr * base * (spec(1.0f) + b.f0 * ((1.0f - e) / e));
    *pdf = ggx_d_visible(b.ggx, wo, h) / (4.0f * fmaxf(dot(wo, h), 1e-8f));
    return;
  }
  *f = bsdf_eval<KM>(b, wo, wi);
  *pdf = bsdf_pdf<KM>(b, wo, wi);
}

// Coated lobe sampling (bsdf.rs:164-182).
__device__ __forceinline__ bool coated_sample(Ggx ggx, float eta, const Spec& base, V3 wo, float u0, float u1,
                                              float u2, BsdfSample* out) {
  if (wo.z <= 0.0f) return false;
  float ps = coat_spec_prob(wo.z, eta, base);
  V3 wi;
  if (u0 < ps) {
    V3 h = ggx_sample_h(ggx, wo, u1, u2);
    wi = reflect(wo, h);
  } else {
    wi = cosine_hemisphere(u1, u2);
  }
  if (wi.z <= 0.0f) return false;
  float p;
  Spec f;
  coated_eval_pdf(ggx, eta, base, wo, wi, &f, &p);
  if (p <= 0.0f) return false;
  out->wi = wi;
  out->f = f;
  out->pdf = p;
  out->delta = out->transmit = out->terminate_secondary = false;
  return true;
}

// bsdf.rs:133-239
template <unsigned KM = KM_ALL>
__device__ bool bsdf_sample(const Bsdf& b, V3 wo, float u0, float u1, float u2, BsdfSample* out) {
  out->delta = out->transmit = out->terminate_secondary = false;
  switch (b.kind) {
    case B_CONDUCTOR: {
      if constexpr (!KM_HAS(KM, B_CONDUCTOR)) return false;
      if (wo.z <= 0.0f) return false;
      if (is_smooth(b.ggx)) {
        V3 wi{-wo.x, -wo.y, wo.z};
        out->wi = wi;
        out->f = fresnel_conductor(wo.z, b.eta, b.k) / fmaxf(wi.z, 1e-8f);
        out->pdf = 1.0f;
        out->delta = true;
        return true;
      }
      V3 h = ggx_sample_h(b.ggx, wo, u1, u2);
      V3 wi = reflect(wo, h);
      if (wi.z <= 0.0f) return false;
      out->wi = wi;
      out->pdf = ggx_d_visible(b.ggx, wo, h) / (4.0f * fmaxf(dot(wo, h), 1e-8f));
      out->f = bsdf_eval<KM>(b, wo, wi);
      return true;
    }
    case B_COATED:
      if constexpr (!KM_HAS(KM, B_COATED)) return false;
      return coated_sample(b.ggx, b.eta1, b.base, wo, u0, u1, u2, out);
    case B_DIFFUSE: {
      if constexpr (!KM_HAS(KM, B_DIFFUSE)) return false;
      if (wo.z <= 0.0f) return false;
      V3 wi = cosine_hemisphere(u1, u2);
      float p = wi.z * ARGENT_FRAC_1_PI_F;
      if (p <= 0.0f) return false;
      out->wi = wi;
      out->f = b.base * ARGENT_FRAC_1_PI_F;
      out->pdf = p;
      return true;
    }
    case B_DIELECTRIC: {
      if constexpr (!KM_HAS(KM, B_DIELECTRIC)) return false;
      bool dispersive = (max_value(b.eta) - min_value(b.eta)) > 1e-5f;
      float e0 = b.eta.v[0];
      float cos_o = wo.z;
      float f0 = fresnel_dielectric(cos_o, e0);
      if (u0 < f0) {
        V3 wi{-wo.x, -wo.y, wo.z};
        float c = fmaxf(fabsf(wi.z), 1e-8f);
        Spec f;
#pragma unroll
        for (int i = 0; i < 4; ++i) f.v[i] = fresnel_dielectric(cos_o, b.eta.v[i]);
        out->wi = wi;
        out->f = f / c;
        out->pdf = f0;
        out->delta = true;
        return true;
      }
      bool entering = cos_o > 0.0f;
      float etap = entering ? e0 : 1.0f / e0;
      V3 nn = entering ? V3{0.0f, 0.0f, 1.0f} : V3{0.0f, 0.0f, -1.0f};
      V3 wi;
      if (!refract(wo, nn, etap, &wi)) return false;
      float c = fmaxf(fabsf(wi.z), 1e-8f);
      float ft = (1.0f - f0) / (c * etap * etap);
      out->wi = wi;
      out->f = spec(ft);
      out->pdf = 1.0f - f0;
      out->delta = true;
      out->transmit = true;
      out->terminate_secondary = dispersive;
      return true;
    }
    case B_OPAL: {
      if constexpr (!KM_HAS(KM, B_OPAL)) return false;
      if (wo.z <= 0.0f) return false;
      V3 wi;
      if (u0 < b.w) {
        Frame fr = make_frame(b.n);
        V3 wol = to_local(fr, wo);
        if (wol.z <= 0.0f) return false;
        V3 h = ggx_sample_h(b.ggx, wol, u1, u2);
        wi = to_world(fr, reflect(wol, h));
      } else {
        BsdfSample s;
        if (!coated_sample(ggx_from_roughness(0.12f), 1.45f, b.base, wo, (u0 - b.w) / fmaxf(1.0f - b.w, 1e-6f), u1, u2,
                           &s))
          return false;
        wi = s.wi;
      }
      if (wi.z <= 0.0f) return false;
      float p = bsdf_pdf<KM>(b, wo, wi);
      if (p <= 0.0f) return false;
      out->wi = wi;
      out->f = bsdf_eval<KM>(b, wo, wi);
      out->pdf = p;
      return true;
    }
    default:
      return false;
  }
}

// ---------------------------------------------------------------- materials

// material.rs:196-205
__device__ __forceinline__ uint32_t hash3(int32_t i, int32_t j, int32_t k, uint32_t salt) {
  uint32_t h = ((uint32_t)i * 0x8da6b343u) ^ ((uint32_t)j * 0xd8163841u) ^ ((uint32_t)k * 0xcb1ab31fu) ^ salt;
  return hash32(h);
}
__device__ __forceinline__ float unit01(uint32_t h) { return (float)(h >> 8) / 16777216.0f; }

// material.rs:208-237: jittered-grid Voronoi over 27 cells.
__device__ void opal_domain(V3 p, V3* dir, float* spacing, float* brightness) {
  int32_t fx = (int32_t)floorf(p.x), fy = (int32_t)floorf(p.y), fz = (int32_t)floorf(p.z);
  float bd = 3.40282347e38f;
  int32_t bi = 0, bj = 0, bk = 0;
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        int32_t i = fx + dx, j = fy + dy, k = fz + dz;
        V3 c{(float)i + unit01(hash3(i, j, k, 1)), (float)j + unit01(hash3(i, j, k, 2)),
             (float)k + unit01(hash3(i, j, k, 3))};
        float d2 = length_squared(c - p);
        if (d2 < bd) {
          bd = d2;
          bi = i;
          bj = j;
          bk = k;
        }
      }
  float z = 2.0f * unit01(hash3(bi, bj, bk, 4)) - 1.0f;
  float phi = (2.0f * ARGENT_PI_F) * unit01(hash3(bi, bj, bk, 5));
  float r = sqrtf(fmaxf(1.0f - z * z, 0.0f));
  float sp, cp;
  sincosf(phi, &sp, &cp);
  *dir = V3{r * cp, r * sp, z};
  *spacing = 190.0f + 75.0f * unit01(hash3(bi, bj, bk, 6));
  *brightness = 0.35f + 0.65f * powf(unit01(hash3(bi, bj, bk, 7)), 0.7f);
}

__device__ __forceinline__ bool mat_is_transmissive(const ArgentMaterial* m) {
  return m->kind == ARGENT_MAT_GEM && m->gem_kind == ARGENT_GEM_TRANSPARENT;
}
__device__ __forceinline__ bool mat_has_medium(const ArgentMaterial* m) {
  return m->kind == ARGENT_MAT_GEM && (m->gem_kind == ARGENT_GEM_TRANSPARENT || m->gem_kind == ARGENT_GEM_OPAL);
}

struct HitCtx {
  V3 p_obj, n_world;
  const Frame* frame;
  float turn_s, turn_c;  // sin/cos of +turntable angle (object -> world)
};

// Material classes: the shading kernel a hit goes to.
#define CLS_TERMINAL 0    // miss or panel: emission only, no surface
#define CLS_METAL 1       // Metal (conductor; the patina layer is coated)
#define CLS_COATED 2      // Plastic, opaque gem
#define CLS_DIELECTRIC 3  // transparent gem (and a gem of opal kind)
#define CLS_OTHER 4       // Opal, Diffuse, Black
#define NUM_CLS 5

__host__ __device__ inline int material_class(int kind, int gem_kind) {
  switch (kind) {
    case ARGENT_MAT_METAL:
      return CLS_METAL;
    case ARGENT_MAT_PLASTIC:
      return CLS_COATED;
    case ARGENT_MAT_GEM:
      return gem_kind == ARGENT_GEM_OPAQUE ? CLS_COATED : CLS_DIELECTRIC;
    default:
      return CLS_OTHER;
  }
}

// BSDF kinds each class can produce.
template <int CLS>
struct ClassKinds {
  static constexpr unsigned value = CLS == CLS_METAL        ? ((1u << B_CONDUCTOR) | (1u << B_COATED))
                                    : CLS == CLS_COATED     ? (1u << B_COATED)
                                    : CLS == CLS_DIELECTRIC ? (1u << B_DIELECTRIC)
                                    : CLS == CLS_OTHER      ? ((1u << B_OPAL) | (1u << B_DIFFUSE) | (1u << B_BLACK))
                                                            : 0u;
};

// material.rs:96-138
template <int CLS = -1>
__device__ Bsdf material_bsdf(const ArgentMaterial* m, const Wavelengths& wl, float mask, float u, const HitCtx& ctx) {
  Bsdf b;
  b.kind = B_BLACK;
  b.ggx = Ggx{1e-4f};
  b.eta1 = 1.0f;
  b.w = 0.0f;
  b.spacing_nm = b.strength = 0.0f;
  b.n = V3{0, 0, 1};
  constexpr bool any = CLS < 0;
  switch (m->kind) {
    case ARGENT_MAT_OPAL: {
      if constexpr (!(any || CLS == CLS_OTHER)) return b;
      V3 dir;
      float spacing, brightness;
      opal_domain(ctx.p_obj / m->cell_mm, &dir, &spacing, &brightness);
      V3 nw = normalize(ctx.n_world * 1.2f + rot_y_sc(dir, ctx.turn_s, ctx.turn_c));
      V3 n = to_local(*ctx.frame, nw);
      if (n.z < 0.0f) n = -n;
      b.kind = B_OPAL;
      b.n = n;
      b.ggx = ggx_from_roughness(0.22f);
      b.spacing_nm = spacing;
      b.strength = m->strength * brightness;
#pragma unroll
      for (int i = 0; i < 4; ++i) b.lambda.v[i] = wl.lambda[i];
      b.base = tab_sample(m->spec_a, wl);
      b.w = 0.6f;
      return b;
    }
    case ARGENT_MAT_METAL: {
      if constexpr (!(any || CLS == CLS_METAL)) return b;
      if (m->has_patina) {
        float t = rclamp((mask - m->patina_lo) / fmaxf(m->patina_hi - m->patina_lo, 1e-4f), 0.0f, 1.0f);
        float w = m->patina_strength * t * t * (3.0f - 2.0f * t);
        if (u < w) {
          b.kind = B_COATED;
          b.ggx = Ggx{m->patina_alpha};
          b.eta1 = m->patina_eta;
          b.base = tab_sample(m->spec_a, wl);
          return b;
        }
      }
      b.kind = B_CONDUCTOR;
      b.ggx = Ggx{m->alpha};
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        b.eta.v[i] = grid_eval(m->nk_eta, wl.lambda[i]);
        b.k.v[i] = grid_eval(m->nk_k, wl.lambda[i]);
      }
      return b;
    }
    case ARGENT_MAT_GEM: {
      if constexpr (!(any || CLS == CLS_COATED || CLS == CLS_DIELECTRIC)) return b;
      if (m->gem_kind == ARGENT_GEM_OPAQUE) {
        b.kind = B_COATED;
        b.ggx = ggx_from_roughness(0.06f);
        b.eta1 = tab_eval(m->spec_a, 550.0f);
        b.base = m->has_opaque_base ? tab_sample(m->spec_b2, wl) : spec(0.01f);
        return b;
      }
      b.kind = B_DIELECTRIC;
      b.eta = tab_sample(m->spec_a, wl);
      return b;
    }
    case ARGENT_MAT_PLASTIC:
      if constexpr (!(any || CLS == CLS_COATED)) return b;
      b.kind = B_COATED;
      b.ggx = Ggx{m->alpha};
      b.eta1 = m->eta;
      b.base = tab_sample(m->spec_a, wl);
      return b;
    case ARGENT_MAT_DIFFUSE:
      if constexpr (!(any || CLS == CLS_OTHER)) return b;
      b.kind = B_DIFFUSE;
      b.base = tab_sample(m->spec_a, wl);
      return b;
    default:
      return b;
  }
}

// metals.rs:95-100
__device__ __forceinline__ float mat_r0(const ArgentMaterial* m, float l) {
  float n = grid_eval(m->nk_eta, l);
  float k = grid_eval(m->nk_k, l);
  return ((n - 1.0f) * (n - 1.0f) + k * k) / ((n + 1.0f) * (n + 1.0f) + k * k);
}

// material.rs:157-177
__device__ void guide_rgb(const ArgentMaterial* m, float cavity, float out[3]) {
  const float L[3] = {610.0f, 550.0f, 465.0f};
  switch (m->kind) {
    case ARGENT_MAT_METAL: {
      for (int i = 0; i < 3; ++i) out[i] = mat_r0(m, L[i]);
      if (m->has_patina) {
        float t = rclamp((cavity - m->patina_lo) / fmaxf(m->patina_hi - m->patina_lo, 1e-4f), 0.0f, 1.0f);
        float w = m->patina_strength * t * t * (3.0f - 2.0f * t);
        for (int i = 0; i < 3; ++i) out[i] = out[i] * (1.0f - w) + tab_eval(m->spec_a, L[i]) * w;
      }
      return;
    }
    case ARGENT_MAT_GEM:
      out[0] = out[1] = out[2] = 1.0f;
      return;
    case ARGENT_MAT_OPAL:
    case ARGENT_MAT_PLASTIC:
    case ARGENT_MAT_DIFFUSE:
      for (int i = 0; i < 3; ++i) out[i] = tab_eval(m->spec_a, L[i]);
      return;
    default:
      out[0] = out[1] = out[2] = 0.0f;
  }
}

}  // namespace dev
