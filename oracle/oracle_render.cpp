// oracle_render.cpp — CPU restatement of argent's spectral path tracer:
// render_pass (core/src/render.rs), trace (integrator.rs), Scene
// (scene.rs), lights (light.rs, envmap.rs), materials (material.rs), BSDFs
// (bsdf.rs, microfacet.rs), camera (camera.rs) and white balance (color.rs).
// TEST INFRASTRUCTURE ONLY: this is the checker for the CUDA path.
#include <omp.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "../argent_b200/csrc/data/spectral_tables.h"
#include "../include/argent_gpu.h"
#include "oracle_api.h"
#include "oracle_bvh.h"

namespace orc {

// ---------------------------------------------------------------- CIE (cie.rs)
static const float CIE_Y_INTEGRAL = 106.85692f;  // cie.rs:29

// cie.rs:38-49
static inline void xyz_bar(float lambda, float out[3]) {
  float x = lambda - 360.0f;
  if (!(x >= 0.0f && x <= 470.0f)) {
    out[0] = out[1] = out[2] = 0.0f;
    return;
  }
  size_t i = std::min((size_t)x, (size_t)469);
  float t = x - (float)i;
  const float* a = &ARGENT_CMF_1931_2DEG[3 * i];
  const float* b = &ARGENT_CMF_1931_2DEG[3 * (i + 1)];
  out[0] = a[0] + (b[0] - a[0]) * t;
  out[1] = a[1] + (b[1] - a[1]) * t;
  out[2] = a[2] + (b[2] - a[2]) * t;
}

// cie.rs:55-70
static inline void to_xyz(const Spec& l, const Wavelengths& wl, float xyz[3]) {
  xyz[0] = xyz[1] = xyz[2] = 0.0f;
  for (int i = 0; i < N; ++i) {
    float p = wl.pdf[i];
    if (p == 0.0f || l.v[i] == 0.0f) continue;
    float c[3];
    xyz_bar(wl.lambda[i], c);
    float w = l.v[i] / p;
    xyz[0] += c[0] * w;
    xyz[1] += c[1] * w;
    xyz[2] += c[2] * w;
  }
  float s = 1.0f / ((float)N * CIE_Y_INTEGRAL);
  xyz[0] *= s;
  xyz[1] *= s;
  xyz[2] *= s;
}

// ---------------------------------------------------------------- color.rs
typedef float M3[3][3];
static const M3 BRADFORD = {{0.8951f, 0.2664f, -0.1614f}, {-0.7502f, 1.7135f, 0.0367f}, {0.0389f, -0.0685f, 1.0296f}};
static const M3 BRADFORD_INV = {
    {0.986993f, -0.147054f, 0.159963f}, {0.432305f, 0.51836f, 0.049291f}, {-0.008529f, 0.040043f, 0.968487f}};
static const M3 XYZ_TO_SRGB = {
    {3.2404542f, -1.5371385f, -0.4985314f}, {-0.969266f, 1.8760108f, 0.041556f}, {0.0556434f, -0.2040259f, 1.0572252f}};
static const float D65_WHITE[3] = {0.95047f, 1.0f, 1.08883f};

static void m3_mul(const M3 a, const M3 b, M3 r) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      float s = 0.0f;  // Iterator::sum starts at 0.0 (color.rs:13)
      for (int k = 0; k < 3; ++k) s += a[i][k] * b[k][j];
      r[i][j] = s;
    }
}
static void m3_apply(const M3 m, const float v[3], float out[3]) {
  for (int i = 0; i < 3; ++i) out[i] = m[i][0] * v[0] + m[i][1] * v[1] + m[i][2] * v[2];
}
// color.rs:48-55
static void camera_matrix(bool has_white, const float w[3], M3 out) {
  if (!has_white) {
    std::memcpy(out, XYZ_TO_SRGB, sizeof(M3));
    return;
  }
  float src[3], dst[3];
  m3_apply(BRADFORD, w, src);
  m3_apply(BRADFORD, D65_WHITE, dst);
  M3 d = {{dst[0] / src[0], 0, 0}, {0, dst[1] / src[1], 0}, {0, 0, dst[2] / src[2]}};
  M3 t, cat;
  m3_mul(d, BRADFORD, t);
  m3_mul(BRADFORD_INV, t, cat);
  m3_mul(XYZ_TO_SRGB, cat, out);
}

// ---------------------------------------------------------------- microfacet.rs
static inline float tan2(V3 w) {
  float c2 = w.z * w.z;
  return rmax(1.0f - c2, 0.0f) / rmax(c2, 1e-12f);
}

struct EnergyTable {
  float e[32 * 32];
};
static const EnergyTable& energy_table();

// microfacet.rs:16-91
struct Ggx {
  float alpha;
  static Ggx from_roughness(float r) {
    float rr = rclamp(r, 0.0f, 1.0f);
    return Ggx{rmax(rr * rr, 1e-4f)};
  }
  bool is_smooth() const { return alpha < 1.5e-3f; }
  float d(V3 h) const {
    if (h.z <= 0.0f) return 0.0f;
    float a2 = alpha * alpha;
    float c2 = h.z * h.z;
    float k = c2 * (a2 - 1.0f) + 1.0f;
    return a2 / (PI_F * k * k);
  }
  float lambda(V3 w) const {
    float t2 = tan2(w);
    if (!std::isfinite(t2)) return 0.0f;
    return 0.5f * (-1.0f + std::sqrt(1.0f + alpha * alpha * t2));
  }
  float g1(V3 w) const { return 1.0f / (1.0f + lambda(w)); }
  float g2(V3 wo, V3 wi) const { return 1.0f / (1.0f + lambda(wo) + lambda(wi)); }
  float d_visible(V3 wo, V3 h) const {
    float c = rmax(std::fabs(wo.z), 1e-8f);
    return g1(wo) * rmax(dot(wo, h), 0.0f) * d(h) / c;
  }
  V3 sample_h(V3 wo, float u1, float u2) const {
    float a = alpha;
    V3 vh = normalize(V3(a * wo.x, a * wo.y, wo.z));
    float lensq = vh.x * vh.x + vh.y * vh.y;
    V3 t1 = lensq > 1e-12f ? V3(-vh.y, vh.x, 0.0f) / std::sqrt(lensq) : V3(1, 0, 0);
    V3 t2 = cross(vh, t1);
    float r = std::sqrt(u1);
    float phi = 2.0f * PI_F * u2;
    float p1 = r * std::cos(phi);
    float p2 = r * std::sin(phi);
    float s = 0.5f * (1.0f + vh.z);
    p2 = (1.0f - s) * std::sqrt(rmax(1.0f - p1 * p1, 0.0f)) + s * p2;
    V3 nh = t1 * p1 + t2 * p2 + vh * std::sqrt(rmax(1.0f - p1 * p1 - p2 * p2, 0.0f));
    return normalize(V3(a * nh.x, a * nh.y, rmax(nh.z, 1e-6f)));
  }
  float e(float cos_o) const;
};

// microfacet.rs:100-109
static float energy_lookup(const EnergyTable& t, float mu, float alpha) {
  const int EN = 32;
  float x = rmin(rclamp(mu, 0.0f, 1.0f) * (float)(EN - 1), (float)(EN - 1) - 1e-4f);
  float y = rmin(rclamp(std::sqrt(alpha), 0.0f, 1.0f) * (float)(EN - 1), (float)(EN - 1) - 1e-4f);
  size_t xi = (size_t)x, yi = (size_t)y;
  float fx = x - (float)xi, fy = y - (float)yi;
  auto g = [&](size_t i, size_t j) { return t.e[j * EN + i]; };
  float a = g(xi, yi) * (1.0f - fx) + g(xi + 1, yi) * fx;
  float b = g(xi, yi + 1) * (1.0f - fx) + g(xi + 1, yi + 1) * fx;
  return rclamp(a * (1.0f - fy) + b * fy, 0.05f, 1.0f);
}
float Ggx::e(float cos_o) const { return energy_lookup(energy_table(), cos_o, alpha); }

// microfacet.rs:112-140
static const EnergyTable& energy_table() {
  static EnergyTable t;
  static std::once_flag once;
  std::call_once(once, [] {
    const int EN = 32;
    for (int j = 0; j < EN; ++j) {
      float r = (float)j / (float)(EN - 1);
      Ggx g{rmax(r * r, 1e-4f)};
      for (int i = 0; i < EN; ++i) {
        float mu = rmax((float)i / (float)(EN - 1), 1e-3f);
        V3 wo(std::sqrt(1.0f - mu * mu), 0.0f, mu);
        const int n = 24;
        float sum = 0.0f;
        for (int a = 0; a < n; ++a)
          for (int b = 0; b < n; ++b) {
            float u1 = ((float)a + 0.5f) / (float)n;
            float u2 = ((float)b + 0.5f) / (float)n;
            V3 h = g.sample_h(wo, u1, u2);
            V3 wi = reflect(wo, h);
            if (wi.z > 0.0f) sum += g.g2(wo, wi) / g.g1(wo);
          }
        t.e[j * EN + i] = sum / (float)(n * n);
      }
    }
  });
  return t;
}

// ---------------------------------------------------------------- bsdf.rs
enum BsdfKind { B_CONDUCTOR, B_COATED, B_DIFFUSE, B_DIELECTRIC, B_BLACK, B_OPAL };

struct BsdfSample {
  V3 wi;
  Spec f;
  float pdf;
  bool delta, transmit, terminate_secondary;
};

struct Bsdf {
  BsdfKind kind;
  Ggx ggx;
  Spec eta, k;   // conductor (eta, k); dielectric eta
  float eta1;    // coated eta
  Spec base;     // coated base; diffuse albedo; opal body
  // opal
  V3 n;
  float spacing_nm, strength, w;
  Spec lambda;

  bool is_delta() const {
    if (kind == B_DIELECTRIC) return true;
    if (kind == B_CONDUCTOR) return ggx.is_smooth();
    return false;
  }
  Spec eval(V3 wo, V3 wi) const;
  float pdf(V3 wo, V3 wi) const;
  bool sample(V3 wo, float u0, float u1, float u2, BsdfSample* out) const;
};

static Bsdf make_coated(Ggx g, float eta, Spec base) {
  Bsdf b;
  b.kind = B_COATED;
  b.ggx = g;
  b.eta1 = eta;
  b.base = base;
  return b;
}

// bsdf.rs:257-264
static inline float coat_spec_prob(float cos_o, float eta, const Spec& base) {
  float f = fresnel_dielectric(cos_o, eta);
  float d = base.average() * (1.0f - f);
  return rclamp(f / rmax(f + d, 1e-6f), 0.15f, 0.95f);
}
// bsdf.rs:219-225
static inline float bragg(float spacing_nm, float cos_t, float l) {
  float peak = 2.0f * spacing_nm * 1.37f * rclamp(cos_t, 0.0f, 1.0f);
  float sigma = 0.045f * rmax(peak, 1.0f);
  float x = (l - peak) / sigma;
  return std::exp(-0.5f * x * x);
}
// bsdf.rs:227-244
static Spec opal_flake_eval(V3 n, Ggx ggx, float spacing, float strength, const Spec& lambda, V3 wo, V3 wi) {
  Frame fr(n);
  V3 a = fr.to_local(wo), b = fr.to_local(wi);
  if (a.z <= 0.0f || b.z <= 0.0f) return Spec();
  V3 h = normalize(a + b);
  float g = ggx.d(h) * ggx.g2(a, b) / (4.0f * a.z * b.z);
  float cos_t = dot(a, h);
  Spec r;
  for (int i = 0; i < N; ++i) r.v[i] = strength * bragg(spacing, cos_t, lambda.v[i]);
  return r * (g * b.z / rmax(wi.z, 1e-6f));
}
// bsdf.rs:246-254
static float opal_flake_pdf(V3 n, Ggx ggx, V3 wo, V3 wi) {
  Frame fr(n);
  V3 a = fr.to_local(wo), b = fr.to_local(wi);
  if (a.z <= 0.0f || b.z <= 0.0f) return 0.0f;
  V3 h = normalize(a + b);
  return ggx.d_visible(a, h) / (4.0f * rmax(dot(a, h), 1e-8f));
}

// bsdf.rs:53-95 (eval)
Spec Bsdf::eval(V3 wo, V3 wi) const {
  switch (kind) {
    case B_CONDUCTOR: {
      if (wo.z <= 0.0f || wi.z <= 0.0f || ggx.is_smooth()) return Spec();
      V3 h = normalize(wo + wi);
      Spec f = fresnel_conductor(dot(wo, h), eta, k);
      float base_ = ggx.d(h) * ggx.g2(wo, wi) / (4.0f * wo.z * wi.z);
      float e = ggx.e(wo.z);
      Spec f0 = fresnel_conductor(1.0f, eta, k);
      return f * base_ * (Spec(1.0f) + f0 * ((1.0f - e) / e));
    }
    case B_COATED: {
      if (wo.z <= 0.0f || wi.z <= 0.0f) return Spec();
      V3 h = normalize(wo + wi);
      float fs = fresnel_dielectric(dot(wo, h), eta1);
      float spec = ggx.d(h) * ggx.g2(wo, wi) * fs / (4.0f * wo.z * wi.z);
      float fo = fresnel_dielectric(wo.z, eta1);
      float fi = fresnel_dielectric(wi.z, eta1);
      return base * ((1.0f - fo) * (1.0f - fi) * FRAC_1_PI_F) + Spec(spec);
    }
    case B_DIFFUSE: {
      if (wo.z <= 0.0f || wi.z <= 0.0f) return Spec();
      return base * FRAC_1_PI_F;
    }
    case B_OPAL: {
      if (wo.z <= 0.0f || wi.z <= 0.0f) return Spec();
      Spec b = make_coated(Ggx::from_roughness(0.12f), 1.45f, base).eval(wo, wi);
      Spec flake = opal_flake_eval(n, ggx, spacing_nm, strength, lambda, wo, wi);
      return b * (1.0f - w) + flake * w;
    }
    default:
      return Spec();
  }
}

// bsdf.rs:97-131 (pdf)
float Bsdf::pdf(V3 wo, V3 wi) const {
  switch (kind) {
    case B_CONDUCTOR: {
      if (wo.z <= 0.0f || wi.z <= 0.0f || ggx.is_smooth()) return 0.0f;
      V3 h = normalize(wo + wi);
      return ggx.d_visible(wo, h) / (4.0f * rmax(dot(wo, h), 1e-8f));
    }
    case B_COATED: {
      if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f;
      float ps = coat_spec_prob(wo.z, eta1, base);
      V3 h = normalize(wo + wi);
      float p_spec = ggx.d_visible(wo, h) / (4.0f * rmax(dot(wo, h), 1e-8f));
      return ps * p_spec + (1.0f - ps) * wi.z * FRAC_1_PI_F;
    }
    case B_DIFFUSE:
      if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f;
      return wi.z * FRAC_1_PI_F;
    case B_OPAL: {
      if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f;
      float pb = make_coated(Ggx::from_roughness(0.12f), 1.45f, base).pdf(wo, wi);
      return pb * (1.0f - w) + opal_flake_pdf(n, ggx, wo, wi) * w;
    }
    default:
      return 0.0f;
  }
}

// bsdf.rs:133-239 (sample)
bool Bsdf::sample(V3 wo, float u0, float u1, float u2, BsdfSample* out) const {
  switch (kind) {
    case B_CONDUCTOR: {
      if (wo.z <= 0.0f) return false;
      if (ggx.is_smooth()) {
        V3 wi(-wo.x, -wo.y, wo.z);
        Spec f = fresnel_conductor(wo.z, eta, k) / rmax(wi.z, 1e-8f);
        *out = BsdfSample{wi, f, 1.0f, true, false, false};
        return true;
      }
      V3 h = ggx.sample_h(wo, u1, u2);
      V3 wi = reflect(wo, h);
      if (wi.z <= 0.0f) return false;
      float pdf_ = ggx.d_visible(wo, h) / (4.0f * rmax(dot(wo, h), 1e-8f));
      Spec f = eval(wo, wi);
      *out = BsdfSample{wi, f, pdf_, false, false, false};
      return true;
    }
    case B_COATED: {
      if (wo.z <= 0.0f) return false;
      float ps = coat_spec_prob(wo.z, eta1, base);
      V3 wi;
      if (u0 < ps) {
        V3 h = ggx.sample_h(wo, u1, u2);
        wi = reflect(wo, h);
      } else {
        wi = cosine_hemisphere(u1, u2);
      }
      if (wi.z <= 0.0f) return false;
      float p = pdf(wo, wi);
      if (p <= 0.0f) return false;
      *out = BsdfSample{wi, eval(wo, wi), p, false, false, false};
      return true;
    }
    case B_DIFFUSE: {
      if (wo.z <= 0.0f) return false;
      V3 wi = cosine_hemisphere(u1, u2);
      float p = wi.z * FRAC_1_PI_F;
      if (p <= 0.0f) return false;
      *out = BsdfSample{wi, base * FRAC_1_PI_F, p, false, false, false};
      return true;
    }
    case B_DIELECTRIC: {
      bool dispersive = (eta.max_value() - eta.min_value()) > 1e-5f;
      float e0 = eta.v[0];
      float cos_o = wo.z;
      float f0 = fresnel_dielectric(cos_o, e0);
      if (u0 < f0) {
        V3 wi(-wo.x, -wo.y, wo.z);
        float c = rmax(std::fabs(wi.z), 1e-8f);
        Spec f;
        for (int i = 0; i < N; ++i) f.v[i] = fresnel_dielectric(cos_o, eta.v[i]);
        f = f / c;
        *out = BsdfSample{wi, f, f0, true, false, false};
        return true;
      }
      bool entering = cos_o > 0.0f;
      float etap = entering ? e0 : 1.0f / e0;
      V3 nn = entering ? V3(0, 0, 1) : V3(0, 0, -1);
      V3 wi;
      if (!refract(wo, nn, etap, &wi)) return false;
      float c = rmax(std::fabs(wi.z), 1e-8f);
      float ft = (1.0f - f0) / (c * etap * etap);
      *out = BsdfSample{wi, Spec(ft), 1.0f - f0, true, true, dispersive};
      return true;
    }
    case B_OPAL: {
      if (wo.z <= 0.0f) return false;
      V3 wi;
      if (u0 < w) {
        Frame fr(n);
        V3 wol = fr.to_local(wo);
        if (wol.z <= 0.0f) return false;
        V3 h = ggx.sample_h(wol, u1, u2);
        wi = fr.to_world(reflect(wol, h));
      } else {
        Bsdf b = make_coated(Ggx::from_roughness(0.12f), 1.45f, base);
        BsdfSample s;
        if (!b.sample(wo, (u0 - w) / rmax(1.0f - w, 1e-6f), u1, u2, &s)) return false;
        wi = s.wi;
      }
      if (wi.z <= 0.0f) return false;
      float p = pdf(wo, wi);
      if (p <= 0.0f) return false;
      *out = BsdfSample{wi, eval(wo, wi), p, false, false, false};
      return true;
    }
    default:
      return false;
  }
}

// ---------------------------------------------------------------- materials
struct Material {
  ArgentMaterial d;  // the description (tables)
  bool is_transmissive() const { return d.kind == ARGENT_MAT_GEM && d.gem_kind == ARGENT_GEM_TRANSPARENT; }
  bool wants_flat_normals() const { return is_transmissive(); }
  bool has_medium() const {
    return d.kind == ARGENT_MAT_GEM && (d.gem_kind == ARGENT_GEM_TRANSPARENT || d.gem_kind == ARGENT_GEM_OPAL);
  }
};

// material.rs:196-205
static inline uint32_t hash3(int32_t i, int32_t j, int32_t k, uint32_t salt) {
  uint32_t h = ((uint32_t)i * 0x8da6b343u) ^ ((uint32_t)j * 0xd8163841u) ^ ((uint32_t)k * 0xcb1ab31fu) ^ salt;
  return hash32(h);
}
static inline float unit(uint32_t h) { return (float)(h >> 8) / 16777216.0f; }

struct OpalDomain {
  V3 dir;
  float spacing, brightness;
};
// material.rs:208-237
static OpalDomain opal_domain(V3 p) {
  int32_t fx = (int32_t)std::floor(p.x), fy = (int32_t)std::floor(p.y), fz = (int32_t)std::floor(p.z);
  float bd = 3.40282347e38f;
  int32_t bi = 0, bj = 0, bk = 0;
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        int32_t i = fx + dx, j = fy + dy, k = fz + dz;
        V3 c((float)i + unit(hash3(i, j, k, 1)), (float)j + unit(hash3(i, j, k, 2)),
             (float)k + unit(hash3(i, j, k, 3)));
        float d2 = length_squared(c - p);
        if (d2 < bd) {
          bd = d2;
          bi = i;
          bj = j;
          bk = k;
        }
      }
  float z = 2.0f * unit(hash3(bi, bj, bk, 4)) - 1.0f;
  float phi = (2.0f * PI_F) * unit(hash3(bi, bj, bk, 5));
  float r = std::sqrt(rmax(1.0f - z * z, 0.0f));
  OpalDomain o;
  o.dir = V3(r * std::cos(phi), r * std::sin(phi), z);
  o.spacing = 190.0f + 75.0f * unit(hash3(bi, bj, bk, 6));
  o.brightness = 0.35f + 0.65f * std::pow(unit(hash3(bi, bj, bk, 7)), 0.7f);
  return o;
}

struct HitCtx {
  V3 p_obj, n_world;
  const Frame* frame;
  float turn_deg;
};

// material.rs:96-138
static Bsdf material_bsdf(const Material& m, const Wavelengths& wl, float mask, float u, const HitCtx& ctx) {
  const ArgentMaterial& d = m.d;
  Bsdf b;
  b = Bsdf();
  switch (d.kind) {
    case ARGENT_MAT_OPAL: {
      V3 pc = ctx.p_obj / d.cell_mm;
      OpalDomain od = opal_domain(pc);
      V3 nw = normalize(ctx.n_world * 1.2f + rot_y(od.dir, ctx.turn_deg));
      V3 n = ctx.frame->to_local(nw);
      if (n.z < 0.0f) n = -n;
      b.kind = B_OPAL;
      b.n = n;
      b.ggx = Ggx::from_roughness(0.22f);
      b.spacing_nm = od.spacing;
      b.strength = d.strength * od.brightness;
      for (int i = 0; i < N; ++i) b.lambda.v[i] = wl.lambda[i];
      b.base = tab_sample(d.spec_a, wl);
      b.w = 0.6f;
      return b;
    }
    case ARGENT_MAT_METAL: {
      if (d.has_patina) {
        float t = rclamp((mask - d.patina_lo) / rmax(d.patina_hi - d.patina_lo, 1e-4f), 0.0f, 1.0f);
        float w = d.patina_strength * t * t * (3.0f - 2.0f * t);
        if (u < w) return make_coated(Ggx{d.patina_alpha}, d.patina_eta, tab_sample(d.spec_a, wl));
      }
      b.kind = B_CONDUCTOR;
      b.ggx = Ggx{d.alpha};
      for (int i = 0; i < N; ++i) {
        b.eta.v[i] = grid_eval(d.nk_eta, wl.lambda[i]);
        b.k.v[i] = grid_eval(d.nk_k, wl.lambda[i]);
      }
      return b;
    }
    case ARGENT_MAT_GEM: {
      if (d.gem_kind == ARGENT_GEM_OPAQUE) {
        Spec base = d.has_opaque_base ? tab_sample(d.spec_b2, wl) : Spec(0.01f);
        return make_coated(Ggx::from_roughness(0.06f), tab_eval(d.spec_a, 550.0f), base);
      }
      b.kind = B_DIELECTRIC;
      b.eta = tab_sample(d.spec_a, wl);
      return b;
    }
    case ARGENT_MAT_PLASTIC:
      return make_coated(Ggx{d.alpha}, d.eta, tab_sample(d.spec_a, wl));
    case ARGENT_MAT_DIFFUSE:
      b.kind = B_DIFFUSE;
      b.base = tab_sample(d.spec_a, wl);
      return b;
    default:
      b.kind = B_BLACK;
      return b;
  }
}

// Normal-incidence reflectance of an n,k table (metals.rs:95-100).
static inline float r0_of(const ArgentMaterial& d, float l) {
  float n = grid_eval(d.nk_eta, l);
  float k = grid_eval(d.nk_k, l);
  return ((n - 1.0f) * (n - 1.0f) + k * k) / ((n + 1.0f) * (n + 1.0f) + k * k);
}

// material.rs:157-177
static void guide_rgb(const Material& m, float cavity, float out[3]) {
  static const float L[3] = {610.0f, 550.0f, 465.0f};
  const ArgentMaterial& d = m.d;
  switch (d.kind) {
    case ARGENT_MAT_METAL: {
      for (int i = 0; i < 3; ++i) out[i] = r0_of(d, L[i]);
      if (d.has_patina) {
        float t = rclamp((cavity - d.patina_lo) / rmax(d.patina_hi - d.patina_lo, 1e-4f), 0.0f, 1.0f);
        float w = d.patina_strength * t * t * (3.0f - 2.0f * t);
        for (int i = 0; i < 3; ++i) out[i] = out[i] * (1.0f - w) + tab_eval(d.spec_a, L[i]) * w;
      }
      return;
    }
    case ARGENT_MAT_GEM:
      out[0] = out[1] = out[2] = 1.0f;
      return;
    case ARGENT_MAT_OPAL:
    case ARGENT_MAT_PLASTIC:
    case ARGENT_MAT_DIFFUSE:
      for (int i = 0; i < 3; ++i) out[i] = tab_eval(d.spec_a, L[i]);
      return;
    default:
      out[0] = out[1] = out[2] = 0.0f;
  }
}

// ---------------------------------------------------------------- lights (light.rs)
struct Panel {
  V3 center, hu, hv, n;
  float area;
  bool emits, camera_visible;
  float feather;
  std::vector<float> emission;

  // light.rs:50-63
  bool intersect(const Ray& ray, float t_max, float* t_out) const {
    float denom = dot(ray.d, n);
    if (std::fabs(denom) < 1e-9f) return false;
    float t = dot(center - ray.o, n) / denom;
    if (t <= 1e-6f || t >= t_max) return false;
    V3 p = ray.at(t) - center;
    float a = dot(p, hu) / length_squared(hu);
    float b = dot(p, hv) / length_squared(hv);
    if (std::fabs(a) <= 1.0f && std::fabs(b) <= 1.0f) {
      *t_out = t;
      return true;
    }
    return false;
  }
  // light.rs:76-93
  float profile(V3 p) const {
    if (feather <= 0.0f) return 1.0f;
    V3 q = p - center;
    float a = rmin(std::fabs(dot(q, hu) / length_squared(hu)), 1.0f);
    float b = rmin(std::fabs(dot(q, hv) / length_squared(hv)), 1.0f);
    auto f = [&](float x) {
      float start = 1.0f - feather;
      if (x <= start) return 1.0f;
      float t = (x - start) / feather;
      return 1.0f - 0.75f * t * t * (3.0f - 2.0f * t);
    };
    return f(a) * f(b);
  }
  // light.rs:67-72
  Spec le(V3 p, V3 dir, const Wavelengths& wl) const {
    if (emits && dot(dir, n) < 0.0f) return tab_sample(emission.data(), wl) * profile(p);
    return Spec();
  }
  V3 sample_point(float u, float v) const { return center + hu * (2.0f * u - 1.0f) + hv * (2.0f * v - 1.0f); }
};

struct Floor {
  bool enabled;
  float y;
  int material;
  float fade_start, fade_end;
  // light.rs:142-148
  bool intersect(const Ray& ray, float t_max, float* t_out) const {
    if (std::fabs(ray.d.y) < 1e-9f) return false;
    float t = (y - ray.o.y) / ray.d.y;
    if (t > 1e-5f && t < t_max) {
      *t_out = t;
      return true;
    }
    return false;
  }
  // light.rs:152-162
  float presence(V3 p) const {
    float r = std::sqrt(p.x * p.x + p.z * p.z);
    if (r <= fade_start) return 1.0f;
    if (r >= fade_end) return 0.0f;
    float t = (r - fade_start) / (fade_end - fade_start);
    return 1.0f - t * t * (3.0f - 2.0f * t);
  }
};

// ---------------------------------------------------------------- envmap.rs
static double planck(float lambda_nm, float t) {
  if (t <= 0.0f) return 0.0;
  double c = 299792458.0, h = 6.62606957e-34, kb = 1.3806488e-23;
  double l = (double)lambda_nm * 1e-9;
  double le = (2.0 * h * c * c) / (std::pow(l, 5) * (std::exp((h * c) / (l * kb * (double)t)) - 1.0));
  return le;
}

// envmap.rs:178-257 (LinearRgb)
struct LinearRgb {
  float basis[3][471];
  float inv[3][3];
  static const LinearRgb& get();
  void weights(const float rgb[3], float out[3]) const {
    for (int i = 0; i < 3; ++i) out[i] = inv[i][0] * rgb[0] + inv[i][1] * rgb[1] + inv[i][2] * rgb[2];
  }
  float eval(const float w[3], float l) const {
    float x = rclamp(l - 360.0f, 0.0f, 469.999f);
    size_t i = (size_t)x;
    float f = x - (float)i;
    float v = 0.0f;
    for (int c = 0; c < 3; ++c) v += w[c] * (basis[c][i] * (1.0f - f) + basis[c][i + 1] * f);
    return rmax(v, 0.0f);
  }
};

static float smoothstep_e(float e0, float e1, float x) {
  float t = rclamp((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}

const LinearRgb& LinearRgb::get() {
  static LinearRgb L;
  static std::once_flag once;
  std::call_once(once, [] {
    // Blackbody::new(6504): peak-normalised Planck (spectrum.rs:104-108, 138-143).
    float kelvin = 6504.0f;
    float peak = 2.897772e-3f / kelvin * 1e9f;
    float norm = 1.0f / (float)planck(peak, kelvin);
    for (int i = 0; i < 471; ++i) {
      float l = 360.0f + (float)i;
      float wb = 1.0f - smoothstep_e(470.0f, 515.0f, l);
      float wr = smoothstep_e(565.0f, 610.0f, l);
      float wg = rmax(1.0f - wb - wr, 0.0f);
      float e = (float)planck(l, kelvin) * norm;
      L.basis[0][i] = wr * e;
      L.basis[1][i] = wg * e;
      L.basis[2][i] = wb * e;
    }
    float m[3][3];
    for (int j = 0; j < 3; ++j) {
      float xyz[3] = {0, 0, 0};
      for (int i = 0; i < 471; ++i) {
        float c[3];
        xyz_bar(360.0f + (float)i, c);
        for (int k = 0; k < 3; ++k) xyz[k] += c[k] * L.basis[j][i];
      }
      float s[3] = {xyz[0] / CIE_Y_INTEGRAL, xyz[1] / CIE_Y_INTEGRAL, xyz[2] / CIE_Y_INTEGRAL};
      // cie.rs:74-81
      float rgb[3] = {3.2404542f * s[0] - 1.5371385f * s[1] - 0.4985314f * s[2],
                      -0.969266f * s[0] + 1.8760108f * s[1] + 0.041556f * s[2],
                      0.0556434f * s[0] - 0.2040259f * s[1] + 1.0572252f * s[2]};
      for (int i = 0; i < 3; ++i) m[i][j] = rgb[i];
    }
    // envmap.rs:259-268
    float a = m[0][0], b = m[0][1], c = m[0][2], d = m[1][0], e = m[1][1], f = m[1][2], g = m[2][0], h = m[2][1],
          ii = m[2][2];
    float det = a * (e * ii - f * h) - b * (d * ii - f * g) + c * (d * h - e * g);
    float k = 1.0f / det;
    float inv[3][3] = {{(e * ii - f * h) * k, (c * h - b * ii) * k, (b * f - c * e) * k},
                       {(f * g - d * ii) * k, (a * ii - c * g) * k, (c * d - a * f) * k},
                       {(d * h - e * g) * k, (b * g - a * h) * k, (a * e - b * d) * k}};
    std::memcpy(L.inv, inv, sizeof(inv));
  });
  return L;
}

struct EnvMap {
  int width = 0, height = 0;
  std::vector<float> weights;  // 3 per texel
  std::vector<float> marginal, conditional;
  float total = 0.0f;
  float rotation_deg = 0.0f;

  // envmap.rs:141-177
  void load(const float* rgb, int w, int h, float rot) {
    width = w;
    height = h;
    rotation_deg = rot;
    const LinearRgb& lin = LinearRgb::get();
    weights.resize((size_t)w * h * 3);
    for (size_t i = 0; i < (size_t)w * h; ++i) lin.weights(&rgb[3 * i], &weights[3 * i]);
    conditional.assign((size_t)(w + 1) * h, 0.0f);
    std::vector<float> row_sum(h);
    for (int y = 0; y < h; ++y) {
      float s = std::sin(PI_F * ((float)y + 0.5f) / (float)h);
      size_t base = (size_t)y * (w + 1);
      float acc = 0.0f;
      conditional[base] = 0.0f;
      for (int x = 0; x < w; ++x) {
        const float* c = &rgb[3 * ((size_t)y * w + x)];
        acc += rmax(0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2], 0.0f) * s + 1e-6f;
        conditional[base + x + 1] = acc;
      }
      row_sum[y] = acc;
      for (int x = 0; x <= w; ++x) conditional[base + x] /= acc;
    }
    marginal.assign(h + 1, 0.0f);
    float acc = 0.0f;
    for (int y = 0; y < h; ++y) {
      acc += row_sum[y];
      marginal[y + 1] = acc;
    }
    total = acc / ((float)w * (float)h);
    for (auto& v : marginal) v /= acc;
  }
  // envmap.rs:345-351
  void uv(V3 dir, float* u, float* v) const {
    V3 d = rot_y(dir, -rotation_deg);
    float uu = 0.5f + std::atan2(d.x, -d.z) / (2.0f * PI_F);
    *v = std::acos(rclamp(d.y, -1.0f, 1.0f)) / PI_F;
    // rem_euclid(1.0)
    float r = std::fmod(uu, 1.0f);
    if (r < 0.0f) r += 1.0f;
    *u = r;
  }
  V3 dir(float u, float v) const {
    float phi = (u - 0.5f) * 2.0f * PI_F;
    float theta = v * PI_F;
    float st = std::sin(theta), ct = std::cos(theta);
    V3 d(st * std::sin(phi), ct, -st * std::cos(phi));
    return rot_y(d, rotation_deg);
  }
  size_t texel(float u, float v) const {
    uint32_t x = std::min((uint32_t)sat_u32(u * (float)width), (uint32_t)(width - 1));
    uint32_t y = std::min((uint32_t)sat_u32(v * (float)height), (uint32_t)(height - 1));
    return (size_t)y * width + x;
  }
  static uint32_t sat_u32(float f) {
    if (!(f > 0.0f)) return 0;
    if (f >= 4294967296.0f) return 0xffffffffu;
    return (uint32_t)f;
  }
  Spec eval(V3 d, const Wavelengths& wl) const {
    float u, v;
    uv(d, &u, &v);
    const float* w = &weights[3 * texel(u, v)];
    const LinearRgb& lin = LinearRgb::get();
    Spec r;
    for (int k = 0; k < N; ++k) r.v[k] = lin.eval(w, wl.lambda[k]);
    return r;
  }
  // envmap.rs:375-387
  float pdf(V3 d) const {
    float u, v;
    uv(d, &u, &v);
    float st = std::sin(PI_F * v);
    if (st <= 1e-6f) return 0.0f;
    size_t x = std::min((size_t)sat_u32(u * (float)width), (size_t)width - 1);
    size_t y = std::min((size_t)sat_u32(v * (float)height), (size_t)height - 1);
    size_t row = y * (width + 1);
    float pc = (conditional[row + x + 1] - conditional[row + x]) * (float)width;
    float pm = (marginal[y + 1] - marginal[y]) * (float)height;
    return pc * pm / (2.0f * PI_F * PI_F * st);
  }
  // envmap.rs:390-402
  V3 sample(float u1, float u2, float* pdf_out) const {
    auto pp = [](const float* a, size_t n, float u) {
      size_t lo = 0, hi = n;
      while (lo < hi) {
        size_t mid = (lo + hi) / 2;
        if (a[mid] <= u)
          lo = mid + 1;
        else
          hi = mid;
      }
      return lo;
    };
    size_t y = std::min(std::max(pp(marginal.data(), marginal.size(), u1), (size_t)1), (size_t)height) - 1;
    size_t row = y * (width + 1);
    const float* cond = &conditional[row];
    size_t x = std::min(std::max(pp(cond, (size_t)width + 1, u2), (size_t)1), (size_t)width) - 1;
    float fy = (u1 - marginal[y]) / rmax(marginal[y + 1] - marginal[y], 1e-12f);
    float fx = (u2 - cond[x]) / rmax(cond[x + 1] - cond[x], 1e-12f);
    float u = ((float)x + rclamp(fx, 0.0f, 0.999f)) / (float)width;
    float v = ((float)y + rclamp(fy, 0.0f, 0.999f)) / (float)height;
    V3 d = dir(u, v);
    *pdf_out = pdf(d);
    return d;
  }
};

// light.rs:103-127
struct Env {
  bool is_map = false;
  float power = 1.0f;
  std::vector<float> top, horizon, bottom;
  EnvMap map;
  Spec eval(V3 dir, const Wavelengths& wl) const {
    if (is_map) return map.eval(dir, wl);
    float y = rclamp(dir.y, -1.0f, 1.0f);
    if (y >= 0.0f) {
      float t = std::pow(y, power);
      return spec_lerp(t, tab_sample(horizon.data(), wl), tab_sample(top.data(), wl));
    }
    float t = std::pow(-y, 0.5f);
    return spec_lerp(t, tab_sample(horizon.data(), wl), tab_sample(bottom.data(), wl));
  }
};

// ---------------------------------------------------------------- scene.rs
enum HitKind { H_NONE, H_PIECE, H_PANEL, H_FLOOR };
struct SceneHit {
  HitKind kind = H_NONE;
  float t = 0.0f;
  V3 p, p_obj, ng, ns;
  uint16_t material = 0;
  float cavity = 0.0f;
  int panel = -1;
};

}  // namespace orc

struct oracle_scene {
  std::vector<orc::V3> positions, normals;
  std::vector<uint32_t> triangles;
  std::vector<uint16_t> tri_material;
  std::vector<float> cavity;
  bool has_cavity = false;
  orc::Bvh bvh;
  std::vector<orc::Material> materials;
  std::vector<orc::Panel> panels;
  orc::Env env;
  orc::Floor floor;
  float turntable_deg = 0.0f;
  bool has_white = false;
  float white[3] = {0, 0, 0};
  std::vector<int> lights;
  std::vector<float> light_cdf;
  float env_pick = 0.0f;
};

namespace orc {

// spectrum.rs:413-420, evaluated on a 1 nm table (exact at whole nm).
static float luminance_y_table(const float* t) {
  double y = 0.0;
  for (int i = 0; i <= 470; ++i) {
    float c[3];
    xyz_bar(360.0f + (float)i, c);
    y += (double)tab_eval(t, 360.0f + (float)i) * (double)c[1];
  }
  return (float)(y / (double)CIE_Y_INTEGRAL);
}

// scene.rs:88-110
static void rebuild_lights(oracle_scene* s) {
  s->lights.clear();
  s->light_cdf.clear();
  float acc = 0.0f;
  for (size_t i = 0; i < s->panels.size(); ++i) {
    const Panel& p = s->panels[i];
    if (p.emits) {
      float power = p.area * rmax(luminance_y_table(p.emission.data()), 1e-6f);
      acc += power;
      s->lights.push_back((int)i);
      s->light_cdf.push_back(acc);
    }
  }
  if (acc > 0.0f)
    for (auto& c : s->light_cdf) c /= acc;
  if (s->env.is_map)
    s->env_pick = s->lights.empty() ? 1.0f : 0.5f;
  else
    s->env_pick = 0.0f;
}

static inline V3 to_object(const oracle_scene* s, V3 v) {
  return s->turntable_deg == 0.0f ? v : rot_y(v, -s->turntable_deg);
}
static inline V3 to_world(const oracle_scene* s, V3 v) {
  return s->turntable_deg == 0.0f ? v : rot_y(v, s->turntable_deg);
}

// scene.rs:169-218
static SceneHit scene_intersect(const oracle_scene* s, const Ray& ray, bool camera_ray) {
  SceneHit best;
  float t_max = INFINITY;
  Ray oray{to_object(s, ray.o), to_object(s, ray.d)};
  TriHit h;
  if (s->bvh.intersect(oray, t_max, &h)) {
    t_max = h.t;
    const uint32_t* tri = &s->triangles[3 * (size_t)h.prim];
    V3 a = s->positions[tri[0]], b = s->positions[tri[1]], c = s->positions[tri[2]];
    V3 ng = normalize(cross(b - a, c - a));
    float w = 1.0f - h.u - h.v;
    uint16_t mat = s->tri_material.empty() ? 0 : s->tri_material[h.prim];
    bool flat = s->materials[mat].wants_flat_normals();
    V3 ns;
    if (flat || s->normals.empty()) {
      ns = ng;
    } else {
      V3 na = s->normals[tri[0]], nb = s->normals[tri[1]], nc = s->normals[tri[2]];
      V3 n = na * w + nb * h.u + nc * h.v;
      ns = length_squared(n) > 1e-12f ? normalize(n) : ng;
    }
    float cav = 0.0f;
    if (s->has_cavity) cav = s->cavity[tri[0]] * w + s->cavity[tri[1]] * h.u + s->cavity[tri[2]] * h.v;
    V3 p_obj = a * w + b * h.u + c * h.v;
    best.kind = H_PIECE;
    best.t = h.t;
    best.p = to_world(s, p_obj);
    best.p_obj = p_obj;
    best.ng = to_world(s, ng);
    best.ns = to_world(s, ns);
    best.material = mat;
    best.cavity = cav;
  }
  for (size_t i = 0; i < s->panels.size(); ++i) {
    const Panel& p = s->panels[i];
    if (camera_ray && !p.camera_visible) continue;
    float t;
    if (p.intersect(ray, t_max, &t)) {
      t_max = t;
      best = SceneHit();
      best.kind = H_PANEL;
      best.t = t;
      best.panel = (int)i;
    }
  }
  if (s->floor.enabled) {
    float t;
    if (s->floor.intersect(ray, t_max, &t)) {
      best = SceneHit();
      best.kind = H_FLOOR;
      best.t = t;
      best.p = ray.at(t);
    }
  }
  return best;
}

// scene.rs:123-140
static float sky_visibility(const oracle_scene* s, V3 from, V3 dir) {
  Ray oray{to_object(s, from), to_object(s, dir)};
  if (s->bvh.occluded(oray, INFINITY)) return 0.0f;
  Ray ray{from, dir};
  for (const Panel& p : s->panels) {
    float t;
    if (p.intersect(ray, INFINITY, &t)) return 0.0f;
  }
  if (s->floor.enabled) {
    float t;
    if (s->floor.intersect(ray, INFINITY, &t)) return 1.0f - s->floor.presence(ray.at(t));
  }
  return 1.0f;
}

// scene.rs:143-147
static float light_pick_pdf(const oracle_scene* s, int panel) {
  for (size_t k = 0; k < s->lights.size(); ++k) {
    if (s->lights[k] == panel) {
      float lo = k == 0 ? 0.0f : s->light_cdf[k - 1];
      return s->light_cdf[k] - lo;
    }
  }
  return 0.0f;
}

// scene.rs:149-156
static bool pick_light(const oracle_scene* s, float u, int* li, float* pick) {
  if (s->lights.empty()) return false;
  size_t k = 0;
  {
    size_t lo = 0, hi = s->light_cdf.size();
    while (lo < hi) {
      size_t mid = (lo + hi) / 2;
      if (s->light_cdf[mid] < u)
        lo = mid + 1;
      else
        hi = mid;
    }
    k = std::min(lo, s->lights.size() - 1);
  }
  float lo = k == 0 ? 0.0f : s->light_cdf[k - 1];
  *li = s->lights[k];
  *pick = s->light_cdf[k] - lo;
  return true;
}

// scene.rs:222-243
static bool visible(const oracle_scene* s, V3 from, V3 to, int ignore_panel) {
  V3 d = to - from;
  float dist = length(d);
  V3 dir = d / dist;
  float t_max = dist * (1.0f - 1e-4f);
  Ray oray{to_object(s, from), to_object(s, dir)};
  if (s->bvh.occluded(oray, t_max)) return false;
  Ray ray{from, dir};
  for (size_t i = 0; i < s->panels.size(); ++i) {
    float t;
    if ((int)i != ignore_panel && s->panels[i].intersect(ray, t_max, &t)) return false;
  }
  if (s->floor.enabled) {
    float t;
    if (s->floor.intersect(ray, t_max, &t)) return false;
  }
  return true;
}

// ---------------------------------------------------------------- integrator.rs
// integrator.rs:35-48
static inline void add_clamped(Spec* l, const Spec& c, bool clamp, float m) {
  if (clamp) {
    float mx = c.max_value();
    if (mx > m)
      *l = *l + c * (m / mx);
    else
      *l = *l + c;
  } else {
    *l = *l + c;
  }
}

struct Guides {
  float albedo[3] = {0, 0, 0};
  float normal[3] = {0, 0, 0};
};

// integrator.rs:50-221
static Spec trace(const oracle_scene* sc, Ray ray, Wavelengths* wl, Sampler* s, const ArgentPathSettings& ps,
                  Guides* guides) {
  Spec l;
  Spec beta(1.0f);
  bool specular = true;
  bool rough_seen = false;
  float prev_pdf = 1.0f;
  int medium = -1;  // material index whose absorption fills the current medium
  const V3 floor_n(0, 1, 0);
  const EnvMap* env_map = sc->env.is_map ? &sc->env.map : nullptr;

  for (uint32_t depth = 0; depth < ps.max_depth; ++depth) {
    bool clamp = rough_seen;
    s->set_dim(8 + depth * 8);
    SceneHit hit = scene_intersect(sc, ray, depth == 0);
    if (medium >= 0 && hit.kind != H_NONE) {
      Spec sig = tab_sample(sc->materials[medium].d.spec_b, *wl);
      Spec e;
      for (int i = 0; i < N; ++i) e.v[i] = -sig.v[i] * hit.t;
      beta = beta * spec_exp(e);
    }
    auto env_weight = [&](V3 dir) -> float {
      if (env_map && !specular) {
        float pl = sc->env_pick * env_map->pdf(dir);
        return prev_pdf * prev_pdf / (prev_pdf * prev_pdf + pl * pl);
      }
      return 1.0f;
    };
    V3 p, p_obj, ng, ns;
    int mat_id;
    float cavity;
    if (hit.kind == H_NONE) {
      add_clamped(&l, beta * sc->env.eval(ray.d, *wl) * env_weight(ray.d), clamp, ps.clamp_indirect);
      break;
    } else if (hit.kind == H_PANEL) {
      const Panel& panel = sc->panels[hit.panel];
      Spec le = panel.le(ray.at(hit.t), ray.d, *wl);
      if (!le.is_black()) {
        if (specular) {
          add_clamped(&l, beta * le, clamp, ps.clamp_indirect);
        } else {
          float cos_l = rmax(std::fabs(dot(-ray.d, panel.n)), 1e-8f);
          float p_light =
              (1.0f - sc->env_pick) * light_pick_pdf(sc, hit.panel) * hit.t * hit.t / (cos_l * panel.area);
          float w = prev_pdf * prev_pdf / (prev_pdf * prev_pdf + p_light * p_light);
          add_clamped(&l, beta * le * w, clamp, ps.clamp_indirect);
        }
      }
      break;
    } else if (hit.kind == H_FLOOR) {
      if (s->next_random() >= sc->floor.presence(hit.p)) {
        add_clamped(&l, beta * sc->env.eval(ray.d, *wl) * env_weight(ray.d), clamp, ps.clamp_indirect);
        break;
      }
      V3 n = ray.d.y < 0.0f ? floor_n : -floor_n;
      p = hit.p;
      p_obj = hit.p;
      ng = n;
      ns = n;
      mat_id = sc->floor.material;
      cavity = 0.0f;
    } else {
      p = hit.p;
      p_obj = hit.p_obj;
      ng = hit.ng;
      ns = hit.ns;
      mat_id = hit.material;
      cavity = hit.cavity;
    }

    const Material& mat = sc->materials[mat_id];
    V3 wo_w = -ray.d;
    bool transmissive = mat.is_transmissive();
    V3 nsu = ns, ngu = ng;
    if (!transmissive && dot(ng, wo_w) < 0.0f) {
      nsu = -ns;
      ngu = -ng;
    }
    if (!transmissive && dot(nsu, wo_w) <= 0.0f) nsu = ngu;
    Frame frame(nsu);
    V3 wo = frame.to_local(wo_w);
    HitCtx ctx{p_obj, nsu, &frame, sc->turntable_deg};
    float ub = s->next();
    Bsdf bsdf = material_bsdf(mat, *wl, cavity, ub, ctx);
    if (depth == 0) {
      guide_rgb(mat, cavity, guides->albedo);
      guides->normal[0] = nsu.x;
      guides->normal[1] = nsu.y;
      guides->normal[2] = nsu.z;
    }

    // Next-event estimation.
    if (!bsdf.is_delta()) {
      float ul = s->next();
      float u1, u2;
      s->next2(&u1, &u2);
      if (env_map && ul < sc->env_pick) {
        float pdf_dir;
        V3 dir = env_map->sample(u1, u2, &pdf_dir);
        if (pdf_dir > 0.0f && dot(dir, ngu) > 0.0f) {
          V3 wi = frame.to_local(dir);
          Spec f = bsdf.eval(wo, wi);
          if (!f.is_black()) {
            float p_light = sc->env_pick * pdf_dir;
            float p_bsdf = bsdf.pdf(wo, wi);
            float w = p_light * p_light / (p_light * p_light + p_bsdf * p_bsdf);
            float vis = sky_visibility(sc, offset_origin(p, ngu, dir), dir);
            if (vis > 0.0f) {
              Spec le = env_map->eval(dir, *wl);
              Spec c = beta * f * le * (std::fabs(wi.z) * w * vis / p_light);
              add_clamped(&l, c, rough_seen, ps.clamp_indirect);
            }
          }
        }
      } else {
        int li;
        float pick;
        float ulp = sc->env_pick > 0.0f ? (ul - sc->env_pick) / (1.0f - sc->env_pick) : ul;
        if (pick_light(sc, ulp, &li, &pick)) {
          pick = pick * (1.0f - sc->env_pick);
          const Panel& panel = sc->panels[li];
          V3 lp = panel.sample_point(u1, u2);
          V3 to = lp - p;
          float d2 = length_squared(to);
          V3 dir = to / std::sqrt(d2);
          float cos_l = dot(-dir, panel.n);
          if (cos_l > 0.0f && dot(dir, ngu) > 0.0f) {
            V3 wi = frame.to_local(dir);
            Spec f = bsdf.eval(wo, wi);
            if (!f.is_black()) {
              float p_light = pick * d2 / (cos_l * panel.area);
              float p_bsdf = bsdf.pdf(wo, wi);
              float w = p_light * p_light / (p_light * p_light + p_bsdf * p_bsdf);
              V3 origin = offset_origin(p, ngu, dir);
              if (visible(sc, origin, lp, li)) {
                Spec le = panel.le(lp, dir, *wl);
                Spec c = beta * f * le * (std::fabs(wi.z) * w / p_light);
                add_clamped(&l, c, rough_seen, ps.clamp_indirect);
              }
            }
          }
        }
      }
    } else {
      s->next();
      float a, b;
      s->next2(&a, &b);
    }

    // Continue the path.
    float u0 = s->next();
    float u1, u2;
    s->next2(&u1, &u2);
    BsdfSample smp;
    if (!bsdf.sample(wo, u0, u1, u2, &smp)) break;
    if (smp.pdf <= 0.0f || smp.f.is_black()) break;
    V3 wi_w = frame.to_world(smp.wi);
    float side = dot(wi_w, ngu) * dot(wo_w, ngu);
    if ((!smp.transmit && side <= 0.0f) || (smp.transmit && side >= 0.0f)) break;
    if (smp.terminate_secondary) terminate_secondary(wl);
    beta = beta * (smp.f * (std::fabs(smp.wi.z) / smp.pdf));
    if (!beta.is_finite()) break;
    specular = smp.delta;
    if (!smp.delta) rough_seen = true;
    prev_pdf = smp.pdf;
    if (smp.transmit) medium = (wo.z > 0.0f && mat.has_medium()) ? mat_id : -1;
    ray = Ray{offset_origin(p, ngu, wi_w), wi_w};

    if (depth >= ps.rr_depth) {
      float survive = rmin(beta.max_value(), 0.95f);
      if (survive <= 0.0f || s->next_random() >= survive) break;
      beta = beta / survive;
    }
  }
  return l;
}

// camera.rs:57-69
static Ray camera_ray(const ArgentCamera& c, float sx, float sy, float lu, float lv) {
  V3 pos(c.pos[0], c.pos[1], c.pos[2]), fwd(c.forward[0], c.forward[1], c.forward[2]),
      right(c.right[0], c.right[1], c.right[2]), up(c.up[0], c.up[1], c.up[2]);
  float x = (sx + c.shift[0]) * c.half_w;
  float y = (sy + c.shift[1]) * c.half_h;
  V3 dir = normalize(fwd + right * x + up * y);
  if (c.lens_radius <= 0.0f) return Ray{pos, dir};
  float ft = c.focus_dist / dot(dir, fwd);
  V3 p_focus = pos + dir * ft;
  float dx, dy;
  disk(lu, lv, &dx, &dy);
  V3 o = pos + right * (dx * c.lens_radius) + up * (dy * c.lens_radius);
  return Ray{o, normalize(p_focus - o)};
}

}  // namespace orc

using namespace orc;

extern "C" {

oracle_scene* oracle_scene_create(const float* positions, uint32_t nv, const float* normals, const uint32_t* tris,
                                  uint32_t nt, const uint16_t* tri_material, const float* cavity,
                                  const ArgentSceneDesc* desc) {
  oracle_scene* s = new oracle_scene();
  s->positions.resize(nv);
  for (uint32_t i = 0; i < nv; ++i) s->positions[i] = V3(positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]);
  if (normals) {
    s->normals.resize(nv);
    for (uint32_t i = 0; i < nv; ++i) s->normals[i] = V3(normals[3 * i], normals[3 * i + 1], normals[3 * i + 2]);
  }
  s->triangles.assign(tris, tris + 3 * (size_t)nt);
  if (tri_material) s->tri_material.assign(tri_material, tri_material + nt);
  if (cavity) {
    s->cavity.assign(cavity, cavity + nv);
    s->has_cavity = true;
  }
  s->bvh = Bvh::build(positions, tris, nt);
  for (int i = 0; i < desc->num_materials; ++i) {
    Material m;
    m.d = desc->materials[i];
    s->materials.push_back(m);
  }
  for (int i = 0; i < desc->num_panels; ++i) {
    const ArgentPanel& d = desc->panels[i];
    Panel p;
    p.center = V3(d.center[0], d.center[1], d.center[2]);
    p.hu = V3(d.hu[0], d.hu[1], d.hu[2]);
    p.hv = V3(d.hv[0], d.hv[1], d.hv[2]);
    V3 c = cross(p.hu, p.hv);  // light.rs:30-33
    p.n = normalize(c);
    p.area = 4.0f * length(c);
    p.emits = d.emits != 0;
    p.camera_visible = d.camera_visible != 0;
    p.feather = d.feather;
    p.emission.assign(d.emission, d.emission + ARGENT_SPEC_LEN);
    s->panels.push_back(p);
  }
  if (desc->env) {
    const ArgentEnv& e = *desc->env;
    if (e.kind == ARGENT_ENV_MAP) {
      s->env.is_map = true;
      s->env.map.load(e.rgb, e.width, e.height, e.rotation_deg);
    } else {
      s->env.power = e.power;
      s->env.top.assign(e.top, e.top + ARGENT_SPEC_LEN);
      s->env.horizon.assign(e.horizon, e.horizon + ARGENT_SPEC_LEN);
      s->env.bottom.assign(e.bottom, e.bottom + ARGENT_SPEC_LEN);
    }
  } else {
    s->env.top.assign(ARGENT_SPEC_LEN, 0.0f);
    s->env.horizon.assign(ARGENT_SPEC_LEN, 0.0f);
    s->env.bottom.assign(ARGENT_SPEC_LEN, 0.0f);
  }
  s->floor.enabled = desc->floor.enabled != 0;
  s->floor.y = desc->floor.y;
  s->floor.material = desc->floor.material;
  s->floor.fade_start = desc->floor.fade_start;
  s->floor.fade_end = desc->floor.fade_end;
  s->turntable_deg = desc->turntable_deg;
  s->has_white = desc->has_white != 0;
  for (int i = 0; i < 3; ++i) s->white[i] = desc->white_xyz[i];
  rebuild_lights(s);
  return s;
}

void oracle_scene_destroy(oracle_scene* s) { delete s; }

void oracle_scene_set_turntable(oracle_scene* s, float deg) { s->turntable_deg = deg; }

// render.rs:67-115 over rows [y0, y1).  color/albedo/normal receive
// argent's film sums (camera RGB) for those rows; xyz (optional, double)
// receives the same samples' XYZ sums.  threads <= 0 uses OpenMP's default.
void oracle_render_pass(const oracle_scene* sc, const ArgentCamera* cam, const ArgentPathSettings* ps, uint32_t w,
                        uint32_t h, uint32_t first, uint32_t count, uint32_t seed, uint32_t y0, uint32_t y1,
                        float* color, float* albedo, float* normal, double* xyz, int threads) {
  float aspect_sx = 2.0f / (float)w;
  float aspect_sy = 2.0f / (float)h;
  uint32_t seed_h = hash32(seed ^ 0xa511e9b3u);
  M3 cam_m;
  camera_matrix(sc->has_white, sc->white, cam_m);
  (void)energy_table();
  (void)LinearRgb::get();
  int nthr = threads > 0 ? threads : omp_get_max_threads();
  // Work is handed out 16 pixels at a time, so a band of a few rows keeps
  // every thread busy (pixels are independent: each writes only its own
  // sums).
  const int64_t npix = (int64_t)(y1 > y0 ? y1 - y0 : 0) * (int64_t)w;
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthr)
  for (int64_t ip = 0; ip < npix; ++ip) {
    uint32_t y = y0 + (uint32_t)(ip / w);
    {
      uint32_t x = (uint32_t)(ip % w);
      uint32_t pix_seed = hash32((y * w + x) ^ seed_h);
      float acc[3] = {0, 0, 0}, aacc[3] = {0, 0, 0}, nacc[3] = {0, 0, 0};
      double xacc[3] = {0, 0, 0};
      for (uint32_t si = first; si < first + count; ++si) {
        Sampler s(pix_seed, si);
        float jx = tent(s.next(), 1.0f);
        float jy = tent(s.next(), 1.0f);
        float lu, lv;
        s.next2(&lu, &lv);
        Wavelengths wl = sample_visible(s.next());
        float sx = (((float)x + 0.5f + jx) * aspect_sx) - 1.0f;
        float sy = 1.0f - (((float)y + 0.5f + jy) * aspect_sy);
        Ray ray = camera_ray(*cam, sx, sy, lu, lv);
        Guides g;
        Spec l = trace(sc, ray, &wl, &s, *ps, &g);
        float xyz_s[3], rgb[3];
        to_xyz(l, wl, xyz_s);
        m3_apply(cam_m, xyz_s, rgb);
        if (std::isfinite(rgb[0]) && std::isfinite(rgb[1]) && std::isfinite(rgb[2])) {
          for (int c = 0; c < 3; ++c) {
            acc[c] += rgb[c];
            xacc[c] += (double)xyz_s[c];
          }
        }
        for (int c = 0; c < 3; ++c) {
          aacc[c] += g.albedo[c];
          nacc[c] += g.normal[c];
        }
      }
      size_t o = 3 * ((size_t)y * w + x);
      for (int c = 0; c < 3; ++c) {
        if (color) color[o + c] += acc[c];
        if (albedo) albedo[o + c] += aacc[c];
        if (normal) normal[o + c] += nacc[c];
        if (xyz) xyz[o + c] += xacc[c];
      }
    }
  }
}

void oracle_camera_matrix(int has_white, const float* white, float* out9) {
  M3 m;
  camera_matrix(has_white != 0, white, m);
  std::memcpy(out9, m, sizeof(m));
}

// Trace one path from an explicit camera sample, for unit checks.
void oracle_trace_sample(const oracle_scene* sc, const ArgentCamera* cam, const ArgentPathSettings* ps, uint32_t w,
                         uint32_t h, uint32_t x, uint32_t y, uint32_t si, uint32_t seed, float* xyz_out) {
  uint32_t seed_h = hash32(seed ^ 0xa511e9b3u);
  uint32_t pix_seed = hash32((y * w + x) ^ seed_h);
  Sampler s(pix_seed, si);
  float jx = tent(s.next(), 1.0f);
  float jy = tent(s.next(), 1.0f);
  float lu, lv;
  s.next2(&lu, &lv);
  Wavelengths wl = sample_visible(s.next());
  float sx = (((float)x + 0.5f + jx) * (2.0f / (float)w)) - 1.0f;
  float sy = 1.0f - (((float)y + 0.5f + jy) * (2.0f / (float)h));
  Ray ray = camera_ray(*cam, sx, sy, lu, lv);
  Guides g;
  Spec l = trace(sc, ray, &wl, &s, *ps, &g);
  to_xyz(l, wl, xyz_out);
}

// ---- primitive checks against argent's unit tests
float oracle_fresnel_dielectric(float c, float eta) { return fresnel_dielectric(c, eta); }
float oracle_fresnel_conductor(float c, float eta, float k) { return fresnel_conductor1(c, eta, k); }
float oracle_ggx_e(float roughness, float cos_o) { return Ggx::from_roughness(roughness).e(cos_o); }
void oracle_ggx_sample_h(float roughness, const float* wo, float u1, float u2, float* h_out) {
  V3 h = Ggx::from_roughness(roughness).sample_h(V3(wo[0], wo[1], wo[2]), u1, u2);
  h_out[0] = h.x;
  h_out[1] = h.y;
  h_out[2] = h.z;
}
void oracle_energy_table(float* out1024) { std::memcpy(out1024, energy_table().e, sizeof(float) * 1024); }
void oracle_sample_visible(float u, float* lambda4, float* pdf4) {
  Wavelengths w = sample_visible(u);
  for (int i = 0; i < 4; ++i) {
    lambda4[i] = w.lambda[i];
    pdf4[i] = w.pdf[i];
  }
}
void oracle_to_xyz(const float* l4, const float* lambda4, const float* pdf4, float* xyz) {
  Spec l(l4[0], l4[1], l4[2], l4[3]);
  Wavelengths w;
  for (int i = 0; i < 4; ++i) {
    w.lambda[i] = lambda4[i];
    w.pdf[i] = pdf4[i];
  }
  to_xyz(l, w, xyz);
}
void oracle_xyz_bar(float lambda, float* out3) { xyz_bar(lambda, out3); }
void oracle_linear_rgb(float* basis3x471, float* inv9) {
  const LinearRgb& L = LinearRgb::get();
  std::memcpy(basis3x471, L.basis, sizeof(L.basis));
  std::memcpy(inv9, L.inv, sizeof(L.inv));
}
uint32_t oracle_hash32(uint32_t x) { return hash32(x); }
// Draw `ndims` successive Sampler::next() values (with set_dim jumps given by
// dims, or sequential when dims is NULL).
void oracle_sampler_next(uint32_t pixel_seed, uint32_t index, uint32_t ndims, float* out) {
  Sampler s(pixel_seed, index);
  for (uint32_t i = 0; i < ndims; ++i) out[i] = s.next();
}
void oracle_sampler_random(uint32_t pixel_seed, uint32_t index, uint32_t n, float* out) {
  Sampler s(pixel_seed, index);
  for (uint32_t i = 0; i < n; ++i) out[i] = s.next_random();
}
void oracle_sobol_4d(uint32_t index, uint32_t set, uint32_t seed, float* out4) { sample_4d(index, set, seed, out4); }
void oracle_sobol_raw(uint32_t index, int dim, uint32_t* out) { *out = sobol_dim(index, dim); }

}  // extern "C"
