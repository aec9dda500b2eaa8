// spectral.cuh — hero-wavelength spectra on the device: `Spec`,
// `Wavelengths`, table lookups, Fresnel, GGX and the CIE projection
// (argent-spectra spec.rs, fresnel.rs, cie.rs; argent-core tab.rs,
// microfacet.rs).
#pragma once
#include "dev_math.cuh"
#include "tables.cuh"

namespace dev {

#define ARGENT_NW 4  // wavelengths per path (spec.rs:6)

// spec.rs:13-76
struct Spec {
  float v[4];
};
__device__ __forceinline__ Spec spec(float s) { return Spec{{s, s, s, s}}; }
__device__ __forceinline__ Spec spec4(float4 a) { return Spec{{a.x, a.y, a.z, a.w}}; }
__device__ __forceinline__ float4 to_f4(const Spec& s) { return make_float4(s.v[0], s.v[1], s.v[2], s.v[3]); }
__device__ __forceinline__ Spec operator+(const Spec& a, const Spec& b) {
  return Spec{{a.v[0] + b.v[0], a.v[1] + b.v[1], a.v[2] + b.v[2], a.v[3] + b.v[3]}};
}
__device__ __forceinline__ Spec operator*(const Spec& a, const Spec& b) {
  return Spec{{a.v[0] * b.v[0], a.v[1] * b.v[1], a.v[2] * b.v[2], a.v[3] * b.v[3]}};
}
__device__ __forceinline__ Spec operator*(const Spec& a, float s) {
  return Spec{{a.v[0] * s, a.v[1] * s, a.v[2] * s, a.v[3] * s}};
}
__device__ __forceinline__ Spec operator/(const Spec& a, float s) {
  return Spec{{a.v[0] / s, a.v[1] / s, a.v[2] / s, a.v[3] / s}};
}
__device__ __forceinline__ float max_value(const Spec& a) {
  float m = -3.40282347e38f;
#pragma unroll
  for (int i = 0; i < 4; ++i) m = fmaxf(m, a.v[i]);
  return m;
}
__device__ __forceinline__ float min_value(const Spec& a) {
  float m = 3.40282347e38f;
#pragma unroll
  for (int i = 0; i < 4; ++i) m = fminf(m, a.v[i]);
  return m;
}
__device__ __forceinline__ float average(const Spec& a) { return (((0.0f + a.v[0]) + a.v[1]) + a.v[2] + a.v[3]) / 4.0f; }
__device__ __forceinline__ bool is_black(const Spec& a) {
  return a.v[0] == 0.0f && a.v[1] == 0.0f && a.v[2] == 0.0f && a.v[3] == 0.0f;
}
__device__ __forceinline__ bool is_finite(const Spec& a) {
  return isfinite(a.v[0]) && isfinite(a.v[1]) && isfinite(a.v[2]) && isfinite(a.v[3]);
}
__device__ __forceinline__ Spec lerp(float t, const Spec& a, const Spec& b) { return a * (1.0f - t) + b * t; }

struct Wavelengths {
  float lambda[4];
  float pdf[4];
};

// spec.rs:209-220
__device__ __forceinline__ float sample_visible_wavelength(float u) {
  return 538.0f - 138.88889f * atanhf(0.8569106f - 1.827502f * u);
}
__device__ __forceinline__ float visible_wavelength_pdf(float lambda) {
  if (!(lambda >= 360.0f && lambda <= 830.0f)) return 0.0f;
  float c = coshf(0.0072f * (lambda - 538.0f));
  return 0.0039398042f / (c * c);
}
// spec.rs:157-169
__device__ __forceinline__ Wavelengths sample_visible(float u) {
  Wavelengths w;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    float up = u + (float)i / 4.0f;
    if (up > 1.0f) up -= 1.0f;
    w.lambda[i] = sample_visible_wavelength(up);
    w.pdf[i] = visible_wavelength_pdf(w.lambda[i]);
  }
  return w;
}
// spec.rs:187-199
__device__ __forceinline__ void terminate_secondary(Wavelengths* w) {
  if (w->pdf[1] == 0.0f && w->pdf[2] == 0.0f && w->pdf[3] == 0.0f) return;
  w->pdf[1] = w->pdf[2] = w->pdf[3] = 0.0f;
  w->pdf[0] /= 4.0f;
}

// A 1 nm table over 360..=830 nm (tab.rs:20-27).
__device__ __forceinline__ float tab_eval(const float* __restrict__ values, float l) {
  float x = rclamp(l - 360.0f, 0.0f, 470.0f);
  int i = (int)x;
  i = i > 469 ? 469 : i;
  float f = x - (float)i;
  return __ldg(values + i) * (1.0f - f) + __ldg(values + i + 1) * f;
}
__device__ __forceinline__ Spec tab_sample(const float* __restrict__ values, const Wavelengths& wl) {
  Spec r;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.v[i] = tab_eval(values, wl.lambda[i]);
  return r;
}
// `Piecewise::eval` on the uniform 5 nm grid (spectrum.rs:80-93): the
// index is the last grid wavelength <= l, found directly instead of by
// binary search (same index, same interpolation).
__device__ __forceinline__ float grid_eval(const float* __restrict__ values, float l) {
  if (l <= 360.0f) return __ldg(values);
  if (l >= 830.0f) return __ldg(values + 94);
  int i = (int)((l - 360.0f) / 5.0f);
  i = i < 0 ? 0 : (i > 93 ? 93 : i);
  if (360.0f + 5.0f * (float)(i + 1) <= l) ++i;
  if (360.0f + 5.0f * (float)i > l) --i;
  float li = 360.0f + 5.0f * (float)i;
  float li1 = 360.0f + 5.0f * (float)(i + 1);
  float t = (l - li) / (li1 - li);
  return __ldg(values + i) * (1.0f - t) + __ldg(values + i + 1) * t;
}

// fresnel.rs:11-27
__device__ __forceinline__ float fresnel_dielectric(float cos_theta_i, float eta) {
  float cos_i = rclamp(cos_theta_i, -1.0f, 1.0f);
  if (cos_i < 0.0f) {
    eta = 1.0f / eta;
    cos_i = -cos_i;
  }
  float sin2_i = 1.0f - cos_i * cos_i;
  float sin2_t = sin2_i / (eta * eta);
  if (sin2_t >= 1.0f) return 1.0f;
  float cos_t = sqrtf(fmaxf(1.0f - sin2_t, 0.0f));
  float r_parl = (eta * cos_i - cos_t) / (eta * cos_i + cos_t);
  float r_perp = (cos_i - eta * cos_t) / (cos_i + eta * cos_t);
  return 0.5f * (r_parl * r_parl + r_perp * r_perp);
}

// fresnel.rs:81-93: exact unpolarised conductor Fresnel, complex f32.
__device__ __forceinline__ float fresnel_conductor1(float cos_theta_i, float eta, float k) {
  float cos_i = rclamp(cos_theta_i, 0.0f, 1.0f);
  float sin2_i = 1.0f - cos_i * cos_i;
  // e*e
  float ee_re = eta * eta - k * k, ee_im = eta * k + k * eta;
  // sin2_t = (sin2_i + 0i) / e^2
  float dd = ee_re * ee_re + ee_im * ee_im;
  float st_re = (sin2_i * ee_re + 0.0f * ee_im) / dd;
  float st_im = (0.0f * ee_re - sin2_i * ee_im) / dd;
  // cos_t = sqrt(1 - sin2_t)
  float a_re = 1.0f - st_re, a_im = 0.0f - st_im;
  float ct_re, ct_im;
  {
    float n = sqrtf(a_re * a_re + a_im * a_im);
    if (n == 0.0f) {
      ct_re = 0.0f;
      ct_im = 0.0f;
    } else {
      float t1 = sqrtf(0.5f * (n + fabsf(a_re)));
      float t2 = 0.5f * a_im / t1;
      if (a_re >= 0.0f) {
        ct_re = t1;
        ct_im = t2;
      } else {
        ct_re = fabsf(t2);
        ct_im = copysignf(t1, a_im);
      }
    }
  }
  // r_parl = (e*cos_i - cos_t) / (e*cos_i + cos_t)
  float ec_re = eta * cos_i, ec_im = k * cos_i;
  float n1_re = ec_re - ct_re, n1_im = ec_im - ct_im;
  float d1_re = ec_re + ct_re, d1_im = ec_im + ct_im;
  float dd1 = d1_re * d1_re + d1_im * d1_im;
  float rp_re = (n1_re * d1_re + n1_im * d1_im) / dd1;
  float rp_im = (n1_im * d1_re - n1_re * d1_im) / dd1;
  // r_perp = (cos_i - e*cos_t) / (cos_i + e*cos_t)
  float ect_re = eta * ct_re - k * ct_im, ect_im = eta * ct_im + k * ct_re;
  float n2_re = cos_i - ect_re, n2_im = 0.0f - ect_im;
  float d2_re = cos_i + ect_re, d2_im = 0.0f + ect_im;
  float dd2 = d2_re * d2_re + d2_im * d2_im;
  float rs_re = (n2_re * d2_re + n2_im * d2_im) / dd2;
  float rs_im = (n2_im * d2_re - n2_re * d2_im) / dd2;
  return 0.5f * ((rp_re * rp_re + rp_im * rp_im) + (rs_re * rs_re + rs_im * rs_im));
}
__device__ __forceinline__ Spec fresnel_conductor(float c, const Spec& eta, const Spec& k) {
  Spec r;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.v[i] = fresnel_conductor1(c, eta.v[i], k.v[i]);
  return r;
}

// microfacet.rs: GGX with VNDF sampling and the energy table.

struct Ggx {
  float alpha;
};
__device__ __forceinline__ Ggx ggx_from_roughness(float r) {
  float rr = rclamp(r, 0.0f, 1.0f);
  return Ggx{fmaxf(rr * rr, 1e-4f)};
}
__device__ __forceinline__ bool is_smooth(Ggx g) { return g.alpha < 1.5e-3f; }
__device__ __forceinline__ float tan2(V3 w) {
  float c2 = w.z * w.z;
  return fmaxf(1.0f - c2, 0.0f) / fmaxf(c2, 1e-12f);
}
__device__ __forceinline__ float ggx_d(Ggx g, V3 h) {
  if (h.z <= 0.0f) return 0.0f;
  float a2 = g.alpha * g.alpha;
  float c2 = h.z * h.z;
  float k = c2 * (a2 - 1.0f) + 1.0f;
  return a2 / (ARGENT_PI_F * k * k);
}
__device__ __forceinline__ float ggx_lambda(Ggx g, V3 w) {
  float t2 = tan2(w);
  if (!isfinite(t2)) return 0.0f;
  return 0.5f * (-1.0f + sqrtf(1.0f + g.alpha * g.alpha * t2));
}
__device__ __forceinline__ float ggx_g1(Ggx g, V3 w) { return 1.0f / (1.0f + ggx_lambda(g, w)); }
__device__ __forceinline__ float ggx_g2(Ggx g, V3 wo, V3 wi) {
  return 1.0f / (1.0f + ggx_lambda(g, wo) + ggx_lambda(g, wi));
}
__device__ __forceinline__ float ggx_d_visible(Ggx g, V3 wo, V3 h) {
  float c = fmaxf(fabsf(wo.z), 1e-8f);
  return ggx_g1(g, wo) * fmaxf(dot(wo, h), 0.0f) * ggx_d(g, h) / c;
}
__device__ __forceinline__ V3 ggx_sample_h(Ggx g, V3 wo, float u1, float u2) {
  float a = g.alpha;
  V3 vh = normalize(V3{a * wo.x, a * wo.y, wo.z});
  float lensq = vh.x * vh.x + vh.y * vh.y;
  V3 t1 = lensq > 1e-12f ? V3{-vh.y, vh.x, 0.0f} / sqrtf(lensq) : V3{1.0f, 0.0f, 0.0f};
  V3 t2 = cross(vh, t1);
  float r = sqrtf(u1);
  float phi = 2.0f * ARGENT_PI_F * u2;
  float sp, cp;
  sincosf(phi, &sp, &cp);
  float p1 = r * cp;
  float p2 = r * sp;
  float s = 0.5f * (1.0f + vh.z);
  p2 = (1.0f - s) * sqrtf(fmaxf(1.0f - p1 * p1, 0.0f)) + s * p2;
  V3 nh = t1 * p1 + t2 * p2 + vh * sqrtf(fmaxf(1.0f - p1 * p1 - p2 * p2, 0.0f));
  return normalize(V3{a * nh.x, a * nh.y, fmaxf(nh.z, 1e-6f)});
}
// microfacet.rs:100-109
__device__ __forceinline__ float ggx_e(Ggx g, float mu) {
  const int EN = 32;
  float x = fminf(rclamp(mu, 0.0f, 1.0f) * (float)(EN - 1), (float)(EN - 1) - 1e-4f);
  float y = fminf(rclamp(sqrtf(g.alpha), 0.0f, 1.0f) * (float)(EN - 1), (float)(EN - 1) - 1e-4f);
  int xi = (int)x, yi = (int)y;
  float fx = x - (float)xi, fy = y - (float)yi;
  float g00 = d_energy_table[yi * EN + xi], g10 = d_energy_table[yi * EN + xi + 1];
  float g01 = d_energy_table[(yi + 1) * EN + xi], g11 = d_energy_table[(yi + 1) * EN + xi + 1];
  float a = g00 * (1.0f - fx) + g10 * fx;
  float b = g01 * (1.0f - fx) + g11 * fx;
  return rclamp(a * (1.0f - fy) + b * fy, 0.05f, 1.0f);
}

// cie.rs:38-70
#define ARGENT_CIE_Y_INTEGRAL 106.85692f

__device__ __forceinline__ void xyz_bar(float lambda, float out[3]) {
  float x = lambda - 360.0f;
  if (!(x >= 0.0f && x <= 470.0f)) {
    out[0] = out[1] = out[2] = 0.0f;
    return;
  }
  int i = (int)x;
  i = i > 469 ? 469 : i;
  float t = x - (float)i;
  const float* a = d_cmf + 3 * i;
  const float* b = a + 3;
  out[0] = a[0] + (b[0] - a[0]) * t;
  out[1] = a[1] + (b[1] - a[1]) * t;
  out[2] = a[2] + (b[2] - a[2]) * t;
}
__device__ __forceinline__ void to_xyz(const Spec& l, const Wavelengths& wl, float xyz[3]) {
  xyz[0] = xyz[1] = xyz[2] = 0.0f;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    float p = wl.pdf[i];
    if (p == 0.0f || l.v[i] == 0.0f) continue;
    float c[3];
    xyz_bar(wl.lambda[i], c);
    float w = l.v[i] / p;
    xyz[0] += c[0] * w;
    xyz[1] += c[1] * w;
    xyz[2] += c[2] * w;
  }
  float s = 1.0f / (4.0f * ARGENT_CIE_Y_INTEGRAL);
  xyz[0] *= s;
  xyz[1] *= s;
  xyz[2] *= s;
}

}  // namespace dev
