// scene_prep.cpp — see scene_prep.h.  Restates the host-side table builds of
// argent-core (scene.rs, envmap.rs, microfacet.rs, color.rs) for the device
// scene; built with -ffp-contract=off so each product/sum rounds like
// argent's f32 code.
#include "scene_prep.h"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "../data/spectral_tables.h"

namespace argent {
namespace {

const float CIE_Y_INTEGRAL = 106.85692f;  // cie.rs:29

void xyz_bar(float lambda, float out[3]) {
  float x = lambda - 360.0f;
  if (!(x >= 0.0f && x <= 470.0f)) {
    out[0] = out[1] = out[2] = 0.0f;
    return;
  }
  size_t i = std::min((size_t)x, (size_t)469);
  float t = x - (float)i;
  const float* a = &ARGENT_CMF_1931_2DEG[3 * i];
  const float* b = &ARGENT_CMF_1931_2DEG[3 * (i + 1)];
  for (int k = 0; k < 3; ++k) out[k] = a[k] + (b[k] - a[k]) * t;
}

float tab_eval(const float* values, float l) {
  float x = l - 360.0f;
  if (x < 0.0f) x = 0.0f;
  if (x > 470.0f) x = 470.0f;
  int i = std::min((int)x, 469);
  float f = x - (float)i;
  return values[i] * (1.0f - f) + values[i + 1] * f;
}

double planck(float lambda_nm, float t) {
  if (t <= 0.0f) return 0.0;
  double c = 299792458.0, h = 6.62606957e-34, kb = 1.3806488e-23;
  double l = (double)lambda_nm * 1e-9;
  return (2.0 * h * c * c) / (std::pow(l, 5) * (std::exp((h * c) / (l * kb * (double)t)) - 1.0));
}

float smoothstep_e(float e0, float e1, float x) {
  float t = (x - e0) / (e1 - e0);
  if (t < 0.0f) t = 0.0f;
  if (t > 1.0f) t = 1.0f;
  return t * t * (3.0f - 2.0f * t);
}

struct V {
  float x, y, z;
};
V vsub(V a, V b) { return V{a.x - b.x, a.y - b.y, a.z - b.z}; }
V vadd(V a, V b) { return V{a.x + b.x, a.y + b.y, a.z + b.z}; }
V vmul(V a, float s) { return V{a.x * s, a.y * s, a.z * s}; }
float vdot(V a, V b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
V vcross(V a, V b) { return V{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
V vnorm(V a) { return vmul(a, 1.0f / std::sqrt(vdot(a, a))); }

// microfacet.rs:71-85
V ggx_sample_h(float a, V wo, float u1, float u2) {
  V vh = vnorm(V{a * wo.x, a * wo.y, wo.z});
  float lensq = vh.x * vh.x + vh.y * vh.y;
  V t1 = lensq > 1e-12f ? vmul(V{-vh.y, vh.x, 0.0f}, 1.0f) : V{1, 0, 0};
  if (lensq > 1e-12f) {
    float s = std::sqrt(lensq);
    t1 = V{-vh.y / s, vh.x / s, 0.0f / s};
  }
  V t2 = vcross(vh, t1);
  float r = std::sqrt(u1);
  float phi = 2.0f * 3.14159265358979323846f * u2;
  float p1 = r * std::cos(phi);
  float p2 = r * std::sin(phi);
  float s = 0.5f * (1.0f + vh.z);
  p2 = (1.0f - s) * std::sqrt(std::fmax(1.0f - p1 * p1, 0.0f)) + s * p2;
  V nh = vadd(vadd(vmul(t1, p1), vmul(t2, p2)), vmul(vh, std::sqrt(std::fmax(1.0f - p1 * p1 - p2 * p2, 0.0f))));
  return vnorm(V{a * nh.x, a * nh.y, std::fmax(nh.z, 1e-6f)});
}
float ggx_lambda(float a, V w) {
  float c2 = w.z * w.z;
  float t2 = std::fmax(1.0f - c2, 0.0f) / std::fmax(c2, 1e-12f);
  if (!std::isfinite(t2)) return 0.0f;
  return 0.5f * (-1.0f + std::sqrt(1.0f + a * a * t2));
}

}  // namespace

float luminance_y_table(const float* t) {
  double y = 0.0;
  for (int i = 0; i <= 470; ++i) {
    float c[3];
    xyz_bar(360.0f + (float)i, c);
    y += (double)tab_eval(t, 360.0f + (float)i) * (double)c[1];
  }
  return (float)(y / (double)CIE_Y_INTEGRAL);
}

void panel_frame(const ArgentPanel& p, float n[3], float* area, float* hu_l2, float* hv_l2) {
  V hu{p.hu[0], p.hu[1], p.hu[2]}, hv{p.hv[0], p.hv[1], p.hv[2]};
  V c = vcross(hu, hv);
  V nn = vnorm(c);
  n[0] = nn.x;
  n[1] = nn.y;
  n[2] = nn.z;
  *area = 4.0f * std::sqrt(vdot(c, c));
  *hu_l2 = vdot(hu, hu);
  *hv_l2 = vdot(hv, hv);
}

LightTable build_lights(const ArgentSceneDesc& desc) {
  LightTable t;
  float acc = 0.0f;
  for (int i = 0; i < desc.num_panels; ++i) {
    const ArgentPanel& p = desc.panels[i];
    if (!p.emits) continue;
    float n[3], area, a2, b2;
    panel_frame(p, n, &area, &a2, &b2);
    float power = area * std::fmax(luminance_y_table(p.emission), 1e-6f);
    acc += power;
    t.lights.push_back(i);
    t.cdf.push_back(acc);
  }
  if (acc > 0.0f)
    for (auto& c : t.cdf) c /= acc;
  bool is_map = desc.env && desc.env->kind == ARGENT_ENV_MAP;
  t.env_pick = is_map ? (t.lights.empty() ? 1.0f : 0.5f) : 0.0f;
  return t;
}

void linear_rgb(float basis[3][471], float inv[3][3]) {
  float kelvin = 6504.0f;
  float peak = 2.897772e-3f / kelvin * 1e9f;
  float norm = 1.0f / (float)planck(peak, kelvin);
  for (int i = 0; i < 471; ++i) {
    float l = 360.0f + (float)i;
    float wb = 1.0f - smoothstep_e(470.0f, 515.0f, l);
    float wr = smoothstep_e(565.0f, 610.0f, l);
    float wg = std::fmax(1.0f - wb - wr, 0.0f);
    float e = (float)planck(l, kelvin) * norm;
    basis[0][i] = wr * e;
    basis[1][i] = wg * e;
    basis[2][i] = wb * e;
  }
  float m[3][3];
  for (int j = 0; j < 3; ++j) {
    float xyz[3] = {0, 0, 0};
    for (int i = 0; i < 471; ++i) {
      float c[3];
      xyz_bar(360.0f + (float)i, c);
      for (int k = 0; k < 3; ++k) xyz[k] += c[k] * basis[j][i];
    }
    float s[3] = {xyz[0] / CIE_Y_INTEGRAL, xyz[1] / CIE_Y_INTEGRAL, xyz[2] / CIE_Y_INTEGRAL};
    float rgb[3] = {3.2404542f * s[0] - 1.5371385f * s[1] - 0.4985314f * s[2],
                    -0.969266f * s[0] + 1.8760108f * s[1] + 0.041556f * s[2],
                    0.0556434f * s[0] - 0.2040259f * s[1] + 1.0572252f * s[2]};
    for (int i = 0; i < 3; ++i) m[i][j] = rgb[i];
  }
  float a = m[0][0], b = m[0][1], c = m[0][2], d = m[1][0], e = m[1][1], f = m[1][2], g = m[2][0], h = m[2][1],
        ii = m[2][2];
  float det = a * (e * ii - f * h) - b * (d * ii - f * g) + c * (d * h - e * g);
  float k = 1.0f / det;
  float r[3][3] = {{(e * ii - f * h) * k, (c * h - b * ii) * k, (b * f - c * e) * k},
                   {(f * g - d * ii) * k, (a * ii - c * g) * k, (c * d - a * f) * k},
                   {(d * h - e * g) * k, (b * g - a * h) * k, (a * e - b * d) * k}};
  std::memcpy(inv, r, sizeof(r));
}

EnvTables build_env(const float* rgb, int w, int h) {
  EnvTables t;
  t.width = w;
  t.height = h;
  float basis[3][471], inv[3][3];
  linear_rgb(basis, inv);
  t.weights.resize((size_t)w * h * 3);
  for (size_t i = 0; i < (size_t)w * h; ++i) {
    const float* c = &rgb[3 * i];
    for (int k = 0; k < 3; ++k) t.weights[3 * i + k] = inv[k][0] * c[0] + inv[k][1] * c[1] + inv[k][2] * c[2];
  }
  t.conditional.assign((size_t)(w + 1) * h, 0.0f);
  std::vector<float> row_sum(h);
  for (int y = 0; y < h; ++y) {
    float s = std::sin(3.14159265358979323846f * ((float)y + 0.5f) / (float)h);
    size_t base = (size_t)y * (w + 1);
    float acc = 0.0f;
    for (int x = 0; x < w; ++x) {
      const float* c = &rgb[3 * ((size_t)y * w + x)];
      acc += std::fmax(0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2], 0.0f) * s + 1e-6f;
      t.conditional[base + x + 1] = acc;
    }
    row_sum[y] = acc;
    for (int x = 0; x <= w; ++x) t.conditional[base + x] /= acc;
  }
  t.marginal.assign(h + 1, 0.0f);
  float acc = 0.0f;
  for (int y = 0; y < h; ++y) {
    acc += row_sum[y];
    t.marginal[y + 1] = acc;
  }
  t.total = acc / ((float)w * (float)h);
  for (auto& v : t.marginal) v /= acc;
  return t;
}

void ggx_energy_table(float out[32 * 32]) {
  const int EN = 32;
  for (int j = 0; j < EN; ++j) {
    float r = (float)j / (float)(EN - 1);
    float a = std::fmax(r * r, 1e-4f);
    for (int i = 0; i < EN; ++i) {
      float mu = std::fmax((float)i / (float)(EN - 1), 1e-3f);
      V wo{std::sqrt(1.0f - mu * mu), 0.0f, mu};
      const int n = 24;
      float sum = 0.0f;
      float g1 = 1.0f / (1.0f + ggx_lambda(a, wo));
      for (int p = 0; p < n; ++p)
        for (int q = 0; q < n; ++q) {
          float u1 = ((float)p + 0.5f) / (float)n;
          float u2 = ((float)q + 0.5f) / (float)n;
          V hh = ggx_sample_h(a, wo, u1, u2);
          // reflect(wo, h) = -wo + h * (2 (wo.h))
          float k = 2.0f * vdot(wo, hh);
          V wi = vadd(V{-wo.x, -wo.y, -wo.z}, vmul(hh, k));
          if (wi.z > 0.0f) {
            float g2 = 1.0f / (1.0f + ggx_lambda(a, wo) + ggx_lambda(a, wi));
            sum += g2 / g1;
          }
        }
      out[j * EN + i] = sum / (float)(n * n);
    }
  }
}

void camera_matrix(bool has_white, const float w[3], float out[9]) {
  static const float BR[3][3] = {{0.8951f, 0.2664f, -0.1614f}, {-0.7502f, 1.7135f, 0.0367f}, {0.0389f, -0.0685f, 1.0296f}};
  static const float BRI[3][3] = {
      {0.986993f, -0.147054f, 0.159963f}, {0.432305f, 0.51836f, 0.049291f}, {-0.008529f, 0.040043f, 0.968487f}};
  static const float XS[3][3] = {
      {3.2404542f, -1.5371385f, -0.4985314f}, {-0.969266f, 1.8760108f, 0.041556f}, {0.0556434f, -0.2040259f, 1.0572252f}};
  static const float D65W[3] = {0.95047f, 1.0f, 1.08883f};
  if (!has_white) {
    std::memcpy(out, XS, sizeof(XS));
    return;
  }
  auto apply = [](const float m[3][3], const float v[3], float o[3]) {
    for (int i = 0; i < 3; ++i) o[i] = m[i][0] * v[0] + m[i][1] * v[1] + m[i][2] * v[2];
  };
  auto mul = [](const float a[3][3], const float b[3][3], float r[3][3]) {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        float s = 0.0f;
        for (int k = 0; k < 3; ++k) s += a[i][k] * b[k][j];
        r[i][j] = s;
      }
  };
  float src[3], dst[3];
  apply(BR, w, src);
  apply(BR, D65W, dst);
  float d[3][3] = {{dst[0] / src[0], 0, 0}, {0, dst[1] / src[1], 0}, {0, 0, dst[2] / src[2]}};
  float t[3][3], cat[3][3], r[3][3];
  mul(d, BR, t);
  mul(BRI, t, cat);
  mul(XS, cat, r);
  std::memcpy(out, r, sizeof(r));
}

void sobol_directions(uint32_t out[4][32]) {
  for (int j = 0; j < 32; ++j) out[0][j] = 1u << (31 - j);
  // (degree, coefficient bits, initial m) of x+1, x^2+x+1, x^3+x+1.
  const int deg[4] = {0, 1, 2, 3};
  const uint32_t coef[4] = {0, 0, 1, 1};
  const uint32_t m0[4][3] = {{0, 0, 0}, {1, 0, 0}, {1, 3, 0}, {1, 3, 1}};
  for (int d = 1; d < 4; ++d) {
    int s = deg[d];
    uint32_t m[32];
    for (int k = 0; k < s; ++k) m[k] = m0[d][k];
    for (int k = s; k < 32; ++k) {
      uint32_t r = m[k - s] ^ (m[k - s] << s);
      for (int i = 1; i < s; ++i)
        if ((coef[d] >> (s - 1 - i)) & 1u) r ^= m[k - i] << i;
      m[k] = r;
    }
    for (int j = 0; j < 32; ++j) out[d][j] = m[j] << (31 - j);
  }
}

}  // namespace argent
