// oracle_denoise.cpp — TEST INFRASTRUCTURE ONLY (the checker for the device
// denoiser; nothing in the product links it).  A plain restatement of
// argent's built-in à-trous denoiser, crates/argent-post/src/denoise.rs:535-712.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "oracle_api.h"

namespace {

const int PASSES = 5;
const float SIGMA_LUM = 4.0f;
const float INV_SIGMA_ALBEDO2 = 1.0f / 0.01f;
const float DEMOD_FLOOR = 0.02f;
const float B3[5] = {1.0f / 16.0f, 1.0f / 4.0f, 3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};

float lum(const float* p) { return 0.2126f * p[0] + 0.7152f * p[1] + 0.0722f * p[2]; }
float clean_radiance(float v) { return std::isfinite(v) ? std::max(v, 0.0f) : 0.0f; }
float clean_unit(float v, float lo) { return std::isfinite(v) ? std::min(std::max(v, lo), 1.0f) : 0.0f; }

// denoise.rs:547-578
std::vector<float> blur_sep(const std::vector<float>& src, int w, int h, const std::vector<float>& k) {
  int r = (int)k.size() / 2;
  std::vector<float> tmp((size_t)w * h), out((size_t)w * h);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      float acc = 0.0f, ws = 0.0f;
      for (int i = 0; i < (int)k.size(); ++i) {
        int xx = x + i - r;
        if (xx >= 0 && xx < w) {
          acc += k[i] * src[(size_t)y * w + xx];
          ws += k[i];
        }
      }
      tmp[(size_t)y * w + x] = acc / ws;
    }
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      float acc = 0.0f, ws = 0.0f;
      for (int i = 0; i < (int)k.size(); ++i) {
        int yy = y + i - r;
        if (yy >= 0 && yy < h) {
          acc += k[i] * tmp[(size_t)yy * w + x];
          ws += k[i];
        }
      }
      out[(size_t)y * w + x] = acc / ws;
    }
  return out;
}

float powi128(float d) {
  float r = 1.0f, a = d;
  for (int b = 128; b; b >>= 1) {
    if (b & 1) r *= a;
    a *= a;
  }
  return r;
}

}  // namespace

extern "C" {

void oracle_atrous(uint32_t wu, uint32_t hu, const float* color, const float* albedo, const float* normal,
                   float* out) {
  int w = (int)wu, h = (int)hu;
  size_t np = (size_t)w * h;
  if (np == 0) return;
  if (normal && !albedo) normal = nullptr;
  std::vector<float> demod, ga, gn;
  if (albedo) {
    demod.resize(3 * np);
    ga.resize(3 * np);
    for (size_t i = 0; i < 3 * np; ++i) {
      ga[i] = clean_unit(albedo[i], 0.0f);
      demod[i] = std::max(clean_unit(albedo[i], 0.0f), DEMOD_FLOOR);
    }
  }
  if (normal) {
    gn.resize(3 * np);
    for (size_t p = 0; p < np; ++p) {
      float v[3];
      for (int c = 0; c < 3; ++c) v[c] = std::isfinite(normal[3 * p + c]) ? normal[3 * p + c] : 0.0f;
      float len = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      for (int c = 0; c < 3; ++c) gn[3 * p + c] = len > 1e-6f ? v[c] / len : 0.0f;
    }
  }
  std::vector<float> sig(3 * np);
  for (size_t i = 0; i < 3 * np; ++i) sig[i] = albedo ? clean_radiance(color[i]) / demod[i] : clean_radiance(color[i]);
  std::vector<float> l(np);
  for (size_t p = 0; p < np; ++p) l[p] = lum(&sig[3 * p]);
  // noise_variance, denoise.rs:582-586
  std::vector<float> mean = blur_sep(l, w, h, {1.0f, 1.0f, 1.0f});
  std::vector<float> resid(np);
  for (size_t p = 0; p < np; ++p) resid[p] = 1.125f * (l[p] - mean[p]) * (l[p] - mean[p]);
  std::vector<float> var = blur_sep(resid, w, h, {1.0f, 1.0f, 1.0f, 1.0f, 1.0f});
  for (int pass = 0; pass < PASSES; ++pass) {
    std::vector<float> var_blur = blur_sep(var, w, h, {0.25f, 0.5f, 0.25f});
    int step = 1 << pass;
    std::vector<float> nsig(3 * np), nvar(np);
    for (int y = 0; y < h; ++y)
      for (int x = 0; x < w; ++x) {
        size_t p = (size_t)y * w + x;
        float lp = l[p];
        float inv_sl = 1.0f / (SIGMA_LUM * std::sqrt(std::max(var_blur[p], 0.0f)) + 1e-10f);
        const float* ap = albedo ? &ga[3 * p] : nullptr;
        const float* npn = normal ? &gn[3 * p] : nullptr;
        float acc[3] = {0, 0, 0}, ws = 0.0f, wv = 0.0f;
        for (int ky = 0; ky < 5; ++ky) {
          int qy = y + (ky - 2) * step;
          if (qy < 0 || qy >= h) continue;
          for (int kx = 0; kx < 5; ++kx) {
            int qx = x + (kx - 2) * step;
            if (qx < 0 || qx >= w) continue;
            size_t q = (size_t)qy * w + qx;
            float e = std::fabs(l[q] - lp) * inv_sl;
            if (ap) {
              const float* aq = &ga[3 * q];
              float d0 = ap[0] - aq[0], d1 = ap[1] - aq[1], d2 = ap[2] - aq[2];
              e += (d0 * d0 + d1 * d1 + d2 * d2) * INV_SIGMA_ALBEDO2;
            }
            float wgt = B3[kx] * B3[ky] * std::exp(-e);
            if (npn) {
              const float* nq = &gn[3 * q];
              bool pz = npn[0] == 0.0f && npn[1] == 0.0f && npn[2] == 0.0f;
              bool qz = nq[0] == 0.0f && nq[1] == 0.0f && nq[2] == 0.0f;
              if (!pz && !qz) wgt *= powi128(std::max(npn[0] * nq[0] + npn[1] * nq[1] + npn[2] * nq[2], 0.0f));
            }
            for (int c = 0; c < 3; ++c) acc[c] += wgt * sig[3 * q + c];
            ws += wgt;
            wv += wgt * wgt * var[q];
          }
        }
        for (int c = 0; c < 3; ++c) nsig[3 * p + c] = acc[c] / ws;
        nvar[p] = wv / (ws * ws);
      }
    sig.swap(nsig);
    var.swap(nvar);
    for (size_t p = 0; p < np; ++p) l[p] = lum(&sig[3 * p]);
  }
  for (size_t i = 0; i < 3 * np; ++i) out[i] = albedo ? sig[i] * demod[i] : sig[i];
}

}  // extern "C"
