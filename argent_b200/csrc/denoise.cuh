// denoise.cuh — argent's built-in à-trous denoiser on the device
// (crates/argent-post/src/denoise.rs:535-700): an edge-avoiding à-trous
// wavelet filter (Dammertz et al. 2010) with SVGF-style luminance edge
// stopping (Schied et al. 2017), 5 passes of the 5x5 B3-spline kernel with
// holes 1, 2, 4, 8, 16, albedo demodulation, normal and albedo weights.
//
// Every per-pixel sum runs in argent's order (kernel taps in index order,
// borders renormalised) and the library has no FMA contraction, so the
// result differs from argent's only through expf (CUDA against the host's).
// One image: all buffers are w*h, row-major; colours are 3 floats per pixel.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace dn {

#define DN_PASSES 5
#define DN_SIGMA_LUM 4.0f
#define DN_INV_SIGMA_ALBEDO2 100.0f  // 1 / 0.01
#define DN_DEMOD_FLOOR 0.02f

__device__ __forceinline__ float clean_radiance(float v) { return isfinite(v) ? fmaxf(v, 0.0f) : 0.0f; }
__device__ __forceinline__ float clean_unit(float v, float lo) {
  return isfinite(v) ? fminf(fmaxf(v, lo), 1.0f) : 0.0f;
}
__device__ __forceinline__ float lum(float r, float g, float b) { return 0.2126f * r + 0.7152f * g + 0.0722f * b; }

// denoise.rs:675-704: guides, demodulated signal and its luminance.
__global__ void k_dn_prep(const float* color, const float* albedo, const float* normal, uint32_t np, float* sig,
                          float* l, float* demod, float* g_albedo, float* g_normal) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x) {
    size_t o = 3 * (size_t)p;
    float s[3];
    for (int c = 0; c < 3; ++c) s[c] = clean_radiance(color[o + c]);
    if (albedo) {
      for (int c = 0; c < 3; ++c) {
        float a = clean_unit(albedo[o + c], 0.0f);
        float d = fmaxf(a, DN_DEMOD_FLOOR);
        g_albedo[o + c] = a;
        demod[o + c] = d;
        s[c] = s[c] / d;
      }
    }
    if (normal) {
      float v[3];
      for (int c = 0; c < 3; ++c) v[c] = isfinite(normal[o + c]) ? normal[o + c] : 0.0f;
      float len = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      for (int c = 0; c < 3; ++c) g_normal[o + c] = len > 1e-6f ? v[c] / len : 0.0f;
    }
    for (int c = 0; c < 3; ++c) sig[o + c] = s[c];
    l[p] = lum(s[0], s[1], s[2]);
  }
}

struct Taps {
  float k[5];
  int n;
};

// blur_sep (denoise.rs:547-578), one direction: symmetric taps, the weight
// sum of the taps inside the image renormalises at the borders.
__global__ void k_dn_blur(const float* src, float* dst, uint32_t w, uint32_t h, Taps t, int vertical) {
  uint32_t np = w * h;
  int r = t.n / 2;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x) {
    int x = (int)(p % w), y = (int)(p / w);
    float acc = 0.0f, ws = 0.0f;
    for (int i = 0; i < t.n; ++i) {
      if (vertical) {
        int yy = y + i - r;
        if (yy >= 0 && yy < (int)h) {
          acc += t.k[i] * src[(size_t)yy * w + x];
          ws += t.k[i];
        }
      } else {
        int xx = x + i - r;
        if (xx >= 0 && xx < (int)w) {
          acc += t.k[i] * src[(size_t)y * w + xx];
          ws += t.k[i];
        }
      }
    }
    dst[p] = acc / ws;
  }
}

// noise_variance's residual (denoise.rs:582-586): 9/8 (v - mean)^2.
__global__ void k_dn_resid(const float* l, const float* mean, uint32_t np, float* out) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x) {
    float d = l[p] - mean[p];
    out[p] = 1.125f * d * d;
  }
}

__device__ __forceinline__ float pow128(float d) {
  // powi(d, 128): seven squarings, as binary exponentiation does it.
  float x = d;
#pragma unroll
  for (int i = 0; i < 7; ++i) x = x * x;
  return x;
}

// atrous_pass (denoise.rs:593-650).
__global__ void __launch_bounds__(256) k_dn_atrous(const float* sig, const float* l, const float* var,
                                                   const float* var_blur, const float* g_albedo,
                                                   const float* g_normal, uint32_t w, uint32_t h, int step,
                                                   float* out, float* out_var, float* out_l) {
  const float B3[5] = {1.0f / 16.0f, 1.0f / 4.0f, 3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};
  uint32_t np = w * h;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x) {
    int x = (int)(p % w), y = (int)(p / w);
    float lp = l[p];
    float inv_sl = 1.0f / (DN_SIGMA_LUM * sqrtf(fmaxf(var_blur[p], 0.0f)) + 1e-10f);
    float ap[3] = {0, 0, 0}, npv[3] = {0, 0, 0};
    if (g_albedo)
      for (int c = 0; c < 3; ++c) ap[c] = g_albedo[3 * (size_t)p + c];
    if (g_normal)
      for (int c = 0; c < 3; ++c) npv[c] = g_normal[3 * (size_t)p + c];
    bool np_zero = npv[0] == 0.0f && npv[1] == 0.0f && npv[2] == 0.0f;
    float acc[3] = {0, 0, 0}, ws = 0.0f, wv = 0.0f;
    for (int ky = 0; ky < 5; ++ky) {
      int qy = y + (ky - 2) * step;
      if (qy < 0 || qy >= (int)h) continue;
      float hy = B3[ky];
      for (int kx = 0; kx < 5; ++kx) {
        int qx = x + (kx - 2) * step;
        if (qx < 0 || qx >= (int)w) continue;
        float hx = B3[kx];
        size_t q = (size_t)qy * w + qx;
        float e = fabsf(l[q] - lp) * inv_sl;
        if (g_albedo) {
          float d0 = ap[0] - g_albedo[3 * q], d1 = ap[1] - g_albedo[3 * q + 1], d2 = ap[2] - g_albedo[3 * q + 2];
          e += (d0 * d0 + d1 * d1 + d2 * d2) * DN_INV_SIGMA_ALBEDO2;
        }
        float wgt = hx * hy * expf(-e);
        if (g_normal) {
          float n0 = g_normal[3 * q], n1 = g_normal[3 * q + 1], n2 = g_normal[3 * q + 2];
          bool nq_zero = n0 == 0.0f && n1 == 0.0f && n2 == 0.0f;
          if (!np_zero && !nq_zero) {
            float d = fmaxf(npv[0] * n0 + npv[1] * n1 + npv[2] * n2, 0.0f);
            wgt *= pow128(d);
          }
        }
        acc[0] += wgt * sig[3 * q];
        acc[1] += wgt * sig[3 * q + 1];
        acc[2] += wgt * sig[3 * q + 2];
        ws += wgt;
        wv += wgt * wgt * var[q];
      }
    }
    float r[3] = {acc[0] / ws, acc[1] / ws, acc[2] / ws};
    for (int c = 0; c < 3; ++c) out[3 * (size_t)p + c] = r[c];
    out_var[p] = wv / (ws * ws);
    out_l[p] = lum(r[0], r[1], r[2]);
  }
}

// denoise.rs:705-711: remodulate by the demodulation albedo.
__global__ void k_dn_remod(float* sig, const float* demod, uint32_t np) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < 3 * np; i += gridDim.x * blockDim.x)
    sig[i] = sig[i] * demod[i];
}

}  // namespace dn
