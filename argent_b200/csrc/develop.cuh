// develop.cuh — argent-post's `develop` fast path on the device
// (crates/argent-post/src/tonemap.rs:311-391): per pixel, exposure and
// sanitise, the operator (AgX through the per-grade bit-pattern curves, or
// ACES fitted / Khronos PBR Neutral / Reinhard / clamp), saturation, the
// sRGB (or AgX display) encode table, TPDF dither and 8-bit quantisation.
// The tables come from the host (host/develop.cpp) and every step rounds as
// argent's f32 code does (no FMA contraction), so the 8-bit output is
// argent's byte for byte.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace dv {

struct DevTables {
  float k;
  int op;
  float sat;
  int pick0, pick1, pick2;
  const float* curves;
  uint32_t curve_base, curve_len;
  const float* enc;
  float enc_lo, enc_scale;
  uint32_t enc_last;
};

#define DV_CURVE_SHIFT 14u

__device__ __forceinline__ float sanitize(float v) { return isnan(v) ? 0.0f : fminf(fmaxf(v, 0.0f), 65504.0f); }

__device__ __forceinline__ void mat3(const float m[9], const float v[3], float o[3]) {
  o[0] = m[0] * v[0] + m[1] * v[1] + m[2] * v[2];
  o[1] = m[3] * v[0] + m[4] * v[1] + m[5] * v[2];
  o[2] = m[6] * v[0] + m[7] * v[1] + m[8] * v[2];
}

// BitCurve::eval (tonemap.rs:249-258)
__device__ __forceinline__ float curve_eval(const DevTables& t, int c, float v) {
  const float* tab = t.curves + (size_t)c * t.curve_len;
  float lo = __uint_as_float(t.curve_base << DV_CURVE_SHIFT);
  float hi = __uint_as_float((t.curve_base + t.curve_len - 1) << DV_CURVE_SHIFT);
  uint32_t bits = __float_as_uint(fminf(fmaxf(v, lo), hi));
  uint32_t k = (bits >> DV_CURVE_SHIFT) - t.curve_base;
  float f = (float)(bits & ((1u << DV_CURVE_SHIFT) - 1u)) * (1.0f / (float)(1u << DV_CURVE_SHIFT));
  k = min(k, t.curve_len - 2);
  return __ldg(tab + k) * (1.0f - f) + __ldg(tab + k + 1) * f;
}

// Lut1::eval (color.rs:54-63)
__device__ __forceinline__ float enc_eval(const DevTables& t, float x) {
  float u = (x - t.enc_lo) * t.enc_scale;
  u = u >= 0.0f ? fminf(u, (float)t.enc_last) : 0.0f;
  uint32_t i = min((uint32_t)u, t.enc_last - 1);
  float f = u - (float)i;
  return __ldg(t.enc + i) * (1.0f - f) + __ldg(t.enc + i + 1) * f;
}

__device__ __forceinline__ float luma(const float v[3]) { return 0.2126f * v[0] + 0.7152f * v[1] + 0.0722f * v[2]; }

// tonemap.rs:135-141
__device__ __forceinline__ void saturate(float v[3], float sat) {
  if (sat == 1.0f) {
    for (int c = 0; c < 3; ++c) v[c] = fminf(fmaxf(v[c], 0.0f), 1.0f);
    return;
  }
  float l = luma(v);
  for (int c = 0; c < 3; ++c) v[c] = fminf(fmaxf(l + sat * (v[c] - l), 0.0f), 1.0f);
}

// splitmix64 finaliser (tonemap.rs:336-343)
__device__ __forceinline__ uint64_t hash64(uint64_t x) {
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ull;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

// tonemap.rs:357-367
__device__ __forceinline__ uint8_t quantize8(float v, float n) {
  if (v <= 0.0f) return 0;
  if (v >= 1.0f) return 255;
  int q = (int)(v * 255.0f + 0.5f + n);
  return (uint8_t)min(max(q, 0), 255);
}

// One thread per pixel; the dither index is the pixel's position y*w + x.
__global__ void __launch_bounds__(256) k_develop(const float* rgb, uint32_t np, DevTables t, uint8_t* out) {
  // Minimal AgX inset/outset (tonemap.rs:71-80) and Hill's ACES fit
  // matrices (tonemap.rs:158-160), as rows.
  const float INSET[9] = {0.84247906f, 0.0784336f, 0.079223745f, 0.042328242f, 0.8784686f,
                          0.07916613f, 0.042375655f, 0.0784336f,  0.879143f};
  const float OUTSET[9] = {1.196879f,   -0.09802088f, -0.09902974f, -0.05289685f, 1.1519031f,
                           -0.09896118f, -0.052971635f, -0.09804345f, 1.1510737f};
  const float ACES_IN[9] = {0.59719f, 0.35458f, 0.04823f, 0.07600f, 0.90834f, 0.01566f, 0.02840f, 0.13383f, 0.83777f};
  const float ACES_OUT[9] = {1.60475f,  -0.53108f, -0.07367f, -0.10208f, 1.10813f,
                             -0.00605f, -0.00327f, -0.07276f, 1.07602f};
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x) {
    float x[3];
    for (int c = 0; c < 3; ++c) x[c] = sanitize(rgb[3 * (size_t)p + c] * t.k);
    float s[3];
    if (t.op == 0) {
      float v[3], e[3];
      mat3(INSET, x, v);
      e[0] = curve_eval(t, t.pick0, v[0]);
      e[1] = curve_eval(t, t.pick1, v[1]);
      e[2] = curve_eval(t, t.pick2, v[2]);
      if (t.sat != 1.0f) saturate(e, t.sat);
      float o[3];
      mat3(OUTSET, e, o);
      for (int c = 0; c < 3; ++c) s[c] = enc_eval(t, o[c]);
    } else {
      float d[3];
      if (t.op == 1) {
        float v[3];
        mat3(ACES_IN, x, v);
        for (int c = 0; c < 3; ++c) {
          float a = v[c] * (v[c] + 0.0245786f) - 0.000090537f;
          float b = v[c] * (0.983729f * v[c] + 0.432951f) + 0.238081f;
          v[c] = a / b;
        }
        mat3(ACES_OUT, v, d);
        for (int c = 0; c < 3; ++c) d[c] = fminf(fmaxf(d[c], 0.0f), 1.0f);
      } else if (t.op == 2) {
        // Khronos PBR Neutral (tonemap.rs:171-187)
        const float START = 0.8f - 0.04f, DESAT = 0.15f;
        for (int c = 0; c < 3; ++c) d[c] = x[c];
        float mn = fminf(fminf(d[0], d[1]), d[2]);
        float offset = mn < 0.08f ? mn - 6.25f * mn * mn : 0.04f;
        for (int c = 0; c < 3; ++c) d[c] = d[c] - offset;
        float peak = fmaxf(fmaxf(d[0], d[1]), d[2]);
        if (peak >= START) {
          float dd = 1.0f - START;
          float new_peak = 1.0f - dd * dd / (peak + dd - START);
          for (int c = 0; c < 3; ++c) d[c] = d[c] * (new_peak / peak);
          float g = 1.0f - 1.0f / (DESAT * (peak - new_peak) + 1.0f);
          for (int c = 0; c < 3; ++c) d[c] = d[c] + (new_peak - d[c]) * g;
        }
      } else if (t.op == 3) {
        for (int c = 0; c < 3; ++c) d[c] = x[c] / (1.0f + x[c]);
      } else {
        for (int c = 0; c < 3; ++c) d[c] = x[c];
      }
      saturate(d, t.sat);
      for (int c = 0; c < 3; ++c) s[c] = enc_eval(t, d[c]);
    }
    // tpdf3 (tonemap.rs:345-355)
    uint64_t h = hash64((uint64_t)p ^ 0x9e3779b97f4a7c15ull);
    const float S = 1.0f / 1024.0f;
    for (int c = 0; c < 3; ++c) {
      float u0 = (float)((h >> (20 * c)) & 0x3ffu), u1 = (float)((h >> (20 * c + 10)) & 0x3ffu);
      float n = (u0 + u1 + 1.0f) * S - 1.0f;
      out[3 * (size_t)p + c] = quantize8(s[c], n);
    }
  }
}

}  // namespace dv
