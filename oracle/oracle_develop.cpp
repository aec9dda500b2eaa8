// oracle_develop.cpp — TEST INFRASTRUCTURE ONLY (the checker for the device
// develop; nothing in the product links it).  A plain restatement of
// argent's tone mapping and develop, crates/argent-post/src/tonemap.rs and
// color.rs: the exact per-pixel operators (`tonemap_pixel`), the per-grade
// tables and fast path (`Prepared`) and `develop`.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "oracle_api.h"

namespace {

const float INSET[3][3] = {{0.84247906f, 0.0784336f, 0.079223745f},
                           {0.042328242f, 0.8784686f, 0.07916613f},
                           {0.042375655f, 0.0784336f, 0.879143f}};
const float OUTSET[3][3] = {{1.196879f, -0.09802088f, -0.09902974f},
                            {-0.05289685f, 1.1519031f, -0.09896118f},
                            {-0.052971635f, -0.09804345f, 1.1510737f}};
const float MIN_EV = -12.47393f, MAX_EV = 4.026069f;
const float ACES_IN[3][3] = {{0.59719f, 0.35458f, 0.04823f}, {0.07600f, 0.90834f, 0.01566f}, {0.02840f, 0.13383f, 0.83777f}};
const float ACES_OUT[3][3] = {
    {1.60475f, -0.53108f, -0.07367f}, {-0.10208f, 1.10813f, -0.00605f}, {-0.00327f, -0.07276f, 1.07602f}};

struct V {
  float c[3];
};
V mat3(const float m[3][3], V v) {
  V o;
  for (int r = 0; r < 3; ++r) o.c[r] = m[r][0] * v.c[0] + m[r][1] * v.c[1] + m[r][2] * v.c[2];
  return o;
}
float clampf(float x, float lo, float hi) { return std::min(std::max(x, lo), hi); }
float luma(V v) { return 0.2126f * v.c[0] + 0.7152f * v.c[1] + 0.0722f * v.c[2]; }
// tonemap.rs:116-120
float log_encode(float v) {
  float ev = clampf(std::log2(std::max(v, 1e-10f)), MIN_EV, MAX_EV);
  return (ev - MIN_EV) / (MAX_EV - MIN_EV);
}
// tonemap.rs:123-126
float sigmoid(float x) {
  return ((((((15.5f * x - 40.14f) * x + 31.96f) * x - 6.868f) * x + 0.4298f) * x + 0.1191f) * x) - 0.00232f;
}
// tonemap.rs:129-133
float sop(float x, float s, float o, float p) {
  float v = clampf(x * s + o, 0.0f, 1.0f);
  return p == 1.0f ? v : std::pow(v, p);
}
// tonemap.rs:135-141
V saturate(V v, float sat) {
  if (sat == 1.0f) {
    for (float& c : v.c) c = clampf(c, 0.0f, 1.0f);
    return v;
  }
  float l = luma(v);
  for (float& c : v.c) c = clampf(l + sat * (c - l), 0.0f, 1.0f);
  return v;
}
// tonemap.rs:92-99
void cdl(int look, float slope[3], float off[3], float pw[3], float* sat) {
  for (int c = 0; c < 3; ++c) slope[c] = 1.0f, off[c] = 0.0f, pw[c] = 1.0f;
  *sat = 1.0f;
  if (look == 1) {
    for (int c = 0; c < 3; ++c) pw[c] = 1.35f;
    *sat = 1.4f;
  } else if (look == 2) {
    slope[1] = 0.9f;
    slope[2] = 0.5f;
    for (int c = 0; c < 3; ++c) pw[c] = 0.8f;
    *sat = 1.3f;
  }
}
// tonemap.rs:162-169
V aces(V x) {
  V v = mat3(ACES_IN, x);
  for (float& c : v.c) {
    float a = c * (c + 0.0245786f) - 0.000090537f;
    float b = c * (0.983729f * c + 0.432951f) + 0.238081f;
    c = a / b;
  }
  V o = mat3(ACES_OUT, v);
  for (float& c : o.c) c = clampf(c, 0.0f, 1.0f);
  return o;
}
// tonemap.rs:171-187
V khronos(V c) {
  const float START = 0.8f - 0.04f, DESAT = 0.15f;
  float x = std::min(std::min(c.c[0], c.c[1]), c.c[2]);
  float offset = x < 0.08f ? x - 6.25f * x * x : 0.04f;
  for (float& v : c.c) v = v - offset;
  float peak = std::max(std::max(c.c[0], c.c[1]), c.c[2]);
  if (peak < START) return c;
  float d = 1.0f - START;
  float np = 1.0f - d * d / (peak + d - START);
  for (float& v : c.c) v = v * (np / peak);
  float g = 1.0f - 1.0f / (DESAT * (peak - np) + 1.0f);
  for (float& v : c.c) v = v + (np - v) * g;
  return c;
}
float sanitize(float v) { return std::isnan(v) ? 0.0f : clampf(v, 0.0f, 65504.0f); }
float expo(float ev) { return std::isfinite(ev) ? std::pow(2.0f, ev) : 1.0f; }
// color.rs:10-19
float srgb(float x) {
  if (x <= 0.0031308f) return 12.92f * std::max(x, 0.0f);
  if (x >= 1.0f) return 1.0f;
  return 1.055f * std::pow(x, 1.0f / 2.4f) - 0.055f;
}

// tonemap.rs:201-213
V tonemap_pixel(V rgb, float ev, int op, int look, float saturation) {
  float k = expo(ev);
  V x;
  for (int c = 0; c < 3; ++c) x.c[c] = sanitize(rgb.c[c] * k);
  float sat = std::isfinite(saturation) ? std::max(saturation, 0.0f) : 1.0f;
  if (op == 0) {
    float s[3], o[3], p[3], ls;
    cdl(look, s, o, p, &ls);
    V v = mat3(INSET, x), e;
    for (int c = 0; c < 3; ++c) e.c[c] = sop(sigmoid(log_encode(v.c[c])), s[c], o[c], p[c]);
    e = saturate(e, ls * sat);
    V out = mat3(OUTSET, e);
    for (float& c : out.c) c = std::min(std::pow(std::max(c, 0.0f), 2.2f), 1.0f);
    return out;
  }
  if (op == 1) return saturate(aces(x), sat);
  if (op == 2) return saturate(khronos(x), sat);
  if (op == 3) {
    for (float& c : x.c) c = c / (1.0f + c);
    return saturate(x, sat);
  }
  return saturate(x, sat);
}

float bitsf(uint32_t u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}
uint32_t fbits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}

const uint32_t SHIFT = 14;

// BitCurve (tonemap.rs:233-258)
struct Curve {
  uint32_t base;
  std::vector<float> t;
  float eval(float v) const {
    float lo = bitsf(base << SHIFT), hi = bitsf((base + (uint32_t)t.size() - 1) << SHIFT);
    uint32_t b = fbits(std::min(std::max(v, lo), hi));
    size_t k = (b >> SHIFT) - base;
    float f = (float)(b & ((1u << SHIFT) - 1)) * (1.0f / (float)(1u << SHIFT));
    k = std::min(k, t.size() - 2);
    return t[k] * (1.0f - f) + t[k + 1] * f;
  }
};

// Lut1 (color.rs:37-64)
struct Lut {
  float lo, scale;
  size_t last;
  std::vector<float> t;
  Lut(float lo_, float hi, int n, float (*f)(float)) {
    for (int i = 0; i <= n; ++i) t.push_back(f(lo_ + (hi - lo_) * (float)i / (float)n));
    lo = lo_;
    scale = (float)n / (hi - lo_);
    last = (size_t)n;
  }
  float eval(float x) const {
    float u = (x - lo) * scale;
    u = u >= 0.0f ? std::min(u, (float)last) : 0.0f;
    size_t i = std::min((size_t)u, last - 1);
    float f = u - (float)i;
    return t[i] * (1.0f - f) + t[i + 1] * f;
  }
};

float agx_enc(float o) { return srgb(std::min(std::pow(std::max(o, 0.0f), 2.2f), 1.0f)); }

// tonemap.rs:336-343
uint64_t hash64(uint64_t x) {
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ull;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

// tonemap.rs:357-367
uint8_t q8(float v, float n) {
  if (v <= 0.0f) return 0;
  if (v >= 1.0f) return 255;
  int q = (int)(v * 255.0f + 0.5f + n);
  return (uint8_t)std::min(std::max(q, 0), 255);
}

}  // namespace

extern "C" {

void oracle_tonemap_pixel(const float* rgb, float ev, int op, int look, float saturation, float* out) {
  V v = tonemap_pixel(V{{rgb[0], rgb[1], rgb[2]}}, ev, op, look, saturation);
  for (int c = 0; c < 3; ++c) out[c] = v.c[c];
}

float oracle_srgb_encode(float x) { return srgb(x); }

// Prepared::encoded (tonemap.rs:285-333) for n pixels, then (when out8 is
// given) develop's dither and quantisation (tonemap.rs:345-391), the pixel
// index being the position in the array.
void oracle_develop(const float* rgb, uint64_t n, float ev, int op, int look, float saturation, float* enc_out,
                    uint8_t* out8) {
  float k = expo(ev);
  float sat = std::isfinite(saturation) ? std::max(saturation, 0.0f) : 1.0f;
  std::vector<Curve> curves;
  int pick[3] = {0, 0, 0};
  float csat = sat;
  float s[3], o[3], p[3], ls;
  cdl(look, s, o, p, &ls);
  if (op == 0) {
    bool shared = true;
    for (int c = 1; c < 3; ++c) shared = shared && s[c] == s[0] && o[c] == o[0] && p[c] == p[0];
    int nc = shared ? 1 : 3;
    float lo = std::pow(2.0f, MIN_EV) * 0.999f, hi = std::pow(2.0f, MAX_EV) * 1.001f;
    uint32_t base = fbits(lo) >> SHIFT, top = (fbits(hi) >> SHIFT) + 1;
    for (int c = 0; c < nc; ++c) {
      Curve cv;
      cv.base = base;
      for (uint32_t kk = base; kk <= top; ++kk)
        cv.t.push_back(sop(sigmoid(log_encode(bitsf(kk << SHIFT))), s[c], o[c], p[c]));
      curves.push_back(cv);
    }
    for (int c = 0; c < 3; ++c) pick[c] = shared ? 0 : c;
    csat = ls * sat;
  }
  Lut enc = op == 0 ? Lut(0.0f, 1.25f, 4096, agx_enc) : Lut(0.0f, 1.0f, 4096, srgb);
  for (uint64_t i = 0; i < n; ++i) {
    V x;
    for (int c = 0; c < 3; ++c) x.c[c] = sanitize(rgb[3 * i + c] * k);
    V e;
    if (op == 0) {
      V v = mat3(INSET, x);
      for (int c = 0; c < 3; ++c) e.c[c] = curves[pick[c]].eval(v.c[c]);
      if (csat != 1.0f) e = saturate(e, csat);
      V ot = mat3(OUTSET, e);
      for (int c = 0; c < 3; ++c) e.c[c] = enc.eval(ot.c[c]);
    } else {
      V d = op == 1 ? aces(x) : op == 2 ? khronos(x) : x;
      if (op == 3)
        for (float& c : d.c) c = c / (1.0f + c);
      d = saturate(d, csat);
      for (int c = 0; c < 3; ++c) e.c[c] = enc.eval(d.c[c]);
    }
    if (enc_out)
      for (int c = 0; c < 3; ++c) enc_out[3 * i + c] = e.c[c];
    if (out8) {
      uint64_t h = hash64(i ^ 0x9e3779b97f4a7c15ull);
      for (int c = 0; c < 3; ++c) {
        float u0 = (float)((h >> (20 * c)) & 0x3ff), u1 = (float)((h >> (20 * c + 10)) & 0x3ff);
        out8[3 * i + c] = q8(e.c[c], (u0 + u1 + 1.0f) * (1.0f / 1024.0f) - 1.0f);
      }
    }
  }
}

}  // extern "C"
