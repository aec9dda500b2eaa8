// develop.cpp — argent-post's per-grade develop tables (tonemap.rs:233-309,
// color.rs:37-64), built with the host's f32 log2/pow exactly as argent's
// Rust, which calls the platform libm, builds them.
#include "develop.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace argent {

namespace {

const float AGX_MIN_EV = -12.47393f;
const float AGX_MAX_EV = 4.026069f;

float bits_f(uint32_t u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}
uint32_t f_bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}
float fclamp(float x, float lo, float hi) { return std::min(std::max(x, lo), hi); }

// tonemap.rs:116-120
float agx_log_encode(float v) {
  float ev = fclamp(std::log2(std::max(v, 1e-10f)), AGX_MIN_EV, AGX_MAX_EV);
  return (ev - AGX_MIN_EV) / (AGX_MAX_EV - AGX_MIN_EV);
}
// tonemap.rs:123-126
float agx_sigmoid(float x) {
  return ((((((15.5f * x - 40.14f) * x + 31.96f) * x - 6.868f) * x + 0.4298f) * x + 0.1191f) * x) - 0.00232f;
}
// tonemap.rs:129-133
float cdl_sop(float x, float slope, float offset, float power) {
  float v = fclamp(x * slope + offset, 0.0f, 1.0f);
  return power == 1.0f ? v : std::pow(v, power);
}
// color.rs:10-19
float srgb_encode(float x) {
  if (x <= 0.0031308f) return 12.92f * std::max(x, 0.0f);
  if (x >= 1.0f) return 1.0f;
  return 1.055f * std::pow(x, 1.0f / 2.4f) - 0.055f;
}

// tonemap.rs:92-99
void look_cdl(int look, float slope[3], float offset[3], float power[3], float* sat) {
  for (int c = 0; c < 3; ++c) {
    slope[c] = 1.0f;
    offset[c] = 0.0f;
    power[c] = 1.0f;
  }
  *sat = 1.0f;
  if (look == AGX_PUNCHY) {
    for (int c = 0; c < 3; ++c) power[c] = 1.35f;
    *sat = 1.4f;
  } else if (look == AGX_GOLDEN) {
    slope[1] = 0.9f;
    slope[2] = 0.5f;
    for (int c = 0; c < 3; ++c) power[c] = 0.8f;
    *sat = 1.3f;
  }
}

void lut1(DevelopTables& t, float lo, float hi, int segments, float (*f)(float)) {
  int n = std::max(segments, 2);
  t.enc.resize(n + 1);
  for (int i = 0; i <= n; ++i) t.enc[i] = f(lo + (hi - lo) * (float)i / (float)n);
  t.enc_lo = lo;
  t.enc_scale = (float)n / (hi - lo);
  t.enc_last = (uint32_t)n;
}

float agx_encode(float o) { return srgb_encode(std::min(std::pow(std::max(o, 0.0f), 2.2f), 1.0f)); }

}  // namespace

DevelopTables develop_tables(float exposure_ev, int op, int look, float saturation) {
  DevelopTables t;
  // tonemap.rs:195-199, 287-288
  t.k = std::isfinite(exposure_ev) ? std::pow(2.0f, exposure_ev) : 1.0f;
  float sat = std::isfinite(saturation) ? std::max(saturation, 0.0f) : 1.0f;
  t.op = op;
  t.ncurves = 0;
  t.pick[0] = t.pick[1] = t.pick[2] = 0;
  t.curve_base = 0;
  t.curve_len = 0;
  if (op == TM_AGX) {
    float slope[3], offset[3], power[3], lsat;
    look_cdl(look, slope, offset, power, &lsat);
    bool shared = true;
    for (int c = 1; c < 3; ++c)
      shared = shared && slope[c] == slope[0] && offset[c] == offset[0] && power[c] == power[0];
    int n = shared ? 1 : 3;
    // BitCurve::new (tonemap.rs:240-247)
    float lo = std::pow(2.0f, AGX_MIN_EV) * 0.999f;
    float hi = std::pow(2.0f, AGX_MAX_EV) * 1.001f;
    uint32_t base = f_bits(lo) >> CURVE_SHIFT;
    uint32_t top = (f_bits(hi) >> CURVE_SHIFT) + 1;
    t.curve_base = base;
    t.curve_len = top - base + 1;
    t.curves.resize((size_t)n * t.curve_len);
    for (int c = 0; c < n; ++c)
      for (uint32_t kk = base; kk <= top; ++kk)
        t.curves[(size_t)c * t.curve_len + (kk - base)] =
            cdl_sop(agx_sigmoid(agx_log_encode(bits_f(kk << CURVE_SHIFT))), slope[c], offset[c], power[c]);
    t.ncurves = n;
    for (int c = 0; c < 3; ++c) t.pick[c] = shared ? 0 : c;
    t.sat = lsat * sat;
    lut1(t, 0.0f, 1.25f, LUT_SEGMENTS, agx_encode);
  } else {
    t.sat = sat;
    lut1(t, 0.0f, 1.0f, LUT_SEGMENTS, srgb_encode);
  }
  return t;
}

}  // namespace argent
