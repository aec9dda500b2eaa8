// dev_math.cuh — device vector helpers with argent's operation order.
//
// The library is compiled with --fmad=false, so each expression below rounds
// every multiply and add separately, like argent's Rust build (no FMA
// contraction).  glam's Vec3A order is kept: dot is (x*x' + y*y') + z*z',
// normalize is v * (1/sqrt(dot)), and vector min/max are the SSE forms
// (a<b ? a : b) argent's slab tests rely on.  Scalar min/max follow Rust's
// f32::min/max (NaN-dropping), i.e. fminf/fmaxf.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace dev {

#define ARGENT_PI_F 3.14159265358979323846f
#define ARGENT_FRAC_1_PI_F 0.318309886183790671538f

struct V3 {
  float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 operator/(V3 a, float s) { return V3{a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ float dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
  return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float length_squared(V3 a) { return dot(a, a); }
__device__ __forceinline__ float length(V3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ V3 normalize(V3 a) { return a * (1.0f / sqrtf(dot(a, a))); }
__device__ __forceinline__ float sse_min(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float sse_max(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float max_element_abs(V3 a) {
  return sse_max(sse_max(fabsf(a.x), fabsf(a.z)), fabsf(a.y));
}
__device__ __forceinline__ float rclamp(float v, float lo, float hi) {
  float r = v;
  if (r < lo) r = lo;
  if (r > hi) r = hi;
  return r;
}

// geom.rs:26-30
__device__ __forceinline__ V3 offset_origin(V3 p, V3 ng, V3 dir) {
  float scale = 1e-4f * (1.0f + max_element_abs(p));
  V3 n = dot(ng, dir) >= 0.0f ? ng : -ng;
  return p + n * scale;
}

// geom.rs:33-66
struct Frame {
  V3 t, b, n;
};
__device__ __forceinline__ Frame make_frame(V3 n) {
  float sign = copysignf(1.0f, n.z);
  float a = -1.0f / (sign + n.z);
  float bb = n.x * n.y * a;
  Frame f;
  f.t = V3{1.0f + sign * n.x * n.x * a, sign * bb, -sign * n.x};
  f.b = V3{bb, sign + n.y * n.y * a, -n.y};
  f.n = n;
  return f;
}
__device__ __forceinline__ V3 to_local(const Frame& f, V3 v) { return V3{dot(v, f.t), dot(v, f.b), dot(v, f.n)}; }
__device__ __forceinline__ V3 to_world(const Frame& f, V3 v) { return f.t * v.x + f.b * v.y + f.n * v.z; }

__device__ __forceinline__ V3 reflect(V3 wo, V3 n) { return -wo + n * (2.0f * dot(wo, n)); }
__device__ __forceinline__ bool refract(V3 wi, V3 n, float eta, V3* out) {
  float cos_i = dot(n, wi);
  float sin2_i = fmaxf(1.0f - cos_i * cos_i, 0.0f);
  float sin2_t = sin2_i / (eta * eta);
  if (sin2_t >= 1.0f) return false;
  float cos_t = sqrtf(1.0f - sin2_t);
  *out = (-wi) / eta + n * (cos_i / eta - cos_t);
  return true;
}

// Rotation about +Y with a precomputed (sin, cos) (geom.rs:92-96).
__device__ __forceinline__ V3 rot_y_sc(V3 v, float s, float c) { return V3{c * v.x + s * v.z, v.y, -s * v.x + c * v.z}; }

__device__ __forceinline__ V3 ld3(const float* p) { return V3{p[0], p[1], p[2]}; }

}  // namespace dev
