// oracle_core.h — CPU restatement of argent's vector, sampling and spectral
// primitives.  TEST INFRASTRUCTURE ONLY: the oracle is the checker that the
// CUDA path is compared against.  Nothing in the product links or calls it.
//
// Arithmetic follows the reference operation by operation so that results
// match bit for bit where the reference is deterministic.  The oracle is
// built with -ffp-contract=off so no multiply-add is fused.  glam's Vec3A
// (x86 SSE) semantics are followed:
//  - dot is (x*x' + y*y') + z*z';
//  - the cross product is the component-wise a.y*b.z - a.z*b.y form;
//  - normalize is v * (1/sqrt(dot(v,v)));
//  - vector min/max are the SSE forms (a<b ? a : b), which propagate the
//    second operand when either is NaN.
// Scalar f32::min / f32::max follow Rust and drop a NaN operand (fminf/fmaxf).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

namespace orc {

static const float PI_F = 3.14159265358979323846f;
static const float FRAC_1_PI_F = 0.318309886183790671538f;

static inline float rmin(float a, float b) { return std::fmin(a, b); }  // f32::min
static inline float rmax(float a, float b) { return std::fmax(a, b); }  // f32::max
static inline float rclamp(float v, float lo, float hi) {                // f32::clamp
  float r = v;
  if (r < lo) r = lo;
  if (r > hi) r = hi;
  return r;
}
static inline float copysign1(float v) { return std::copysign(1.0f, v); }

// glam::Vec3A with SSE semantics (core/src/geom.rs:3).
struct V3 {
  float x, y, z;
  V3() : x(0), y(0), z(0) {}
  V3(float a, float b, float c) : x(a), y(b), z(c) {}
  static V3 splat(float v) { return V3(v, v, v); }
  float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
static inline V3 operator+(V3 a, V3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 operator-(V3 a, V3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 operator-(V3 a) { return V3(-a.x, -a.y, -a.z); }
static inline V3 operator*(V3 a, float s) { return V3(a.x * s, a.y * s, a.z * s); }
static inline V3 operator*(V3 a, V3 b) { return V3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline V3 operator/(V3 a, float s) { return V3(a.x / s, a.y / s, a.z / s); }
static inline V3 operator/(V3 a, V3 b) { return V3(a.x / b.x, a.y / b.y, a.z / b.z); }
static inline float dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static inline V3 cross(V3 a, V3 b) {
  return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float length_squared(V3 a) { return dot(a, a); }
static inline float length(V3 a) { return std::sqrt(dot(a, a)); }
static inline V3 normalize(V3 a) { return a * (1.0f / std::sqrt(dot(a, a))); }
static inline float sse_min(float a, float b) { return a < b ? a : b; }
static inline float sse_max(float a, float b) { return a > b ? a : b; }
static inline V3 vmin(V3 a, V3 b) { return V3(sse_min(a.x, b.x), sse_min(a.y, b.y), sse_min(a.z, b.z)); }
static inline V3 vmax(V3 a, V3 b) { return V3(sse_max(a.x, b.x), sse_max(a.y, b.y), sse_max(a.z, b.z)); }
static inline V3 vabs(V3 a) { return V3(std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)); }
static inline float max_element(V3 a) { return sse_max(sse_max(a.x, a.z), a.y); }
static inline float min_element(V3 a) { return sse_min(sse_min(a.x, a.z), a.y); }

struct Ray {
  V3 o, d;
  V3 at(float t) const { return o + d * t; }
};

// geom.rs:26-30
static inline V3 offset_origin(V3 p, V3 ng, V3 dir) {
  float scale = 1e-4f * (1.0f + max_element(vabs(p)));
  V3 n = dot(ng, dir) >= 0.0f ? ng : -ng;
  return p + n * scale;
}

// geom.rs:33-66 (Duff et al. 2017 basis)
struct Frame {
  V3 t, b, n;
  explicit Frame(V3 nn) {
    float sign = copysign1(nn.z);
    float a = -1.0f / (sign + nn.z);
    float bb = nn.x * nn.y * a;
    t = V3(1.0f + sign * nn.x * nn.x * a, sign * bb, -sign * nn.x);
    b = V3(bb, sign + nn.y * nn.y * a, -nn.y);
    n = nn;
  }
  V3 to_local(V3 v) const { return V3(dot(v, t), dot(v, b), dot(v, n)); }
  V3 to_world(V3 v) const { return t * v.x + b * v.y + n * v.z; }
};

// geom.rs:68-84
static inline V3 reflect(V3 wo, V3 n) { return -wo + n * (2.0f * dot(wo, n)); }
static inline bool refract(V3 wi, V3 n, float eta, V3* out) {
  float cos_i = dot(n, wi);
  float sin2_i = rmax(1.0f - cos_i * cos_i, 0.0f);
  float sin2_t = sin2_i / (eta * eta);
  if (sin2_t >= 1.0f) return false;
  float cos_t = std::sqrt(1.0f - sin2_t);
  *out = -wi / eta + n * (cos_i / eta - cos_t);
  return true;
}

// geom.rs:92-96: rotation about +Y.  `deg.to_radians()` is deg * (pi/180) in f32.
static inline V3 rot_y(V3 v, float deg) {
  float r = deg * (PI_F / 180.0f);
  float s = std::sin(r), c = std::cos(r);
  return V3(c * v.x + s * v.z, v.y, -s * v.x + c * v.z);
}

// ------------------------------------------------------------------ sampling
// sampler.rs:18-25
static inline uint32_t hash32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// Owen-scrambled Sobol, Burley 2020 ("Practical Hash-based Owen Scrambling",
// JCGT 9(4)), with 4-dimensional padding.  argent calls the sobol_burley
// 0.5.0 crate here (sampler.rs:48), whose source is not available; this is
// the published algorithm, shared bit for bit with the CUDA sampler.
static const uint32_t SOBOL_MAX_DIM = 256;  // sobol_burley::NUM_DIMENSIONS

struct SobolDirs {
  uint32_t v[4][32];
  SobolDirs() {
    // dim 0: van der Corput; dims 1..3 from the primitive polynomials
    // x+1, x^2+x+1, x^3+x+1 with initial m = {1}, {1,3}, {1,3,1}.
    for (int j = 0; j < 32; ++j) v[0][j] = 1u << (31 - j);
    const int s_[4] = {0, 1, 2, 3};
    const uint32_t a_[4] = {0, 0, 1, 1};
    const uint32_t m0[4][3] = {{0, 0, 0}, {1, 0, 0}, {1, 3, 0}, {1, 3, 1}};
    for (int d = 1; d < 4; ++d) {
      int s = s_[d];
      uint32_t m[32];
      for (int k = 0; k < s; ++k) m[k] = m0[d][k];
      for (int k = s; k < 32; ++k) {
        uint32_t r = m[k - s] ^ (m[k - s] << s);
        for (int i = 1; i < s; ++i)
          if ((a_[d] >> (s - 1 - i)) & 1u) r ^= m[k - i] << i;
        m[k] = r;
      }
      for (int j = 0; j < 32; ++j) v[d][j] = m[j] << (31 - j);
    }
  }
};
extern const SobolDirs SOBOL_DIRS;

static inline uint32_t reverse_bits(uint32_t x) {
  x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
  x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
  x = ((x >> 4) & 0x0f0f0f0fu) | ((x & 0x0f0f0f0fu) << 4);
  x = ((x >> 8) & 0x00ff00ffu) | ((x & 0x00ff00ffu) << 8);
  return (x >> 16) | (x << 16);
}
static inline uint32_t lk_permutation(uint32_t x, uint32_t seed) {
  x += seed;
  x ^= x * 0x6c50b47cu;
  x ^= x * 0xb82f1e52u;
  x ^= x * 0xc7afe638u;
  x ^= x * 0x8d22f6e6u;
  return x;
}
static inline uint32_t nested_uniform_scramble(uint32_t x, uint32_t seed) {
  return reverse_bits(lk_permutation(reverse_bits(x), seed));
}
static inline uint32_t hash_combine(uint32_t seed, uint32_t v) {
  return seed ^ (v + 0x9e3779b9u + (seed << 6) + (seed >> 2));
}
static inline uint32_t sobol_dim(uint32_t index, int d) {
  uint32_t x = 0;
  for (int j = 0; index; index >>= 1, ++j)
    if (index & 1u) x ^= SOBOL_DIRS.v[d][j];
  return x;
}
static inline void sample_4d(uint32_t index, uint32_t set, uint32_t seed, float out[4]) {
  uint32_t sseed = hash_combine(seed, hash32(set));
  uint32_t shuffled = nested_uniform_scramble(index, sseed);
  for (int d = 0; d < 4; ++d) {
    uint32_t x = sobol_dim(shuffled, d);
    x = nested_uniform_scramble(x, hash_combine(sseed, hash32((uint32_t)d + 1u)));
    out[d] = (float)(x >> 8) * (1.0f / 16777216.0f);
  }
}

// sampler.rs:5-77
struct Sampler {
  uint32_t index, seed, dim;
  uint64_t rng;
  float block[4];
  uint32_t block_set;
  Sampler(uint32_t pixel_seed, uint32_t sample_index)
      : index(sample_index), seed(pixel_seed), dim(0),
        rng((((uint64_t)pixel_seed << 32) | (uint64_t)sample_index) ^ 0x9e3779b97f4a7c15ull),
        block_set(0xffffffffu) {
    block[0] = block[1] = block[2] = block[3] = 0.0f;
  }
  float next() {
    uint32_t d = dim;
    dim += 1;
    if (d < SOBOL_MAX_DIM && index < (1u << 16)) {
      uint32_t set = d / 4;
      if (set != block_set) {
        sample_4d(index, set, seed, block);
        block_set = set;
      }
      return rmin(block[d % 4], 0.99999994f);
    }
    return next_random();
  }
  void next2(float* a, float* b) {
    *a = next();
    *b = next();
  }
  float next_random() {
    rng = rng * 6364136223846793005ull + 1442695040888963407ull;
    uint64_t x = ((rng >> 18) ^ rng) >> 27;
    uint32_t rot = (uint32_t)(rng >> 59);
    uint32_t v32 = (uint32_t)x;
    uint32_t v = (v32 >> rot) | (v32 << ((32 - rot) & 31));
    return (float)(v >> 8) * (1.0f / 16777216.0f);
  }
  void set_dim(uint32_t d) { dim = d; }
};

// sampler.rs:81-100
static inline float tent(float u, float r) {
  float uu = 2.0f * u;
  if (uu < 1.0f) return r * (std::sqrt(uu) - 1.0f);
  return r * (1.0f - std::sqrt(2.0f - uu));
}
static inline void disk(float u, float v, float* ox, float* oy) {
  float a = 2.0f * u - 1.0f;
  float b = 2.0f * v - 1.0f;
  if (a == 0.0f && b == 0.0f) {
    *ox = 0.0f;
    *oy = 0.0f;
    return;
  }
  float r, phi;
  if (std::fabs(a) > std::fabs(b)) {
    r = a;
    phi = (PI_F / 4.0f) * (b / a);
  } else {
    r = b;
    phi = (PI_F / 2.0f) - (PI_F / 4.0f) * (a / b);
  }
  *ox = r * std::cos(phi);
  *oy = r * std::sin(phi);
}
static inline V3 cosine_hemisphere(float u, float v) {
  float x, y;
  disk(u, v, &x, &y);
  float z = std::sqrt(rmax(1.0f - x * x - y * y, 0.0f));
  return V3(x, y, z);
}

// ------------------------------------------------------------------ spectra
static const int N = 4;  // spec.rs:6

// spec.rs:13-76
struct Spec {
  float v[N];
  Spec() { v[0] = v[1] = v[2] = v[3] = 0.0f; }
  explicit Spec(float s) { v[0] = v[1] = v[2] = v[3] = s; }
  Spec(float a, float b, float c, float d) {
    v[0] = a;
    v[1] = b;
    v[2] = c;
    v[3] = d;
  }
  float& operator[](int i) { return v[i]; }
  float operator[](int i) const { return v[i]; }
  float max_value() const {
    float m = -3.40282347e38f;  // f32::MIN, folded with f32::max
    for (int i = 0; i < N; ++i) m = rmax(m, v[i]);
    return m;
  }
  float min_value() const {
    float m = 3.40282347e38f;
    for (int i = 0; i < N; ++i) m = rmin(m, v[i]);
    return m;
  }
  float average() const {
    float s = 0.0f;
    for (int i = 0; i < N; ++i) s += v[i];
    return s / (float)N;
  }
  bool is_black() const {
    for (int i = 0; i < N; ++i)
      if (v[i] != 0.0f) return false;
    return true;
  }
  bool is_finite() const {
    for (int i = 0; i < N; ++i)
      if (!std::isfinite(v[i])) return false;
    return true;
  }
};
static inline Spec operator+(Spec a, Spec b) {
  Spec r;
  for (int i = 0; i < N; ++i) r.v[i] = a.v[i] + b.v[i];
  return r;
}
static inline Spec operator-(Spec a, Spec b) {
  Spec r;
  for (int i = 0; i < N; ++i) r.v[i] = a.v[i] - b.v[i];
  return r;
}
static inline Spec operator*(Spec a, Spec b) {
  Spec r;
  for (int i = 0; i < N; ++i) r.v[i] = a.v[i] * b.v[i];
  return r;
}
static inline Spec operator*(Spec a, float s) {
  Spec r;
  for (int i = 0; i < N; ++i) r.v[i] = a.v[i] * s;
  return r;
}
static inline Spec operator/(Spec a, float s) {
  Spec r;
  for (int i = 0; i < N; ++i) r.v[i] = a.v[i] / s;
  return r;
}
static inline Spec spec_exp(Spec a) {
  Spec r;
  for (int i = 0; i < N; ++i) r.v[i] = std::exp(a.v[i]);
  return r;
}
static inline Spec spec_lerp(float t, Spec a, Spec b) { return a * (1.0f - t) + b * t; }

struct Wavelengths {
  float lambda[N];
  float pdf[N];
};

// spec.rs:209-220
static inline float sample_visible_wavelength(float u) {
  return 538.0f - 138.88889f * std::atanh(0.8569106f - 1.827502f * u);
}
static inline float visible_wavelength_pdf(float lambda) {
  if (!(lambda >= 360.0f && lambda <= 830.0f)) return 0.0f;
  float c = std::cosh(0.0072f * (lambda - 538.0f));
  return 0.0039398042f / (c * c);
}
// spec.rs:157-169
static inline Wavelengths sample_visible(float u) {
  Wavelengths w;
  for (int i = 0; i < N; ++i) {
    float up = u + (float)i / (float)N;
    if (up > 1.0f) up -= 1.0f;
    w.lambda[i] = sample_visible_wavelength(up);
    w.pdf[i] = visible_wavelength_pdf(w.lambda[i]);
  }
  return w;
}
// spec.rs:187-199
static inline bool secondary_terminated(const Wavelengths& w) {
  for (int i = 1; i < N; ++i)
    if (w.pdf[i] != 0.0f) return false;
  return true;
}
static inline void terminate_secondary(Wavelengths* w) {
  if (secondary_terminated(*w)) return;
  for (int i = 1; i < N; ++i) w->pdf[i] = 0.0f;
  w->pdf[0] /= (float)N;
}

// A 1 nm table over 360..=830 (core/src/tab.rs:20-27).
static inline float tab_eval(const float* values, float l) {
  float x = rclamp(l - 360.0f, 0.0f, 470.0f);
  int i = (int)x;
  if (i > 469) i = 469;
  float f = x - (float)i;
  return values[i] * (1.0f - f) + values[i + 1] * f;
}
static inline Spec tab_sample(const float* values, const Wavelengths& wl) {
  Spec r;
  for (int i = 0; i < N; ++i) r.v[i] = tab_eval(values, wl.lambda[i]);
  return r;
}
// `Piecewise::eval` on the 5 nm n,k grid (spectrum.rs:80-93).
static inline float grid_eval(const float* values, float l) {
  if (l <= 360.0f) return values[0];
  if (l >= 830.0f) return values[94];
  // partition_point(|x| x <= l) - 1 over lambda_i = 360 + 5 i
  int lo = 0, hi = 95;
  while (lo < hi) {
    int mid = (lo + hi) / 2;
    float lm = 360.0f + 5.0f * (float)mid;
    if (lm <= l)
      lo = mid + 1;
    else
      hi = mid;
  }
  int i = lo - 1;
  float li = 360.0f + 5.0f * (float)i;
  float li1 = 360.0f + 5.0f * (float)(i + 1);
  float t = (l - li) / (li1 - li);
  return values[i] * (1.0f - t) + values[i + 1] * t;
}

// fresnel.rs:11-27
static inline float fresnel_dielectric(float cos_theta_i, float eta) {
  float cos_i = rclamp(cos_theta_i, -1.0f, 1.0f);
  if (cos_i < 0.0f) {
    eta = 1.0f / eta;
    cos_i = -cos_i;
  }
  float sin2_i = 1.0f - cos_i * cos_i;
  float sin2_t = sin2_i / (eta * eta);
  if (sin2_t >= 1.0f) return 1.0f;
  float cos_t = std::sqrt(rmax(1.0f - sin2_t, 0.0f));
  float r_parl = (eta * cos_i - cos_t) / (eta * cos_i + cos_t);
  float r_perp = (cos_i - eta * cos_t) / (cos_i + eta * cos_t);
  return 0.5f * (r_parl * r_parl + r_perp * r_perp);
}

// fresnel.rs:29-78 complex helpers
struct Cf {
  float re, im;
};
static inline Cf c_add(Cf a, Cf b) { return Cf{a.re + b.re, a.im + b.im}; }
static inline Cf c_sub(Cf a, Cf b) { return Cf{a.re - b.re, a.im - b.im}; }
static inline Cf c_mul(Cf a, Cf b) { return Cf{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
static inline Cf c_scale(Cf a, float s) { return Cf{a.re * s, a.im * s}; }
static inline Cf c_div(Cf a, Cf b) {
  float d = b.re * b.re + b.im * b.im;
  return Cf{(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}
static inline float c_norm(Cf a) { return a.re * a.re + a.im * a.im; }
static inline Cf c_sqrt(Cf a) {
  float n = std::sqrt(c_norm(a));
  if (n == 0.0f) return Cf{0.0f, 0.0f};
  float t1 = std::sqrt(0.5f * (n + std::fabs(a.re)));
  float t2 = 0.5f * a.im / t1;
  if (a.re >= 0.0f) return Cf{t1, t2};
  return Cf{std::fabs(t2), std::copysign(t1, a.im)};
}
// fresnel.rs:81-93
static inline float fresnel_conductor1(float cos_theta_i, float eta, float k) {
  float cos_i = rclamp(cos_theta_i, 0.0f, 1.0f);
  float sin2_i = 1.0f - cos_i * cos_i;
  Cf e{eta, k};
  Cf sin2_t = c_div(Cf{sin2_i, 0.0f}, c_mul(e, e));
  Cf cos_t = c_sqrt(c_sub(Cf{1.0f, 0.0f}, sin2_t));
  Cf ec = c_scale(e, cos_i);
  Cf r_parl = c_div(c_sub(ec, cos_t), c_add(ec, cos_t));
  Cf ci{cos_i, 0.0f};
  Cf ect = c_mul(e, cos_t);
  Cf r_perp = c_div(c_sub(ci, ect), c_add(ci, ect));
  return 0.5f * (c_norm(r_parl) + c_norm(r_perp));
}
static inline Spec fresnel_conductor(float cos_theta_i, const Spec& eta, const Spec& k) {
  Spec r;
  for (int i = 0; i < N; ++i) r.v[i] = fresnel_conductor1(cos_theta_i, eta.v[i], k.v[i]);
  return r;
}

}  // namespace orc
