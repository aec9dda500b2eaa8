// spectra.cpp — host restatement of argent-spectra's table builders and of
// argent-core's material constructors (argent_host.h).  Built with
// -ffp-contract=off; f64 where argent uses f64.
//
//   metals::get                     spectra/src/metals.rs:110-177
//   Alloy::ior, karat_gold, bronze  spectra/src/alloys.rs:142-489
//   Blackbody, planck, luminance_y  spectra/src/spectrum.rs:95-143, 413-420
//   RgbAlbedo (sigmoid fit)         spectra/src/spectrum.rs:145-375
//   RgbIlluminant                   spectra/src/spectrum.rs:377-409
//   d65, d65_normalized, weights    spectra/src/cie.rs:94-172
//   gems::get                       spectra/src/gems.rs:152-440
//   Material::*                     core/src/material.rs:38-153
//   tab::bake                       core/src/tab.rs:8-32
#include <algorithm>
#include <array>
#include <cctype>
#include <cmath>
#include <cstring>
#include <functional>
#include <mutex>
#include <string>
#include <vector>

#include "../../../include/argent_host.h"
#include "../data/spectral_tables.h"

namespace {

const float CIE_Y_INTEGRAL = 106.85692f;
const int GRID_LEN = 95;

std::string lower(const char* s) {
  std::string r(s ? s : "");
  size_t a = r.find_first_not_of(" \t\n"), b = r.find_last_not_of(" \t\n");
  r = a == std::string::npos ? std::string() : r.substr(a, b - a + 1);
  for (auto& c : r) c = (char)std::tolower((unsigned char)c);
  return r;
}

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

// Piecewise linear spectrum (spectrum.rs:43-93).
struct Piecewise {
  std::vector<float> lambda, value;
  float eval(float l) const {
    size_t n = lambda.size();
    if (l <= lambda[0]) return value[0];
    if (l >= lambda[n - 1]) return value[n - 1];
    size_t i = (size_t)(std::upper_bound(lambda.begin(), lambda.end(), l) - lambda.begin()) - 1;
    float t = (l - lambda[i]) / (lambda[i + 1] - lambda[i]);
    return value[i] * (1.0f - t) + value[i + 1] * t;
  }
};

typedef std::function<float(float)> Spectrum;

// spectrum.rs:413-420
float luminance_y(const Spectrum& s) {
  double y = 0.0;
  for (int i = 0; i <= 470; ++i) {
    float l = 360.0f + (float)i;
    float c[3];
    xyz_bar(l, c);
    y += (double)s(l) * (double)c[1];
  }
  return (float)(y / (double)CIE_Y_INTEGRAL);
}

// tab.rs:8-32: 1 nm table of s over 360..=830.
void bake(const Spectrum& s, float out[471]) {
  for (int i = 0; i < 471; ++i) out[i] = s(360.0f + (float)i);
}

// cie.rs:94-103
const Piecewise& d65() {
  static Piecewise p;
  static std::once_flag once;
  std::call_once(once, [] {
    for (int i = 0; i < 107; ++i) {
      p.lambda.push_back(300.0f + 5.0f * (float)i);
      p.value.push_back(ARGENT_D65_300_830_5NM[i]);
    }
  });
  return p;
}
// cie.rs:107-113
const Piecewise& d65_normalized() {
  static Piecewise p;
  static std::once_flag once;
  std::call_once(once, [] {
    const Piecewise& d = d65();
    float y = luminance_y([&](float l) { return d.eval(l); });
    p = d;
    for (auto& v : p.value) v *= 1.0f / y;
  });
  return p;
}

// spectrum.rs:126-136
float planck(float lambda_nm, float t) {
  if (t <= 0.0f) return 0.0f;
  double c = 299792458.0, h = 6.62606957e-34, kb = 1.3806488e-23;
  double l = (double)lambda_nm * 1e-9;
  double le = (2.0 * h * c * c) / (std::pow(l, 5) * (std::exp((h * c) / (l * kb * (double)t)) - 1.0));
  return (float)le;
}
// Blackbody::new (spectrum.rs:104-108): peak-normalised.
struct Blackbody {
  float kelvin, norm;
  explicit Blackbody(float k) : kelvin(k) {
    float peak = 2.897772e-3f / k * 1e9f;
    norm = 1.0f / planck(peak, k);
  }
  float eval(float l) const { return planck(l, kelvin) * norm; }
};

// ----------------------------------------------------------------- sigmoid albedo
const float SIG_L0 = 360.0f, SIG_DL = 470.0f;

float sigmoid(float x) {
  if (std::fabs(x) > 1e8f) return x > 0.0f ? 1.0f : 0.0f;
  return 0.5f + 0.5f * x / std::sqrt(1.0f + x * x);
}

struct Quadrature {
  std::vector<double> t;
  std::vector<std::array<double, 3>> w;
};

// cie.rs:132-152
const std::vector<std::array<double, 3>>& d65_cmf_weights() {
  static std::vector<std::array<double, 3>> w;
  static std::once_flag once;
  std::call_once(once, [] {
    const Piecewise& d = d65();
    w.assign(471, {0.0, 0.0, 0.0});
    double ny = 0.0;
    for (int i = 0; i < 471; ++i) {
      double e = (double)d.eval(360.0f + (float)i);
      for (int k = 0; k < 3; ++k) w[i][k] = e * (double)ARGENT_CMF_1931_2DEG[3 * i + k];
      ny += w[i][1];
    }
    for (auto& row : w)
      for (auto& v : row) v /= ny;
  });
  return w;
}

// spectrum.rs:244-257
const Quadrature& fine_quadrature() {
  static Quadrature q;
  static std::once_flag once;
  std::call_once(once, [] {
    const double M[3][3] = {{3.2404542, -1.5371385, -0.4985314}, {-0.969266, 1.8760108, 0.041556},
                            {0.0556434, -0.2040259, 1.0572252}};
    const auto& xyz = d65_cmf_weights();
    for (size_t j = 0; j < xyz.size(); ++j) {
      std::array<double, 3> r;
      for (int k = 0; k < 3; ++k) r[k] = M[k][0] * xyz[j][0] + M[k][1] * xyz[j][1] + M[k][2] * xyz[j][2];
      q.w.push_back(r);
      q.t.push_back((double)j / (double)SIG_DL);
    }
  });
  return q;
}
// spectrum.rs:262-277
const Quadrature& coarse_quadrature() {
  static Quadrature q;
  static std::once_flag once;
  std::call_once(once, [] {
    const Quadrature& f = fine_quadrature();
    size_t bins = (f.t.size() - 1) / 5 + 1;
    q.w.assign(bins, {0.0, 0.0, 0.0});
    for (size_t i = 0; i < f.w.size(); ++i) {
      size_t b = std::min((i + 2) / 5, bins - 1);
      for (int k = 0; k < 3; ++k) q.w[b][k] += f.w[i][k];
    }
    for (size_t b = 0; b < bins; ++b) q.t.push_back((double)(5 * b) / (double)SIG_DL);
  });
  return q;
}

std::array<double, 3> sigmoid_rgb(const double c[3], const Quadrature& q) {
  std::array<double, 3> acc = {0.0, 0.0, 0.0};
  for (size_t j = 0; j < q.t.size(); ++j) {
    double t = q.t[j];
    double x = (c[0] * t + c[1]) * t + c[2];
    double s = 0.5 + 0.5 * x / std::sqrt(1.0 + x * x);
    for (int k = 0; k < 3; ++k) acc[k] += s * q.w[j][k];
  }
  return acc;
}

// spectrum.rs:293-316
bool solve3(double a[3][3], double b[3], double x[3]) {
  for (int col = 0; col < 3; ++col) {
    // Iterator::max_by keeps the last of equal maxima.
    int piv = col;
    for (int i = col; i < 3; ++i)
      if (std::fabs(a[i][col]) >= std::fabs(a[piv][col])) piv = i;
    if (std::fabs(a[piv][col]) < 1e-300) return false;
    for (int k = 0; k < 3; ++k) std::swap(a[col][k], a[piv][k]);
    std::swap(b[col], b[piv]);
    for (int r = col + 1; r < 3; ++r) {
      double f = a[r][col] / a[col][col];
      for (int k = col; k < 3; ++k) a[r][k] -= f * a[col][k];
      b[r] -= f * b[col];
    }
  }
  for (int r = 2; r >= 0; --r) {
    double s = 0.0;
    for (int k = r + 1; k < 3; ++k) s += a[r][k] * x[k];
    x[r] = (b[r] - s) / a[r][r];
  }
  for (int i = 0; i < 3; ++i)
    if (!std::isfinite(x[i])) return false;
  return true;
}

// spectrum.rs:320-357
void newton(double c[3], const double goal[3], const Quadrature& q, int max_iter, double tol) {
  for (int it = 0; it < max_iter; ++it) {
    double f[3] = {-goal[0], -goal[1], -goal[2]};
    double jac[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (size_t j = 0; j < q.t.size(); ++j) {
      double t = q.t[j];
      double x = (c[0] * t + c[1]) * t + c[2];
      double r = 1.0 / std::sqrt(1.0 + x * x);
      double s = 0.5 + 0.5 * x * r;
      double d = 0.5 * r * r * r;
      double dx[3] = {d * t * t, d * t, d};
      for (int k = 0; k < 3; ++k) {
        f[k] += s * q.w[j][k];
        for (int m = 0; m < 3; ++m) jac[k][m] += dx[m] * q.w[j][k];
      }
    }
    double f2 = f[0] * f[0] + f[1] * f[1] + f[2] * f[2];
    if (f2 < tol) return;
    double rhs[3] = {-f[0], -f[1], -f[2]};
    double step[3];
    if (!solve3(jac, rhs, step)) return;
    double alpha = 1.0;
    for (;;) {
      double cn[3] = {c[0] + alpha * step[0], c[1] + alpha * step[1], c[2] + alpha * step[2]};
      auto r = sigmoid_rgb(cn, q);
      double e[3] = {r[0] - goal[0], r[1] - goal[1], r[2] - goal[2]};
      if (e[0] * e[0] + e[1] * e[1] + e[2] * e[2] < f2) {
        c[0] = cn[0];
        c[1] = cn[1];
        c[2] = cn[2];
        break;
      }
      alpha *= 0.5;
      if (alpha < 1e-6) return;
    }
  }
}

// spectrum.rs:360-375
bool solve_sigmoid(const float target_f[3], float out[3]) {
  const Quadrature& coarse = coarse_quadrature();
  const Quadrature& fine = fine_quadrature();
  double target[3] = {target_f[0], target_f[1], target_f[2]};
  double g0 = std::min(std::max((target[0] + target[1] + target[2]) / 3.0, 0.02), 0.98);
  double u = 2.0 * g0 - 1.0;
  double c[3] = {0.0, 0.0, u / std::sqrt(1.0 - u * u)};
  auto start = sigmoid_rgb(c, coarse);
  const int STEPS = 8;
  for (int k = 1; k <= STEPS; ++k) {
    double a = (double)k / (double)STEPS;
    double goal[3];
    for (int i = 0; i < 3; ++i) goal[i] = start[i] + (target[i] - start[i]) * a;
    newton(c, goal, coarse, 30, 1e-10);
  }
  newton(c, target, fine, 30, 1e-16);
  for (int i = 0; i < 3; ++i)
    if (!std::isfinite(c[i])) return false;
  for (int i = 0; i < 3; ++i) out[i] = (float)c[i];
  return true;
}

// RgbAlbedo (spectrum.rs:181-233).
struct RgbAlbedo {
  bool constant = true;
  float value = 0.0f;
  float c[3] = {0, 0, 0};
  explicit RgbAlbedo(const float rgb_in[3]) {
    float rgb[3];
    for (int i = 0; i < 3; ++i) rgb[i] = std::isnan(rgb_in[i]) ? 0.0f : std::min(std::max(rgb_in[i], 0.0f), 1.0f);
    if (rgb[0] == rgb[1] && rgb[1] == rgb[2]) {
      value = rgb[0];
      return;
    }
    if (solve_sigmoid(rgb, c)) {
      constant = false;
    } else {
      value = (rgb[0] + rgb[1] + rgb[2]) / 3.0f;
    }
  }
  float eval(float l) const {
    if (constant) return value;
    float t = (l - SIG_L0) * (1.0f / SIG_DL);
    return sigmoid((c[0] * t + c[1]) * t + c[2]);
  }
};

// RgbIlluminant (spectrum.rs:387-409).
struct RgbIlluminant {
  RgbAlbedo albedo;
  float scale;
  static RgbAlbedo make(const float rgb_in[3], float* scale) {
    float rgb[3];
    for (int i = 0; i < 3; ++i) rgb[i] = std::isfinite(rgb_in[i]) ? std::max(rgb_in[i], 0.0f) : 0.0f;
    float m = 0.0f;
    for (int i = 0; i < 3; ++i) m = std::fmax(m, rgb[i]);
    *scale = 2.0f * m;
    if (m > 0.0f) {
      float q[3] = {rgb[0] / *scale, rgb[1] / *scale, rgb[2] / *scale};
      return RgbAlbedo(q);
    }
    float z[3] = {0, 0, 0};
    return RgbAlbedo(z);
  }
  explicit RgbIlluminant(const float rgb[3]) : albedo(make(rgb, &scale)) {}
  float eval(float l) const { return scale * albedo.eval(l) * d65_normalized().eval(l); }
};

// ----------------------------------------------------------------- metals
int metal_index(const std::string& n) {
  static const char* names[13][3] = {
      {"ag", "silver", ""},    {"au", "gold", ""},      {"cu", "copper", ""},   {"pt", "platinum", ""},
      {"pd", "palladium", ""}, {"rh", "rhodium", ""},   {"ni", "nickel", ""},   {"ti", "titanium", ""},
      {"al", "aluminium", "aluminum"}, {"cr", "chromium", "chrome"}, {"fe", "iron", ""}, {"zn", "zinc", ""},
      {"sn", "tin", ""}};
  for (int i = 0; i < 13; ++i)
    for (int k = 0; k < 3; ++k)
      if (names[i][k][0] && n == names[i][k]) return i;
  return -1;
}

struct Cx {
  double re, im;
};
Cx cadd(Cx a, Cx b) { return Cx{a.re + b.re, a.im + b.im}; }
Cx csub(Cx a, Cx b) { return Cx{a.re - b.re, a.im - b.im}; }
Cx cscale(Cx a, double s) { return Cx{a.re * s, a.im * s}; }
Cx from_nk(float n, float k) {
  double nn = n, kk = k;
  return Cx{nn * nn - kk * kk, 2.0 * nn * kk};
}
// alloys.rs:331-336
Cx csqrt(Cx a) {
  double m = std::hypot(a.re, a.im);
  double n = std::sqrt(std::max(0.5 * (m + a.re), 0.0));
  double k = std::sqrt(std::max(0.5 * (m - a.re), 0.0));
  return Cx{n, a.im < 0.0 ? -k : k};
}

typedef std::array<Cx, GRID_LEN> Grid;
const double HC_EV_NM = 1239.84193;
const double EPS0_OVER_HBAR = 8.8541878128e-12 / 6.582119569e-16;
const double EDGE_AU = 2.40, EDGE_CU = 2.10;
const double RHO_AU_CU = 20e-8;
const double DRUDE_AU[2] = {8.849, 0.0735}, DRUDE_AG[2] = {9.146, 0.0255}, DRUDE_CU[2] = {9.087, 0.1180};
const float DENSITY_AU = 19.32f, DENSITY_AG = 10.49f, DENSITY_CU = 8.96f;

double grid_lambda(int i) { return (double)(360.0f + 5.0f * (float)i); }

Grid eps_of(const float* nk190) {
  Grid g;
  for (int i = 0; i < GRID_LEN; ++i) g[i] = from_nk(nk190[2 * i], nk190[2 * i + 1]);
  return g;
}
Cx drude(double wp, double g, double e) {
  double d = e * e + g * g;
  return Cx{-wp * wp / d, wp * wp * g / (e * d)};
}
Grid interband(const Grid& eps, const double dr[2]) {
  Grid out = eps;
  for (int i = 0; i < GRID_LEN; ++i) {
    double e = HC_EV_NM / grid_lambda(i);
    out[i] = csub(csub(out[i], drude(dr[0], dr[1], e)), Cx{1.0, 0.0});
  }
  return out;
}
Cx grid_at(const Grid& g, double lambda) {
  double x = std::min(std::max((lambda - 360.0) / 5.0, 0.0), (double)(GRID_LEN - 1));
  size_t i = std::min((size_t)x, (size_t)(GRID_LEN - 2));
  double t = x - (double)i;
  return cadd(cscale(g[i], 1.0 - t), cscale(g[i + 1], t));
}
void to_ior(const Grid& eps, float eta[95], float k[95]) {
  for (int i = 0; i < GRID_LEN; ++i) {
    Cx nk = csqrt(eps[i]);
    eta[i] = std::fmax((float)nk.re, 1e-4f);
    k[i] = std::fmax((float)nk.im, 0.0f);
  }
}
void pure(int idx, float eta[95], float k[95]) {
  for (int i = 0; i < GRID_LEN; ++i) {
    eta[i] = ARGENT_METAL_NK[idx][2 * i];
    k[i] = ARGENT_METAL_NK[idx][2 * i + 1];
  }
}
// metals::get(..).eta.eval(l) for grid points is exact; for mix_permittivity
// argent evaluates the Piecewise at grid wavelengths, which returns the rows.
std::vector<double> volume_fractions(const std::vector<std::pair<float, float>>& parts) {
  std::vector<double> v;
  for (auto& p : parts) v.push_back((double)(std::fmax(p.first, 0.0f) / p.second));
  double s = 0.0;
  for (double x : v) s += x;
  if (s > 0.0)
    for (double& x : v) x /= s;
  return v;
}

// alloys.rs:407-418
void mix_permittivity(const std::vector<std::pair<float, const float*>>& parts, float eta[95], float k[95]) {
  double total = 0.0;
  for (auto& p : parts) total += (double)std::fmax(p.first, 0.0f);
  Grid eps;
  for (auto& e : eps) e = Cx{0.0, 0.0};
  for (int i = 0; i < GRID_LEN; ++i)
    for (auto& p : parts) {
      double w = total > 0.0 ? (double)std::fmax(p.first, 0.0f) / total : 0.0;
      eps[i] = cadd(eps[i], cscale(from_nk(p.second[2 * i], p.second[2 * i + 1]), w));
    }
  to_ior(eps, eta, k);
}

// alloys.rs:423-460
void karat_gold(float au, float ag, float cu, float eta[95], float k[95]) {
  if (std::fmax(au, 0.0f) + std::fmax(ag, 0.0f) + std::fmax(cu, 0.0f) <= 0.0f) {
    pure(1, eta, k);
    return;
  }
  auto v = volume_fractions({{au, DENSITY_AU}, {ag, DENSITY_AG}, {cu, DENSITY_CU}});
  double fau = v[0], fag = v[1], fcu = v[2];
  Grid e_au = eps_of(ARGENT_METAL_NK[1]), e_ag = eps_of(ARGENT_METAL_NK[0]), e_cu = eps_of(ARGENT_METAL_NK[2]);
  Grid eps;
  for (int i = 0; i < GRID_LEN; ++i) {
    Cx excess = cscale(Cx{(double)ARGENT_AU_AG_EXCESS_50[2 * i], (double)ARGENT_AU_AG_EXCESS_50[2 * i + 1]},
                       4.0 * fau * fag);
    eps[i] = cadd(cadd(cadd(cscale(e_au[i], fau), cscale(e_ag[i], fag)), cscale(e_cu[i], fcu)), excess);
  }
  if (fau > 0.0 && fcu > 0.0) {
    double edge = (fau * EDGE_AU + fcu * EDGE_CU) / (fau + fcu);
    struct M {
      double f;
      const Grid* e;
      const double* dr;
      double edge;
    } ms[2] = {{fau, &e_au, DRUDE_AU, EDGE_AU}, {fcu, &e_cu, DRUDE_CU, EDGE_CU}};
    for (auto& m : ms) {
      Grid ib = interband(*m.e, m.dr);
      double shift = edge - m.edge;
      for (int i = 0; i < GRID_LEN; ++i) {
        double e = HC_EV_NM / grid_lambda(i);
        Cx moved = grid_at(ib, HC_EV_NM / (e - shift));
        eps[i] = cadd(eps[i], cscale(csub(moved, ib[i]), m.f));
      }
    }
  }
  double wp2 = fau * std::pow(DRUDE_AU[0], 2) + fag * std::pow(DRUDE_AG[0], 2) + fcu * std::pow(DRUDE_CU[0], 2);
  double g0 = fau * DRUDE_AU[1] + fag * DRUDE_AG[1] + fcu * DRUDE_CU[1];
  double dg = EPS0_OVER_HBAR * wp2 * 4.0 * RHO_AU_CU * fau * fcu;
  if (dg > 0.0) {
    double wp = std::sqrt(wp2);
    for (int i = 0; i < GRID_LEN; ++i) {
      double en = HC_EV_NM / grid_lambda(i);
      eps[i] = csub(cadd(eps[i], drude(wp, g0 + dg, en)), drude(wp, g0, en));
    }
  }
  to_ior(eps, eta, k);
}

// alloys.rs:464-489
void bronze(float eta[95], float k[95]) {
  const double M_CU = 63.546, M_SN = 118.71, M_ZN = 65.38;
  double x_sn = (0.12 / M_SN) / (0.12 / M_SN + 0.88 / M_CU);
  double ea = 1.0 + 3.0 * x_sn;
  auto ea_brass = [&](double zn) { return 1.0 + (zn / M_ZN) / (zn / M_ZN + (1.0 - zn) / M_CU); };
  double ea15 = ea_brass(0.15), ea30 = ea_brass(0.30);
  double t = (ea - ea15) / (ea30 - ea15);
  Grid q_cu = eps_of(ARGENT_CU_QUERRY), q15 = eps_of(ARGENT_CU85ZN15_QUERRY), q30 = eps_of(ARGENT_CU70ZN30_QUERRY);
  Grid jc_cu = eps_of(ARGENT_METAL_NK[2]);
  double drho = (x_sn * 100.0 * 2.88 - (ea - 1.0) * 100.0 * 0.30) * 1e-8;
  double wp = DRUDE_CU[0], g = DRUDE_CU[1];
  double dg = EPS0_OVER_HBAR * wp * wp * drho;
  Grid eps;
  for (int i = 0; i < GRID_LEN; ++i) {
    Cx brass = cadd(cscale(q15[i], 1.0 - t), cscale(q30[i], t));
    double en = HC_EV_NM / grid_lambda(i);
    eps[i] = csub(cadd(cadd(jc_cu[i], csub(brass, q_cu[i])), drude(wp, g + dg, en)), drude(wp, g, en));
  }
  to_ior(eps, eta, k);
}

// Alloy::from_name (alloys.rs:260-280) -> canonical key
std::string alloy_key(const char* name) {
  std::string s = lower(name);
  for (auto& c : s)
    if (c == '_' || c == ' ') c = '-';
  struct {
    const char* key;
    const char* aliases[8];
  } table[] = {
      {"sterling", {"silver", "sterling", "925", "sterling-silver", nullptr}},
      {"fine-silver", {"fine-silver", "999", nullptr}},
      {"gold14k", {"gold", "yellow", "gold14k", "14k", "gold-filled", "gf", "yellow-gold", nullptr}},
      {"gold24k", {"gold24k", "24k", nullptr}},
      {"gold18k", {"gold18k", "18k", nullptr}},
      {"gold10k", {"gold10k", "10k", nullptr}},
      {"rose14k", {"rose", "rose-gold", "rose14k", nullptr}},
      {"white14k", {"white", "white-gold", "white14k", nullptr}},
      {"platinum", {"platinum", "pt", nullptr}},
      {"palladium", {"palladium", "pd", nullptr}},
      {"rhodium", {"rhodium", "rh", nullptr}},
      {"copper", {"copper", "cu", nullptr}},
      {"bronze", {"bronze", nullptr}},
      {"brass", {"brass", nullptr}},
  };
  for (auto& e : table)
    for (int i = 0; e.aliases[i]; ++i)
      if (s == e.aliases[i]) return e.key;
  return "";
}

bool alloy_ior(const std::string& key, float eta[95], float k[95]) {
  if (key == "fine-silver") pure(0, eta, k);
  else if (key == "gold24k") pure(1, eta, k);
  else if (key == "white14k" || key == "rhodium") pure(5, eta, k);
  else if (key == "platinum") pure(3, eta, k);
  else if (key == "palladium") pure(4, eta, k);
  else if (key == "copper") pure(2, eta, k);
  else if (key == "sterling") {
    auto v = volume_fractions({{0.925f, DENSITY_AG}, {0.075f, DENSITY_CU}});
    mix_permittivity({{(float)v[0], ARGENT_METAL_NK[0]}, {(float)v[1], ARGENT_METAL_NK[2]}}, eta, k);
  } else if (key == "gold18k") karat_gold(0.75f, 0.125f, 0.125f, eta, k);
  else if (key == "gold14k") karat_gold(0.585f, 0.2075f, 0.2075f, eta, k);
  else if (key == "gold10k") karat_gold(0.417f, 0.2915f, 0.2915f, eta, k);
  else if (key == "rose14k") karat_gold(0.585f, 0.09f, 0.325f, eta, k);
  else if (key == "brass") {
    for (int i = 0; i < GRID_LEN; ++i) {
      eta[i] = ARGENT_CU70ZN30_QUERRY[2 * i];
      k[i] = ARGENT_CU70ZN30_QUERRY[2 * i + 1];
    }
  } else if (key == "bronze") bronze(eta, k);
  else return false;
  return true;
}

// ----------------------------------------------------------------- gems (gems.rs)
const float HC = 1239.8419f;
const float FWHM_TO_SIGMA = 1.0f / 2.35482f;
struct Sellmeier {
  float b[3], c[3];
  float eval(float lambda_nm) const {
    float l2 = (lambda_nm * 1e-3f) * (lambda_nm * 1e-3f);
    float n2 = 1.0f;
    for (int i = 0; i < 3; ++i) n2 += b[i] * l2 / (l2 - c[i]);
    return std::sqrt(std::fmax(n2, 1.0f));
  }
};
struct Cauchy {
  float a, b;
  static Cauchy from_gemological(float n_d, float bg) {
    auto inv2 = [](float nm) { return 1.0f / ((nm * 1e-3f) * (nm * 1e-3f)); };
    float b = bg / (inv2(430.8f) - inv2(686.7f));
    return Cauchy{n_d - b * inv2(589.3f), b};
  }
  float eval(float lambda_nm) const {
    float l = lambda_nm * 1e-3f;
    return a + b / (l * l);
  }
};
struct Band {
  float center_nm, fwhm_low_ev, fwhm_high_ev, peak;
  float eval_ev(float e) const {
    float e0 = HC / center_nm;
    float w = (e < e0 ? fwhm_low_ev : fwhm_high_ev) * FWHM_TO_SIGMA;
    float z = (e - e0) / w;
    return peak * std::exp(-0.5f * z * z);
  }
};
Band band(float c, float f, float p) { return Band{c, f, f, p}; }
Band split(float c, float lo, float hi, float p) { return Band{c, lo, hi, p}; }
struct Urbach {
  float edge_nm, at_edge, slope_ev;
};
struct Bands {
  float floor;
  std::vector<Band> bands;
  bool has_urbach;
  Urbach u;
  float eval(float lambda_nm) const {
    float e = HC / std::fmax(lambda_nm, 1.0f);
    float s = floor;
    for (auto& b : bands) s += b.eval_ev(e);
    if (has_urbach) s += u.at_edge * std::exp(std::fmin((e - HC / u.edge_nm) / u.slope_ev, 60.0f));
    return std::fmax(s, 0.0f);
  }
};

// gems.rs:262-268 dispersion formulas
const Sellmeier DIAMOND{{4.3356f, 0.3306f, 0.0f}, {0.011236f, 0.030625f, 0.0f}};
// The gems workload's stated alternate fit (B = [0.4336, 3.3248],
// C = [0.0106, 0.0321] um^2; n_D about 2.261), not one of argent's gems.
const Sellmeier DIAMOND_ALT{{0.4336f, 3.3248f, 0.0f}, {0.0106f, 0.0321f, 0.0f}};
const Sellmeier CUBIC_ZIRCONIA{{1.347091f, 2.117788f, 9.452943f}, {0.003911627f, 0.027801894f, 591.4901f}};
const Sellmeier MOISSANITE{{0.20075f, 5.54861f, 35.65066f}, {-12.07224f, 0.02641f, 1268.247f}};
const Sellmeier CORUNDUM_O{{1.4313493f, 0.65054713f, 5.3414021f}, {0.005279926f, 0.014238265f, 325.0178f}};
const Sellmeier QUARTZ_O{{0.28604141f, 1.0704408f, 1.1020224f}, {0.0f, 0.0100586f, 100.0f}};
const Sellmeier SPINEL{{1.8938f, 3.0755f, 0.0f}, {0.009884336f, 250.46228f, 0.0f}};
const Sellmeier N_BK7{{1.0396121f, 0.23179234f, 1.0104695f}, {0.0060006987f, 0.020017914f, 103.56065f}};

struct GemDef {
  int kind;  // ARGENT_GEM_*
  Spectrum ior;
  Spectrum absorption;
  bool has_body;
  float body[3];
};

Spectrum sell(const Sellmeier& s) { return [s](float l) { return s.eval(l); }; }
Spectrum cauchy(float nd, float bg) {
  Cauchy c = Cauchy::from_gemological(nd, bg);
  return [c](float l) { return c.eval(l); };
}
Spectrum bands(Bands b) { return [b](float l) { return b.eval(l); }; }
Spectrum constant(float v) { return [v](float) { return v; }; }

bool gem_def(const std::string& name_in, GemDef* g) {
  std::string n = name_in;
  for (auto& c : n)
    if (c == '-' || c == ' ') c = '_';
  const Urbach NO{0, 0, 0};
  auto T = [&](Spectrum ior, Spectrum ab) {
    *g = GemDef{ARGENT_GEM_TRANSPARENT, ior, ab, false, {0, 0, 0}};
    return true;
  };
  auto OP = [&](float nd, float bg, float r, float gg, float b) {
    *g = GemDef{ARGENT_GEM_OPAQUE, cauchy(nd, bg), constant(20.0f), true, {r, gg, b}};
    return true;
  };
  Bands SAPPHIRE{0.0706f, {band(565, 0.62f, 0.5615f), band(700, 0.50f, 0.9784f), band(450, 0.08f, 0.15f),
                            band(388, 0.06f, 0.20f), band(377, 0.06f, 0.25f)}, true, {360, 0.3f, 0.12f}};
  Bands RUBY{0.005f, {split(556, 0.24f, 0.50f, 1.9751f), split(405, 0.40f, 0.60f, 2.9627f)}, true, {360, 0.5f, 0.15f}};
  Bands PINK{0.003f, {split(556, 0.24f, 0.50f, 0.2785f), split(405, 0.40f, 0.60f, 0.4177f)}, false, NO};
  Bands EMERALD{0.1395f, {split(610, 0.36f, 0.44f, 0.40f), split(430, 0.40f, 0.50f, 0.6177f), band(830, 0.55f, 0.171f)},
                false, NO};
  Bands AQUA{0.0324f, {band(820, 0.65f, 0.764f), band(427, 0.10f, 0.03f), band(370, 0.12f, 0.06f)}, false, NO};
  Bands MORG{0.0067f, {band(495, 0.45f, 0.0976f), band(560, 0.35f, 0.0329f)}, true, {400, 0.18f, 0.25f}};
  Bands AMETH{0.0471f, {band(545, 0.65f, 0.3908f), band(357, 0.50f, 0.035f)}, false, NO};
  Bands CITR{0.0008f, {}, true, {420, 0.8236f, 0.36f}};
  Bands SMOKY{0.0791f, {band(460, 0.90f, 0.4317f), band(620, 0.75f, 0.30f)}, true, {380, 0.6f, 0.25f}};
  Bands PERI{0.035f, {band(850, 0.55f, 1.0f), band(1050, 0.55f, 6.0f), band(1250, 0.55f, 3.0f), band(453, 0.10f, 0.20f),
                      band(473, 0.10f, 0.12f), band(493, 0.10f, 0.18f)}, true, {400, 0.9f, 0.25f}};
  Bands BTOPAZ{0.0083f, {band(640, 0.65f, 0.2855f)}, false, NO};
  Bands GARNET{0.0815f, {band(505, 0.10f, 0.6f), band(527, 0.10f, 1.6124f), band(576, 0.12f, 2.25f),
                          band(460, 0.35f, 0.6986f), band(615, 0.15f, 0.30f), band(430, 0.12f, 0.20f)},
               true, {400, 1.0f, 0.25f}};
  Bands TSAV{0.1083f, {split(605, 0.42f, 0.48f, 0.478f), split(430, 0.42f, 0.48f, 1.192f)}, false, NO};
  Bands SPRED{0.008f, {split(545, 0.24f, 0.50f, 2.5937f), split(395, 0.40f, 0.60f, 3.8905f)}, false, NO};
  Bands TANZ{0.146f, {band(595, 0.38f, 0.7046f), band(530, 0.35f, 0.208f)}, false, NO};
  Bands TOURM{0.0365f, {band(720, 0.55f, 1.5f), band(470, 0.45f, 0.72f)}, false, NO};
  Bands MOISS_ABS{0.0005f, {}, true, {380, 0.05f, 0.08f}};
  if (n == "diamond") return T(sell(DIAMOND), constant(0.0f));
  if (n == "diamond_alt") return T(sell(DIAMOND_ALT), constant(0.0f));
  if (n == "cubic_zirconia" || n == "cz" || n == "zirconia") return T(sell(CUBIC_ZIRCONIA), constant(0.0005f));
  if (n == "moissanite") return T(sell(MOISSANITE), bands(MOISS_ABS));
  if (n == "sapphire" || n == "blue_sapphire") return T(sell(CORUNDUM_O), bands(SAPPHIRE));
  if (n == "ruby") return T(sell(CORUNDUM_O), bands(RUBY));
  if (n == "pink_sapphire") return T(sell(CORUNDUM_O), bands(PINK));
  if (n == "emerald") return T(cauchy(1.580f, 0.014f), bands(EMERALD));
  if (n == "aquamarine") return T(cauchy(1.577f, 0.014f), bands(AQUA));
  if (n == "morganite") return T(cauchy(1.585f, 0.014f), bands(MORG));
  if (n == "amethyst") return T(sell(QUARTZ_O), bands(AMETH));
  if (n == "citrine") return T(sell(QUARTZ_O), bands(CITR));
  if (n == "smoky_quartz" || n == "smoky") return T(sell(QUARTZ_O), bands(SMOKY));
  if (n == "peridot" || n == "olivine") return T(cauchy(1.672f, 0.020f), bands(PERI));
  if (n == "blue_topaz") return T(cauchy(1.613f, 0.014f), bands(BTOPAZ));
  if (n == "white_topaz" || n == "topaz") return T(cauchy(1.613f, 0.014f), constant(0.0005f));
  if (n == "garnet" || n == "almandine" || n == "almandite") return T(cauchy(1.790f, 0.027f), bands(GARNET));
  if (n == "tsavorite") return T(cauchy(1.740f, 0.027f), bands(TSAV));
  if (n == "spinel" || n == "red_spinel") return T(sell(SPINEL), bands(SPRED));
  if (n == "tanzanite") return T(cauchy(1.694f, 0.030f), bands(TANZ));
  if (n == "tourmaline" || n == "green_tourmaline") return T(cauchy(1.635f, 0.017f), bands(TOURM));
  if (n == "onyx" || n == "black_onyx") return OP(1.537f, 0.013f, 0.012f, 0.012f, 0.013f);
  if (n == "obsidian") return OP(1.490f, 0.010f, 0.016f, 0.015f, 0.015f);
  if (n == "turquoise") return OP(1.620f, 0.010f, 0.080f, 0.456f, 0.429f);
  if (n == "lapis" || n == "lapis_lazuli") return OP(1.500f, 0.010f, 0.019f, 0.120f, 0.332f);
  if (n == "opal" || n == "white_opal") {
    *g = GemDef{ARGENT_GEM_OPAL, cauchy(1.450f, 0.0115f), constant(0.05f), true, {0.55f, 0.58f, 0.62f}};
    return true;
  }
  if (n == "black_opal") {
    *g = GemDef{ARGENT_GEM_OPAL, cauchy(1.450f, 0.0115f), constant(1.5f), true, {0.012f, 0.012f, 0.018f}};
    return true;
  }
  if (n == "glass" || n == "bk7" || n == "n_bk7" || n == "crown_glass") {
    Piecewise p;
    const float tab[17][2] = {{350, 3.335e-3f}, {365, 1.177e-3f}, {370, 9.308e-4f}, {380, 6.859e-4f},
                              {390, 4.424e-4f}, {400, 3.213e-4f}, {405, 2.810e-4f}, {420, 2.810e-4f},
                              {436, 3.213e-4f}, {460, 2.810e-4f}, {500, 2.407e-4f}, {546, 1.603e-4f},
                              {580, 2.005e-4f}, {620, 2.407e-4f}, {660, 2.407e-4f}, {700, 1.603e-4f},
                              {1060, 1.202e-4f}};
    for (auto& r : tab) {
      p.lambda.push_back(r[0]);
      p.value.push_back(r[1]);
    }
    return T(sell(N_BK7), [p](float l) { return p.eval(l); });
  }
  return false;
}

void zero_material(ArgentMaterial* m) { std::memset(m, 0, sizeof(*m)); }

float ggx_alpha(float r) {
  float rr = std::min(std::max(r, 0.0f), 1.0f);
  return std::fmax(rr * rr, 1e-4f);
}

void bake_albedo(const float rgb[3], float out[471]) {
  RgbAlbedo a(rgb);
  bake([&](float l) { return a.eval(l); }, out);
}

}  // namespace

extern "C" {

int argent_metal_nk(const char* name, float* eta, float* k) {
  int i = metal_index(lower(name));
  if (i < 0 || !eta || !k) return ARGENT_E_INVALID;
  pure(i, eta, k);
  return ARGENT_OK;
}

int argent_alloy_nk(const char* name, float* eta, float* k) {
  std::string key = alloy_key(name);
  if (key.empty() || !eta || !k) return ARGENT_E_INVALID;
  return alloy_ior(key, eta, k) ? ARGENT_OK : ARGENT_E_INVALID;
}

int argent_karat_gold_nk(float au, float ag, float cu, float* eta, float* k) {
  if (!eta || !k) return ARGENT_E_INVALID;
  karat_gold(au, ag, cu, eta, k);
  return ARGENT_OK;
}

float argent_luminance_y(const float* table) {
  return luminance_y([&](float l) {
    float x = std::min(std::max(l - 360.0f, 0.0f), 470.0f);
    int i = std::min((int)x, 469);
    float f = x - (float)i;
    return table[i] * (1.0f - f) + table[i + 1] * f;
  });
}

void argent_bake_emitter(float kelvin, float intensity, float* out) {
  Blackbody bb(kelvin);
  float y = std::fmax(luminance_y([&](float l) { return bb.eval(l); }), 1e-9f);
  float s = intensity / y;
  bake([&](float l) { return bb.eval(l) * s; }, out);
}

void argent_bake_rgb_albedo(const float* rgb, float* out) { bake_albedo(rgb, out); }

int argent_rgb_albedo_coefficients(const float* rgb, float* c3) {
  RgbAlbedo a(rgb);
  if (a.constant) return 0;
  for (int i = 0; i < 3; ++i) c3[i] = a.c[i];
  return 1;
}

void argent_bake_rgb_illuminant(const float* rgb, float* out) {
  RgbIlluminant il(rgb);
  bake([&](float l) { return il.eval(l); }, out);
}

// cie.rs:156-172: linear sRGB of a reflectance table under D65.
void argent_reflectance_srgb(const float* table, float* rgb) {
  const auto& w = d65_cmf_weights();
  double acc[3] = {0, 0, 0};
  for (int i = 0; i < 471; ++i)
    for (int k = 0; k < 3; ++k) acc[k] += (double)table[i] * w[i][k];
  float x = (float)acc[0], y = (float)acc[1], z = (float)acc[2];
  rgb[0] = 3.2404542f * x - 1.5371385f * y - 0.4985314f * z;
  rgb[1] = -0.969266f * x + 1.8760108f * y + 0.041556f * z;
  rgb[2] = 0.0556434f * x - 0.2040259f * y + 1.0572252f * z;
}

// ComplexIor::f0_srgb (metals.rs:102-107): r0(λ) at each nm under D65.
void argent_nk_f0_srgb(const float* eta, const float* k, float* rgb) {
  Piecewise pe, pk;
  for (int i = 0; i < GRID_LEN; ++i) {
    pe.lambda.push_back(360.0f + 5.0f * (float)i);
    pe.value.push_back(eta[i]);
    pk.lambda.push_back(360.0f + 5.0f * (float)i);
    pk.value.push_back(k[i]);
  }
  float t[471];
  for (int i = 0; i < 471; ++i) {
    float l = 360.0f + (float)i;
    float n = pe.eval(l), kk = pk.eval(l);
    t[i] = ((n - 1.0f) * (n - 1.0f) + kk * kk) / ((n + 1.0f) * (n + 1.0f) + kk * kk);
  }
  argent_reflectance_srgb(t, rgb);
}

// color.rs:32-45
void argent_blackbody_white(float kelvin, float* xyz) {
  Blackbody bb(kelvin);
  float acc[3] = {0, 0, 0};
  float l = 360.0f;
  while (l <= 830.0f) {
    float c[3];
    xyz_bar(l, c);
    float e = bb.eval(l);
    for (int i = 0; i < 3; ++i) acc[i] += c[i] * e;
    l += 1.0f;
  }
  xyz[0] = acc[0] / acc[1];
  xyz[1] = 1.0f;
  xyz[2] = acc[2] / acc[1];
}

int argent_gem_tables(const char* name, int32_t* kind, float* ior, float* absorption, float* body_rgb) {
  GemDef g;
  if (!gem_def(lower(name), &g)) return ARGENT_E_INVALID;
  if (kind) *kind = g.kind;
  if (ior) bake(g.ior, ior);
  if (absorption) bake(g.absorption, absorption);
  if (body_rgb) {
    for (int i = 0; i < 3; ++i) body_rgb[i] = g.has_body ? g.body[i] : -1.0f;
  }
  return ARGENT_OK;
}

// Gemological figures of a stone's dispersion formula, unbaked
// (gems.rs:115-140): n_d, n_F - n_C, n_G - n_B.
int argent_gem_dispersion(const char* name, float* n_d, float* fire, float* bg) {
  GemDef g;
  if (!gem_def(lower(name), &g)) return ARGENT_E_INVALID;
  *n_d = g.ior(587.56f);
  *fire = g.ior(486.13f) - g.ior(656.27f);
  *bg = g.ior(430.8f) - g.ior(686.7f);
  return ARGENT_OK;
}

// Material::metal(alloy, roughness).with_patina(default_patina(strength, alloy))
// (material.rs:39-48, 142-149).  patina_strength < 0 leaves the patina off.
int argent_material_metal(const char* alloy, float roughness, float patina_strength, ArgentMaterial* m) {
  if (!m) return ARGENT_E_INVALID;
  zero_material(m);
  std::string key = alloy_key(alloy);
  if (key.empty()) return ARGENT_E_INVALID;
  m->kind = ARGENT_MAT_METAL;
  m->alpha = ggx_alpha(roughness);
  alloy_ior(key, m->nk_eta, m->nk_k);
  if (patina_strength >= 0.0f) {
    m->has_patina = 1;
    m->patina_strength = patina_strength;
    m->patina_lo = 0.18f;
    m->patina_hi = 0.62f;
    m->patina_alpha = ggx_alpha(0.42f);
    m->patina_eta = 1.9f;
    float base[3];
    if (key == "sterling" || key == "fine-silver") {
      base[0] = 0.018f; base[1] = 0.018f; base[2] = 0.02f;
    } else if (key == "bronze" || key == "brass" || key == "copper") {
      base[0] = 0.03f; base[1] = 0.016f; base[2] = 0.008f;
    } else {
      base[0] = 0.03f; base[1] = 0.02f; base[2] = 0.01f;
    }
    bake_albedo(base, m->spec_a);
  }
  return ARGENT_OK;
}

// Metal with explicit n,k rows (e.g. karat_gold for a custom mix).
int argent_material_metal_nk(const float* eta, const float* k, float roughness, ArgentMaterial* m) {
  if (!m || !eta || !k) return ARGENT_E_INVALID;
  zero_material(m);
  m->kind = ARGENT_MAT_METAL;
  m->alpha = ggx_alpha(roughness);
  std::memcpy(m->nk_eta, eta, sizeof(float) * GRID_LEN);
  std::memcpy(m->nk_k, k, sizeof(float) * GRID_LEN);
  return ARGENT_OK;
}

// Material::opal (material.rs:63-66)
void argent_material_opal(int black, float cell_mm, ArgentMaterial* m) {
  zero_material(m);
  m->kind = ARGENT_MAT_OPAL;
  float body[3] = {0.55f, 0.58f, 0.62f};
  if (black) {
    body[0] = 0.012f;
    body[1] = 0.012f;
    body[2] = 0.018f;
  }
  bake_albedo(body, m->spec_a);
  m->cell_mm = cell_mm;
  m->strength = black ? 1.0f : 0.7f;
}

// Material::gem (material.rs:50-60)
int argent_material_gem(const char* name, ArgentMaterial* m) {
  if (!m) return ARGENT_E_INVALID;
  std::string l = lower(name);
  if (l.find("opal") != std::string::npos) {
    argent_material_opal(l.find("black") != std::string::npos || l == "opal", 0.35f, m);
    return ARGENT_OK;
  }
  GemDef g;
  if (!gem_def(l, &g)) return ARGENT_E_INVALID;
  zero_material(m);
  m->kind = ARGENT_MAT_GEM;
  m->gem_kind = g.kind;
  bake(g.ior, m->spec_a);
  bake(g.absorption, m->spec_b);
  if (g.has_body) {
    m->has_opaque_base = 1;
    bake_albedo(g.body, m->spec_b2);
  }
  return ARGENT_OK;
}

// Material::plastic (material.rs:73-75)
void argent_material_plastic(const float* rgb, float eta, float roughness, ArgentMaterial* m) {
  zero_material(m);
  m->kind = ARGENT_MAT_PLASTIC;
  m->eta = eta;
  m->alpha = ggx_alpha(roughness);
  bake_albedo(rgb, m->spec_a);
}

// Material::diffuse (material.rs:77-79)
void argent_material_diffuse(const float* rgb, ArgentMaterial* m) {
  zero_material(m);
  m->kind = ARGENT_MAT_DIFFUSE;
  bake_albedo(rgb, m->spec_a);
}

void argent_material_black(ArgentMaterial* m) {
  zero_material(m);
  m->kind = ARGENT_MAT_BLACK;
}

}  // extern "C"
