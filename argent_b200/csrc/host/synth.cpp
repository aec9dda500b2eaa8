// synth.cpp — procedural jewelry meshes for the workloads (argent_host.h).
// The ring follows argent-mesh's `torus_profile` vertex and triangle order
// (argent-mesh/src/synth.rs:153-173); the noise lattices use argent's hash32
// (argent-core/src/sampler.rs:18-25).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../../include/argent_host.h"

namespace {

const float TAU_F = 6.28318530717958647692f;

uint32_t hash32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

float lattice(int32_t i, int32_t j, int32_t k, uint32_t seed) {
  uint32_t h = hash32(((uint32_t)i * 0x8da6b343u) ^ ((uint32_t)j * 0xd8163841u) ^ ((uint32_t)k * 0xcb1ab31fu) ^
                      hash32(seed));
  return (float)(h >> 8) * (1.0f / 16777216.0f);
}

float smooth(float t) { return t * t * (3.0f - 2.0f * t); }

// Trilinear value noise in [0, 1).
float value_noise3(float x, float y, float z, uint32_t seed) {
  float fx = std::floor(x), fy = std::floor(y), fz = std::floor(z);
  int32_t ix = (int32_t)fx, iy = (int32_t)fy, iz = (int32_t)fz;
  float tx = smooth(x - fx), ty = smooth(y - fy), tz = smooth(z - fz);
  float c[2][2][2];
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int d = 0; d < 2; ++d) c[a][b][d] = lattice(ix + a, iy + b, iz + d, seed);
  auto lerp = [](float a, float b, float t) { return a + (b - a) * t; };
  float x00 = lerp(c[0][0][0], c[1][0][0], tx), x10 = lerp(c[0][1][0], c[1][1][0], tx);
  float x01 = lerp(c[0][0][1], c[1][0][1], tx), x11 = lerp(c[0][1][1], c[1][1][1], tx);
  return lerp(lerp(x00, x10, ty), lerp(x01, x11, ty), tz);
}

// 2D Perlin gradient noise, roughly in [-0.7, 0.7].
float perlin2(float x, float y, uint32_t seed) {
  float fx = std::floor(x), fy = std::floor(y);
  int32_t ix = (int32_t)fx, iy = (int32_t)fy;
  float dx = x - fx, dy = y - fy;
  auto grad = [&](int32_t i, int32_t j, float px, float py) {
    float a = lattice(i, j, 0x5eed, seed) * TAU_F;
    return std::cos(a) * px + std::sin(a) * py;
  };
  auto fade = [](float t) { return t * t * t * (t * (t * 6.0f - 15.0f) + 10.0f); };
  float u = fade(dx), v = fade(dy);
  float n00 = grad(ix, iy, dx, dy), n10 = grad(ix + 1, iy, dx - 1.0f, dy);
  float n01 = grad(ix, iy + 1, dx, dy - 1.0f), n11 = grad(ix + 1, iy + 1, dx - 1.0f, dy - 1.0f);
  float a = n00 + (n10 - n00) * u, b = n01 + (n11 - n01) * u;
  return a + (b - a) * v;
}

void torus_triangles(uint32_t nu, uint32_t nv, std::vector<uint32_t>& t) {
  auto id = [&](uint32_t i, uint32_t j) { return (i % nu) * nv + (j % nv); };
  t.reserve(6ull * nu * nv);
  for (uint32_t i = 0; i < nu; ++i)
    for (uint32_t j = 0; j < nv; ++j) {
      t.push_back(id(i, j));
      t.push_back(id(i + 1, j));
      t.push_back(id(i + 1, j + 1));
      t.push_back(id(i, j));
      t.push_back(id(i + 1, j + 1));
      t.push_back(id(i, j + 1));
    }
}

void vertex_normals(const std::vector<float>& p, const std::vector<uint32_t>& t, std::vector<float>& n) {
  n.assign(p.size(), 0.0f);
  for (size_t f = 0; f < t.size(); f += 3) {
    const float* a = &p[3 * (size_t)t[f]];
    const float* b = &p[3 * (size_t)t[f + 1]];
    const float* c = &p[3 * (size_t)t[f + 2]];
    float e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    float e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
    float fn[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    for (int k = 0; k < 3; ++k)
      for (int q = 0; q < 3; ++q) n[3 * (size_t)t[f + k] + q] += fn[q];
  }
  for (size_t v = 0; v < n.size(); v += 3) {
    float l = std::sqrt(n[v] * n[v] + n[v + 1] * n[v + 1] + n[v + 2] * n[v + 2]);
    if (l > 0.0f)
      for (int q = 0; q < 3; ++q) n[v + q] /= l;
  }
}

int fill(ArgentMesh* out, const std::vector<float>& p, const std::vector<uint32_t>& t, const std::vector<uint16_t>& m) {
  std::memset(out, 0, sizeof(*out));
  std::vector<float> n;
  vertex_normals(p, t, n);
  out->nv = (uint32_t)(p.size() / 3);
  out->nt = (uint32_t)(t.size() / 3);
  out->positions = (float*)std::malloc(p.size() * sizeof(float));
  out->normals = (float*)std::malloc(n.size() * sizeof(float));
  out->tris = (uint32_t*)std::malloc(t.size() * sizeof(uint32_t));
  out->tri_material = (uint16_t*)std::malloc((t.size() / 3) * sizeof(uint16_t));
  if (!out->positions || !out->normals || !out->tris || !out->tri_material) {
    argent_mesh_free(out);
    return ARGENT_E_OOM;
  }
  std::memcpy(out->positions, p.data(), p.size() * sizeof(float));
  std::memcpy(out->normals, n.data(), n.size() * sizeof(float));
  std::memcpy(out->tris, t.data(), t.size() * sizeof(uint32_t));
  if (m.empty())
    std::memset(out->tri_material, 0, (t.size() / 3) * sizeof(uint16_t));
  else
    std::memcpy(out->tri_material, m.data(), m.size() * sizeof(uint16_t));
  return ARGENT_OK;
}

}  // namespace

extern "C" {

void argent_mesh_free(ArgentMesh* m) {
  if (!m) return;
  std::free(m->positions);
  std::free(m->normals);
  std::free(m->tris);
  std::free(m->tri_material);
  std::memset(m, 0, sizeof(*m));
}

int argent_synth_ring(float R, float r, uint32_t nu, uint32_t nv, float amp, float cell_mm, uint32_t seed,
                      ArgentMesh* out) {
  if (!out || nu < 3 || nv < 3 || !(cell_mm > 0.0f) || (uint64_t)nu * nv * 2 >= (1ull << 27)) return ARGENT_E_INVALID;
  std::vector<float> p;
  p.reserve(3ull * nu * nv);
  for (uint32_t i = 0; i < nu; ++i) {
    float u = TAU_F * (float)i / (float)nu;
    float cu = std::cos(u), su = std::sin(u);
    for (uint32_t j = 0; j < nv; ++j) {
      float v = TAU_F * (float)j / (float)nv;
      float cv = std::cos(v), sv = std::sin(v);
      float rad = R + r * cv, z = r * sv;
      float x = rad * cu, y = rad * su;
      // tube normal
      float nx = cv * cu, ny = cv * su, nz = sv;
      float d = amp * (2.0f * value_noise3(x / cell_mm, y / cell_mm, z / cell_mm, seed) - 1.0f);
      p.push_back(x + nx * d);
      p.push_back(y + ny * d);
      p.push_back(z + nz * d);
    }
  }
  std::vector<uint32_t> t;
  torus_triangles(nu, nv, t);
  return fill(out, p, t, {});
}

int argent_synth_signet(float R, float r, uint32_t nu, uint32_t nv, float bezel_w, float bezel_d, float emboss_mm,
                        uint32_t seed, uint32_t mask_seed, ArgentMesh* out) {
  if (!out || nu < 3 || nv < 3 || (uint64_t)nu * nv * 2 >= (1ull << 27)) return ARGENT_E_INVALID;
  const float half_w = 0.5f * bezel_w, half_d = 0.5f * bezel_d;
  const float y_top = R + r + 1.5f;  // raised bezel plate
  std::vector<float> p;
  p.reserve(3ull * nu * nv);
  for (uint32_t i = 0; i < nu; ++i) {
    float u = TAU_F * (float)i / (float)nu;
    float cu = std::cos(u), su = std::sin(u);
    // bezel weight: 1 over the top where the band is within the plate's width
    float xc = R * cu, yc = R * su;
    float wu = yc > 0.0f ? 1.0f - smooth(std::fmin(std::fmax((std::fabs(xc) - (half_w - 1.5f)) / 1.5f, 0.0f), 1.0f)) : 0.0f;
    for (uint32_t j = 0; j < nv; ++j) {
      float v = TAU_F * (float)j / (float)nv;
      float cv = std::cos(v), sv = std::sin(v);
      float rad = R + r * cv;
      float x = rad * cu, y = rad * su, z = r * sv;
      if (wu > 0.0f) {
        // widen the section across the band toward the plate depth
        z = z * (1.0f + wu * (half_d / r - 1.0f));
        // push the outer half of the section up to the plate
        float f = smooth(std::fmin(std::fmax(cv / 0.6f, 0.0f), 1.0f)) * wu;
        if (f > 0.0f) {
          float top = y_top + emboss_mm * perlin2(x / 1.5f, z / 1.5f, seed);
          float yy = y + (top - y) * f;
          y = std::fmax(y, yy);
        }
      }
      p.push_back(x);
      p.push_back(y);
      p.push_back(z);
    }
  }
  std::vector<uint32_t> t;
  torus_triangles(nu, nv, t);
  std::vector<uint16_t> m(t.size() / 3);
  for (size_t f = 0; f < m.size(); ++f) {
    const float* a = &p[3 * (size_t)t[3 * f]];
    const float* b = &p[3 * (size_t)t[3 * f + 1]];
    const float* c = &p[3 * (size_t)t[3 * f + 2]];
    float cx = (a[0] + b[0] + c[0]) / 3.0f, cy = (a[1] + b[1] + c[1]) / 3.0f, cz = (a[2] + b[2] + c[2]) / 3.0f;
    m[f] = value_noise3(cx / 2.0f, cy / 2.0f, cz / 2.0f, mask_seed) > 0.5f ? 1 : 0;
  }
  return fill(out, p, t, m);
}

}  // extern "C"

// ------------------------------------------------------------------ gems workload
namespace {

struct Plane {
  float n[3], d;  // n . x <= d
};

// Round brilliant of girdle radius 1 centred on the origin, table up (+y),
// as the intersection of its facet half-spaces: table, 8 stars, 8 bezels,
// 16 upper girdle halves, a 32-facet girdle band, 16 lower girdle halves and
// 8 pavilion mains (57 cut facets + girdle).  Proportions: table 57 %, crown
// 34.5 deg, pavilion 40.75 deg, girdle 3 %.
std::vector<Plane> brilliant_planes() {
  std::vector<Plane> ps;
  const float PI_F = 3.14159265358979f;
  auto deg = [&](float a) { return a * PI_F / 180.0f; };
  const float girdle_half = 0.015f;
  const float crown_a = deg(34.5f), pav_a = deg(40.75f);
  const float table_r = 0.57f;
  const float crown_h = girdle_half + (1.0f - table_r) * std::tan(crown_a);
  const float culet_y = -girdle_half - std::tan(pav_a) * 1.0f;
  // A facet inclined `tilt` from the horizontal has its outward normal
  // tilted `tilt` from the vertical, toward azimuth az.
  auto add = [&](float az, float tilt, float px, float py, float pz) {
    float n[3] = {std::cos(az) * std::sin(tilt), std::cos(tilt), std::sin(az) * std::sin(tilt)};
    ps.push_back(Plane{{n[0], n[1], n[2]}, n[0] * px + n[1] * py + n[2] * pz});
  };
  auto addn = [&](float az, float tilt, float px, float py, float pz) {  // pavilion side (normal points down)
    float n[3] = {std::cos(az) * std::sin(tilt), -std::cos(tilt), std::sin(az) * std::sin(tilt)};
    ps.push_back(Plane{{n[0], n[1], n[2]}, n[0] * px + n[1] * py + n[2] * pz});
  };
  ps.push_back(Plane{{0, 1, 0}, crown_h});  // table
  for (int k = 0; k < 8; ++k) {
    float az = deg(45.0f * k);
    // bezel: through the girdle top at az, crown angle
    add(az, crown_a, std::cos(az), girdle_half, std::sin(az));
    // star: shallower, through the table edge between two bezels
    float az2 = az + deg(22.5f);
    add(az2, deg(21.7f), table_r * std::cos(az2), crown_h, table_r * std::sin(az2));
    // pavilion main: through the culet
    addn(az, pav_a, 0.0f, culet_y, 0.0f);
  }
  for (int k = 0; k < 16; ++k) {
    float az = deg(22.5f * k + 11.25f);
    add(az, deg(42.0f), std::cos(az), girdle_half, std::sin(az));    // upper girdle half
    addn(az, deg(42.0f), std::cos(az), -girdle_half, std::sin(az));  // lower girdle half
  }
  for (int k = 0; k < 32; ++k) {  // girdle band
    float az = deg(11.25f * k);
    ps.push_back(Plane{{std::cos(az), 0.0f, std::sin(az)}, 1.0f});
  }
  return ps;
}

// Convex polytope -> triangles (fan per facet).
void polytope(const std::vector<Plane>& ps, std::vector<float>& pos, std::vector<uint32_t>& tri) {
  const size_t n = ps.size();
  std::vector<std::vector<std::array<float, 3>>> face(n);
  for (size_t a = 0; a < n; ++a)
    for (size_t b = a + 1; b < n; ++b)
      for (size_t c = b + 1; c < n; ++c) {
        const float* A = ps[a].n;
        const float* B = ps[b].n;
        const float* C = ps[c].n;
        double det = A[0] * ((double)B[1] * C[2] - (double)B[2] * C[1]) - A[1] * ((double)B[0] * C[2] - (double)B[2] * C[0]) +
                     A[2] * ((double)B[0] * C[1] - (double)B[1] * C[0]);
        if (std::fabs(det) < 1e-9) continue;
        double da = ps[a].d, db = ps[b].d, dc = ps[c].d;
        double x = (da * ((double)B[1] * C[2] - (double)B[2] * C[1]) - A[1] * (db * C[2] - (double)B[2] * dc) +
                    A[2] * (db * C[1] - (double)B[1] * dc)) / det;
        double y = (A[0] * (db * C[2] - (double)B[2] * dc) - da * ((double)B[0] * C[2] - (double)B[2] * C[0]) +
                    A[2] * ((double)B[0] * dc - db * C[0])) / det;
        double z = (A[0] * ((double)B[1] * dc - db * C[1]) - A[1] * ((double)B[0] * dc - db * C[0]) +
                    da * ((double)B[0] * C[1] - (double)B[1] * C[0])) / det;
        bool inside = true;
        for (size_t q = 0; q < n && inside; ++q)
          if (ps[q].n[0] * x + ps[q].n[1] * y + ps[q].n[2] * z > ps[q].d + 1e-5) inside = false;
        if (!inside) continue;
        std::array<float, 3> v = {(float)x, (float)y, (float)z};
        for (size_t f : {a, b, c}) {
          bool dup = false;
          for (auto& w : face[f])
            if (std::fabs(w[0] - v[0]) + std::fabs(w[1] - v[1]) + std::fabs(w[2] - v[2]) < 1e-5f) dup = true;
          if (!dup) face[f].push_back(v);
        }
      }
  for (size_t f = 0; f < n; ++f) {
    auto& vs = face[f];
    if (vs.size() < 3) continue;
    float c[3] = {0, 0, 0};
    for (auto& v : vs)
      for (int k = 0; k < 3; ++k) c[k] += v[k] / (float)vs.size();
    // in-plane basis
    const float* nn = ps[f].n;
    float t[3] = {1, 0, 0};
    if (std::fabs(nn[0]) > 0.9f) t[0] = 0, t[1] = 1;
    float u[3] = {t[1] * nn[2] - t[2] * nn[1], t[2] * nn[0] - t[0] * nn[2], t[0] * nn[1] - t[1] * nn[0]};
    float w[3] = {nn[1] * u[2] - nn[2] * u[1], nn[2] * u[0] - nn[0] * u[2], nn[0] * u[1] - nn[1] * u[0]};
    std::sort(vs.begin(), vs.end(), [&](const std::array<float, 3>& p, const std::array<float, 3>& q) {
      float px = (p[0] - c[0]) * u[0] + (p[1] - c[1]) * u[1] + (p[2] - c[2]) * u[2];
      float py = (p[0] - c[0]) * w[0] + (p[1] - c[1]) * w[1] + (p[2] - c[2]) * w[2];
      float qx = (q[0] - c[0]) * u[0] + (q[1] - c[1]) * u[1] + (q[2] - c[2]) * u[2];
      float qy = (q[0] - c[0]) * w[0] + (q[1] - c[1]) * w[1] + (q[2] - c[2]) * w[2];
      return std::atan2(py, px) < std::atan2(qy, qx);
    });
    uint32_t base = (uint32_t)(pos.size() / 3);
    for (auto& v : vs)
      for (int k = 0; k < 3; ++k) pos.push_back(v[k]);
    // orient the fan so its winding gives the outward normal
    for (size_t i = 1; i + 1 < vs.size(); ++i) {
      float e1[3], e2[3];
      for (int k = 0; k < 3; ++k) {
        e1[k] = vs[i][k] - vs[0][k];
        e2[k] = vs[i + 1][k] - vs[0][k];
      }
      float cn[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
      bool out = cn[0] * nn[0] + cn[1] * nn[1] + cn[2] * nn[2] > 0.0f;
      tri.push_back(base);
      tri.push_back(base + (uint32_t)(out ? i : i + 1));
      tri.push_back(base + (uint32_t)(out ? i + 1 : i));
    }
  }
}

void append_torus(std::vector<float>& p, std::vector<uint32_t>& t, std::vector<uint16_t>& m, float R, float r,
                  uint32_t nu, uint32_t nv, const float c[3], const float ax[3], const float ay[3], const float az[3],
                  uint16_t mat) {
  // torus around local z, placed with basis (ax, ay, az) at c
  uint32_t base = (uint32_t)(p.size() / 3);
  for (uint32_t i = 0; i < nu; ++i) {
    float u = TAU_F * (float)i / (float)nu;
    for (uint32_t j = 0; j < nv; ++j) {
      float v = TAU_F * (float)j / (float)nv;
      float rad = R + r * std::cos(v);
      float l[3] = {rad * std::cos(u), rad * std::sin(u), r * std::sin(v)};
      for (int k = 0; k < 3; ++k) p.push_back(c[k] + ax[k] * l[0] + ay[k] * l[1] + az[k] * l[2]);
    }
  }
  auto id = [&](uint32_t i, uint32_t j) { return base + (i % nu) * nv + (j % nv); };
  for (uint32_t i = 0; i < nu; ++i)
    for (uint32_t j = 0; j < nv; ++j) {
      uint32_t q[6] = {id(i, j), id(i + 1, j), id(i + 1, j + 1), id(i, j), id(i + 1, j + 1), id(i, j + 1)};
      for (int k = 0; k < 6; ++k) t.push_back(q[k]);
      m.push_back(mat);
      m.push_back(mat);
    }
}

void append_stone(std::vector<float>& p, std::vector<uint32_t>& t, std::vector<uint16_t>& m,
                  const std::vector<float>& sp, const std::vector<uint32_t>& st, float radius, const float c[3],
                  const float ax[3], const float ay[3], const float az[3], uint16_t mat) {
  uint32_t base = (uint32_t)(p.size() / 3);
  for (size_t i = 0; i < sp.size(); i += 3) {
    float l[3] = {sp[i] * radius, sp[i + 1] * radius, sp[i + 2] * radius};
    for (int k = 0; k < 3; ++k) p.push_back(c[k] + ax[k] * l[0] + ay[k] * l[1] + az[k] * l[2]);
  }
  for (uint32_t i : st) t.push_back(base + i);
  for (size_t i = 0; i < st.size() / 3; ++i) m.push_back(mat);
}

}  // namespace

extern "C" {

// Gems workload: an 18k setting (torus shank + 37 prong cups, each a small
// torus collar and four torus prongs) holding one round brilliant of
// girdle radius `center_mm` on top and 36 smaller brilliants of girdle radius
// `stone_mm` around the shank.  Materials: 0 = metal, 1 = centre stone,
// 2..5 = the four side-stone gems, chosen per stone by `seed`.  `shank_nu`,
// `shank_nv` set the shank tessellation (the setting's triangle count).
int argent_synth_gem_ring(uint32_t shank_nu, uint32_t shank_nv, float center_mm, float stone_mm, uint32_t seed,
                          ArgentMesh* out) {
  if (!out || shank_nu < 3 || shank_nv < 3) return ARGENT_E_INVALID;
  std::vector<float> p;
  std::vector<uint32_t> t;
  std::vector<uint16_t> m;
  const float R = 9.0f, r = 1.1f;
  const float X[3] = {1, 0, 0}, Y[3] = {0, 1, 0}, Z[3] = {0, 0, 1};
  const float O[3] = {0, 0, 0};
  append_torus(p, t, m, R, r, shank_nu, shank_nv, O, X, Y, Z, 0);
  std::vector<float> sp;
  std::vector<uint32_t> st;
  polytope(brilliant_planes(), sp, st);
  // centre stone on top of the shank, table up
  const float ctop[3] = {0.0f, R + r + 0.9f * center_mm, 0.0f};
  append_stone(p, t, m, sp, st, center_mm, ctop, X, Y, Z, 1);
  auto cup = [&](const float c[3], const float ax[3], const float ay[3], const float az[3], float rad, uint32_t res) {
    // collar under the girdle (local y is the stone's up axis)
    float cc[3] = {c[0] - ay[0] * 0.05f * rad, c[1] - ay[1] * 0.05f * rad, c[2] - ay[2] * 0.05f * rad};
    // the torus axis is local z: map (x, y, z)_torus -> (ax, az, ay) so it lies in the girdle plane
    append_torus(p, t, m, rad * 1.05f, 0.08f * rad + 0.05f, res, res / 4, cc, ax, az, ay, 0);
    for (int k = 0; k < 4; ++k) {
      float a = TAU_F * (float)k / 4.0f + 0.39f;
      float px = std::cos(a) * rad * 1.02f, pz = std::sin(a) * rad * 1.02f;
      float pc[3];
      for (int q = 0; q < 3; ++q) pc[q] = c[q] + ax[q] * px + az[q] * pz + ay[q] * 0.1f * rad;
      float prx[3] = {-std::sin(a) * ax[0] + std::cos(a) * az[0], -std::sin(a) * ax[1] + std::cos(a) * az[1],
                      -std::sin(a) * ax[2] + std::cos(a) * az[2]};
      float pry[3] = {std::cos(a) * ax[0] + std::sin(a) * az[0], std::cos(a) * ax[1] + std::sin(a) * az[1],
                      std::cos(a) * ax[2] + std::sin(a) * az[2]};
      append_torus(p, t, m, 0.25f * rad, 0.06f * rad + 0.03f, res / 2, res / 8 + 3, pc, pry, ay, prx, 0);
    }
  };
  cup(ctop, X, Y, Z, center_mm, 256);
  // 36 side stones around the shank's outer surface, tables facing outward
  uint32_t h = seed * 0x9e3779b9u + 0x7f4a7c15u;
  for (int i = 0; i < 36; ++i) {
    float a = TAU_F * ((float)i + 0.5f) / 36.0f;
    float dir[3] = {std::cos(a), std::sin(a), 0.0f};
    // skip the centre stone's seat on top
    float rr = R + r + 0.35f * stone_mm;
    float c[3] = {dir[0] * rr, dir[1] * rr, 0.0f};
    const float* up = dir;
    float ax2[3] = {-dir[1], dir[0], 0.0f};
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    h *= 0x846ca68bu;
    h ^= h >> 16;
    uint16_t gem_slot = (uint16_t)(2 + (h >> 30));
    append_stone(p, t, m, sp, st, stone_mm, c, ax2, up, Z, gem_slot);
    cup(c, ax2, up, Z, stone_mm, 64);
  }
  return fill(out, p, t, m);
}

}  // extern "C"
