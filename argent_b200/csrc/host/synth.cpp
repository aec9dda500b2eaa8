// synth.cpp — procedural jewelry meshes for the workloads (argent_host.h).
// The ring follows argent-mesh's `torus_profile` vertex and triangle order
// (argent-mesh/src/synth.rs:153-173); the noise lattices use argent's hash32
// (argent-core/src/sampler.rs:18-25).
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
