// oracle_cavity.cpp — TEST INFRASTRUCTURE ONLY (the checker for the cavity
// mask; nothing in the product links it).  A plain, single-threaded
// restatement of argent's per-vertex patina mask,
// crates/argent-mesh/src/cavity.rs, with ambient occlusion run on argent's
// own BVH (oracle_bvh.cpp) through the Occluder of
// crates/argent-core/src/scene.rs:40-44.
//
// glam 0.34.1 (Cargo.lock) is not vendored.  Vec3::normalize_or_zero and
// Vec3::any_orthonormal_pair are restated from glam's documented behaviour:
// the pair is the branchless basis of Duff et al. 2017 ("Building an
// Orthonormal Basis, Revisited", JCGT 6(1)) with sign = signum(z)
// (f32::signum gives +1 for +0.0), in glam's scalar operation order.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <vector>

#include "oracle_api.h"
#include "oracle_bvh.h"

using orc::V3;

namespace {

// util.rs:244-257
uint32_t hash32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
float unit_f32(uint32_t h) { return (float)(h >> 8) * (1.0f / 16777216.0f); }

V3 vec_normalize_or_zero(V3 v) {
  float rcp = 1.0f / std::sqrt((v.x * v.x + v.y * v.y) + v.z * v.z);
  if (std::isfinite(rcp) && rcp > 0.0f) return V3(v.x * rcp, v.y * rcp, v.z * rcp);
  return V3(0, 0, 0);
}

void any_orthonormal_pair(V3 n, V3* t, V3* b) {
  float sign = std::signbit(n.z) ? -1.0f : 1.0f;
  float a = -1.0f / (sign + n.z);
  float bb = n.x * n.y * a;
  *t = V3(1.0f + sign * n.x * n.x * a, sign * bb, -sign * n.x);
  *b = V3(bb, sign + n.y * n.y * a, -n.y);
}

float smoothstep(float e0, float e1, float x) {
  float t = std::min(std::max((x - e0) / (e1 - e0), 0.0f), 1.0f);
  return t * t * (3.0f - 2.0f * t);
}

struct D {
  double x, y, z;
};
D dd(const float* p) { return {(double)p[0], (double)p[1], (double)p[2]}; }
D dsub(D a, D b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
double ddot(D a, D b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
D dcross(D a, D b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
double dlen(D a) { return std::sqrt(ddot(a, a)); }
D dnorm0(D a) {
  double r = 1.0 / dlen(a);
  if (std::isfinite(r) && r > 0.0) return {a.x * r, a.y * r, a.z * r};
  return {0, 0, 0};
}

}  // namespace

extern "C" {

// normals.rs:226-242: angle-weighted vertex normals.
void oracle_smooth_vertex_normals(const float* pos, uint32_t nv, const uint32_t* tris, uint32_t nt, float* out) {
  std::vector<D> acc(nv, D{0, 0, 0});
  for (uint32_t f = 0; f < nt; ++f) {
    const uint32_t* t = tris + 3 * (size_t)f;
    D n = dcross(dsub(dd(pos + 3 * t[1]), dd(pos + 3 * t[0])), dsub(dd(pos + 3 * t[2]), dd(pos + 3 * t[0])));
    double l = dlen(n);
    float fn[3] = {0.0f, 0.0f, 0.0f};
    if (l > 0.0) {
      fn[0] = (float)(n.x / l);
      fn[1] = (float)(n.y / l);
      fn[2] = (float)(n.z / l);
    }
    for (int k = 0; k < 3; ++k) {
      D p = dd(pos + 3 * t[k]);
      D ea = dsub(dd(pos + 3 * t[(k + 1) % 3]), p);
      D eb = dsub(dd(pos + 3 * t[(k + 2) % 3]), p);
      double ang = std::atan2(dlen(dcross(ea, eb)), ddot(ea, eb));
      acc[t[k]].x += ang * fn[0];
      acc[t[k]].y += ang * fn[1];
      acc[t[k]].z += ang * fn[2];
    }
  }
  for (uint32_t v = 0; v < nv; ++v) {
    double l = dlen(acc[v]);
    bool ok = l > 1e-300;
    out[3 * v] = ok ? (float)(acc[v].x / l) : 0.0f;
    out[3 * v + 1] = ok ? (float)(acc[v].y / l) : 0.0f;
    out[3 * v + 2] = ok ? (float)(acc[v].z / l) : 1.0f;
  }
}

// cavity.rs:96-135, on argent's BVH.
void oracle_ambient_occlusion(const float* pos, uint32_t nv, const float* normals, const uint32_t* tris, uint32_t nt,
                              uint32_t samples, float distance, float* out) {
  orc::Bvh bvh = orc::Bvh::build(pos, tris, nt);
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t v = 0; v < nv; ++v)
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], pos[3 * (size_t)v + k]);
      hi[k] = std::max(hi[k], pos[3 * (size_t)v + k]);
    }
  float ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
  float diag = std::sqrt((ex * ex + ey * ey) + ez * ez);
  float eps = std::max(2e-4f * diag, 1e-3f);
  uint32_t n = std::max(samples, 1u);
  for (uint32_t v = 0; v < nv; ++v) {
    V3 nn = vec_normalize_or_zero(V3(normals[3 * v], normals[3 * v + 1], normals[3 * v + 2]));
    if (nn.x == 0.0f && nn.y == 0.0f && nn.z == 0.0f) {
      out[v] = 0.0f;
      continue;
    }
    V3 t, b;
    any_orthonormal_pair(nn, &t, &b);
    V3 o(pos[3 * v] + nn.x * eps, pos[3 * v + 1] + nn.y * eps, pos[3 * v + 2] + nn.z * eps);
    uint32_t h = hash32(v ^ 0x5bd1e995u);
    float rot = unit_f32(h);
    float jit = unit_f32(hash32(h));
    uint32_t hits = 0;
    for (uint32_t k = 0; k < n; ++k) {
      float u1 = std::min(((float)k + jit) / (float)n, 0.999999f);
      float x = (float)k * 0.618034f + rot;
      float u2 = x - std::trunc(x);
      float r = std::sqrt(u1);
      float phi = 6.28318530717958647692f * u2;
      float c = r * std::cos(phi), s = r * std::sin(phi), w = std::sqrt(1.0f - u1);
      orc::Ray ray;
      ray.o = o;
      ray.d = V3((t.x * c + b.x * s) + nn.x * w, (t.y * c + b.y * s) + nn.y * w, (t.z * c + b.z * s) + nn.z * w);
      if (bvh.occluded(ray, distance)) ++hits;
    }
    out[v] = (float)hits / (float)n;
  }
}

// cavity.rs:137-236.
void oracle_concavity(const float* pos, uint32_t nv, const float* normals, const uint32_t* tris, uint32_t nt,
                      float radius, float* out) {
  if (nv == 0 || !(radius > 0.0f)) {
    for (uint32_t v = 0; v < nv; ++v) out[v] = 0.0f;
    return;
  }
  std::vector<double> varea(nv, 0.0);
  for (uint32_t f = 0; f < nt; ++f) {
    const uint32_t* t = tris + 3 * (size_t)f;
    double ar = 0.5 * dlen(dcross(dsub(dd(pos + 3 * t[1]), dd(pos + 3 * t[0])),
                                  dsub(dd(pos + 3 * t[2]), dd(pos + 3 * t[0])))) / 3.0;
    for (int k = 0; k < 3; ++k) varea[t[k]] += ar;
  }
  float lo[3] = {INFINITY, INFINITY, INFINITY};
  for (uint32_t v = 0; v < nv; ++v)
    for (int k = 0; k < 3; ++k) lo[k] = std::min(lo[k], pos[3 * (size_t)v + k]);
  double h = (double)radius / 2.0;
  const uint64_t M = (1ull << 21) - 1;
  auto cellc = [&](const float* p, int k) -> uint64_t {
    double q = std::max(((double)p[k] - (double)lo[k]) / h, 0.0);
    uint64_t c = q >= 1.8446744073709552e19 ? ~0ull : (uint64_t)q;
    return std::min(c, M);
  };
  std::vector<std::pair<uint64_t, uint32_t>> order;
  for (uint32_t v = 0; v < nv; ++v) {
    const float* p = pos + 3 * (size_t)v;
    order.push_back({(cellc(p, 0) << 42) | (cellc(p, 1) << 21) | cellc(p, 2), v});
  }
  std::sort(order.begin(), order.end());
  std::vector<uint64_t> ckey;
  std::vector<double> cm;
  std::vector<D> cp, cn;
  std::vector<uint32_t> cell_of(nv);
  for (size_t i = 0; i < order.size();) {
    size_t e = i;
    double m = 0.0;
    D p{0, 0, 0}, n{0, 0, 0};
    while (e < order.size() && order[e].first == order[i].first) {
      uint32_t v = order[e].second;
      double w = std::max(varea[v], 1e-12);
      m += w;
      p.x += pos[3 * v] * w;
      p.y += pos[3 * v + 1] * w;
      p.z += pos[3 * v + 2] * w;
      n.x += normals[3 * v] * w;
      n.y += normals[3 * v + 1] * w;
      n.z += normals[3 * v + 2] * w;
      cell_of[v] = (uint32_t)ckey.size();
      ++e;
    }
    ckey.push_back(order[i].first);
    cm.push_back(m);
    cp.push_back({p.x / m, p.y / m, p.z / m});
    cn.push_back(dnorm0(n));
    i = e;
  }
  int64_t reach = (int64_t)std::ceil((double)radius / h) + 1;
  double max_d = (double)radius + 2.0 * h;
  double r2 = (double)radius * (double)radius;
  double inv2s2 = 1.0 / (2.0 * (0.5 * (double)radius) * (0.5 * (double)radius));
  std::vector<std::vector<uint32_t>> nbr(ckey.size());
  for (size_t ci = 0; ci < ckey.size(); ++ci) {
    int64_t bx = (int64_t)(ckey[ci] >> 42), by = (int64_t)((ckey[ci] >> 21) & M), bz = (int64_t)(ckey[ci] & M);
    for (int64_t dx = -reach; dx <= reach; ++dx)
      for (int64_t dy = -reach; dy <= reach; ++dy)
        for (int64_t dz = -reach; dz <= reach; ++dz) {
          int64_t x = bx + dx, y = by + dy, z = bz + dz;
          if (x < 0 || y < 0 || z < 0 || x > (int64_t)M || y > (int64_t)M || z > (int64_t)M) continue;
          uint64_t key = ((uint64_t)x << 42) | ((uint64_t)y << 21) | (uint64_t)z;
          auto it = std::lower_bound(ckey.begin(), ckey.end(), key);
          if (it == ckey.end() || *it != key) continue;
          size_t j = (size_t)(it - ckey.begin());
          if (dlen(dsub(cp[j], cp[ci])) <= max_d) nbr[ci].push_back((uint32_t)j);
        }
  }
  for (uint32_t v = 0; v < nv; ++v) {
    D p = dd(pos + 3 * (size_t)v);
    D n = dnorm0(dd(normals + 3 * (size_t)v));
    if (n.x == 0.0 && n.y == 0.0 && n.z == 0.0) {
      out[v] = 0.0f;
      continue;
    }
    double sw = 0.0, st = 0.0;
    D sd{0, 0, 0};
    for (uint32_t j : nbr[cell_of[v]]) {
      D d = dsub(cp[j], p);
      double dist2 = ddot(d, d);
      if (dist2 > r2 || ddot(cn[j], n) < -0.5) continue;
      double w = cm[j] * std::exp(-dist2 * inv2s2);
      sw += w;
      sd.x += d.x * w;
      sd.y += d.y * w;
      sd.z += d.z * w;
      double dn = ddot(d, n);
      st += w * (dist2 - dn * dn);
    }
    if (sw <= 0.0 || st <= 1e-18) {
      out[v] = 0.0f;
      continue;
    }
    double hgt = ddot(D{sd.x / sw, sd.y / sw, sd.z / sw}, n);
    double mean_curv = 2.0 * hgt / (st / sw);
    out[v] = (float)std::min(std::max(mean_curv * (double)radius, -4.0), 4.0);
  }
}

// cavity.rs:241-299 with weld.rs:92 at eps 0 (exact duplicates, -0 == +0,
// unique ids in first-occurrence order).
void oracle_smooth(const float* pos, uint32_t nv, const uint32_t* tris, uint32_t nt, float* values,
                   uint32_t iterations, float lambda) {
  if (nv == 0) return;
  std::map<std::array<uint32_t, 3>, uint32_t> first;
  std::vector<uint32_t> canon(nv);
  uint32_t nc = 0;
  for (uint32_t v = 0; v < nv; ++v) {
    std::array<uint32_t, 3> k;
    for (int c = 0; c < 3; ++c) {
      float f = pos[3 * (size_t)v + c] + 0.0f;
      std::memcpy(&k[c], &f, 4);
    }
    auto it = first.find(k);
    if (it == first.end()) {
      first[k] = nc;
      canon[v] = nc++;
    } else {
      canon[v] = it->second;
    }
  }
  std::vector<double> sum(nc, 0.0);
  std::vector<uint32_t> cnt(nc, 0);
  for (uint32_t v = 0; v < nv; ++v) {
    sum[canon[v]] += values[v];
    cnt[canon[v]]++;
  }
  std::vector<float> x(nc);
  for (uint32_t c = 0; c < nc; ++c) x[c] = (float)(sum[c] / (double)std::max(cnt[c], 1u));
  if (iterations > 0 && nt > 0) {
    std::vector<std::vector<uint32_t>> adj(nc);
    std::vector<uint64_t> edges;
    for (uint32_t f = 0; f < nt; ++f) {
      uint64_t c[3] = {canon[tris[3 * f]], canon[tris[3 * f + 1]], canon[tris[3 * f + 2]]};
      for (int k = 0; k < 3; ++k) {
        edges.push_back((c[k] << 32) | c[(k + 1) % 3]);
        edges.push_back((c[(k + 1) % 3] << 32) | c[k]);
      }
    }
    std::sort(edges.begin(), edges.end());
    edges.erase(std::unique(edges.begin(), edges.end()), edges.end());
    for (uint64_t e : edges) adj[e >> 32].push_back((uint32_t)e);
    std::vector<float> y(nc);
    for (uint32_t it = 0; it < iterations; ++it) {
      for (uint32_t i = 0; i < nc; ++i) {
        if (adj[i].empty()) {
          y[i] = x[i];
          continue;
        }
        float s = 0.0f;
        for (uint32_t j : adj[i])
          if (j != i) s += x[j];
        y[i] = x[i] + lambda * (s / (float)adj[i].size() - x[i]);
      }
      std::swap(x, y);
    }
  }
  for (uint32_t v = 0; v < nv; ++v) values[v] = x[canon[v]];
}

// cavity.rs:52-78: patina_mask.  normals may be NULL (smooth normals are
// computed, cavity.rs:80-86).
void oracle_patina_mask(const float* pos, uint32_t nv, const float* normals, const uint32_t* tris, uint32_t nt,
                        uint32_t ao_samples, float ao_distance, float curvature_radius, float concavity_weight,
                        uint32_t smooth_iterations, float* out) {
  if (nv == 0 || nt == 0) {
    for (uint32_t v = 0; v < nv; ++v) out[v] = 0.0f;
    return;
  }
  std::vector<float> nrm(3 * (size_t)nv);
  if (normals)
    std::memcpy(nrm.data(), normals, nrm.size() * sizeof(float));
  else
    oracle_smooth_vertex_normals(pos, nv, tris, nt, nrm.data());
  std::vector<float> ao(nv, 0.0f), cav(nv, 0.0f);
  if (ao_samples > 0 && ao_distance > 0.0f)
    oracle_ambient_occlusion(pos, nv, nrm.data(), tris, nt, ao_samples, ao_distance, ao.data());
  float w = std::min(std::max(concavity_weight, 0.0f), 1.0f);
  if (w > 0.0f && curvature_radius > 0.0f) oracle_concavity(pos, nv, nrm.data(), tris, nt, curvature_radius, cav.data());
  for (uint32_t v = 0; v < nv; ++v) {
    float at = smoothstep(0.04f, 0.55f, ao[v]);
    float ct = smoothstep(0.02f, 0.5f, cav[v]);
    out[v] = smoothstep(0.05f, 0.9f, (1.0f - w) * at + w * ct);
  }
  oracle_smooth(pos, nv, tris, nt, out, smooth_iterations, 0.5f);
  for (uint32_t v = 0; v < nv; ++v) out[v] = std::min(std::max(out[v], 0.0f), 1.0f);
}

}  // extern "C"
