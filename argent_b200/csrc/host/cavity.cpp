// cavity.cpp — the host half of argent's per-vertex patina mask
// (crates/argent-mesh/src/cavity.rs): the concavity estimate, the Laplacian
// smoothing over welded positions, the smooth vertex normals used when a
// mesh has none, and the final contrast blend.  The ambient-occlusion half
// (48 any-hit rays per vertex) runs on the device (argent_gpu.cu,
// k_cavity_ao) over the uploaded piece's BVH.
#include "cavity.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <unordered_map>
#include <vector>

namespace argent {

namespace {

template <class F>
void parallel_for(size_t n, F f) {
  unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
  if (n < 4096 || nt == 1) {
    for (size_t i = 0; i < n; ++i) f(i);
    return;
  }
  std::atomic<size_t> next{0};
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nt; ++t)
    th.emplace_back([&] {
      for (;;) {
        size_t b = next.fetch_add(1024);
        if (b >= n) break;
        size_t e = std::min(n, b + 1024);
        for (size_t i = b; i < e; ++i) f(i);
      }
    });
  for (auto& t : th) t.join();
}

struct D3 {
  double x, y, z;
};
inline D3 d3(const float* p) { return {p[0], p[1], p[2]}; }
inline D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline D3 add(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline D3 mul(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline D3 cross(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double len(D3 a) { return std::sqrt(dot(a, a)); }
inline D3 normalize_or_zero(D3 a) {
  // glam DVec3::normalize_or_zero: scale by 1/length when that is finite and positive.
  double r = 1.0 / len(a);
  if (std::isfinite(r) && r > 0.0) return mul(a, r);
  return {0, 0, 0};
}

float smoothstep(float e0, float e1, float x) {
  float t = std::min(std::max((x - e0) / (e1 - e0), 0.0f), 1.0f);
  return t * t * (3.0f - 2.0f * t);
}

}  // namespace

// normals.rs:226-242 (face_normals: unit normal per face, zero when
// degenerate; angle-weighted accumulation in f64; [0, 0, 1] when nothing
// accumulates).
void smooth_vertex_normals(const float* pos, uint32_t nv, const uint32_t* tris, uint32_t nt, float* out) {
  std::vector<D3> acc(nv, D3{0, 0, 0});
  for (uint32_t f = 0; f < nt; ++f) {
    const uint32_t* t = tris + 3 * (size_t)f;
    D3 a = d3(pos + 3 * (size_t)t[0]), b = d3(pos + 3 * (size_t)t[1]), c = d3(pos + 3 * (size_t)t[2]);
    D3 n = cross(sub(b, a), sub(c, a));
    double l = len(n);
    float fn[3] = {0, 0, 0};
    if (l > 0.0) {
      fn[0] = (float)(n.x / l);
      fn[1] = (float)(n.y / l);
      fn[2] = (float)(n.z / l);
    }
    for (int k = 0; k < 3; ++k) {
      uint32_t v = t[k];
      D3 p = d3(pos + 3 * (size_t)v);
      D3 ea = sub(d3(pos + 3 * (size_t)t[(k + 1) % 3]), p);
      D3 eb = sub(d3(pos + 3 * (size_t)t[(k + 2) % 3]), p);
      double ang = std::atan2(len(cross(ea, eb)), dot(ea, eb));
      acc[v].x += ang * fn[0];
      acc[v].y += ang * fn[1];
      acc[v].z += ang * fn[2];
    }
  }
  for (uint32_t v = 0; v < nv; ++v) {
    double l = len(acc[v]);
    if (l > 1e-300) {
      out[3 * v] = (float)(acc[v].x / l);
      out[3 * v + 1] = (float)(acc[v].y / l);
      out[3 * v + 2] = (float)(acc[v].z / l);
    } else {
      out[3 * v] = 0.0f;
      out[3 * v + 1] = 0.0f;
      out[3 * v + 2] = 1.0f;
    }
  }
}

// cavity.rs:137-236: mean curvature x radius from area-weighted cell
// centroids within `radius` (cells of radius/2 on a 21-bit-per-axis grid).
void concavity(const float* pos, uint32_t nv, const uint32_t* tris, uint32_t nt, const float* normals, float radius,
               float* out) {
  if (nv == 0 || !(radius > 0.0f)) {
    std::fill(out, out + nv, 0.0f);
    return;
  }
  std::vector<double> varea(nv, 0.0);
  for (uint32_t f = 0; f < nt; ++f) {
    const uint32_t* t = tris + 3 * (size_t)f;
    D3 a = d3(pos + 3 * (size_t)t[0]), b = d3(pos + 3 * (size_t)t[1]), c = d3(pos + 3 * (size_t)t[2]);
    double ar = 0.5 * len(cross(sub(b, a), sub(c, a))) / 3.0;
    for (int k = 0; k < 3; ++k) varea[t[k]] += ar;
  }
  float lo[3] = {pos[0], pos[1], pos[2]};
  for (uint32_t v = 1; v < nv; ++v)
    for (int k = 0; k < 3; ++k) lo[k] = std::min(lo[k], pos[3 * (size_t)v + k]);
  D3 lod{lo[0], lo[1], lo[2]};
  double h = (double)radius / 2.0;
  const uint64_t M = (1ull << 21) - 1;
  auto key_of = [&](const float* p) -> uint64_t {
    // (p - lo) / h per axis; `x.max(0.0) as u64` truncates and saturates
    double qq[3] = {(d3(p).x - lod.x) / h, (d3(p).y - lod.y) / h, (d3(p).z - lod.z) / h};
    uint64_t c[3];
    for (int k = 0; k < 3; ++k) {
      double x = std::max(qq[k], 0.0);
      c[k] = x >= 18446744073709551615.0 ? ~0ull : (uint64_t)x;
      c[k] = std::min(c[k], M);
    }
    return (c[0] << 42) | (c[1] << 21) | c[2];
  };
  std::vector<std::pair<uint64_t, uint32_t>> order(nv);
  parallel_for(nv, [&](size_t i) { order[i] = {key_of(pos + 3 * i), (uint32_t)i}; });
  std::sort(order.begin(), order.end());
  struct Cell {
    uint64_t key;
    double m;
    D3 p, n;
  };
  std::vector<Cell> cells;
  std::vector<uint32_t> cell_of(nv, 0);
  for (size_t i = 0; i < order.size();) {
    uint64_t k = order[i].first;
    double m = 0.0;
    D3 p{0, 0, 0}, n{0, 0, 0};
    size_t e = i;
    while (e < order.size() && order[e].first == k) {
      uint32_t v = order[e].second;
      double w = std::max(varea[v], 1e-12);
      m += w;
      p = add(p, mul(d3(pos + 3 * (size_t)v), w));
      n = add(n, mul(d3(normals + 3 * (size_t)v), w));
      cell_of[v] = (uint32_t)cells.size();
      ++e;
    }
    cells.push_back({k, m, mul(p, 1.0 / m), normalize_or_zero(n)});
    i = e;
  }
  std::vector<uint64_t> keys(cells.size());
  for (size_t i = 0; i < cells.size(); ++i) keys[i] = cells[i].key;
  const int64_t reach = (int64_t)std::ceil((double)radius / h) + 1;
  const int64_t lim = (int64_t)M;
  const double max_d = (double)radius + 2.0 * h;
  std::vector<std::vector<uint32_t>> nbr(cells.size());
  parallel_for(cells.size(), [&](size_t ci) {
    const Cell& c = cells[ci];
    int64_t base[3] = {(int64_t)(c.key >> 42), (int64_t)((c.key >> 21) & M), (int64_t)(c.key & M)};
    for (int64_t dx = -reach; dx <= reach; ++dx)
      for (int64_t dy = -reach; dy <= reach; ++dy)
        for (int64_t dz = -reach; dz <= reach; ++dz) {
          int64_t q[3] = {base[0] + dx, base[1] + dy, base[2] + dz};
          if (q[0] < 0 || q[0] > lim || q[1] < 0 || q[1] > lim || q[2] < 0 || q[2] > lim) continue;
          uint64_t key = ((uint64_t)q[0] << 42) | ((uint64_t)q[1] << 21) | (uint64_t)q[2];
          auto it = std::lower_bound(keys.begin(), keys.end(), key);
          if (it != keys.end() && *it == key) {
            size_t j = (size_t)(it - keys.begin());
            if (len(sub(cells[j].p, c.p)) <= max_d) nbr[ci].push_back((uint32_t)j);
          }
        }
  });
  const double r2 = (double)radius * (double)radius;
  const double inv2s2 = 1.0 / (2.0 * std::pow(0.5 * (double)radius, 2));
  parallel_for(nv, [&](size_t v) {
    D3 p = d3(pos + 3 * v);
    D3 n = normalize_or_zero(d3(normals + 3 * v));
    if (n.x == 0.0 && n.y == 0.0 && n.z == 0.0) {
      out[v] = 0.0f;
      return;
    }
    double sw = 0.0, st = 0.0;
    D3 sd{0, 0, 0};
    for (uint32_t j : nbr[cell_of[v]]) {
      const Cell& c = cells[j];
      D3 d = sub(c.p, p);
      double dist2 = dot(d, d);
      if (dist2 > r2 || dot(c.n, n) < -0.5) continue;
      double w = c.m * std::exp(-dist2 * inv2s2);
      sw += w;
      sd = add(sd, mul(d, w));
      double dn = dot(d, n);
      st += w * (dist2 - dn * dn);
    }
    if (sw <= 0.0 || st <= 1e-18) {
      out[v] = 0.0f;
      return;
    }
    double hgt = dot(mul(sd, 1.0 / sw), n);
    double dt2 = st / sw;
    double mean_curv = 2.0 * hgt / dt2;
    out[v] = (float)std::min(std::max(mean_curv * (double)radius, -4.0), 4.0);
  });
}

// cavity.rs:241-299: x <- x + lambda (mean(neighbours) - x) over the edges
// of the mesh with exactly coincident positions welded (weld.rs:92, eps 0).
void smooth_values(const float* pos, uint32_t nv, const uint32_t* tris, uint32_t nt, float* values,
                   uint32_t iterations, float lambda) {
  if (nv == 0) return;
  // Weld: canonical index per position, -0.0 and +0.0 collide (weld.rs:148-151).
  struct Key {
    uint32_t a, b, c;
    bool operator==(const Key& o) const { return a == o.a && b == o.b && c == o.c; }
  };
  struct KeyHash {
    size_t operator()(const Key& k) const {
      return ((size_t)k.a * 0x9E3779B97F4A7C15ull) ^ ((size_t)k.b * 0xC2B2AE3D27D4EB4Full) ^ (size_t)k.c;
    }
  };
  auto bits = [](float x) {
    float y = x + 0.0f;
    uint32_t u;
    std::memcpy(&u, &y, 4);
    return u;
  };
  // Canonical indices in first-occurrence order, as weld.rs:219-233 numbers
  // its unique positions (the order fixes the summation order below).
  std::vector<std::pair<Key, uint32_t>> ks(nv);
  for (uint32_t v = 0; v < nv; ++v)
    ks[v] = {Key{bits(pos[3 * (size_t)v]), bits(pos[3 * (size_t)v + 1]), bits(pos[3 * (size_t)v + 2])}, v};
  std::sort(ks.begin(), ks.end(), [](const std::pair<Key, uint32_t>& x, const std::pair<Key, uint32_t>& y) {
    if (x.first.a != y.first.a) return x.first.a < y.first.a;
    if (x.first.b != y.first.b) return x.first.b < y.first.b;
    if (x.first.c != y.first.c) return x.first.c < y.first.c;
    return x.second < y.second;
  });
  std::vector<uint32_t> head(nv);
  for (uint32_t i = 0, g = 0; i < nv; ++i) {
    if (i > 0 && !(ks[i].first == ks[i - 1].first)) g = i;
    head[ks[i].second] = ks[g].second;  // smallest vertex index of the run
  }
  std::vector<uint32_t> canon(nv);
  uint32_t nc = 0;
  for (uint32_t v = 0; v < nv; ++v) canon[v] = head[v] == v ? nc++ : canon[head[v]];
  std::vector<double> sum(nc, 0.0);
  std::vector<uint32_t> cnt(nc, 0);
  for (uint32_t v = 0; v < nv; ++v) {
    sum[canon[v]] += values[v];
    cnt[canon[v]] += 1;
  }
  std::vector<float> x(nc);
  for (uint32_t c = 0; c < nc; ++c) x[c] = (float)(sum[c] / (double)std::max(cnt[c], 1u));
  if (iterations > 0 && nt > 0) {
    std::vector<uint64_t> edges;
    edges.reserve(6 * (size_t)nt);
    for (uint32_t f = 0; f < nt; ++f) {
      uint64_t c0 = canon[tris[3 * (size_t)f]], c1 = canon[tris[3 * (size_t)f + 1]], c2 = canon[tris[3 * (size_t)f + 2]];
      edges.push_back((c0 << 32) | c1);
      edges.push_back((c1 << 32) | c0);
      edges.push_back((c1 << 32) | c2);
      edges.push_back((c2 << 32) | c1);
      edges.push_back((c2 << 32) | c0);
      edges.push_back((c0 << 32) | c2);
    }
    std::sort(edges.begin(), edges.end());
    edges.erase(std::unique(edges.begin(), edges.end()), edges.end());
    std::vector<uint32_t> off(nc + 1, 0);
    for (uint64_t e : edges) off[(e >> 32) + 1] += 1;
    for (uint32_t i = 0; i < nc; ++i) off[i + 1] += off[i];
    std::vector<uint32_t> nb(edges.size());
    for (size_t i = 0; i < edges.size(); ++i) nb[i] = (uint32_t)edges[i];
    std::vector<float> y(x);
    for (uint32_t it = 0; it < iterations; ++it) {
      parallel_for(nc, [&](size_t i) {
        uint32_t a = off[i], b = off[i + 1];
        float xi = x[i];
        if (b > a) {
          float s = 0.0f;
          for (uint32_t k = a; k < b; ++k)
            if (nb[k] != i) s += x[nb[k]];
          float m = s / (float)(b - a);
          y[i] = xi + lambda * (m - xi);
        } else {
          y[i] = xi;
        }
      });
      std::swap(x, y);
    }
  }
  for (uint32_t v = 0; v < nv; ++v) values[v] = x[canon[v]];
}

// cavity.rs:52-78: contrast-shaped blend of AO and concavity, smoothed,
// clamped to [0, 1].
void patina_blend(const float* pos, uint32_t nv, const uint32_t* tris, uint32_t nt, const float* ao, const float* cav,
                  float concavity_weight, uint32_t smooth_iterations, float* out) {
  float w = std::min(std::max(concavity_weight, 0.0f), 1.0f);
  for (uint32_t v = 0; v < nv; ++v) {
    float at = smoothstep(0.04f, 0.55f, ao[v]);
    float ct = smoothstep(0.02f, 0.5f, cav[v]);
    out[v] = smoothstep(0.05f, 0.9f, (1.0f - w) * at + w * ct);
  }
  smooth_values(pos, nv, tris, nt, out, smooth_iterations, 0.5f);
  for (uint32_t v = 0; v < nv; ++v) out[v] = std::min(std::max(out[v], 0.0f), 1.0f);
}

}  // namespace argent
