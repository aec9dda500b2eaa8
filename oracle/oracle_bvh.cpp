// oracle_bvh.cpp — CPU restatement of argent's BVH build and traversal
// (crates/argent-core/src/bvh.rs).  TEST INFRASTRUCTURE ONLY.
//
// The build reproduces argent's node layout and leaf order exactly (same
// binned SAH, same in-place partition, same DFS layout and 4-wide collapse),
// so closest-hit ties resolve the way argent resolves them.
#include "oracle_bvh.h"

#include <algorithm>

namespace orc {

const SobolDirs SOBOL_DIRS;

namespace {

const int BINS = 16;      // bvh.rs:101
const size_t MAX_LEAF = 4;  // bvh.rs:102

struct BuildPrim {
  Aabb bounds;
  V3 centroid;
  uint32_t id;
};

struct Sub {
  std::vector<Node> nodes;
  std::vector<uint32_t> prims;
};

Node make_node(const Aabb& b, uint32_t index, uint32_t count) {
  Node n;
  n.min[0] = b.min.x;
  n.min[1] = b.min.y;
  n.min[2] = b.min.z;
  n.max[0] = b.max.x;
  n.max[1] = b.max.y;
  n.max[2] = b.max.z;
  n.index = index;
  n.count = count;
  return n;
}

// bvh.rs:412-417
Sub leaf(BuildPrim* prims, size_t n, const Aabb& bounds) {
  Sub s;
  s.nodes.push_back(make_node(bounds, 0, (uint32_t)n));
  for (size_t i = 0; i < n; ++i) s.prims.push_back(prims[i].id);
  return s;
}

Sub build_rec(BuildPrim* prims, size_t n);

// bvh.rs:497-533
Sub combine(const Aabb& bounds, BuildPrim* prims, size_t n, size_t mid) {
  Sub ls = build_rec(prims, mid);
  Sub rs = build_rec(prims + mid, n - mid);
  Sub out;
  out.nodes.reserve(1 + ls.nodes.size() + rs.nodes.size());
  out.nodes.push_back(make_node(bounds, 1, 0));
  uint32_t l_rest_base = 3;
  uint32_t r_rest_base = l_rest_base + ((uint32_t)ls.nodes.size() - 1);
  auto remap = [](const Node& node, uint32_t base_rest, uint32_t prim_off) {
    Node nd = node;
    if (nd.count > 0)
      nd.index += prim_off;
    else
      nd.index = base_rest + (nd.index - 1);
    return nd;
  };
  uint32_t lp = 0;
  uint32_t rp = (uint32_t)ls.prims.size();
  out.nodes.push_back(remap(ls.nodes[0], l_rest_base, lp));
  out.nodes.push_back(remap(rs.nodes[0], r_rest_base, rp));
  for (size_t i = 1; i < ls.nodes.size(); ++i) out.nodes.push_back(remap(ls.nodes[i], l_rest_base, lp));
  for (size_t i = 1; i < rs.nodes.size(); ++i) out.nodes.push_back(remap(rs.nodes[i], r_rest_base, rp));
  out.prims = std::move(ls.prims);
  out.prims.insert(out.prims.end(), rs.prims.begin(), rs.prims.end());
  return out;
}

// Rust `as usize` of an f32: saturating, NaN -> 0.
inline size_t sat_usize(float f) {
  if (!(f > 0.0f)) return 0;
  if (f >= 1.8446744e19f) return (size_t)-1;
  return (size_t)f;
}

// bvh.rs:419-495
Sub build_rec(BuildPrim* prims, size_t n) {
  Aabb bounds = Aabb::empty();
  Aabb cb = Aabb::empty();
  for (size_t i = 0; i < n; ++i) {
    bounds = bounds.uni(prims[i].bounds);
    cb.grow(prims[i].centroid);
  }
  if (n <= MAX_LEAF) return leaf(prims, n, bounds);
  V3 ext = cb.max - cb.min;
  int axis = (ext.x >= ext.y && ext.x >= ext.z) ? 0 : (ext.y >= ext.z ? 1 : 2);
  float lo = cb.min[axis];
  float span = ext[axis];
  if (span <= 1e-12f) return combine(bounds, prims, n, n / 2);
  Aabb bin_b[BINS];
  size_t bin_n[BINS];
  for (int i = 0; i < BINS; ++i) {
    bin_b[i] = Aabb::empty();
    bin_n[i] = 0;
  }
  float k = (float)BINS / span;
  auto bin_of = [&](float c) { return std::min(sat_usize((c - lo) * k), (size_t)(BINS - 1)); };
  for (size_t i = 0; i < n; ++i) {
    size_t b = bin_of(prims[i].centroid[axis]);
    bin_n[b] += 1;
    bin_b[b] = bin_b[b].uni(prims[i].bounds);
  }
  float left_area[BINS - 1];
  size_t left_n[BINS - 1];
  Aabb acc = Aabb::empty();
  size_t cnt = 0;
  for (int i = 0; i < BINS - 1; ++i) {
    acc = acc.uni(bin_b[i]);
    cnt += bin_n[i];
    left_area[i] = cnt > 0 ? acc.area() : 0.0f;
    left_n[i] = cnt;
  }
  float best_cost = INFINITY;
  size_t best_bin = 0;
  acc = Aabb::empty();
  cnt = 0;
  for (int i = BINS - 1; i >= 1; --i) {
    acc = acc.uni(bin_b[i]);
    cnt += bin_n[i];
    size_t ln = left_n[i - 1];
    if (ln == 0 || cnt == 0) continue;
    float cost = left_area[i - 1] * (float)ln + acc.area() * (float)cnt;
    if (cost < best_cost) {
      best_cost = cost;
      best_bin = (size_t)i;
    }
  }
  float leaf_cost = bounds.area() * (float)n;
  if (!std::isfinite(best_cost) || (n <= 16 && best_cost >= leaf_cost)) {
    if (n <= 16) return leaf(prims, n, bounds);
    return combine(bounds, prims, n, n / 2);
  }
  size_t split_bin = best_bin;
  size_t i = 0, j = n;
  while (i < j) {
    if (bin_of(prims[i].centroid[axis]) < split_bin) {
      i += 1;
    } else {
      j -= 1;
      std::swap(prims[i], prims[j]);
    }
  }
  size_t mid = (i == 0 || i == n) ? n / 2 : i;
  return combine(bounds, prims, n, mid);
}

float node_area(const Node& n) {
  float e0 = n.max[0] - n.min[0], e1 = n.max[1] - n.min[1], e2 = n.max[2] - n.min[2];
  return e0 * e1 + e1 * e2 + e2 * e0;
}

// bvh.rs:303-378
uint32_t collapse_build(const std::vector<Node>& nodes, uint32_t root, std::vector<Node4>& wide) {
  uint32_t me = (uint32_t)wide.size();
  Node4 blank;
  for (int c = 0; c < 4; ++c) {
    blank.min_x[c] = blank.min_y[c] = blank.min_z[c] = INFINITY;
    blank.max_x[c] = blank.max_y[c] = blank.max_z[c] = -INFINITY;
    blank.child[c] = EMPTY_CHILD;
    blank.count[c] = 0;
  }
  wide.push_back(blank);
  const Node& r = nodes[root];
  std::vector<uint32_t> kids;
  if (r.count > 0)
    kids.push_back(root);
  else {
    kids.push_back(r.index);
    kids.push_back(r.index + 1);
  }
  while (kids.size() < 4) {
    int best = -1;
    float best_a = 0.0f;
    for (size_t i = 0; i < kids.size(); ++i) {
      const Node& n = nodes[kids[i]];
      if (n.count == 0) {
        float a = node_area(n);
        if (best < 0 || a > best_a) {
          best = (int)i;
          best_a = a;
        }
      }
    }
    if (best < 0) break;
    Node n = nodes[kids[best]];
    kids[best] = kids.back();  // swap_remove
    kids.pop_back();
    kids.push_back(n.index);
    kids.push_back(n.index + 1);
  }
  Node4 node = wide[me];
  for (size_t c = 0; c < kids.size(); ++c) {
    const Node& n = nodes[kids[c]];
    node.min_x[c] = n.min[0];
    node.min_y[c] = n.min[1];
    node.min_z[c] = n.min[2];
    node.max_x[c] = n.max[0];
    node.max_y[c] = n.max[1];
    node.max_z[c] = n.max[2];
    if (n.count > 0) {
      node.child[c] = LEAF | n.index;
      node.count[c] = n.count;
    } else {
      node.child[c] = 0xffffffffu - 1;
    }
  }
  wide[me] = node;
  for (size_t c = 0; c < kids.size(); ++c) {
    if (nodes[kids[c]].count == 0) {
      uint32_t w = collapse_build(nodes, kids[c], wide);
      wide[me].child[c] = w;
    }
  }
  return me;
}

// bvh.rs:280-299, with glam's SSE min/max semantics.
inline uint32_t slab4(const Node4& n, V3 o, V3 inv, float t_max, float tmin_out[4]) {
  uint32_t mask = 0;
  for (int c = 0; c < 4; ++c) {
    float tx0 = (n.min_x[c] - o.x) * inv.x;
    float tx1 = (n.max_x[c] - o.x) * inv.x;
    float ty0 = (n.min_y[c] - o.y) * inv.y;
    float ty1 = (n.max_y[c] - o.y) * inv.y;
    float tz0 = (n.min_z[c] - o.z) * inv.z;
    float tz1 = (n.max_z[c] - o.z) * inv.z;
    float tmin = sse_max(sse_max(sse_max(sse_min(tx0, tx1), sse_min(ty0, ty1)), sse_min(tz0, tz1)), 0.0f);
    float tmax = sse_min(sse_min(sse_min(sse_max(tx0, tx1), sse_max(ty0, ty1)), sse_max(tz0, tz1)), t_max);
    tmin_out[c] = tmin;
    if (tmin <= tmax) mask |= 1u << c;
  }
  return mask;
}

}  // namespace

Bvh Bvh::build(const float* positions, const uint32_t* triangles, uint32_t nt) {
  auto p = [&](uint32_t i) { return V3(positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]); };
  std::vector<BuildPrim> prims(nt);
  for (uint32_t i = 0; i < nt; ++i) {
    Aabb b = Aabb::empty();
    b.grow(p(triangles[3 * i]));
    b.grow(p(triangles[3 * i + 1]));
    b.grow(p(triangles[3 * i + 2]));
    prims[i].centroid = b.centroid();
    prims[i].bounds = b;
    prims[i].id = i;
  }
  Bvh bvh;
  Sub sub;
  if (prims.empty()) {
    Node z;
    std::memset(&z, 0, sizeof(z));
    sub.nodes.push_back(z);
  } else {
    sub = build_rec(prims.data(), prims.size());
  }
  bvh.tris.resize(sub.prims.size());
  for (size_t i = 0; i < sub.prims.size(); ++i) {
    const uint32_t* t = &triangles[3 * (size_t)sub.prims[i]];
    V3 v0 = p(t[0]);
    bvh.tris[i].v0 = v0;
    bvh.tris[i].e1 = p(t[1]) - v0;
    bvh.tris[i].e2 = p(t[2]) - v0;
  }
  // argent's collapse indexes past the end for an empty piece; the oracle
  // simply keeps no wide nodes (every query misses, bvh.rs:160, 217).
  if (!prims.empty()) collapse_build(sub.nodes, 0, bvh.wide);
  bvh.nodes = std::move(sub.nodes);
  bvh.prim_ids = std::move(sub.prims);
  return bvh;
}

Aabb Bvh::bounds() const {
  Aabb a;
  a.min = V3(nodes[0].min[0], nodes[0].min[1], nodes[0].min[2]);
  a.max = V3(nodes[0].max[0], nodes[0].max[1], nodes[0].max[2]);
  return a;
}

// bvh.rs:159-212
bool Bvh::intersect(const Ray& ray, float t_max, TriHit* out, uint32_t* max_stack) const {
  if (tris.empty()) return false;
  V3 inv = V3(1.0f / ray.d.x, 1.0f / ray.d.y, 1.0f / ray.d.z);
  float best_t = t_max;
  bool have = false;
  uint32_t bi = 0;
  float bu = 0, bv = 0;
  struct Entry {
    uint32_t entry, count;
    float tn;
  };
  Entry stack[192];
  size_t sp = 0;
  stack[sp++] = Entry{0, 0, 0.0f};
  uint32_t deepest = 1;
  while (sp > 0) {
    sp -= 1;
    Entry e = stack[sp];
    if (e.tn > best_t) continue;
    if (e.entry & LEAF) {
      uint32_t start = e.entry & ~LEAF;
      for (uint32_t i = start; i < start + e.count; ++i) {
        float t, u, v;
        if (tri_intersect(tris[i], ray, best_t, &t, &u, &v)) {
          best_t = t;
          have = true;
          bi = i;
          bu = u;
          bv = v;
        }
      }
      continue;
    }
    const Node4& n = wide[e.entry];
    float tmin[4];
    uint32_t mask = slab4(n, ray.o, inv, best_t, tmin);
    int order_c[4];
    float order_t[4];
    int k = 0;
    for (int c = 0; c < 4; ++c) {
      if (mask & (1u << c)) {
        float t = tmin[c];
        int j = k;
        while (j > 0 && order_t[j - 1] < t) {
          order_c[j] = order_c[j - 1];
          order_t[j] = order_t[j - 1];
          j -= 1;
        }
        order_c[j] = c;
        order_t[j] = t;
        k += 1;
      }
    }
    for (int q = 0; q < k; ++q) {
      if (sp >= 192) {  // argent would panic on the index; the oracle stops here
        if (max_stack) *max_stack = 0xffffffffu;
        return false;
      }
      stack[sp++] = Entry{n.child[order_c[q]], n.count[order_c[q]], order_t[q]};
    }
    if (sp > deepest) deepest = (uint32_t)sp;
  }
  if (max_stack && *max_stack != 0xffffffffu && deepest > *max_stack) *max_stack = deepest;
  if (!have) return false;
  out->t = best_t;
  out->u = bu;
  out->v = bv;
  out->prim = prim_ids[bi];
  return true;
}

// bvh.rs:216-247
bool Bvh::occluded(const Ray& ray, float t_max) const {
  if (tris.empty()) return false;
  V3 inv = V3(1.0f / ray.d.x, 1.0f / ray.d.y, 1.0f / ray.d.z);
  struct Entry {
    uint32_t entry, count;
  };
  Entry stack[192];
  stack[0] = Entry{0, 0};
  size_t sp = 1;
  while (sp > 0) {
    sp -= 1;
    Entry e = stack[sp];
    if (e.entry & LEAF) {
      uint32_t start = e.entry & ~LEAF;
      for (uint32_t i = start; i < start + e.count; ++i) {
        float t, u, v;
        if (tri_intersect(tris[i], ray, t_max, &t, &u, &v)) return true;
      }
      continue;
    }
    const Node4& n = wide[e.entry];
    float tmin[4];
    uint32_t mask = slab4(n, ray.o, inv, t_max, tmin);
    for (int c = 0; c < 4; ++c) {
      if (mask & (1u << c)) {
        if (sp >= 192) return false;
        stack[sp++] = Entry{n.child[c], n.count[c]};
      }
    }
  }
  return false;
}

// bvh.rs:250-275 (argent's test-only binary traversal) and slab :382-388.
bool Bvh::intersect_binary(const Ray& ray, float t_max, TriHit* out) const {
  if (tris.empty()) return false;
  V3 inv = V3(1.0f / ray.d.x, 1.0f / ray.d.y, 1.0f / ray.d.z);
  float best_t = t_max;
  bool have = false;
  uint32_t bi = 0;
  float bu = 0, bv = 0;
  std::vector<uint32_t> stack{0};
  while (!stack.empty()) {
    uint32_t idx = stack.back();
    stack.pop_back();
    const Node& node = nodes[idx];
    V3 mn(node.min[0], node.min[1], node.min[2]), mx(node.max[0], node.max[1], node.max[2]);
    V3 t0 = (mn - ray.o) * inv;
    V3 t1 = (mx - ray.o) * inv;
    float tmin = rmax(max_element(vmin(t0, t1)), 0.0f);
    float tmax = rmin(min_element(vmax(t0, t1)), best_t);
    if (!(tmin <= tmax)) continue;
    if (node.count > 0) {
      for (uint32_t i = node.index; i < node.index + node.count; ++i) {
        float t, u, v;
        if (tri_intersect(tris[i], ray, best_t, &t, &u, &v)) {
          best_t = t;
          have = true;
          bi = i;
          bu = u;
          bv = v;
        }
      }
    } else {
      stack.push_back(node.index);
      stack.push_back(node.index + 1);
    }
  }
  if (!have) return false;
  out->t = best_t;
  out->u = bu;
  out->v = bv;
  out->prim = prim_ids[bi];
  return true;
}

}  // namespace orc

// ------------------------------------------------------------------ C API
#include <omp.h>

#include "oracle_api.h"

struct oracle_bvh {
  orc::Bvh bvh;
  uint32_t max_stack = 0;
};

namespace {
inline orc::Ray to_ray(const ArgentRay& r) {
  return orc::Ray{orc::V3(r.o[0], r.o[1], r.o[2]), orc::V3(r.d[0], r.d[1], r.d[2])};
}
inline int nthreads(int t) { return t > 0 ? t : omp_get_max_threads(); }
}  // namespace

extern "C" {

oracle_bvh* oracle_bvh_create(const float* positions, uint32_t nv, const uint32_t* tris, uint32_t nt) {
  (void)nv;
  oracle_bvh* b = new oracle_bvh();
  b->bvh = orc::Bvh::build(positions, tris, nt);
  return b;
}

void oracle_bvh_destroy(oracle_bvh* b) { delete b; }

void oracle_bvh_intersect(const oracle_bvh* b, const ArgentRay* rays, uint64_t n, ArgentHit* hits, int threads) {
  uint32_t deepest = 0;
#pragma omp parallel num_threads(nthreads(threads))
  {
    uint32_t local = 0;
#pragma omp for schedule(dynamic, 4096)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
      orc::TriHit h;
      if (b->bvh.intersect(to_ray(rays[i]), rays[i].tmax, &h, &local)) {
        hits[i] = ArgentHit{h.t, h.u, h.v, h.prim};
      } else {
        hits[i] = ArgentHit{0.0f, 0.0f, 0.0f, ARGENT_NO_HIT};
      }
    }
#pragma omp critical
    if (local > deepest) deepest = local;
  }
  oracle_bvh* mb = const_cast<oracle_bvh*>(b);
  if (deepest > mb->max_stack) mb->max_stack = deepest;
}

void oracle_bvh_occluded(const oracle_bvh* b, const ArgentRay* rays, uint64_t n, uint8_t* occ, int threads) {
#pragma omp parallel for schedule(dynamic, 4096) num_threads(nthreads(threads))
  for (int64_t i = 0; i < (int64_t)n; ++i) occ[i] = b->bvh.occluded(to_ray(rays[i]), rays[i].tmax) ? 1 : 0;
}

void oracle_bvh_intersect_binary(const oracle_bvh* b, const ArgentRay* rays, uint64_t n, ArgentHit* hits) {
  for (uint64_t i = 0; i < n; ++i) {
    orc::TriHit h;
    if (b->bvh.intersect_binary(to_ray(rays[i]), rays[i].tmax, &h))
      hits[i] = ArgentHit{h.t, h.u, h.v, h.prim};
    else
      hits[i] = ArgentHit{0.0f, 0.0f, 0.0f, ARGENT_NO_HIT};
  }
}

static inline orc::Tri make_tri(const float* p, const uint32_t* t) {
  orc::V3 v0(p[3 * t[0]], p[3 * t[0] + 1], p[3 * t[0] + 2]);
  orc::V3 v1(p[3 * t[1]], p[3 * t[1] + 1], p[3 * t[1] + 2]);
  orc::V3 v2(p[3 * t[2]], p[3 * t[2] + 1], p[3 * t[2] + 2]);
  return orc::Tri{v0, v1 - v0, v2 - v0};
}

// bvh.rs:560-570 (argent's brute-force test helper, returning the hit too)
void oracle_brute_intersect(const float* positions, const uint32_t* tris, uint32_t nt, const ArgentRay* rays,
                            uint64_t n, ArgentHit* hits, int threads) {
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads(threads))
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    orc::Ray r = to_ray(rays[i]);
    float best = rays[i].tmax;
    ArgentHit h{0.0f, 0.0f, 0.0f, ARGENT_NO_HIT};
    for (uint32_t k = 0; k < nt; ++k) {
      float t, u, v;
      if (orc::tri_intersect(make_tri(positions, &tris[3 * (size_t)k]), r, best, &t, &u, &v)) {
        best = t;
        h = ArgentHit{t, u, v, k};
      }
    }
    hits[i] = h;
  }
}

int oracle_tri_hit(const float* positions, const uint32_t* tris, uint32_t prim, const ArgentRay* r, float* t,
                   float* u, float* v) {
  return orc::tri_intersect(make_tri(positions, &tris[3 * (size_t)prim]), to_ray(*r), r->tmax, t, u, v) ? 1 : 0;
}

void oracle_bvh_stats(const oracle_bvh* b, uint64_t* binary_nodes, uint64_t* wide_nodes, uint32_t* max_stack) {
  *binary_nodes = b->bvh.nodes.size();
  *wide_nodes = b->bvh.wide.size();
  *max_stack = b->max_stack;
}

}  // extern "C"
