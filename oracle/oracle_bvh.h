// oracle_bvh.h — CPU restatement of argent's BVH (crates/argent-core/src/bvh.rs).
// TEST INFRASTRUCTURE ONLY (see oracle_core.h).
#pragma once
#include <cstdint>
#include <vector>

#include "oracle_core.h"

namespace orc {

// bvh.rs:11-42
struct Aabb {
  V3 min, max;
  static Aabb empty() {
    Aabb a;
    a.min = V3::splat(INFINITY);
    a.max = V3::splat(-INFINITY);
    return a;
  }
  void grow(V3 p) {
    min = vmin(min, p);
    max = vmax(max, p);
  }
  Aabb uni(const Aabb& o) const {
    Aabb r;
    r.min = vmin(min, o.min);
    r.max = vmax(max, o.max);
    return r;
  }
  float area() const {
    V3 e = vmax(max - min, V3(0, 0, 0));
    return 2.0f * (e.x * e.y + e.y * e.z + e.z * e.x);
  }
  V3 centroid() const { return (min + max) * 0.5f; }
};

// bvh.rs:44-53
struct Node {
  float min[3];
  uint32_t index;
  float max[3];
  uint32_t count;
};

// bvh.rs:55-61
struct Tri {
  V3 v0, e1, e2;
};

// bvh.rs:82-96 (SoA 4-wide node)
struct Node4 {
  float min_x[4], min_y[4], min_z[4], max_x[4], max_y[4], max_z[4];
  uint32_t child[4];
  uint32_t count[4];
};

static const uint32_t LEAF = 1u << 31;
static const uint32_t EMPTY_CHILD = 0xffffffffu;

struct TriHit {
  float t, u, v;
  uint32_t prim;
};

struct Bvh {
  std::vector<Node> nodes;
  std::vector<Node4> wide;
  std::vector<Tri> tris;
  std::vector<uint32_t> prim_ids;

  static Bvh build(const float* positions, const uint32_t* triangles, uint32_t nt);
  bool intersect(const Ray& ray, float t_max, TriHit* out, uint32_t* max_stack = nullptr) const;
  bool occluded(const Ray& ray, float t_max) const;
  bool intersect_binary(const Ray& ray, float t_max, TriHit* out) const;
  Aabb bounds() const;
};

// bvh.rs:391-410 (Moller-Trumbore, argent's operation order)
static inline bool tri_intersect(const Tri& tri, const Ray& ray, float t_max, float* t_out, float* u_out,
                                 float* v_out) {
  V3 p = cross(ray.d, tri.e2);
  float det = dot(tri.e1, p);
  if (std::fabs(det) < 1e-14f) return false;
  float inv_det = 1.0f / det;
  V3 s = ray.o - tri.v0;
  float u = dot(s, p) * inv_det;
  if (!(u >= 0.0f && u <= 1.0f)) return false;
  V3 q = cross(s, tri.e1);
  float v = dot(ray.d, q) * inv_det;
  if (v < 0.0f || u + v > 1.0f) return false;
  float t = dot(tri.e2, q) * inv_det;
  if (t > 1e-7f && t < t_max) {
    *t_out = t;
    *u_out = u;
    *v_out = v;
    return true;
  }
  return false;
}

}  // namespace orc
