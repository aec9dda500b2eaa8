// traverse.cuh — closest-hit and any-hit traversal of the compressed 8-wide
// BVH (layout in host/bvh_build.h).  Replaces `Bvh::intersect` and
// `Bvh::occluded` (crates/argent-core/src/bvh.rs:159-247).
//
// Exactness.  The triangle test is argent's Moller-Trumbore in argent's
// operation order (bvh.rs:391-410), rounded exactly like the f32 Rust code
// (the library is compiled with --fmad=false; the box decode uses explicit
// round-to-nearest intrinsics).  Child boxes are quantised conservatively
// (decoded lo <= true lo, decoded hi >= true hi), and the slab test keeps
// argent's arithmetic ((plane - o) * inv, SSE min/max), so every box argent's
// traversal enters is entered here too.  The closest hit is the minimum of
// (t, original triangle index) over all triangles that pass the test, which
// does not depend on the tree.  argent instead keeps the first of equal-t
// hits in its own traversal order; the parity tests bucket such exact ties.
#pragma once
#include "dev_math.cuh"
#include "tables.cuh"

namespace dev {

#define ARGENT_STACK_SIZE 160
#define ARGENT_LEAF_BIT 0x80000000u
#define ARGENT_NO_HIT_U 0xFFFFFFFFu

// Status bits written (atomicOr) to the context's device status word.
#define ARGENT_STATUS_STACK_OVERFLOW 1u

struct DevPiece {
  const uint4* nodes;    // 5 x uint4 per wide node
  const float4* tris;    // 3 x float4 per triangle, BVH order
  const float4* pos;     // vertex positions (w unused)
  const float4* nrm;     // vertex normals or nullptr
  const uint4* tri_idx;  // (a, b, c, material) per original triangle
  const float* cavity;   // per vertex or nullptr
  uint32_t num_tris;
};

// Moller-Trumbore, bvh.rs:391-410.  Returns t > 0 on a hit, else -1.
__device__ __forceinline__ bool mt_hit(const float4* tri, V3 o, V3 d, float t_max, float* t_out, float* u_out,
                                       float* v_out, uint32_t* prim_out) {
  float4 a = __ldg(tri);
  float4 b = __ldg(tri + 1);
  float4 c = __ldg(tri + 2);
  V3 v0{a.x, a.y, a.z}, e1{b.x, b.y, b.z}, e2{c.x, c.y, c.z};
  V3 p = cross(d, e2);
  float det = dot(e1, p);
  if (fabsf(det) < 1e-14f) return false;
  float inv_det = __fdiv_rn(1.0f, det);
  V3 s = o - v0;
  float u = dot(s, p) * inv_det;
  if (!(u >= 0.0f && u <= 1.0f)) return false;
  V3 q = cross(s, e1);
  float v = dot(d, q) * inv_det;
  if (v < 0.0f || u + v > 1.0f) return false;
  float t = dot(e2, q) * inv_det;
  if (t > 1e-7f && t < t_max) {
    *t_out = t;
    *u_out = u;
    *v_out = v;
    *prim_out = __float_as_uint(a.w);
    return true;
  }
  return false;
}

struct NodeView {
  float ox, oy, oz;
  float sx, sy, sz;
  uint32_t imask, child_base, tri_base, leaf_counts, present;
  uint32_t qlx0, qlx1, qly0, qly1, qlz0, qlz1, qhx0, qhx1, qhy0, qhy1, qhz0, qhz1;
};

__device__ __forceinline__ NodeView load_node(const uint4* nodes, uint32_t idx) {
  const uint4* p = nodes + 5 * (size_t)idx;
  uint4 w0 = __ldg(p), w1 = __ldg(p + 1), w2 = __ldg(p + 2), w3 = __ldg(p + 3), w4 = __ldg(p + 4);
  NodeView n;
  n.ox = __uint_as_float(w0.x);
  n.oy = __uint_as_float(w0.y);
  n.oz = __uint_as_float(w0.z);
  n.sx = __uint_as_float((w0.w & 0xffu) << 23);
  n.sy = __uint_as_float(((w0.w >> 8) & 0xffu) << 23);
  n.sz = __uint_as_float(((w0.w >> 16) & 0xffu) << 23);
  n.imask = w0.w >> 24;
  n.child_base = w1.x;
  n.tri_base = w1.y;
  n.leaf_counts = w1.z;
  n.present = w1.w & 0xffu;
  n.qlx0 = w2.x; n.qlx1 = w2.y; n.qly0 = w2.z; n.qly1 = w2.w;
  n.qlz0 = w3.x; n.qlz1 = w3.y; n.qhx0 = w3.z; n.qhx1 = w3.w;
  n.qhy0 = w4.x; n.qhy1 = w4.y; n.qhz0 = w4.z; n.qhz1 = w4.w;
  return n;
}

__device__ __forceinline__ uint32_t qbyte(uint32_t w0, uint32_t w1, int c) {
  return ((c < 4 ? w0 : w1) >> (8 * (c & 3))) & 0xffu;
}
__device__ __forceinline__ float decode(float origin, uint32_t q, float scale) {
  return __fadd_rn(origin, __fmul_rn((float)q, scale));
}

// Reference to a child: an interior node index, or a leaf
// (LEAF_BIT | (count-1) << 27 | first triangle).
__device__ __forceinline__ uint32_t child_ref(const NodeView& n, int c) {
  uint32_t below = (1u << c) - 1u;
  if ((n.imask >> c) & 1u) return n.child_base + __popc(n.imask & below);
  uint32_t leafmask = n.present & ~n.imask;
  uint32_t lc = n.leaf_counts & ((1u << (4 * c)) - 1u);
  uint32_t x = (lc & 0x0F0F0F0Fu) + ((lc >> 4) & 0x0F0F0F0Fu);
  uint32_t off = ((x * 0x01010101u) >> 24) + __popc(leafmask & below);
  uint32_t cnt1 = (n.leaf_counts >> (4 * c)) & 15u;
  return ARGENT_LEAF_BIT | (cnt1 << 27) | (n.tri_base + off);
}

// Slab test of child c, bvh.rs:280-299 (SSE min/max).  Returns tmin or -1
// (as "no hit") in *hit.
__device__ __forceinline__ bool slab_child(const NodeView& n, int c, V3 o, V3 inv, float t_max, float* tmin_out) {
  float lx = decode(n.ox, qbyte(n.qlx0, n.qlx1, c), n.sx);
  float hx = decode(n.ox, qbyte(n.qhx0, n.qhx1, c), n.sx);
  float ly = decode(n.oy, qbyte(n.qly0, n.qly1, c), n.sy);
  float hy = decode(n.oy, qbyte(n.qhy0, n.qhy1, c), n.sy);
  float lz = decode(n.oz, qbyte(n.qlz0, n.qlz1, c), n.sz);
  float hz = decode(n.oz, qbyte(n.qhz0, n.qhz1, c), n.sz);
  float tx0 = __fmul_rn(__fsub_rn(lx, o.x), inv.x);
  float tx1 = __fmul_rn(__fsub_rn(hx, o.x), inv.x);
  float ty0 = __fmul_rn(__fsub_rn(ly, o.y), inv.y);
  float ty1 = __fmul_rn(__fsub_rn(hy, o.y), inv.y);
  float tz0 = __fmul_rn(__fsub_rn(lz, o.z), inv.z);
  float tz1 = __fmul_rn(__fsub_rn(hz, o.z), inv.z);
  float tmin = sse_max(sse_max(sse_max(sse_min(tx0, tx1), sse_min(ty0, ty1)), sse_min(tz0, tz1)), 0.0f);
  float tmax = sse_min(sse_min(sse_min(sse_max(tx0, tx1), sse_max(ty0, ty1)), sse_max(tz0, tz1)), t_max);
  *tmin_out = tmin;
  return tmin <= tmax;
}

struct TraceHit {
  float t, u, v;
  uint32_t prim;
};

// Adds one ray's node and triangle visits to the instrumentation counters.
__device__ __forceinline__ void count_visits(int base, uint32_t nodes, uint32_t tris) {
  if (d_trav_counting) {
    atomicAdd(&d_trav_counts[base], 1ull);
    atomicAdd(&d_trav_counts[base + 1], (unsigned long long)nodes);
    atomicAdd(&d_trav_counts[base + 2], (unsigned long long)tris);
  }
}

// Sorts 8 keys ascending (Batcher odd-even merge network, 19 comparators).
#define ARGENT_CX(a, b)                      \
  {                                          \
    uint32_t lo_ = min(k[a], k[b]);          \
    uint32_t hi_ = max(k[a], k[b]);          \
    k[a] = lo_;                              \
    k[b] = hi_;                              \
  }
__device__ __forceinline__ void sort8(uint32_t k[8]) {
  ARGENT_CX(0, 1) ARGENT_CX(2, 3) ARGENT_CX(4, 5) ARGENT_CX(6, 7)
  ARGENT_CX(0, 2) ARGENT_CX(1, 3) ARGENT_CX(4, 6) ARGENT_CX(5, 7)
  ARGENT_CX(1, 2) ARGENT_CX(5, 6)
  ARGENT_CX(0, 4) ARGENT_CX(1, 5) ARGENT_CX(2, 6) ARGENT_CX(3, 7)
  ARGENT_CX(2, 4) ARGENT_CX(3, 5)
  ARGENT_CX(1, 2) ARGENT_CX(3, 4) ARGENT_CX(5, 6)
}
#undef ARGENT_CX

// Closest hit with t in (1e-7, t_max).  Ties at equal t go to the lower
// original triangle index.
//
// Order of visits: the children a node's slab test keeps are sorted by
// entry distance and the nearest is entered at once; the others are pushed
// far-to-near.  The sort key is the entry distance with its 3 low mantissa
// bits replaced by the child slot; the truncated distance is what the stack
// keeps for pruning, which can only keep more nodes than the exact value.
// The visit order changes how much is pruned, never the result: a triangle
// whose hit is the final best has box entry <= that distance <= the running
// best at every point, so its box is always entered.
__device__ __noinline__ TraceHit trace_closest(const DevPiece& pc, V3 o, V3 d, float t_max, uint32_t* status) {
  TraceHit best{t_max, 0.0f, 0.0f, ARGENT_NO_HIT_U};
  if (pc.num_tris == 0) return best;
  V3 inv{__fdiv_rn(1.0f, d.x), __fdiv_rn(1.0f, d.y), __fdiv_rn(1.0f, d.z)};
  uint2 stack[ARGENT_STACK_SIZE];
  int sp = 0;
  uint32_t n_nodes = 0, n_tris = 0;
  uint32_t ref = 0u;
  bool have = true;
  for (;;) {
    if (!have) {
      if (sp == 0) break;
      --sp;
      ref = stack[sp].x;
      if (__uint_as_float(stack[sp].y) > best.t) continue;
    }
    have = false;
    if (ref & ARGENT_LEAF_BIT) {
      uint32_t start = ref & 0x07FFFFFFu;
      uint32_t cnt = ((ref >> 27) & 15u) + 1u;
      n_tris += cnt;
      for (uint32_t i = 0; i < cnt; ++i) {
        float t, u, v;
        uint32_t prim;
        // Accept t == best.t too, so equal-t ties resolve by index.
        float lim = best.t;
        if (mt_hit(pc.tris + 3 * (size_t)(start + i), o, d, t_max, &t, &u, &v, &prim)) {
          if (t < lim || (t == lim && prim < best.prim)) {
            best.t = t;
            best.u = u;
            best.v = v;
            best.prim = prim;
          }
        }
      }
      continue;
    }
    NodeView n = load_node(pc.nodes, ref);
    ++n_nodes;
    uint32_t k[8];
    int nh = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      k[c] = 0xFFFFFFFFu;
      float tc;
      if (((n.present >> c) & 1u) && slab_child(n, c, o, inv, best.t, &tc)) {
        k[c] = (__float_as_uint(tc) & ~7u) | (uint32_t)c;
        ++nh;
      }
    }
    if (nh == 0) continue;
    if (sp + nh - 1 > ARGENT_STACK_SIZE) {
      atomicOr(status, ARGENT_STATUS_STACK_OVERFLOW);
      break;
    }
    sort8(k);
#pragma unroll
    for (int j = 7; j >= 1; --j) {
      if (j < nh) stack[sp++] = make_uint2(child_ref(n, (int)(k[j] & 7u)), k[j] & ~7u);
    }
    ref = child_ref(n, (int)(k[0] & 7u));
    have = true;
  }
  count_visits(0, n_nodes, n_tris);
  return best;
}

// Any hit with t in (1e-7, t_max), bvh.rs:216-247.
__device__ __noinline__ bool trace_any(const DevPiece& pc, V3 o, V3 d, float t_max, uint32_t* status) {
  if (pc.num_tris == 0) return false;
  V3 inv{__fdiv_rn(1.0f, d.x), __fdiv_rn(1.0f, d.y), __fdiv_rn(1.0f, d.z)};
  uint32_t stack[ARGENT_STACK_SIZE];
  int sp = 0;
  uint32_t n_nodes = 0, n_tris = 0;
  stack[sp++] = 0u;
  while (sp > 0) {
    uint32_t ref = stack[--sp];
    if (ref & ARGENT_LEAF_BIT) {
      uint32_t start = ref & 0x07FFFFFFu;
      uint32_t cnt = ((ref >> 27) & 15u) + 1u;
      for (uint32_t i = 0; i < cnt; ++i) {
        float t, u, v;
        uint32_t prim;
        ++n_tris;
        if (mt_hit(pc.tris + 3 * (size_t)(start + i), o, d, t_max, &t, &u, &v, &prim)) {
          count_visits(3, n_nodes, n_tris);
          return true;
        }
      }
      continue;
    }
    NodeView n = load_node(pc.nodes, ref);
    ++n_nodes;
    uint32_t hitmask = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      float tmin;
      if ((n.present >> c) & 1u) {
        if (slab_child(n, c, o, inv, t_max, &tmin)) hitmask |= 1u << c;
      }
    }
    if (sp + __popc(hitmask) > ARGENT_STACK_SIZE) {
      atomicOr(status, ARGENT_STATUS_STACK_OVERFLOW);
      return false;
    }
    while (hitmask) {
      int c = __ffs(hitmask) - 1;
      hitmask &= hitmask - 1u;
      stack[sp++] = child_ref(n, c);
    }
  }
  count_visits(3, n_nodes, n_tris);
  return false;
}

}  // namespace dev
