// traverse.cuh — closest-hit and any-hit traversal of the compressed 8-wide
// BVH (layout in host/bvh_build.h).  Replaces `Bvh::intersect` and
// `Bvh::occluded` (crates/argent-core/src/bvh.rs:159-247).
//
// Exactness.  The triangle test is argent's Moller-Trumbore in argent's
// operation order (bvh.rs:391-410), rounded exactly like the f32 Rust code
// (the library is compiled with --fmad=false).  The closest hit is the
// minimum of (t, original triangle index) over all triangles that pass the
// test, which does not depend on the tree; argent instead keeps the first of
// equal-t hits in its own traversal order, and the parity tests bucket such
// exact ties.  The tree only decides which triangles are tested, so box
// culling must be conservative: child boxes are quantised outward (decoded
// lo <= true lo, decoded hi >= true hi), and the slab interval is widened by
// a bound on its own rounding error (node_ray), so a box whose exact
// interval holds a hit distance is entered whenever argent's slab test
// (bvh.rs:280-299), whose rounding is within that bound, would enter it.
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

// Watertight ray-triangle test (Woop, Benthin and Wald, "Watertight
// Ray/Triangle Intersection", JCGT 2(1), 2013), the optional alternative to
// argent's Moller-Trumbore.  The ray is sheared so that it runs along +z of
// a permuted frame (kz = the axis of largest |d|); the three 2D edge
// functions of the sheared vertices decide the hit.  Two triangles sharing
// an edge evaluate that edge's function from the same two vertices with the
// same arithmetic, so their signs agree and no ray passes between them; an
// edge function of exactly zero is recomputed in double precision so that
// its sign is exact.  Both faces count (argent's test is two-sided too).
// The record holds the three original vertices (v0, v1, v2); the hit's
// (u, v) weigh v1 and v2, as Moller-Trumbore's do.
__device__ __forceinline__ float pick3(float x, float y, float z, int k) { return k == 0 ? x : (k == 1 ? y : z); }

__device__ __forceinline__ bool wt_hit(float4 a, float4 b, float4 c, V3 o, V3 d, float t_max, float* t_out,
                                       float* u_out, float* v_out) {
  float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  int kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
  int kx = kz == 2 ? 0 : kz + 1;
  int ky = kx == 2 ? 0 : kx + 1;
  float dz = pick3(d.x, d.y, d.z, kz);
  if (dz < 0.0f) {
    int t = kx;
    kx = ky;
    ky = t;
  }
  float sx = __fdiv_rn(pick3(d.x, d.y, d.z, kx), dz), sy = __fdiv_rn(pick3(d.x, d.y, d.z, ky), dz);
  float sz = __fdiv_rn(1.0f, dz);
  // Vertices relative to the origin, then permuted (x, y, z) = (kx, ky, kz).
  V3 A = V3{a.x, a.y, a.z} - o, B = V3{b.x, b.y, b.z} - o, C = V3{c.x, c.y, c.z} - o;
  float Akz = pick3(A.x, A.y, A.z, kz), Bkz = pick3(B.x, B.y, B.z, kz), Ckz = pick3(C.x, C.y, C.z, kz);
  float Ax = __fsub_rn(pick3(A.x, A.y, A.z, kx), __fmul_rn(sx, Akz));
  float Ay = __fsub_rn(pick3(A.x, A.y, A.z, ky), __fmul_rn(sy, Akz));
  float Bx = __fsub_rn(pick3(B.x, B.y, B.z, kx), __fmul_rn(sx, Bkz));
  float By = __fsub_rn(pick3(B.x, B.y, B.z, ky), __fmul_rn(sy, Bkz));
  float Cx = __fsub_rn(pick3(C.x, C.y, C.z, kx), __fmul_rn(sx, Ckz));
  float Cy = __fsub_rn(pick3(C.x, C.y, C.z, ky), __fmul_rn(sy, Ckz));
  float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
  float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
  float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
  if (U == 0.0f || V == 0.0f || W == 0.0f) {
    // The product of two floats is exact in double, so the difference of
    // two such products has the exact sign.
    U = (float)__dsub_rn(__dmul_rn((double)Cx, (double)By), __dmul_rn((double)Cy, (double)Bx));
    V = (float)__dsub_rn(__dmul_rn((double)Ax, (double)Cy), __dmul_rn((double)Ay, (double)Cx));
    W = (float)__dsub_rn(__dmul_rn((double)Bx, (double)Ay), __dmul_rn((double)By, (double)Ax));
  }
  if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
  float det = __fadd_rn(__fadd_rn(U, V), W);
  if (det == 0.0f) return false;
  float T = __fadd_rn(__fadd_rn(__fmul_rn(U, __fmul_rn(sz, Akz)), __fmul_rn(V, __fmul_rn(sz, Bkz))),
                      __fmul_rn(W, __fmul_rn(sz, Ckz)));
  float inv = __fdiv_rn(1.0f, det);
  float t = __fmul_rn(T, inv);
  if (!(t > 1e-7f && t < t_max)) return false;
  *t_out = t;
  *u_out = __fmul_rn(V, inv);
  *v_out = __fmul_rn(W, inv);
  return true;
}

// The triangle test a record asks for: the bits of its second word's w are
// 0 for argent's Moller-Trumbore (record = v0, e1, e2) and
// ARGENT_TRI_REC_WATERTIGHT for the watertight test (record = v0, v1, v2).
#define ARGENT_TRI_REC_WATERTIGHT 1u
// 0 compiles the watertight branch out of the leaf test (pieces can then
// only use Moller-Trumbore; argent_piece_set_triangle_test still rewrites
// the records, which such a build would misread).
#ifndef ARGENT_WATERTIGHT_OPTION
#define ARGENT_WATERTIGHT_OPTION 1
#endif

// Moller-Trumbore, bvh.rs:391-410 (or the watertight test, by the
// record's marker).  True on a hit with t in (1e-7, t_max).
__device__ __forceinline__ bool mt_hit(const float4* tri, V3 o, V3 d, float t_max, float* t_out, float* u_out,
                                       float* v_out, uint32_t* prim_out) {
  float4 a = __ldg(tri);
  float4 b = __ldg(tri + 1);
  float4 c = __ldg(tri + 2);
#if ARGENT_WATERTIGHT_OPTION
  if (__float_as_uint(b.w) == ARGENT_TRI_REC_WATERTIGHT) {
    if (!wt_hit(a, b, c, o, d, t_max, t_out, u_out, v_out)) return false;
    *prim_out = __float_as_uint(a.w);
    return true;
  }
#endif
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

// Read-only 16-byte load of BVH node data with the L2 "evict last"
// priority: every ray walks the upper levels and the node array is a small
// share of what passes through L2 (path state streams through it once per
// kernel), so nodes are kept in preference to the streaming data.
__device__ __forceinline__ uint4 ld_node16(const uint4* ptr) {
  uint4 r;
  uint64_t pol;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  asm("ld.global.nc.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
      : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
      : "l"(ptr), "l"(pol));
  return r;
}

__device__ __forceinline__ NodeView load_node(const uint4* nodes, uint32_t idx) {
  const uint4* p = nodes + 5 * (size_t)idx;
  uint4 w0 = ld_node16(p), w1 = ld_node16(p + 1), w2 = ld_node16(p + 2), w3 = ld_node16(p + 3),
        w4 = ld_node16(p + 4);
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

// Byte c of the packed plane words (w0: children 0-3, w1: 4-7) as an exact
// float, without an integer-to-float conversion (those issue on the narrow
// XU pipe): the byte is placed in the mantissa of 2^23, and 2^23 is
// subtracted exactly.
__device__ __forceinline__ float qf(uint32_t w0, uint32_t w1, int c) {
  return __fadd_rn(__uint_as_float(__byte_perm(c < 4 ? w0 : w1, 0x4B000000u, 0x7440u | (uint32_t)(c & 3))),
                   -8388608.0f);
}

// A ray prepared for the node-space slab test: the inverse direction with
// magnitudes capped at 2^64 (a zero component gives +-2^64, so no 0 * inf
// arises), and per axis whether the ray runs toward -axis.
struct RayQ {
  V3 o;
  float ix, iy, iz;
  bool nx, ny, nz;
};

__device__ __forceinline__ float capped_inv(float d) {
  const float cap = 18446744073709551616.0f;  // 2^64
  return fminf(fmaxf(__fdiv_rn(1.0f, d), -cap), cap);
}

__device__ __forceinline__ RayQ make_rayq(V3 o, V3 d) {
  RayQ r;
  r.o = o;
  r.ix = capped_inv(d.x);
  r.iy = capped_inv(d.y);
  r.iz = capped_inv(d.z);
  r.nx = signbit(r.ix);
  r.ny = signbit(r.iy);
  r.nz = signbit(r.iz);
  return r;
}

// One axis of a node seen from a ray.  A plane q of the axis is at
// t = (origin + q * scale - o) * inv = q * a + b, with a = scale * inv
// (exact: scale is a power of two) and b = (origin - o) * inv.  Computed as
// fma(q, a, b), t differs from the exact value by at most about
// 3 * 2^-24 * (|origin - o| + 255 * scale) * |inv|; the slack e is 2^-18
// times that magnitude (64 units of rounding), and is subtracted from the
// near plane's bias and added to the far plane's.  The near plane is the
// low one unless the ray runs toward -axis.
struct AxisQ {
  float a, bn, bf;
  uint32_t n0, n1, f0, f1;
};

__device__ __forceinline__ AxisQ axis_q(float origin, float scale, float o, float inv, bool neg, uint32_t lo0,
                                        uint32_t lo1, uint32_t hi0, uint32_t hi1) {
  AxisQ q;
  float dd = __fsub_rn(origin, o);
  float b = __fmul_rn(dd, inv);
  float e = __fmul_rn(__fmul_rn(__fadd_rn(fabsf(dd), __fmul_rn(256.0f, scale)), fabsf(inv)), 3.814697265625e-06f);
  q.a = __fmul_rn(scale, inv);
  q.bn = __fsub_rn(b, e);
  q.bf = __fadd_rn(b, e);
  q.n0 = neg ? hi0 : lo0;
  q.n1 = neg ? hi1 : lo1;
  q.f0 = neg ? lo0 : hi0;
  q.f1 = neg ? lo1 : hi1;
  return q;
}

struct NodeQ {
  AxisQ x, y, z;
};

// The whole box of a node, planes 0 and 255 on every axis (it holds every
// child box), with the slack of axis_q.  Reads only the node's first 16
// bytes.  A ray that misses the root's box misses the piece.
__device__ __forceinline__ bool node_box_hit(const uint4* nodes, uint32_t idx, const RayQ& r, float t_max) {
  uint4 w0 = ld_node16(nodes + 5 * (size_t)idx);
  float o[3] = {__uint_as_float(w0.x), __uint_as_float(w0.y), __uint_as_float(w0.z)};
  float ro[3] = {r.o.x, r.o.y, r.o.z};
  float iv[3] = {r.ix, r.iy, r.iz};
  float tmin = 0.0f, tmax = t_max;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    float scale = __uint_as_float(((w0.w >> (8 * k)) & 0xffu) << 23);
    float dd = __fsub_rn(o[k], ro[k]);
    float b = __fmul_rn(dd, iv[k]);
    float e = __fmul_rn(__fmul_rn(__fadd_rn(fabsf(dd), __fmul_rn(256.0f, scale)), fabsf(iv[k])), 3.814697265625e-06f);
    float t1 = __fmaf_rn(255.0f, __fmul_rn(scale, iv[k]), b);
    tmin = fmaxf(tmin, __fsub_rn(fminf(b, t1), e));
    tmax = fminf(tmax, __fadd_rn(fmaxf(b, t1), e));
  }
  return tmin <= tmax;
}

__device__ __forceinline__ NodeQ node_ray(const NodeView& n, const RayQ& r) {
  NodeQ q;
  q.x = axis_q(n.ox, n.sx, r.o.x, r.ix, r.nx, n.qlx0, n.qlx1, n.qhx0, n.qhx1);
  q.y = axis_q(n.oy, n.sy, r.o.y, r.iy, r.ny, n.qly0, n.qly1, n.qhy0, n.qhy1);
  q.z = axis_q(n.oz, n.sz, r.o.z, r.iz, r.nz, n.qlz0, n.qlz1, n.qhz0, n.qhz1);
  return q;
}

// Widened slab interval of child c, clipped to [0, t_max]; true when it is
// not empty.  *tmin_out = its entry distance.
__device__ __forceinline__ bool child_q(const NodeQ& q, int c, float t_max, float* tmin_out) {
  float tnx = __fmaf_rn(qf(q.x.n0, q.x.n1, c), q.x.a, q.x.bn);
  float tny = __fmaf_rn(qf(q.y.n0, q.y.n1, c), q.y.a, q.y.bn);
  float tnz = __fmaf_rn(qf(q.z.n0, q.z.n1, c), q.z.a, q.z.bn);
  float tfx = __fmaf_rn(qf(q.x.f0, q.x.f1, c), q.x.a, q.x.bf);
  float tfy = __fmaf_rn(qf(q.y.f0, q.y.f1, c), q.y.a, q.y.bf);
  float tfz = __fmaf_rn(qf(q.z.f0, q.z.f1, c), q.z.a, q.z.bf);
  float tmin = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, 0.0f));
  float tmax = fminf(fminf(tfx, tfy), fminf(tfz, t_max));
  *tmin_out = tmin;
  return tmin <= tmax;
}

// Traversal stacks.  LocalStack keeps a thread's whole stack in its local
// memory.  ShortStack keeps the top S entries in shared memory (a ring per
// thread: entry k in row k % S of the thread's column, so the 32 threads of
// a warp touch 32 consecutive words and no bank twice) and moves older
// entries to a local-memory spill array only while the stack is deeper than
// S: a push that wraps onto an occupied row first writes that row's entry to
// spill[sp - S], and a pop that uncovers a spilled entry moves it back into
// the freed row.  The order of entries is the same either way, so
// traversals, pruning and results do not depend on the stack kind.
template <typename E>
struct LocalStack {
  E* a;
  __device__ __forceinline__ void push(int& sp, E e) { a[sp++] = e; }
  __device__ __forceinline__ E pop(int& sp) { return a[--sp]; }
};

template <typename E, int S, int STRIDE>
struct ShortStack {
  static_assert((S & (S - 1)) == 0, "ring size must be a power of two");
  E* sh;     // this thread's column in the block's shared ring array
  E* spill;  // this thread's local spill array
  __device__ __forceinline__ void push(int& sp, E e) {
    E* row = sh + (sp & (S - 1)) * STRIDE;
    if (sp >= S) spill[sp - S] = *row;
    *row = e;
    ++sp;
  }
  __device__ __forceinline__ E pop(int& sp) {
    --sp;
    E* row = sh + (sp & (S - 1)) * STRIDE;
    E e = *row;
    if (sp >= S) *row = spill[sp - S];
    return e;
  }
};

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
    int kind = base / 3;
    int bin = nodes == 0 ? 0 : nodes < 2 ? 1 : nodes < 4 ? 2 : nodes < 8 ? 3 : nodes < 16 ? 4 : nodes < 64 ? 5
              : nodes < 256 ? 6 : 7;
    atomicAdd(&d_trav_hist[8 * kind + bin], 1ull);
    atomicMax(&d_trav_max[kind], nodes);
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

// Children's push order: 1 = all entered children sorted by entry distance
// (the nearest popped first), 0 = the nearest entered at once and the rest
// pushed in slot order.  Hits do not depend on it (see below).  Measured on
// B200 with eight lanes: sorted 1.752 G path-samples/s on the signet still
// and 1.17 G on the gems, nearest-first 1.737 G and 1.144 G (it visits a
// few more nodes, and needs a few more registers), so sorting stays.
#ifndef ARGENT_SORTED_PUSH
#define ARGENT_SORTED_PUSH 1
#endif

// Closest hit with t in (1e-7, t_max).  Ties at equal t go to the lower
// original triangle index.
//
// Order of visits: of the children a node's slab test keeps, the nearest
// by entry distance is entered at once; the others are pushed with their
// entry distances (ARGENT_SORTED_PUSH: far-to-near).  The key is the entry
// distance with its 3 low mantissa bits replaced by the child slot; the
// truncated distance is what the stack keeps for pruning, which can only
// keep more nodes than the exact value.
// The visit order changes how much is pruned, never the result: a triangle
// whose hit is the final best has box entry <= that distance <= the running
// best at every point, so its box is always entered.
//
// The traversal is resumable: closest_begin sets it up and each
// closest_step visits one node or one leaf, so a kernel can interleave the
// steps of rays that start at different times (persistent lanes that take a
// new ray as soon as theirs finishes).  The stack (LocalStack or
// ShortStack) lives with the caller.
struct ClosestTrav {
  V3 o, d;
  RayQ rq;
  float t_max;
  TraceHit best;
  uint32_t ref;
  int sp;
  bool have;
  uint32_t n_nodes, n_tris;
};

// Returns false when the traversal is already over (empty piece, or a ray
// that misses the piece's box); s.best is then a miss.
__device__ __forceinline__ bool closest_begin(const DevPiece& pc, ClosestTrav& s, V3 o, V3 d, float t_max) {
  s.o = o;
  s.d = d;
  s.t_max = t_max;
  s.best = TraceHit{t_max, 0.0f, 0.0f, ARGENT_NO_HIT_U};
  s.ref = 0u;
  s.sp = 0;
  s.have = false;
  s.n_nodes = 0;
  s.n_tris = 0;
  if (pc.num_tris == 0) return false;
  s.rq = make_rayq(o, d);
  if (!node_box_hit(pc.nodes, 0u, s.rq, t_max)) return false;
  s.have = true;
  return true;
}

// Makes the next node or leaf current (popping entries that the running
// best has pruned); false when the traversal is over.
template <class ST>
__device__ __forceinline__ bool closest_next(ClosestTrav& s, ST& stack) {
  if (s.have) return true;
  while (s.sp > 0) {
    uint2 e = stack.pop(s.sp);
    if (__uint_as_float(e.y) <= s.best.t) {
      s.ref = e.x;
      s.have = true;
      return true;
    }
  }
  return false;
}

__device__ __forceinline__ bool trav_at_leaf(uint32_t ref) { return (ref & ARGENT_LEAF_BIT) != 0; }

// Visits the current node or leaf (closest_next returned true); true while
// the traversal has more to visit.
template <class ST>
__device__ __forceinline__ bool closest_visit(const DevPiece& pc, ClosestTrav& s, ST& stack, uint32_t* status) {
  s.have = false;
  uint32_t ref = s.ref;
  if (ref & ARGENT_LEAF_BIT) {
    uint32_t start = ref & 0x07FFFFFFu;
    uint32_t cnt = ((ref >> 27) & 15u) + 1u;
    s.n_tris += cnt;
    for (uint32_t i = 0; i < cnt; ++i) {
      float t, u, v;
      uint32_t prim;
      // Accept t == best.t too, so equal-t ties resolve by index.
      float lim = s.best.t;
      if (mt_hit(pc.tris + 3 * (size_t)(start + i), s.o, s.d, s.t_max, &t, &u, &v, &prim)) {
        if (t < lim || (t == lim && prim < s.best.prim)) {
          s.best.t = t;
          s.best.u = u;
          s.best.v = v;
          s.best.prim = prim;
        }
      }
    }
    return s.sp > 0;
  }
  NodeView n = load_node(pc.nodes, ref);
  ++s.n_nodes;
  NodeQ nq = node_ray(n, s.rq);
  uint32_t k[8];
  int nh = 0;
  uint32_t hm = 0;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    float tc;
    bool h = child_q(nq, c, s.best.t, &tc) && ((n.present >> c) & 1u);
    k[c] = h ? ((__float_as_uint(tc) & ~7u) | (uint32_t)c) : 0xFFFFFFFFu;
    nh += h ? 1 : 0;
    hm |= h ? (1u << c) : 0u;
  }
  if (d_trav_counting) atomicAdd(&d_trav_child_hits[nh], 1ull);
  if (nh == 0) return s.sp > 0;
  if (s.sp + nh - 1 > ARGENT_STACK_SIZE) {
    atomicOr(status, ARGENT_STATUS_STACK_OVERFLOW);
    s.sp = 0;
    return false;
  }
#if ARGENT_SORTED_PUSH
  sort8(k);
#pragma unroll
  for (int j = 7; j >= 1; --j) {
    if (j < nh) stack.push(s.sp, make_uint2(child_ref(n, (int)(k[j] & 7u)), k[j] & ~7u));
  }
  s.ref = child_ref(n, (int)(k[0] & 7u));
#else
  // Descend into the nearest child; push the others (nh - 1: none in three
  // visits of four, and at most one in more than nine of ten) in slot order
  // with their entry distances, so popping still prunes them against the
  // running best.  The loop runs as many times as the lane has children to
  // push, where the sort costs 19 compare-exchanges and eight guarded
  // pushes on every visit.
  uint32_t kmin = min(min(min(k[0], k[1]), min(k[2], k[3])), min(min(k[4], k[5]), min(k[6], k[7])));
  uint32_t near = kmin & 7u;
  uint32_t rest = hm & ~(1u << near);
  while (rest) {
    int c = __ffs(rest) - 1;
    rest &= rest - 1u;
    uint32_t kc = c == 0 ? k[0] : c == 1 ? k[1] : c == 2 ? k[2] : c == 3 ? k[3]
                : c == 4 ? k[4] : c == 5 ? k[5] : c == 6 ? k[6] : k[7];
    stack.push(s.sp, make_uint2(child_ref(n, c), kc & ~7u));
  }
  s.ref = child_ref(n, (int)near);
#endif
  s.have = true;
  return true;
}

// Visits one node or one leaf; true when the traversal has finished.
template <class ST>
__device__ __forceinline__ bool closest_step(const DevPiece& pc, ClosestTrav& s, ST& stack, uint32_t* status) {
  if (!closest_next(s, stack)) return true;
  return !closest_visit(pc, s, stack, status);
}

__device__ __noinline__ TraceHit trace_closest(const DevPiece& pc, V3 o, V3 d, float t_max, uint32_t* status) {
  ClosestTrav s;
  uint2 arr[ARGENT_STACK_SIZE];
  LocalStack<uint2> stack{arr};
  if (closest_begin(pc, s, o, d, t_max))
    while (!closest_step(pc, s, stack, status)) {
    }
  count_visits(0, s.n_nodes, s.n_tris);
  return s.best;
}

// Any hit with t in (1e-7, t_max), bvh.rs:216-247, resumable like the
// closest-hit traversal.
struct AnyTrav {
  V3 o, d;
  RayQ rq;
  float t_max;
  int sp;
  uint32_t ref;
  bool have;  // ref holds a popped entry not yet visited
  uint32_t n_nodes, n_tris;
};

#define ARGENT_ANY_RUNNING 0
#define ARGENT_ANY_HIT 1
#define ARGENT_ANY_CLEAR 2

// The test any_begin starts with: false when the piece is empty or the ray
// (up to t_max) misses its box, so nothing of the piece can occlude it.
__device__ __forceinline__ bool piece_may_occlude(const DevPiece& pc, V3 o, V3 d, float t_max) {
  if (pc.num_tris == 0) return false;
  return node_box_hit(pc.nodes, 0u, make_rayq(o, d), t_max);
}

// Returns ARGENT_ANY_RUNNING, or ARGENT_ANY_CLEAR when the ray misses the
// piece outright.
template <class ST>
__device__ __forceinline__ int any_begin(const DevPiece& pc, AnyTrav& s, ST& stack, V3 o, V3 d, float t_max) {
  s.o = o;
  s.d = d;
  s.t_max = t_max;
  s.sp = 0;
  s.have = false;
  s.n_nodes = 0;
  s.n_tris = 0;
  if (pc.num_tris == 0) return ARGENT_ANY_CLEAR;
  s.rq = make_rayq(o, d);
  if (!node_box_hit(pc.nodes, 0u, s.rq, t_max)) return ARGENT_ANY_CLEAR;
  stack.push(s.sp, 0u);
  return ARGENT_ANY_RUNNING;
}

// Pops the next node or leaf into s.ref; false when none is left.
template <class ST>
__device__ __forceinline__ bool any_next(AnyTrav& s, ST& stack) {
  if (s.have) return true;
  if (s.sp == 0) return false;
  s.ref = stack.pop(s.sp);
  s.have = true;
  return true;
}

// Visits s.ref: ARGENT_ANY_HIT, or ARGENT_ANY_RUNNING / ARGENT_ANY_CLEAR by
// whether entries remain.
template <class ST>
__device__ __forceinline__ int any_visit(const DevPiece& pc, AnyTrav& s, ST& stack, uint32_t* status) {
  s.have = false;
  uint32_t ref = s.ref;
  if (ref & ARGENT_LEAF_BIT) {
    uint32_t start = ref & 0x07FFFFFFu;
    uint32_t cnt = ((ref >> 27) & 15u) + 1u;
    for (uint32_t i = 0; i < cnt; ++i) {
      float t, u, v;
      uint32_t prim;
      ++s.n_tris;
      if (mt_hit(pc.tris + 3 * (size_t)(start + i), s.o, s.d, s.t_max, &t, &u, &v, &prim)) return ARGENT_ANY_HIT;
    }
    return s.sp == 0 ? ARGENT_ANY_CLEAR : ARGENT_ANY_RUNNING;
  }
  NodeView n = load_node(pc.nodes, ref);
  ++s.n_nodes;
  NodeQ nq = node_ray(n, s.rq);
  uint32_t hitmask = 0;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    float tmin;
    if (child_q(nq, c, s.t_max, &tmin)) hitmask |= 1u << c;
  }
  hitmask &= n.present;
  if (d_trav_counting) atomicAdd(&d_trav_child_hits[9 + __popc(hitmask)], 1ull);
  if (s.sp + __popc(hitmask) > ARGENT_STACK_SIZE) {
    atomicOr(status, ARGENT_STATUS_STACK_OVERFLOW);
    s.sp = 0;
    return ARGENT_ANY_CLEAR;
  }
  while (hitmask) {
    int c = __ffs(hitmask) - 1;
    hitmask &= hitmask - 1u;
    stack.push(s.sp, child_ref(n, c));
  }
  return s.sp == 0 ? ARGENT_ANY_CLEAR : ARGENT_ANY_RUNNING;
}

// Visits one node or one leaf.
template <class ST>
__device__ __forceinline__ int any_step(const DevPiece& pc, AnyTrav& s, ST& stack, uint32_t* status) {
  if (!any_next(s, stack)) return ARGENT_ANY_CLEAR;
  return any_visit(pc, s, stack, status);
}

__device__ __noinline__ bool trace_any(const DevPiece& pc, V3 o, V3 d, float t_max, uint32_t* status) {
  AnyTrav s;
  uint32_t arr[ARGENT_STACK_SIZE];
  LocalStack<uint32_t> stack{arr};
  int r = any_begin(pc, s, stack, o, d, t_max);
  while (r == ARGENT_ANY_RUNNING) r = any_step(pc, s, stack, status);
  count_visits(3, s.n_nodes, s.n_tris);
  return r == ARGENT_ANY_HIT;
}

}  // namespace dev
