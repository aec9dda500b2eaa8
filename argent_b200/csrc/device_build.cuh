// device_build.cuh — the piece BVH built on the device, for fast piece
// swaps (argent builds on the host at every prepare, bvh.rs:117-146).
//
// A linear BVH (Karras 2012, "Maximizing parallelism in the construction of
// BVHs, octrees, and k-d trees"): 63-bit Morton codes of the triangle
// centroids, a radix sort, the binary radix tree (one thread per internal
// node), boxes bottom-up, then the same collapse to 8-wide nodes the host
// builder does (open the interior child of largest area until 8 children;
// subtrees of at most 4 triangles become leaves), level by level, writing
// the same 80-byte node and 48-byte triangle layouts (host/bvh_build.h) with
// the same conservative plane quantisation.  The traversal does not depend
// on which builder made the tree: every closest hit is the minimum of
// (t, triangle index) over the triangles whose Moller-Trumbore test passes.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace db {

#define DB_LEAF_MAX 4
#define DB_ERR_EXTENT 1u
#define DB_ERR_QUANT 2u

struct Bin {
  float* lo;  // 3 per node
  float* hi;
  uint32_t* first;
  uint32_t* last;
  int32_t* left;
  int32_t* right;
  int32_t* parent;
  uint32_t* flag;
};

// Per triangle: box and centroid; block-reduced centroid bounds.  Launched
// with 256 threads per block.
__global__ void __launch_bounds__(256) k_tri_boxes(const float4* pos, const uint4* tri, uint32_t n, float* tlo,
                                                   float* thi, float* cen, float* blk_lo, float* blk_hi) {
  __shared__ float slo[3][256], shi[3][256];
  float clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    uint4 q = tri[t];
    float4 a = pos[q.x], b = pos[q.y], c = pos[q.z];
    float lo[3] = {fminf(fminf(a.x, b.x), c.x), fminf(fminf(a.y, b.y), c.y), fminf(fminf(a.z, b.z), c.z)};
    float hi[3] = {fmaxf(fmaxf(a.x, b.x), c.x), fmaxf(fmaxf(a.y, b.y), c.y), fmaxf(fmaxf(a.z, b.z), c.z)};
    for (int k = 0; k < 3; ++k) {
      tlo[3 * (size_t)t + k] = lo[k];
      thi[3 * (size_t)t + k] = hi[k];
      float m = 0.5f * lo[k] + 0.5f * hi[k];
      cen[3 * (size_t)t + k] = m;
      clo[k] = fminf(clo[k], m);
      chi[k] = fmaxf(chi[k], m);
    }
  }
  for (int k = 0; k < 3; ++k) {
    slo[k][threadIdx.x] = clo[k];
    shi[k][threadIdx.x] = chi[k];
  }
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int k = 0; k < 3; ++k) {
        slo[k][threadIdx.x] = fminf(slo[k][threadIdx.x], slo[k][threadIdx.x + s]);
        shi[k][threadIdx.x] = fmaxf(shi[k][threadIdx.x], shi[k][threadIdx.x + s]);
      }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; ++k) {
      blk_lo[3 * blockIdx.x + k] = slo[k][0];
      blk_hi[3 * blockIdx.x + k] = shi[k][0];
    }
}

__device__ __forceinline__ uint64_t spread21(uint32_t v) {
  uint64_t x = v & 0x1fffffu;
  x = (x | x << 32) & 0x1f00000000ffffull;
  x = (x | x << 16) & 0x1f0000ff0000ffull;
  x = (x | x << 8) & 0x100f00f00f00f00full;
  x = (x | x << 4) & 0x10c30c30c30c30c3ull;
  x = (x | x << 2) & 0x1249249249249249ull;
  return x;
}

// 63-bit Morton code of each centroid within the centroid bounds (every
// thread reduces the few per-block partials itself).
__global__ void k_morton(const float* cen, uint32_t n, const float* blk_lo, const float* blk_hi, uint32_t nblk,
                         uint64_t* keys, uint32_t* vals) {
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t b = 0; b < nblk; ++b)
    for (int k = 0; k < 3; ++k) {
      lo[k] = fminf(lo[k], blk_lo[3 * b + k]);
      hi[k] = fmaxf(hi[k], blk_hi[3 * b + k]);
    }
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    uint32_t q[3];
    for (int k = 0; k < 3; ++k) {
      float ext = hi[k] - lo[k];
      float u = ext > 0.0f ? (cen[3 * (size_t)t + k] - lo[k]) / ext : 0.0f;
      u = fminf(fmaxf(u, 0.0f), 1.0f);
      q[k] = (uint32_t)fminf(u * 2097152.0f, 2097151.0f);
    }
    keys[t] = (spread21(q[0]) << 2) | (spread21(q[1]) << 1) | spread21(q[2]);
    vals[t] = t;
  }
}

// Karras' common-prefix length of sorted keys i and j (-1 outside the
// array; equal keys fall back to the indices).
__device__ __forceinline__ int delta(const uint64_t* keys, int64_t n, int64_t i, int64_t j) {
  if (j < 0 || j >= n) return -1;
  uint64_t a = keys[i], b = keys[j];
  if (a == b) return 64 + __clz((uint32_t)(i ^ j));
  return __clzll(a ^ b);
}

// Internal node i of the binary radix tree (Karras 2012, Fig. 4).  Binary
// ids: internal nodes 0 .. n-2, leaf k (sorted position k) at n-1+k.
__global__ void k_radix_tree(const uint64_t* keys, uint32_t n, Bin bn) {
  int64_t N = n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N - 1; i += (int64_t)gridDim.x * blockDim.x) {
    int d = delta(keys, N, i, i + 1) - delta(keys, N, i, i - 1) >= 0 ? 1 : -1;
    int dmin = delta(keys, N, i, i - d);
    int64_t lmax = 2;
    while (delta(keys, N, i, i + lmax * d) > dmin) lmax *= 2;
    int64_t l = 0;
    for (int64_t t = lmax / 2; t >= 1; t /= 2)
      if (delta(keys, N, i, i + (l + t) * d) > dmin) l += t;
    int64_t j = i + l * d;
    int dnode = delta(keys, N, i, j);
    int64_t s = 0, t = l;
    do {
      t = (t + 1) / 2;
      if (delta(keys, N, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    int64_t gamma = i + s * d + (d < 0 ? -1 : 0);
    int64_t lo = i < j ? i : j, hi = i < j ? j : i;
    int32_t left = (lo == gamma) ? (int32_t)(N - 1 + gamma) : (int32_t)gamma;
    int32_t right = (hi == gamma + 1) ? (int32_t)(N - 1 + gamma + 1) : (int32_t)(gamma + 1);
    bn.left[i] = left;
    bn.right[i] = right;
    bn.first[i] = (uint32_t)lo;
    bn.last[i] = (uint32_t)hi;
    bn.parent[left] = (int32_t)i;
    bn.parent[right] = (int32_t)i;
  }
}

// Boxes bottom-up: each leaf writes its box and climbs; the second child to
// arrive at a node computes the node's box and continues.
__global__ void k_boxes_up(const float* tlo, const float* thi, const uint32_t* vals, uint32_t n, Bin bn) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    uint32_t leaf = n - 1 + k, t = vals[k];
    for (int a = 0; a < 3; ++a) {
      bn.lo[3 * (size_t)leaf + a] = tlo[3 * (size_t)t + a];
      bn.hi[3 * (size_t)leaf + a] = thi[3 * (size_t)t + a];
    }
    bn.first[leaf] = k;
    bn.last[leaf] = k;
    bn.left[leaf] = -1;
    bn.right[leaf] = -1;
    __threadfence();
    int32_t p = n > 1 ? bn.parent[leaf] : -1;
    while (p >= 0) {
      if (atomicAdd(bn.flag + p, 1u) == 0) break;
      int32_t l = bn.left[p], r = bn.right[p];
      for (int a = 0; a < 3; ++a) {
        bn.lo[3 * (size_t)p + a] = fminf(__ldcg(bn.lo + 3 * (size_t)l + a), __ldcg(bn.lo + 3 * (size_t)r + a));
        bn.hi[3 * (size_t)p + a] = fmaxf(__ldcg(bn.hi + 3 * (size_t)l + a), __ldcg(bn.hi + 3 * (size_t)r + a));
      }
      __threadfence();
      p = p == 0 ? -1 : bn.parent[p];
    }
  }
}

// host/bvh_build.h decode_plane: origin + q * 2^(e-127), one rounding.
__device__ __forceinline__ float decode_plane(float origin, uint32_t q, uint32_t e) {
  return __fadd_rn(origin, __fmul_rn((float)q, __uint_as_float(e << 23)));
}
// Largest q with decode(q) <= v (host/bvh_build.cpp quant_lo).
__device__ uint32_t quant_lo(float origin, float v, uint32_t e) {
  double qd = floor(((double)v - (double)origin) / (double)__uint_as_float(e << 23));
  int q = (int)fmin(fmax(qd, 0.0), 255.0);
  while (q > 0 && decode_plane(origin, (uint32_t)q, e) > v) --q;
  while (q < 255 && decode_plane(origin, (uint32_t)(q + 1), e) <= v) ++q;
  return (uint32_t)q;
}
// Smallest q with decode(q) >= v; false when no byte reaches v.
__device__ bool quant_hi(float origin, float v, uint32_t e, uint32_t* out) {
  double qd = ceil(((double)v - (double)origin) / (double)__uint_as_float(e << 23));
  int q = (int)fmin(fmax(qd, 0.0), 255.0);
  while (q < 255 && decode_plane(origin, (uint32_t)q, e) < v) ++q;
  while (q > 0 && decode_plane(origin, (uint32_t)(q - 1), e) >= v) --q;
  if (decode_plane(origin, (uint32_t)q, e) < v) return false;
  *out = (uint32_t)q;
  return true;
}

struct Collapse {
  const int2* in;  // (wide node, binary node) of this level
  uint32_t n_in;
  int2* out;
  uint32_t* n_out;
  uint32_t* node_count;
  uint32_t* tri_count;
  uint4* nodes;  // 5 per wide node
  float4* tris;  // 3 per triangle
  const float4* pos;
  const uint4* tri;
  const uint32_t* vals;
  uint32_t* err;
};

__device__ __forceinline__ bool leafish(const Bin& bn, uint32_t n, int32_t b) {
  return (uint32_t)b >= n - 1 || bn.last[b] - bn.first[b] + 1 <= DB_LEAF_MAX;
}
__device__ __forceinline__ float half_area(const Bin& bn, int32_t b) {
  float e0 = bn.hi[3 * (size_t)b] - bn.lo[3 * (size_t)b], e1 = bn.hi[3 * (size_t)b + 1] - bn.lo[3 * (size_t)b + 1],
        e2 = bn.hi[3 * (size_t)b + 2] - bn.lo[3 * (size_t)b + 2];
  return e0 * e1 + e1 * e2 + e2 * e0;
}

// One level of the collapse: each item fills one wide node from the binary
// subtree below it (host/bvh_build.cpp Collapser::fill) and queues its
// interior children for the next level.
__global__ void k_collapse(Collapse c, Bin bn, uint32_t n) {
  for (uint32_t it = blockIdx.x * blockDim.x + threadIdx.x; it < c.n_in; it += gridDim.x * blockDim.x) {
    int2 item = c.in[it];
    int32_t kids[8];
    int nk = 0;
    if (leafish(bn, n, item.y)) {
      kids[nk++] = item.y;
    } else {
      kids[nk++] = bn.left[item.y];
      kids[nk++] = bn.right[item.y];
    }
    while (nk < 8) {
      int best = -1;
      float best_a = -1.0f;
      for (int i = 0; i < nk; ++i)
        if (!leafish(bn, n, kids[i])) {
          float a = half_area(bn, kids[i]);
          if (a > best_a) {
            best = i;
            best_a = a;
          }
        }
      if (best < 0) break;
      int32_t open = kids[best];
      for (int i = nk; i > best + 1; --i) kids[i] = kids[i - 1];
      kids[best] = bn.left[open];
      kids[best + 1] = bn.right[open];
      ++nk;
    }
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = 0; i < nk; ++i)
      for (int a = 0; a < 3; ++a) {
        lo[a] = fminf(lo[a], bn.lo[3 * (size_t)kids[i] + a]);
        hi[a] = fmaxf(hi[a], bn.hi[3 * (size_t)kids[i] + a]);
      }
    uint32_t e[3];
    for (int a = 0; a < 3; ++a) {
      float ext = hi[a] - lo[a];
      int ee = -120;
      if (ext > 0.0f) {
        int ex;
        frexp((double)ext / 255.0, &ex);
        ee = ex;
      }
      ee = max(ee, -120);
      if (ee > 60) {
        atomicOr(c.err, DB_ERR_EXTENT);
        ee = 60;
      }
      uint32_t qh;
      while (ee <= 60 && !quant_hi(lo[a], hi[a], (uint32_t)(ee + 127), &qh)) ++ee;
      if (ee > 60) {
        atomicOr(c.err, DB_ERR_QUANT);
        ee = 60;
      }
      e[a] = (uint32_t)(ee + 127);
    }
    uint32_t n_int = 0, n_tri = 0;
    for (int i = 0; i < nk; ++i) {
      if (leafish(bn, n, kids[i]))
        n_tri += bn.last[kids[i]] - bn.first[kids[i]] + 1;
      else
        ++n_int;
    }
    uint32_t child_base = n_int ? atomicAdd(c.node_count, n_int) : 0u;
    uint32_t tri_base = n_tri ? atomicAdd(c.tri_count, n_tri) : 0u;
    uint32_t imask = 0, present = 0, counts = 0;
    uint32_t q[6][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}, {0, 0}, {0, 0}};  // qlo x,y,z then qhi x,y,z
    uint32_t slot = 0, toff = 0;
    for (int i = 0; i < nk; ++i) {
      int32_t k = kids[i];
      present |= 1u << i;
      for (int a = 0; a < 3; ++a) {
        uint32_t ql = quant_lo(lo[a], bn.lo[3 * (size_t)k + a], e[a]);
        uint32_t qh = 255;
        if (!quant_hi(lo[a], bn.hi[3 * (size_t)k + a], e[a], &qh)) atomicOr(c.err, DB_ERR_QUANT);
        q[a][i >> 2] |= ql << (8 * (i & 3));
        q[3 + a][i >> 2] |= qh << (8 * (i & 3));
      }
      if (leafish(bn, n, k)) {
        uint32_t f = bn.first[k], l = bn.last[k];
        counts |= (l - f) << (4 * i);
        for (uint32_t s = f; s <= l; ++s) {
          uint32_t t = c.vals[s];
          uint4 ti = c.tri[t];
          float4 a = c.pos[ti.x], b = c.pos[ti.y], d = c.pos[ti.z];
          size_t o = 3 * (size_t)(tri_base + toff);
          c.tris[o] = make_float4(a.x, a.y, a.z, __uint_as_float(t));
          c.tris[o + 1] = make_float4(__fsub_rn(b.x, a.x), __fsub_rn(b.y, a.y), __fsub_rn(b.z, a.z), 0.0f);
          c.tris[o + 2] = make_float4(__fsub_rn(d.x, a.x), __fsub_rn(d.y, a.y), __fsub_rn(d.z, a.z), 0.0f);
          ++toff;
        }
      } else {
        imask |= 1u << i;
        uint32_t o = atomicAdd(c.n_out, 1u);
        c.out[o] = make_int2((int)(child_base + slot), k);
        ++slot;
      }
    }
    uint4* w = c.nodes + 5 * (size_t)item.x;
    w[0] = make_uint4(__float_as_uint(lo[0]), __float_as_uint(lo[1]), __float_as_uint(lo[2]),
                      e[0] | (e[1] << 8) | (e[2] << 16) | (imask << 24));
    w[1] = make_uint4(child_base, tri_base, counts, present);
    w[2] = make_uint4(q[0][0], q[0][1], q[1][0], q[1][1]);
    w[3] = make_uint4(q[2][0], q[2][1], q[3][0], q[3][1]);
    w[4] = make_uint4(q[4][0], q[4][1], q[5][0], q[5][1]);
  }
}

}  // namespace db
