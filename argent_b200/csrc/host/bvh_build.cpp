// bvh_build.cpp — host build of the compressed 8-wide BVH (see bvh_build.h).
//
// Binary stage: binned SAH over all three axes (16 bins), leaves of at most
// 4 triangles, built in parallel over subtrees.  Unlike argent's build
// (bvh.rs:419-495, longest axis only), every axis is binned, which gives a
// cheaper tree for the same triangles; closest hits do not depend on the tree.
// Past depth 48 the build falls back to median splits so the tree depth, and
// with it the device traversal stack, stays bounded.
//
// Wide stage: each wide node opens its largest-area interior child until it
// holds eight children (the rule argent's 4-wide collapse uses,
// bvh.rs:324-341, extended to eight), then quantises the children's boxes
// conservatively against the node origin.
#include "bvh_build.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <thread>

namespace argent {
namespace {

struct Box {
  float lo[3], hi[3];
  void reset() {
    for (int a = 0; a < 3; ++a) {
      lo[a] = INFINITY;
      hi[a] = -INFINITY;
    }
  }
  void grow(const Box& b) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], b.lo[a]);
      hi[a] = std::max(hi[a], b.hi[a]);
    }
  }
  void grow_pt(const float* p) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], p[a]);
      hi[a] = std::max(hi[a], p[a]);
    }
  }
  float half_area() const {
    float e0 = std::max(hi[0] - lo[0], 0.0f), e1 = std::max(hi[1] - lo[1], 0.0f), e2 = std::max(hi[2] - lo[2], 0.0f);
    return e0 * e1 + e1 * e2 + e2 * e0;
  }
};

struct BNode {
  Box box;
  int32_t left = -1, right = -1;
  uint32_t start = 0, count = 0;  // leaf when count > 0
  uint32_t span = 0;              // triangles of the subtree, at ref[start ..)
};

// Subtrees of at most this many triangles become one leaf of the wide tree
// (the binary build's triangles of a subtree are contiguous in `ref`).  A
// node visit costs several times a triangle test, so a wide node whose
// children are two leaves of two triangles is better as one leaf of four.
// Leaves hold at most 16 triangles (a 4-bit count).  0 keeps the binary
// tree's leaves.  Measured on B200 (eight lanes): merging subtrees of up to
// 4 triangles cut the signet's wide nodes from 298k to 222k and its node
// visits per path-sample from 3.80 to 3.68, with the signet unchanged
// (1.754-1.757 G path-samples/s against 1.755-1.759 G) and the gems 0.8 %
// faster; up to 6 or 8 triangles ran 1-6 % slower (more triangle tests on
// the dependent chain than node visits saved).
#ifndef ARGENT_LEAF_MERGE
#define ARGENT_LEAF_MERGE 4
#endif
static_assert(ARGENT_LEAF_MERGE <= 16, "wide-tree leaves hold at most 16 triangles");

const int BINS = 16;
const uint32_t MAX_LEAF = 4;
const int MEDIAN_DEPTH = 48;
const uint32_t PARALLEL_MIN = 1u << 16;

struct Builder {
  const std::vector<Box>& prim_box;
  const std::vector<float>& cent;  // 3 per prim
  std::vector<uint32_t>& ref;
  std::vector<BNode>& nodes;
  std::atomic<uint32_t> next{0};
  std::atomic<int> threads_left;

  Builder(const std::vector<Box>& pb, const std::vector<float>& c, std::vector<uint32_t>& r, std::vector<BNode>& n,
          int threads)
      : prim_box(pb), cent(c), ref(r), nodes(n), threads_left(threads) {}

  uint32_t alloc() { return next.fetch_add(1); }

  void make_leaf(uint32_t id, uint32_t begin, uint32_t end, const Box& b) {
    BNode& n = nodes[id];
    n.box = b;
    n.start = begin;
    n.count = end - begin;
    n.span = end - begin;
  }

  // Returns the split position or `begin` when the range should be a leaf.
  uint32_t split(uint32_t begin, uint32_t end, const Box& bounds, int depth) {
    uint32_t n = end - begin;
    Box cb;
    cb.reset();
    for (uint32_t i = begin; i < end; ++i) cb.grow_pt(&cent[3 * (size_t)ref[i]]);
    float ext[3] = {cb.hi[0] - cb.lo[0], cb.hi[1] - cb.lo[1], cb.hi[2] - cb.lo[2]};
    int long_axis = (ext[0] >= ext[1] && ext[0] >= ext[2]) ? 0 : (ext[1] >= ext[2] ? 1 : 2);
    auto median = [&]() {
      uint32_t mid = begin + n / 2;
      int a = long_axis;
      std::nth_element(ref.begin() + begin, ref.begin() + mid, ref.begin() + end,
                       [&](uint32_t x, uint32_t y) { return cent[3 * (size_t)x + a] < cent[3 * (size_t)y + a]; });
      return mid;
    };
    if (depth >= MEDIAN_DEPTH) return n <= MAX_LEAF ? begin : median();
    float best_cost = INFINITY;
    int best_axis = -1, best_bin = 0;
    for (int a = 0; a < 3; ++a) {
      if (!(ext[a] > 0.0f)) continue;
      Box bb[BINS];
      uint32_t bn[BINS] = {0};
      for (int i = 0; i < BINS; ++i) bb[i].reset();
      float k = (float)BINS / ext[a];
      for (uint32_t i = begin; i < end; ++i) {
        uint32_t p = ref[i];
        int b = (int)((cent[3 * (size_t)p + a] - cb.lo[a]) * k);
        b = std::min(std::max(b, 0), BINS - 1);
        bn[b]++;
        bb[b].grow(prim_box[p]);
      }
      float left_area[BINS];
      uint32_t left_n[BINS];
      Box acc;
      acc.reset();
      uint32_t cnt = 0;
      for (int i = 0; i < BINS - 1; ++i) {
        acc.grow(bb[i]);
        cnt += bn[i];
        left_area[i] = acc.half_area();
        left_n[i] = cnt;
      }
      acc.reset();
      cnt = 0;
      for (int i = BINS - 1; i >= 1; --i) {
        acc.grow(bb[i]);
        cnt += bn[i];
        uint32_t ln = left_n[i - 1];
        if (ln == 0 || cnt == 0) continue;
        float cost = left_area[i - 1] * (float)ln + acc.half_area() * (float)cnt;
        if (cost < best_cost) {
          best_cost = cost;
          best_axis = a;
          best_bin = i;
        }
      }
    }
    float leaf_cost = bounds.half_area() * (float)n;
    if (n <= MAX_LEAF && !(best_cost + bounds.half_area() < leaf_cost)) return begin;
    if (best_axis < 0) return n <= MAX_LEAF ? begin : median();
    int a = best_axis;
    float k = (float)BINS / ext[a];
    auto left_of = [&](uint32_t p) {
      int b = (int)((cent[3 * (size_t)p + a] - cb.lo[a]) * k);
      b = std::min(std::max(b, 0), BINS - 1);
      return b < best_bin;
    };
    uint32_t* mid = std::partition(ref.data() + begin, ref.data() + end, left_of);
    uint32_t m = (uint32_t)(mid - ref.data());
    if (m == begin || m == end) return n <= MAX_LEAF ? begin : median();
    return m;
  }

  void build(uint32_t id, uint32_t begin, uint32_t end, int depth) {
    Box b;
    b.reset();
    for (uint32_t i = begin; i < end; ++i) b.grow(prim_box[ref[i]]);
    uint32_t m = split(begin, end, b, depth);
    if (m == begin) {
      make_leaf(id, begin, end, b);
      return;
    }
    uint32_t l = alloc(), r = alloc();
    nodes[id].box = b;
    nodes[id].left = (int32_t)l;
    nodes[id].right = (int32_t)r;
    nodes[id].count = 0;
    nodes[id].start = begin;
    nodes[id].span = end - begin;
    if (end - begin >= PARALLEL_MIN && threads_left.fetch_sub(1) > 1) {
      std::thread t([&, l, begin, m, depth] { build(l, begin, m, depth + 1); });
      build(r, m, end, depth + 1);
      t.join();
      threads_left.fetch_add(1);
    } else {
      build(l, begin, m, depth + 1);
      build(r, m, end, depth + 1);
    }
  }
};

// Largest q with decode(q) <= v, and smallest q with decode(q) >= v.
uint8_t quant_lo(float origin, float v, uint8_t e) {
  union {
    uint32_t u;
    float f;
  } s;
  s.u = (uint32_t)e << 23;
  double qd = std::floor(((double)v - (double)origin) / (double)s.f);
  int q = (int)std::min(std::max(qd, 0.0), 255.0);
  while (q > 0 && decode_plane(origin, (uint8_t)q, e) > v) --q;
  while (q < 255 && decode_plane(origin, (uint8_t)(q + 1), e) <= v) ++q;
  return (uint8_t)q;
}
bool quant_hi(float origin, float v, uint8_t e, uint8_t* out) {
  union {
    uint32_t u;
    float f;
  } s;
  s.u = (uint32_t)e << 23;
  double qd = std::ceil(((double)v - (double)origin) / (double)s.f);
  int q = (int)std::min(std::max(qd, 0.0), 255.0);
  while (q < 255 && decode_plane(origin, (uint8_t)q, e) < v) ++q;
  while (q > 0 && decode_plane(origin, (uint8_t)(q - 1), e) >= v) --q;
  if (decode_plane(origin, (uint8_t)q, e) < v) return false;
  *out = (uint8_t)q;
  return true;
}

struct Collapser {
  const std::vector<BNode>& bn;
  const std::vector<uint32_t>& ref;
  const float* pos;
  const uint32_t* tris;
  WideBvh& out;

  TriRecord make_tri(uint32_t prim) const {
    const uint32_t* t = &tris[3 * (size_t)prim];
    TriRecord r;
    std::memset(&r, 0, sizeof(r));
    for (int a = 0; a < 3; ++a) {
      float v0 = pos[3 * (size_t)t[0] + a];
      r.v0[a] = v0;
      r.e1[a] = pos[3 * (size_t)t[1] + a] - v0;
      r.e2[a] = pos[3 * (size_t)t[2] + a] - v0;
    }
    r.prim = prim;
    return r;
  }

  // A binary node the wide tree stores as one leaf: a leaf, or a subtree
  // small enough to merge.  The collapse first opens binary nodes (largest
  // half-area first) until a wide node has eight children, so wide nodes
  // stay full; an interior child still left then becomes a leaf if it is
  // small enough, instead of a wide node of two or three small leaves.
  static bool as_leaf(const BNode& n) { return n.count > 0 || n.span <= (uint32_t)ARGENT_LEAF_MERGE; }
  static uint32_t leaf_count(const BNode& n) { return n.count > 0 ? n.count : n.span; }

  // Fills wide node `me` from binary node `root`; returns the depth below.
  uint32_t fill(uint32_t me, uint32_t root) {
    std::vector<uint32_t> kids;
    const BNode& r = bn[root];
    if (as_leaf(r))
      kids.push_back(root);
    else {
      kids.push_back((uint32_t)r.left);
      kids.push_back((uint32_t)r.right);
    }
    while (kids.size() < 8) {
      int best = -1;
      float best_a = -1.0f;
      for (size_t i = 0; i < kids.size(); ++i) {
        const BNode& n = bn[kids[i]];
        if (n.count == 0) {
          float a = n.box.half_area();
          if (a > best_a) {
            best = (int)i;
            best_a = a;
          }
        }
      }
      if (best < 0) break;
      uint32_t open = kids[best];
      kids[best] = (uint32_t)bn[open].left;
      kids.insert(kids.begin() + best + 1, (uint32_t)bn[open].right);
    }
    Box nb;
    nb.reset();
    for (uint32_t k : kids) nb.grow(bn[k].box);
    WideNode w;
    std::memset(&w, 0, sizeof(w));
    uint8_t e[3];
    for (int a = 0; a < 3; ++a) {
      w.origin[a] = nb.lo[a];
      float ext = nb.hi[a] - nb.lo[a];
      int ee;
      if (!(ext > 0.0f)) {
        ee = -120;
      } else {
        int ex;
        std::frexp((double)ext / 255.0, &ex);  // ext/255 = m * 2^ex, m in [0.5, 1)
        ee = ex;
      }
      ee = std::max(ee, -120);
      // The device slab test multiplies scale by 1/d (capped at 2^64);
      // scale <= 2^60 keeps that product finite.
      if (ee > 60) throw std::runtime_error("piece extent too large for the node quantisation");
      for (;;) {
        uint8_t eb = (uint8_t)(ee + 127);
        uint8_t qh;
        if (quant_hi(w.origin[a], nb.hi[a], eb, &qh)) break;
        ++ee;
      }
      e[a] = (uint8_t)(ee + 127);
    }
    w.ex = e[0];
    w.ey = e[1];
    w.ez = e[2];
    uint32_t n_interior = 0;
    for (uint32_t k : kids)
      if (!as_leaf(bn[k])) ++n_interior;
    uint32_t child_base = (uint32_t)out.nodes.size();
    out.nodes.resize(out.nodes.size() + n_interior);
    w.child_base = child_base;
    w.tri_base = (uint32_t)out.tris.size();
    for (size_t c = 0; c < kids.size(); ++c) {
      const BNode& k = bn[kids[c]];
      w.present |= 1u << c;
      for (int a = 0; a < 3; ++a) {
        w.qlo[a][c] = quant_lo(w.origin[a], k.box.lo[a], e[a]);
        uint8_t qh = 255;
        if (!quant_hi(w.origin[a], k.box.hi[a], e[a], &qh)) throw std::runtime_error("quantisation failed");
        w.qhi[a][c] = qh;
      }
      if (as_leaf(k)) {
        uint32_t cnt = leaf_count(k);
        if (cnt > 16) throw std::runtime_error("leaf larger than 16 triangles");
        w.leaf_counts |= (cnt - 1) << (4 * c);
        for (uint32_t i = k.start; i < k.start + cnt; ++i) out.tris.push_back(make_tri(ref[i]));
      } else {
        w.imask |= (uint8_t)(1u << c);
      }
    }
    out.nodes[me] = w;
    uint32_t depth = 1, slot = 0;
    for (size_t c = 0; c < kids.size(); ++c) {
      if (!as_leaf(bn[kids[c]])) {
        uint32_t d = 1 + fill(child_base + slot, kids[c]);
        depth = std::max(depth, d);
        ++slot;
      }
    }
    return depth;
  }
};

}  // namespace

WideBvh build_wide_bvh(const float* positions, uint32_t nv, const uint32_t* tris, uint32_t nt, int threads) {
  WideBvh out;
  if (nt == 0) return out;
  if (nt >= (1u << 27)) throw std::runtime_error("piece exceeds 2^27 triangles");
  for (uint64_t i = 0; i < 3ull * nt; ++i)
    if (tris[i] >= nv) throw std::runtime_error("triangle index out of range");
  std::vector<Box> pbox(nt);
  std::vector<float> cent(3 * (size_t)nt);
  for (uint32_t i = 0; i < nt; ++i) {
    Box b;
    b.reset();
    for (int k = 0; k < 3; ++k) b.grow_pt(&positions[3 * (size_t)tris[3 * (size_t)i + k]]);
    pbox[i] = b;
    for (int a = 0; a < 3; ++a) cent[3 * (size_t)i + a] = (b.lo[a] + b.hi[a]) * 0.5f;
  }
  std::vector<uint32_t> ref(nt);
  for (uint32_t i = 0; i < nt; ++i) ref[i] = i;
  std::vector<BNode> nodes(2 * (size_t)nt);
  if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  Builder b(pbox, cent, ref, nodes, std::min(threads, 64));
  uint32_t root = b.alloc();
  b.build(root, 0, nt, 0);
  nodes.resize(b.next.load());
  out.binary_nodes = nodes.size();
  for (int a = 0; a < 3; ++a) {
    out.lo[a] = nodes[root].box.lo[a];
    out.hi[a] = nodes[root].box.hi[a];
  }
  out.nodes.reserve(nodes.size() / 4 + 1);
  out.tris.reserve(nt);
  out.nodes.resize(1);
  Collapser c{nodes, ref, positions, tris, out};
  out.depth = c.fill(0, root);
  return out;
}

}  // namespace argent
