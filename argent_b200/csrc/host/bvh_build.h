// bvh_build.h — host build of the compressed 8-wide BVH the CUDA traversal
// reads.  Replaces argent's binned-SAH binary build + 4-wide collapse
// (crates/argent-core/src/bvh.rs:117-146, 303-378, 419-533) with a layout
// sized for B200 memory transactions: 80-byte nodes (five 16-byte loads)
// holding eight children whose boxes are quantised to 8 bits per plane
// against the node's origin and a power-of-two scale per axis.
#pragma once
#include <cstdint>
#include <vector>

namespace argent {

// One wide node, 80 bytes, 16-byte aligned (five uint4 loads on the device).
//  word 0..2  origin x, y, z (float)
//  word 3     exponent bytes ex, ey, ez (biased like an IEEE float exponent:
//             scale = 2^(e-127)) and the interior-child mask
//  word 4     child_base: index of the first interior child; interior child i
//             lives at child_base + popcount(imask & ((1<<i)-1))
//  word 5     tri_base: first triangle of this node's leaves; leaf children
//             store their triangles contiguously in slot order
//  word 6     leaf counts: nibble i = (triangles in leaf child i) - 1
//  word 7     present mask (low byte): which of the 8 slots hold a child
//  bytes 32..79  qlo_x[8] qlo_y[8] qlo_z[8] qhi_x[8] qhi_y[8] qhi_z[8]
struct alignas(16) WideNode {
  float origin[3];
  uint8_t ex, ey, ez, imask;
  uint32_t child_base;
  uint32_t tri_base;
  uint32_t leaf_counts;
  uint32_t present;
  uint8_t qlo[3][8];
  uint8_t qhi[3][8];
};
static_assert(sizeof(WideNode) == 80, "wide node must be 80 bytes");

// Moller-Trumbore triangle record in BVH order: v0 (w = original triangle
// index as raw bits), e1 = v1 - v0, e2 = v2 - v0, all computed in f32 as
// argent does (bvh.rs:135-143).
struct alignas(16) TriRecord {
  float v0[3];
  uint32_t prim;
  float e1[3];
  uint32_t pad0;
  float e2[3];
  uint32_t pad1;
};
static_assert(sizeof(TriRecord) == 48, "triangle record must be 48 bytes");

struct WideBvh {
  std::vector<WideNode> nodes;
  std::vector<TriRecord> tris;
  uint32_t depth = 0;        // interior levels on the deepest root-to-leaf path
  float lo[3] = {0, 0, 0};   // root bounds (argent's Bvh::bounds, bvh.rs:148-151)
  float hi[3] = {0, 0, 0};
  uint64_t binary_nodes = 0;
};

// Decode one quantised plane exactly as the device does.
inline float decode_plane(float origin, uint8_t q, uint8_t e) {
  union {
    uint32_t u;
    float f;
  } s;
  s.u = (uint32_t)e << 23;
  volatile float prod = (float)q * s.f;  // exact: q <= 255 times a power of two
  return origin + prod;
}

// Builds the wide BVH.  `threads` <= 0 uses the hardware concurrency.
WideBvh build_wide_bvh(const float* positions, uint32_t nv, const uint32_t* tris, uint32_t nt, int threads);

}  // namespace argent
