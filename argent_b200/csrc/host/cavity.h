// cavity.h — host half of the per-vertex patina mask (argent-mesh cavity.rs).
#pragma once
#include <cstdint>

namespace argent {

// Angle-weighted vertex normals (normals.rs:226-242); out has 3 * nv floats.
void smooth_vertex_normals(const float* pos, uint32_t nv, const uint32_t* tris, uint32_t nt, float* out);
// Signed concavity per vertex (cavity.rs:137-236).
void concavity(const float* pos, uint32_t nv, const uint32_t* tris, uint32_t nt, const float* normals, float radius,
               float* out);
// Laplacian smoothing over welded positions (cavity.rs:241-299).
void smooth_values(const float* pos, uint32_t nv, const uint32_t* tris, uint32_t nt, float* values,
                   uint32_t iterations, float lambda);
// Contrast blend of AO and concavity, smoothed and clamped (cavity.rs:52-78).
void patina_blend(const float* pos, uint32_t nv, const uint32_t* tris, uint32_t nt, const float* ao, const float* cav,
                  float concavity_weight, uint32_t smooth_iterations, float* out);

}  // namespace argent
