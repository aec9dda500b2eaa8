// tables.cuh — device-resident lookup tables, filled by the host at context
// creation with cudaMemcpyToSymbol (the library is one translation unit, so
// the definitions live here rather than behind extern declarations).
#pragma once
#include <cstdint>

namespace dev {

// Sobol direction numbers of the sampler's four dimensions, [dim][bit].
__device__ uint32_t d_sobol_dirs[4][32];
// The same generator matrices applied a byte at a time: entry [dim][k][v]
// is the XOR of the direction numbers of the set bits of v << 8k, so a
// 32-bit index costs four lookups per dimension.
__device__ uint32_t d_sobol_bytes[4][4][256];
// GGX single-scattering albedo E(mu, sqrt(alpha)), 32 x 32 (microfacet.rs:93-140).
__device__ float d_energy_table[32 * 32];
// CIE 1931 2-degree colour matching functions, 1 nm, 360..=830 (cie.rs:38-49).
__device__ float d_cmf[471 * 3];
// Traversal instrumentation (off unless the host enables it): closest-hit
// rays, nodes, triangles; any-hit rays, nodes, triangles.
__device__ int d_trav_counting;
__device__ unsigned long long d_trav_counts[6];
// Rays by node visits (bins 0, 1, 2-3, 4-7, 8-15, 16-63, 64-255, 256+),
// closest-hit then any-hit, and the largest visit count of each kind.
__device__ unsigned long long d_trav_hist[16];
__device__ unsigned int d_trav_max[2];
// Node visits by the number of children whose box the ray enters (0..8),
// closest-hit then any-hit.
__device__ unsigned long long d_trav_child_hits[18];
// Paths entering each bounce and shadow rays queued at each bounce (64
// bounces, the path depth limit), summed over the waves run while counting
// is on.
#define ARGENT_BOUNCE_BINS 64
__device__ unsigned long long d_bounce_counts[2 * ARGENT_BOUNCE_BINS];

}  // namespace dev
