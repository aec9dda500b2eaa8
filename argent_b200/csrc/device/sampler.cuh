// sampler.cuh — argent's per-sample dimension stream on the device
// (crates/argent-core/src/sampler.rs:5-100).
//
// Dimensions below 256 of samples with index < 2^16 come from an
// Owen-scrambled Sobol sequence evaluated four dimensions at a time; the rest
// come from argent's PCG-XSH-RR stream.  argent gets the Sobol values from the
// sobol_burley 0.5.0 crate, which is not vendored.  This file implements the
// published method instead (Burley 2020, "Practical Hash-based Owen
// Scrambling", JCGT 9(4)): index shuffling by nested uniform scrambling, the
// first four Sobol dimensions, and an independent scramble per 4-dimension
// set (padding).  The direction numbers of those four dimensions come from
// the primitive polynomials x+1, x^2+x+1 and x^3+x+1.
#pragma once
#include <cstdint>

#include "dev_math.cuh"
#include "tables.cuh"

namespace dev {

#define ARGENT_SOBOL_MAX_DIM 256u


__device__ __forceinline__ uint32_t hash32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
__device__ __forceinline__ uint32_t lk_permutation(uint32_t x, uint32_t seed) {
  x += seed;
  x ^= x * 0x6c50b47cu;
  x ^= x * 0xb82f1e52u;
  x ^= x * 0xc7afe638u;
  x ^= x * 0x8d22f6e6u;
  return x;
}
__device__ __forceinline__ uint32_t nested_uniform_scramble(uint32_t x, uint32_t seed) {
  return __brev(lk_permutation(__brev(x), seed));
}
__device__ __forceinline__ uint32_t hash_combine(uint32_t seed, uint32_t v) {
  return seed ^ (v + 0x9e3779b9u + (seed << 6) + (seed >> 2));
}
__device__ __forceinline__ uint32_t sobol_dim(uint32_t index, int d) {
  const uint32_t* t = &d_sobol_bytes[d][0][0];
  return __ldg(t + (index & 0xffu)) ^ __ldg(t + 256 + ((index >> 8) & 0xffu)) ^
         __ldg(t + 512 + ((index >> 16) & 0xffu)) ^ __ldg(t + 768 + (index >> 24));
}
__device__ __forceinline__ void sample_4d(uint32_t index, uint32_t set, uint32_t seed, float out[4]) {
  uint32_t sseed = hash_combine(seed, hash32(set));
  uint32_t shuffled = nested_uniform_scramble(index, sseed);
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    uint32_t x = sobol_dim(shuffled, d);
    x = nested_uniform_scramble(x, hash_combine(sseed, hash32((uint32_t)d + 1u)));
    out[d] = (float)(x >> 8) * (1.0f / 16777216.0f);
  }
}

struct Sampler {
  uint32_t index, seed, dim;
  uint64_t rng;
  uint32_t block_set;
  float block[4];

  __device__ __forceinline__ void init(uint32_t pixel_seed, uint32_t sample_index) {
    index = sample_index;
    seed = pixel_seed;
    dim = 0;
    rng = (((uint64_t)pixel_seed << 32) | (uint64_t)sample_index) ^ 0x9e3779b97f4a7c15ull;
    block_set = 0xffffffffu;
  }
  // Resume a path: the PCG state travels with the path between kernels.
  __device__ __forceinline__ void resume(uint32_t pixel_seed, uint32_t sample_index, uint64_t rng_state) {
    index = sample_index;
    seed = pixel_seed;
    dim = 0;
    rng = rng_state;
    block_set = 0xffffffffu;
  }
  __device__ __forceinline__ float next_random() {
    rng = rng * 6364136223846793005ull + 1442695040888963407ull;
    uint64_t x = ((rng >> 18) ^ rng) >> 27;
    uint32_t rot = (uint32_t)(rng >> 59);
    uint32_t v = __funnelshift_r((uint32_t)x, (uint32_t)x, rot);
    return (float)(v >> 8) * (1.0f / 16777216.0f);
  }
  __device__ __forceinline__ float next() {
    uint32_t d = dim;
    dim += 1;
    if (d < ARGENT_SOBOL_MAX_DIM && index < (1u << 16)) {
      uint32_t set = d >> 2;
      if (set != block_set) {
        sample_4d(index, set, seed, block);
        block_set = set;
      }
      uint32_t k = d & 3u;
      float v = k == 0 ? block[0] : (k == 1 ? block[1] : (k == 2 ? block[2] : block[3]));
      return fminf(v, 0.99999994f);
    }
    return next_random();
  }
  __device__ __forceinline__ void set_dim(uint32_t d) { dim = d; }
};

// sampler.rs:103-108
__device__ __forceinline__ float tent(float u, float r) {
  float uu = 2.0f * u;
  if (uu < 1.0f) return r * (sqrtf(uu) - 1.0f);
  return r * (1.0f - sqrtf(2.0f - uu));
}
// sampler.rs:111-124
__device__ __forceinline__ void disk(float u, float v, float* ox, float* oy) {
  float a = 2.0f * u - 1.0f;
  float b = 2.0f * v - 1.0f;
  if (a == 0.0f && b == 0.0f) {
    *ox = 0.0f;
    *oy = 0.0f;
    return;
  }
  float r, phi;
  if (fabsf(a) > fabsf(b)) {
    r = a;
    phi = (ARGENT_PI_F / 4.0f) * (b / a);
  } else {
    r = b;
    phi = (ARGENT_PI_F / 2.0f) - (ARGENT_PI_F / 4.0f) * (a / b);
  }
  float s, c;
  sincosf(phi, &s, &c);
  *ox = r * c;
  *oy = r * s;
}
// sampler.rs:127-132
__device__ __forceinline__ V3 cosine_hemisphere(float u, float v) {
  float x, y;
  disk(u, v, &x, &y);
  float z = sqrtf(fmaxf(1.0f - x * x - y * y, 0.0f));
  return V3{x, y, z};
}

}  // namespace dev
