/*
 * argent_host.h — host-side helpers that build the plain-old-data
 * descriptions argent_gpu.h consumes (libargent_host.so, no CUDA needed).
 *
 * In argent these are the callers' own Rust routines: argent-spectra's table
 * builders (alloys, gems, sigmoid albedo, blackbody emitters), argent-core's
 * studio rigs, camera and framing, and argent-mesh's synthetic meshes.  When
 * argent calls the GPU library through its FFI crate it keeps its own Rust
 * versions and passes their tables.  This library restates them in C++ so
 * the C++/Python side (tests, benchmark, serve loop) can build the same
 * inputs.  Each function names the argent routine it restates.
 */
#ifndef ARGENT_HOST_H
#define ARGENT_HOST_H

#include <stdint.h>

#include "argent_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- meshes */

/* A triangle mesh in caller-freeable memory (argent_mesh_free). */
typedef struct ArgentMesh {
  uint32_t nv;
  uint32_t nt;
  float* positions;       /* nv*3 */
  float* normals;         /* nv*3, smooth (area-weighted) vertex normals */
  uint32_t* tris;         /* nt*3 */
  uint16_t* tri_material; /* nt */
} ArgentMesh;

void argent_mesh_free(ArgentMesh* m);

/*
 * Procedural ring: `synth::torus_profile` (argent-mesh/src/synth.rs:153-173)
 * around Z with major radius R and tube radius r, nu x nv quads
 * (2*nu*nv triangles), each vertex pushed along its tube normal by
 * amp * (2*noise - 1), noise = smooth 3D value noise on a lattice of cell
 * `cell_mm` whose lattice values come from argent's hash32 (sampler.rs:18-25)
 * with `seed`.
 */
int argent_synth_ring(float R, float r, uint32_t nu, uint32_t nv, float amp, float cell_mm, uint32_t seed,
                      ArgentMesh* out);

/*
 * Signet ring: the same torus with the top flattened into a bezel_w x
 * bezel_d mm plate (centred on +Y, normal +Y) embossed by a seeded 2D Perlin
 * heightfield of amplitude `emboss_mm`; nu x nv quads.  Triangles get
 * material 0 or 1 from a seeded value-noise mask (polished / satin).
 */
int argent_synth_signet(float R, float r, uint32_t nu, uint32_t nv, float bezel_w, float bezel_d, float emboss_mm,
                        uint32_t seed, uint32_t mask_seed, ArgentMesh* out);

#ifdef __cplusplus
}
#endif

#endif /* ARGENT_HOST_H */
