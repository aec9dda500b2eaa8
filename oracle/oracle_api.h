/*
 * oracle_api.h — C entry points of the CPU oracle (liboracle.so).
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle restates argent's render hot path on
 * the CPU (crates/argent-core/src/{render,integrator,scene,bvh,...}.rs).  Only
 * the tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it,
 * as the checker, never as the measured or shipped path.
 */
#ifndef ARGENT_ORACLE_API_H
#define ARGENT_ORACLE_API_H

#include <stdint.h>

#include "../include/argent_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_bvh oracle_bvh;
typedef struct oracle_scene oracle_scene;

/* BVH (bvh.rs) */
oracle_bvh* oracle_bvh_create(const float* positions, uint32_t nv, const uint32_t* tris, uint32_t nt);
void oracle_bvh_destroy(oracle_bvh* b);
void oracle_bvh_intersect(const oracle_bvh* b, const ArgentRay* rays, uint64_t n, ArgentHit* hits, int threads);
void oracle_bvh_occluded(const oracle_bvh* b, const ArgentRay* rays, uint64_t n, uint8_t* occ, int threads);
void oracle_bvh_intersect_binary(const oracle_bvh* b, const ArgentRay* rays, uint64_t n, ArgentHit* hits);
/* Moller-Trumbore against every triangle, keeping the first strict minimum. */
void oracle_brute_intersect(const float* positions, const uint32_t* tris, uint32_t nt, const ArgentRay* rays,
                            uint64_t n, ArgentHit* hits, int threads);
/* Does triangle `prim` (original index) give a hit at exactly t for ray r? */
int oracle_tri_hit(const float* positions, const uint32_t* tris, uint32_t prim, const ArgentRay* r, float* t,
                   float* u, float* v);
/* Node counts and the deepest traversal stack seen so far. */
void oracle_bvh_stats(const oracle_bvh* b, uint64_t* binary_nodes, uint64_t* wide_nodes, uint32_t* max_stack);

/* Scene and render (scene.rs, render.rs, integrator.rs) */
oracle_scene* oracle_scene_create(const float* positions, uint32_t nv, const float* normals, const uint32_t* tris,
                                  uint32_t nt, const uint16_t* tri_material, const float* cavity,
                                  const ArgentSceneDesc* desc);
void oracle_scene_destroy(oracle_scene* s);
void oracle_scene_set_turntable(oracle_scene* s, float deg);
void oracle_render_pass(const oracle_scene* sc, const ArgentCamera* cam, const ArgentPathSettings* ps, uint32_t w,
                        uint32_t h, uint32_t first, uint32_t count, uint32_t seed, uint32_t y0, uint32_t y1,
                        float* color, float* albedo, float* normal, double* xyz, int threads);
void oracle_trace_sample(const oracle_scene* sc, const ArgentCamera* cam, const ArgentPathSettings* ps, uint32_t w,
                         uint32_t h, uint32_t x, uint32_t y, uint32_t si, uint32_t seed, float* xyz_out);
void oracle_camera_matrix(int has_white, const float* white, float* out9);

/* Cavity mask (argent-mesh cavity.rs; AO on argent's BVH) */
void oracle_smooth_vertex_normals(const float* pos, uint32_t nv, const uint32_t* tris, uint32_t nt, float* out);
void oracle_ambient_occlusion(const float* pos, uint32_t nv, const float* normals, const uint32_t* tris, uint32_t nt,
                              uint32_t samples, float distance, float* out);
void oracle_concavity(const float* pos, uint32_t nv, const float* normals, const uint32_t* tris, uint32_t nt,
                      float radius, float* out);
void oracle_smooth(const float* pos, uint32_t nv, const uint32_t* tris, uint32_t nt, float* values,
                   uint32_t iterations, float lambda);
void oracle_patina_mask(const float* pos, uint32_t nv, const float* normals, const uint32_t* tris, uint32_t nt,
                        uint32_t ao_samples, float ao_distance, float curvature_radius, float concavity_weight,
                        uint32_t smooth_iterations, float* out);

/* À-trous denoiser (argent-post denoise.rs:535-712); albedo/normal may be NULL */
void oracle_atrous(uint32_t w, uint32_t h, const float* color, const float* albedo, const float* normal, float* out);

/* Tone mapping and develop (argent-post tonemap.rs, color.rs) */
void oracle_tonemap_pixel(const float* rgb, float ev, int op, int look, float saturation, float* out);
float oracle_srgb_encode(float x);
void oracle_develop(const float* rgb, uint64_t n, float ev, int op, int look, float saturation, float* enc_out,
                    uint8_t* out8);

/* Primitives, for argent's unit-test known answers */
float oracle_fresnel_dielectric(float c, float eta);
float oracle_fresnel_conductor(float c, float eta, float k);
float oracle_ggx_e(float roughness, float cos_o);
void oracle_ggx_sample_h(float roughness, const float* wo, float u1, float u2, float* h_out);
void oracle_energy_table(float* out1024);
void oracle_sample_visible(float u, float* lambda4, float* pdf4);
void oracle_to_xyz(const float* l4, const float* lambda4, const float* pdf4, float* xyz);
void oracle_xyz_bar(float lambda, float* out3);
void oracle_linear_rgb(float* basis3x471, float* inv9);
uint32_t oracle_hash32(uint32_t x);
void oracle_sampler_next(uint32_t pixel_seed, uint32_t index, uint32_t ndims, float* out);
void oracle_sampler_random(uint32_t pixel_seed, uint32_t index, uint32_t n, float* out);
void oracle_sobol_4d(uint32_t index, uint32_t set, uint32_t seed, float* out4);
void oracle_sobol_raw(uint32_t index, int dim, uint32_t* out);

#ifdef __cplusplus
}
#endif

#endif
