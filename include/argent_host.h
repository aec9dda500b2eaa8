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


/* ---------------------------------------------------------------- spectra
 * Tables are 1 nm over 360..=830 nm (ARGENT_SPEC_LEN); n,k rows are the
 * 5 nm grid (ARGENT_NK_LEN). */

/* metals::get (spectra/src/metals.rs:165): measured n,k of a pure metal. */
int argent_metal_nk(const char* name, float* eta, float* k);
/* Alloy::from_name + Alloy::ior (spectra/src/alloys.rs:142-171, 260-280). */
int argent_alloy_nk(const char* name, float* eta, float* k);
/* karat_gold (alloys.rs:423-460): mass fractions of Au, Ag, Cu. */
int argent_karat_gold_nk(float au, float ag, float cu, float* eta, float* k);
/* ComplexIor::f0_srgb (metals.rs:102-107). */
void argent_nk_f0_srgb(const float* eta, const float* k, float* rgb);
/* luminance_y of a 1 nm table (spectra/src/spectrum.rs:413-420). */
float argent_luminance_y(const float* table);
/* studio::emitter (core/src/studio.rs:15-25): blackbody at `kelvin`,
 * luminance-normalised, times `intensity`, baked to 1 nm (tab.rs:30). */
void argent_bake_emitter(float kelvin, float intensity, float* out);
/* RgbAlbedo::new baked to 1 nm (spectrum.rs:194-233). */
void argent_bake_rgb_albedo(const float* rgb, float* out);
/* RgbAlbedo coefficients in normalised wavelength; returns 0 for a grey. */
int argent_rgb_albedo_coefficients(const float* rgb, float* c3);
/* RgbIlluminant::new baked to 1 nm (spectrum.rs:395-409). */
void argent_bake_rgb_illuminant(const float* rgb, float* out);
/* cie::reflectance_srgb of a 1 nm table (spectra/src/cie.rs:156-172). */
void argent_reflectance_srgb(const float* table, float* rgb);
/* color::blackbody_white (core/src/color.rs:32-45): XYZ with Y = 1. */
void argent_blackbody_white(float kelvin, float* xyz);
/* gems::get (spectra/src/gems.rs:395-440): kind, n(lambda) and absorption
 * (1/mm) baked to 1 nm; body_rgb = -1 when the stone has no body colour. */
int argent_gem_tables(const char* name, int32_t* kind, float* ior, float* absorption, float* body_rgb);
/* GemOptics::n_d / fire / dispersion_bg (gems.rs:115-140). */
int argent_gem_dispersion(const char* name, float* n_d, float* fire, float* bg);

/* ---------------------------------------------------------------- materials
 * The `Material` constructors (core/src/material.rs:38-153). */

/* Material::metal(alloy, roughness).with_patina(default_patina(s, alloy));
 * patina_strength < 0 leaves the patina off. */
int argent_material_metal(const char* alloy, float roughness, float patina_strength, ArgentMaterial* out);
/* A metal from explicit n,k rows. */
int argent_material_metal_nk(const float* eta, const float* k, float roughness, ArgentMaterial* out);
/* Material::gem (material.rs:50-60): opal names give the opal material. */
int argent_material_gem(const char* name, ArgentMaterial* out);
/* Material::opal (material.rs:63-66). */
void argent_material_opal(int black, float cell_mm, ArgentMaterial* out);
/* Material::plastic (material.rs:73-75). */
void argent_material_plastic(const float* rgb, float eta, float roughness, ArgentMaterial* out);
/* Material::diffuse (material.rs:77-79). */
void argent_material_diffuse(const float* rgb, ArgentMaterial* out);
/* Material::Black. */
void argent_material_black(ArgentMaterial* out);

/* ---------------------------------------------------------------- studio, camera */

/* Studio::build(radius) + floor_at (core/src/studio.rs:252-362): up to 16
 * panels, the gradient environment, the floor's material and placement
 * (floor->material is left -1 for the caller to set), and the white point
 * (has_white = 0 keeps the rig's colour). */
int argent_studio_build(const char* name, float radius, float floor_y, ArgentPanel* panels, int32_t* num_panels,
                        ArgentEnv* env, ArgentMaterial* floor_material, ArgentFloor* floor, int32_t* has_white,
                        float* white_xyz);
/* Camera::look_at (core/src/camera.rs:38-54). */
void argent_camera_look_at(const float* pos, const float* target, const float* up_hint, float focal_mm, float f_stop,
                           float aspect, ArgentCamera* out);
/* View::named (core/src/views.rs:17-30). */
int argent_view_named(const char* name, float* azimuth_deg, float* elevation_deg, float* fill);
/* views::frame (core/src/views.rs:45-83). */
void argent_frame(const float* points, uint32_t n, float azimuth_deg, float elevation_deg, float fill, float focal_mm,
                  float f_stop, float aspect, ArgentCamera* out);
/* Seeded synthetic equirect HDRI (linear sRGB, width*height*3): lognormal
 * texels of log-sigma `sigma` plus three hot lobes.  Stands in for a
 * photographed HDR, which the workloads do not ship. */
void argent_synth_hdri(uint32_t width, uint32_t height, float sigma, uint32_t seed, float* rgb);

/*
 * Gems workload piece: a torus shank (shank_nu x shank_nv quads) with 37
 * prong cups (a torus collar and four torus prongs each), one round
 * brilliant of girdle radius center_mm on top and 36 brilliants of girdle
 * radius stone_mm around the shank.  The brilliant is the polytope of its
 * facet half-spaces: table, 8 stars, 8 bezels, 16 upper and 16 lower girdle
 * halves, 8 pavilion mains (57 facets) and a 32-facet girdle band.
 * Material slots: 0 metal, 1 centre stone, 2..5 side stones (by seed).
 */
int argent_synth_gem_ring(uint32_t shank_nu, uint32_t shank_nv, float center_mm, float stone_mm, uint32_t seed,
                          ArgentMesh* out);

#ifdef __cplusplus
}
#endif

#endif /* ARGENT_HOST_H */
