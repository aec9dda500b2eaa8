/*
 * argent_gpu.h — C ABI of the B200 spectral path tracer.
 *
 * This is the drop-in boundary for argent's render hot path.  argent calls
 * `render_pass(scene, cam, film, ps, count, seed)`
 * (crates/argent-core/src/render.rs:67) and
 * `render_image(scene, cam, q, seed)` (crates/argent-core/src/shot.rs:424) as
 * plain Rust functions.  A Rust FFI crate binds the functions below in their
 * place.  Everything above the boundary stays on argent's side: mesh loading,
 * posing, the spectral table builders in argent-spectra, the studio rigs,
 * framing, denoise and tone mapping.  Those produce the plain-old-data
 * descriptions declared here.
 *
 * Conventions:
 *  - Every function returns an int status (ARGENT_OK or ARGENT_E_*).  The
 *    text of the last failure is available from argent_last_error(ctx), or
 *    from argent_last_error(NULL) for failures before a context exists.
 *  - No exception or panic crosses the ABI.
 *  - Handles own device memory.  The caller owns all host arrays.  Uploads
 *    copy them, so a host array may be freed when the call returns.
 *  - A context owns one CUDA stream and is not thread-safe.  Use one
 *    context per worker thread.
 *  - Units are millimetres and nanometres, as in argent.
 */
#ifndef ARGENT_GPU_H
#define ARGENT_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Spectral sampling conventions of argent-spectra. */
#define ARGENT_SPEC_LEN 471  /* 1 nm table over 360..=830 nm (core/src/tab.rs:8-27) */
#define ARGENT_NK_LEN 95     /* 5 nm grid over 360..=830 nm (spectra/src/metals.rs:53-56) */

/* Status codes. */
enum {
  ARGENT_OK = 0,
  ARGENT_E_OOM = 1,      /* device or host allocation failed */
  ARGENT_E_INVALID = 2,  /* bad argument or malformed description */
  ARGENT_E_TIMEOUT = 3,  /* a bounded device wait ran out */
  ARGENT_E_CUDA = 4,     /* a CUDA runtime call failed */
  ARGENT_E_OVERFLOW = 5, /* a traversal stack or queue overflowed (recorded, not trapped) */
  ARGENT_E_BUSY = 6      /* admission refused: not enough device memory budget */
};

typedef struct ArgentCtx ArgentCtx;
typedef struct ArgentPiece ArgentPiece;
typedef struct ArgentScene ArgentScene;
typedef struct ArgentFilm ArgentFilm;

/* ------------------------------------------------------------------ */
/* Scene description (argent-core scene.rs / material.rs / light.rs). */
/* ------------------------------------------------------------------ */

/* Material kinds: the variants of `Material` (core/src/material.rs:27-36). */
enum {
  ARGENT_MAT_METAL = 0,
  ARGENT_MAT_GEM = 1,
  ARGENT_MAT_PLASTIC = 2,
  ARGENT_MAT_OPAL = 3,
  ARGENT_MAT_DIFFUSE = 4,
  ARGENT_MAT_BLACK = 5
};

/* `GemKind` (spectra/src/gems.rs:86-93). */
enum { ARGENT_GEM_TRANSPARENT = 0, ARGENT_GEM_OPAL = 1, ARGENT_GEM_OPAQUE = 2 };

/*
 * One material slot.  The fields a kind does not use are ignored.
 *  METAL:   nk_eta/nk_k = the alloy's n,k on the 5 nm grid (`ComplexIor`),
 *           alpha = GGX alpha.  Optional patina (material.rs:15-24):
 *           spec_a = tarnish base albedo (1 nm table).
 *  GEM:     spec_a = n(lambda) (1 nm table), spec_b = absorption in 1/mm
 *           (1 nm table).  For ARGENT_GEM_OPAQUE, spec_b2 = body albedo table
 *           when has_opaque_base, else a constant 0.01 is used (material.rs:127-131).
 *  PLASTIC: spec_a = base albedo table, eta, alpha.
 *  OPAL:    spec_a = body albedo table, cell_mm, strength.
 *  DIFFUSE: spec_a = albedo table.
 *  BLACK:   nothing.
 * `alpha` is already mapped from perceptual roughness
 * (alpha = max(clamp(r,0,1)^2, 1e-4), microfacet.rs:22-25).
 */
typedef struct ArgentMaterial {
  int32_t kind;
  int32_t gem_kind;
  float alpha;
  float eta;
  float cell_mm;
  float strength;
  int32_t has_patina;
  float patina_strength;
  float patina_lo;
  float patina_hi;
  float patina_alpha;
  float patina_eta;
  int32_t has_opaque_base;
  float nk_eta[ARGENT_NK_LEN];
  float nk_k[ARGENT_NK_LEN];
  float spec_a[ARGENT_SPEC_LEN];
  float spec_b[ARGENT_SPEC_LEN];
  float spec_b2[ARGENT_SPEC_LEN];
} ArgentMaterial;

/*
 * A rectangular softbox or flag (`Panel`, core/src/light.rs:10-27).
 * The library derives n = normalize(hu x hv) and area = 4 |hu x hv|
 * exactly as `Panel::new` (light.rs:30-33) does.
 */
typedef struct ArgentPanel {
  float center[3];
  float hu[3];
  float hv[3];
  int32_t emits;          /* 0 = flag (black card) */
  int32_t camera_visible;
  float feather;
  float emission[ARGENT_SPEC_LEN]; /* radiance table when emits */
} ArgentPanel;

/* `Env` (light.rs:103-109). */
enum { ARGENT_ENV_GRADIENT = 0, ARGENT_ENV_MAP = 1 };

typedef struct ArgentEnv {
  int32_t kind;
  /* Gradient: tables for the three bands and the blend power. */
  float power;
  float top[ARGENT_SPEC_LEN];
  float horizon[ARGENT_SPEC_LEN];
  float bottom[ARGENT_SPEC_LEN];
  /* Map: equirectangular linear-sRGB texels, exposure already applied,
   * row-major, width*height*3 floats (envmap.rs:141-177 input). */
  int32_t width;
  int32_t height;
  const float* rgb;
  float rotation_deg;
} ArgentEnv;

/* `Floor` (light.rs:133-138). */
typedef struct ArgentFloor {
  int32_t enabled;
  float y;
  int32_t material;
  float fade_start;
  float fade_end;
} ArgentFloor;

/* Everything `Scene::new` takes besides the piece (scene.rs:47-64, 82). */
typedef struct ArgentSceneDesc {
  const ArgentMaterial* materials;
  int32_t num_materials;
  const ArgentPanel* panels;
  int32_t num_panels;
  const ArgentEnv* env;
  ArgentFloor floor;
  float turntable_deg;
  int32_t has_white;   /* 0 = D65 (scene.white = None) */
  float white_xyz[3];
} ArgentSceneDesc;

/* `Camera` (core/src/camera.rs:17-29): a plain copy of its fields. */
typedef struct ArgentCamera {
  float pos[3];
  float forward[3];
  float right[3];
  float up[3];
  float half_w;
  float half_h;
  float lens_radius;
  float focus_dist;
  float shift[2];
} ArgentCamera;

/* `PathSettings` (core/src/integrator.rs:10-24). */
typedef struct ArgentPathSettings {
  uint32_t max_depth;
  float clamp_indirect;
  uint32_t rr_depth;
} ArgentPathSettings;

/* A ray for the traversal entry points: origin, t_max, direction. */
typedef struct ArgentRay {
  float o[3];
  float tmax;
  float d[3];
  float pad;
} ArgentRay;

/* Closest-hit result; prim = ARGENT_NO_HIT on a miss (bvh.rs:63-70). */
#define ARGENT_NO_HIT 0xFFFFFFFFu
typedef struct ArgentHit {
  float t;
  float u;
  float v;
  uint32_t prim;
} ArgentHit;

/* Context limits; zero fields take defaults.  Path state is 244 bytes per
 * slot per lane and grows on demand to what a render needs, so the defaults
 * (8 lanes of 2^24 slots) hold about 33 GB once a large frame has run. */
typedef struct ArgentLimits {
  uint64_t wave_paths;      /* path slots per wavefront wave (default 2^24, at most 2^30) */
  uint64_t memory_budget;   /* bytes the serve loop may hold (default 3/4 of free) */
  uint32_t lanes;           /* concurrent waves, each with its own stream and path state (default 8, at most 16) */
  uint32_t reserved;
} ArgentLimits;

/* Film flags. */
enum {
  ARGENT_FILM_KAHAN = 1,      /* FP32 sums with Kahan compensation (default) */
  ARGENT_FILM_FP64 = 2,       /* FP64 sums (oracle-grade accumulation) */
  ARGENT_FILM_PROGRESSIVE = 4 /* with KAHAN: FP64 sums join once a pass takes the film past
                                 ARGENT_FILM_FP64_AFTER samples (long progressive renders),
                                 seeded with the compensated FP32 sums */
};
#define ARGENT_FILM_FP64_AFTER 4096

/* ------------------------------------------------------------------ */
/* Context, piece, scene, film.                                       */
/* ------------------------------------------------------------------ */

/* New context on `device`.  Replaces nothing in argent: argent has no device. */
int argent_ctx_create(int device, const ArgentLimits* limits, ArgentCtx** out);
void argent_ctx_destroy(ArgentCtx* ctx);
const char* argent_last_error(const ArgentCtx* ctx);
/* Block until the context's stream is idle. */
int argent_ctx_sync(ArgentCtx* ctx);
/* The context's cudaStream_t, as a void pointer. */
void* argent_ctx_stream(ArgentCtx* ctx);

/*
 * Upload a piece and build its acceleration structure.  Replaces
 * `Piece::new` + `Bvh::build` (core/src/scene.rs:22-32, bvh.rs:117-146).
 * positions: nv*3 floats; normals: nv*3 floats or NULL (flat shading, as
 * argent does for a mesh without normals, scene.rs:181); tris: nt*3 indices;
 * tri_material: nt slots or NULL (all 0); cavity: nv floats or NULL.
 */
int argent_piece_upload(ArgentCtx* ctx, const float* positions, uint32_t nv, const float* normals,
                        const uint32_t* tris, uint32_t nt, const uint16_t* tri_material,
                        const float* cavity, ArgentPiece** out);
void argent_piece_destroy(ArgentPiece* piece);
/*
 * Same arguments and result as argent_piece_upload, with the BVH built on
 * the device: a linear BVH (63-bit Morton codes, radix sort, Karras radix
 * tree) collapsed to the same 8-wide nodes.  For piece swaps: it builds
 * much faster than the host SAH tree, which traces faster.  Closest
 * hits are the same for either tree (the minimum of (t, triangle index)
 * over the triangles hit).  Replaces `Bvh::build` (bvh.rs:117-146).
 */
int argent_piece_upload_device_bvh(ArgentCtx* ctx, const float* positions, uint32_t nv, const float* normals,
                                   const uint32_t* tris, uint32_t nt, const uint16_t* tri_material,
                                   const float* cavity, ArgentPiece** out);
/*
 * The ray-triangle test of a piece's traversals.  ARGENT_TRI_MOLLER_TRUMBORE
 * (the default) is argent's `tri_intersect` (bvh.rs:391-410) in argent's
 * operation order, which gives bit-exact closest hits.  ARGENT_TRI_WATERTIGHT
 * is Woop, Benthin and Wald's watertight test (JCGT 2013): no ray passes
 * between two triangles that share an edge, at the price of hits that can
 * differ from argent's at edges and in the last bits of t.  Rewrites the
 * piece's triangle records on the device after the context's work is done;
 * scenes built on the piece use the new test from their next render.
 */
enum { ARGENT_TRI_MOLLER_TRUMBORE = 0, ARGENT_TRI_WATERTIGHT = 1 };
int argent_piece_set_triangle_test(ArgentCtx* ctx, ArgentPiece* piece, int test);
/* Root bounds, as `Piece::bounds` (scene.rs:34-37). */
int argent_piece_bounds(const ArgentPiece* piece, float lo[3], float hi[3]);
/* Bytes the piece holds on the device. */
uint64_t argent_piece_device_bytes(const ArgentPiece* piece);

/* Build a scene around a piece.  Replaces `Scene::new` + `rebuild_lights`
 * (scene.rs:82-110) and, for a map environment, `EnvData::load`'s table build
 * (envmap.rs:141-177).  The piece must outlive the scene. */
int argent_scene_upload(ArgentCtx* ctx, ArgentPiece* piece, const ArgentSceneDesc* desc, ArgentScene** out);
void argent_scene_destroy(ArgentScene* scene);
/* Replace the turntable angle of an uploaded scene (scene.rs:53-55). */
int argent_scene_set_turntable(ArgentScene* scene, float turntable_deg);

/* A film of width x height pixels.  Replaces `Film::new` (render.rs:24-27). */
int argent_film_create(ArgentCtx* ctx, uint32_t width, uint32_t height, uint32_t flags, ArgentFilm** out);
void argent_film_destroy(ArgentFilm* film);
/* `Film::clear` (render.rs:29-34). */
int argent_film_clear(ArgentFilm* film);
/* `film.samples`: the next sample index (render.rs:19-20, 70). */
uint32_t argent_film_samples(const ArgentFilm* film);
/*
 * Averages as `Film::color`, `Film::albedo`, `Film::normal` (render.rs:36-62):
 * width*height*3 floats each, any pointer may be NULL.  color is camera RGB
 * (the scene's white balance applied, render.rs:74,96).
 */
int argent_film_read(ArgentFilm* film, float* color, float* albedo, float* normal);
/* Average CIE XYZ per pixel (width*height*3), before the camera matrix. */
int argent_film_read_xyz(ArgentFilm* film, float* xyz);

/*
 * Render `count` more samples per pixel.  Replaces `render_pass`
 * (render.rs:67-115) with the same semantics: sample indices run from
 * film.samples to film.samples+count-1, per-pixel seeding
 * hash32((y*w+x) ^ hash32(seed ^ 0xa511e9b3)), non-finite samples dropped.
 * Asynchronous on the context stream; argent_film_read synchronises.
 */
int argent_render_pass(ArgentCtx* ctx, ArgentScene* scene, const ArgentCamera* camera, ArgentFilm* film,
                       const ArgentPathSettings* settings, uint32_t count, uint32_t seed);

/* ------------------------------------------------------------------ */
/* Traversal primitives.                                              */
/* ------------------------------------------------------------------ */

/*
 * Closest hit of n object-space rays against a piece, t in (1e-7, tmax).
 * Replaces `Bvh::intersect` (bvh.rs:159-212); prim is the original triangle
 * index.  Host arrays; synchronous.
 */
int argent_trace_closest(ArgentCtx* ctx, ArgentPiece* piece, const ArgentRay* rays, uint64_t n, ArgentHit* hits);
/* Any hit; occluded[i] = 1 when some triangle has t in (1e-7, tmax).
 * Replaces `Bvh::occluded` (bvh.rs:216-247).  Host arrays; synchronous. */
int argent_trace_anyhit(ArgentCtx* ctx, ArgentPiece* piece, const ArgentRay* rays, uint64_t n, uint8_t* occluded);
/*
 * Allocation-free closest hit.  No counterpart in argent.  Same inputs,
 * outputs and results as argent_trace_closest (host arrays, synchronous),
 * but it allocates nothing: no cudaMalloc, cudaFree or allocating library
 * call.  It is for callers that cannot allocate device memory while they run.
 * One example is a serve loop that admits renders against a fixed
 * device-memory budget and issues probe rays (autofocus, picking) between
 * them: an allocation could fail under load or evict a resident scene, and
 * cudaMalloc/cudaFree can synchronise the device and stall renders in
 * flight on other streams.
 * Limit: n <= 262,144 rays (2^18); larger n returns ARGENT_E_INVALID.  The
 * device staging is one static array of 12 MiB (rays then hits) that every
 * GPU loading the library holds until exit.  The first call on a context
 * looks up the array's device address (cudaGetSymbolAddress) with the
 * context's device current and keeps it in the context; make that first call
 * before any stream capture.  A device reset (cudaDeviceReset) ends every
 * context on the device, and a context created after it looks the address
 * up again.  A call with the context's profiling on records its launch like
 * the other trace entry points (events, no device memory).  All calls share
 * the array and it keeps the last call's contents: calls that overlap on the
 * GPU (e.g. two contexts on one device used from two threads) race.
 */
int argent_trace_closest_noalloc(ArgentCtx* ctx, ArgentPiece* piece, const ArgentRay* rays, uint64_t n,
                                 ArgentHit* hits);
/* Device-pointer variants (asynchronous on the context stream). */
int argent_trace_closest_device(ArgentCtx* ctx, ArgentPiece* piece, const ArgentRay* d_rays, uint64_t n,
                                ArgentHit* d_hits);
int argent_trace_anyhit_device(ArgentCtx* ctx, ArgentPiece* piece, const ArgentRay* d_rays, uint64_t n,
                               uint8_t* d_occluded);

/* ------------------------------------------------------------------ */
/* Batched renders (argent `turntable` / `sheet` loops).              */
/* ------------------------------------------------------------------ */

/*
 * One item of a batch: a render_pass call.  The items of one batch run as
 * one persistent launch sequence in which waves of different items
 * overlap.  Each item's film receives the samples argent_render_pass would
 * render for the same arguments, each bit for bit; the film adds them in
 * runs per wave, so where the batch packs an item's samples into other runs
 * (an item that starts in a wave another item began) its film values differ
 * from argent_render_pass's by float rounding only.  Items may share a film:
 * they render one after another, as consecutive argent_render_pass calls
 * would.  Replaces the per-frame `render_image` loops of `render_reel`
 * (argent/src/jobs.rs:595-713) and `sheet_prepared` (jobs.rs:857-889).
 */
typedef struct ArgentBatchItem {
  ArgentScene* scene;
  ArgentCamera camera;
  ArgentFilm* film;
  ArgentPathSettings settings;
  uint32_t count;
  uint32_t seed;
} ArgentBatchItem;

int argent_render_batch(ArgentCtx* ctx, const ArgentBatchItem* items, uint32_t n);

/* ------------------------------------------------------------------ */
/* Autotuning (no counterpart in argent).                             */
/* ------------------------------------------------------------------ */

typedef struct ArgentTuneResult {
  uint32_t lanes;
  uint32_t reserved;
  uint64_t wave_paths;
  double path_samples_per_s;
} ArgentTuneResult;

/*
 * Times `count` samples of the given frame (after one warm-up pass) for each
 * lane count in {2, 4, 8, 12, 16} and wave size in {2^21 .. 2^25} whose path
 * state fits in half of the free device memory and keeps the fastest; then,
 * at that lane count and wave size, searches one knob at a time: blocks per
 * SM of each shading class the scene uses ({2, 3, 4, 5, 6, 8}) and of the
 * traversals ({4, 6, 8}), keeping a value only when it is faster.  The best
 * tuning becomes the context's (argent_ctx_tuning reads it) and the path
 * state of unused lanes is freed.  results (may be NULL when max_results is
 * 0) receives up to max_results lane/wave measurements; *n_results the
 * number taken.  Renders into a scratch film.
 */
int argent_autotune(ArgentCtx* ctx, ArgentScene* scene, const ArgentCamera* camera,
                    const ArgentPathSettings* settings, uint32_t width, uint32_t height, uint32_t count,
                    ArgentTuneResult* results, uint32_t max_results, uint32_t* n_results);
/*
 * Launch configuration of a context's renders: what argent_autotune
 * searches.  Grid sizes change only how work is spread over the SMs, never
 * a film (every kernel takes its work from a queue counter, and film sums
 * are added in wave order).
 */
typedef struct ArgentTuning {
  uint32_t lanes;                  /* concurrent waves, 1..16 */
  uint32_t trace_blocks_per_sm;    /* blocks of 128 per SM launched for the closest-hit and shadow
                                      traversals; 0 = as many as are resident */
  uint64_t wave_paths;             /* path slots per wave, 2^16..2^30 */
  uint32_t shade_blocks_per_sm[5]; /* per material class (misses and panels, metal, coated,
                                      dielectric, other); 0 = the built-in default */
  uint32_t reserved;
} ArgentTuning;
int argent_ctx_tuning(const ArgentCtx* ctx, ArgentTuning* out);
/* Applies a tuning (e.g. one argent_autotune found for the same kind of
 * render earlier); waits for the context stream first. */
int argent_ctx_set_tuning(ArgentCtx* ctx, const ArgentTuning* tuning);
/* The context's current lanes and wave size. */
int argent_ctx_config(const ArgentCtx* ctx, uint32_t* lanes, uint64_t* wave_paths);
/*
 * Sets the lanes (1..16) and the wave size (2^16..2^30 path slots) that the
 * context's next calls use, e.g. a configuration argent_autotune found
 * earlier for the same kind of render.  Waits for the context stream first.
 * Lane buffers grow on first use; lanes left unused keep theirs.  Films do
 * not depend on the configuration beyond the order of their FP32 sums.
 */
int argent_ctx_set_config(ArgentCtx* ctx, uint32_t lanes, uint64_t wave_paths);

/* Kernels the library has launched on this context since creation. */
uint64_t argent_ctx_kernel_launches(const ArgentCtx* ctx);

/* ------------------------------------------------------------------ */
/* Denoise (argent-post denoise.rs, the built-in à-trous backend).    */
/* ------------------------------------------------------------------ */

/*
 * argent's à-trous denoiser (argent-post/src/denoise.rs:535-712: 5 passes
 * of the 5x5 B3 kernel with holes 1..16, luminance edge stopping against a
 * per-pixel noise estimate, normal weight max(0, n.n')^128, albedo weight
 * exp(-|da|^2 / 0.01), albedo demodulation) on the device.  color, albedo,
 * normal and out are width*height*3 floats in host memory; albedo and
 * normal may be NULL (a normal without an albedo is ignored, as with argent's
 * OIDN path).  Replaces `denoise(.., DenoiseBackend::Atrous)`.
 */
int argent_denoise_atrous(ArgentCtx* ctx, uint32_t width, uint32_t height, const float* color, const float* albedo,
                          const float* normal, float* out);
/* The film's colour denoised with its albedo and normal guides, without the
 * averages leaving the device (the `render_image` hand-off, shot.rs:424-444);
 * out receives width*height*3 floats of camera RGB. */
int argent_film_denoise(ArgentFilm* film, float* out);

/* ------------------------------------------------------------------ */
/* Develop (argent-post tonemap.rs): the 8-bit hand-off.              */
/* ------------------------------------------------------------------ */

/* `ToneMap` and `AgxLook` (argent-post/src/tonemap.rs:38-55). */
enum { ARGENT_TM_AGX = 0, ARGENT_TM_ACES = 1, ARGENT_TM_KHRONOS = 2, ARGENT_TM_REINHARD = 3, ARGENT_TM_CLAMP = 4 };
enum { ARGENT_AGX_BASE = 0, ARGENT_AGX_PUNCHY = 1, ARGENT_AGX_GOLDEN = 2 };

/* `Grade` (tonemap.rs:57-68); argent's default is AgX Punchy, 0 EV,
 * saturation 1.  `look` is used by AgX only. */
typedef struct ArgentGrade {
  float exposure_ev;
  int32_t tonemap;
  int32_t look;
  float saturation;
} ArgentGrade;

/*
 * argent_post::develop (tonemap.rs:369-391): exposure, tone map, saturation,
 * sRGB encode through argent's per-grade tables, TPDF dither, 8 bits.  rgb is
 * width*height*3 floats of scene-linear camera RGB in host memory; out
 * receives width*height*3 bytes, byte-identical to argent's develop.
 */
int argent_develop(ArgentCtx* ctx, uint32_t width, uint32_t height, const float* rgb, const ArgentGrade* grade,
                   uint8_t* out);
/* The film's colour (denoised with its guides when `denoise` is non-zero)
 * developed to 8-bit sRGB without leaving the device: render_image + develop
 * (shot.rs:424-444, serve/live.rs:200).  out receives width*height*3 bytes. */
int argent_film_develop(ArgentFilm* film, const ArgentGrade* grade, int denoise, uint8_t* out);

/* ------------------------------------------------------------------ */
/* Cavity mask (argent-mesh cavity.rs), the patina input of `Piece`.  */
/* ------------------------------------------------------------------ */

/* `PatinaSettings` (argent-mesh/src/cavity.rs:24-42).  argent's defaults:
 * 48 samples, ao_distance 1.2 mm, curvature_radius 0.4 mm, concavity_weight
 * 0.35, 3 smoothing passes; `Prepared::build` scales the two distances by
 * the piece radius (core/src/shot.rs:137-141). */
typedef struct ArgentPatinaSettings {
  uint32_t ao_samples;
  float ao_distance;
  float curvature_radius;
  float concavity_weight;
  uint32_t smooth_iterations;
} ArgentPatinaSettings;

/*
 * Fraction of `samples` cosine-weighted hemisphere rays per vertex blocked
 * within `distance` (cavity::ambient_occlusion, cavity.rs:96-135), traced on
 * the device against the uploaded piece.  positions/normals are the nv
 * vertices the piece was uploaded with (normals already chosen: the mesh's,
 * or argent_mesh_smooth_normals); ao receives nv floats.
 */
int argent_piece_ambient_occlusion(ArgentCtx* ctx, ArgentPiece* piece, const float* positions, const float* normals,
                                   uint32_t nv, uint32_t samples, float distance, float* ao);
/*
 * cavity::patina_mask (cavity.rs:52-78): device AO, host concavity and
 * Laplacian smoothing, then the contrast blend; mask receives nv values in
 * [0, 1] for `argent_piece_upload`'s cavity argument.  normals may be NULL
 * (smooth vertex normals, cavity.rs:80-86).  The mesh must be the one the
 * piece was uploaded from.
 */
int argent_piece_patina_mask(ArgentCtx* ctx, ArgentPiece* piece, const float* positions, const float* normals,
                             uint32_t nv, const uint32_t* tris, uint32_t nt, const ArgentPatinaSettings* settings,
                             float* mask);
/* Host helpers with argent-mesh's public semantics (no device needed):
 * normals::smooth_vertex_normals (normals.rs:226-242), cavity::concavity
 * (cavity.rs:137-236) and cavity::smooth (cavity.rs:241-299). */
int argent_mesh_smooth_normals(const float* positions, uint32_t nv, const uint32_t* tris, uint32_t nt, float* out);
int argent_mesh_concavity(const float* positions, uint32_t nv, const float* normals, const uint32_t* tris, uint32_t nt,
                          float radius, float* out);
int argent_mesh_smooth(const float* positions, uint32_t nv, const uint32_t* tris, uint32_t nt, float* values,
                       uint32_t iterations, float lambda);

/* ------------------------------------------------------------------ */
/* Serving: continuous batching of render requests.                   */
/* ------------------------------------------------------------------ */

/*
 * Replaces serve's job loop for stills (argent/src/serve/queue.rs:599-617:
 * one job at a time, render_pass in chunks sized for ~1.5 s, seed 7, a
 * cancel check between chunks) and its progressive live passes
 * (serve/live.rs:747, 767).  Here requests in flight share batches: each
 * argent_serve_step issues one batch (as argent_render_batch) of chunks,
 * whole samples of the requests' frames, up to the step's budget.  The
 * budget is a quarter of the pending work, between step_path_samples and
 * step_path_samples_max.  Requests whose remaining work is under a
 * sixteenth of it finish in that batch (together up to half the budget);
 * the rest of the budget goes to the other active requests strictly in
 * urgency order (a request reached with no budget left waits; the first
 * one reached always takes at least one sample).  Urgency is the priority
 * value minus the time waited over aging_ms (lower first; ties in
 * submission order).  Chunks continue each film's sample indices, so a
 * finished film holds what one argent_render_pass of `spp` samples with the
 * same seed gives (up to the order of the FP32 sums).
 *
 * With `overlap` set, a step issues its batch while the previous one still
 * runs (at most two in flight) and waits only for the older one, so the
 * device does not drain between steps; without it each step waits for its
 * own batch.
 *
 * Admission: a queued request becomes active, in urgency order, while
 * fewer than max_active are active and its film fits in film_budget
 * together with the films in use and pooled (pooled films of other sizes
 * are freed first).  Films are pooled by (width, height, flags).
 *
 * Threads: submit, poll, cancel, release and stats may be called from any
 * thread.  step and read use the context and must be called from the one
 * thread that owns it.  A request's scene must outlive the request.
 */
typedef struct ArgentServe ArgentServe;

typedef struct ArgentServeConfig {
  uint64_t film_budget;       /* device bytes for films in use and pooled; 0 = 8 GiB */
  uint32_t max_active;        /* requests rendered together; 0 = 64 */
  uint32_t aging_ms;          /* waiting this long raises a request one priority level; 0 = 250 */
  uint64_t step_path_samples; /* least path-samples per step; 0 = 2^26 (about 45 ms of rendering) */
  uint64_t step_path_samples_max; /* a step takes a quarter of the pending work, up to this;
                                     0 = 2 x step_path_samples */
  uint32_t overlap;           /* 1 = keep the next batch in flight while one runs */
  uint32_t max_pending;       /* requests queued or active at most: a submit beyond it returns
                                 ARGENT_E_BUSY (argent refuses a job when 24 wait, queue.rs:28,364);
                                 0 = no bound */
  uint64_t max_pending_path_samples; /* work not yet rendered, at most: a submit that would take the
                                        path-samples still to render of the queued and active requests
                                        past it returns ARGENT_E_BUSY, unless no request of its
                                        priority is pending (so no class is shut out); bounds the
                                        wait of every admitted request under overload; 0 = no bound */
} ArgentServeConfig;

typedef struct ArgentServeRequest {
  ArgentScene* scene;
  ArgentCamera camera;
  ArgentPathSettings settings;
  uint32_t width, height;
  uint32_t spp;        /* samples per pixel in total */
  uint32_t seed;       /* render seed (serve uses 7 for stills, queue.rs:613) */
  uint32_t film_flags; /* ARGENT_FILM_*; 0 = Kahan */
  int32_t priority;    /* lower values are served first */
} ArgentServeRequest;

enum {
  ARGENT_REQ_QUEUED = 0,
  ARGENT_REQ_ACTIVE = 1,
  ARGENT_REQ_DONE = 2,
  ARGENT_REQ_CANCELLED = 3,
  ARGENT_REQ_FAILED = 4
};

typedef struct ArgentServeStatus {
  int32_t state;    /* ARGENT_REQ_* */
  uint32_t samples; /* samples accumulated so far */
  uint32_t spp;
  uint32_t reserved;
  double t_submit, t_start, t_done; /* seconds on the serve's steady clock; -1 = not yet */
} ArgentServeStatus;

int argent_serve_create(ArgentCtx* ctx, const ArgentServeConfig* cfg, ArgentServe** out);
/* Frees every film the serve holds; the context stays. */
void argent_serve_destroy(ArgentServe* serve);
/* Queues a request.  ARGENT_E_BUSY if its film alone exceeds film_budget. */
int argent_serve_submit(ArgentServe* serve, const ArgentServeRequest* req, uint64_t* ticket);
int argent_serve_poll(ArgentServe* serve, uint64_t ticket, ArgentServeStatus* status);
/* Marks a queued or active request; it is cancelled at the next step that
 * finds none of its batches in flight. */
int argent_serve_cancel(ArgentServe* serve, uint64_t ticket);
/* One scheduling round: completions of finished batches, cancellations,
 * admission, one batch issued, and a wait for its batch (or, with overlap,
 * for the older batch in flight).  *pending (may be NULL) = requests still
 * queued or active.  A failed batch marks its requests ARGENT_REQ_FAILED
 * and returns the code. */
int argent_serve_step(ArgentServe* serve, uint32_t* pending);
/* Averages of a finished request's film (as argent_film_read; any pointer
 * may be NULL), then forgets the request and pools its film. */
int argent_serve_read(ArgentServe* serve, uint64_t ticket, float* color, float* albedo, float* normal);
/* Forgets a finished, cancelled or failed request without reading it
 * (ARGENT_E_BUSY while a batch holding a chunk of it still runs). */
int argent_serve_release(ArgentServe* serve, uint64_t ticket);
/* Steps that ran a batch, path-samples rendered, film bytes in use. */
int argent_serve_stats(ArgentServe* serve, uint64_t* steps, uint64_t* path_samples, uint64_t* film_bytes_in_use);
/* Seconds on the serve's steady clock (the clock of ArgentServeStatus). */
double argent_serve_now(ArgentServe* serve);

/* ------------------------------------------------------------------ */
/* Measurement (no counterpart in argent, whose only timing is wall   */
/* clock around render_pass, argent/src/jobs.rs:501-504).             */
/* ------------------------------------------------------------------ */

/* Kernel classes for argent_ctx_kernel_times. */
enum {
  ARGENT_KC_RAYGEN = 0,
  ARGENT_KC_INTERSECT = 1,
  ARGENT_KC_SHADE = 2,
  ARGENT_KC_SHADOW = 3,
  ARGENT_KC_FILM = 4,
  ARGENT_KC_TRACE = 5,
  /* The shading kernel of each material class; ARGENT_KC_SHADE is their sum. */
  ARGENT_KC_SHADE_TERMINAL = 6,
  ARGENT_KC_SHADE_METAL = 7,
  ARGENT_KC_SHADE_COATED = 8,
  ARGENT_KC_SHADE_DIELECTRIC = 9,
  ARGENT_KC_SHADE_OTHER = 10,
  ARGENT_KC_COUNT = 11
};
/* While on, every launch is bracketed by CUDA events on the context stream;
 * turning it on or off resets the totals. */
int argent_ctx_set_profiling(ArgentCtx* ctx, int on);
/* Summed device time (ms) and launch count per kernel class since the last
 * reset; synchronises the stream.  ms and launches hold ARGENT_KC_COUNT. */
int argent_ctx_kernel_times(ArgentCtx* ctx, double* ms, uint64_t* launches);
/* Renders that are not overlapped and not instrumented are captured as CUDA
 * graphs and replayed when the same waves come again (on by default); off
 * also frees the captured graphs. */
int argent_ctx_set_graphs(ArgentCtx* ctx, int on);
/* Ray sharing for batches (off by default).  argent's reel renders every
 * metal variant of a frame on its own (jobs.rs:595-713); variants that differ
 * only in their materials -- the same piece, turntable angle, panels, floor,
 * camera, film size, samples and seed -- trace the same rays until their
 * paths part.  While on, the renders of one argent_render_batch (or serve
 * step) that match so are laid out side by side in the waves, and a ray
 * bit-identical to the same pixel-sample's ray of the first of them takes
 * that ray's closest hit or shadow visibility instead of being traced again;
 * a first hit on a material whose record equals the first render's (the
 * studio floor) takes that render's shading too.
 * Every hit record and radiance sample equals the unshared render's, and a
 * batch's films equal each render's own argent_render_pass bit for bit (the
 * waves give every pixel the same runs of samples); a serve step's chunks
 * agree with the render alone to float rounding, as unshared ones do.  Costs
 * 33 bytes per path slot per lane in use. */
int argent_ctx_set_ray_sharing(ArgentCtx* ctx, int on);
/* Traversal visit counters: on = count, and reset to zero. */
int argent_ctx_set_counting(ArgentCtx* ctx, int on);
/* out[6] = closest-hit rays, nodes, triangles; any-hit rays, nodes,
 * triangles, counted since the last argent_ctx_set_counting. */
int argent_ctx_traversal_counts(ArgentCtx* ctx, uint64_t* out);
/* out[18]: rays by node visits in bins 0, 1, 2-3, 4-7, 8-15, 16-63, 64-255,
 * 256+ (closest-hit out[0..7], any-hit out[8..15]), then the largest node
 * count of a closest-hit ray and of an any-hit ray, since the last
 * argent_ctx_set_counting. */
int argent_ctx_traversal_histogram(ArgentCtx* ctx, uint64_t* out);
/* out[18]: interior node visits by the number of children whose box the ray
 * enters, 0..8 (closest hit out[0..8], any hit out[9..17]), since the last
 * argent_ctx_set_counting. */
int argent_ctx_child_hit_histogram(ArgentCtx* ctx, uint64_t* out);
/* out[128]: paths entering bounce d (out[d]) and shadow rays queued at
 * bounce d (out[64 + d]), d < 64, summed over the waves run since the last
 * argent_ctx_set_counting that turned counting on. */
int argent_ctx_bounce_counts(ArgentCtx* ctx, uint64_t* out);

#ifdef __cplusplus
}
#endif

#endif /* ARGENT_GPU_H */
