// internal.cuh — the objects behind the opaque handles of argent_gpu.h and
// the device-side scene, job and wave descriptors.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/argent_gpu.h"
#include "device/traverse.cuh"

// Status bits (device status word) beyond the traversal ones.
#define ARGENT_STATUS_QUEUE_OVERFLOW 2u
#define ARGENT_STATUS_TIMEOUT 4u

#define ARGENT_MAX_PANELS 16
#define ARGENT_MAX_DEPTH 64

namespace dev {

struct DevPanel {
  float c[3], hu[3], hv[3], n[3];
  float area, feather, hu_l2, hv_l2;
  int32_t emits, camera_visible;
  const float* emission;  // 471-entry table
};

// Everything a path needs from its scene, in device memory.
struct DevScene {
  DevPiece piece;
  const ArgentMaterial* mats;
  int32_t num_mats;
  int32_t num_panels;
  DevPanel panels[ARGENT_MAX_PANELS];
  int32_t num_lights;
  int32_t lights[ARGENT_MAX_PANELS];
  float light_cdf[ARGENT_MAX_PANELS];
  float env_pick;
  // environment
  int32_t env_is_map;
  float env_power;
  const float* env_top;
  const float* env_horizon;
  const float* env_bottom;
  int32_t map_w, map_h;
  const float* map_weights;  // 3 per texel
  const float* map_cond;     // (w+1) per row
  const float* map_marg;     // h+1
  const float* lin_basis;    // 3 x 471
  float map_to_local_s, map_to_local_c;  // rot_y(-rotation)
  float map_to_world_s, map_to_world_c;  // rot_y(+rotation)
  // floor
  int32_t floor_enabled;
  float floor_y;
  int32_t floor_material;
  float fade_start, fade_end;
  // turntable
  int32_t has_turn;
  float to_obj_s, to_obj_c;      // rot_y(-turn)
  float to_world_s, to_world_c;  // rot_y(+turn)
  float cam_m[9];
  // Shading class of each material slot and of the floor's material.
  uint8_t mat_class[256];
  int32_t floor_class;
  uint32_t class_mask;  // classes a path of this scene can reach
};

// One render_pass worth of work.
struct DevJob {
  const DevScene* scene;
  ArgentCamera cam;
  uint32_t w, h;
  uint32_t first;   // film.samples before this pass
  uint32_t seed_h;  // hash32(seed ^ 0xa511e9b3)
  uint32_t max_depth, rr_depth;
  float clamp_indirect;
  float* film_xyz;       // 3 per pixel
  float* film_comp;      // Kahan compensation, 3 per pixel (or null)
  double* film_xyz64;    // FP64 sums (or null)
  float* film_albedo;    // 3 per pixel
  float* film_normal;    // 3 per pixel
  // Ray sharing, for a job that follows another in its group: the material
  // slots whose records equal the leader's (bit i of share_mat[i / 32]), and
  // whether everything else shading reads (lights, environment, floor,
  // turntable, path settings) equals the leader's.  A bounce-0 hit on such a
  // material is shaded exactly as the leader's, so it takes the leader's
  // result (k_shade_copy).
  uint32_t share_mat[8];
  uint32_t share_rest;
};

// A contiguous run of path slots in a wave: pixels [p0, p0+pn) of job
// `job`, samples first+s0 .. first+s0+sn-1; slot = slot_begin + k*pn + p.
// With ray sharing, the segments of jobs that trace the same rays (same
// piece, camera, seed and samples; other materials) follow each other with
// the same pixels and samples, and `lead` is the first such segment's
// slot_begin (the slot of the same pixel-sample there is lead + k*pn + p);
// ~0u when the segment leads or shares nothing.
struct DevSegment {
  uint32_t slot_begin, job, p0, pn, s0, sn, lead;
};

#define ARGENT_MAX_SEGMENTS 64
struct WaveDesc {
  uint32_t num_segments;
  uint32_t num_slots;
  DevSegment seg[ARGENT_MAX_SEGMENTS];
};

}  // namespace dev

// Path state of one wave, structure of arrays (capacity = wave_paths).
struct WaveBuffers {
  uint64_t cap = 0;
  float4 *o = nullptr, *d = nullptr, *beta = nullptr, *L = nullptr, *lambda = nullptr, *pdf = nullptr;
  float4 *hit = nullptr, *albedo = nullptr, *normal = nullptr;
  float4 *sh_o = nullptr, *sh_d = nullptr, *sh_c = nullptr;
  uint4* meta = nullptr;
  unsigned long long* rng = nullptr;
  uint32_t *q0 = nullptr, *q1 = nullptr, *qc = nullptr;
  uint32_t* counters = nullptr;
  std::vector<void*> allocs;
  uint64_t bytes = 0;
  // Ray sharing (allocated on the first wave that shares rays): per slot its
  // leader's slot and its shadow record of the current depth (position,
  // depth + 1); per shadow record whether it reached its light; the queues of
  // rays to trace and of rays that take their leader's result, for closest
  // hits and for shadow rays.
  uint64_t share_cap = 0, share_bytes = 0;
  uint32_t* lead = nullptr;
  uint32_t* qsc = nullptr;  // bounce-0 paths that take their leader's shading
  uint2* shrec = nullptr;
  uint8_t* vis = nullptr;
  uint32_t *qt = nullptr, *qx = nullptr, *qst = nullptr, *qsx = nullptr;
  std::vector<void*> share_allocs;
  void release_share() {
    for (void* a : share_allocs) cudaFree(a);
    share_allocs.clear();
    lead = qt = qx = qst = qsx = qsc = nullptr;
    shrec = nullptr;
    vis = nullptr;
    share_cap = 0;
    bytes -= share_bytes;
    share_bytes = 0;
  }
  void release() {
    for (void* a : allocs) cudaFree(a);
    allocs.clear();
    release_share();
    cap = 0;
    bytes = 0;
  }
};

// Per-kernel-class CUDA event pairs recorded while profiling is on.
enum { KC_RAYGEN = 0, KC_INTERSECT, KC_SHADE, KC_SHADOW, KC_FILM, KC_TRACE, KC_SHADE_CLS0, KC_COUNT = KC_SHADE_CLS0 + 5 };
struct KernelProfile {
  bool on = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev[KC_COUNT];
  std::vector<cudaEvent_t> pool;
  double ms[KC_COUNT] = {};
  uint64_t n[KC_COUNT] = {};
};

// Waves rotate over `lanes` lanes (default 8, at most ARGENT_LANES), each
// with its own stream and path state, so that one wave's kernels fill the
// SMs that another wave's kernel tails and small late-bounce launches leave
// idle.  Lane 0 runs on the context stream.
#define ARGENT_LANES 16
#define ARGENT_GRAPH_CACHE 8

struct ArgentCtx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t lane_stream[ARGENT_LANES] = {};
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  cudaEvent_t film_ev[ARGENT_LANES] = {};
  // Waves rotate over the lanes across calls: the next call starts at
  // next_lane, and, while an overlapped batch may still run, its first film
  // pass waits for the film pass of the last wave before it (on
  // last_film_lane), so films accumulate in wave order also when batches
  // overlap.
  int next_lane = 0, last_film_lane = -1;
  // Completion stream of batches that do not join the context stream, and
  // whether one may still run (cleared by argent_ctx_sync and by a joined
  // batch, which orders everything after it).
  cudaStream_t aux_stream = nullptr;
  bool overlapped_pending = false;
  // Job records of joined batches (kept, so captured graphs can point at it).
  dev::DevJob* d_jobs_buf = nullptr;
  size_t d_jobs_cap = 0;
  // Captured batches: the launch sequence of a joined batch, keyed by
  // everything its kernel parameters depend on, least recently used evicted.
  struct GraphEntry {
    std::vector<uint8_t> key;
    cudaGraphExec_t exec;
    uint64_t kernels;
    uint64_t last_use;
  };
  std::vector<GraphEntry> graph_cache;
  uint64_t graph_clock = 0;
  bool graphs_on = true;
  // Batches trace the rays that renders have in common once
  // (argent_ctx_set_ray_sharing).
  bool share_rays = false;
  // Scene data uploaded once per distinct content (environment maps and
  // their sampling tables, emission and sky spectra), shared by the scenes
  // that hold it and freed with the last of them: metal variants of one
  // studio then read one copy, which keeps one map in L2 instead of one per
  // scene.
  struct SharedBlob {
    uint64_t hash = 0;
    std::vector<uint8_t> host;
    void* dev = nullptr;
    int refs = 0;
  };
  std::vector<SharedBlob> blobs;
  std::mutex blob_mu;  // scenes may be uploaded and destroyed from several threads
  int num_sms = 148;
  int lanes = 8;
  // Launch tuning (argent_ctx_set_tuning / argent_autotune); 0 = default.
  int trace_bpsm = 0;
  int shade_bpsm[5] = {0, 0, 0, 0, 0};
  bool counting = false;  // traversal instrumentation on (argent_ctx_set_counting)
  ArgentLimits limits{};
  std::string err;
  uint64_t launches = 0;
  uint32_t* d_status = nullptr;
  bool tables_ready = false;
  WaveBuffers wave[ARGENT_LANES];
  KernelProfile prof;
  float* resolve = nullptr;  // film-read staging (grown on demand)
  size_t resolve_floats = 0;
  // Device address of the allocation-free entry point's static array,
  // looked up by this context's first call of it.
  void* noalloc_addr = nullptr;
  // Runtime errors found pending (from earlier calls) when a batch was
  // issued; cleared there, counted for diagnosis.
  uint64_t stale_errors = 0;
};

struct ArgentPiece {
  ArgentCtx* ctx = nullptr;
  dev::DevPiece dev{};
  std::vector<void*> allocs;
  uint64_t bytes = 0;
  uint32_t nv = 0, nt = 0, depth = 0, max_material = 0;
  float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  int tri_test = 0;  // ARGENT_TRI_MOLLER_TRUMBORE or ARGENT_TRI_WATERTIGHT
};

struct ArgentScene {
  ArgentCtx* ctx = nullptr;
  ArgentPiece* piece = nullptr;
  dev::DevScene host{};           // host copy of the device descriptor
  dev::DevScene* d_scene = nullptr;
  std::vector<void*> allocs;
  std::vector<void*> shared;  // blobs held in ctx->blobs
  std::vector<ArgentMaterial> mats_host;  // the material records, for ray sharing's comparisons
  uint64_t bytes = 0;
  float cam_m[9];
  // Pinned staging copy for stream-ordered descriptor updates (turntable),
  // and the event that marks its last copy done.
  dev::DevScene* staged = nullptr;
  cudaEvent_t staged_ev = nullptr;
};

struct ArgentFilm {
  ArgentCtx* ctx = nullptr;
  uint32_t w = 0, h = 0, flags = 0;
  uint32_t samples = 0;
  float* xyz = nullptr;
  float* comp = nullptr;
  double* xyz64 = nullptr;
  float* albedo = nullptr;
  float* normal = nullptr;
  bool has_matrix = false;
  float cam_m[9];
  uint64_t bytes = 0;
};

int set_error(const ArgentCtx* ctx, int code, const std::string& msg);
int ctx_check_status(ArgentCtx* ctx);
int grid_for(const ArgentCtx* ctx, const void* kernel, int block, uint64_t n);
