// render_impl.cuh — the wavefront path tracer.
//
// argent renders one path per (pixel, sample) with a recursive-free bounce
// loop (integrator.rs:50-221) called from a rayon row loop
// (render.rs:67-115).  Here a wave of up to `wave_paths` paths advances one
// bounce at a time through four kernels:
//   k_intersect  closest hit: piece BVH (object space), panels, floor
//   k_shade      emission + MIS, BSDF, next-event sample, continuation, RR;
//                survivors and shadow rays are appended to queues by warp
//                ballot + one atomic per warp
//   k_shadow     any-hit of the piece BVH for the shadow queue; unoccluded
//                rays add their (already clamped) contribution to L
//   k_film       per pixel: XYZ of each finished sample, non-finite samples
//                dropped, FP32 Kahan (or FP64) accumulation into the film
// k_raygen starts a wave.  Each path keeps its PCG state between kernels, so
// the dimension stream is the one argent's single-threaded loop would draw.
#pragma once
#include "device/bsdf.cuh"
#include "device/sampler.cuh"
#include "device/spectral.cuh"
#include "device/traverse.cuh"
#include "host/scene_prep.h"
#include "internal.cuh"

namespace dev {

// Hit record encoding (w component of the hit float4).
// Minimum resident blocks of 128 threads per SM for the traversal kernels
// (the register budget ptxas gets: 8 blocks = 64 registers per thread).
#ifndef ARGENT_TRAV_BLOCKS
#define ARGENT_TRAV_BLOCKS 8
#endif
#define HIT_MISS 0xFFFFFFFFu
#define HIT_FLOOR 0xFFFFFFFEu
#define HIT_PANEL 0xF0000000u

// ---------------------------------------------------------------- lights

// |fl(x / y)| <= 1, as argent's `(q.dot(hu) / hu.length_squared()).abs() <= 1.0`
// rounds it.  For a finite y > 0: |x| <= y passes without the division;
// |x| above y (1 + 2^-22), rounded up, fails (the quotient then exceeds
// 1 + 2^-22, which rounds above 1); only the band between, and any other y,
// divides.
__device__ __forceinline__ bool ratio_within_1(float x, float y) {
  float ax = fabsf(x);
  if (y > 0.0f && y < INFINITY) {
    if (ax <= y) return true;
    if (ax > __fmul_ru(y, 1.0000002384185791f)) return false;
  }
  return fabsf(x / y) <= 1.0f;
}

// light.rs:50-63
__device__ __forceinline__ bool panel_intersect(const DevPanel& p, V3 o, V3 d, float t_max, float* t_out) {
  V3 n = ld3(p.n);
  float denom = dot(d, n);
  if (fabsf(denom) < 1e-9f) return false;
  float num = dot(ld3(p.c) - o, n);
  // A zero numerator or one of the other sign gives t <= 0, which argent's
  // t <= 1e-6 test rejects; skipping the division there changes nothing.
  if (num == 0.0f || (signbit(num) != signbit(denom))) return false;
  float t = num / denom;
  if (t <= 1e-6f || t >= t_max) return false;
  V3 q = (o + d * t) - ld3(p.c);
  if (ratio_within_1(dot(q, ld3(p.hu)), p.hu_l2) && ratio_within_1(dot(q, ld3(p.hv)), p.hv_l2)) {
    *t_out = t;
    return true;
  }
  return false;
}
// light.rs:76-93
__device__ __forceinline__ float panel_profile(const DevPanel& p, V3 x) {
  if (p.feather <= 0.0f) return 1.0f;
  V3 q = x - ld3(p.c);
  float a = fminf(fabsf(dot(q, ld3(p.hu)) / p.hu_l2), 1.0f);
  float b = fminf(fabsf(dot(q, ld3(p.hv)) / p.hv_l2), 1.0f);
  float start = 1.0f - p.feather;
  float fa = 1.0f, fb = 1.0f;
  if (a > start) {
    float t = (a - start) / p.feather;
    fa = 1.0f - 0.75f * t * t * (3.0f - 2.0f * t);
  }
  if (b > start) {
    float t = (b - start) / p.feather;
    fb = 1.0f - 0.75f * t * t * (3.0f - 2.0f * t);
  }
  return fa * fb;
}
// light.rs:67-72
__device__ __forceinline__ Spec panel_le(const DevPanel& p, V3 x, V3 dir, const Wavelengths& wl) {
  if (p.emits && dot(dir, ld3(p.n)) < 0.0f) return tab_sample(p.emission, wl) * panel_profile(p, x);
  return spec(0.0f);
}
// light.rs:142-148
__device__ __forceinline__ bool floor_intersect(const DevScene* sc, V3 o, V3 d, float t_max, float* t_out) {
  if (fabsf(d.y) < 1e-9f) return false;
  float t = (sc->floor_y - o.y) / d.y;
  if (t > 1e-5f && t < t_max) {
    *t_out = t;
    return true;
  }
  return false;
}
// light.rs:152-162
__device__ __forceinline__ float floor_presence(const DevScene* sc, V3 p) {
  float r = sqrtf(p.x * p.x + p.z * p.z);
  if (r <= sc->fade_start) return 1.0f;
  if (r >= sc->fade_end) return 0.0f;
  float t = (r - sc->fade_start) / (sc->fade_end - sc->fade_start);
  return 1.0f - t * t * (3.0f - 2.0f * t);
}

// ---------------------------------------------------------------- environment (envmap.rs)
__device__ __forceinline__ void env_uv(const DevScene* sc, V3 dir, float* u, float* v) {
  V3 d = rot_y_sc(dir, sc->map_to_local_s, sc->map_to_local_c);
  float uu = 0.5f + atan2f(d.x, -d.z) / (2.0f * ARGENT_PI_F);
  *v = acosf(rclamp(d.y, -1.0f, 1.0f)) / ARGENT_PI_F;
  float r = fmodf(uu, 1.0f);
  if (r < 0.0f) r += 1.0f;
  *u = r;
}
__device__ __forceinline__ uint32_t sat_u32(float f) {
  if (!(f > 0.0f)) return 0u;
  if (f >= 4294967296.0f) return 0xffffffffu;
  return (uint32_t)f;
}
__device__ __forceinline__ float lin_eval(const DevScene* sc, const float* w, float l) {
  float x = rclamp(l - 360.0f, 0.0f, 469.999f);
  int i = (int)x;
  float f = x - (float)i;
  float v = 0.0f;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float* b = sc->lin_basis + 471 * c;
    v += w[c] * (__ldg(b + i) * (1.0f - f) + __ldg(b + i + 1) * f);
  }
  return fmaxf(v, 0.0f);
}
// The texel a direction falls in, and its v; the map's eval and pdf of one
// direction share it.
struct EnvTexel {
  uint32_t x, y;
  float v;
};
__device__ __forceinline__ EnvTexel env_texel(const DevScene* sc, V3 dir) {
  float u, v;
  env_uv(sc, dir, &u, &v);
  EnvTexel t;
  t.x = min(sat_u32(u * (float)sc->map_w), (uint32_t)sc->map_w - 1u);
  t.y = min(sat_u32(v * (float)sc->map_h), (uint32_t)sc->map_h - 1u);
  t.v = v;
  return t;
}
__device__ Spec envmap_eval_at(const DevScene* sc, EnvTexel t, const Wavelengths& wl) {
  const float* wp = sc->map_weights + 3 * ((size_t)t.y * sc->map_w + t.x);
  float w[3] = {__ldg(wp), __ldg(wp + 1), __ldg(wp + 2)};
  Spec r;
#pragma unroll
  for (int k = 0; k < 4; ++k) r.v[k] = lin_eval(sc, w, wl.lambda[k]);
  return r;
}
// envmap.rs:375-387
__device__ float envmap_pdf_at(const DevScene* sc, EnvTexel t) {
  float st = sinf(ARGENT_PI_F * t.v);
  if (st <= 1e-6f) return 0.0f;
  size_t row = (size_t)t.y * (sc->map_w + 1);
  float pc = (__ldg(sc->map_cond + row + t.x + 1) - __ldg(sc->map_cond + row + t.x)) * (float)sc->map_w;
  float pm = (__ldg(sc->map_marg + t.y + 1) - __ldg(sc->map_marg + t.y)) * (float)sc->map_h;
  return pc * pm / (2.0f * ARGENT_PI_F * ARGENT_PI_F * st);
}
__device__ __forceinline__ uint32_t partition_le(const float* a, uint32_t n, float u) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (__ldg(a + mid) <= u)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}
// envmap.rs:390-402
__device__ V3 envmap_sample(const DevScene* sc, float u1, float u2, float* pdf_out, EnvTexel* texel) {
  uint32_t w = (uint32_t)sc->map_w, h = (uint32_t)sc->map_h;
  uint32_t y = min(max(partition_le(sc->map_marg, h + 1, u1), 1u), h) - 1u;
  const float* cond = sc->map_cond + (size_t)y * (w + 1);
  uint32_t x = min(max(partition_le(cond, w + 1, u2), 1u), w) - 1u;
  float my = __ldg(sc->map_marg + y), my1 = __ldg(sc->map_marg + y + 1);
  float cx = __ldg(cond + x), cx1 = __ldg(cond + x + 1);
  float fy = (u1 - my) / fmaxf(my1 - my, 1e-12f);
  float fx = (u2 - cx) / fmaxf(cx1 - cx, 1e-12f);
  float u = ((float)x + rclamp(fx, 0.0f, 0.999f)) / (float)w;
  float v = ((float)y + rclamp(fy, 0.0f, 0.999f)) / (float)h;
  float phi = (u - 0.5f) * 2.0f * ARGENT_PI_F;
  float theta = v * ARGENT_PI_F;
  float st, ct, sp, cp;
  sincosf(theta, &st, &ct);
  sincosf(phi, &sp, &cp);
  V3 d = rot_y_sc(V3{st * sp, ct, -st * cp}, sc->map_to_world_s, sc->map_to_world_c);
  *texel = env_texel(sc, d);
  *pdf_out = envmap_pdf_at(sc, *texel);
  return d;
}
// light.rs:111-127.  MAP false: the caller's scenes have no env map.
template <bool MAP>
__device__ Spec env_eval(const DevScene* sc, V3 dir, const Wavelengths& wl) {
  if (MAP && sc->env_is_map) return envmap_eval_at(sc, env_texel(sc, dir), wl);
  float y = rclamp(dir.y, -1.0f, 1.0f);
  if (y >= 0.0f) {
    float t = powf(y, sc->env_power);
    return lerp(t, tab_sample(sc->env_horizon, wl), tab_sample(sc->env_top, wl));
  }
  float t = powf(-y, 0.5f);
  return lerp(t, tab_sample(sc->env_horizon, wl), tab_sample(sc->env_bottom, wl));
}

// scene.rs:143-147
__device__ __forceinline__ float light_pick_pdf(const DevScene* sc, int panel) {
  for (int k = 0; k < sc->num_lights; ++k)
    if (sc->lights[k] == panel) return sc->light_cdf[k] - (k == 0 ? 0.0f : sc->light_cdf[k - 1]);
  return 0.0f;
}

// integrator.rs:35-48
__device__ __forceinline__ void add_clamped(Spec* l, const Spec& c, bool clamp, float m) {
  if (clamp) {
    float mx = max_value(c);
    *l = (mx > m) ? (*l + c * (m / mx)) : (*l + c);
  } else {
    *l = *l + c;
  }
}
__device__ __forceinline__ Spec clamped(const Spec& c, bool clamp, float m) {
  if (clamp) {
    float mx = max_value(c);
    if (mx > m) return c * (m / mx);
  }
  return c;
}

// ---------------------------------------------------------------- wave kernels

struct WaveArgs {
  const DevJob* jobs;
  float4 *o, *d, *beta, *L, *lambda, *pdf, *hit, *albedo, *normal, *sh_o, *sh_d, *sh_c;
  uint4* meta;
  unsigned long long* rng;
  uint32_t *q_in, *q_out;  // active paths entering / leaving a bounce
  uint32_t* qc;            // NUM_CLS shade queues of `cap` entries
  uint32_t cap;
  uint32_t* counters;
  uint32_t* status;
  // When every path of the wave belongs to one scene: that scene, a copy of
  // its piece descriptor and its turntable rotation, so the traversal
  // kernels read them from the parameter bank instead of following
  // meta -> job -> scene for each ray (null otherwise).
  const DevScene* uscene;
  DevPiece upiece;
  int32_t u_has_turn;
  float u_to_obj_s, u_to_obj_c;
  // Ray sharing, for a wave whose segments share rays (null otherwise): per
  // slot its leader's slot (~0u for none) and its shadow record of the
  // current depth (position, depth + 1); per shadow record whether it
  // reached its light; the queues of closest rays to trace (qt) and to take
  // from their leader (qx), and the same for shadow records (qst, qsx).
  // Whether a path is alive at a depth is in bits 2..7 of its meta.w (the
  // depth it was last continued to).
  uint32_t* lead;
  uint2* shrec;
  uint8_t* vis;
  uint32_t *qt, *qx, *qst, *qsx;
  uint32_t* qsc;  // bounce-0 paths that take their leader's shading
};

// Queue counters of one wave: active paths per bounce, shade-queue lengths
// per bounce and class, shadow rays per bounce.  Each queue also has a work
// counter (CNT_WORK) from which the kernel that drains it takes batches.
#define CNT_ACT(d) (d)
#define CNT_CLS(d, c) ((ARGENT_MAX_DEPTH + 2) + (d) * NUM_CLS + (c))
#define CNT_SH(d) ((ARGENT_MAX_DEPTH + 2) * (1 + NUM_CLS) + (d))
// Ray sharing: closest rays to trace and to take from their leaders, shadow
// records to trace and to take from their leaders.
#define CNT_TR(d) ((ARGENT_MAX_DEPTH + 2) * (2 + NUM_CLS) + (d))
#define CNT_CP(d) ((ARGENT_MAX_DEPTH + 2) * (3 + NUM_CLS) + (d))
#define CNT_STR(d) ((ARGENT_MAX_DEPTH + 2) * (4 + NUM_CLS) + (d))
#define CNT_SCP(d) ((ARGENT_MAX_DEPTH + 2) * (5 + NUM_CLS) + (d))
// Ray sharing: bounce-0 paths that take their leader's shading.
#define CNT_SC(d) ((ARGENT_MAX_DEPTH + 2) * (6 + NUM_CLS) + (d))
#define CNT_QUEUES ((ARGENT_MAX_DEPTH + 2) * (7 + NUM_CLS))
#define CNT_WORK(q) (CNT_QUEUES + (q))
#define CNT_TOTAL (2 * CNT_QUEUES)

// Dynamic work distribution over a queue: a warp takes 32 consecutive
// entries at a time.  Its first batch is fixed by its index in the grid; the
// later ones come from the queue's work counter (zeroed with the queue
// counters), so warps whose rays finish early take more batches.  The loop
// condition is warp-uniform, as the ballots in the loop bodies require.
__device__ __forceinline__ uint32_t warp_first_batch() {
  return (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32u;
}
__device__ __forceinline__ uint32_t warp_next_batch(uint32_t* work) {
  uint32_t b = 0;
  if ((threadIdx.x & 31) == 0) b = atomicAdd(work, 32u);
  return __shfl_sync(0xffffffffu, b, 0) + gridDim.x * blockDim.x;
}

__device__ __forceinline__ const DevSegment& find_segment(const WaveDesc& w, uint32_t slot) {
  uint32_t s = 0;
  while (s + 1 < w.num_segments && slot >= w.seg[s + 1].slot_begin) ++s;
  return w.seg[s];
}

// camera.rs:57-69
__device__ __forceinline__ void camera_ray(const ArgentCamera& c, float sx, float sy, float lu, float lv, V3* o,
                                           V3* d) {
  V3 pos = ld3(c.pos), fwd = ld3(c.forward), right = ld3(c.right), up = ld3(c.up);
  float x = (sx + c.shift[0]) * c.half_w;
  float y = (sy + c.shift[1]) * c.half_h;
  V3 dir = normalize(fwd + right * x + up * y);
  if (c.lens_radius <= 0.0f) {
    *o = pos;
    *d = dir;
    return;
  }
  float ft = c.focus_dist / dot(dir, fwd);
  V3 p_focus = pos + dir * ft;
  float dx, dy;
  disk(lu, lv, &dx, &dy);
  V3 oo = pos + right * (dx * c.lens_radius) + up * (dy * c.lens_radius);
  *o = oo;
  *d = normalize(p_focus - oo);
}

// render.rs:82-93: one camera sample per slot.
__global__ void __launch_bounds__(256) k_raygen(WaveArgs a, WaveDesc w) {
  if (blockIdx.x == 0) {
    for (int i = threadIdx.x; i < CNT_TOTAL; i += blockDim.x) a.counters[i] = (i == CNT_ACT(0)) ? w.num_slots : 0u;
  }
  for (uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < w.num_slots; slot += gridDim.x * blockDim.x) {
    const DevSegment& sg = find_segment(w, slot);
    const DevJob& job = a.jobs[sg.job];
    uint32_t k = slot - sg.slot_begin;
    uint32_t pix = sg.p0 + k % sg.pn;
    uint32_t si = job.first + sg.s0 + k / sg.pn;
    uint32_t x = pix % job.w, y = pix / job.w;
    if (a.lead) {
      a.lead[slot] = sg.lead == ~0u ? ~0u : sg.lead + k;
      a.shrec[slot] = make_uint2(0u, 0u);  // no shadow record yet
    }
    uint32_t pix_seed = hash32((y * job.w + x) ^ job.seed_h);
    Sampler s;
    s.init(pix_seed, si);
    float jx = tent(s.next(), 1.0f);
    float jy = tent(s.next(), 1.0f);
    float lu = s.next();
    float lv = s.next();
    Wavelengths wl = sample_visible(s.next());
    float aspect_sx = 2.0f / (float)job.w;
    float aspect_sy = 2.0f / (float)job.h;
    float sx = (((float)x + 0.5f + jx) * aspect_sx) - 1.0f;
    float sy = 1.0f - (((float)y + 0.5f + jy) * aspect_sy);
    V3 o, d;
    camera_ray(job.cam, sx, sy, lu, lv, &o, &d);
    // The throughput (1 at bounce 0) and the guides are not stored here: the
    // bounce-0 shading takes beta = 1 and writes every path's guides (zero
    // where it has none), so ray generation writes 48 B less per path.  A
    // job without bounces zeroes its guides here, for the film pass.
    a.o[slot] = make_float4(o.x, o.y, o.z, 0.0f);
    a.d[slot] = make_float4(d.x, d.y, d.z, 1.0f);  // w = prev_pdf
    a.L[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    a.lambda[slot] = make_float4(wl.lambda[0], wl.lambda[1], wl.lambda[2], wl.lambda[3]);
    a.pdf[slot] = make_float4(wl.pdf[0], wl.pdf[1], wl.pdf[2], wl.pdf[3]);
    if (job.max_depth == 0) {
      a.albedo[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      a.normal[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    // flags: bit0 specular, bit1 rough_seen, bits 8..15 medium (material+1), bits 16..31 job
    a.meta[slot] = make_uint4(pix, si, pix_seed, 1u | (sg.job << 16));
    a.rng[slot] = s.rng;
    a.q_in[slot] = slot;
  }
}

// Warp-aggregated queue append: one atomic per warp, ballot prefix for the
// lane offsets.  Every lane of the warp must call it.
__device__ __forceinline__ void warp_append(bool pred, uint32_t value, uint32_t* counter, uint32_t* queue,
                                            uint32_t cap, uint32_t* status) {
  unsigned m = __ballot_sync(0xffffffffu, pred);
  if (!m) return;
  int lane = threadIdx.x & 31;
  int leader = __ffs(m) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(m));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (pred) {
    uint32_t pos = base + __popc(m & ((1u << lane) - 1u));
    if (pos < cap)
      queue[pos] = value;
    else
      atomicOr(status, ARGENT_STATUS_QUEUE_OVERFLOW);
  }
}

// Shadow-ray append from inside shading's divergent NEE branch: the lanes
// that reach it together take one run of queue positions with one atomic
// (the active mask is the group; lanes that arrive apart take runs of their
// own).  The record is written where it is built, so its twelve values are
// not held through the continuation sample.  The order of the records in the
// queue does not matter: each adds to its own path's radiance.
__device__ __forceinline__ void push_shadow(const WaveArgs& a, int depth, float4 o, float4 d, float4 c) {
  unsigned m = __activemask();
  int lane = threadIdx.x & 31;
  int leader = __ffs(m) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(a.counters + CNT_SH(depth), (uint32_t)__popc(m));
  base = __shfl_sync(m, base, leader);
  uint32_t pos = base + __popc(m & ((1u << lane) - 1u));
  if (pos < a.cap) {
    a.sh_o[pos] = o;
    a.sh_d[pos] = d;
    a.sh_c[pos] = c;
  } else {
    atomicOr(a.status, ARGENT_STATUS_QUEUE_OVERFLOW);
  }
}

// Persistent-lane work fetch, shared by k_intersect and k_shadow: a warp
// keeps each lane on one queue entry and, when at least ARGENT_REFILL lanes
// are idle (or all are), hands them the next entries in one atomic.  The
// warp's first 32 entries are fixed by its index in the grid, as in
// warp_first_batch.  Returns the queue index given to this lane (or ~0u)
// and clears *more once the queue has run out; the decisions are
// warp-uniform.
#ifndef ARGENT_REFILL
#define ARGENT_REFILL 16
#endif
#ifndef ARGENT_FIN_BATCH
#define ARGENT_FIN_BATCH 24
#endif
__device__ __forceinline__ uint32_t lane_refill(bool idle, bool* first, bool* more, uint32_t count, uint32_t* work) {
  const unsigned lane = threadIdx.x & 31;
  unsigned need = __ballot_sync(0xffffffffu, idle);
  if (!*more || need == 0 || (!*first && __popc(need) < ARGENT_REFILL && need != 0xffffffffu)) return ~0u;
  uint32_t b;
  if (*first) {
    b = warp_first_batch();
    *first = false;
  } else {
    uint32_t t = 0;
    if (lane == 0) t = atomicAdd(work, (uint32_t)__popc(need));
    b = __shfl_sync(0xffffffffu, t, 0) + gridDim.x * blockDim.x;
  }
  if (b + (uint32_t)__popc(need) >= count) *more = false;
  if (!idle) return ~0u;
  uint32_t j = b + (uint32_t)__popc(need & ((1u << lane) - 1u));
  return j < count ? j : ~0u;
}

// scene.rs:169-218: closest hit of every active path (piece BVH in object
// space, then panels, then floor), then the path is queued for the shading
// kernel of its hit's material class.  Persistent lanes step their BVH
// traversals one node or leaf at a time and take a new path as soon as
// theirs is done.
// Rows of the traversal kernels' shared-memory stack rings (ShortStack);
// 0 keeps the whole stack in local memory.  The kernels run 128 threads per
// block.  Measured on B200 (signet still, eight lanes): local stacks 1.756 G
// path-samples/s, rings of 8 rows 1.727 G, of 16 rows 1.722 G -- the rings'
// shared memory (8-16 KB per block) costs the other lanes' kernels L1 and
// co-residency more than the stack traffic it saves (the local stack hits
// in L1), so the default is 0.
#ifndef ARGENT_SHORT_STACK
#define ARGENT_SHORT_STACK 0
#endif
#ifndef ARGENT_SHORT_STACK_ANY
#define ARGENT_SHORT_STACK_ANY 0
#endif
#if ARGENT_SHORT_STACK > 0
#define ARGENT_CLOSEST_STACK(name)                                             \
  __shared__ uint2 name##_ring[ARGENT_SHORT_STACK * 128];                      \
  uint2 name##_spill[ARGENT_STACK_SIZE];                                       \
  ShortStack<uint2, ARGENT_SHORT_STACK, 128> name{name##_ring + threadIdx.x, name##_spill}
#else
#define ARGENT_CLOSEST_STACK(name)   \
  uint2 name##_arr[ARGENT_STACK_SIZE]; \
  LocalStack<uint2> name { name##_arr }
#endif
#if ARGENT_SHORT_STACK_ANY > 0
#define ARGENT_ANY_STACK(name)                                                     \
  __shared__ uint32_t name##_ring[ARGENT_SHORT_STACK_ANY * 128];                   \
  uint32_t name##_spill[ARGENT_STACK_SIZE];                                        \
  ShortStack<uint32_t, ARGENT_SHORT_STACK_ANY, 128> name{name##_ring + threadIdx.x, name##_spill}
#else
#define ARGENT_ANY_STACK(name)          \
  uint32_t name##_arr[ARGENT_STACK_SIZE]; \
  LocalStack<uint32_t> name { name##_arr }
#endif

template <bool U>
__global__ void __launch_bounds__(128, ARGENT_TRAV_BLOCKS) k_intersect(WaveArgs a, int depth) {
  // With ray sharing, the rays that take their leader's hit are left out
  // (k_share_split) and the rest come from the trace queue.
  const uint32_t cq = a.lead ? CNT_TR(depth) : CNT_ACT(depth);
  const uint32_t count = a.counters[cq];
  uint32_t* work = a.counters + CNT_WORK(cq);
  const uint32_t* qin = a.lead ? a.qt : a.q_in;
  ARGENT_CLOSEST_STACK(stack);
  ClosestTrav s;
  const DevScene* sc = U ? a.uscene : nullptr;
  uint32_t slot = 0;
  bool active = false, running = false, first = true, more = true;
  for (;;) {
    uint32_t j = lane_refill(!active, &first, &more, count, work);
    if (j != ~0u) {
      slot = qin[j];
      if (!U) sc = a.jobs[a.meta[slot].w >> 16].scene;
      float4 of = a.o[slot], df = a.d[slot];
      V3 oo{of.x, of.y, of.z}, od{df.x, df.y, df.z};
      if (U ? a.u_has_turn : sc->has_turn) {
        float ts = U ? a.u_to_obj_s : sc->to_obj_s, tc = U ? a.u_to_obj_c : sc->to_obj_c;
        oo = rot_y_sc(oo, ts, tc);
        od = rot_y_sc(od, ts, tc);
      }
      running = closest_begin(U ? a.upiece : sc->piece, s, oo, od, INFINITY);
      active = true;
    }
    if (__ballot_sync(0xffffffffu, active) == 0 && !more) break;
    // One step: the lanes at a leaf or the lanes at a node, whichever are
    // more, visit it; the others wait, so the warp runs one of the two
    // code paths per step instead of both.
    if (active && running) running = closest_next(s, stack);
    {
      bool at_leaf = active && running && trav_at_leaf(s.ref);
      bool at_node = active && running && !trav_at_leaf(s.ref);
      bool leaves = __popc(__ballot_sync(0xffffffffu, at_leaf)) >= __popc(__ballot_sync(0xffffffffu, at_node));
      if (leaves ? at_leaf : at_node) running = closest_visit(U ? a.upiece : sc->piece, s, stack, a.status);
    }
    // Lanes whose traversal is over wait until ARGENT_FIN_BATCH of them (or
    // every active lane) can record their hits together: the panel and
    // floor tests and the queue appends then run once for many lanes.
    bool waiting = active && !running;
    unsigned wm = __ballot_sync(0xffffffffu, waiting);
    unsigned rm = __ballot_sync(0xffffffffu, active && running);
    if (wm == 0 || (__popc(wm) < ARGENT_FIN_BATCH && rm != 0)) continue;
    bool fin = waiting;
    int cls = -1;
    if (fin) {
      count_visits(0, s.n_nodes, s.n_tris);
      float4 of = a.o[slot], df = a.d[slot];
      V3 o{of.x, of.y, of.z}, d{df.x, df.y, df.z};
      float t_max = INFINITY;
      float4 rec = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(HIT_MISS));
      cls = CLS_TERMINAL;
      if (s.best.prim != ARGENT_NO_HIT_U) {
        t_max = s.best.t;
        rec = make_float4(s.best.t, s.best.u, s.best.v, __uint_as_float(s.best.prim));
        cls = sc->mat_class[__ldg(&(U ? a.upiece : sc->piece).tri_idx[s.best.prim].w)];
      }
      for (int p = 0; p < sc->num_panels; ++p) {
        const DevPanel& pn = sc->panels[p];
        if (depth == 0 && !pn.camera_visible) continue;
        float t;
        if (panel_intersect(pn, o, d, t_max, &t)) {
          t_max = t;
          rec = make_float4(t, 0.0f, 0.0f, __uint_as_float(HIT_PANEL | (uint32_t)p));
          cls = CLS_TERMINAL;
        }
      }
      if (sc->floor_enabled) {
        float t;
        if (floor_intersect(sc, o, d, t_max, &t)) {
          rec = make_float4(t, 0.0f, 0.0f, __uint_as_float(HIT_FLOOR));
          cls = sc->floor_class;
        }
      }
      a.hit[slot] = rec;
      active = false;
    }
    if (__ballot_sync(0xffffffffu, fin)) {
#pragma unroll
      for (int c = 0; c < NUM_CLS; ++c)
        warp_append(cls == c, slot, a.counters + CNT_CLS(depth, c), a.qc + (size_t)c * a.cap, a.cap, a.status);
    }
  }
}

// A shadow ray that misses the piece's box is unoccluded: its contribution
// is added here exactly as k_shadow adds a clear ray's (the stored radiance
// plus c), and the ray is not queued.  The terminal class keeps its
// radiance in `L` (stored at the end); the others read and write it here.
template <int CLS>
__device__ __forceinline__ void add_unoccluded(const WaveArgs& a, uint32_t slot, Spec* L, const Spec& c) {
  if constexpr (CLS == CLS_TERMINAL) {
    *L = *L + c;
  } else {
    float4 l = a.L[slot];
    a.L[slot] = make_float4(l.x + c.v[0], l.y + c.v[1], l.z + c.v[2], l.w + c.v[3]);
  }
}

struct ShadeOut {
  bool alive;
  bool shadow;
  float4 sh_o, sh_d, sh_c;
};

// Classes whose shadow records are appended inside the NEE branch
// (push_shadow) rather than by the whole warp after the bounce.  Measured on
// B200: the coated class (the studio floor) spills 20 B instead of 68 B and
// runs 3-4 % faster (88 -> 85 ms per signet frame, the frame 0.4-1.1 %);
// with every class appending inline the white studio's diffuse ("other")
// class ran 7 % slower, so the others keep the warp-wide append.
template <int CLS>
struct InlineShadow {
  static constexpr bool value = CLS == CLS_COATED;
};

// integrator.rs:59-218, one bounce of one path whose hit belongs to class
// CLS: CLS_TERMINAL takes misses and panel hits, the other classes take
// surface hits (piece or floor) of their materials.  MAP false compiles the
// env-map code out, for waves whose scenes have none.
template <int CLS, bool MAP>
__device__ __forceinline__ ShadeOut shade_path(const WaveArgs& a, uint32_t slot, int depth) {
  constexpr unsigned KM = ClassKinds<CLS>::value;
  ShadeOut out;
  out.alive = false;
  out.shadow = false;
  uint4 meta = a.meta[slot];
  const DevJob& job = a.jobs[meta.w >> 16];
  const DevScene* sc = job.scene;
  uint32_t flags = meta.w;
  bool specular = flags & 1u;
  bool rough_seen = (flags >> 1) & 1u;
  uint32_t medium = (flags >> 8) & 0xffu;
  Sampler s;
  s.resume(meta.z, meta.y, a.rng[slot]);
  s.set_dim(8u + (uint32_t)depth * 8u);
  float4 of = a.o[slot], df = a.d[slot], hf = a.hit[slot];
  V3 ro{of.x, of.y, of.z}, rd{df.x, df.y, df.z};
  float prev_pdf = df.w;
  Spec beta = depth == 0 ? spec(1.0f) : spec4(a.beta[slot]);
  bool guided = false;  // bounce 0: this path's guides are written
  // Radiance changes here only for terminal hits and floor fade misses, and
  // the wavelength pdfs only when a dispersive refraction terminates the
  // secondaries: the other classes read and write them only where they do.
  constexpr bool kPdf = KM_HAS(KM, B_DIELECTRIC);
  Spec L = CLS == CLS_TERMINAL ? spec4(a.L[slot]) : spec(0.0f);
  float4 lf = a.lambda[slot], pf = kPdf ? a.pdf[slot] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  Wavelengths wl{{lf.x, lf.y, lf.z, lf.w}, {pf.x, pf.y, pf.z, pf.w}};
  bool clamp = rough_seen;
  float cl = job.clamp_indirect;
  uint32_t kind = __float_as_uint(hf.w);
  float t = hf.x;

  if (medium && kind != HIT_MISS) {
    Spec sig = tab_sample(sc->mats[medium - 1].spec_b, wl);
    Spec e;
#pragma unroll
    for (int i = 0; i < 4; ++i) e.v[i] = expf(-sig.v[i] * t);
    beta = beta * e;
  }
  const bool env_map = MAP && sc->env_is_map != 0;
  V3 p, p_obj, ng, ns;
  uint32_t mat_id = 0;
  float cavity = 0.0f;
  bool done = false;
  if (CLS == CLS_TERMINAL && kind == HIT_MISS) {
    float w = 1.0f;
    Spec le;
    if (env_map) {
      EnvTexel et = env_texel(sc, rd);
      if (!specular) {
        float pl = sc->env_pick * envmap_pdf_at(sc, et);
        w = prev_pdf * prev_pdf / (prev_pdf * prev_pdf + pl * pl);
      }
      le = envmap_eval_at(sc, et, wl);
    } else {
      le = env_eval<false>(sc, rd, wl);
    }
    add_clamped(&L, beta * le * w, clamp, cl);
    done = true;
  } else if (CLS == CLS_TERMINAL) {  // panel (light.rs:67-72, integrator.rs:84-98)
    int idx = (int)(kind & 0x0FFFFFFFu);
    const DevPanel& pn = sc->panels[idx];
    Spec le = panel_le(pn, ro + rd * t, rd, wl);
    if (!is_black(le)) {
      if (specular) {
        add_clamped(&L, beta * le, clamp, cl);
      } else {
        float cos_l = fmaxf(fabsf(dot(-rd, ld3(pn.n))), 1e-8f);
        float p_light = (1.0f - sc->env_pick) * light_pick_pdf(sc, idx) * t * t / (cos_l * pn.area);
        float w = prev_pdf * prev_pdf / (prev_pdf * prev_pdf + p_light * p_light);
        add_clamped(&L, beta * le * w, clamp, cl);
      }
    }
    done = true;
  } else if (kind == HIT_FLOOR) {
    V3 fp = ro + rd * t;
    if (s.next_random() >= floor_presence(sc, fp)) {
      float w = 1.0f;
      Spec le;
      if (env_map) {
        EnvTexel et = env_texel(sc, rd);
        if (!specular) {
          float pl = sc->env_pick * envmap_pdf_at(sc, et);
          w = prev_pdf * prev_pdf / (prev_pdf * prev_pdf + pl * pl);
        }
        le = envmap_eval_at(sc, et, wl);
      } else {
        le = env_eval<false>(sc, rd, wl);
      }
      if constexpr (CLS != CLS_TERMINAL) L = spec4(a.L[slot]);
      add_clamped(&L, beta * le * w, clamp, cl);
      if constexpr (CLS != CLS_TERMINAL) a.L[slot] = to_f4(L);
      done = true;
    } else {
      V3 n = rd.y < 0.0f ? V3{0.0f, 1.0f, 0.0f} : V3{0.0f, -1.0f, 0.0f};
      p = fp;
      p_obj = fp;
      ng = n;
      ns = n;
      mat_id = (uint32_t)sc->floor_material;
    }
  } else {
    // scene.rs:174-201: hit attributes of the piece.
    const DevPiece& pc = sc->piece;
    uint4 tri = __ldg(pc.tri_idx + kind);
    float4 fa = __ldg(pc.pos + tri.x), fb = __ldg(pc.pos + tri.y), fc = __ldg(pc.pos + tri.z);
    V3 A{fa.x, fa.y, fa.z}, B{fb.x, fb.y, fb.z}, C{fc.x, fc.y, fc.z};
    float hu = hf.y, hv = hf.z;
    V3 ngo = normalize(cross(B - A, C - A));
    float w = 1.0f - hu - hv;
    mat_id = tri.w;
    const ArgentMaterial* m = sc->mats + mat_id;
    bool flat = m->kind == ARGENT_MAT_GEM && m->gem_kind == ARGENT_GEM_TRANSPARENT;
    V3 nso;
    if (flat || pc.nrm == nullptr) {
      nso = ngo;
    } else {
      float4 na = __ldg(pc.nrm + tri.x), nb = __ldg(pc.nrm + tri.y), nc = __ldg(pc.nrm + tri.z);
      V3 n = V3{na.x, na.y, na.z} * w + V3{nb.x, nb.y, nb.z} * hu + V3{nc.x, nc.y, nc.z} * hv;
      nso = length_squared(n) > 1e-12f ? normalize(n) : ngo;
    }
    if (pc.cavity) cavity = __ldg(pc.cavity + tri.x) * w + __ldg(pc.cavity + tri.y) * hu + __ldg(pc.cavity + tri.z) * hv;
    p_obj = A * w + B * hu + C * hv;
    if (sc->has_turn) {
      p = rot_y_sc(p_obj, sc->to_world_s, sc->to_world_c);
      ng = rot_y_sc(ngo, sc->to_world_s, sc->to_world_c);
      ns = rot_y_sc(nso, sc->to_world_s, sc->to_world_c);
    } else {
      p = p_obj;
      ng = ngo;
      ns = nso;
    }
  }

  if constexpr (CLS != CLS_TERMINAL) {
  if (!done) {
    const ArgentMaterial* mat = sc->mats + mat_id;
    V3 wo_w = -rd;
    bool transmissive = mat_is_transmissive(mat);
    V3 nsu = ns, ngu = ng;
    if (!transmissive && dot(ng, wo_w) < 0.0f) {
      nsu = -ns;
      ngu = -ng;
    }
    if (!transmissive && dot(nsu, wo_w) <= 0.0f) nsu = ngu;
    Frame frame = make_frame(nsu);
    V3 wo = to_local(frame, wo_w);
    HitCtx ctx{p_obj, nsu, &frame, sc->to_world_s, sc->to_world_c};
    if (!sc->has_turn) {
      ctx.turn_s = 0.0f;
      ctx.turn_c = 1.0f;
    }
    float ub = s.next();
    Bsdf bsdf = material_bsdf<CLS>(mat, wl, cavity, ub, ctx);
    if (bsdf.kind == B_CONDUCTOR && !is_smooth(bsdf.ggx)) {
      bsdf.f0 = fresnel_conductor(1.0f, bsdf.eta, bsdf.k);
      bsdf.e_wo = ggx_e(bsdf.ggx, wo.z);
    }
    if (depth == 0) {
      float g[3];
      guide_rgb(mat, cavity, g);
      a.albedo[slot] = make_float4(g[0], g[1], g[2], 0.0f);
      a.normal[slot] = make_float4(nsu.x, nsu.y, nsu.z, 0.0f);
      guided = true;
    }

    // Next-event estimation (integrator.rs:130-178).
    if (!bsdf_is_delta(bsdf)) {
      float ul = s.next();
      float u1 = s.next();
      float u2 = s.next();
      // The light sample: the env map (with probability env_pick when the
      // scene has one) or a panel by the power CDF.  From the BSDF value on,
      // both take one code path (MIS weight, the panel and floor visibility
      // tests, the shadow ray), so a warp whose paths chose different lights
      // evaluates the BSDF once.  The arithmetic of each case is unchanged:
      // a panel sample's visibility factor is exactly 1.
      const bool use_env = env_map && ul < sc->env_pick;
      bool valid = false;
      V3 dir{0.0f, 0.0f, 0.0f};  // toward the sample, from p
      V3 lp{0.0f, 0.0f, 0.0f};   // the point on the sampled panel
      EnvTexel etx{0u, 0u, 0.0f};  // the map texel of a map sample
      float p_light = 0.0f;
      int li = -1;  // the sampled panel, left out of the visibility test
      if (use_env) {
        float pdf_dir;
        dir = envmap_sample(sc, u1, u2, &pdf_dir, &etx);
        valid = pdf_dir > 0.0f && dot(dir, ngu) > 0.0f;
        p_light = sc->env_pick * pdf_dir;
      } else if (sc->num_lights > 0) {
        // scene.rs:149-156
        float u = sc->env_pick > 0.0f ? (ul - sc->env_pick) / (1.0f - sc->env_pick) : ul;
        int k = 0;
        {
          int lo = 0, hi = sc->num_lights;
          while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (sc->light_cdf[mid] < u)
              lo = mid + 1;
            else
              hi = mid;
          }
          k = min(lo, sc->num_lights - 1);
        }
        float pick = sc->light_cdf[k] - (k == 0 ? 0.0f : sc->light_cdf[k - 1]);
        li = sc->lights[k];
        pick = pick * (1.0f - sc->env_pick);
        const DevPanel& pn = sc->panels[li];
        lp = ld3(pn.c) + ld3(pn.hu) * (2.0f * u1 - 1.0f) + ld3(pn.hv) * (2.0f * u2 - 1.0f);
        V3 to = lp - p;
        float d2 = length_squared(to);
        dir = to / sqrtf(d2);
        float cos_l = dot(-dir, ld3(pn.n));
        valid = cos_l > 0.0f && dot(dir, ngu) > 0.0f;
        p_light = pick * d2 / (cos_l * pn.area);
      }
      if (valid) {
        V3 wi = to_local(frame, dir);
        Spec f;
        float p_bsdf;
        bsdf_eval_pdf<KM>(bsdf, wo, wi, &f, &p_bsdf);
        if (!is_black(f)) {
          float w = p_light * p_light / (p_light * p_light + p_bsdf * p_bsdf);
          // sky_visibility (scene.rs:123-140) for the map, visible
          // (scene.rs:222-243) for a panel: panels and floor here, the piece
          // in k_shadow.
          V3 origin = offset_origin(p, ngu, dir);
          V3 sdir = dir;
          float t_max = INFINITY;
          if (!use_env) {
            V3 dd = lp - origin;
            float dist = length(dd);
            sdir = dd / dist;
            t_max = dist * (1.0f - 1e-4f);
          }
          float vis = 1.0f;
          for (int q = 0; q < sc->num_panels && vis > 0.0f; ++q) {
            float tt;
            if (q != li && panel_intersect(sc->panels[q], origin, sdir, t_max, &tt)) vis = 0.0f;
          }
          if (vis > 0.0f && sc->floor_enabled) {
            float tt;
            if (floor_intersect(sc, origin, sdir, t_max, &tt))
              vis = use_env ? 1.0f - floor_presence(sc, origin + sdir * tt) : 0.0f;
          }
          if (vis > 0.0f) {
            Spec le = use_env ? envmap_eval_at(sc, etx, wl) : panel_le(sc->panels[li], lp, dir, wl);
            Spec c = beta * f * le * (fabsf(wi.z) * w * vis / p_light);
            c = clamped(c, rough_seen, cl);
            V3 oo = origin, od = sdir;
            if (sc->has_turn) {
              oo = rot_y_sc(origin, sc->to_obj_s, sc->to_obj_c);
              od = rot_y_sc(sdir, sc->to_obj_s, sc->to_obj_c);
            }
            if (piece_may_occlude(sc->piece, oo, od, t_max)) {
              float4 so = make_float4(oo.x, oo.y, oo.z, t_max);
              float4 sd = make_float4(od.x, od.y, od.z, __uint_as_float(slot));
              if constexpr (InlineShadow<CLS>::value) {
                push_shadow(a, depth, so, sd, to_f4(c));
              } else {
                out.shadow = true;
                out.sh_o = so;
                out.sh_d = sd;
                out.sh_c = to_f4(c);
              }
            } else {
              add_unoccluded<CLS>(a, slot, &L, c);
            }
          }
        }
      }
    } else {
      s.next();
      s.next();
      s.next();
    }

    // Continue the path (integrator.rs:180-218).
    float u0 = s.next();
    float u1 = s.next();
    float u2 = s.next();
    BsdfSample smp;
    bool cont = bsdf_sample<KM>(bsdf, wo, u0, u1, u2, &smp);
    if (cont && (smp.pdf <= 0.0f || is_black(smp.f))) cont = false;
    V3 wi_w;
    if (cont) {
      wi_w = to_world(frame, smp.wi);
      float side = dot(wi_w, ngu) * dot(wo_w, ngu);
      if ((!smp.transmit && side <= 0.0f) || (smp.transmit && side >= 0.0f)) cont = false;
    }
    if (cont) {
      if (smp.terminate_secondary) terminate_secondary(&wl);
      beta = beta * (smp.f * (fabsf(smp.wi.z) / smp.pdf));
      if (!is_finite(beta)) cont = false;
    }
    if (cont) {
      specular = smp.delta;
      if (!smp.delta) rough_seen = true;
      prev_pdf = smp.pdf;
      if (smp.transmit) medium = (wo.z > 0.0f && mat_has_medium(mat)) ? mat_id + 1u : 0u;
      ro = offset_origin(p, ngu, wi_w);
      rd = wi_w;
      if ((uint32_t)depth >= job.rr_depth) {
        float survive = fminf(max_value(beta), 0.95f);
        if (survive <= 0.0f || s.next_random() >= survive)
          cont = false;
        else
          beta = beta / survive;
      }
    }
    out.alive = cont && ((uint32_t)depth + 1u < job.max_depth);
    // Store the state the next bounce (or the film) reads.
    a.beta[slot] = to_f4(beta);
    if constexpr (kPdf) a.pdf[slot] = make_float4(wl.pdf[0], wl.pdf[1], wl.pdf[2], wl.pdf[3]);
    if (out.alive) {
      a.o[slot] = make_float4(ro.x, ro.y, ro.z, 0.0f);
      a.d[slot] = make_float4(rd.x, rd.y, rd.z, prev_pdf);
      // Bits 2..7: the depth the path is alive at (ray sharing reads it).
      uint32_t nf = (flags & 0xffff0000u) | (specular ? 1u : 0u) | (rough_seen ? 2u : 0u) |
                    ((((uint32_t)depth + 1u) & 63u) << 2) | (medium << 8);
      a.meta[slot].w = nf;
      a.rng[slot] = s.rng;
    }
  }
  }
  if constexpr (CLS == CLS_TERMINAL) a.L[slot] = to_f4(L);
  if (depth == 0 && !guided) {
    // A camera ray that ends at its first hit (miss, panel, faded floor)
    // has no guides: the film adds zeros.
    a.albedo[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    a.normal[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  }
  return out;
}

// Register budgets of the shading classes.  Metal and the other surface
// classes are capped at 128 registers (4 blocks of 128 per SM) instead of up
// to ~166; lower caps spill them heavily and run slower.  The coated class
// (the studio floor, the largest shading launch) runs at 96 registers, 5
// blocks, with about 60 B of spill, on a grid of its own 5 blocks per SM.
// The dielectric class fits 96 registers without spilling.  The terminal,
// dielectric and other classes launch on a grid of ARGENT_SHADE_BLOCKS (4)
// blocks per SM, metal and coated on grids of their own occupancy:
// wider grids for the terminal (8) and dielectric (5) classes took SMs from
// the other lanes' kernels and ran slower.
#ifndef ARGENT_SHADE_BLOCKS
#define ARGENT_SHADE_BLOCKS 4
#endif
#ifndef ARGENT_SHADE_BLOCKS_DIELECTRIC
#define ARGENT_SHADE_BLOCKS_DIELECTRIC 5
#endif
#ifndef ARGENT_SHADE_BLOCKS_COATED
#define ARGENT_SHADE_BLOCKS_COATED 5
#endif
#ifndef ARGENT_SHADE_BLOCKS_METAL
#define ARGENT_SHADE_BLOCKS_METAL ARGENT_SHADE_BLOCKS
#endif
template <int CLS, bool MAP>
__global__ void __launch_bounds__(128, CLS == CLS_TERMINAL      ? 1
                                       : CLS == CLS_DIELECTRIC ? ARGENT_SHADE_BLOCKS_DIELECTRIC
                                       : CLS == CLS_COATED     ? ARGENT_SHADE_BLOCKS_COATED
                                       : CLS == CLS_METAL      ? ARGENT_SHADE_BLOCKS_METAL
                                                               : ARGENT_SHADE_BLOCKS)
    k_shade(WaveArgs a, int depth) {
  uint32_t count = a.counters[CNT_CLS(depth, CLS)];
  const uint32_t* q = a.qc + (size_t)CLS * a.cap;
  uint32_t cap = a.cap;
  uint32_t* next_counter = a.counters + CNT_ACT(depth + 1);
  uint32_t* work = a.counters + CNT_WORK(CNT_CLS(depth, CLS));
  for (uint32_t base = warp_first_batch(); base < count; base = warp_next_batch(work)) {
    uint32_t i = base + (threadIdx.x & 31);
    ShadeOut r;
    r.alive = false;
    r.shadow = false;
    uint32_t slot = 0;
    if (i < count) {
      slot = q[i];
      r = shade_path<CLS, MAP>(a, slot, depth);
    }
    warp_append(r.alive, slot, next_counter, a.q_out, cap, a.status);
    if constexpr (!InlineShadow<CLS>::value) {
      // Shadow rays: the record is written at the queue position.
      unsigned m = __ballot_sync(0xffffffffu, r.shadow);
      if (m) {
        int lane = threadIdx.x & 31;
        int leader = __ffs(m) - 1;
        uint32_t sbase = 0;
        if (lane == leader) sbase = atomicAdd(a.counters + CNT_SH(depth), (uint32_t)__popc(m));
        sbase = __shfl_sync(0xffffffffu, sbase, leader);
        if (r.shadow) {
          uint32_t pos = sbase + __popc(m & ((1u << lane) - 1u));
          if (pos < cap) {
            a.sh_o[pos] = r.sh_o;
            a.sh_d[pos] = r.sh_d;
            a.sh_c[pos] = r.sh_c;
          } else {
            atomicOr(a.status, ARGENT_STATUS_QUEUE_OVERFLOW);
          }
        }
      }
    }
  }
}

// scene.rs:123-140 (piece part): any hit of the piece for each shadow ray;
// unoccluded rays add their contribution to L.  Persistent lanes, so a
// lane whose ray ends early takes a new one instead of idling until the
// slowest ray of its warp ends.
template <bool U>
__global__ void __launch_bounds__(128, ARGENT_TRAV_BLOCKS) k_shadow(WaveArgs a, int depth) {
  // With ray sharing, the records that take their leader's visibility are
  // left out (k_shadow_split) and the rest come through the trace queue;
  // each traced record's visibility is kept for its followers.
  const uint32_t cq = a.lead ? CNT_STR(depth) : CNT_SH(depth);
  const uint32_t count = a.counters[cq];
  uint32_t* work = a.counters + CNT_WORK(cq);
  ARGENT_ANY_STACK(stack);
  AnyTrav s;
  const DevScene* sc = nullptr;
  uint32_t idx = 0;
  int state = ARGENT_ANY_CLEAR;
  bool active = false, first = true, more = true;
  for (;;) {
    uint32_t j = lane_refill(!active, &first, &more, count, work);
    if (j != ~0u) {
      idx = a.lead ? a.qst[j] : j;
      float4 so = __ldcs(a.sh_o + idx), sd = __ldcs(a.sh_d + idx);
      if (!U) sc = a.jobs[a.meta[__float_as_uint(sd.w)].w >> 16].scene;
      state = any_begin(U ? a.upiece : sc->piece, s, stack, V3{so.x, so.y, so.z}, V3{sd.x, sd.y, sd.z}, so.w);
      active = true;
    }
    if (__ballot_sync(0xffffffffu, active) == 0 && !more) break;
    if (active && state == ARGENT_ANY_RUNNING && !any_next(s, stack)) state = ARGENT_ANY_CLEAR;
    {
      bool run = active && state == ARGENT_ANY_RUNNING;
      bool at_leaf = run && trav_at_leaf(s.ref);
      bool at_node = run && !trav_at_leaf(s.ref);
      bool leaves = __popc(__ballot_sync(0xffffffffu, at_leaf)) >= __popc(__ballot_sync(0xffffffffu, at_node));
      if (leaves ? at_leaf : at_node) state = any_visit(U ? a.upiece : sc->piece, s, stack, a.status);
    }
    if (active && state != ARGENT_ANY_RUNNING) {
      count_visits(3, s.n_nodes, s.n_tris);
      if (a.vis) a.vis[idx] = state == ARGENT_ANY_CLEAR ? 1u : 0u;
      if (state == ARGENT_ANY_CLEAR) {
        uint32_t slot = __float_as_uint(__ldcs(a.sh_d + idx).w);
        float4 c = __ldcs(a.sh_c + idx);
        float4 l = a.L[slot];
        a.L[slot] = make_float4(l.x + c.x, l.y + c.y, l.z + c.z, l.w + c.w);
      }
      active = false;
    }
  }
}

// ---------------------------------------------------------------- ray sharing
// Renders of one batch that differ only in their materials (metal variants
// of a piece under the same camera, seed and samples) trace the same rays
// until their paths part (a different sampled lobe, Russian roulette on a
// different throughput).  Their segments sit side by side in a wave; before
// each traversal a path whose leader (the same pixel-sample of the first
// render) is alive with a bit-identical ray takes the leader's result, so
// every shared ray is traced once.  Identical rays in identical geometry
// have identical closest hits and identical visibility, so the records and
// films equal those of tracing every ray.  Likewise a hit on a surface whose
// material (and everything else shading reads) equals the leader's, reached
// in the leader's path state, takes the leader's shading.

// The depth path `slot` was last continued to (0 from ray generation): it is
// alive at `depth` exactly when this equals `depth`.
__device__ __forceinline__ uint32_t alive_depth(const WaveArgs& a, uint32_t slot) {
  return (reinterpret_cast<const uint32_t*>(a.meta + slot)[3] >> 2) & 63u;
}

__device__ __forceinline__ bool same_bits3(float4 a, float4 b) {
  return __float_as_uint(a.x) == __float_as_uint(b.x) && __float_as_uint(a.y) == __float_as_uint(b.y) &&
         __float_as_uint(a.z) == __float_as_uint(b.z);
}

// Shading class of a hit record, for a path of scene `sc` (the classes
// k_intersect gives: miss and panels terminal, the floor's material class,
// the hit triangle's material class).
__device__ __forceinline__ int hit_class(const DevScene* sc, const DevPiece& pc, float4 rec) {
  uint32_t kind = __float_as_uint(rec.w);
  if (kind == HIT_FLOOR) return sc->floor_class;
  if (kind >= HIT_PANEL) return CLS_TERMINAL;
  return sc->mat_class[__ldg(&pc.tri_idx[kind].w)];
}

// Block-aggregated reservation for the streaming passes below: the threads
// of the block with `pred` set take consecutive positions behind `counter`
// with one atomic per block (a pass over tens of millions of entries is
// otherwise bound by the atomics on one counter); returns this thread's
// position (meaningful where `pred` is set).  Every thread of the block must
// call it; `sw` is the block's scratch of blockDim.x / 32 + 1 words.
__device__ __forceinline__ uint32_t block_reserve(bool pred, uint32_t* counter, uint32_t* sw) {
  const unsigned m = __ballot_sync(0xffffffffu, pred);
  const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u, nw = blockDim.x >> 5;
  if (lane == 0) sw[warp] = (uint32_t)__popc(m);
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t total = 0;
    for (unsigned w = 0; w < nw; ++w) {
      uint32_t c = sw[w];
      sw[w] = total;
      total += c;
    }
    sw[nw] = total ? atomicAdd(counter, total) : 0u;
  }
  __syncthreads();
  const uint32_t pos = sw[nw] + sw[warp] + (uint32_t)__popc(m & ((1u << lane) - 1u));
  __syncthreads();  // sw is reused by the next reservation
  return pos;
}

// Block-aggregated queue append (block_reserve, then the entry).
__device__ __forceinline__ void block_append(bool pred, uint32_t value, uint32_t* counter, uint32_t* queue,
                                             uint32_t cap, uint32_t* status, uint32_t* sw) {
  const uint32_t pos = block_reserve(pred, counter, sw);
  if (pred) {
    if (pos < cap)
      queue[pos] = value;
    else
      atomicOr(status, ARGENT_STATUS_QUEUE_OVERFLOW);
  }
}

// Before k_intersect: splits the alive paths of `depth` into those that take
// their leader's hit (qx) and those to trace (qt).
__global__ void __launch_bounds__(256) k_share_split(WaveArgs a, int depth) {
  __shared__ uint32_t sw[256 / 32 + 1];
  const uint32_t count = min(a.counters[CNT_ACT(depth)], a.cap);
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = blockIdx.x * blockDim.x; base < count; base += stride) {
    uint32_t i = base + threadIdx.x;
    bool valid = i < count, share = false;
    uint32_t slot = 0;
    if (valid) {
      slot = a.q_in[i];
      uint32_t ld = a.lead[slot];
      if (ld != ~0u && alive_depth(a, ld) == (uint32_t)depth)
        share = same_bits3(a.o[slot], a.o[ld]) && same_bits3(a.d[slot], a.d[ld]);
    }
    block_append(valid && share, slot, a.counters + CNT_CP(depth), a.qx, a.cap, a.status, sw);
    block_append(valid && !share, slot, a.counters + CNT_TR(depth), a.qt, a.cap, a.status, sw);
  }
}

// True when path `slot` enters shading at `depth` (> 0) in the same state as
// path `l`: throughput, radiance, wavelengths and their pdfs, sampler state,
// the previous bounce's pdf and its flags (specular, rough, medium).  The
// rays and hits are already equal.
__device__ __forceinline__ bool same_state(const WaveArgs& a, uint32_t slot, uint32_t l) {
  auto eq4 = [](float4 x, float4 y) { return same_bits3(x, y) && __float_as_uint(x.w) == __float_as_uint(y.w); };
  return eq4(a.beta[slot], a.beta[l]) && eq4(a.L[slot], a.L[l]) && eq4(a.lambda[slot], a.lambda[l]) &&
         eq4(a.pdf[slot], a.pdf[l]) && a.rng[slot] == a.rng[l] &&
         __float_as_uint(a.d[slot].w) == __float_as_uint(a.d[l].w) &&
         ((reinterpret_cast<const uint32_t*>(a.meta + slot)[3] ^ reinterpret_cast<const uint32_t*>(a.meta + l)[3]) &
          0xffffu) == 0u;
}

// After k_intersect: the paths of qx take their leaders' hit records and
// join the shade queue of their own material's class.  A path that hits a
// surface whose material record and everything else shading reads equal the
// leader's (the job's share masks), and enters shading in its leader's state
// -- at bounce 0 always (the same camera sample), later while its path has
// met only such materials -- goes to qsc instead and takes the leader's
// shading (k_shade_copy).
template <bool U>
__global__ void __launch_bounds__(256) k_hit_copy(WaveArgs a, int depth) {
  __shared__ uint32_t sw[256 / 32 + 1];
  const uint32_t count = min(a.counters[CNT_CP(depth)], a.cap);
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = blockIdx.x * blockDim.x; base < count; base += stride) {
    uint32_t i = base + threadIdx.x;
    int cls = -1;
    uint32_t slot = 0;
    bool same_shading = false;
    if (i < count) {
      slot = a.qx[i];
      float4 rec = a.hit[a.lead[slot]];
      a.hit[slot] = rec;
      const DevJob& job = a.jobs[a.meta[slot].w >> 16];
      const DevScene* sc = U ? a.uscene : job.scene;
      const DevPiece& pc = U ? a.upiece : sc->piece;
      cls = hit_class(sc, pc, rec);
      // Surface hits only: a miss or panel hit costs less to shade than to
      // copy.
      if (job.share_rest && cls != CLS_TERMINAL) {
        uint32_t kind = __float_as_uint(rec.w);
        uint32_t m = kind == HIT_FLOOR ? (uint32_t)sc->floor_material : __ldg(&pc.tri_idx[kind].w);
        same_shading =
            ((job.share_mat[m >> 5] >> (m & 31u)) & 1u) && (depth == 0 || same_state(a, slot, a.lead[slot]));
      }
      if (same_shading) cls = -1;
    }
    if (__syncthreads_or(same_shading))
      block_append(same_shading, slot, a.counters + CNT_SC(depth), a.qsc, a.cap, a.status, sw);
    for (int c = 0; c < NUM_CLS; ++c)
      if (__syncthreads_or(cls == c))
        block_append(cls == c, slot, a.counters + CNT_CLS(depth, c), a.qc + (size_t)c * a.cap, a.cap, a.status,
                     sw);
  }
}

// After the shading kernels and k_shadow_index: each path of qsc takes its
// leader's shaded state (radiance, throughput, guides, the next ray and
// sampler state, its flags but for its own job index), continues if the
// leader continues, and gets a copy of the leader's shadow record.
__global__ void __launch_bounds__(256) k_shade_copy(WaveArgs a, int depth) {
  __shared__ uint32_t sw[256 / 32 + 1];
  const uint32_t count = min(a.counters[CNT_SC(depth)], a.cap);
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = blockIdx.x * blockDim.x; base < count; base += stride) {
    uint32_t i = base + threadIdx.x;
    bool alive = false, shadow = false;
    uint32_t slot = 0, rec = 0;
    if (i < count) {
      slot = a.qsc[i];
      uint32_t l = a.lead[slot];
      a.L[slot] = a.L[l];
      a.beta[slot] = a.beta[l];
      a.lambda[slot] = a.lambda[l];
      a.pdf[slot] = a.pdf[l];
      a.albedo[slot] = a.albedo[l];
      a.normal[slot] = a.normal[l];
      a.o[slot] = a.o[l];
      a.d[slot] = a.d[l];
      a.rng[slot] = a.rng[l];
      uint32_t* mw = reinterpret_cast<uint32_t*>(a.meta + slot) + 3;
      *mw = (reinterpret_cast<const uint32_t*>(a.meta + l)[3] & 0xffffu) | (*mw & 0xffff0000u);
      alive = alive_depth(a, l) == (uint32_t)depth + 1u;
      uint2 sr = a.shrec[l];
      shadow = sr.y == (uint32_t)depth + 1u;
      rec = sr.x;
    }
    block_append(alive, slot, a.counters + CNT_ACT(depth + 1), a.q_out, a.cap, a.status, sw);
    // The shadow record: the leader's, with this path's slot.
    const uint32_t pos = block_reserve(shadow, a.counters + CNT_SH(depth), sw);
    if (shadow) {
      if (pos < a.cap) {
        float4 sd = a.sh_d[rec];
        a.sh_o[pos] = a.sh_o[rec];
        a.sh_d[pos] = make_float4(sd.x, sd.y, sd.z, __uint_as_float(slot));
        a.sh_c[pos] = a.sh_c[rec];
      } else {
        atomicOr(a.status, ARGENT_STATUS_QUEUE_OVERFLOW);
      }
    }
  }
}

// Before k_shadow_split: each path's shadow record of this depth, by slot
// (position, depth + 1).
__global__ void __launch_bounds__(256) k_shadow_index(WaveArgs a, int depth) {
  const uint32_t count = min(a.counters[CNT_SH(depth)], a.cap);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    a.shrec[__float_as_uint(a.sh_d[i].w)] = make_uint2(i, (uint32_t)depth + 1u);
}

// Before k_shadow: a shadow record whose path's leader wrote a record at
// this depth with the same origin, t_max and direction takes that record's
// visibility (qsx); the others are traced (qst).
__global__ void __launch_bounds__(256) k_shadow_split(WaveArgs a, int depth) {
  __shared__ uint32_t sw[256 / 32 + 1];
  const uint32_t count = min(a.counters[CNT_SH(depth)], a.cap);
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = blockIdx.x * blockDim.x; base < count; base += stride) {
    uint32_t i = base + threadIdx.x;
    bool valid = i < count, share = false;
    if (valid) {
      float4 so = a.sh_o[i], sd = a.sh_d[i];
      uint32_t ld = a.lead[__float_as_uint(sd.w)];
      if (ld != ~0u) {
        uint2 lr = a.shrec[ld];
        if (lr.y == (uint32_t)depth + 1u) {
          float4 lo = a.sh_o[lr.x];
          share = same_bits3(so, lo) && __float_as_uint(so.w) == __float_as_uint(lo.w) &&
                  same_bits3(sd, a.sh_d[lr.x]);
        }
      }
    }
    block_append(valid && share, i, a.counters + CNT_SCP(depth), a.qsx, a.cap, a.status, sw);
    block_append(valid && !share, i, a.counters + CNT_STR(depth), a.qst, a.cap, a.status, sw);
  }
}

// After k_shadow: a record of qsx whose leader's record reached its light
// adds its contribution, as k_shadow adds a clear ray's.
__global__ void __launch_bounds__(256) k_shadow_copy(WaveArgs a, int depth) {
  const uint32_t count = min(a.counters[CNT_SCP(depth)], a.cap);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    uint32_t r = a.qsx[i];
    uint32_t slot = __float_as_uint(a.sh_d[r].w);
    if (a.vis[a.shrec[a.lead[slot]].x]) {
      float4 c = a.sh_c[r];
      float4 l = a.L[slot];
      a.L[slot] = make_float4(l.x + c.x, l.y + c.y, l.z + c.z, l.w + c.w);
    }
  }
}

// Instrumentation: adds a finished wave's queue lengths per bounce to
// d_bounce_counts (one thread per bounce).
static_assert(ARGENT_BOUNCE_BINS == ARGENT_MAX_DEPTH, "one bounce counter per depth");
__global__ void k_count_bounces(const uint32_t* counters, int depths) {
  int d = threadIdx.x;
  if (d < depths) {
    atomicAdd(&d_bounce_counts[d], (unsigned long long)counters[CNT_ACT(d)]);
    atomicAdd(&d_bounce_counts[ARGENT_BOUNCE_BINS + d], (unsigned long long)counters[CNT_SH(d)]);
  }
}

// render.rs:96-111 + Film sums.
__global__ void __launch_bounds__(256) k_film(WaveArgs a, WaveDesc w) {
  uint32_t total = 0;
  for (uint32_t s = 0; s < w.num_segments; ++s) total += w.seg[s].pn;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    uint32_t s = 0, off = t;
    while (off >= w.seg[s].pn) {
      off -= w.seg[s].pn;
      ++s;
    }
    const DevSegment& sg = w.seg[s];
    const DevJob& job = a.jobs[sg.job];
    const float* m = job.scene->cam_m;
    float acc[3] = {0.0f, 0.0f, 0.0f}, aacc[3] = {0.0f, 0.0f, 0.0f}, nacc[3] = {0.0f, 0.0f, 0.0f};
    double acc64[3] = {0.0, 0.0, 0.0};
    for (uint32_t k = 0; k < sg.sn; ++k) {
      uint32_t slot = sg.slot_begin + k * sg.pn + off;
      float4 lf = a.L[slot], wlf = a.lambda[slot], pf = a.pdf[slot];
      Spec L{{lf.x, lf.y, lf.z, lf.w}};
      Wavelengths wl{{wlf.x, wlf.y, wlf.z, wlf.w}, {pf.x, pf.y, pf.z, pf.w}};
      float xyz[3];
      to_xyz(L, wl, xyz);
      float r0 = m[0] * xyz[0] + m[1] * xyz[1] + m[2] * xyz[2];
      float r1 = m[3] * xyz[0] + m[4] * xyz[1] + m[5] * xyz[2];
      float r2 = m[6] * xyz[0] + m[7] * xyz[1] + m[8] * xyz[2];
      if (isfinite(r0) && isfinite(r1) && isfinite(r2)) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          acc[c] += xyz[c];
          acc64[c] += (double)xyz[c];
        }
      }
      float4 al = a.albedo[slot], nr = a.normal[slot];
      aacc[0] += al.x;
      aacc[1] += al.y;
      aacc[2] += al.z;
      nacc[0] += nr.x;
      nacc[1] += nr.y;
      nacc[2] += nr.z;
    }
    size_t o = 3 * (size_t)(sg.p0 + off);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (job.film_comp) {
        // Kahan-compensated running sum.
        float sum = job.film_xyz[o + c];
        float y = acc[c] - job.film_comp[o + c];
        float tt = sum + y;
        job.film_comp[o + c] = (tt - sum) - y;
        job.film_xyz[o + c] = tt;
      } else {
        job.film_xyz[o + c] += acc[c];
      }
      if (job.film_xyz64) job.film_xyz64[o + c] += acc64[c];
      job.film_albedo[o + c] += aacc[c];
      job.film_normal[o + c] += nacc[c];
    }
  }
}

}  // namespace dev
