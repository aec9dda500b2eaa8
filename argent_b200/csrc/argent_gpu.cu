// argent_gpu.cu — the C ABI of include/argent_gpu.h: context, piece, scene,
// film, render_pass, batch and traversal entry points.  Kernels live in the
// device/*.cuh headers included here.
#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/argent_gpu.h"
#include "data/spectral_tables.h"
#include "device/dev_math.cuh"
#include "device/traverse.cuh"
#include "host/bvh_build.h"
#include "host/scene_prep.h"
#include "host/cavity.h"
#include "internal.cuh"
#include "render_impl.cuh"
#include "denoise.cuh"
#include "develop.cuh"
#include "device_build.cuh"
#include "host/develop.h"

using namespace dev;

namespace {

thread_local std::string g_last_error;

}  // namespace

// ------------------------------------------------------------------ helpers

#define ARGENT_CK(ctx, call)                                                   \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      return set_error((ctx), ARGENT_E_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    }                                                                          \
  } while (0)

int set_error(const ArgentCtx* ctx, int code, const std::string& msg) {
  g_last_error = msg;
  if (ctx) const_cast<ArgentCtx*>(ctx)->err = msg;
  return code;
}

// ------------------------------------------------------------------ kernels

__global__ void k_trace_closest(DevPiece pc, const ArgentRay* __restrict__ rays, uint64_t n, ArgentHit* hits,
                                uint32_t* status) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const float4* rp = reinterpret_cast<const float4*>(rays + i);
    float4 a = __ldg(rp), b = __ldg(rp + 1);
    TraceHit h = trace_closest(pc, V3{a.x, a.y, a.z}, V3{b.x, b.y, b.z}, a.w, status);
    ArgentHit o;
    if (h.prim == ARGENT_NO_HIT_U) {
      o.t = 0.0f;
      o.u = 0.0f;
      o.v = 0.0f;
    } else {
      o.t = h.t;
      o.u = h.u;
      o.v = h.v;
    }
    o.prim = h.prim;
    reinterpret_cast<float4*>(hits)[i] = make_float4(o.t, o.u, o.v, __uint_as_float(o.prim));
  }
}

__global__ void k_trace_any(DevPiece pc, const ArgentRay* __restrict__ rays, uint64_t n, uint8_t* occ,
                            uint32_t* status) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const float4* rp = reinterpret_cast<const float4*>(rays + i);
    float4 a = __ldg(rp), b = __ldg(rp + 1);
    occ[i] = trace_any(pc, V3{a.x, a.y, a.z}, V3{b.x, b.y, b.z}, a.w, status) ? 1 : 0;
  }
}

// Rewrites every triangle record of a piece for a triangle test: (v0, e1,
// e2) with e = v - v0 rounded as the host builder rounds it (argent's
// Moller-Trumbore), or the three original vertices (v0, v1, v2) marked
// watertight.  The record's original index (v0.w) names its vertices.
__global__ void k_tri_records(float4* tris, const uint4* __restrict__ tri_idx, const float4* __restrict__ pos,
                              uint32_t n, int watertight) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t prim = __float_as_uint(tris[3 * (size_t)i].w);
    uint4 t = __ldg(tri_idx + prim);
    float4 a = __ldg(pos + t.x), b = __ldg(pos + t.y), c = __ldg(pos + t.z);
    tris[3 * (size_t)i] = make_float4(a.x, a.y, a.z, __uint_as_float(prim));
    if (watertight) {
      tris[3 * (size_t)i + 1] = make_float4(b.x, b.y, b.z, __uint_as_float(ARGENT_TRI_REC_WATERTIGHT));
      tris[3 * (size_t)i + 2] = make_float4(c.x, c.y, c.z, 0.0f);
    } else {
      tris[3 * (size_t)i + 1] = make_float4(__fsub_rn(b.x, a.x), __fsub_rn(b.y, a.y), __fsub_rn(b.z, a.z), 0.0f);
      tris[3 * (size_t)i + 2] = make_float4(__fsub_rn(c.x, a.x), __fsub_rn(c.y, a.y), __fsub_rn(c.z, a.z), 0.0f);
    }
  }
}

// ------------------------------------------------------------------ cavity ambient occlusion

// cavity.rs:96-135, one thread per (vertex, sample): the ray from the
// vertex nudged eps along its normal, direction from a cosine-weighted
// stratified hemisphere rotated by a vertex hash, tested for any hit within
// `distance` (the Occluder of scene.rs:40-44).  Consecutive threads are
// samples of one vertex, so a warp's rays share an origin.  glam's
// normalize_or_zero and any_orthonormal_pair (Duff et al. 2017, sign =
// signum(z)) are restated in glam's scalar operation order.
__global__ void __launch_bounds__(128) k_cavity_ao(DevPiece pc, const float* __restrict__ normals, uint32_t nv,
                                                   uint32_t n, float distance, float eps, uint32_t* counts,
                                                   uint32_t* status) {
  uint64_t total = (uint64_t)nv * n;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t v = (uint32_t)(i / n), k = (uint32_t)(i % n);
    float nx = normals[3 * (size_t)v], ny = normals[3 * (size_t)v + 1], nz = normals[3 * (size_t)v + 2];
    float rcp = __fdiv_rn(1.0f, __fsqrt_rn((nx * nx + ny * ny) + nz * nz));
    if (!(isfinite(rcp) && rcp > 0.0f)) continue;
    nx *= rcp;
    ny *= rcp;
    nz *= rcp;
    float sign = signbit(nz) ? -1.0f : 1.0f;
    float a = __fdiv_rn(-1.0f, sign + nz);
    float bb = nx * ny * a;
    float tx = 1.0f + sign * nx * nx * a, ty = sign * bb, tz = -sign * nx;
    float bx = bb, by = sign + ny * ny * a, bz = -ny;
    float4 p = __ldg(pc.pos + v);
    V3 o{p.x + nx * eps, p.y + ny * eps, p.z + nz * eps};
    uint32_t h = hash32(v ^ 0x5bd1e995u);
    float rot = (float)(h >> 8) * (1.0f / 16777216.0f);
    float jit = (float)(hash32(h) >> 8) * (1.0f / 16777216.0f);
    float u1 = fminf(__fdiv_rn((float)k + jit, (float)n), 0.999999f);
    float x = (float)k * 0.618034f + rot;
    float u2 = x - truncf(x);
    float r = __fsqrt_rn(u1);
    float phi = 6.28318530717958647692f * u2;
    float c = r * cosf(phi), sn = r * sinf(phi), w = __fsqrt_rn(1.0f - u1);
    V3 d{(tx * c + bx * sn) + nx * w, (ty * c + by * sn) + ny * w, (tz * c + bz * sn) + nz * w};
    if (trace_any(pc, o, d, distance, status)) atomicAdd(counts + v, 1u);
  }
}

__global__ void k_cavity_ao_finish(const uint32_t* counts, uint32_t nv, uint32_t n, float* out) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x)
    out[v] = __fdiv_rn((float)counts[v], (float)n);
}

// ------------------------------------------------------------------ context

int ctx_check_status(ArgentCtx* ctx) {
  uint32_t st = 0;
  ARGENT_CK(ctx, cudaMemcpyAsync(&st, ctx->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
  ARGENT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  if (st) {
    ARGENT_CK(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(uint32_t), ctx->stream));
    ARGENT_CK(ctx, cudaStreamSynchronize(ctx->stream));
    std::string m = "device status:";
    if (st & ARGENT_STATUS_STACK_OVERFLOW) m += " traversal stack overflow;";
    if (st & ARGENT_STATUS_QUEUE_OVERFLOW) m += " queue overflow;";
    if (st & ARGENT_STATUS_TIMEOUT) m += " bounded wait expired;";
    return set_error(ctx, (st & ARGENT_STATUS_TIMEOUT) ? ARGENT_E_TIMEOUT : ARGENT_E_OVERFLOW, m);
  }
  return ARGENT_OK;
}

int grid_for(const ArgentCtx* ctx, const void* kernel, int block, uint64_t n) {
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0);
  per_sm = std::max(per_sm, 1);
  uint64_t full = (n + block - 1) / block;
  uint64_t g = std::min<uint64_t>(full, (uint64_t)ctx->num_sms * per_sm);
  return (int)std::max<uint64_t>(g, 1);
}

// ------------------------------------------------------------------ kernel timing

static cudaEvent_t prof_event(ArgentCtx* ctx) {
  if (!ctx->prof.pool.empty()) {
    cudaEvent_t e = ctx->prof.pool.back();
    ctx->prof.pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Brackets one launch with events on its stream when profiling.
struct ProfScope {
  ArgentCtx* ctx;
  int kind;
  cudaStream_t s;
  cudaEvent_t a = nullptr;
  ProfScope(ArgentCtx* c, int k, cudaStream_t st = nullptr) : ctx(c), kind(k), s(st ? st : c->stream) {
    if (ctx->prof.on) {
      a = prof_event(ctx);
      cudaEventRecord(a, s);
    }
  }
  ~ProfScope() {
    if (a) {
      cudaEvent_t b = prof_event(ctx);
      cudaEventRecord(b, s);
      ctx->prof.ev[kind].push_back({a, b});
    }
  }
};

static void prof_collect(ArgentCtx* ctx) {
  cudaStreamSynchronize(ctx->stream);
  for (int k = 0; k < KC_COUNT; ++k) {
    for (auto& pr : ctx->prof.ev[k]) {
      float ms = 0.0f;
      if (cudaEventElapsedTime(&ms, pr.first, pr.second) == cudaSuccess) ctx->prof.ms[k] += ms;
      ctx->prof.n[k] += 1;
      ctx->prof.pool.push_back(pr.first);
      ctx->prof.pool.push_back(pr.second);
    }
    ctx->prof.ev[k].clear();
  }
}

extern "C" {

const char* argent_last_error(const ArgentCtx* ctx) {
  if (ctx) return ctx->err.c_str();
  return g_last_error.c_str();
}

int argent_ctx_create(int device, const ArgentLimits* limits, ArgentCtx** out) {
  if (!out) return set_error(nullptr, ARGENT_E_INVALID, "argent_ctx_create: out is NULL");
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0)
    return set_error(nullptr, ARGENT_E_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
  if (device < 0 || device >= count) return set_error(nullptr, ARGENT_E_INVALID, "device index out of range");
  ArgentCtx* ctx = new ArgentCtx();
  ctx->device = device;
  if (limits) ctx->limits = *limits;
  if (ctx->limits.wave_paths == 0) ctx->limits.wave_paths = 1ull << 24;
  if (ctx->limits.wave_paths > (1ull << 30) || ctx->limits.lanes > ARGENT_LANES) {
    delete ctx;
    return set_error(nullptr, ARGENT_E_INVALID, "wave_paths above 2^30 or more than 16 lanes");
  }
  ctx->lanes = ctx->limits.lanes ? (int)ctx->limits.lanes : 8;
  cudaError_t r = cudaSetDevice(device);
  if (r == cudaSuccess) r = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  for (int l = 0; l < ctx->lanes && r == cudaSuccess; ++l)
    r = cudaStreamCreateWithFlags(&ctx->lane_stream[l], cudaStreamNonBlocking);
  if (r == cudaSuccess) r = cudaStreamCreateWithFlags(&ctx->aux_stream, cudaStreamNonBlocking);
  if (r == cudaSuccess) r = cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming);
  if (r == cudaSuccess) r = cudaEventCreateWithFlags(&ctx->join_ev, cudaEventDisableTiming);
  for (int l = 0; l < ctx->lanes && r == cudaSuccess; ++l)
    r = cudaEventCreateWithFlags(&ctx->film_ev[l], cudaEventDisableTiming);
  if (r == cudaSuccess) r = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (r == cudaSuccess) r = cudaMalloc(&ctx->d_status, sizeof(uint32_t) * 4);
  if (r == cudaSuccess) r = cudaMemset(ctx->d_status, 0, sizeof(uint32_t) * 4);
  if (r != cudaSuccess) {
    std::string m = std::string("context setup failed: ") + cudaGetErrorString(r);
    argent_ctx_destroy(ctx);
    return set_error(nullptr, ARGENT_E_CUDA, m);
  }
  if (ctx->limits.memory_budget == 0) {
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    ctx->limits.memory_budget = (uint64_t)(fr / 4 * 3);
  }
  *out = ctx;
  return ARGENT_OK;
}

void argent_ctx_destroy(ArgentCtx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (int l = 0; l < ARGENT_LANES; ++l)
    if (ctx->lane_stream[l]) cudaStreamSynchronize(ctx->lane_stream[l]);
  if (ctx->aux_stream) cudaStreamSynchronize(ctx->aux_stream);
  prof_collect(ctx);
  for (cudaEvent_t e : ctx->prof.pool) cudaEventDestroy(e);
  for (int l = 0; l < ARGENT_LANES; ++l) ctx->wave[l].release();
  for (auto& b : ctx->blobs) cudaFree(b.dev);
  ctx->blobs.clear();
  if (ctx->d_status) cudaFree(ctx->d_status);
  if (ctx->resolve) cudaFree(ctx->resolve);
  if (ctx->d_jobs_buf) cudaFree(ctx->d_jobs_buf);
  for (auto& g : ctx->graph_cache) cudaGraphExecDestroy(g.exec);
  for (int l = 0; l < ARGENT_LANES; ++l)
    if (ctx->lane_stream[l]) cudaStreamDestroy(ctx->lane_stream[l]);
  if (ctx->aux_stream) cudaStreamDestroy(ctx->aux_stream);
  if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
  if (ctx->join_ev) cudaEventDestroy(ctx->join_ev);
  for (int l = 0; l < ARGENT_LANES; ++l)
    if (ctx->film_ev[l]) cudaEventDestroy(ctx->film_ev[l]);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

int argent_ctx_sync(ArgentCtx* ctx) {
  if (!ctx) return set_error(nullptr, ARGENT_E_INVALID, "ctx is NULL");
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  ARGENT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  for (int l = 0; l < ARGENT_LANES; ++l)
    if (ctx->lane_stream[l]) ARGENT_CK(ctx, cudaStreamSynchronize(ctx->lane_stream[l]));
  if (ctx->aux_stream) ARGENT_CK(ctx, cudaStreamSynchronize(ctx->aux_stream));
  ctx->overlapped_pending = false;
  return ctx_check_status(ctx);
}

void* argent_ctx_stream(ArgentCtx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

uint64_t argent_ctx_kernel_launches(const ArgentCtx* ctx) { return ctx ? ctx->launches : 0; }

// ------------------------------------------------------------------ piece

void argent_piece_destroy(ArgentPiece* p) {
  if (!p) return;
  cudaSetDevice(p->ctx->device);
  for (void* a : p->allocs) cudaFree(a);
  delete p;
}

int argent_piece_upload(ArgentCtx* ctx, const float* positions, uint32_t nv, const float* normals,
                        const uint32_t* tris, uint32_t nt, const uint16_t* tri_material, const float* cavity,
                        ArgentPiece** out) {
  if (!ctx || !out) return set_error(ctx, ARGENT_E_INVALID, "argent_piece_upload: NULL argument");
  *out = nullptr;
  if ((nv && !positions) || (nt && !tris)) return set_error(ctx, ARGENT_E_INVALID, "piece arrays are NULL");
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  argent::WideBvh bvh;
  try {
    bvh = argent::build_wide_bvh(positions, nv, tris, nt, 0);
  } catch (const std::exception& e) {
    return set_error(ctx, ARGENT_E_INVALID, std::string("BVH build: ") + e.what());
  }
  if ((uint64_t)bvh.depth * 7 + 1 > ARGENT_STACK_SIZE)
    return set_error(ctx, ARGENT_E_INVALID, "BVH too deep for the traversal stack");
  ArgentPiece* p = new ArgentPiece();
  p->ctx = ctx;
  p->nv = nv;
  p->nt = nt;
  p->depth = bvh.depth;
  for (int a = 0; a < 3; ++a) {
    p->lo[a] = bvh.lo[a];
    p->hi[a] = bvh.hi[a];
  }
  std::vector<float4> pos4(nv), nrm4;
  for (uint32_t i = 0; i < nv; ++i) pos4[i] = make_float4(positions[3 * i], positions[3 * i + 1], positions[3 * i + 2], 0);
  if (normals) {
    nrm4.resize(nv);
    for (uint32_t i = 0; i < nv; ++i) nrm4[i] = make_float4(normals[3 * i], normals[3 * i + 1], normals[3 * i + 2], 0);
  }
  std::vector<uint4> tidx(nt);
  for (uint32_t i = 0; i < nt; ++i)
    tidx[i] = make_uint4(tris[3 * i], tris[3 * i + 1], tris[3 * i + 2], tri_material ? tri_material[i] : 0u);
  p->max_material = 0;
  for (uint32_t i = 0; tri_material && i < nt; ++i) p->max_material = std::max<uint32_t>(p->max_material, tri_material[i]);
  auto up = [&](const void* src, size_t bytes, void** dst) -> cudaError_t {
    *dst = nullptr;
    if (bytes == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(dst, bytes);
    if (e != cudaSuccess) return e;
    p->allocs.push_back(*dst);
    p->bytes += bytes;
    return cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream);
  };
  void *dn = nullptr, *dt = nullptr, *dp = nullptr, *dnr = nullptr, *di = nullptr, *dc = nullptr;
  cudaError_t e = up(bvh.nodes.data(), bvh.nodes.size() * sizeof(argent::WideNode), &dn);
  if (e == cudaSuccess) e = up(bvh.tris.data(), bvh.tris.size() * sizeof(argent::TriRecord), &dt);
  if (e == cudaSuccess) e = up(pos4.data(), pos4.size() * sizeof(float4), &dp);
  if (e == cudaSuccess && normals) e = up(nrm4.data(), nrm4.size() * sizeof(float4), &dnr);
  if (e == cudaSuccess) e = up(tidx.data(), tidx.size() * sizeof(uint4), &di);
  if (e == cudaSuccess && cavity) e = up(cavity, (size_t)nv * sizeof(float), &dc);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    std::string m = std::string("piece upload: ") + cudaGetErrorString(e);
    argent_piece_destroy(p);
    return set_error(ctx, e == cudaErrorMemoryAllocation ? ARGENT_E_OOM : ARGENT_E_CUDA, m);
  }
  p->dev.nodes = (const uint4*)dn;
  p->dev.tris = (const float4*)dt;
  p->dev.pos = (const float4*)dp;
  p->dev.nrm = (const float4*)dnr;
  p->dev.tri_idx = (const uint4*)di;
  p->dev.cavity = (const float*)dc;
  p->dev.num_tris = nt;
  *out = p;
  return ARGENT_OK;
}

}  // extern "C"

namespace {

// Stream-ordered temporaries of one device build, freed together.
struct BuildTemps {
  cudaStream_t st;
  std::vector<void*> ptrs;
  cudaError_t err = cudaSuccess;
  template <class T>
  T* get(size_t count) {
    void* p = nullptr;
    if (err == cudaSuccess) err = cudaMallocAsync(&p, std::max<size_t>(count, 1) * sizeof(T), st);
    if (err == cudaSuccess) ptrs.push_back(p);
    return (T*)p;
  }
  ~BuildTemps() {
    for (void* p : ptrs) cudaFreeAsync(p, st);
  }
};

// Builds the 8-wide BVH of the piece's uploaded triangles on the device
// (device_build.cuh) and stores nodes, triangle records, depth and bounds
// in `p`.  `tidx` holds the piece's triangles (x, y, z = vertex indices).
std::string device_bvh(ArgentCtx* ctx, ArgentPiece* p, const float4* pos, const uint4* tidx, uint32_t nt) {
  cudaStream_t st = ctx->stream;
  const size_t n = nt, nb = 2 * n - 1;
  BuildTemps tmp{st};
  const uint32_t tpb = 256;
  const uint32_t nblk = (uint32_t)std::min<size_t>((n + tpb - 1) / tpb, (size_t)148 * 8);
  float* tlo = tmp.get<float>(3 * n);
  float* thi = tmp.get<float>(3 * n);
  float* cen = tmp.get<float>(3 * n);
  float* blo = tmp.get<float>(3 * (size_t)nblk);
  float* bhi = tmp.get<float>(3 * (size_t)nblk);
  uint64_t* k0 = tmp.get<uint64_t>(n);
  uint64_t* k1 = tmp.get<uint64_t>(n);
  uint32_t* v0 = tmp.get<uint32_t>(n);
  uint32_t* v1 = tmp.get<uint32_t>(n);
  db::Bin bn;
  bn.lo = tmp.get<float>(3 * nb);
  bn.hi = tmp.get<float>(3 * nb);
  bn.first = tmp.get<uint32_t>(nb);
  bn.last = tmp.get<uint32_t>(nb);
  bn.left = tmp.get<int32_t>(nb);
  bn.right = tmp.get<int32_t>(nb);
  bn.parent = tmp.get<int32_t>(nb);
  bn.flag = tmp.get<uint32_t>(nb);
  int2* qa = tmp.get<int2>(n);
  int2* qb = tmp.get<int2>(n);
  uint32_t* ctr = tmp.get<uint32_t>(4);  // n_out, node_count, tri_count, err
  const size_t max_nodes = std::max<size_t>(1, n - 1);
  uint4* nodes = tmp.get<uint4>(5 * max_nodes);
  if (tmp.err != cudaSuccess) return std::string("device BVH temporaries: ") + cudaGetErrorString(tmp.err);

  void* dt = nullptr;
  cudaError_t e = cudaMalloc(&dt, n * sizeof(argent::TriRecord));
  if (e != cudaSuccess) return std::string("device BVH triangles: ") + cudaGetErrorString(e);
  p->allocs.push_back(dt);
  p->bytes += n * sizeof(argent::TriRecord);

  db::k_tri_boxes<<<nblk, tpb, 0, st>>>(pos, tidx, nt, tlo, thi, cen, blo, bhi);
  const uint32_t grid = nblk;
  db::k_morton<<<grid, tpb, 0, st>>>(cen, nt, blo, bhi, nblk, k0, v0);
  size_t sort_bytes = 0;
  e = cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, k0, k1, v0, v1, (int)n, 0, 63, st);
  void* sort_tmp = tmp.get<uint8_t>(sort_bytes);
  if (e == cudaSuccess) e = tmp.err;
  if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(sort_tmp, sort_bytes, k0, k1, v0, v1, (int)n, 0, 63, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(bn.flag, 0, nb * sizeof(uint32_t), st);
  if (e != cudaSuccess) return std::string("device BVH sort: ") + cudaGetErrorString(e);
  ctx->launches += 4;
  if (n > 1) {
    db::k_radix_tree<<<grid, tpb, 0, st>>>(k1, nt, bn);
    ++ctx->launches;
  }
  db::k_boxes_up<<<grid, tpb, 0, st>>>(tlo, thi, v1, nt, bn);
  ++ctx->launches;

  const uint32_t init[4] = {0, 1, 0, 0};
  const int2 root = make_int2(0, 0);  // wide node 0 <- binary root (internal 0, or leaf 0 when n = 1)
  e = cudaMemcpyAsync(ctr, init, sizeof(init), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(qa, &root, sizeof(root), cudaMemcpyHostToDevice, st);
  uint32_t n_in = 1, depth = 0;
  db::Collapse c{};
  c.n_out = ctr;
  c.node_count = ctr + 1;
  c.tri_count = ctr + 2;
  c.err = ctr + 3;
  c.nodes = nodes;
  c.tris = (float4*)dt;
  c.pos = pos;
  c.tri = tidx;
  c.vals = v1;
  while (e == cudaSuccess && n_in > 0) {
    if (++depth > 64) return "device BVH collapse did not finish in 64 levels";
    c.in = qa;
    c.n_in = n_in;
    c.out = qb;
    e = cudaMemsetAsync(ctr, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) break;
    uint32_t g = (uint32_t)std::min<size_t>((n_in + 127) / 128, (size_t)148 * 16);
    db::k_collapse<<<g, 128, 0, st>>>(c, bn, nt);
    ++ctx->launches;
    e = cudaMemcpyAsync(&n_in, ctr, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    std::swap(qa, qb);
  }
  uint32_t got[4] = {0, 0, 0, 0};
  float box[6];
  if (e == cudaSuccess) e = cudaMemcpyAsync(got, ctr, sizeof(got), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(box, bn.lo, 3 * sizeof(float), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(box + 3, bn.hi, 3 * sizeof(float), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return std::string("device BVH build: ") + cudaGetErrorString(e);
  if (got[3] & DB_ERR_EXTENT) return "piece extent too large for the node quantisation";
  if (got[3]) return "device BVH quantisation failed";
  if (got[2] != nt || got[1] == 0 || got[1] > max_nodes)
    return "device BVH build lost triangles or nodes";
  if ((uint64_t)depth * 7 + 1 > ARGENT_STACK_SIZE) return "BVH too deep for the traversal stack";

  void* dn = nullptr;
  const size_t node_bytes = (size_t)got[1] * sizeof(argent::WideNode);
  e = cudaMalloc(&dn, node_bytes);
  if (e != cudaSuccess) return std::string("device BVH nodes: ") + cudaGetErrorString(e);
  p->allocs.push_back(dn);
  p->bytes += node_bytes;
  e = cudaMemcpyAsync(dn, nodes, node_bytes, cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return std::string("device BVH nodes: ") + cudaGetErrorString(e);
  p->dev.nodes = (const uint4*)dn;
  p->dev.tris = (const float4*)dt;
  p->depth = depth;
  for (int a = 0; a < 3; ++a) {
    p->lo[a] = box[a];
    p->hi[a] = box[3 + a];
  }
  return "";
}

}  // namespace

extern "C" {

int argent_piece_upload_device_bvh(ArgentCtx* ctx, const float* positions, uint32_t nv, const float* normals,
                                   const uint32_t* tris, uint32_t nt, const uint16_t* tri_material,
                                   const float* cavity, ArgentPiece** out) {
  if (!ctx || !out) return set_error(ctx, ARGENT_E_INVALID, "argent_piece_upload_device_bvh: NULL argument");
  *out = nullptr;
  if ((nv && !positions) || (nt && !tris)) return set_error(ctx, ARGENT_E_INVALID, "piece arrays are NULL");
  // An empty piece has nothing to build: the host path makes the same empty piece.
  if (nt == 0) return argent_piece_upload(ctx, positions, nv, normals, tris, nt, tri_material, cavity, out);
  if (nt >= (1u << 27)) return set_error(ctx, ARGENT_E_INVALID, "device BVH build takes fewer than 2^27 triangles");
  for (uint64_t i = 0; i < 3ull * nt; ++i)
    if (tris[i] >= nv) return set_error(ctx, ARGENT_E_INVALID, "triangle index out of range");
  for (uint64_t i = 0; i < 3ull * nv; ++i)
    if (!std::isfinite(positions[i])) return set_error(ctx, ARGENT_E_INVALID, "non-finite vertex position");
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  ArgentPiece* p = new ArgentPiece();
  p->ctx = ctx;
  p->nv = nv;
  p->nt = nt;
  std::vector<float4> pos4(nv), nrm4;
  for (uint32_t i = 0; i < nv; ++i) pos4[i] = make_float4(positions[3 * i], positions[3 * i + 1], positions[3 * i + 2], 0);
  if (normals) {
    nrm4.resize(nv);
    for (uint32_t i = 0; i < nv; ++i) nrm4[i] = make_float4(normals[3 * i], normals[3 * i + 1], normals[3 * i + 2], 0);
  }
  std::vector<uint4> tidx(nt);
  for (uint32_t i = 0; i < nt; ++i)
    tidx[i] = make_uint4(tris[3 * i], tris[3 * i + 1], tris[3 * i + 2], tri_material ? tri_material[i] : 0u);
  for (uint32_t i = 0; tri_material && i < nt; ++i) p->max_material = std::max<uint32_t>(p->max_material, tri_material[i]);
  auto up = [&](const void* src, size_t bytes, void** dst) -> cudaError_t {
    *dst = nullptr;
    if (bytes == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(dst, bytes);
    if (e != cudaSuccess) return e;
    p->allocs.push_back(*dst);
    p->bytes += bytes;
    return cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream);
  };
  void *dp = nullptr, *dnr = nullptr, *di = nullptr, *dc = nullptr;
  cudaError_t e = up(pos4.data(), pos4.size() * sizeof(float4), &dp);
  if (e == cudaSuccess && normals) e = up(nrm4.data(), nrm4.size() * sizeof(float4), &dnr);
  if (e == cudaSuccess) e = up(tidx.data(), tidx.size() * sizeof(uint4), &di);
  if (e == cudaSuccess && cavity) e = up(cavity, (size_t)nv * sizeof(float), &dc);
  if (e != cudaSuccess) {
    cudaStreamSynchronize(ctx->stream);
    std::string m = std::string("piece upload: ") + cudaGetErrorString(e);
    argent_piece_destroy(p);
    return set_error(ctx, e == cudaErrorMemoryAllocation ? ARGENT_E_OOM : ARGENT_E_CUDA, m);
  }
  std::string err = device_bvh(ctx, p, (const float4*)dp, (const uint4*)di, nt);
  cudaStreamSynchronize(ctx->stream);
  if (!err.empty()) {
    argent_piece_destroy(p);
    return set_error(ctx, ARGENT_E_INVALID, err);
  }
  p->dev.pos = (const float4*)dp;
  p->dev.nrm = (const float4*)dnr;
  p->dev.tri_idx = (const uint4*)di;
  p->dev.cavity = (const float*)dc;
  p->dev.num_tris = nt;
  *out = p;
  return ARGENT_OK;
}

int argent_piece_set_triangle_test(ArgentCtx* ctx, ArgentPiece* piece, int test) {
  if (!ctx || !piece) return set_error(ctx, ARGENT_E_INVALID, "argent_piece_set_triangle_test: NULL argument");
  if (piece->ctx != ctx) return set_error(ctx, ARGENT_E_INVALID, "piece belongs to another context");
  if (test != ARGENT_TRI_MOLLER_TRUMBORE && test != ARGENT_TRI_WATERTIGHT)
    return set_error(ctx, ARGENT_E_INVALID, "unknown triangle test");
  if (piece->nt == 0) return ARGENT_OK;
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  // Renders in flight read the records: rewrite them only once the
  // context's work is done.
  ARGENT_CK(ctx, cudaDeviceSynchronize());
  int grid = grid_for(ctx, (const void*)k_tri_records, 256, piece->nt);
  k_tri_records<<<grid, 256, 0, ctx->stream>>>(const_cast<float4*>(piece->dev.tris), piece->dev.tri_idx,
                                                piece->dev.pos, piece->nt, test == ARGENT_TRI_WATERTIGHT ? 1 : 0);
  ctx->launches++;
  ARGENT_CK(ctx, cudaGetLastError());
  ARGENT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  piece->tri_test = test;
  return ARGENT_OK;
}

int argent_piece_bounds(const ArgentPiece* p, float lo[3], float hi[3]) {
  if (!p || !lo || !hi) return set_error(nullptr, ARGENT_E_INVALID, "argent_piece_bounds: NULL argument");
  for (int a = 0; a < 3; ++a) {
    lo[a] = p->lo[a];
    hi[a] = p->hi[a];
  }
  return ARGENT_OK;
}

uint64_t argent_piece_device_bytes(const ArgentPiece* p) { return p ? p->bytes : 0; }

// ------------------------------------------------------------------ traversal entry points

int argent_trace_closest_device(ArgentCtx* ctx, ArgentPiece* piece, const ArgentRay* d_rays, uint64_t n,
                                ArgentHit* d_hits) {
  if (!ctx || !piece) return set_error(ctx, ARGENT_E_INVALID, "NULL argument");
  if (n == 0) return ARGENT_OK;
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  int block = 128;
  int grid = grid_for(ctx, (const void*)k_trace_closest, block, n);
  {
    ProfScope ps(ctx, KC_TRACE);
    k_trace_closest<<<grid, block, 0, ctx->stream>>>(piece->dev, d_rays, n, d_hits, ctx->d_status);
  }
  ctx->launches++;
  ARGENT_CK(ctx, cudaGetLastError());
  return ARGENT_OK;
}

int argent_trace_anyhit_device(ArgentCtx* ctx, ArgentPiece* piece, const ArgentRay* d_rays, uint64_t n,
                               uint8_t* d_occ) {
  if (!ctx || !piece) return set_error(ctx, ARGENT_E_INVALID, "NULL argument");
  if (n == 0) return ARGENT_OK;
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  int block = 128;
  int grid = grid_for(ctx, (const void*)k_trace_any, block, n);
  {
    ProfScope ps(ctx, KC_TRACE);
    k_trace_any<<<grid, block, 0, ctx->stream>>>(piece->dev, d_rays, n, d_occ, ctx->d_status);
  }
  ctx->launches++;
  ARGENT_CK(ctx, cudaGetLastError());
  return ARGENT_OK;
}

int argent_trace_closest(ArgentCtx* ctx, ArgentPiece* piece, const ArgentRay* rays, uint64_t n, ArgentHit* hits) {
  if (!ctx || !piece || (n && (!rays || !hits))) return set_error(ctx, ARGENT_E_INVALID, "NULL argument");
  if (n == 0) return ARGENT_OK;
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  void *dr = nullptr, *dh = nullptr;
  ARGENT_CK(ctx, cudaMallocAsync(&dr, n * sizeof(ArgentRay), ctx->stream));
  cudaError_t e = cudaMallocAsync(&dh, n * sizeof(ArgentHit), ctx->stream);
  if (e != cudaSuccess) {
    cudaFreeAsync(dr, ctx->stream);
    return set_error(ctx, ARGENT_E_OOM, "trace buffers");
  }
  e = cudaMemcpyAsync(dr, rays, n * sizeof(ArgentRay), cudaMemcpyHostToDevice, ctx->stream);
  int rc = ARGENT_OK;
  if (e == cudaSuccess) rc = argent_trace_closest_device(ctx, piece, (const ArgentRay*)dr, n, (ArgentHit*)dh);
  if (e == cudaSuccess && rc == ARGENT_OK)
    e = cudaMemcpyAsync(hits, dh, n * sizeof(ArgentHit), cudaMemcpyDeviceToHost, ctx->stream);
  cudaFreeAsync(dr, ctx->stream);
  cudaFreeAsync(dh, ctx->stream);
  cudaError_t s = cudaStreamSynchronize(ctx->stream);
  if (e == cudaSuccess) e = s;
  if (rc != ARGENT_OK) return rc;
  if (e != cudaSuccess) return set_error(ctx, ARGENT_E_CUDA, std::string("trace: ") + cudaGetErrorString(e));
  return ctx_check_status(ctx);
}

int argent_trace_anyhit(ArgentCtx* ctx, ArgentPiece* piece, const ArgentRay* rays, uint64_t n, uint8_t* occluded) {
  if (!ctx || !piece || (n && (!rays || !occluded))) return set_error(ctx, ARGENT_E_INVALID, "NULL argument");
  if (n == 0) return ARGENT_OK;
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  void *dr = nullptr, *dh = nullptr;
  ARGENT_CK(ctx, cudaMallocAsync(&dr, n * sizeof(ArgentRay), ctx->stream));
  cudaError_t e = cudaMallocAsync(&dh, n, ctx->stream);
  if (e != cudaSuccess) {
    cudaFreeAsync(dr, ctx->stream);
    return set_error(ctx, ARGENT_E_OOM, "trace buffers");
  }
  e = cudaMemcpyAsync(dr, rays, n * sizeof(ArgentRay), cudaMemcpyHostToDevice, ctx->stream);
  int rc = ARGENT_OK;
  if (e == cudaSuccess) rc = argent_trace_anyhit_device(ctx, piece, (const ArgentRay*)dr, n, (uint8_t*)dh);
  if (e == cudaSuccess && rc == ARGENT_OK) e = cudaMemcpyAsync(occluded, dh, n, cudaMemcpyDeviceToHost, ctx->stream);
  cudaFreeAsync(dr, ctx->stream);
  cudaFreeAsync(dh, ctx->stream);
  cudaError_t s = cudaStreamSynchronize(ctx->stream);
  if (e == cudaSuccess) e = s;
  if (rc != ARGENT_OK) return rc;
  if (e != cudaSuccess) return set_error(ctx, ARGENT_E_CUDA, std::string("trace: ") + cudaGetErrorString(e));
  return ctx_check_status(ctx);
}

}  // extern "C"

// ------------------------------------------------------------------ à-trous denoise

namespace {

// argent-post's atrous (denoise.rs:653-712) on device buffers: d_color
// (and the optional guides) in, d_out out; w*h pixels, 3 floats each.
int run_atrous(ArgentCtx* ctx, uint32_t w, uint32_t h, const float* d_color, const float* d_albedo,
               const float* d_normal, float* d_out) {
  size_t np = (size_t)w * h;
  cudaStream_t st = ctx->stream;
  float* base = nullptr;
  // sig, sig2, demod, g_albedo, g_normal (3 np each); l, l2, var, var2, vb, tmp, tmp2 (np each)
  size_t total = 15 * np + 7 * np;
  ARGENT_CK(ctx, cudaMallocAsync((void**)&base, total * sizeof(float), st));
  float *sig = base, *sig2 = sig + 3 * np, *demod = sig2 + 3 * np, *ga = demod + 3 * np, *gn = ga + 3 * np;
  float *l = gn + 3 * np, *l2 = l + np, *var = l2 + np, *var2 = var + np, *vb = var2 + np, *tmp = vb + np,
        *tmp2 = tmp + np;
  int grid = (int)std::min<size_t>((np + 255) / 256, (size_t)ctx->num_sms * 8);
  grid = std::max(grid, 1);
  auto blur = [&](const float* src, float* dst, std::initializer_list<float> k) {
    dn::Taps t{};
    t.n = 0;
    for (float v : k) t.k[t.n++] = v;
    dn::k_dn_blur<<<grid, 256, 0, st>>>(src, tmp2, w, h, t, 0);
    dn::k_dn_blur<<<grid, 256, 0, st>>>(tmp2, dst, w, h, t, 1);
    ctx->launches += 2;
  };
  dn::k_dn_prep<<<grid, 256, 0, st>>>(d_color, d_albedo, d_normal, (uint32_t)np, sig, l, demod, ga, gn);
  ctx->launches++;
  // noise_variance (denoise.rs:582-586)
  blur(l, tmp, {1.0f, 1.0f, 1.0f});
  dn::k_dn_resid<<<grid, 256, 0, st>>>(l, tmp, (uint32_t)np, vb);
  ctx->launches++;
  blur(vb, var, {1.0f, 1.0f, 1.0f, 1.0f, 1.0f});
  for (int pass = 0; pass < DN_PASSES; ++pass) {
    blur(var, vb, {0.25f, 0.5f, 0.25f});
    dn::k_dn_atrous<<<grid, 256, 0, st>>>(sig, l, var, vb, d_albedo ? ga : nullptr, d_normal ? gn : nullptr, w, h,
                                          1 << pass, sig2, var2, l2);
    ctx->launches++;
    std::swap(sig, sig2);
    std::swap(var, var2);
    std::swap(l, l2);
  }
  if (d_albedo) {
    dn::k_dn_remod<<<grid, 256, 0, st>>>(sig, demod, (uint32_t)np);
    ctx->launches++;
  }
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_out, sig, 3 * np * sizeof(float), cudaMemcpyDeviceToDevice, st);
  cudaFreeAsync(base, st);
  if (e != cudaSuccess) return set_error(ctx, ARGENT_E_CUDA, std::string("denoise: ") + cudaGetErrorString(e));
  return ARGENT_OK;
}

}  // namespace

extern "C" {

int argent_denoise_atrous(ArgentCtx* ctx, uint32_t width, uint32_t height, const float* color, const float* albedo,
                          const float* normal, float* out) {
  if (!ctx || (width && height && (!color || !out))) return set_error(ctx, ARGENT_E_INVALID, "NULL argument");
  if (normal && !albedo) normal = nullptr;  // a lone normal is ignored, as with OIDN (denoise.rs:16-17)
  size_t np = (size_t)width * height;
  if (np == 0) return ARGENT_OK;
  if (np > (1ull << 31)) return set_error(ctx, ARGENT_E_INVALID, "image too large");
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  float* d = nullptr;
  ARGENT_CK(ctx, cudaMallocAsync((void**)&d, 12 * np * sizeof(float), ctx->stream));
  float *dc = d, *da = albedo ? d + 3 * np : nullptr, *dn_ = normal ? d + 6 * np : nullptr, *dout = d + 9 * np;
  cudaError_t e = cudaMemcpyAsync(dc, color, 3 * np * sizeof(float), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess && da) e = cudaMemcpyAsync(da, albedo, 3 * np * sizeof(float), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess && dn_) e = cudaMemcpyAsync(dn_, normal, 3 * np * sizeof(float), cudaMemcpyHostToDevice, ctx->stream);
  int rc = e == cudaSuccess ? run_atrous(ctx, width, height, dc, da, dn_, dout) : ARGENT_E_CUDA;
  if (rc == ARGENT_OK) e = cudaMemcpyAsync(out, dout, 3 * np * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
  cudaFreeAsync(d, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (rc != ARGENT_OK) return rc;
  if (e != cudaSuccess) return set_error(ctx, ARGENT_E_CUDA, std::string("denoise: ") + cudaGetErrorString(e));
  return ctx_check_status(ctx);
}

}  // extern "C"

// ------------------------------------------------------------------ develop

namespace {

// Uploads the grade's tables and develops d_rgb (w*h camera RGB on the
// device) into d_out (w*h*3 bytes on the device).
int run_develop(ArgentCtx* ctx, uint32_t w, uint32_t h, const float* d_rgb, const ArgentGrade* g, uint8_t* d_out) {
  if (g->tonemap < ARGENT_TM_AGX || g->tonemap > ARGENT_TM_CLAMP || g->look < ARGENT_AGX_BASE ||
      g->look > ARGENT_AGX_GOLDEN)
    return set_error(ctx, ARGENT_E_INVALID, "unknown tone map or AgX look");
  argent::DevelopTables t = argent::develop_tables(g->exposure_ev, g->tonemap, g->look, g->saturation);
  size_t nc = t.curves.size(), ne = t.enc.size();
  float* d_tab = nullptr;
  ARGENT_CK(ctx, cudaMallocAsync((void**)&d_tab, (nc + ne) * sizeof(float), ctx->stream));
  cudaError_t e = cudaSuccess;
  if (nc) e = cudaMemcpyAsync(d_tab, t.curves.data(), nc * sizeof(float), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_tab + nc, t.enc.data(), ne * sizeof(float), cudaMemcpyHostToDevice, ctx->stream);
  dv::DevTables dt;
  dt.k = t.k;
  dt.op = t.op;
  dt.sat = t.sat;
  dt.pick0 = t.pick[0];
  dt.pick1 = t.pick[1];
  dt.pick2 = t.pick[2];
  dt.curves = d_tab;
  dt.curve_base = t.curve_base;
  dt.curve_len = t.curve_len;
  dt.enc = d_tab + nc;
  dt.enc_lo = t.enc_lo;
  dt.enc_scale = t.enc_scale;
  dt.enc_last = t.enc_last;
  size_t np = (size_t)w * h;
  int grid = (int)std::min<size_t>((np + 255) / 256, (size_t)ctx->num_sms * 8);
  if (e == cudaSuccess) {
    dv::k_develop<<<std::max(grid, 1), 256, 0, ctx->stream>>>(d_rgb, (uint32_t)np, dt, d_out);
    ctx->launches++;
    e = cudaGetLastError();
  }
  cudaFreeAsync(d_tab, ctx->stream);
  if (e != cudaSuccess) return set_error(ctx, ARGENT_E_CUDA, std::string("develop: ") + cudaGetErrorString(e));
  return ARGENT_OK;
}

}  // namespace

extern "C" {

int argent_develop(ArgentCtx* ctx, uint32_t width, uint32_t height, const float* rgb, const ArgentGrade* grade,
                   uint8_t* out) {
  if (!ctx || !grade || (width && height && (!rgb || !out))) return set_error(ctx, ARGENT_E_INVALID, "NULL argument");
  size_t np = (size_t)width * height;
  if (np == 0) return ARGENT_OK;
  if (np > (1ull << 31)) return set_error(ctx, ARGENT_E_INVALID, "image too large");
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  float* d_rgb = nullptr;
  uint8_t* d_out = nullptr;
  ARGENT_CK(ctx, cudaMallocAsync((void**)&d_rgb, 3 * np * sizeof(float), ctx->stream));
  ARGENT_CK(ctx, cudaMallocAsync((void**)&d_out, 3 * np, ctx->stream));
  cudaError_t e = cudaMemcpyAsync(d_rgb, rgb, 3 * np * sizeof(float), cudaMemcpyHostToDevice, ctx->stream);
  int rc = e == cudaSuccess ? run_develop(ctx, width, height, d_rgb, grade, d_out) : ARGENT_E_CUDA;
  if (rc == ARGENT_OK) e = cudaMemcpyAsync(out, d_out, 3 * np, cudaMemcpyDeviceToHost, ctx->stream);
  cudaFreeAsync(d_rgb, ctx->stream);
  cudaFreeAsync(d_out, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (rc != ARGENT_OK) return rc;
  if (e != cudaSuccess) return set_error(ctx, ARGENT_E_CUDA, std::string("develop: ") + cudaGetErrorString(e));
  return ctx_check_status(ctx);
}

}  // extern "C"

// ------------------------------------------------------------------ cavity mask

extern "C" {

int argent_mesh_smooth_normals(const float* positions, uint32_t nv, const uint32_t* tris, uint32_t nt, float* out) {
  if ((nv && (!positions || !out)) || (nt && !tris)) return set_error(nullptr, ARGENT_E_INVALID, "NULL argument");
  for (uint64_t i = 0; i < 3ull * nt; ++i)
    if (tris[i] >= nv) return set_error(nullptr, ARGENT_E_INVALID, "triangle index out of range");
  argent::smooth_vertex_normals(positions, nv, tris, nt, out);
  return ARGENT_OK;
}

int argent_mesh_concavity(const float* positions, uint32_t nv, const float* normals, const uint32_t* tris, uint32_t nt,
                          float radius, float* out) {
  if ((nv && (!positions || !normals || !out)) || (nt && !tris))
    return set_error(nullptr, ARGENT_E_INVALID, "NULL argument");
  for (uint64_t i = 0; i < 3ull * nt; ++i)
    if (tris[i] >= nv) return set_error(nullptr, ARGENT_E_INVALID, "triangle index out of range");
  argent::concavity(positions, nv, tris, nt, normals, radius, out);
  return ARGENT_OK;
}

int argent_mesh_smooth(const float* positions, uint32_t nv, const uint32_t* tris, uint32_t nt, float* values,
                       uint32_t iterations, float lambda) {
  if ((nv && (!positions || !values)) || (nt && !tris)) return set_error(nullptr, ARGENT_E_INVALID, "NULL argument");
  for (uint64_t i = 0; i < 3ull * nt; ++i)
    if (tris[i] >= nv) return set_error(nullptr, ARGENT_E_INVALID, "triangle index out of range");
  argent::smooth_values(positions, nv, tris, nt, values, iterations, lambda);
  return ARGENT_OK;
}

int argent_piece_ambient_occlusion(ArgentCtx* ctx, ArgentPiece* piece, const float* positions, const float* normals,
                                   uint32_t nv, uint32_t samples, float distance, float* ao) {
  if (!ctx || !piece || (nv && (!positions || !normals || !ao))) return set_error(ctx, ARGENT_E_INVALID, "NULL argument");
  if (nv != piece->nv) return set_error(ctx, ARGENT_E_INVALID, "vertex count differs from the uploaded piece");
  if (nv == 0) return ARGENT_OK;
  if (piece->nt == 0 || samples == 0 || !(distance > 0.0f)) {
    std::fill(ao, ao + nv, 0.0f);
    return ARGENT_OK;
  }
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  // cavity.rs:87-90: eps = max(2e-4 * |hi - lo|, 1e-3) over the vertices.
  float lo[3] = {positions[0], positions[1], positions[2]}, hi[3] = {positions[0], positions[1], positions[2]};
  for (uint32_t v = 1; v < nv; ++v)
    for (int k = 0; k < 3; ++k) {
      float x = positions[3 * (size_t)v + k];
      lo[k] = x < lo[k] ? x : lo[k];
      hi[k] = x > hi[k] ? x : hi[k];
    }
  float ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
  float diag = std::sqrt((ex * ex + ey * ey) + ez * ez);
  float eps = std::max(2e-4f * diag, 1e-3f);
  float* d_n = nullptr;
  uint32_t* d_cnt = nullptr;
  float* d_ao = nullptr;
  ARGENT_CK(ctx, cudaMallocAsync((void**)&d_n, 3ull * nv * sizeof(float), ctx->stream));
  ARGENT_CK(ctx, cudaMallocAsync((void**)&d_cnt, (size_t)nv * sizeof(uint32_t), ctx->stream));
  ARGENT_CK(ctx, cudaMallocAsync((void**)&d_ao, (size_t)nv * sizeof(float), ctx->stream));
  ARGENT_CK(ctx, cudaMemcpyAsync(d_n, normals, 3ull * nv * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  ARGENT_CK(ctx, cudaMemsetAsync(d_cnt, 0, (size_t)nv * sizeof(uint32_t), ctx->stream));
  uint64_t total = (uint64_t)nv * samples;
  int grid = grid_for(ctx, (const void*)k_cavity_ao, 128, total);
  {
    ProfScope ps(ctx, KC_TRACE);
    k_cavity_ao<<<grid, 128, 0, ctx->stream>>>(piece->dev, d_n, nv, samples, distance, eps, d_cnt, ctx->d_status);
  }
  int g2 = (int)std::min<uint64_t>((nv + 255) / 256, (uint64_t)ctx->num_sms * 8);
  k_cavity_ao_finish<<<std::max(g2, 1), 256, 0, ctx->stream>>>(d_cnt, nv, samples, d_ao);
  ctx->launches += 2;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(ao, d_ao, (size_t)nv * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
  cudaFreeAsync(d_n, ctx->stream);
  cudaFreeAsync(d_cnt, ctx->stream);
  cudaFreeAsync(d_ao, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return set_error(ctx, ARGENT_E_CUDA, std::string("ambient occlusion: ") + cudaGetErrorString(e));
  return ctx_check_status(ctx);
}

int argent_piece_patina_mask(ArgentCtx* ctx, ArgentPiece* piece, const float* positions, const float* normals,
                             uint32_t nv, const uint32_t* tris, uint32_t nt, const ArgentPatinaSettings* settings,
                             float* mask) {
  if (!ctx || !piece || !settings || (nv && (!positions || !mask)) || (nt && !tris))
    return set_error(ctx, ARGENT_E_INVALID, "NULL argument");
  if (nv != piece->nv || nt != piece->nt)
    return set_error(ctx, ARGENT_E_INVALID, "mesh differs from the uploaded piece");
  for (uint64_t i = 0; i < 3ull * nt; ++i)
    if (tris[i] >= nv) return set_error(ctx, ARGENT_E_INVALID, "triangle index out of range");
  if (nv == 0) return ARGENT_OK;
  if (nt == 0) {
    std::fill(mask, mask + nv, 0.0f);
    return ARGENT_OK;
  }
  std::vector<float> nrm(3 * (size_t)nv);
  if (normals)
    std::memcpy(nrm.data(), normals, nrm.size() * sizeof(float));
  else
    argent::smooth_vertex_normals(positions, nv, tris, nt, nrm.data());
  std::vector<float> ao(nv, 0.0f), cav(nv, 0.0f);
  if (settings->ao_samples > 0 && settings->ao_distance > 0.0f) {
    int rc = argent_piece_ambient_occlusion(ctx, piece, positions, nrm.data(), nv, settings->ao_samples,
                                            settings->ao_distance, ao.data());
    if (rc != ARGENT_OK) return rc;
  }
  float w = std::min(std::max(settings->concavity_weight, 0.0f), 1.0f);
  if (w > 0.0f && settings->curvature_radius > 0.0f)
    argent::concavity(positions, nv, tris, nt, nrm.data(), settings->curvature_radius, cav.data());
  argent::patina_blend(positions, nv, tris, nt, ao.data(), cav.data(), settings->concavity_weight,
                       settings->smooth_iterations, mask);
  return ARGENT_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ device tables

static int ensure_tables(ArgentCtx* ctx) {
  if (ctx->tables_ready) return ARGENT_OK;
  uint32_t dirs[4][32];
  argent::sobol_directions(dirs);
  static float energy[32 * 32];
  static std::once_flag once;
  std::call_once(once, [] { argent::ggx_energy_table(energy); });
  ARGENT_CK(ctx, cudaMemcpyToSymbol(dev::d_sobol_dirs, dirs, sizeof(dirs)));
  static uint32_t bytes[4][4][256];
  for (int d = 0; d < 4; ++d)
    for (int k = 0; k < 4; ++k)
      for (int v = 0; v < 256; ++v) {
        uint32_t x = 0;
        for (int j = 0; j < 8; ++j)
          if ((v >> j) & 1) x ^= dirs[d][8 * k + j];
        bytes[d][k][v] = x;
      }
  ARGENT_CK(ctx, cudaMemcpyToSymbol(dev::d_sobol_bytes, bytes, sizeof(bytes)));
  ARGENT_CK(ctx, cudaMemcpyToSymbol(dev::d_energy_table, energy, sizeof(energy)));
  ARGENT_CK(ctx, cudaMemcpyToSymbol(dev::d_cmf, ARGENT_CMF_1931_2DEG, sizeof(float) * 471 * 3));
  ctx->tables_ready = true;
  return ARGENT_OK;
}

// Streams and events for lanes 0 .. n-1 (created once, kept).
static int ensure_lane_streams(ArgentCtx* ctx, int n) {
  for (int l = 0; l < n; ++l)
    if (!ctx->lane_stream[l]) ARGENT_CK(ctx, cudaStreamCreateWithFlags(&ctx->lane_stream[l], cudaStreamNonBlocking));
  for (int l = 0; l < n; ++l)
    if (!ctx->film_ev[l]) ARGENT_CK(ctx, cudaEventCreateWithFlags(&ctx->film_ev[l], cudaEventDisableTiming));
  return ARGENT_OK;
}

// Grows lane `lane`'s path state to at least `cap` slots (never shrinks, so
// small renders after large ones reuse the buffers).
static int ensure_wave(ArgentCtx* ctx, int lane, uint64_t cap) {
  WaveBuffers& w = ctx->wave[lane];
  if (w.cap >= cap) return ARGENT_OK;
  // Waves of earlier batches may still run on this lane.
  if (w.cap > 0) ARGENT_CK(ctx, cudaStreamSynchronize(ctx->lane_stream[lane]));
  w.release();
  auto alloc = [&](void** p, size_t bytes) -> bool {
    if (cudaMalloc(p, bytes) != cudaSuccess) return false;
    w.allocs.push_back(*p);
    w.bytes += bytes;
    return true;
  };
  bool ok = true;
  float4** f4[] = {&w.o, &w.d, &w.beta, &w.L, &w.lambda, &w.pdf, &w.hit, &w.albedo, &w.normal, &w.sh_o, &w.sh_d, &w.sh_c};
  for (float4** p : f4) ok = ok && alloc((void**)p, cap * sizeof(float4));
  ok = ok && alloc((void**)&w.meta, cap * sizeof(uint4));
  ok = ok && alloc((void**)&w.rng, cap * sizeof(unsigned long long));
  ok = ok && alloc((void**)&w.q0, cap * sizeof(uint32_t));
  ok = ok && alloc((void**)&w.q1, cap * sizeof(uint32_t));
  ok = ok && alloc((void**)&w.qc, (size_t)NUM_CLS * cap * sizeof(uint32_t));
  ok = ok && alloc((void**)&w.counters, CNT_TOTAL * sizeof(uint32_t));
  if (!ok) {
    w.release();
    return set_error(ctx, ARGENT_E_OOM, "wave buffers: out of device memory");
  }
  w.cap = cap;
  return ARGENT_OK;
}

// Grows lane `lane`'s ray-sharing buffers to at least `cap` slots.
static int ensure_share(ArgentCtx* ctx, int lane, uint64_t cap) {
  WaveBuffers& w = ctx->wave[lane];
  if (w.share_cap >= cap) return ARGENT_OK;
  if (w.share_cap > 0) ARGENT_CK(ctx, cudaStreamSynchronize(ctx->lane_stream[lane]));
  w.release_share();
  auto alloc = [&](void** p, size_t bytes) -> bool {
    if (cudaMalloc(p, bytes) != cudaSuccess) return false;
    w.share_allocs.push_back(*p);
    w.share_bytes += bytes;
    w.bytes += bytes;
    return true;
  };
  bool ok = alloc((void**)&w.lead, cap * sizeof(uint32_t)) &&
            alloc((void**)&w.shrec, cap * sizeof(uint2)) && alloc((void**)&w.vis, cap * sizeof(uint8_t)) &&
            alloc((void**)&w.qt, cap * sizeof(uint32_t)) && alloc((void**)&w.qx, cap * sizeof(uint32_t)) &&
            alloc((void**)&w.qst, cap * sizeof(uint32_t)) && alloc((void**)&w.qsx, cap * sizeof(uint32_t)) &&
            alloc((void**)&w.qsc, cap * sizeof(uint32_t));
  if (!ok) {
    w.release_share();
    return set_error(ctx, ARGENT_E_OOM, "ray-sharing buffers: out of device memory");
  }
  w.share_cap = cap;
  return ARGENT_OK;
}

// ------------------------------------------------------------------ wave driver

namespace {

// True when two scenes give every ray the same closest hit and the same
// visibility: the same piece (its BVH and triangle records), the same
// turntable rotation, the same panels (as k_intersect tests them) and the
// same floor plane.  Materials, lights' emission and the environment may
// differ.
bool same_geometry(const ArgentScene* a, const ArgentScene* b) {
  if (a == b) return true;
  const dev::DevScene &x = a->host, &y = b->host;
  auto bits = [](float f) {
    uint32_t u;
    std::memcpy(&u, &f, sizeof(u));
    return u;
  };
  if (a->piece != b->piece || x.has_turn != y.has_turn) return false;
  if (x.has_turn && (bits(x.to_obj_s) != bits(y.to_obj_s) || bits(x.to_obj_c) != bits(y.to_obj_c))) return false;
  if (x.num_panels != y.num_panels || x.floor_enabled != y.floor_enabled) return false;
  if (x.floor_enabled && bits(x.floor_y) != bits(y.floor_y)) return false;
  for (int p = 0; p < x.num_panels; ++p) {
    const dev::DevPanel &u = x.panels[p], &v = y.panels[p];
    if (std::memcmp(u.c, v.c, sizeof(u.c)) || std::memcmp(u.hu, v.hu, sizeof(u.hu)) ||
        std::memcmp(u.hv, v.hv, sizeof(u.hv)) || std::memcmp(u.n, v.n, sizeof(u.n)) ||
        bits(u.hu_l2) != bits(v.hu_l2) || bits(u.hv_l2) != bits(v.hv_l2) || u.camera_visible != v.camera_visible)
      return false;
  }
  return true;
}

// True when the traversal kernels may take scene `b`'s paths as `a`'s: the
// same geometry and the same shading class for every material slot and the
// floor (what k_intersect reads from a wave's one scene).
bool same_traversal(const ArgentScene* a, const ArgentScene* b) {
  return a == b || (same_geometry(a, b) && a->host.floor_class == b->host.floor_class &&
                    std::memcmp(a->host.mat_class, b->host.mat_class, sizeof(a->host.mat_class)) == 0);
}

// Sets `f`'s ray-sharing masks against its group's leader `l` (scenes ls,
// fs): the material slots with byte-equal records and shading classes, and
// whether the rest of what shading reads is equal (the scene descriptor but
// for its materials, their classes and the film's camera matrix; the path
// settings).  Environment tables and emission spectra of equal content are
// one blob, so their pointers compare equal.  The descriptors are zeroed
// before they are filled, so their padding compares equal too; a mismatch
// could only turn sharing off.
void share_masks(const dev::DevJob& l, const ArgentScene* ls, const ArgentScene* fs, dev::DevJob* f) {
  std::memset(f->share_mat, 0, sizeof(f->share_mat));
  f->share_rest = 0;
  dev::DevScene a = ls->host, b = fs->host;
  for (dev::DevScene* x : {&a, &b}) {
    x->mats = nullptr;
    x->num_mats = 0;
    std::memset(x->mat_class, 0, sizeof(x->mat_class));
    x->floor_class = 0;
    x->class_mask = 0;
    std::memset(x->cam_m, 0, sizeof(x->cam_m));
  }
  const bool rest = std::memcmp(&a, &b, sizeof(a)) == 0 && l.max_depth == f->max_depth &&
                    l.rr_depth == f->rr_depth && std::memcmp(&l.clamp_indirect, &f->clamp_indirect, 4) == 0;
  if (!rest) return;
  f->share_rest = 1;
  const size_t n = std::min(ls->mats_host.size(), fs->mats_host.size());
  for (size_t i = 0; i < n && i < 256; ++i)
    if (ls->host.mat_class[i] == fs->host.mat_class[i] &&
        std::memcmp(&ls->mats_host[i], &fs->mats_host[i], sizeof(ArgentMaterial)) == 0)
      f->share_mat[i / 32] |= 1u << (i % 32);
}

// Groups of jobs that trace the same rays: the same film size, samples,
// seed and camera over the same geometry.  With sharing off, or for a job
// with no partner, a group is the job alone.  Groups are listed in the order
// of their first jobs, at most 16 jobs each.
std::vector<std::vector<uint32_t>> plan_groups(bool share, const std::vector<dev::DevJob>& jobs,
                                               const std::vector<uint32_t>& counts,
                                               const std::vector<const ArgentScene*>& scenes) {
  std::vector<std::vector<uint32_t>> groups;
  std::vector<bool> taken(jobs.size(), false);
  for (uint32_t j = 0; j < jobs.size(); ++j) {
    if (taken[j]) continue;
    taken[j] = true;
    groups.push_back({j});
    if (!share) continue;
    const dev::DevJob& a = jobs[j];
    for (uint32_t i = j + 1; i < jobs.size() && groups.back().size() < 16; ++i) {
      const dev::DevJob& b = jobs[i];
      if (taken[i] || b.w != a.w || b.h != a.h || b.first != a.first || b.seed_h != a.seed_h ||
          counts[i] != counts[j] || std::memcmp(&a.cam, &b.cam, sizeof(a.cam)) != 0 ||
          !same_geometry(scenes[j], scenes[i]))
        continue;
      taken[i] = true;
      groups.back().push_back(i);
    }
  }
  return groups;
}

// Splits every group of jobs into (pixel range, sample range) chunks of at
// most `cap` paths and packs them, in order, into waves.  A group of k jobs
// takes k segments with the same pixels and samples per chunk, side by side,
// the first leading the others.
std::vector<dev::WaveDesc> plan_waves(const std::vector<dev::DevJob>& jobs, const std::vector<uint32_t>& counts,
                                      const std::vector<std::vector<uint32_t>>& groups, uint64_t cap,
                                      std::vector<uint32_t>* wave_depth) {
  std::vector<dev::WaveDesc> waves;
  dev::WaveDesc cur{};
  uint32_t cur_depth = 0;
  auto flush = [&]() {
    if (cur.num_segments) {
      waves.push_back(cur);
      wave_depth->push_back(cur_depth);
    }
    cur = dev::WaveDesc{};
    cur_depth = 0;
  };
  // k_film adds each segment's sums to its pixels without atomics, so a wave
  // never holds two segments over the same pixels of one film: another run
  // of the same render's pixels (a group's runs are shorter than a wave), or
  // a later batch item rendering into the same film.
  auto clashes = [&](uint32_t job, uint32_t p0, uint32_t pn) {
    for (uint32_t i = 0; i < cur.num_segments; ++i) {
      const dev::DevSegment& q = cur.seg[i];
      if (jobs[q.job].film_xyz == jobs[job].film_xyz && q.p0 < p0 + pn && p0 < q.p0 + q.pn) return true;
    }
    return false;
  };
  for (const std::vector<uint32_t>& g : groups) {
    const uint32_t j0 = g[0];
    const uint64_t k = g.size();
    uint32_t P = jobs[j0].w * jobs[j0].h;
    uint32_t count = counts[j0];
    if (P == 0 || count == 0) continue;
    uint32_t depth = 0;
    for (uint32_t j : g) depth = std::max(depth, jobs[j].max_depth);
    // A group takes the samples per pixel and wave that one of its renders
    // would take alone in an empty wave (sn1), on fewer pixels per wave: the
    // film then sums every pixel's samples in the same runs as the render
    // alone, so its values are the same bit for bit.
    const uint64_t pn1 = std::min<uint64_t>(P, cap);
    const uint64_t sn1 = k > 1 ? std::max<uint64_t>(1, std::min<uint64_t>(count, cap / pn1)) : count;
    uint32_t pn_max = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(P, cap / (k * (k > 1 ? sn1 : 1))));
    for (uint32_t p0 = 0; p0 < P; p0 += pn_max) {
      uint32_t pn = std::min(pn_max, P - p0);
      uint32_t s0 = 0;
      while (s0 < count) {
        uint64_t room = cap - cur.num_slots;
        uint64_t want = k > 1 ? std::min<uint64_t>(count - s0, sn1) : 1;
        bool clash = false;
        for (uint32_t j : g) clash = clash || clashes(j, p0, pn);
        if (room < k * pn * want || cur.num_segments + k > ARGENT_MAX_SEGMENTS || clash) {
          flush();
          room = cap;
        }
        uint32_t sn = (uint32_t)std::min<uint64_t>(count - s0, room / (k * pn));
        if (k > 1) sn = (uint32_t)std::min<uint64_t>(sn, sn1);
        const uint32_t lead = cur.num_slots;
        for (uint64_t m = 0; m < k; ++m) {
          dev::DevSegment& sg = cur.seg[cur.num_segments++];
          sg.slot_begin = cur.num_slots;
          sg.job = g[m];
          sg.p0 = p0;
          sg.pn = pn;
          sg.s0 = s0;
          sg.sn = sn;
          sg.lead = m == 0 ? ~0u : lead;
          cur.num_slots += pn * sn;
        }
        cur_depth = std::max(cur_depth, depth);
        s0 += sn;
      }
    }
  }
  flush();
  return waves;
}

}  // namespace

static void fill_args(dev::WaveArgs& a, const WaveBuffers& wb) {
  a.o = wb.o;
  a.d = wb.d;
  a.beta = wb.beta;
  a.L = wb.L;
  a.lambda = wb.lambda;
  a.pdf = wb.pdf;
  a.hit = wb.hit;
  a.albedo = wb.albedo;
  a.normal = wb.normal;
  a.sh_o = wb.sh_o;
  a.sh_d = wb.sh_d;
  a.sh_c = wb.sh_c;
  a.meta = wb.meta;
  a.rng = wb.rng;
  a.counters = wb.counters;
  a.qc = wb.qc;
  a.cap = (uint32_t)wb.cap;
}

// Persistent grids of class CLS's two shading kernels (without and with the
// env-map code) for queues of up to `cap` paths.
template <int CLS>
static void shade_grids(const ArgentCtx* ctx, uint64_t cap, int grid[2]) {
  grid[0] = grid_for(ctx, (const void*)dev::k_shade<CLS, false>, 128, cap);
  grid[1] = grid_for(ctx, (const void*)dev::k_shade<CLS, true>, 128, cap);
}

// One shading launch of class CLS; `map` tells whether any scene of the wave
// has an env map.
template <int CLS>
static void launch_shade(bool map, const int grid[2], cudaStream_t st, const dev::WaveArgs& a, int depth) {
  if (map)
    dev::k_shade<CLS, true><<<grid[1], 128, 0, st>>>(a, depth);
  else
    dev::k_shade<CLS, false><<<grid[0], 128, 0, st>>>(a, depth);
}

// Renders every job's samples, wave by wave.  Wave i runs on lane i % 2
// (its own stream and path state); the film kernels of successive waves are
// chained by events, so films accumulate in wave order exactly as on one
// stream.  The lanes fork from and join back into the context stream.
// Plans and launches the waves of `jobs`.  With `done` null the lanes join
// the context stream at the end (work after this call on the context stream
// sees the films finished); otherwise the lanes do not join: `done` is
// recorded once the batch has finished, and the next batch's waves queue
// behind this one's on each lane, so consecutive batches overlap.
static int run_jobs(ArgentCtx* ctx, const std::vector<dev::DevJob>& jobs, const std::vector<uint32_t>& counts,
                    const std::vector<const ArgentScene*>& job_scenes, cudaEvent_t done = nullptr) {
  int rc = ensure_tables(ctx);
  if (rc != ARGENT_OK) return rc;
  // Waves of up to wave_paths slots; a call with fewer path-samples than
  // that plans one wave of its own size (at least 2^16 slots).
  uint64_t total = 0;
  for (size_t j = 0; j < jobs.size(); ++j) total += (uint64_t)jobs[j].w * jobs[j].h * counts[j];
  uint32_t cap = (uint32_t)std::min<uint64_t>(ctx->limits.wave_paths, std::max<uint64_t>(total, 1u << 16));
  std::vector<uint32_t> depths;
  const std::vector<std::vector<uint32_t>> groups = plan_groups(ctx->share_rays, jobs, counts, job_scenes);
  std::vector<dev::WaveDesc> waves = plan_waves(jobs, counts, groups, cap, &depths);
  if (waves.empty()) return ARGENT_OK;
  // Followers of a group: which of their materials (and whether the rest of
  // what shading reads) equal the leader's.
  std::vector<dev::DevJob> shared_jobs;
  const std::vector<dev::DevJob>* job_list = &jobs;
  for (const auto& g : groups) {
    if (g.size() < 2) continue;
    if (shared_jobs.empty()) shared_jobs = jobs;
    for (size_t m = 1; m < g.size(); ++m)
      share_masks(jobs[g[0]], job_scenes[g[0]], job_scenes[g[m]], &shared_jobs[g[m]]);
    job_list = &shared_jobs;
  }
  rc = ensure_lane_streams(ctx, ctx->lanes);
  if (rc != ARGENT_OK) return rc;
  const int nlanes = ctx->lanes;
  // A joined batch with no overlapped batch in flight starts on lane 0: every
  // lane is idle once the context stream reaches it, and a fixed first lane
  // keeps its captured graph reusable whatever ran before (a 1-wave render in
  // between would otherwise shift the lanes and force a new capture).
  // Overlapped batches continue the rotation, so consecutive ones spread
  // over the lanes.
  const int start = (done == nullptr && !ctx->overlapped_pending) ? 0 : ctx->next_lane % nlanes;
  const int used = (int)std::min<size_t>((size_t)nlanes, waves.size());
  for (int k = 0; k < used; ++k) {
    rc = ensure_wave(ctx, (start + k) % nlanes, cap);
    if (rc != ARGENT_OK) return rc;
  }
  // Waves whose segments share rays, and their lanes' sharing buffers.
  std::vector<uint8_t> wshare(waves.size(), 0);
  for (size_t wi = 0; wi < waves.size(); ++wi) {
    for (uint32_t sgi = 0; sgi < waves[wi].num_segments; ++sgi)
      if (waves[wi].seg[sgi].lead != ~0u) wshare[wi] = 1;
    if (wshare[wi]) {
      rc = ensure_share(ctx, (int)((start + wi) % nlanes), cap);
      if (rc != ARGENT_OK) return rc;
    }
  }
  // Joined batches (done == null) read their job records from a buffer the
  // context keeps; overlapped ones from their own, freed when they finish.
  const bool joined = done == nullptr;
  dev::DevJob* d_jobs = nullptr;
  if (joined) {
    if (ctx->d_jobs_cap < jobs.size()) {
      if (ctx->d_jobs_buf) {
        ARGENT_CK(ctx, cudaStreamSynchronize(ctx->stream));
        cudaFree(ctx->d_jobs_buf);
      }
      ctx->d_jobs_buf = nullptr;
      ctx->d_jobs_cap = 0;
      size_t n = std::max<size_t>(jobs.size(), 64);
      if (cudaMalloc((void**)&ctx->d_jobs_buf, n * sizeof(dev::DevJob)) != cudaSuccess)
        return set_error(ctx, ARGENT_E_OOM, "job records: out of device memory");
      ctx->d_jobs_cap = n;
    }
    d_jobs = ctx->d_jobs_buf;
  } else {
    ARGENT_CK(ctx, cudaMallocAsync((void**)&d_jobs, jobs.size() * sizeof(dev::DevJob), ctx->stream));
  }
  // Pageable source: the call returns once the bytes are staged.
  ARGENT_CK(ctx, cudaMemcpyAsync(d_jobs, job_list->data(), jobs.size() * sizeof(dev::DevJob), cudaMemcpyHostToDevice,
                                 ctx->stream));
  dev::WaveArgs args[ARGENT_LANES];
  for (int l = 0; l < ARGENT_LANES; ++l) {
    args[l] = dev::WaveArgs{};
    args[l].jobs = d_jobs;
    args[l].status = ctx->d_status;
    fill_args(args[l], ctx->wave[l]);
  }
  int g_ray = grid_for(ctx, (const void*)dev::k_raygen, 256, cap);
  // Traversal grids: every resident block, or the tuned blocks per SM.
  auto tuned_grid = [&](int g, int bpsm) {
    if (bpsm <= 0) return g;
    uint64_t want = std::min<uint64_t>((cap + 127) / 128, (uint64_t)ctx->num_sms * bpsm);
    return (int)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)g));
  };
  int g_int[2] = {tuned_grid(grid_for(ctx, (const void*)dev::k_intersect<false>, 128, cap), ctx->trace_bpsm),
                  tuned_grid(grid_for(ctx, (const void*)dev::k_intersect<true>, 128, cap), ctx->trace_bpsm)};
  // Shading grids: ARGENT_SHADE_BLOCKS blocks per SM for the terminal,
  // dielectric and other classes; the metal and coated classes size their
  // own from their occupancy; a tuned class takes its tuned blocks per SM
  // (blocks beyond those resident wait for a free slot, and the persistent
  // loops take whatever work is left).
  int g_sh[NUM_CLS][2];
  const int g_shared = (int)std::max<uint64_t>(
      1, std::min<uint64_t>((cap + 127) / 128, (uint64_t)ctx->num_sms * ARGENT_SHADE_BLOCKS));
  for (int c = 0; c < NUM_CLS; ++c) g_sh[c][0] = g_sh[c][1] = g_shared;
  shade_grids<CLS_METAL>(ctx, cap, g_sh[CLS_METAL]);
  shade_grids<CLS_COATED>(ctx, cap, g_sh[CLS_COATED]);
  for (int c = 0; c < NUM_CLS; ++c) {
    if (ctx->shade_bpsm[c] <= 0) continue;
    g_sh[c][0] = g_sh[c][1] = (int)std::max<uint64_t>(
        1, std::min<uint64_t>((cap + 127) / 128, (uint64_t)ctx->num_sms * ctx->shade_bpsm[c]));
  }
  int g_any[2] = {tuned_grid(grid_for(ctx, (const void*)dev::k_shadow<false>, 128, cap), ctx->trace_bpsm),
                  tuned_grid(grid_for(ctx, (const void*)dev::k_shadow<true>, 128, cap), ctx->trace_bpsm)};
  int g_film = grid_for(ctx, (const void*)dev::k_film, 256, cap);
  int g_split = grid_for(ctx, (const void*)dev::k_share_split, 256, cap);
  // Per wave: its classes, whether any of its scenes has an env map (the
  // shading kernels without one leave the map code out) and, when its scenes
  // all trace alike (one scene, or metal variants of one: same_traversal),
  // the first of them for the traversal kernels' uniform form.
  std::vector<uint32_t> wclasses(waves.size()), wmap(waves.size());
  std::vector<const ArgentScene*> wone(waves.size());
  for (size_t wi = 0; wi < waves.size(); ++wi) {
    const dev::WaveDesc& w = waves[wi];
    uint32_t classes = 1u << CLS_TERMINAL, map = 0;
    const ArgentScene* one = job_scenes[w.seg[0].job];
    for (uint32_t sgi = 0; sgi < w.num_segments; ++sgi) {
      const ArgentScene* sc = job_scenes[w.seg[sgi].job];
      classes |= sc->host.class_mask;
      if (sc->host.env_is_map) map = 1;
      if (one && !same_traversal(one, sc)) one = nullptr;
    }
    wclasses[wi] = classes;
    wmap[wi] = map;
    wone[wi] = one;
  }
  // The first film pass waits for the last one before this batch only while
  // an overlapped batch may still be adding to films.  After a joined batch
  // the context stream already orders it: this batch forks from that stream
  // once the joined batch's lanes have joined it.  (A joined batch may have
  // been captured as a graph, and an event recorded during a capture is no
  // event to wait on outside it.)
  const bool chain_first = ctx->overlapped_pending;
  const int last_lane = (int)((start + waves.size() - 1) % nlanes);
  cudaStream_t join = joined ? ctx->stream : ctx->aux_stream;

  // Issues the batch: fork from the context stream, each wave's kernels on
  // its lane, join.  Counts the kernels it launches.
  // The step of the issue that failed first, for the error text.
  const char* stage = "fork";
  auto issue = [&](uint64_t* kernels) -> cudaError_t {
    // Launch errors are reported by cudaPeekAtLastError right after the
    // launch that caused them, so the failing step is named.
    auto launched = [&](cudaError_t& e, const char* what) {
      if (e != cudaSuccess) return;
      e = cudaPeekAtLastError();
      if (e != cudaSuccess) stage = what;
    };
    // An error left by an earlier, unrelated runtime call on this thread
    // (already reported by whichever call made it) is not this batch's.
    cudaError_t stale = cudaGetLastError();
    if (stale != cudaSuccess) ctx->stale_errors++;
    cudaError_t e = cudaEventRecord(ctx->fork_ev, ctx->stream);
    for (int k = 0; k < used && e == cudaSuccess; ++k)
      e = cudaStreamWaitEvent(ctx->lane_stream[(start + k) % nlanes], ctx->fork_ev, 0);
    if (e == cudaSuccess) stage = "waves";
    int prev_film = chain_first ? ctx->last_film_lane : -1;
    for (size_t wi = 0; wi < waves.size() && e == cudaSuccess; ++wi) {
      const dev::WaveDesc& w = waves[wi];
      int lane = (int)((start + wi) % nlanes);
      cudaStream_t st = ctx->lane_stream[lane];
      dev::WaveArgs& a = args[lane];
      const WaveBuffers& wb = ctx->wave[lane];
      const uint32_t classes = wclasses[wi];
      const bool map = wmap[wi] != 0;
      const ArgentScene* one = wone[wi];
      const int uni = one ? 1 : 0;
      a.uscene = one ? one->d_scene : nullptr;
      a.upiece = one ? one->host.piece : dev::DevPiece{};
      a.u_has_turn = one ? one->host.has_turn : 0;
      a.u_to_obj_s = one ? one->host.to_obj_s : 0.0f;
      a.u_to_obj_c = one ? one->host.to_obj_c : 1.0f;
      a.q_in = wb.q0;
      a.q_out = wb.q1;
      const bool shared = wshare[wi] != 0;
      a.lead = shared ? wb.lead : nullptr;
      a.shrec = shared ? wb.shrec : nullptr;
      a.vis = shared ? wb.vis : nullptr;
      a.qt = shared ? wb.qt : nullptr;
      a.qx = shared ? wb.qx : nullptr;
      a.qst = shared ? wb.qst : nullptr;
      a.qsx = shared ? wb.qsx : nullptr;
      a.qsc = shared ? wb.qsc : nullptr;
      {
        ProfScope ps(ctx, KC_RAYGEN, st);
        dev::k_raygen<<<g_ray, 256, 0, st>>>(a, w);
      }
      launched(e, "k_raygen");
      ++*kernels;
      for (uint32_t depth = 0; depth < depths[wi] && depth < ARGENT_MAX_DEPTH; ++depth) {
        a.q_in = (depth & 1) ? wb.q1 : wb.q0;
        a.q_out = (depth & 1) ? wb.q0 : wb.q1;
        {
          ProfScope ps(ctx, KC_INTERSECT, st);
          if (shared) {
            dev::k_share_split<<<g_split, 256, 0, st>>>(a, (int)depth);
            ++*kernels;
          }
          if (uni)
            dev::k_intersect<true><<<g_int[1], 128, 0, st>>>(a, (int)depth);
          else
            dev::k_intersect<false><<<g_int[0], 128, 0, st>>>(a, (int)depth);
          if (shared) {
            if (uni)
              dev::k_hit_copy<true><<<g_split, 256, 0, st>>>(a, (int)depth);
            else
              dev::k_hit_copy<false><<<g_split, 256, 0, st>>>(a, (int)depth);
            ++*kernels;
          }
        }
        launched(e, "k_intersect");
        {
          // One timing scope per class launch (profiling only); the shade
          // total is their sum.
          if (classes & (1u << CLS_TERMINAL)) {
            ProfScope ps(ctx, KC_SHADE_CLS0 + CLS_TERMINAL, st);
            launch_shade<CLS_TERMINAL>(map, g_sh[CLS_TERMINAL], st, a, (int)depth);
          }
          if (classes & (1u << CLS_METAL)) {
            ProfScope ps(ctx, KC_SHADE_CLS0 + CLS_METAL, st);
            launch_shade<CLS_METAL>(map, g_sh[CLS_METAL], st, a, (int)depth);
          }
          if (classes & (1u << CLS_COATED)) {
            ProfScope ps(ctx, KC_SHADE_CLS0 + CLS_COATED, st);
            launch_shade<CLS_COATED>(map, g_sh[CLS_COATED], st, a, (int)depth);
          }
          if (classes & (1u << CLS_DIELECTRIC)) {
            ProfScope ps(ctx, KC_SHADE_CLS0 + CLS_DIELECTRIC, st);
            launch_shade<CLS_DIELECTRIC>(map, g_sh[CLS_DIELECTRIC], st, a, (int)depth);
          }
          if (classes & (1u << CLS_OTHER)) {
            ProfScope ps(ctx, KC_SHADE_CLS0 + CLS_OTHER, st);
            launch_shade<CLS_OTHER>(map, g_sh[CLS_OTHER], st, a, (int)depth);
          }
          *kernels += __builtin_popcount(classes);
        }
        launched(e, "k_shade");
        {
          ProfScope ps(ctx, KC_SHADOW, st);
          if (shared) {
            dev::k_shadow_index<<<g_split, 256, 0, st>>>(a, (int)depth);
            dev::k_shade_copy<<<g_split, 256, 0, st>>>(a, (int)depth);
            dev::k_shadow_split<<<g_split, 256, 0, st>>>(a, (int)depth);
            *kernels += 3;
          }
          if (uni)
            dev::k_shadow<true><<<g_any[1], 128, 0, st>>>(a, (int)depth);
          else
            dev::k_shadow<false><<<g_any[0], 128, 0, st>>>(a, (int)depth);
          if (shared) {
            dev::k_shadow_copy<<<g_split, 256, 0, st>>>(a, (int)depth);
            ++*kernels;
          }
        }
        launched(e, "k_shadow");
        *kernels += 2;
      }
      if (ctx->counting) {
        dev::k_count_bounces<<<1, ARGENT_MAX_DEPTH, 0, st>>>(wb.counters, (int)std::min<uint32_t>(depths[wi],
                                                                                              ARGENT_MAX_DEPTH));
        ++*kernels;
      }
      // Films accumulate in wave order: wait for the previous wave's film pass.
      if (e == cudaSuccess && prev_film >= 0 && prev_film != lane) {
        e = cudaStreamWaitEvent(st, ctx->film_ev[prev_film], 0);
        if (e != cudaSuccess) stage = "film chain";
      }
      {
        ProfScope ps(ctx, KC_FILM, st);
        dev::k_film<<<g_film, 256, 0, st>>>(a, w);
      }
      launched(e, "k_film");
      if (e == cudaSuccess) e = cudaEventRecord(ctx->film_ev[lane], st);
      prev_film = lane;
      ++*kernels;
    }
    if (e == cudaSuccess) stage = "join";
    for (int k = 0; k < used && e == cudaSuccess; ++k) {
      e = cudaEventRecord(ctx->join_ev, ctx->lane_stream[(start + k) % nlanes]);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(join, ctx->join_ev, 0);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    return e;
  };

  cudaError_t e = cudaSuccess;
  uint64_t kernels = 0;
  // A joined batch without instrumentation is captured once as a CUDA graph
  // and replayed while the same waves come again (a render repeated with new
  // films, cameras or seeds changes only the job records).
  const bool graphs = joined && !chain_first && !ctx->prof.on && !ctx->counting && ctx->graphs_on;
  if (graphs) {
    std::vector<uint8_t> key;
    auto put = [&](const void* p, size_t n) {
      const uint8_t* b = (const uint8_t*)p;
      key.insert(key.end(), b, b + n);
    };
    put(&nlanes, sizeof(nlanes));
    put(&start, sizeof(start));
    put(&cap, sizeof(cap));
    put(g_int, sizeof(g_int));
    put(g_any, sizeof(g_any));
    put(g_sh, sizeof(g_sh));
    put(&d_jobs, sizeof(d_jobs));
    for (int k = 0; k < used; ++k) {
      put(&args[(start + k) % nlanes], sizeof(dev::WaveArgs));
      const WaveBuffers& wb = ctx->wave[(start + k) % nlanes];
      const void* sp[8] = {wb.lead, wb.shrec, wb.vis, wb.qt, wb.qx, wb.qst, wb.qsx, wb.qsc};
      put(sp, sizeof(sp));
    }
    for (size_t wi = 0; wi < waves.size(); ++wi) {
      const dev::WaveDesc& w = waves[wi];
      put(&w.num_segments, sizeof(w.num_segments));
      put(&w.num_slots, sizeof(w.num_slots));
      put(w.seg, w.num_segments * sizeof(dev::DevSegment));
      put(&depths[wi], sizeof(uint32_t));
      put(&wclasses[wi], sizeof(uint32_t));
      put(&wmap[wi], sizeof(uint32_t));
      const ArgentScene* one = wone[wi];
      const void* sp = one ? (const void*)one->d_scene : nullptr;
      put(&sp, sizeof(sp));
      if (one) {
        put(&one->host.piece, sizeof(one->host.piece));
        put(&one->host.has_turn, sizeof(one->host.has_turn));
        put(&one->host.to_obj_s, sizeof(float));
        put(&one->host.to_obj_c, sizeof(float));
      }
    }
    ArgentCtx::GraphEntry* hit = nullptr;
    for (auto& g : ctx->graph_cache)
      if (g.key == key) hit = &g;
    if (!hit) {
      cudaGraph_t graph = nullptr;
      cudaGraphExec_t exec = nullptr;
      e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        cudaError_t ie = issue(&kernels);
        e = cudaStreamEndCapture(ctx->stream, &graph);
        if (ie != cudaSuccess) e = ie;
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
      if (graph) cudaGraphDestroy(graph);
      if (e != cudaSuccess) {
        if (exec) cudaGraphExecDestroy(exec);
        return set_error(ctx, ARGENT_E_CUDA, std::string("render graph: ") + cudaGetErrorString(e));
      }
      if (ctx->graph_cache.size() >= ARGENT_GRAPH_CACHE) {
        auto lru = std::min_element(ctx->graph_cache.begin(), ctx->graph_cache.end(),
                                    [](const ArgentCtx::GraphEntry& x, const ArgentCtx::GraphEntry& y) {
                                      return x.last_use < y.last_use;
                                    });
        cudaGraphExecDestroy(lru->exec);
        ctx->graph_cache.erase(lru);
      }
      ctx->graph_cache.push_back(ArgentCtx::GraphEntry{std::move(key), exec, kernels, 0});
      hit = &ctx->graph_cache.back();
    }
    hit->last_use = ++ctx->graph_clock;
    e = cudaGraphLaunch(hit->exec, ctx->stream);
    kernels = hit->kernels;
  } else {
    e = issue(&kernels);
  }
  ctx->launches += kernels;
  ctx->next_lane = (int)((start + waves.size()) % nlanes);
  ctx->last_film_lane = last_lane;
  if (!joined) {
    cudaFreeAsync(d_jobs, join);
    if (e == cudaSuccess) e = cudaEventRecord(done, join);
    ctx->overlapped_pending = true;
  } else {
    // This batch's first film pass waited for the overlapped batches' last
    // one and its lanes joined the context stream, so work issued after it
    // is ordered after every film pass so far.
    ctx->overlapped_pending = false;
  }
  if (e != cudaSuccess)
    return set_error(ctx, ARGENT_E_CUDA, std::string("render launch (") + stage + "): " + cudaGetErrorString(e));
  return ARGENT_OK;
}

extern "C" {

// ------------------------------------------------------------------ scene

// 64-bit hash of a byte string, eight bytes at a time (a multiply-xorshift
// mix per word); equal hashes are confirmed by comparing the bytes.
static uint64_t blob_hash(const void* src, size_t bytes) {
  const uint8_t* p = (const uint8_t*)src;
  uint64_t h = 0x9e3779b97f4a7c15ull ^ bytes;
  size_t i = 0;
  for (; i + 8 <= bytes; i += 8) {
    uint64_t w;
    std::memcpy(&w, p + i, 8);
    h = (h ^ w) * 0xff51afd7ed558ccdull;
    h ^= h >> 32;
  }
  for (; i < bytes; ++i) h = (h ^ p[i]) * 0x100000001b3ull;
  return h;
}

// The device copy of `bytes` bytes equal to `src`: an existing blob of the
// same content gains a holder, or a new one is uploaded.  The pointer is
// added to `held`; null when the device is out of memory.
static void* intern_blob(ArgentCtx* ctx, const void* src, size_t bytes, std::vector<void*>* held) {
  uint64_t h = blob_hash(src, bytes);
  std::lock_guard<std::mutex> lock(ctx->blob_mu);
  for (auto& b : ctx->blobs) {
    if (b.hash == h && b.host.size() == bytes && std::memcmp(b.host.data(), src, bytes) == 0) {
      ++b.refs;
      held->push_back(b.dev);
      return b.dev;
    }
  }
  ArgentCtx::SharedBlob b;
  if (cudaMalloc(&b.dev, bytes) != cudaSuccess) return nullptr;
  if (cudaMemcpy(b.dev, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(b.dev);
    return nullptr;
  }
  b.hash = h;
  b.host.assign((const uint8_t*)src, (const uint8_t*)src + bytes);
  b.refs = 1;
  ctx->blobs.push_back(std::move(b));
  held->push_back(ctx->blobs.back().dev);
  return ctx->blobs.back().dev;
}

static void release_blob(ArgentCtx* ctx, void* dev) {
  std::lock_guard<std::mutex> lock(ctx->blob_mu);
  for (size_t i = 0; i < ctx->blobs.size(); ++i) {
    if (ctx->blobs[i].dev != dev) continue;
    if (--ctx->blobs[i].refs == 0) {
      cudaFree(dev);
      ctx->blobs.erase(ctx->blobs.begin() + (long)i);
    }
    return;
  }
}

void argent_scene_destroy(ArgentScene* s) {
  if (!s) return;
  cudaSetDevice(s->ctx->device);
  cudaStreamSynchronize(s->ctx->stream);
  for (void* a : s->allocs) cudaFree(a);
  for (void* b : s->shared) release_blob(s->ctx, b);
  if (s->staged) cudaFreeHost(s->staged);
  if (s->staged_ev) cudaEventDestroy(s->staged_ev);
  delete s;
}

static void set_turn(dev::DevScene& h, float deg) {
  h.has_turn = deg != 0.0f ? 1 : 0;
  float r_obj = (-deg) * (3.14159265358979323846f / 180.0f);
  float r_w = deg * (3.14159265358979323846f / 180.0f);
  h.to_obj_s = std::sin(r_obj);
  h.to_obj_c = std::cos(r_obj);
  h.to_world_s = std::sin(r_w);
  h.to_world_c = std::cos(r_w);
}

int argent_scene_upload(ArgentCtx* ctx, ArgentPiece* piece, const ArgentSceneDesc* desc, ArgentScene** out) {
  if (!ctx || !piece || !desc || !out) return set_error(ctx, ARGENT_E_INVALID, "argent_scene_upload: NULL argument");
  *out = nullptr;
  if (desc->num_materials <= 0 || !desc->materials)
    return set_error(ctx, ARGENT_E_INVALID, "a scene needs at least one material");
  if (desc->num_materials > 65535) return set_error(ctx, ARGENT_E_INVALID, "too many materials");
  if (piece->max_material >= (uint32_t)desc->num_materials)
    return set_error(ctx, ARGENT_E_INVALID, "tri_material refers past the material list");
  if (desc->num_materials > 254) return set_error(ctx, ARGENT_E_INVALID, "at most 254 materials per scene");
  if (desc->num_panels < 0 || desc->num_panels > ARGENT_MAX_PANELS)
    return set_error(ctx, ARGENT_E_INVALID, "at most 16 panels per scene");
  if (desc->num_panels > 0 && !desc->panels) return set_error(ctx, ARGENT_E_INVALID, "panels is NULL");
  if (desc->floor.enabled && (desc->floor.material < 0 || desc->floor.material >= desc->num_materials))
    return set_error(ctx, ARGENT_E_INVALID, "floor material out of range");
  for (int i = 0; i < desc->num_materials; ++i) {
    const ArgentMaterial& m = desc->materials[i];
    if (m.kind < ARGENT_MAT_METAL || m.kind > ARGENT_MAT_BLACK)
      return set_error(ctx, ARGENT_E_INVALID, "unknown material kind");
    if (m.kind == ARGENT_MAT_OPAL && !(m.cell_mm > 0.0f))
      return set_error(ctx, ARGENT_E_INVALID, "opal cell size must be positive");
  }
  const ArgentEnv* env = desc->env;
  bool is_map = env && env->kind == ARGENT_ENV_MAP;
  if (is_map && (env->width <= 0 || env->height <= 0 || !env->rgb))
    return set_error(ctx, ARGENT_E_INVALID, "environment map needs width, height and texels");
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  ArgentScene* s = new ArgentScene();
  s->ctx = ctx;
  s->piece = piece;
  dev::DevScene& h = s->host;
  std::memset(&h, 0, sizeof(h));
  h.piece = piece->dev;
  auto up = [&](const void* src, size_t bytes) -> void* {
    void* d = nullptr;
    if (cudaMalloc(&d, bytes) != cudaSuccess) return nullptr;
    s->allocs.push_back(d);
    s->bytes += bytes;
    if (cudaMemcpy(d, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
    return d;
  };
  // Data that other scenes of the context may hold too: one device copy.
  auto share = [&](const void* src, size_t bytes) -> void* { return intern_blob(ctx, src, bytes, &s->shared); };
  bool ok = true;
  h.mats = (const ArgentMaterial*)up(desc->materials, sizeof(ArgentMaterial) * desc->num_materials);
  s->mats_host.assign(desc->materials, desc->materials + desc->num_materials);
  ok = ok && h.mats;
  h.num_mats = desc->num_materials;
  h.num_panels = desc->num_panels;
  for (int i = 0; ok && i < desc->num_panels; ++i) {
    const ArgentPanel& p = desc->panels[i];
    dev::DevPanel& dp = h.panels[i];
    for (int a = 0; a < 3; ++a) {
      dp.c[a] = p.center[a];
      dp.hu[a] = p.hu[a];
      dp.hv[a] = p.hv[a];
    }
    argent::panel_frame(p, dp.n, &dp.area, &dp.hu_l2, &dp.hv_l2);
    dp.feather = p.feather;
    dp.emits = p.emits ? 1 : 0;
    dp.camera_visible = p.camera_visible ? 1 : 0;
    dp.emission = p.emits ? (const float*)share(p.emission, sizeof(float) * ARGENT_SPEC_LEN) : nullptr;
    ok = ok && (!p.emits || dp.emission);
  }
  argent::LightTable lt = argent::build_lights(*desc);
  h.num_lights = (int)lt.lights.size();
  for (size_t i = 0; i < lt.lights.size(); ++i) {
    h.lights[i] = lt.lights[i];
    h.light_cdf[i] = lt.cdf[i];
  }
  h.env_pick = lt.env_pick;
  static const float zeros[ARGENT_SPEC_LEN] = {0};
  if (is_map) {
    argent::EnvTables et = argent::build_env(env->rgb, env->width, env->height);
    float basis[3][471], inv[3][3];
    argent::linear_rgb(basis, inv);
    h.env_is_map = 1;
    h.map_w = env->width;
    h.map_h = env->height;
    h.map_weights = (const float*)share(et.weights.data(), et.weights.size() * sizeof(float));
    h.map_cond = (const float*)share(et.conditional.data(), et.conditional.size() * sizeof(float));
    h.map_marg = (const float*)share(et.marginal.data(), et.marginal.size() * sizeof(float));
    h.lin_basis = (const float*)share(basis, sizeof(basis));
    ok = ok && h.map_weights && h.map_cond && h.map_marg && h.lin_basis;
    float r_l = (-env->rotation_deg) * (3.14159265358979323846f / 180.0f);
    float r_w = env->rotation_deg * (3.14159265358979323846f / 180.0f);
    h.map_to_local_s = std::sin(r_l);
    h.map_to_local_c = std::cos(r_l);
    h.map_to_world_s = std::sin(r_w);
    h.map_to_world_c = std::cos(r_w);
  } else {
    h.env_is_map = 0;
    h.env_power = env ? env->power : 1.0f;
    h.env_top = (const float*)share(env ? env->top : zeros, sizeof(float) * ARGENT_SPEC_LEN);
    h.env_horizon = (const float*)share(env ? env->horizon : zeros, sizeof(float) * ARGENT_SPEC_LEN);
    h.env_bottom = (const float*)share(env ? env->bottom : zeros, sizeof(float) * ARGENT_SPEC_LEN);
    ok = ok && h.env_top && h.env_horizon && h.env_bottom;
  }
  h.floor_enabled = desc->floor.enabled ? 1 : 0;
  h.floor_y = desc->floor.y;
  h.floor_material = desc->floor.material;
  h.fade_start = desc->floor.fade_start;
  h.fade_end = desc->floor.fade_end;
  set_turn(h, desc->turntable_deg);
  h.class_mask = 1u << CLS_TERMINAL;
  for (int i = 0; i < desc->num_materials; ++i) {
    int c = dev::material_class(desc->materials[i].kind, desc->materials[i].gem_kind);
    h.mat_class[i] = (uint8_t)c;
    if (desc->floor.enabled && i == desc->floor.material) h.class_mask |= 1u << c;
  }
  for (uint32_t i = 0; i <= piece->max_material && (int)i < desc->num_materials; ++i)
    h.class_mask |= 1u << h.mat_class[i];
  h.floor_class = desc->floor.enabled ? h.mat_class[desc->floor.material] : CLS_TERMINAL;
  argent::camera_matrix(desc->has_white != 0, desc->white_xyz, h.cam_m);
  std::memcpy(s->cam_m, h.cam_m, sizeof(s->cam_m));
  if (ok) {
    s->d_scene = (dev::DevScene*)up(&h, sizeof(h));
    ok = s->d_scene != nullptr;
  }
  if (!ok) {
    argent_scene_destroy(s);
    return set_error(ctx, ARGENT_E_OOM, "scene upload: out of device memory");
  }
  *out = s;
  return ARGENT_OK;
}

int argent_scene_set_turntable(ArgentScene* s, float deg) {
  if (!s) return set_error(nullptr, ARGENT_E_INVALID, "scene is NULL");
  ArgentCtx* ctx = s->ctx;
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  // Stream-ordered, without waiting for the renders already queued (they
  // keep their angle): the descriptor goes through a pinned staging copy,
  // rewritten only once its previous copy has run.
  if (!s->staged) {
    ARGENT_CK(ctx, cudaMallocHost((void**)&s->staged, sizeof(dev::DevScene)));
    ARGENT_CK(ctx, cudaEventCreateWithFlags(&s->staged_ev, cudaEventDisableTiming));
  } else {
    ARGENT_CK(ctx, cudaEventSynchronize(s->staged_ev));
  }
  set_turn(s->host, deg);
  *s->staged = s->host;
  ARGENT_CK(ctx, cudaMemcpyAsync(s->d_scene, s->staged, sizeof(dev::DevScene), cudaMemcpyHostToDevice, ctx->stream));
  ARGENT_CK(ctx, cudaEventRecord(s->staged_ev, ctx->stream));
  return ARGENT_OK;
}

// ------------------------------------------------------------------ film

void argent_film_destroy(ArgentFilm* f) {
  if (!f) return;
  cudaSetDevice(f->ctx->device);
  cudaStreamSynchronize(f->ctx->stream);
  cudaFree(f->xyz);
  cudaFree(f->comp);
  cudaFree(f->xyz64);
  cudaFree(f->albedo);
  cudaFree(f->normal);
  delete f;
}

int argent_film_create(ArgentCtx* ctx, uint32_t width, uint32_t height, uint32_t flags, ArgentFilm** out) {
  if (!ctx || !out) return set_error(ctx, ARGENT_E_INVALID, "argent_film_create: NULL argument");
  *out = nullptr;
  if (width == 0 || height == 0 || (uint64_t)width * height > (1ull << 31))
    return set_error(ctx, ARGENT_E_INVALID, "film size out of range");
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  if (flags == 0) flags = ARGENT_FILM_KAHAN;
  ArgentFilm* f = new ArgentFilm();
  f->ctx = ctx;
  f->w = width;
  f->h = height;
  f->flags = flags;
  size_t n = 3ull * width * height;
  bool ok = cudaMalloc(&f->xyz, n * sizeof(float)) == cudaSuccess;
  ok = ok && cudaMalloc(&f->albedo, n * sizeof(float)) == cudaSuccess;
  ok = ok && cudaMalloc(&f->normal, n * sizeof(float)) == cudaSuccess;
  if (ok && (flags & ARGENT_FILM_KAHAN)) ok = cudaMalloc(&f->comp, n * sizeof(float)) == cudaSuccess;
  if (ok && (flags & ARGENT_FILM_FP64)) ok = cudaMalloc(&f->xyz64, n * sizeof(double)) == cudaSuccess;
  if (!ok) {
    argent_film_destroy(f);
    return set_error(ctx, ARGENT_E_OOM, "film: out of device memory");
  }
  f->bytes = n * (3 * sizeof(float) + ((flags & ARGENT_FILM_KAHAN) ? 4 : 0) + ((flags & ARGENT_FILM_FP64) ? 8 : 0));
  int rc = argent_film_clear(f);
  if (rc != ARGENT_OK) {
    argent_film_destroy(f);
    return rc;
  }
  *out = f;
  return ARGENT_OK;
}

int argent_film_clear(ArgentFilm* f) {
  if (!f) return set_error(nullptr, ARGENT_E_INVALID, "film is NULL");
  ArgentCtx* ctx = f->ctx;
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  size_t n = 3ull * f->w * f->h;
  ARGENT_CK(ctx, cudaMemsetAsync(f->xyz, 0, n * sizeof(float), ctx->stream));
  ARGENT_CK(ctx, cudaMemsetAsync(f->albedo, 0, n * sizeof(float), ctx->stream));
  ARGENT_CK(ctx, cudaMemsetAsync(f->normal, 0, n * sizeof(float), ctx->stream));
  if (f->comp) ARGENT_CK(ctx, cudaMemsetAsync(f->comp, 0, n * sizeof(float), ctx->stream));
  if (f->xyz64) ARGENT_CK(ctx, cudaMemsetAsync(f->xyz64, 0, n * sizeof(double), ctx->stream));
  f->samples = 0;
  f->has_matrix = false;
  return ARGENT_OK;
}

uint32_t argent_film_samples(const ArgentFilm* f) { return f ? f->samples : 0; }

static int film_fetch_xyz(ArgentFilm* f, std::vector<double>& xyz) {
  ArgentCtx* ctx = f->ctx;
  size_t n = 3ull * f->w * f->h;
  xyz.assign(n, 0.0);
  if (f->xyz64) {
    ARGENT_CK(ctx, cudaMemcpyAsync(xyz.data(), f->xyz64, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    ARGENT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  } else {
    std::vector<float> tmp(n);
    ARGENT_CK(ctx, cudaMemcpyAsync(tmp.data(), f->xyz, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    ARGENT_CK(ctx, cudaStreamSynchronize(ctx->stream));
    for (size_t i = 0; i < n; ++i) xyz[i] = tmp[i];
  }
  return ctx_check_status(ctx);
}

int argent_film_read_xyz(ArgentFilm* f, float* out) {
  if (!f || !out) return set_error(f ? f->ctx : nullptr, ARGENT_E_INVALID, "NULL argument");
  ARGENT_CK(f->ctx, cudaSetDevice(f->ctx->device));
  std::vector<double> xyz;
  int rc = film_fetch_xyz(f, xyz);
  if (rc != ARGENT_OK) return rc;
  double k = 1.0 / (double)std::max<uint32_t>(f->samples, 1);
  for (size_t i = 0; i < xyz.size(); ++i) out[i] = (float)(xyz[i] * k);
  return ARGENT_OK;
}

// render.rs:36-62: averages; color is the camera matrix applied to XYZ.
}  // extern "C"

namespace {

struct Mat3 {
  float m[9];
};

// Film::color / albedo / normal (render.rs:40-62) per pixel: camera RGB of
// the XYZ sums (((m0 x + m1 y) + m2 z) * k per row), albedo * k, and the
// normal sum scaled by k and normalised (zero when shorter than 1e-6), each
// rounded as the host loops round them (the library has no FMA contraction).
__global__ void __launch_bounds__(256) k_film_resolve(const float* xyz, const double* xyz64, const float* alb,
                                                      const float* nrm, Mat3 mt, float k, uint32_t np, float* color,
                                                      float* albedo, float* normal) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
    size_t o = 3 * (size_t)i;
    if (color) {
      float x, y, z;
      if (xyz64) {
        x = (float)xyz64[o];
        y = (float)xyz64[o + 1];
        z = (float)xyz64[o + 2];
      } else {
        x = xyz[o];
        y = xyz[o + 1];
        z = xyz[o + 2];
      }
      const float* m = mt.m;
#pragma unroll
      for (int c = 0; c < 3; ++c) color[o + c] = (m[3 * c] * x + m[3 * c + 1] * y + m[3 * c + 2] * z) * k;
    }
    if (albedo) {
#pragma unroll
      for (int c = 0; c < 3; ++c) albedo[o + c] = alb[o + c] * k;
    }
    if (normal) {
      float v[3] = {nrm[o] * k, nrm[o + 1] * k, nrm[o + 2] * k};
      float l = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
#pragma unroll
      for (int c = 0; c < 3; ++c) normal[o + c] = l > 1e-6f ? v[c] / l : 0.0f;
    }
  }
}

// Device staging for film reads, grown on demand and kept by the context.
int ensure_resolve(ArgentCtx* ctx, size_t floats) {
  if (ctx->resolve_floats >= floats) return ARGENT_OK;
  if (ctx->resolve) cudaFree(ctx->resolve);
  ctx->resolve = nullptr;
  ctx->resolve_floats = 0;
  if (cudaMalloc(&ctx->resolve, floats * sizeof(float)) != cudaSuccess)
    return set_error(ctx, ARGENT_E_OOM, "film read staging: out of device memory");
  ctx->resolve_floats = floats;
  return ARGENT_OK;
}

}  // namespace

extern "C" {

int argent_film_read(ArgentFilm* f, float* color, float* albedo, float* normal) {
  if (!f) return set_error(nullptr, ARGENT_E_INVALID, "film is NULL");
  ArgentCtx* ctx = f->ctx;
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  size_t np = (size_t)f->w * f->h;
  if (!color && !albedo && !normal) return ARGENT_OK;
  float k = 1.0f / (float)std::max<uint32_t>(f->samples, 1);
  Mat3 mt;
  if (f->has_matrix)
    std::memcpy(mt.m, f->cam_m, sizeof(mt.m));
  else
    argent::camera_matrix(false, nullptr, mt.m);
  int rc = ensure_resolve(ctx, 9 * np);
  if (rc != ARGENT_OK) return rc;
  float* d_color = color ? ctx->resolve : nullptr;
  float* d_albedo = albedo ? ctx->resolve + 3 * np : nullptr;
  float* d_normal = normal ? ctx->resolve + 6 * np : nullptr;
  int grid = (int)std::min<size_t>((np + 255) / 256, (size_t)ctx->num_sms * 8);
  k_film_resolve<<<std::max(grid, 1), 256, 0, ctx->stream>>>(f->xyz, f->xyz64, f->albedo, f->normal, mt, k,
                                                              (uint32_t)np, d_color, d_albedo, d_normal);
  ctx->launches++;
  ARGENT_CK(ctx, cudaGetLastError());
  if (color)
    ARGENT_CK(ctx, cudaMemcpyAsync(color, d_color, 3 * np * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  if (albedo)
    ARGENT_CK(ctx, cudaMemcpyAsync(albedo, d_albedo, 3 * np * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  if (normal)
    ARGENT_CK(ctx, cudaMemcpyAsync(normal, d_normal, 3 * np * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  ARGENT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  return ctx_check_status(ctx);
}

int argent_film_denoise(ArgentFilm* f, float* out) {
  if (!f || !out) return set_error(f ? f->ctx : nullptr, ARGENT_E_INVALID, "NULL argument");
  ArgentCtx* ctx = f->ctx;
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  size_t np = (size_t)f->w * f->h;
  float k = 1.0f / (float)std::max<uint32_t>(f->samples, 1);
  Mat3 mt;
  if (f->has_matrix)
    std::memcpy(mt.m, f->cam_m, sizeof(mt.m));
  else
    argent::camera_matrix(false, nullptr, mt.m);
  int rc = ensure_resolve(ctx, 9 * np);
  if (rc != ARGENT_OK) return rc;
  float *dc = ctx->resolve, *da = ctx->resolve + 3 * np, *dnrm = ctx->resolve + 6 * np;
  int grid = (int)std::min<size_t>((np + 255) / 256, (size_t)ctx->num_sms * 8);
  k_film_resolve<<<std::max(grid, 1), 256, 0, ctx->stream>>>(f->xyz, f->xyz64, f->albedo, f->normal, mt, k,
                                                              (uint32_t)np, dc, da, dnrm);
  ctx->launches++;
  float* dout = nullptr;
  ARGENT_CK(ctx, cudaMallocAsync((void**)&dout, 3 * np * sizeof(float), ctx->stream));
  rc = run_atrous(ctx, f->w, f->h, dc, da, dnrm, dout);
  cudaError_t e = cudaSuccess;
  if (rc == ARGENT_OK) e = cudaMemcpyAsync(out, dout, 3 * np * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
  cudaFreeAsync(dout, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (rc != ARGENT_OK) return rc;
  if (e != cudaSuccess) return set_error(ctx, ARGENT_E_CUDA, std::string("film denoise: ") + cudaGetErrorString(e));
  return ctx_check_status(ctx);
}

int argent_film_develop(ArgentFilm* f, const ArgentGrade* grade, int denoise, uint8_t* out) {
  if (!f || !grade || !out) return set_error(f ? f->ctx : nullptr, ARGENT_E_INVALID, "NULL argument");
  ArgentCtx* ctx = f->ctx;
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  size_t np = (size_t)f->w * f->h;
  float k = 1.0f / (float)std::max<uint32_t>(f->samples, 1);
  Mat3 mt;
  if (f->has_matrix)
    std::memcpy(mt.m, f->cam_m, sizeof(mt.m));
  else
    argent::camera_matrix(false, nullptr, mt.m);
  int rc = ensure_resolve(ctx, 9 * np);
  if (rc != ARGENT_OK) return rc;
  float *dc = ctx->resolve, *da = ctx->resolve + 3 * np, *dnrm = ctx->resolve + 6 * np;
  int grid = (int)std::min<size_t>((np + 255) / 256, (size_t)ctx->num_sms * 8);
  k_film_resolve<<<std::max(grid, 1), 256, 0, ctx->stream>>>(f->xyz, f->xyz64, f->albedo, f->normal, mt, k,
                                                              (uint32_t)np, dc, denoise ? da : nullptr,
                                                              denoise ? dnrm : nullptr);
  ctx->launches++;
  float* dd = nullptr;
  uint8_t* d8 = nullptr;
  ARGENT_CK(ctx, cudaMallocAsync((void**)&dd, 3 * np * sizeof(float), ctx->stream));
  ARGENT_CK(ctx, cudaMallocAsync((void**)&d8, 3 * np, ctx->stream));
  const float* src = dc;
  if (denoise) {
    rc = run_atrous(ctx, f->w, f->h, dc, da, dnrm, dd);
    src = dd;
  }
  if (rc == ARGENT_OK) rc = run_develop(ctx, f->w, f->h, src, grade, d8);
  cudaError_t e = cudaSuccess;
  if (rc == ARGENT_OK) e = cudaMemcpyAsync(out, d8, 3 * np, cudaMemcpyDeviceToHost, ctx->stream);
  cudaFreeAsync(dd, ctx->stream);
  cudaFreeAsync(d8, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (rc != ARGENT_OK) return rc;
  if (e != cudaSuccess) return set_error(ctx, ARGENT_E_CUDA, std::string("film develop: ") + cudaGetErrorString(e));
  return ctx_check_status(ctx);
}

// ------------------------------------------------------------------ render

// Long progressive renders switch their XYZ sums to FP64: the FP32 sums
// with their Kahan compensation seed the FP64 sums (sum - compensation),
// and from then on every film pass adds to both.
__global__ void k_film_promote(const float* xyz, const float* comp, double* xyz64, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    xyz64[i] = (double)xyz[i] - (comp ? (double)comp[i] : 0.0);
}

static int promote_if_long(ArgentFilm* f, uint64_t end_samples) {
  if (!(f->flags & ARGENT_FILM_PROGRESSIVE) || f->xyz64 || end_samples <= ARGENT_FILM_FP64_AFTER) return ARGENT_OK;
  ArgentCtx* ctx = f->ctx;
  size_t n = 3ull * f->w * f->h;
  cudaError_t e = cudaMalloc(&f->xyz64, n * sizeof(double));
  if (e != cudaSuccess) {
    f->xyz64 = nullptr;
    return set_error(ctx, ARGENT_E_OOM, "film: out of device memory for the FP64 sums");
  }
  f->bytes += n * sizeof(double);
  k_film_promote<<<(int)std::min<size_t>((n + 255) / 256, 148 * 16), 256, 0, ctx->stream>>>(f->xyz, f->comp, f->xyz64,
                                                                                          n);
  ctx->launches++;
  ARGENT_CK(ctx, cudaGetLastError());
  return ARGENT_OK;
}

static int make_job(ArgentScene* scene, const ArgentCamera* cam, ArgentFilm* film, const ArgentPathSettings* ps,
                    uint32_t seed, dev::DevJob* j) {
  ArgentCtx* ctx = scene->ctx;
  if (film->ctx != ctx) return set_error(ctx, ARGENT_E_INVALID, "film belongs to another context");
  if (ps->max_depth > ARGENT_MAX_DEPTH) return set_error(ctx, ARGENT_E_INVALID, "max_depth above 64");
  if (film->has_matrix && std::memcmp(film->cam_m, scene->cam_m, sizeof(film->cam_m)) != 0)
    return set_error(ctx, ARGENT_E_INVALID, "film already holds samples under a different white balance");
  std::memset(j, 0, sizeof(*j));
  j->scene = scene->d_scene;
  j->cam = *cam;
  j->w = film->w;
  j->h = film->h;
  j->first = film->samples;
  uint32_t x = seed ^ 0xa511e9b3u;  // render.rs:73
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  j->seed_h = x;
  j->max_depth = ps->max_depth;
  j->rr_depth = ps->rr_depth;
  j->clamp_indirect = ps->clamp_indirect;
  j->film_xyz = film->xyz;
  j->film_comp = film->comp;
  j->film_xyz64 = film->xyz64;
  j->film_albedo = film->albedo;
  j->film_normal = film->normal;
  return ARGENT_OK;
}

int argent_render_pass(ArgentCtx* ctx, ArgentScene* scene, const ArgentCamera* camera, ArgentFilm* film,
                       const ArgentPathSettings* settings, uint32_t count, uint32_t seed) {
  if (!ctx || !scene || !camera || !film || !settings)
    return set_error(ctx, ARGENT_E_INVALID, "argent_render_pass: NULL argument");
  if (scene->ctx != ctx) return set_error(ctx, ARGENT_E_INVALID, "scene belongs to another context");
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  if ((uint64_t)film->samples + count > 0xffffffffull) return set_error(ctx, ARGENT_E_INVALID, "sample index overflow");
  std::vector<dev::DevJob> jobs(1);
  int rc = promote_if_long(film, (uint64_t)film->samples + count);
  if (rc != ARGENT_OK) return rc;
  rc = make_job(scene, camera, film, settings, seed, &jobs[0]);
  if (rc != ARGENT_OK) return rc;
  std::vector<uint32_t> counts{count};
  std::vector<const ArgentScene*> scenes{scene};
  rc = run_jobs(ctx, jobs, counts, scenes);
  if (rc != ARGENT_OK) return rc;
  film->samples += count;
  film->has_matrix = true;
  std::memcpy(film->cam_m, scene->cam_m, sizeof(film->cam_m));
  return ARGENT_OK;
}

int argent_autotune(ArgentCtx* ctx, ArgentScene* scene, const ArgentCamera* camera,
                    const ArgentPathSettings* settings, uint32_t width, uint32_t height, uint32_t count,
                    ArgentTuneResult* results, uint32_t max_results, uint32_t* n_results) {
  if (!ctx || !scene || !camera || !settings || !n_results || (max_results && !results))
    return set_error(ctx, ARGENT_E_INVALID, "argent_autotune: NULL argument");
  if (width == 0 || height == 0 || count == 0) return set_error(ctx, ARGENT_E_INVALID, "empty tuning render");
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  *n_results = 0;
  size_t fr = 0, tot = 0;
  ARGENT_CK(ctx, cudaMemGetInfo(&fr, &tot));
  // A candidate's path state must fit in half of what is free now plus what
  // the context already holds.
  uint64_t held = 0;
  for (int l = 0; l < ARGENT_LANES; ++l) held += ctx->wave[l].bytes;
  uint64_t room = (uint64_t)fr / 2 + held;
  const uint32_t lanes_c[] = {2, 4, 8, 12, 16};
  const uint64_t waves_c[] = {1ull << 21, 1ull << 22, 1ull << 23, 1ull << 24, 1ull << 25};
  uint64_t path_samples = (uint64_t)width * height * count;
  ArgentFilm* film = nullptr;
  int rc = argent_film_create(ctx, width, height, ARGENT_FILM_KAHAN, &film);
  if (rc != ARGENT_OK) return rc;
  int keep_lanes = ctx->lanes;
  uint64_t keep_wave = ctx->limits.wave_paths;
  double best = -1.0;
  int best_lanes = keep_lanes;
  uint64_t best_wave = keep_wave;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (uint32_t L : lanes_c) {
    for (uint64_t W : waves_c) {
      if ((uint64_t)L * W * 244 > room) continue;
      if (W > path_samples * 2 && W > (1ull << 21)) continue;  // waves larger than the render change nothing
      ctx->lanes = (int)L;
      ctx->limits.wave_paths = W;
      rc = argent_film_clear(film);
      if (rc == ARGENT_OK) rc = argent_render_pass(ctx, scene, camera, film, settings, count, 1);  // warm-up
      if (rc == ARGENT_OK) rc = argent_film_clear(film);
      if (rc != ARGENT_OK) break;
      cudaEventRecord(e0, ctx->stream);
      rc = argent_render_pass(ctx, scene, camera, film, settings, count, 1);
      cudaEventRecord(e1, ctx->stream);
      if (rc == ARGENT_OK) rc = argent_ctx_sync(ctx);
      if (rc != ARGENT_OK) break;
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e0, e1);
      double v = ms > 0.0f ? (double)path_samples / (ms * 1e-3) : 0.0;
      if (*n_results < max_results) {
        results[*n_results].lanes = L;
        results[*n_results].reserved = 0;
        results[*n_results].wave_paths = W;
        results[*n_results].path_samples_per_s = v;
      }
      ++*n_results;
      if (v > best) {
        best = v;
        best_lanes = (int)L;
        best_wave = W;
      }
    }
    if (rc != ARGENT_OK) break;
  }
  // Second phase at the best lanes and wave size: blocks per SM of each
  // shading class the scene uses, then of the traversals, one knob at a
  // time; a value is kept only when it is faster by more than 1 %, which
  // is above the run-to-run spread of such a render.
  const int keep_trace = ctx->trace_bpsm;
  int keep_shade[NUM_CLS];
  for (int c = 0; c < NUM_CLS; ++c) keep_shade[c] = ctx->shade_bpsm[c];
  if (rc == ARGENT_OK && best > 0.0) {
    ctx->lanes = best_lanes;
    ctx->limits.wave_paths = best_wave;
    auto measure = [&](double* v) -> int {
      int r = argent_film_clear(film);
      if (r == ARGENT_OK) r = argent_render_pass(ctx, scene, camera, film, settings, count, 1);  // warm-up
      if (r == ARGENT_OK) r = argent_film_clear(film);
      if (r != ARGENT_OK) return r;
      cudaEventRecord(e0, ctx->stream);
      r = argent_render_pass(ctx, scene, camera, film, settings, count, 1);
      cudaEventRecord(e1, ctx->stream);
      if (r == ARGENT_OK) r = argent_ctx_sync(ctx);
      if (r != ARGENT_OK) return r;
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e0, e1);
      *v = ms > 0.0f ? (double)path_samples / (ms * 1e-3) : 0.0;
      return ARGENT_OK;
    };
    double cur = 0.0;
    rc = measure(&cur);
    const uint32_t classes = (1u << CLS_TERMINAL) | scene->host.class_mask;
    const int shade_c[] = {2, 3, 4, 5, 6, 8};
    for (int c = 0; c < NUM_CLS && rc == ARGENT_OK; ++c) {
      if (!((classes >> c) & 1u)) continue;
      int keep = ctx->shade_bpsm[c];
      for (int v : shade_c) {
        ctx->shade_bpsm[c] = v;
        double r = 0.0;
        rc = measure(&r);
        if (rc != ARGENT_OK) break;
        if (r > cur * 1.01) {
          cur = r;
          keep = v;
        }
      }
      ctx->shade_bpsm[c] = keep;
    }
    const int trace_c[] = {4, 6, 8};
    int keep_t = ctx->trace_bpsm;
    for (int v : trace_c) {
      if (rc != ARGENT_OK) break;
      ctx->trace_bpsm = v;
      double r = 0.0;
      rc = measure(&r);
      if (rc == ARGENT_OK && r > cur * 1.01) {
        cur = r;
        keep_t = v;
      }
    }
    ctx->trace_bpsm = keep_t;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  argent_film_destroy(film);
  if (rc != ARGENT_OK) {
    ctx->lanes = keep_lanes;
    ctx->limits.wave_paths = keep_wave;
    ctx->trace_bpsm = keep_trace;
    for (int c = 0; c < NUM_CLS; ++c) ctx->shade_bpsm[c] = keep_shade[c];
    return rc;
  }
  ctx->lanes = best_lanes;
  ctx->limits.wave_paths = best_wave;
  // Free the path state of lanes the chosen configuration does not use.
  ARGENT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  for (int l = best_lanes; l < ARGENT_LANES; ++l) ctx->wave[l].release();
  return ARGENT_OK;
}

int argent_ctx_config(const ArgentCtx* ctx, uint32_t* lanes, uint64_t* wave_paths) {
  if (!ctx) return set_error(nullptr, ARGENT_E_INVALID, "ctx is NULL");
  if (lanes) *lanes = (uint32_t)ctx->lanes;
  if (wave_paths) *wave_paths = ctx->limits.wave_paths;
  return ARGENT_OK;
}

int argent_ctx_tuning(const ArgentCtx* ctx, ArgentTuning* out) {
  if (!ctx || !out) return set_error(ctx, ARGENT_E_INVALID, "argent_ctx_tuning: NULL argument");
  std::memset(out, 0, sizeof(*out));
  out->lanes = (uint32_t)ctx->lanes;
  out->wave_paths = ctx->limits.wave_paths;
  out->trace_blocks_per_sm = (uint32_t)ctx->trace_bpsm;
  for (int c = 0; c < NUM_CLS; ++c) out->shade_blocks_per_sm[c] = (uint32_t)ctx->shade_bpsm[c];
  return ARGENT_OK;
}

int argent_ctx_set_tuning(ArgentCtx* ctx, const ArgentTuning* t) {
  if (!ctx || !t) return set_error(ctx, ARGENT_E_INVALID, "argent_ctx_set_tuning: NULL argument");
  if (t->trace_blocks_per_sm > 64) return set_error(ctx, ARGENT_E_INVALID, "trace_blocks_per_sm above 64");
  for (int c = 0; c < NUM_CLS; ++c)
    if (t->shade_blocks_per_sm[c] > 64) return set_error(ctx, ARGENT_E_INVALID, "shade_blocks_per_sm above 64");
  int rc = argent_ctx_set_config(ctx, t->lanes, t->wave_paths);
  if (rc != ARGENT_OK) return rc;
  ctx->trace_bpsm = (int)t->trace_blocks_per_sm;
  for (int c = 0; c < NUM_CLS; ++c) ctx->shade_bpsm[c] = (int)t->shade_blocks_per_sm[c];
  return ARGENT_OK;
}

int argent_ctx_set_config(ArgentCtx* ctx, uint32_t lanes, uint64_t wave_paths) {
  if (!ctx) return set_error(nullptr, ARGENT_E_INVALID, "ctx is NULL");
  if (lanes < 1 || lanes > ARGENT_LANES || wave_paths < (1ull << 16) || wave_paths > (1ull << 30))
    return set_error(ctx, ARGENT_E_INVALID, "argent_ctx_set_config: lanes must be 1..16 and wave_paths 2^16..2^30");
  // Work already queued keeps the lanes it was issued on; the next call
  // starts its waves at lane 0 of the new rotation.
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  ARGENT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->lanes = (int)lanes;
  ctx->limits.wave_paths = wave_paths;
  ctx->next_lane = 0;
  return ARGENT_OK;
}

}  // extern "C"

// argent_render_batch; with `done` the batch overlaps the next one (run_jobs).
static int render_batch(ArgentCtx* ctx, const ArgentBatchItem* items, uint32_t n, cudaEvent_t done) {
  if (!ctx || (n && !items)) return set_error(ctx, ARGENT_E_INVALID, "argent_render_batch: NULL argument");
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  std::vector<dev::DevJob> jobs(n);
  std::vector<uint32_t> counts(n);
  std::vector<const ArgentScene*> scenes(n);
  // A progressive film that this batch takes past the FP64 threshold gets
  // its FP64 sums before any of its items is planned.
  for (uint32_t i = 0; i < n; ++i) {
    if (!items[i].film || items[i].film->ctx != ctx) continue;  // refused below
    uint64_t end = items[i].film->samples;
    for (uint32_t k = 0; k < n; ++k)
      if (items[k].film == items[i].film) end += items[k].count;
    int rc = promote_if_long(items[i].film, end);
    if (rc != ARGENT_OK) return rc;
  }
  // Items that share a film run one after another: the second starts where
  // the first leaves film.samples.
  std::vector<uint32_t> pending(n, 0);
  for (uint32_t i = 0; i < n; ++i) {
    const ArgentBatchItem& it = items[i];
    if (!it.scene || !it.film) return set_error(ctx, ARGENT_E_INVALID, "batch item without scene or film");
    if (it.scene->ctx != ctx) return set_error(ctx, ARGENT_E_INVALID, "scene belongs to another context");
    uint32_t base = it.film->samples;
    for (uint32_t k = 0; k < i; ++k)
      if (items[k].film == it.film) base += items[k].count;
    int rc = make_job(it.scene, &it.camera, it.film, &it.settings, it.seed, &jobs[i]);
    if (rc != ARGENT_OK) return rc;
    for (uint32_t k = 0; k < i; ++k)
      if (items[k].film == it.film && std::memcmp(items[k].scene->cam_m, it.scene->cam_m, sizeof(float) * 9) != 0)
        return set_error(ctx, ARGENT_E_INVALID, "batch items share a film under different white balances");
    jobs[i].first = base;
    counts[i] = it.count;
    scenes[i] = it.scene;
  }
  int rc = run_jobs(ctx, jobs, counts, scenes, done);
  if (rc != ARGENT_OK) return rc;
  for (uint32_t i = 0; i < n; ++i) {
    items[i].film->samples += items[i].count;
    items[i].film->has_matrix = true;
    std::memcpy(items[i].film->cam_m, items[i].scene->cam_m, sizeof(float) * 9);
  }
  return ARGENT_OK;
}

bool scene_belongs(const ArgentScene* scene, const ArgentCtx* ctx) { return scene && scene->ctx == ctx; }

int render_batch_overlapped(ArgentCtx* ctx, const ArgentBatchItem* items, uint32_t n, cudaEvent_t done) {
  if (!done) return set_error(ctx, ARGENT_E_INVALID, "render_batch_overlapped: no completion event");
  return render_batch(ctx, items, n, done);
}

extern "C" {

int argent_render_batch(ArgentCtx* ctx, const ArgentBatchItem* items, uint32_t n) {
  return render_batch(ctx, items, n, nullptr);
}

}  // extern "C"

extern "C" {

int argent_ctx_set_profiling(ArgentCtx* ctx, int on) {
  if (!ctx) return set_error(nullptr, ARGENT_E_INVALID, "ctx is NULL");
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  prof_collect(ctx);
  ctx->prof.on = on != 0;
  for (int k = 0; k < KC_COUNT; ++k) {
    ctx->prof.ms[k] = 0.0;
    ctx->prof.n[k] = 0;
  }
  return ARGENT_OK;
}

int argent_ctx_kernel_times(ArgentCtx* ctx, double* ms, uint64_t* launches) {
  if (!ctx || !ms || !launches) return set_error(ctx, ARGENT_E_INVALID, "NULL argument");
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  prof_collect(ctx);
  for (int k = 0; k < KC_COUNT; ++k) {
    ms[k] = ctx->prof.ms[k];
    launches[k] = ctx->prof.n[k];
  }
  ms[KC_SHADE] = 0.0;
  launches[KC_SHADE] = 0;
  for (int c = 0; c < 5; ++c) {
    ms[KC_SHADE] += ctx->prof.ms[KC_SHADE_CLS0 + c];
    launches[KC_SHADE] += ctx->prof.n[KC_SHADE_CLS0 + c];
  }
  return ARGENT_OK;
}

int argent_ctx_set_graphs(ArgentCtx* ctx, int on) {
  if (!ctx) return set_error(nullptr, ARGENT_E_INVALID, "ctx is NULL");
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  ctx->graphs_on = on != 0;
  if (!ctx->graphs_on) {
    ARGENT_CK(ctx, cudaStreamSynchronize(ctx->stream));
    for (auto& g : ctx->graph_cache) cudaGraphExecDestroy(g.exec);
    ctx->graph_cache.clear();
  }
  return ARGENT_OK;
}

int argent_ctx_set_ray_sharing(ArgentCtx* ctx, int on) {
  if (!ctx) return set_error(nullptr, ARGENT_E_INVALID, "ctx is NULL");
  ctx->share_rays = on != 0;
  return ARGENT_OK;
}

int argent_ctx_set_counting(ArgentCtx* ctx, int on) {
  if (!ctx) return set_error(nullptr, ARGENT_E_INVALID, "ctx is NULL");
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  ARGENT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  int v = on ? 1 : 0;
  unsigned long long z[16] = {};
  unsigned int zm[2] = {0, 0};
  ARGENT_CK(ctx, cudaMemcpyToSymbol(dev::d_trav_counting, &v, sizeof(v)));
  ARGENT_CK(ctx, cudaMemcpyToSymbol(dev::d_trav_counts, z, 6 * sizeof(unsigned long long)));
  ARGENT_CK(ctx, cudaMemcpyToSymbol(dev::d_trav_hist, z, sizeof(z)));
  ARGENT_CK(ctx, cudaMemcpyToSymbol(dev::d_trav_max, zm, sizeof(zm)));
  unsigned long long zc[18] = {};
  ARGENT_CK(ctx, cudaMemcpyToSymbol(dev::d_trav_child_hits, zc, sizeof(zc)));
  std::vector<unsigned long long> zb(2 * ARGENT_MAX_DEPTH, 0ull);
  ARGENT_CK(ctx, cudaMemcpyToSymbol(dev::d_bounce_counts, zb.data(), zb.size() * sizeof(unsigned long long)));
  ctx->counting = on != 0;
  return ARGENT_OK;
}

int argent_ctx_bounce_counts(ArgentCtx* ctx, uint64_t* out) {
  if (!ctx || !out) return set_error(ctx, ARGENT_E_INVALID, "NULL argument");
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  ARGENT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  unsigned long long b[2 * ARGENT_MAX_DEPTH];
  ARGENT_CK(ctx, cudaMemcpyFromSymbol(b, dev::d_bounce_counts, sizeof(b)));
  for (int i = 0; i < 2 * ARGENT_MAX_DEPTH; ++i) out[i] = b[i];
  return ARGENT_OK;
}

int argent_ctx_traversal_histogram(ArgentCtx* ctx, uint64_t* out18) {
  if (!ctx || !out18) return set_error(ctx, ARGENT_E_INVALID, "NULL argument");
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  ARGENT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  unsigned long long h[16];
  unsigned int m[2];
  ARGENT_CK(ctx, cudaMemcpyFromSymbol(h, dev::d_trav_hist, sizeof(h)));
  ARGENT_CK(ctx, cudaMemcpyFromSymbol(m, dev::d_trav_max, sizeof(m)));
  for (int i = 0; i < 16; ++i) out18[i] = h[i];
  out18[16] = m[0];
  out18[17] = m[1];
  return ARGENT_OK;
}

int argent_ctx_child_hit_histogram(ArgentCtx* ctx, uint64_t* out18) {
  if (!ctx || !out18) return set_error(ctx, ARGENT_E_INVALID, "NULL argument");
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  ARGENT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  unsigned long long h[18];
  ARGENT_CK(ctx, cudaMemcpyFromSymbol(h, dev::d_trav_child_hits, sizeof(h)));
  for (int i = 0; i < 18; ++i) out18[i] = h[i];
  return ARGENT_OK;
}

int argent_ctx_traversal_counts(ArgentCtx* ctx, uint64_t* out6) {
  if (!ctx || !out6) return set_error(ctx, ARGENT_E_INVALID, "NULL argument");
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  ARGENT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  unsigned long long z[6];
  ARGENT_CK(ctx, cudaMemcpyFromSymbol(z, dev::d_trav_counts, sizeof(z)));
  for (int i = 0; i < 6; ++i) out6[i] = z[i];
  return ARGENT_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ allocation-free closest hit
//
// A variant of argent_trace_closest for callers that must not allocate
// device memory while they run (see argent_gpu.h).  Its staging buffers are
// this file-scope array instead of cudaMallocAsync: rays first, then hits.
// Every GPU that loads the library holds the array until the process exits.

#define ARGENT_NOALLOC_MAX_RAYS (1u << 18)

static __device__ __align__(256) unsigned char g_noalloc_scratch[(size_t)ARGENT_NOALLOC_MAX_RAYS *
                                                                 (sizeof(ArgentRay) + sizeof(ArgentHit))];

// Device address of g_noalloc_scratch (in host code the name is only a
// host-side stand-in), looked up by a context's first call with its device
// current and kept in the context.  A context made after a device reset
// looks it up afresh, so it never uses an address of a context that is gone.
static int noalloc_scratch(ArgentCtx* ctx, unsigned char** out) {
  if (!ctx->noalloc_addr) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return set_error(ctx, ARGENT_E_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") +
                                               cudaGetErrorString(e));
    ctx->noalloc_addr = p;
  }
  *out = (unsigned char*)ctx->noalloc_addr;
  return ARGENT_OK;
}

extern "C" int argent_trace_closest_noalloc(ArgentCtx* ctx, ArgentPiece* piece, const ArgentRay* rays, uint64_t n,
                                            ArgentHit* hits) {
  if (!ctx || !piece || (n && (!rays || !hits))) return set_error(ctx, ARGENT_E_INVALID, "NULL argument");
  if (n > ARGENT_NOALLOC_MAX_RAYS)
    return set_error(ctx, ARGENT_E_INVALID,
                     "argent_trace_closest_noalloc: " + std::to_string(n) +
                         " rays exceed the allocation-free maximum of " + std::to_string(ARGENT_NOALLOC_MAX_RAYS));
  if (n == 0) return ARGENT_OK;
  ARGENT_CK(ctx, cudaSetDevice(ctx->device));
  unsigned char* base = nullptr;
  int rc = noalloc_scratch(ctx, &base);
  if (rc != ARGENT_OK) return rc;
  ArgentRay* d_rays = reinterpret_cast<ArgentRay*>(base);
  ArgentHit* d_hits = reinterpret_cast<ArgentHit*>(base + (size_t)ARGENT_NOALLOC_MAX_RAYS * sizeof(ArgentRay));
  // Every hit the call returns is written by the kernel, so nothing in the
  // array has to start at zero; rays are overwritten by this copy.
  ARGENT_CK(ctx, cudaMemcpyAsync(d_rays, rays, n * sizeof(ArgentRay), cudaMemcpyHostToDevice, ctx->stream));
  int block = 128;
  int grid = grid_for(ctx, (const void*)k_trace_closest, block, n);
  {
    ProfScope ps(ctx, KC_TRACE);
    k_trace_closest<<<grid, block, 0, ctx->stream>>>(piece->dev, d_rays, n, d_hits, ctx->d_status);
  }
  ctx->launches++;
  ARGENT_CK(ctx, cudaGetLastError());
  ARGENT_CK(ctx, cudaMemcpyAsync(hits, d_hits, n * sizeof(ArgentHit), cudaMemcpyDeviceToHost, ctx->stream));
  ARGENT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  return ctx_check_status(ctx);
}
