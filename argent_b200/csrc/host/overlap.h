// overlap.h — the library-internal form of argent_render_batch whose lanes
// do not join the context stream: `done` is recorded when the batch has
// finished, and the next batch's waves queue behind this one's on each
// lane, so a scheduler can keep the next batch in flight while one runs.
// Work later on the context stream does not wait for the batch; wait for
// `done` (or argent_ctx_sync) before reading its films.
#pragma once
#include <cuda_runtime.h>

#include "../../../include/argent_gpu.h"

int render_batch_overlapped(ArgentCtx* ctx, const ArgentBatchItem* items, uint32_t n, cudaEvent_t done);

// Whether `scene` was uploaded on `ctx`.
bool scene_belongs(const ArgentScene* scene, const ArgentCtx* ctx);

// The context's device status word (traversal stack or queue overflow,
// expired waits) as a status code, cleared once read.
int ctx_check_status(ArgentCtx* ctx);
