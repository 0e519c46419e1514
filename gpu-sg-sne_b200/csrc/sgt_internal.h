// sgt_internal.h -- context accessors shared by the engine's translation
// units (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "../../include/sgtsne_b200.h"

cudaStream_t sgti_stream(sgt_ctx *ctx);
int sgti_device(sgt_ctx *ctx);
// records msg as the context's last error and returns s
sgt_status sgti_fail(sgt_ctx *ctx, sgt_status s, const std::string &msg);
// Stream-ordered device allocation (free with cudaFreeAsync) from the
// context's memory pool.  The pool keeps the memory of freed buffers for the
// next allocation instead of returning it to the driver at the next
// synchronisation, so creating a job after another one retired maps no new
// pages; sgt_destroy trims the pool.
cudaError_t sgti_alloc(sgt_ctx *ctx, void **p, size_t bytes, cudaStream_t s);
