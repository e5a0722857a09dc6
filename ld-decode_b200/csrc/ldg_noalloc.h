// Internal helpers shared by the context implementation (ldg_abi.cu), the
// allocation-free demod entry point (ldg_noalloc.cu), the mixed-batch queue
// (ldg_queue.cu) and the ingest kernels (ldg_ingest.cu).
#pragma once
#include <string>

#include "ldg_demod.cuh"
#include "ldgpu.h"

namespace ldg {

// Validate `a` for the allocation-free path (device buffers only) and fill
// `p` (all but p->scratch).  grid = ctas, or min(nblocks, max_slots) when
// ctas == 0; ctas > max_slots is rejected.  Allocates nothing.
int noalloc_prepare(ldg_ctx* ctx, const ldg_demod_args* a, int ctas, int max_slots, DemodParams* p, int* grid,
                    int* device);
// Record msg as this thread's ldg_last_error() and return code.
int api_fail(int code, const std::string& msg);

// Validate a batch whose buffers are all device memory and fill `p` from it
// and ctx's filters (scheduling fields zero); `who` names the caller in
// error messages.
int device_params(ldg_ctx* ctx, const ldg_demod_args* a, const std::string& who, DemodParams* p);
int ctx_device(const ldg_ctx* ctx);
void* noalloc_stream(ldg_ctx* ctx, const ldg_demod_args* a);

}  // namespace ldg
