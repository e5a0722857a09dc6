// Per-context state of the single-pass (decoupled look-back) scan behind
// ldg_sync_runs: a ticket counter that is never reset, so a call's tiles are
// the tickets base .. base + ntiles - 1 in the order its CTAs start; per-tile
// flag words tagged with the call's number (flags of earlier calls never
// match); per-tile edge counts and inclusive prefixes.  Calls on a context
// are serialised by its mutex and each waits for its own kernels, so two
// calls never share the state on the GPU.
#pragma once
#include <cuda_runtime.h>

struct ldg_ctx;

namespace ldg {

struct ScanState {
    unsigned long long* ticket;
    unsigned long long* flags;
    long long* agg;
    long long* incl;
    unsigned long long base;
    unsigned long long call;
};

// The state for a call over `ntiles` tiles (grown and zeroed on `st` when
// needed); advances the context's ticket base and call number.
int ctx_scan_state(ldg_ctx* c, long long ntiles, cudaStream_t st, ScanState* out);

// After a failed call: the next call starts from a fresh state.
void ctx_scan_invalidate(ldg_ctx* c);

}  // namespace ldg
