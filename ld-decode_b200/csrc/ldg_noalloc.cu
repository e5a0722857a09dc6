// Allocation-free variant of ldg_demod_blocks.
//
// Who needs it: callers that cannot call cudaMalloc at demodulation time --
// a host process whose device memory is owned by another allocator (a
// framework's caching pool that has reserved the GPU, so a raw cudaMalloc
// would fail or fragment it), or a latency-critical capture loop that must
// not pay cudaMalloc's implicit device-wide synchronisation in the middle of
// a stream of blocks.  ldg_demod_blocks grows a per-context scratch buffer
// with cudaMalloc on first use and stages host buffers through an arena;
// this entry point does neither.
//
// The demodulator's scratch (two parked 16384-point spectra per resident
// CTA, 256 KB per CTA) lives instead in the file-scope device array below,
// sized for kNoAllocSlots CTAs.  Every GPU that loads this library holds
// that array (kNoAllocSlots * 256 KB = 8 MB) until the process exits.  All
// calls share it and it keeps the last call's contents; the kernel writes
// every scratch element before reading it, so nothing needs clearing, but
// two calls that overlap on the GPU (different streams, or different
// contexts on the same device) race on it and must be serialised by the
// caller.
#include <string>

#include "ldg_demod.cuh"
#include "ldg_fft.cuh"
#include "ldg_noalloc.h"
#include "ldgpu.h"

namespace {

constexpr int kNoAllocSlots = 32;
constexpr size_t kSlotFloat2 = ldg::kScratchPerCta / sizeof(float2);

static __device__ __align__(256) float2 g_noalloc_scratch[kNoAllocSlots * kSlotFloat2];

// Device address of the scratch array on the current device.  Looked up on
// every call (cudaGetSymbolAddress allocates nothing and is cheap), so an
// address never outlives the device context it came from: after a
// cudaDeviceReset the next call gets the array of the new context.  The
// host-side symbol itself is not a device address and must never be handed
// to a kernel.
int scratch_address(float2** out) {
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || ptr == nullptr) {
        cudaGetLastError();
        return LDG_ERR_CUDA;
    }
    *out = static_cast<float2*>(ptr);
    return LDG_OK;
}

}  // namespace

extern "C" int ldg_demod_blocks_noalloc(ldg_ctx* ctx, const ldg_demod_args* a, int32_t ctas) {
    ldg::DemodParams p;
    int grid = 0;
    int device = 0;
    int rc = ldg::noalloc_prepare(ctx, a, ctas, kNoAllocSlots, &p, &grid, &device);
    if (rc != LDG_OK || grid == 0) return rc;
    // the symbol lookup and the launch run with the context's device current
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != device && cudaSetDevice(device) != cudaSuccess)
        return ldg::api_fail(LDG_ERR_CUDA, "ldg_demod_blocks_noalloc: cannot make the context's device current");
    struct Restore {
        int prev, dev;
        ~Restore() {
            if (prev >= 0 && prev != dev) cudaSetDevice(prev);
        }
    } restore{prev, device};
    float2* scratch = nullptr;
    rc = scratch_address(&scratch);
    if (rc != LDG_OK)
        return ldg::api_fail(rc, "ldg_demod_blocks_noalloc: cudaGetSymbolAddress of the static scratch failed");
    p.scratch = scratch;
    const cudaError_t e = ldg::launch_demod(p, grid, static_cast<cudaStream_t>(ldg::noalloc_stream(ctx, a)));
    if (e != cudaSuccess)
        return ldg::api_fail(LDG_ERR_CUDA, std::string("demod launch: ") + cudaGetErrorString(e));
    return LDG_OK;
}
