// SM-driven copies through host-mapped pinned memory (see ldg_copy.cuh).
#include "ldg_copy.cuh"
#include "ldg_noalloc.h"
#include "ldgpu.h"

#include <string>

namespace ldg {

namespace {

// 16-byte words when both ends are 16-byte aligned, bytes otherwise.
__global__ void sm_copy_kernel(uint8_t* __restrict__ dst, const uint8_t* __restrict__ src, long long n) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (((reinterpret_cast<uintptr_t>(dst) | reinterpret_cast<uintptr_t>(src)) & 15) == 0) {
        const long long nw = n >> 4;
        const uint4* s = reinterpret_cast<const uint4*>(src);
        uint4* d = reinterpret_cast<uint4*>(dst);
        for (long long i = t; i < nw; i += stride) d[i] = s[i];
        for (long long i = (nw << 4) + t; i < n; i += stride) dst[i] = src[i];
    } else {
        for (long long i = t; i < n; i += stride) dst[i] = src[i];
    }
}

}  // namespace

void* device_view(const void* p) {
    if (!p) return nullptr;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) return const_cast<void*>(p);
    if (a.type == cudaMemoryTypeHost) return a.devicePointer;
    return nullptr;
}

cudaError_t sm_copy(void* dst, const void* src, size_t nbytes, cudaStream_t stream) {
    if (nbytes == 0) return cudaSuccess;
    const long long words = (long long)(nbytes + 15) / 16;
    long long grid = (words + 255) / 256;
    if (grid > 4 * 148) grid = 4 * 148;
    sm_copy_kernel<<<(unsigned)grid, 256, 0, stream>>>(static_cast<uint8_t*>(dst), static_cast<const uint8_t*>(src),
                                                       (long long)nbytes);
    return cudaGetLastError();
}

}  // namespace ldg

extern "C" int ldg_copy_async(void* dst, const void* src, int64_t nbytes, void* stream) {
    if (!dst || !src || nbytes < 0) return ldg::api_fail(LDG_ERR_ARG, "ldg_copy_async: NULL pointer or negative size");
    void* d = ldg::device_view(dst);
    void* s = ldg::device_view(src);
    if (!d || !s)
        return ldg::api_fail(LDG_ERR_ARG, "ldg_copy_async: both buffers must be device memory or pinned host memory");
    const cudaError_t e = ldg::sm_copy(d, s, (size_t)nbytes, (cudaStream_t)stream);
    if (e != cudaSuccess) return ldg::api_fail(LDG_ERR_CUDA, std::string("ldg_copy_async: ") + cudaGetErrorString(e));
    return LDG_OK;
}
