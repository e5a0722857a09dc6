// .lds ingest: DomesdayDuplicator 10-bit packed samples (4 samples in 5
// bytes, most significant bits first) to the signed 16-bit samples the
// reference's loader returns (unpack_data_4_40, lddecode/utils.py:371-391):
// value v of a sample -> (v - 512) << 6.
//
// Each CTA stages a contiguous run of packed bytes in shared memory with
// aligned 4-byte loads, then each thread unpacks groups of 5 bytes and
// writes 4 samples.  HBM-bound: 1.25 bytes read and 2 written per sample.
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "ldg_noalloc.h"
#include "ldgpu.h"

namespace {

constexpr int kThreads = 256;
constexpr int kGroupsPerThread = 4;
constexpr int kGroups = kThreads * kGroupsPerThread;   // 1024 groups = 4096 samples per CTA
constexpr int kBytes = kGroups * 5;                     // 5120 packed bytes per CTA

__device__ __forceinline__ int16_t to_s16(unsigned v) { return (int16_t)(((int)v - 512) * 64); }

// Samples [first, first + n) of the packed buffer; sample k lives in group
// k / 4 (bytes 5 (k / 4) .. +4).  CTA c covers groups [g0 + c * kGroups, ...).
__global__ void __launch_bounds__(kThreads) lds_unpack_kernel(const uint8_t* __restrict__ packed, long long nbytes,
                                                               long long first, long long n,
                                                               int16_t* __restrict__ out) {
    __shared__ __align__(16) uint8_t sb[kBytes + 8];
    const long long g0 = first / 4 + (long long)blockIdx.x * kGroups;  // first group of this CTA
    const long long b0 = g0 * 5;
    // aligned word loads covering [b0, b0 + kBytes)
    const long long a0 = b0 & ~3LL;
    const int lead = (int)(b0 - a0);
    const int nwords = (kBytes + lead + 3) / 4;
    const uint32_t* src = reinterpret_cast<const uint32_t*>(packed + a0);
    for (int w = threadIdx.x; w < nwords; w += kThreads) {
        const long long at = a0 + 4LL * w;
        uint32_t v = 0;
        if (at + 4 <= nbytes) {
            v = __ldcs(src + w);
        } else {
            for (int j = 0; j < 4; ++j)
                if (at + j < nbytes) v |= (uint32_t)packed[at + j] << (8 * j);
        }
        if (4 * w < kBytes + 8) *reinterpret_cast<uint32_t*>(sb + 4 * w) = v;
    }
    __syncthreads();
    for (int gi = threadIdx.x; gi < kGroups; gi += kThreads) {
        const long long g = g0 + gi;
        const long long k0 = 4 * g;  // first sample of the group
        if (k0 >= first + n) break;
        const uint8_t* p = sb + lead + 5 * gi;
        const unsigned c0 = p[0], c1 = p[1], c2 = p[2], c3 = p[3], c4 = p[4];
        const int16_t s[4] = {to_s16((c0 << 2) | (c1 >> 6)), to_s16(((c1 & 0x3F) << 4) | (c2 >> 4)),
                              to_s16(((c2 & 0x0F) << 6) | (c3 >> 2)), to_s16(((c3 & 0x03) << 8) | c4)};
        const long long o = k0 - first;  // output index of sample k0
        if (o >= 0 && o + 4 <= n && ((o & 3) == 0)) {
            // 8-byte store of 4 samples (out is 8-byte aligned when first % 4 == 0)
            uint2 u;
            u.x = (uint32_t)(uint16_t)s[0] | ((uint32_t)(uint16_t)s[1] << 16);
            u.y = (uint32_t)(uint16_t)s[2] | ((uint32_t)(uint16_t)s[3] << 16);
            __stcs(reinterpret_cast<uint2*>(out + o), u);
        } else {
            for (int j = 0; j < 4; ++j)
                if (o + j >= 0 && o + j < n) out[o + j] = s[j];
        }
    }
}

}  // namespace

extern "C" int ldg_unpack_lds(const uint8_t* packed, int64_t nbytes, int64_t first, int64_t n, int16_t* out,
                              void* stream) {
    using ldg::api_fail;
    if (!packed || !out) return api_fail(LDG_ERR_ARG, "ldg_unpack_lds: NULL buffer");
    if (first < 0 || n < 0 || nbytes < 0) return api_fail(LDG_ERR_ARG, "ldg_unpack_lds: negative size");
    if (n == 0) return LDG_OK;
    const long long last_group = (first + n - 1) / 4;
    if ((last_group + 1) * 5 > nbytes)
        return api_fail(LDG_ERR_RANGE, "ldg_unpack_lds: the packed buffer ends before the last sample");
    if ((reinterpret_cast<uintptr_t>(packed) & 3) != 0 || (reinterpret_cast<uintptr_t>(out) & 7) != 0)
        return api_fail(LDG_ERR_ARG, "ldg_unpack_lds: packed must be 4-byte and out 8-byte aligned");
    const long long groups = last_group - first / 4 + 1;
    const long long grid = (groups + kGroups - 1) / kGroups;
    if (grid > 0x7fffffffLL) return api_fail(LDG_ERR_ARG, "ldg_unpack_lds: too many samples");
    lds_unpack_kernel<<<(unsigned)grid, kThreads, 0, (cudaStream_t)stream>>>(packed, nbytes, first, n, out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return api_fail(LDG_ERR_CUDA, std::string("ldg_unpack_lds: ") + cudaGetErrorString(e));
    return LDG_OK;
}
