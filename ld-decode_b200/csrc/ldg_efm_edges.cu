// Zero crossings of the demodulator's EFM output on the GPU: the edges that
// EFM_PLL.process (lddecode/efm_pll.py:124-167) detects one sample at a
// time and feeds to its PLL.  A crossing is a sample whose sign differs
// from the sample before it (negative against not negative); each is kept
// as its position and the two sample values, from which the PLL's
// interpolated fraction -prev / (cur - prev) follows exactly.  With the
// crossings on the host, ldg_efm_pll_process_edges runs the PLL without
// the samples: an EFM stream then crosses PCIe as ~8 bytes per crossing
// (one every ~25 samples of band-limited EFM) instead of 2 bytes per
// sample.
//
// Three launches, as the sync-run scan: crossings counted per tile of 8192
// samples, an exclusive scan of the tile counts (which also writes the
// total where the caller asked, device or host-mapped memory), crossings
// written in order.
#include <stdint.h>

#include <string>

#include "ldg_copy.cuh"
#include "ldgpu.h"

namespace ldg {
int api_fail(int code, const std::string& msg);
}

namespace {

constexpr int kTile = 8192;
constexpr int kThreads = 256;
constexpr int kSteps = kTile / (4 * kThreads);

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// crossing bits of samples base .. base+3 (bit k: sample base+k)
__device__ __forceinline__ unsigned crossings4(const int16_t* __restrict__ x, long long n, long long base,
                                               int has_before) {
    int prev = base > 0 ? (int)x[base - 1] : (has_before ? (int)x[-1] : 0);
    unsigned bits = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (base + k >= n) break;
        const int cur = x[base + k];
        if ((prev ^ cur) < 0) bits |= 1u << k;
        prev = cur;
    }
    return bits;
}

__global__ void __launch_bounds__(kThreads) efm_count_kernel(const int16_t* __restrict__ x, long long n,
                                                             int has_before, int* __restrict__ counts) {
    const long long t0 = (long long)blockIdx.x * kTile;
    int c = 0;
    for (int j = 0; j < kSteps; ++j) {
        const long long base = t0 + (long long)j * 4 * kThreads + 4 * threadIdx.x;
        if (base < n) c += __popc(crossings4(x, n, base, has_before));
    }
    __shared__ int warp_sum[kThreads / 32];
    for (int o = 16; o; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int w = 0; w < kThreads / 32; ++w) s += warp_sum[w];
        counts[blockIdx.x] = s;
    }
}

// exclusive scan of the tile counts (one CTA); the total to *total and, if
// given, to *count_out
__global__ void __launch_bounds__(1024) efm_scan_kernel(const int* __restrict__ counts, long long ntiles,
                                                        long long* __restrict__ offsets, long long* total,
                                                        long long* count_out) {
    __shared__ long long part[1024];
    __shared__ long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (long long base = 0; base < ntiles; base += 1024) {
        const long long i = base + threadIdx.x;
        const long long v = i < ntiles ? counts[i] : 0;
        part[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            const long long add = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
            __syncthreads();
            part[threadIdx.x] += add;
            __syncthreads();
        }
        if (i < ntiles) offsets[i] = carry + part[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry += part[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *total = carry;
        if (count_out) *count_out = carry;
    }
}

__global__ void __launch_bounds__(kThreads) efm_write_kernel(const int16_t* __restrict__ x, long long n,
                                                             int has_before, const long long* __restrict__ offsets,
                                                             ldg_efm_edge* __restrict__ edges, long long cap,
                                                             long long pos_offset) {
    __shared__ int warp_cnt[kThreads / 32];
    const long long t0 = (long long)blockIdx.x * kTile;
    long long out = offsets[blockIdx.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int j = 0; j < kSteps; ++j) {
        const long long base = t0 + (long long)j * 4 * kThreads + 4 * threadIdx.x;
        const unsigned e = base < n ? crossings4(x, n, base, has_before) : 0u;
        const int cnt = __popc(e);
        int inc = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) warp_cnt[warp] = inc;
        __syncthreads();
        int before = 0, chunk = 0;
#pragma unroll
        for (int w = 0; w < kThreads / 32; ++w) {
            before += w < warp ? warp_cnt[w] : 0;
            chunk += warp_cnt[w];
        }
        long long k = out + before + inc - cnt;
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (e & (1u << q)) {
                if (k < cap) {
                    const long long i = base + q;
                    ldg_efm_edge r;
                    r.pos = (int32_t)(pos_offset + i);
                    r.prev = i > 0 ? x[i - 1] : (has_before ? x[-1] : (int16_t)0);
                    r.cur = x[i];
                    edges[k] = r;
                }
                ++k;
            }
        out += chunk;
        __syncthreads();
    }
}

}  // namespace

extern "C" {

int64_t ldg_efm_edges_scratch_bytes(int64_t n) {
    if (n < 0) return -1;
    const long long ntiles = (n + kTile - 1) / kTile;
    return (int64_t)(align256((size_t)ntiles * sizeof(int)) + align256((size_t)ntiles * sizeof(long long)) + 256);
}

int ldg_efm_edges(const int16_t* efm, int64_t n, int32_t has_before, int64_t pos_offset, ldg_efm_edge* edges,
                  int64_t cap, int64_t* count, void* scratch, void* stream) {
    if (!efm || !edges || !scratch || n < 0 || cap < 0)
        return ldg::api_fail(LDG_ERR_ARG, "ldg_efm_edges: NULL buffer or negative size");
    if (pos_offset < 0 || pos_offset + n > (int64_t)INT32_MAX)
        return ldg::api_fail(LDG_ERR_RANGE, "ldg_efm_edges: positions must fit int32 (pos_offset + n)");
    long long* dcount = nullptr;
    if (count) {
        dcount = static_cast<long long*>(ldg::device_view(count));
        if (!dcount)
            return ldg::api_fail(LDG_ERR_ARG, "ldg_efm_edges: count must be device memory or pinned host memory");
    }
    cudaStream_t st = (cudaStream_t)stream;
    const long long ntiles = (n + kTile - 1) / kTile;
    char* p = static_cast<char*>(scratch);
    int* counts = reinterpret_cast<int*>(p);
    long long* offsets = reinterpret_cast<long long*>(p + align256((size_t)ntiles * sizeof(int)));
    long long* total = reinterpret_cast<long long*>(p + align256((size_t)ntiles * sizeof(int)) +
                                                    align256((size_t)ntiles * sizeof(long long)));
    if (ntiles > 0) {
        efm_count_kernel<<<(unsigned)ntiles, kThreads, 0, st>>>(efm, n, has_before, counts);
        efm_scan_kernel<<<1, 1024, 0, st>>>(counts, ntiles, offsets, total, dcount);
        efm_write_kernel<<<(unsigned)ntiles, kThreads, 0, st>>>(efm, n, has_before, offsets, edges, cap, pos_offset);
    } else if (dcount) {
        if (cudaMemsetAsync(dcount, 0, sizeof(long long), st) != cudaSuccess) cudaGetLastError();
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return ldg::api_fail(LDG_ERR_CUDA, std::string("ldg_efm_edges: ") + cudaGetErrorString(e));
    return LDG_OK;
}

}  // extern "C"

namespace {

// one thread per field: its EFM slice [startloc + int(ll[1]), startloc +
// int(ll[end_line])) and the samples at both ends
__global__ void efm_slices_kernel(const long long* __restrict__ startloc, const unsigned long long* __restrict__ llp,
                                  const int* __restrict__ end_line, int n, const int16_t* __restrict__ efm,
                                  long long efm_len, long long* bounds, int16_t* samples) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* ll = reinterpret_cast<const double*>(llp[i]);
    const long long lo = startloc[i] + (long long)ll[1];  // truncation, as int() of the location
    const long long hi = startloc[i] + (long long)ll[end_line[i]];
    bounds[2 * i] = lo;
    bounds[2 * i + 1] = hi;
    samples[2 * i] = lo >= 0 && lo < efm_len ? efm[lo] : (int16_t)0;
    samples[2 * i + 1] = hi - 1 >= 0 && hi - 1 < efm_len ? efm[hi - 1] : (int16_t)0;
}

}  // namespace

extern "C" int ldg_efm_field_slices(const int64_t* startloc, const uint64_t* linelocs, const int32_t* end_line,
                                    int32_t n, const int16_t* efm, int64_t efm_len, int64_t* bounds,
                                    int16_t* samples, void* stream) {
    if (n < 0 || (n > 0 && (!startloc || !linelocs || !end_line || !efm || !bounds || !samples)))
        return ldg::api_fail(LDG_ERR_ARG, "ldg_efm_field_slices: NULL buffer or negative count");
    if (n == 0) return LDG_OK;
    const void* p[5] = {startloc, linelocs, end_line, bounds, samples};
    void* d[5];
    for (int k = 0; k < 5; ++k) {
        d[k] = ldg::device_view(p[k]);
        if (!d[k])
            return ldg::api_fail(LDG_ERR_ARG, "ldg_efm_field_slices: arrays must be device memory or pinned host memory");
    }
    efm_slices_kernel<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(
        static_cast<const long long*>(d[0]), static_cast<const unsigned long long*>(d[1]),
        static_cast<const int*>(d[2]), n, efm, efm_len, static_cast<long long*>(d[3]), static_cast<int16_t*>(d[4]));
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return ldg::api_fail(LDG_ERR_CUDA, std::string("ldg_efm_field_slices: ") + cudaGetErrorString(e));
    return LDG_OK;
}
