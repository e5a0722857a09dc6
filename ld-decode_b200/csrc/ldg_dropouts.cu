// Dropout detection, one CTA per field: Field.dropout_detect
// (lddecode/core.py:2962-2983).
//
//  1. rfstd: FP64 mean, then FP64 mean squared deviation of the field's
//     rfhpf read (nb_std, core.py:2836; numba sums in another order, which
//     moves the result by ~1e-13 relative).
//  2. Sync areas of every line l >= 1 (core.py:2867-2873): whole lines for
//     the vertical-sync lines, otherwise the first hsync_len samples; Python
//     slice bounds, then a prefix maximum of the area ends so that "inside
//     any area" is one binary search plus a forward walk.
//  3. The error mask per sample (core.py:2837-2887) over the field's lines,
//     compacted in order into the field's error list (warp ballots and a
//     block scan per tile of 4096 samples).
//  4. One thread merges the error samples into spans (build_errlist,
//     core.py:2889-2908) and places the spans on TBC lines as it goes
//     (dropout_errlist_to_tbc, core.py:2910-2960), in the reference's
//     FP64 arithmetic.
#include <cuda_runtime.h>
#include <stdint.h>

#include "ldg_dropouts.cuh"

namespace ldg {

namespace {

constexpr int kThreads = kDropThreads;
constexpr int kPer = 8;  // consecutive samples per thread per tile
constexpr int kWarps = kThreads / 32;

__device__ __forceinline__ long long py_index(long long x, long long n) {
    // a slice bound as Python normalises it
    if (x < 0) {
        x += n;
        return x < 0 ? 0 : x;
    }
    return x > n ? n : x;
}

__device__ __forceinline__ bool is_vsync_line(int l, int system, int isfirst) {
    // Field.get_vsync_lines (core.py:2814-2827)
    if (l >= 1 && l < (isfirst ? 10 : 9)) return true;
    return system == 1 && l >= (isfirst ? 311 : 310) && l < 318;
}

__device__ double block_sum(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        double w = threadIdx.x < kWarps ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
        if (threadIdx.x == 0) red[32] = w;
    }
    __syncthreads();
    const double r = red[32];
    __syncthreads();
    return r;
}

struct Emitter {
    int* out;
    int cap;
    int n;
    bool over;
    __device__ void put(int line, long long a, long long b) {
        if (n < cap) {
            out[3 * n] = line;
            out[3 * n + 1] = (int)a;
            out[3 * n + 2] = (int)b;
        } else {
            over = true;
        }
        ++n;
    }
};

// Spans to TBC lines (core.py:2910-2960), fed one span at a time in order.
struct LinePlacer {
    const double* ll;
    int line, end_line, lineoffset;
    double outlinelen;
    double ll0;
    bool placing;          // past the reference's initial skip of spans before line `lineoffset`
    bool have_pending;
    double p0, p1;
    Emitter* em;

    __device__ void place(double c0, double c1) {
        while (line < end_line) {
            const double a = ll[line], b = ll[line + 1];
            if (c0 >= a && c0 <= b) {
                const double span = b - a;
                const long long start = (long long)(((c0 - a) / span) * outlinelen);
                const long long end = (long long)rint(((c1 - a) / span) * outlinelen);
                const int first = line + 1 - lineoffset;
                const long long ol = (long long)outlinelen;
                if (end > ol) {
                    const long long k = end / ol;
                    em->put(first - 1, start, ol);
                    for (long long j = 0; j < k - 1; ++j) em->put((int)(first + j + 1) - 1, 0, ol);
                    em->put((int)(first + k) - 1, 0, end % ol);
                } else {
                    em->put(first - 1, start, end);
                }
                return;
            }
            ++line;
        }
    }
    __device__ void feed(double s0, double s1) {
        if (!placing) {
            if (!have_pending) {
                p0 = s0;
                p1 = s1;
                have_pending = true;
                return;
            }
            if (p0 < ll0) {  // a later span exists: the reference pops on
                p0 = s0;
                p1 = s1;
                return;
            }
            placing = true;
            place(p0, p1);
        }
        place(s0, s1);
    }
    __device__ void finish() {
        if (!placing && have_pending) {
            placing = true;
            place(p0, p1);
        }
    }
};

}  // namespace

__global__ void __launch_bounds__(kThreads) dropout_kernel(const DropField* fields, const DropConsts k, int* errs,
                                                            int* drops, int* counts, double* rfstd_out) {
    __shared__ double red[33];
    __shared__ long long rs[kMaxDropRegions], pm[kMaxDropRegions];
    __shared__ int s_bad;
    __shared__ int s_wsum[kWarps];
    __shared__ long long s_base;
    const DropField f = fields[blockIdx.x];
    const long long n = f.len;
    int* ferr = errs + (size_t)blockIdx.x * k.err_cap;
    if (threadIdx.x == 0) {
        s_bad = 0;
        s_base = 0;
    }

    // ---- 1. rfhpf standard deviation
    double s = 0.0;
    for (long long i = threadIdx.x; i < n; i += kThreads) s += (double)__ldg(f.rfhpf + i);
    const double mean = block_sum(s, red) / (double)n;
    s = 0.0;
    for (long long i = threadIdx.x; i < n; i += kThreads) {
        const double d = (double)__ldg(f.rfhpf + i) - mean;
        s = fma(d, d, s);
    }
    const double rfstd = sqrt(block_sum(s, red) / (double)n);
    const double rf_hi = rfstd * 3.0, rf_lo = -rfstd * 3.0;

    // ---- 2. sync areas
    const int nreg = f.nlines - 1;
    for (int l = 1 + threadIdx.x; l < f.nlines; l += kThreads) {
        const long long a = (long long)f.ll[l];
        long long b;
        if (is_vsync_line(l, k.system, f.isfirst)) {
            if (l + 1 >= f.nlines) {
                atomicOr(&s_bad, 2);
                b = a;
            } else {
                b = (long long)f.ll[l + 1];
            }
        } else {
            b = a + f.hsync_len;
        }
        rs[l - 1] = py_index(a, n);
        pm[l - 1] = py_index(b, n);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int r = 1; r < nreg; ++r) {
            if (rs[r] < rs[r - 1]) s_bad |= 1;
            if (pm[r] < pm[r - 1]) pm[r] = pm[r - 1];
        }
    }
    __syncthreads();
    const int bad = s_bad;
    if (bad) {
        if (threadIdx.x == 0) {
            counts[2 * blockIdx.x] = (bad & 2) ? -3 : -2;
            counts[2 * blockIdx.x + 1] = 0;
            if (rfstd_out) rfstd_out[blockIdx.x] = rfstd;
        }
        return;
    }

    // ---- 3. error mask over [lo, hi), compacted in order
    const long long lo = py_index((long long)f.ll[f.lineoffset + 1], n);
    const long long hi = py_index((long long)f.ll[f.lineoffset + f.linecount + 1], n);
    const float* dm = f.demod;
    const float* d5 = f.d05;
    const float* dr = f.raw;
    const float* hp = f.rfhpf;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (long long t0 = lo; t0 < hi; t0 += (long long)kThreads * kPer) {
        const long long i0 = t0 + (long long)threadIdx.x * kPer;
        unsigned m = 0;
        if (i0 < hi) {
            // last area starting at or before i0
            int lo_r = 0, hi_r = nreg - 1, idx = -1;
            while (lo_r <= hi_r) {
                const int mid = (lo_r + hi_r) >> 1;
                if (rs[mid] <= i0) {
                    idx = mid;
                    lo_r = mid + 1;
                } else {
                    hi_r = mid - 1;
                }
            }
#pragma unroll
            for (int j = 0; j < kPer; ++j) {
                const long long i = i0 + j;
                if (i >= hi) break;
                while (idx + 1 < nreg && rs[idx + 1] <= i) ++idx;
                const bool sync = idx >= 0 && i < pm[idx];
                bool e = false;
                if (i >= k.video_rot) {
                    const double h = (double)__ldg(hp + i - k.video_rot);
                    e = (h < rf_lo) || (h > rf_hi);
                }
                e |= (double)__ldg(dr + i) > k.fhalf;
                const float d = __ldg(dm + i);
                e |= (d < (sync ? k.smin : k.vmin)) || (d > k.vmax);
                const float q = __ldg(d5 + i);
                e |= (q < (sync ? k.smin05 : k.vmin05)) || (q > k.vmax05);
                if (e) m |= 1u << j;
            }
        }
        // block exclusive scan of the per-thread counts
        const int c = __popc(m);
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        if (lane == 31) s_wsum[warp] = incl;
        __syncthreads();
        int woff = 0, total = 0;
        for (int w = 0; w < kWarps; ++w) {
            const int v = s_wsum[w];
            if (w < warp) woff += v;
            total += v;
        }
        long long pos = s_base + woff + incl - c;
        while (m) {
            const int j = __ffs(m) - 1;
            m &= m - 1;
            if (pos < k.err_cap) ferr[pos] = (int)(i0 + j);
            ++pos;
        }
        __syncthreads();
        if (threadIdx.x == 0) s_base += total;
        __syncthreads();
    }

    // ---- 4. spans and TBC lines (one thread, the reference's order)
    if (threadIdx.x != 0) return;
    const long long nerr = s_base;
    if (rfstd_out) rfstd_out[blockIdx.x] = rfstd;
    counts[2 * blockIdx.x + 1] = nerr > k.err_cap ? -1 : (int)nerr;
    if (nerr > k.err_cap) {
        counts[2 * blockIdx.x] = 0;
        return;
    }
    Emitter em{drops + (size_t)blockIdx.x * k.out_cap * 3, k.out_cap, 0, false};
    const double ll0 = f.ll[f.lineoffset];
    if (nerr > 0 && (double)ferr[nerr - 1] > ll0) {
        LinePlacer lp{f.ll, f.lineoffset, f.lineoffset + f.linecount, f.lineoffset, (double)k.outlinelen, ll0,
                      false, false, 0.0, 0.0, &em};
        const double cap = k.freq_mhz * 12.0;
        bool started = false;
        long long firsterr = 0, c0 = 0;
        double c1 = 0.0;
        for (long long j = 0; j < nerr; ++j) {
            const long long e = ferr[j];
            if (!started) {
                if ((double)e >= ll0) {
                    started = true;
                    firsterr = c0 = e;
                    c1 = (double)e;
                }
                continue;
            }
            if (e > c0 && (double)e <= c1 + 20.0) {
                double pad = (double)(e - c0) * 1.7;
                if (cap < pad) pad = cap;
                c1 = (double)c0 + pad;
            } else if (e > firsterr) {
                lp.feed((double)(c0 - 8), c1 + 4.0);
                c0 = e;
                c1 = (double)e;
            }
        }
        if (started) lp.feed((double)c0, c1);
        lp.finish();
    }
    counts[2 * blockIdx.x] = em.over ? -1 : em.n;
}

cudaError_t launch_dropouts(const DropField* fields, int nfields, const DropConsts& k, int* errs, int* drops,
                            int* counts, double* rfstd, cudaStream_t stream) {
    if (nfields <= 0) return cudaSuccess;
    dropout_kernel<<<nfields, kThreads, 0, stream>>>(fields, k, errs, drops, counts, rfstd);
    return cudaGetLastError();
}

}  // namespace ldg
