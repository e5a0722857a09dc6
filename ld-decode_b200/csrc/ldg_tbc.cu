// Time-base correction: resample demodulated fields onto the 4fsc output
// grid (restates Field.computewow_scaled, lddecode/core.py:2591-2623,
// scale_field, lddecode/utils.py:127-183, and hz_to_output_array,
// lddecode/utils.py:1061-1075).
//
// Two kernels per batch of fields:
//   wow_levels_kernel  one CTA per field: the per-line-segment wow factors
//                      (slopes of the expected->actual line-location spline),
//                      their pixel-weighted median and 15*MAD outlier rule ->
//                      one level-adjust factor per segment.
//   tbc_gather_kernel  one thread per output pixel: FP64 spline coordinate,
//                      optional float32 rounding (the reference's own cast),
//                      16-tap windowed-sinc gather with linear interpolation
//                      between LUT phases, level adjust, uint16 conversion.
#include "ldg_tbc.cuh"

namespace ldg {

namespace {

constexpr int kWowThreads = 512;
constexpr int kMaxSeg = kWowThreads;  // segments (lines - 1) per field handled

// The spline segment of output pixel i: j with j*inl <= x < (j+1)*inl,
// x = i * outscale, clamped to [0, nseg-1] (a degree-1 B-spline's interval).
__device__ __forceinline__ int segment_of(double x, double inl, int nseg) {
    int j = (int)floor(x / inl);
    if ((double)j * inl > x) --j;
    if ((double)(j + 1) * inl <= x) ++j;
    return min(max(j, 0), nseg - 1);
}

__device__ __forceinline__ long long first_pixel_at(double xk, double outscale) {
    // smallest i >= 0 with i * outscale >= xk (same FP product as the gather)
    long long i = (long long)ceil(xk / outscale);
    if (i < 0) i = 0;
    while (i > 0 && __dmul_rn((double)(i - 1), outscale) >= xk) --i;
    while (__dmul_rn((double)i, outscale) < xk) ++i;
    return i;
}

// Bitonic sort of (key, weight) pairs, ascending by key, n = kWowThreads.
__device__ void bitonic_sort(double* key, long long* wt) {
    const int t = threadIdx.x;
    for (int k = 2; k <= kWowThreads; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            const int ixj = t ^ j;
            if (ixj > t) {
                const bool up = (t & k) == 0;
                const double a = key[t], b = key[ixj];
                if ((a > b) == up) {
                    key[t] = b;
                    key[ixj] = a;
                    const long long w = wt[t];
                    wt[t] = wt[ixj];
                    wt[ixj] = w;
                }
            }
            __syncthreads();
        }
    }
}

// Weighted median (numpy convention: mean of the two middle elements for an
// even count) of the sorted (key, wt) list, total count n.
__device__ double weighted_median(const double* key, const long long* wt, long long* csum,
                                  long long n) {
    __shared__ double res[2];
    // inclusive prefix sum (serial over <= 512 entries by one thread: cheap)
    if (threadIdx.x == 0) {
        long long acc = 0;
        for (int i = 0; i < kWowThreads; ++i) {
            acc += wt[i];
            csum[i] = acc;
        }
        const long long r1 = (n & 1) ? n / 2 : n / 2 - 1;
        const long long r2 = n / 2;
        double v1 = 0, v2 = 0;
        for (int i = 0; i < kWowThreads; ++i) {
            if (wt[i] == 0) continue;
            const long long lo = csum[i] - wt[i];
            if (r1 >= lo && r1 < csum[i]) v1 = key[i];
            if (r2 >= lo && r2 < csum[i]) v2 = key[i];
        }
        res[0] = (n & 1) ? v2 : (v1 + v2) / 2;
    }
    __syncthreads();
    const double r = res[0];
    __syncthreads();
    return r;
}

}  // namespace

__global__ void __launch_bounds__(kWowThreads) wow_levels_kernel(const TbcField* fields,
                                                                 double threshold_mult) {
    const TbcField& f = fields[blockIdx.x];
    __shared__ double key[kWowThreads];
    __shared__ long long wt[kWowThreads];
    __shared__ long long csum[kWowThreads];
    __shared__ double slope_s[kMaxSeg];
    const int nseg = f.nlines - 1;
    const int t = threadIdx.x;
    if (nseg < 1 || nseg > kMaxSeg) {
        if (t == 0) f.status[0] = LDG_TBC_BAD_LINES;
        return;
    }
    const double inl = f.inlinelen;
    double slope = 0.0;
    long long cnt = 0;
    if (t < nseg) {
        const double y0 = f.linelocs[t], y1 = f.linelocs[t + 1];
        const double w = 1.0 / ((double)(t + 1) * inl - (double)t * inl);
        slope = __dadd_rn(__dmul_rn(y0, -w), __dmul_rn(y1, w));
        // pixels of the wow array [0, nwow) falling in this segment
        const long long lo = (t == 0) ? 0 : first_pixel_at((double)t * inl, f.outscale);
        const long long hi = (t == nseg - 1) ? f.nwow : first_pixel_at((double)(t + 1) * inl, f.outscale);
        const long long a = min(lo, f.nwow), b = min(hi, f.nwow);
        cnt = b > a ? b - a : 0;
        slope_s[t] = slope;
    }
    key[t] = (t < nseg) ? slope : 1.0e300;
    wt[t] = cnt;
    __syncthreads();
    bitonic_sort(key, wt);
    const double med = weighted_median(key, wt, csum, f.nwow);
    // MAD over the same weighted set
    if (t < nseg) {
        key[t] = fabs(slope_s[t] - med);
        wt[t] = cnt;
    } else {
        key[t] = 1.0e300;
        wt[t] = 0;
    }
    __syncthreads();
    bitonic_sort(key, wt);
    const double mad = weighted_median(key, wt, csum, f.nwow);
    const double thr = mad > 0 ? threshold_mult * mad : 0.001;
    if (t < nseg) {
        const double s = slope_s[t];
        f.seg_level[t] = (fabs(s - med) > thr) ? med : s;
    }
}

__global__ void __launch_bounds__(256) tbc_gather_kernel(const TbcField* fields, const float* lut,
                                                         int nfields) {
    const int fi = blockIdx.y;
    if (fi >= nfields) return;
    const TbcField& f = fields[fi];
    const long long nout = (long long)f.linesout * f.outwidth;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nout) return;
    const long long ig = i + (long long)f.outwidth * (f.lineoffset + 1);
    const double inl = f.inlinelen;
    const int nseg = f.nlines - 1;
    const double x = __dmul_rn((double)ig, f.outscale);
    const int j = segment_of(x, inl, nseg);
    const double x0 = (double)j * inl, x1 = (double)(j + 1) * inl;
    const double y0 = f.linelocs[j], y1 = f.linelocs[j + 1];
    const double w = 1.0 / (x1 - x0);
    double c = __dadd_rn(__dmul_rn(y0, __dmul_rn(w, x1 - x)), __dmul_rn(y1, __dmul_rn(w, x - x0)));
    if (f.coord_f32) c = (double)__double2float_rn(c);
    const long long ci = (long long)c;
    const double ph = __dmul_rn(c - (double)ci, 65536.0);
    const int ps = (int)ph;
    const float alpha = __double2float_rn(ph - (double)ps);
    const float* w0 = lut + (size_t)ps * 16;
    const float* w1 = w0 + 16;
    const long long start = ci - 7;
    double acc = 0.0;
    if (start >= 0 && start + 16 <= f.buf_len && ps >= 0 && ps < 65536) {
#pragma unroll
        for (int t = 0; t < 16; ++t) {
            const float ws = __ldg(w0 + t);
            const float wt = fmaf(alpha, __ldg(w1 + t) - ws, ws);
            acc += (double)(__ldg(f.buf + start + t) * wt);
        }
    } else if (f.status) {
        atomicOr(f.status, LDG_TBC_OUT_OF_RANGE);
    }
    const float out = (float)(f.seg_level[j] * acc);
    if (f.out_f32) f.out_f32[i] = out;
    if (f.out_u16) {
        double v = (double)out * f.u16_scale + f.u16_offset + 0.5;
        v = fmin(fmax(v, 0.0), 65535.0);
        f.out_u16[i] = (uint16_t)(unsigned)v;
    }
}

cudaError_t launch_tbc(const TbcField* dfields, int nfields, long long max_nout, const float* lut,
                       double threshold_mult, cudaStream_t stream) {
    if (nfields <= 0) return cudaSuccess;
    wow_levels_kernel<<<nfields, kWowThreads, 0, stream>>>(dfields, threshold_mult);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    dim3 grid((unsigned)((max_nout + 255) / 256), (unsigned)nfields);
    tbc_gather_kernel<<<grid, 256, 0, stream>>>(dfields, lut, nfields);
    return cudaGetLastError();
}

}  // namespace ldg
