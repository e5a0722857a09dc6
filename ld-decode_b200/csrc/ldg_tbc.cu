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
//   tbc_gather_kernel  one thread per output pixels: FP64 spline coordinate,
//                      optional float32 rounding (the reference's own cast),
//                      16-tap windowed-sinc gather with linear interpolation
//                      between LUT phases, level adjust, uint16 conversion.
#include "ldg_tbc.cuh"

namespace ldg {

namespace {

constexpr int kWowThreads = 512;
constexpr int kMaxSeg = kWowThreads;  // segments (lines - 1) per field handled

__device__ __forceinline__ long long first_pixel_at(double xk, double outscale) {
    // smallest i >= 0 with i * outscale >= xk (same FP product as the gather)
    long long i = (long long)ceil(xk / outscale);
    if (i < 0) i = 0;
    while (i > 0 && __dmul_rn((double)(i - 1), outscale) >= xk) --i;  // one or two steps
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
// even count) of the sorted (key, wt) list, total count n.  Block-wide
// inclusive scan of the weights (warp shuffles + one shared pass).
__device__ double weighted_median(const double* key, const long long* wt, long long* csum,
                                  long long n) {
    __shared__ long long warp_tot[kWowThreads / 32];
    __shared__ double res[2];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    long long x = wt[t];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    if (w == 0) {
        long long y = lane < kWowThreads / 32 ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long z = __shfl_up_sync(0xffffffffu, y, o);
            if (lane >= o) y += z;
        }
        if (lane < kWowThreads / 32) warp_tot[lane] = y;
    }
    __syncthreads();
    const long long incl = x + (w ? warp_tot[w - 1] : 0);
    csum[t] = incl;
    const long long r1 = (n & 1) ? n / 2 : n / 2 - 1;
    const long long r2 = n / 2;
    const long long lo = incl - wt[t];
    if (wt[t] > 0) {
        if (r1 >= lo && r1 < incl) res[0] = key[t];
        if (r2 >= lo && r2 < incl) res[1] = key[t];
    }
    __syncthreads();
    const double r = (n & 1) ? res[1] : (res[0] + res[1]) / 2;
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
        f.seg_lo[t] = a;
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
    if (f.smooth_b > 0) {
        // level-adjust IIR (utils.py:141-149), y[0] = la[0], y[i] = a la[i] +
        // b y[i-1]: over segment j (constant level c_j) it is c_j + (y_before
        // - c_j) b^(i - lo_j + 1); the value entering each segment is carried
        // from segment to segment by one thread
        __syncthreads();
        if (t == 0) {
            double y = f.seg_level[0];
            for (int j = 0; j < nseg; ++j) {
                const double c = f.seg_level[j];
                f.seg_start[j] = y;
                const long long hi = (j + 1 < nseg) ? f.seg_lo[j + 1] : f.nwow;
                const long long len = hi - f.seg_lo[j];
                if (len > 0) y = c + (y - c) * pow(f.smooth_b, (double)len);
            }
        }
    }
}

constexpr int kGatherThreads = 256;

// Input coordinate (FP64) of output pixel ig, optionally rounded to float32
// as the reference does; the spline segment j is also returned.  The
// segment is found from x * (1/inlinelen) and then fixed by exact
// comparisons with the integer knots; w = 1/(x1 - x0) = 1/inlinelen is
// precomputed with the same rounding.
__device__ __forceinline__ double pixel_coord(const TbcField& f, long long ig, int nseg, int& j) {
    const double inl = f.inlinelen;
    const double x = __dmul_rn((double)ig, f.outscale);
    j = (int)(x * f.inv_inl);
    j = min(max(j, 0), nseg - 1);
    if (j > 0 && (double)j * inl > x) --j;
    if (j < nseg - 1 && (double)(j + 1) * inl <= x) ++j;
    const double x0 = (double)j * inl, x1 = (double)(j + 1) * inl;
    const double y0 = __ldg(f.linelocs + j), y1 = __ldg(f.linelocs + j + 1);
    const double w = f.inv_inl;
    double c = __dadd_rn(__dmul_rn(y0, __dmul_rn(w, x1 - x)), __dmul_rn(y1, __dmul_rn(w, x - x0)));
    if (f.coord_f32) c = (double)__double2float_rn(c);
    return c;
}

// One warp per 32 consecutive output pixels of one field; blockIdx.y is the
// field.  Each lane computes its own pixel's FP64 coordinate; then groups of
// 8 lanes gather one pixel at a time: lane k of a group reads taps 2k, 2k+1
// of the input and of the two LUT rows, so a pixel's 64-byte input span and
// its two 64-byte LUT rows are each one contiguous access (instead of 16
// scattered ones per lane); the 8 partial sums meet by shuffles.
__global__ void __launch_bounds__(kGatherThreads) tbc_gather_kernel(const TbcField* fields, const float* lut,
                                                                    int nfields) {
    const int fi = blockIdx.y;
    if (fi >= nfields) return;
    const TbcField& f = fields[fi];
    const long long nout = (long long)f.linesout * f.outwidth;
    const long long wbase = (long long)blockIdx.x * kGatherThreads + (threadIdx.x & ~31);
    if (wbase >= nout) return;  // whole warps leave together
    const int lane = threadIdx.x & 31, grp = lane >> 3, k = lane & 7;
    const long long i = wbase + lane;
    const int nseg = f.nlines - 1;
    const long long igbase = (long long)f.outwidth * (f.lineoffset + 1);
    int jj;
    const double cc = pixel_coord(f, igbase + (i < nout ? i : 0), nseg, jj);
    const long long ci = (long long)cc;
    const double ph = __dmul_rn(cc - (double)ci, 65536.0);
    const int ps = (int)ph;
    const float alpha = __double2float_rn(ph - (double)ps);
    const long long st = ci - 7;
    const bool ok = i < nout && st >= 0 && st + 16 <= f.buf_len && ps >= 0 && ps < 65536;
    if (i < nout && !ok && f.status) atomicOr(f.status, LDG_TBC_OUT_OF_RANGE);
    double mine = 0.0;
#pragma unroll 2
    for (int p = 0; p < 8; ++p) {
        const int src = grp * 8 + p;  // the group's p-th pixel
        const long long pst = __shfl_sync(0xffffffffu, st, src);
        const int pps = __shfl_sync(0xffffffffu, ps, src);
        const float pal = __shfl_sync(0xffffffffu, alpha, src);
        const bool pok = __shfl_sync(0xffffffffu, ok, src);
        double part = 0.0;
        if (pok) {
            const float2 a = __ldg(reinterpret_cast<const float2*>(lut + (size_t)pps * 16) + k);
            const float2 b = __ldg(reinterpret_cast<const float2*>(lut + (size_t)(pps + 1) * 16) + k);
            const float* in = f.buf + pst + 2 * k;
            const float x0 = __ldg(in), x1 = __ldg(in + 1);
            const float w0 = fmaf(pal, b.x - a.x, a.x), w1 = fmaf(pal, b.y - a.y, a.y);
            part = (double)(x0 * w0) + (double)(x1 * w1);
        }
        part += __shfl_xor_sync(0xffffffffu, part, 1);
        part += __shfl_xor_sync(0xffffffffu, part, 2);
        part += __shfl_xor_sync(0xffffffffu, part, 4);
        if (k == p) mine = part;
    }
    if (i >= nout) return;
    double level = f.seg_level[jj];
    if (f.smooth_b > 0) {
        const long long ig = igbase + i;  // index into the wow array
        level = level + (f.seg_start[jj] - level) * pow(f.smooth_b, (double)(ig - f.seg_lo[jj] + 1));
    }
    const float out = (float)(level * mine);
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
    const long long per_cta = kGatherThreads;
    const unsigned gx = (unsigned)((max_nout + per_cta - 1) / per_cta);
    for (int off = 0; off < nfields; off += 65535) {  // grid.y limit
        const int n = nfields - off < 65535 ? nfields - off : 65535;
        tbc_gather_kernel<<<dim3(gx, (unsigned)n), kGatherThreads, 0, stream>>>(dfields + off, lut, n);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// RF TBC (Field.rf_tbc, lddecode/core.py:2724-2752): each output line l is
// the cubic scaler (utils.py:37-70) over the raw input between linelocs[l]
// and linelocs[l + 1], both moved back by the video delay, rounded half to
// even and stored as int16.  The arithmetic is the reference's FP64
// expression term by term with every product and sum rounded on its own
// (no fused multiply-adds), so the output is bit-identical.  One CTA per
// (line, field).
__global__ void __launch_bounds__(256) rf_tbc_kernel(const RfTbcField* fields) {
    const RfTbcField& f = fields[blockIdx.y];
    const int line = blockIdx.x;
    if (line >= f.nout) return;
    const int l = f.startline + line;
    const double begin = __dsub_rn(f.ll[l], f.delay);
    const double end = __dsub_rn(f.ll[l + 1], f.delay);
    const double sf = __ddiv_rn(__dsub_rn(end, begin), (double)f.linelen);
    int16_t* out = f.out + (long long)line * f.linelen;
    for (int i = threadIdx.x; i < f.linelen; i += blockDim.x) {
        const double coord = __dadd_rn(__dmul_rn((double)i, sf), begin);
        // taps int(coord) - 1 .. int(coord) + 2 inside the read: 1 <= coord < len - 2
        if (!(coord >= 1.0 && coord < (double)(f.len - 2))) {
            atomicOr(f.status, LDG_TBC_OUT_OF_RANGE);
            out[i] = 0;
            continue;
        }
        const long long ic = (long long)coord;
        const long long s = ic - 1;
        const double p0 = f.in[s], p1 = f.in[s + 1], p2 = f.in[s + 2], p3 = f.in[s + 3];
        const double x = __dsub_rn(coord, (double)ic);
        // p1 + 0.5 x (p2 - p0 + x (2 p0 - 5 p1 + 4 p2 - p3 + x (3 (p1 - p2) + p3 - p0)))
        const double c = __dsub_rn(__dadd_rn(__dmul_rn(3.0, __dsub_rn(p1, p2)), p3), p0);
        const double b = __dadd_rn(
            __dsub_rn(__dadd_rn(__dsub_rn(__dmul_rn(2.0, p0), __dmul_rn(5.0, p1)), __dmul_rn(4.0, p2)), p3),
            __dmul_rn(x, c));
        const double a = __dadd_rn(__dsub_rn(p2, p0), __dmul_rn(x, b));
        const double v = __dadd_rn(p1, __dmul_rn(__dmul_rn(0.5, x), a));
        out[i] = (int16_t)(int)rint(v);
    }
}

cudaError_t launch_rf_tbc(const RfTbcField* dfields, int nfields, int max_lines, cudaStream_t stream) {
    if (nfields <= 0 || max_lines <= 0) return cudaSuccess;
    for (int off = 0; off < nfields; off += 65535) {
        const int n = nfields - off < 65535 ? nfields - off : 65535;
        rf_tbc_kernel<<<dim3((unsigned)max_lines, (unsigned)n), 256, 0, stream>>>(dfields + off);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace ldg
