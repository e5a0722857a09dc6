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
//   wow_spline_kernel  (quadratic / cubic wow interpolation only) one CTA per
//                      field: the spline's pieces, the exact median and MAD
//                      of the per-pixel wow factors by radix selection, and
//                      with level smoothing the IIR's state every 32 pixels.
//   tbc_gather_kernel  one thread per output pixels: FP64 spline coordinate,
//                      optional float32 rounding (the reference's own cast),
//                      16-tap windowed-sinc gather with linear interpolation
//                      between LUT phases, level adjust, uint16 conversion.
#include <climits>

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
    if (f.spline_k >= 2) return;  // wow_spline_kernel's field
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


// ---- quadratic / cubic wow interpolation (core.py:2602-2621) --------------
//
// The reference builds scipy's make_interp_spline through the points
// (i * inlinelen, linelocs[i]): k = 2 with scipy's default knots for even
// degree (the data points' midpoints, the first and last omitted), k = 3
// with natural end conditions (knots at the data points, s'' = 0 at both
// ends).  Here each spline is built directly as piecewise polynomials:
//   cubic      the classic second-derivative form, one tridiagonal system
//              for M_1 .. M_{n-2} (M_0 = M_{n-1} = 0);
//   quadratic  the derivative s' is piecewise linear and continuous over the
//              breakpoints x_0, (x_j + x_{j+1})/2 for j = 1 .. n-3, x_{n-1};
//              its values D_0 .. D_{n-2} at the breakpoints solve one
//              tridiagonal system whose row i states that the integral of s'
//              over [x_i, x_{i+1}] is y_{i+1} - y_i (the trapezoid rule is
//              exact for the linear pieces of s').
// Both systems are diagonally dominant and solved by the Thomas algorithm in
// FP64.  Outside the data range the first and last pieces extend, as scipy's
// BSpline extrapolates.

constexpr int kSplThreads = 1024;
constexpr int kSplMaxLines = 513;
constexpr int kHistBins = 2048;

// Coordinate and wow factor at x from a field's piece table pc (kSplStride
// doubles per piece: left edge, anchor, c0..c3; value c0 + c1 t + c2 t^2 +
// c3 t^3 at t = x - anchor).  The piece is guessed from x / inlinelen (shift
// 0: cubic pieces start at data points; 0.5: quadratic ones at midpoints)
// and fixed by exact comparisons with the left edges.  Every operation is
// an explicitly rounded intrinsic so that the statistics kernel and the
// gather get the same values.
__device__ __forceinline__ void spline_eval(const double* pc, int np, double x, double inv_inl, double shift,
                                            double& coord, double& wow) {
    int p = (int)floor(__dadd_rn(__dmul_rn(x, inv_inl), -shift));
    p = min(max(p, 0), np - 1);
    while (p > 0 && x < pc[p * kSplStride]) --p;
    while (p + 1 < np && x >= pc[(p + 1) * kSplStride]) ++p;
    const double* c = pc + p * kSplStride;
    const double t = __dadd_rn(x, -c[1]);
    coord = __fma_rn(t, __fma_rn(t, __fma_rn(t, c[5], c[4]), c[3]), c[2]);
    wow = __fma_rn(t, __fma_rn(t, __dmul_rn(3.0, c[5]), __dmul_rn(2.0, c[4])), c[3]);
}

// Order-preserving map of a double onto an unsigned 64-bit key.
__device__ __forceinline__ unsigned long long order_key(double v) {
    const unsigned long long u = (unsigned long long)__double_as_longlong(v);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}

__device__ __forceinline__ double key_value(unsigned long long k) {
    const unsigned long long u = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double((long long)u);
}

// The wow factors of pixels i0 .. i1-1 in order (one thread's chunk):
// body(i, wow).  The pixel position i * outscale comes from an exact double
// counter, the piece advances when the position passes the next piece's
// left edge (positions only grow), and the current piece's coefficients
// stay in registers -- the same position, piece and rounded operations as
// spline_eval, so the same wow factor as the gather's, at a fraction of the
// instructions of a search per pixel.
struct WowWalk {
    const double* pc;
    int np;
    double outscale, inv_inl, shift;
    template <class Body>
    __device__ __forceinline__ void operator()(long long i0, long long i1, Body body) const {
        if (i0 >= i1) return;
        double xi = (double)i0;
        double x = __dmul_rn(xi, outscale);
        int p = (int)floor(__dadd_rn(__dmul_rn(x, inv_inl), -shift));
        p = min(max(p, 0), np - 1);
        while (p > 0 && x < pc[p * kSplStride]) --p;
        while (p + 1 < np && x >= pc[(p + 1) * kSplStride]) ++p;
        double next, anc, c3, c4x2, c5x3;
        auto load = [&]() {
            const double* c = pc + p * kSplStride;
            next = p + 1 < np ? pc[(p + 1) * kSplStride] : INFINITY;
            anc = c[1];
            c3 = c[3];
            c4x2 = __dmul_rn(2.0, c[4]);
            c5x3 = __dmul_rn(3.0, c[5]);
        };
        load();
        for (long long i = i0; i < i1; ++i) {
            if (x >= next) {
                while (p + 1 < np && x >= pc[(p + 1) * kSplStride]) ++p;
                load();
            }
            const double t = __dadd_rn(x, -anc);
            body(i, __fma_rn(t, __fma_rn(t, c5x3, c4x2), c3));
            xi = __dadd_rn(xi, 1.0);
            x = __dmul_rn(xi, outscale);
        }
    }
};

constexpr int kCollect = kHistBins / 2;  // keys ranked in shared memory (the histogram's space)

struct SelectShared {
    unsigned warp_sum[32];
    unsigned long long prefix;  // key bits fixed so far
    long long krem;             // wanted rank among the keys that share them
    long long below;            // keys below that set
    unsigned eq;                // keys sharing the prefix (after the last pass: equal to the result)
    unsigned long long wmin[32];
    int ncoll, has_next;        // collected keys; the next key in rank order was among them
    long long cless;            // collected keys below the result
    unsigned long long next;    // that next key
};

// k-th smallest (0-based) of key(i), i in [0, n): most-significant-digit
// radix selection in up to six passes (digits of 11, 11, 11, 11, 11 and 9
// bits) over a shared histogram; the keys are recomputed on every pass.
// Once at most kCollect keys share the digits found so far, one more pass
// collects them into shared memory and the result is found among them by
// exact ranking (each thread counts the keys below and equal to its own),
// which also gives the next key in rank order when it is among them.  Each
// thread walks its own contiguous chunk of pixels and adds runs of equal
// digits at once; the 32 lanes of a warp look at pixels ~n/1024 apart,
// whose digits mostly differ where the runs are short.  On
// return sh.prefix is the key, sh.below the number of keys below it, sh.eq
// the number equal to it.
template <class Visit>
__device__ void radix_select(Visit visit, long long n, long long k, unsigned* hist, SelectShared& sh) {
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    if (t == 0) {
        sh.prefix = 0;
        sh.krem = k;
        sh.below = 0;
        sh.eq = 0;
        sh.has_next = 0;
    }
    unsigned long long mask = 0;
    const long long chunk = (n + kSplThreads - 1) / kSplThreads;
    const long long i0 = (long long)t * chunk, i1 = min(n, i0 + chunk);
    for (int pass = 0; pass < 6; ++pass) {
        const int shift = pass < 5 ? 53 - 11 * pass : 0;
        const unsigned dmask = pass < 5 ? 0x7ffu : 0x1ffu;
        for (int b = t; b < kHistBins; b += kSplThreads) hist[b] = 0;
        __syncthreads();
        const unsigned long long prefix = sh.prefix;
        // runs of one digit (the rule in the high passes, where a whole
        // chunk shares its sign and exponent) are counted in a register
        unsigned run_d = 0xffffffffu, run_n = 0;
        visit(i0, i1, [&](long long, unsigned long long kk) {
            if ((kk & mask) != prefix) return;
            const unsigned d = (unsigned)(kk >> shift) & dmask;
            if (d != run_d) {
                if (run_n) atomicAdd(&hist[run_d], run_n);
                run_d = d;
                run_n = 0;
            }
            ++run_n;
        });
        if (run_n) atomicAdd(&hist[run_d], run_n);
        __syncthreads();
        // the bin holding rank krem: block scan over bin pairs
        const unsigned h0 = hist[2 * t], h1 = hist[2 * t + 1];
        const unsigned s = h0 + h1;
        unsigned incl = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) sh.warp_sum[w] = incl;
        __syncthreads();
        if (w == 0) {
            unsigned y = sh.warp_sum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned z = __shfl_up_sync(0xffffffffu, y, o);
                if (lane >= o) y += z;
            }
            sh.warp_sum[lane] = y;
        }
        __syncthreads();
        const long long excl = (long long)(incl - s) + (w ? (long long)sh.warp_sum[w - 1] : 0);
        const long long kr = sh.krem;
        __syncthreads();
        if (s > 0 && kr >= excl && kr < excl + s) {
            const bool first = kr < excl + h0;
            const long long bel = excl + (first ? 0 : h0);
            sh.prefix = prefix | ((unsigned long long)(2 * t + (first ? 0 : 1)) << shift);
            sh.krem = kr - bel;
            sh.below += bel;
            sh.eq = first ? h0 : h1;
        }
        mask |= (unsigned long long)dmask << shift;
        __syncthreads();
        if (pass < 5 && sh.eq <= (unsigned)kCollect) {  // uniform: a shared value after a barrier
            unsigned long long* coll = reinterpret_cast<unsigned long long*>(hist);
            const unsigned long long pre = sh.prefix;
            if (t == 0) sh.ncoll = 0;
            __syncthreads();
            visit(i0, i1, [&](long long, unsigned long long kk) {
                if ((kk & mask) == pre) {
                    const int pos = atomicAdd(&sh.ncoll, 1);
                    if (pos < kCollect) coll[pos] = kk;
                }
            });
            __syncthreads();
            const int nc = min(sh.ncoll, kCollect);
            const long long kr = sh.krem;
            __syncthreads();
            if (t < nc) {
                const unsigned long long mine = coll[t];
                int less = 0, same = 0;
                for (int q = 0; q < nc; ++q) {
                    const unsigned long long o = coll[q];
                    less += o < mine;
                    same += o == mine;
                }
                // threads holding equal keys store equal values
                if (less <= kr && kr < less + same) {
                    sh.prefix = mine;
                    sh.cless = less;
                    sh.eq = (unsigned)same;
                }
                if (kr + 1 < nc && less <= kr + 1 && kr + 1 < less + same) {
                    sh.next = mine;
                    sh.has_next = 1;
                }
            }
            __syncthreads();
            if (t == 0) sh.below += sh.cless;
            __syncthreads();
            return;
        }
    }
}

// Smallest key(i) above `above` (all ones when there is none).
template <class Visit>
__device__ unsigned long long min_key_above(Visit visit, long long n, unsigned long long above, SelectShared& sh) {
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    unsigned long long m = ~0ull;
    const long long chunk = (n + kSplThreads - 1) / kSplThreads;
    visit((long long)t * chunk, min(n, (long long)t * chunk + chunk), [&](long long, unsigned long long kk) {
        if (kk > above && kk < m) m = kk;
    });
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long y = __shfl_xor_sync(0xffffffffu, m, o);
        m = y < m ? y : m;
    }
    if (lane == 0) sh.wmin[w] = m;
    __syncthreads();
    m = sh.wmin[lane];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long y = __shfl_xor_sync(0xffffffffu, m, o);
        m = y < m ? y : m;
    }
    __syncthreads();
    return m;
}

// numpy median of key(i), i in [0, n): the middle value, or the mean of the
// two middle values for even n.
template <class Visit>
__device__ double select_median(Visit visit, long long n, unsigned* hist, SelectShared& sh) {
    const long long r1 = (n & 1) ? n / 2 : n / 2 - 1;
    radix_select(visit, n, r1, hist, sh);
    const unsigned long long k1 = sh.prefix;
    const long long upto = sh.below + sh.eq;  // keys <= k1
    const bool has_next = sh.has_next != 0;
    const unsigned long long kn = sh.next;
    __syncthreads();
    const double v1 = key_value(k1);
    if (n & 1) return v1;
    const double v2 = has_next ? key_value(kn) : (upto >= r1 + 2 ? v1 : key_value(min_key_above(visit, n, k1, sh)));
    return __dadd_rn(v1, v2) / 2;
}

// One CTA per spline field.  Thread 0 solves the tridiagonal system, the
// pieces are built in parallel (shared table and the field's scratch copy),
// then the median and MAD of the wow factors over the whole wow array [0,
// nwow) are selected exactly, and with level smoothing the IIR runs as a
// scan of affine maps over 1024 contiguous chunks (each chunk's map from one
// pass, the chunks' start values by a block scan, then a second pass that
// records the level just before every 32nd output pixel for the gather).
__global__ void __launch_bounds__(kSplThreads) wow_spline_kernel(const TbcField* fields, double threshold_mult) {
    const TbcField& f = fields[blockIdx.x];
    if (f.spline_k < 2) return;
    __shared__ double pc[kSplStride * kSplMaxLines];
    __shared__ double cp[kSplMaxLines], dp[kSplMaxLines];
    __shared__ unsigned long long hist_mem[kHistBins / 2];  // 8-byte aligned: also the collected keys
    unsigned* hist = reinterpret_cast<unsigned*>(hist_mem);
    __shared__ SelectShared sh;
    __shared__ double wmapA[32], wmapB[32], wy[32];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int n = f.nlines;
    const bool cubic = f.spline_k == 3;
    if (n < 4 || n > kSplMaxLines) {
        if (t == 0) f.status[0] = LDG_TBC_BAD_LINES;
        return;
    }
    const double inl = f.inlinelen;
    const double* y = f.linelocs;
    auto X = [&](int i) { return (double)i * inl; };
    // quadratic breakpoints
    auto BK = [&](int j) {
        return j == 0 ? X(0) : (j == n - 2 ? X(n - 1) : __dmul_rn(__dadd_rn(X(j), X(j + 1)), 0.5));
    };
    if (t == 0) {
        const int m = n - 2 + (cubic ? 0 : 1);  // unknowns
        for (int r = 0; r < m; ++r) {
            double a = 0, b = 0, c = 0, d = 0;
            if (cubic) {
                const int i = r + 1;
                const double h0 = X(i) - X(i - 1), h1 = X(i + 1) - X(i);
                a = h0;
                b = 2.0 * (h0 + h1);
                c = h1;
                d = 6.0 * ((y[i + 1] - y[i]) / h1 - (y[i] - y[i - 1]) / h0);
            } else {
                // integral of s' over [x_r, x_{r+1}], split at breakpoint r when it lies inside
                auto add = [&](double p, double q, int j, double& cj, double& cj1) {
                    const double b0 = BK(j), wj = BK(j + 1) - b0;
                    const double rp = (p - b0) / wj, rq = (q - b0) / wj;
                    const double hw = (q - p) / 2;
                    cj += hw * ((1.0 - rp) + (1.0 - rq));
                    cj1 += hw * (rp + rq);
                };
                if (r == 0) {
                    add(X(0), X(1), 0, b, c);
                } else if (r == n - 2) {
                    add(X(n - 2), X(n - 1), n - 3, a, b);
                } else {
                    add(X(r), BK(r), r - 1, a, b);
                    add(BK(r), X(r + 1), r, b, c);
                }
                d = y[r + 1] - y[r];
            }
            if (r == 0) {
                cp[0] = c / b;
                dp[0] = d / b;
            } else {
                const double den = b - a * cp[r - 1];
                cp[r] = c / den;
                dp[r] = (d - a * dp[r - 1]) / den;
            }
        }
        for (int r = m - 2; r >= 0; --r) dp[r] = dp[r] - cp[r] * dp[r + 1];
    }
    __syncthreads();
    const int np = f.npieces;
    for (int p = t; p < np; p += kSplThreads) {
        double e[kSplStride];
        if (cubic) {
            auto M = [&](int i) { return (i == 0 || i == n - 1) ? 0.0 : dp[i - 1]; };
            const double h = X(p + 1) - X(p);
            const double m0 = M(p), m1 = M(p + 1);
            e[0] = X(p);
            e[1] = X(p);
            e[2] = y[p];
            e[3] = (y[p + 1] - y[p]) / h - h * (2.0 * m0 + m1) / 6.0;
            e[4] = m0 / 2.0;
            e[5] = (m1 - m0) / (6.0 * h);
        } else {
            const double left = BK(p), wp = BK(p + 1) - left;
            const int a = p == 0 ? 0 : (p == n - 3 ? n - 1 : p + 1);
            const double dd = dp[p + 1] - dp[p];
            e[0] = left;
            e[1] = X(a);
            e[2] = y[a];
            e[3] = dp[p] + dd * (X(a) - left) / wp;
            e[4] = dd / (2.0 * wp);
            e[5] = 0.0;
        }
#pragma unroll
        for (int q = 0; q < kSplStride; ++q) {
            pc[p * kSplStride + q] = e[q];
            f.spl[p * kSplStride + q] = e[q];
        }
    }
    __syncthreads();
    const long long L = f.nwow;
    const double shift = cubic ? 0.0 : 0.5;
    const double outscale = f.outscale, inv_inl = f.inv_inl;
    const WowWalk walk{pc, np, outscale, inv_inl, shift};
    const double med = select_median(
        [&](long long a0, long long a1, auto body) {
            walk(a0, a1, [&](long long i, double w) { body(i, order_key(w)); });
        },
        L, hist, sh);
    const double mad = select_median(
        [&](long long a0, long long a1, auto body) {
            walk(a0, a1, [&](long long i, double w) { body(i, order_key(fabs(__dadd_rn(w, -med)))); });
        },
        L, hist, sh);
    const double thr = mad > 0 ? threshold_mult * mad : 0.001;
    if (t == 0) {
        f.stat[0] = med;
        f.stat[1] = thr;
    }
    if (!(f.smooth_b > 0)) return;
    auto level = [&](double wv) { return fabs(__dadd_rn(wv, -med)) > thr ? med : wv; };
    // level-adjust IIR (utils.py:141-149): y[0] = la[0], y[i] = a la[i] + b y[i-1]
    const double a = f.smooth_a, b = f.smooth_b;
    const long long C = (L + kSplThreads - 1) / kSplThreads;
    const long long i0 = (long long)t * C, i1 = min(L, i0 + C);
    double A = 1.0, B = 0.0;  // this chunk as y_out = A y_in + B
    walk(i0, i1, [&](long long i, double wv) {
        const double la = level(wv);
        if (i == 0) {
            A = 0.0;
            B = la;
        } else {
            A = __dmul_rn(b, A);
            B = __dadd_rn(__dmul_rn(a, la), __dmul_rn(b, B));
        }
    });
    // inclusive scan of the maps over the warp, then over the warps
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double Ap = __shfl_up_sync(0xffffffffu, A, o), Bp = __shfl_up_sync(0xffffffffu, B, o);
        if (lane >= o) {
            B = __fma_rn(A, Bp, B);
            A = __dmul_rn(A, Ap);
        }
    }
    if (lane == 31) {
        wmapA[w] = A;
        wmapB[w] = B;
    }
    __syncthreads();
    if (t == 0) {
        double yy = 0.0;
        for (int q = 0; q < 32; ++q) {
            wy[q] = yy;
            yy = __fma_rn(wmapA[q], yy, wmapB[q]);
        }
    }
    __syncthreads();
    const double Ae = __shfl_up_sync(0xffffffffu, A, 1), Be = __shfl_up_sync(0xffffffffu, B, 1);
    double yv = lane == 0 ? wy[w] : __fma_rn(Ae, wy[w], Be);
    // second pass: record y just before output pixel 32*m (wow index igbase + 32*m)
    const long long igbase = (long long)f.outwidth * (f.lineoffset + 1);
    const long long nout = (long long)f.linesout * f.outwidth;
    const long long nyb = (nout + 31) / 32;
    long long mq = (i0 + 1 - igbase + 31) / 32;
    if (i0 + 1 - igbase <= 0) mq = 0;
    walk(i0, i1, [&](long long i, double wv) {
        const double la = level(wv);
        yv = i == 0 ? la : __dadd_rn(__dmul_rn(a, la), __dmul_rn(b, yv));
        if (mq < nyb && i + 1 == igbase + 32 * mq) {
            f.ybefore[mq] = yv;
            ++mq;
        }
    });
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
// 8 lanes gather one pixel at a time (at step p group g takes pixel 4p + g,
// so a step's four pixels are adjacent): lane k of a group reads taps 2k, 2k+1
// of the input and one float4 of the interleaved LUT (the two taps of phase
// ps and their differences to phase ps + 1), so a pixel's 64-byte input
// span and its 128 bytes of LUT are each one contiguous access; the 8
// partial sums meet in a transposing reduction (lane k of group g ends with
// pixel 4k + g) and one shuffle takes each pixel's sum to its own lane.
// One lane's share of a pixel: taps 2k and 2k+1 of the 16 starting at
// buf[st], weights from LUT phase ps (the interleaved float4 of w and the
// next-phase difference) at fraction alpha; float32 products, FP64 sum.
__device__ __forceinline__ double two_taps(const float* buf, const float* lut, int st, int ps, float alpha, int k) {
    const float4 q = __ldg(reinterpret_cast<const float4*>(lut + (size_t)ps * 32) + k);
    const float* in = buf + st + 2 * k;
    const float x0 = __ldg(in), x1 = __ldg(in + 1);
    const float w0 = fmaf(alpha, q.z, q.x), w1 = fmaf(alpha, q.w, q.y);
    return (double)(x0 * w0) + (double)(x1 * w1);
}

// Sum over a group's 8 lanes of their shares of the group's 8 pixels
// (share(p): this lane's share of pixel p), as a transposing reduction: at
// each level a lane keeps half of its pixels and adds the partner's shares
// of them, so lane k ends with the whole sum of pixel k.  The shares are
// formed in the order the reduction consumes them (pixels j and j + 4, for
// j = 0, 2, 1, 3), so at most two partial sums are live beside them.
template <class S>
__device__ __forceinline__ double group_sum(int k, S&& share) {
    const bool h4 = (k & 4) != 0, h2 = (k & 2) != 0, h1 = (k & 1) != 0;
    double b2[2];
#pragma unroll
    for (int jj = 0; jj < 2; ++jj) {
        double b4[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int j = jj + 2 * h;
            const double a = share(j), c = share(j + 4);
            b4[h] = (h4 ? c : a) + __shfl_xor_sync(0xffffffffu, h4 ? a : c, 4);
        }
        b2[jj] = (h2 ? b4[1] : b4[0]) + __shfl_xor_sync(0xffffffffu, h2 ? b4[0] : b4[1], 2);
    }
    return (h1 ? b2[1] : b2[0]) + __shfl_xor_sync(0xffffffffu, h1 ? b2[0] : b2[1], 1);
}

// The group sum with each pixel's first tap and phase in separate shuffles
// (phase -1: a pixel left at 0), for warps whose first taps do not fit
// 16-bit offsets.
__device__ __noinline__ double gather_unpacked(const float* buf, const float* lut, int sti, int psi, float alpha,
                                               int grp, int k) {
    return group_sum(k, [&](int p) {
        const int src = 4 * p + grp;
        const int pst = __shfl_sync(0xffffffffu, sti, src);
        const int pps = __shfl_sync(0xffffffffu, psi, src);
        const float pal = __shfl_sync(0xffffffffu, alpha, src);
        return pps >= 0 ? two_taps(buf, lut, pst, pps, pal, k) : 0.0;
    });
}

__global__ void __launch_bounds__(kGatherThreads, 8) tbc_gather_kernel(const TbcField* fields, const float* lut,
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
    int jj = 0;
    double cc, wv = 0.0;
    if (f.spline_k >= 2) {
        const double x = __dmul_rn((double)(igbase + (i < nout ? i : 0)), f.outscale);
        spline_eval(f.spl, f.npieces, x, f.inv_inl, f.spline_k == 2 ? 0.5 : 0.0, cc, wv);
        if (f.coord_f32) cc = (double)__double2float_rn(cc);
    } else {
        cc = pixel_coord(f, igbase + (i < nout ? i : 0), nseg, jj);
    }
    const long long ci = (long long)cc;
    const double ph = __dmul_rn(cc - (double)ci, 65536.0);
    const int ps = (int)ph;
    const float alpha = __double2float_rn(ph - (double)ps);
    const long long st = ci - 7;
    const bool ok = i < nout && st >= 0 && st + 16 <= f.buf_len && ps >= 0 && ps < 65536;
    if (i < nout && !ok && f.status) atomicOr(f.status, LDG_TBC_OUT_OF_RANGE);
    // first tap as a 32-bit offset (buf_len < 2^31); phase -1 marks a pixel left at 0
    const int sti = ok ? (int)st : 0;
    const int psi = ok ? ps : -1;
    // The 32 pixels' first taps lie within a few hundred samples of each
    // other: as offsets from the warp's lowest one they fit 16 bits, and
    // each pixel's offset and phase travel in one shuffle instead of two
    // (the shuffles share the load pipe's writeback with the tap loads).
    // 0xffff as the offset marks a pixel left at 0.
    const int low = __reduce_min_sync(0xffffffffu, ok ? sti : INT_MAX);
    const bool packed = __all_sync(0xffffffffu, !ok || sti - low < 0xffff);
    const unsigned pk = ok ? ((unsigned)(sti - low) << 16) | (unsigned)ps : 0xffff0000u;
    double held;  // after the group sum: the whole sum of pixel 4 k + grp
    if (packed) {
        held = group_sum(k, [&](int p) {
            // the group's p-th pixel: at each step the four groups take four
            // adjacent pixels, whose 16-tap windows overlap (fewer cache lines
            // per tap load)
            const int src = 4 * p + grp;
            const unsigned q = __shfl_sync(0xffffffffu, pk, src);
            const float pal = __shfl_sync(0xffffffffu, alpha, src);
            return (q >> 16) != 0xffffu ? two_taps(f.buf, lut, low + (int)(q >> 16), (int)(q & 0xffffu), pal, k)
                                        : 0.0;
        });
    } else {
        // first taps too far apart for 16-bit offsets (wild line locations): rare
        held = gather_unpacked(f.buf, lut, sti, psi, alpha, grp, k);
    }
    // pixel `lane` is at lane 8 (lane % 4) + lane / 4
    const double mine = __shfl_sync(0xffffffffu, held, 8 * (lane & 3) + (lane >> 2));
    double level;
    if (f.spline_k >= 2) {
        const double med = f.stat[0];
        level = fabs(__dadd_rn(wv, -med)) > f.stat[1] ? med : wv;
        if (f.smooth_b > 0) {
            // the IIR over this warp's 32 pixels as a scan of affine maps,
            // started from the level just before the warp's first pixel
            double A = f.smooth_b, B = __dmul_rn(f.smooth_a, level);
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const double Ap = __shfl_up_sync(0xffffffffu, A, o), Bp = __shfl_up_sync(0xffffffffu, B, o);
                if (lane >= o) {
                    B = __fma_rn(A, Bp, B);
                    A = __dmul_rn(A, Ap);
                }
            }
            level = __fma_rn(A, f.ybefore[wbase >> 5], B);
        }
    } else {
        level = 0.0;
    }
    if (i >= nout) return;
    if (f.spline_k < 2) {
        level = f.seg_level[jj];
        if (f.smooth_b > 0) {
            const long long ig = igbase + i;  // index into the wow array
            level = level + (f.seg_start[jj] - level) * pow(f.smooth_b, (double)(ig - f.seg_lo[jj] + 1));
        }
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
                       double threshold_mult, bool any_spline, cudaStream_t stream) {
    if (nfields <= 0) return cudaSuccess;
    wow_levels_kernel<<<nfields, kWowThreads, 0, stream>>>(dfields, threshold_mult);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (any_spline) {
        wow_spline_kernel<<<nfields, kSplThreads, 0, stream>>>(dfields, threshold_mult);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
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
