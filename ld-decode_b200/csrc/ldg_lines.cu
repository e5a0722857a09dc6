// Sync-pulse runs and per-line refinement of line locations on the GPU.
//
// ldg_sync_runs: runs of demod_05 at or below the sync threshold over a
// whole capture-wide output array -- the pulses findpulses
// (lddecode/utils.py:1101-1157) finds, for every field read window at once --
// and the mean level inside the long ones (getpulses' VSYNC level check,
// core.py:2242-2322).  Two launches: the edges of every tile counted,
// scanned (decoupled look-back) and written in order by one single-pass
// kernel; then the runs paired and the long runs' interiors averaged, the
// results written straight into the caller's pinned buffers.
//
// ldg_lines_refine: the per-line refinement of Field.process() for all
// fields of a capture (pulse-level line locations from the host chain):
//   lines_hsync_kernel   one CTA per field: refine_linelocs_hsync
//                        (core.py:2483-2551), compute_deriv_error
//                        (2553-2564); NTSC: the colour-burst zero crossings
//                        of compute_line_bursts (2998-3047, clb_findbursts
//                        utils.py:1339-1368) per line; PAL:
//                        refine_linelocs_pilot twice (3054-3093) and
//                        fix_badlines (2566-2589) -> final line locations;
//                        PAL: the burst levels and line 7-19 burst crossings
//                        of determine_field_number (3095-3203).
//   pal_sequence_kernel  PAL, one warp walking the fields in order: the
//                        8-field sequence (field phase IDs).
//   burst_round_kernel   NTSC, one CTA per field, twice, and
//   burst_verify_kernel  one CTA walking the fields in order: the burst
//                        phase of every line starts from the previous
//                        field's phase_adjust_median (compute_burst_offsets,
//                        core.py:3360-3388), two passes of the phase
//                        update, the field's median and its field-1/4 flag;
//                        speculated in parallel, verified in order.
//   burst_apply_kernel   NTSC, one CTA per field: refine_linelocs_burst
//                        (3390-3440), fix_badlines with linelocs2 as backup,
//                        the 117.25-degree subcarrier shift (3493-3495).
// Positions, fits and phases are FP64; samples are the float32 outputs.
#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>

#include "ldg_copy.cuh"
#include "ldg_scan.cuh"
#include "ldgpu.h"

struct ldg_ctx;

namespace ldg {
int lines_fail(int code, const std::string& msg);
int ctx_device(const ldg_ctx* c);
std::mutex& ctx_mutex(ldg_ctx* c);
int ctx_lines_scratch(ldg_ctx* c, size_t need, void** out);
int ctx_host_word(ldg_ctx* c, long long** host, long long** dev);
}  // namespace ldg

namespace {

constexpr int kMaxL = LDG_CHAIN_MAX_LINES;
constexpr int kEdgeTile = 16384;  // samples per sync-run scan tile
constexpr int kEdgeThreads = 256;
constexpr int kLineThreads = 352;   // >= proclines (326 PAL)
constexpr int kBurstLines = 266;    // compute_burst_offsets covers lines 0..265
constexpr int kPilotLines = 323;    // refine_linelocs_pilot covers lines 0..322
constexpr int kZc = 16;             // clb_findbursts' fixed zero-crossing slots
constexpr int kBurstThreads = 288;  // >= kBurstLines, whole warps
constexpr int kHsWin = 512;         // samples of a line's H-sync window in shared memory (40 MSPS needs ~480)

// ---------------------------------------------------------------- sync runs

__device__ __forceinline__ bool below(const float* x, long long i, double thr) { return (double)x[i] <= thr; }

// the below-threshold flags of samples base .. base+3 (bit k: sample
// base+k; none at or past n); a float4 load when the array is 16-byte aligned
__device__ __forceinline__ unsigned four_flags(const float* __restrict__ x, long long n, long long base, double thr,
                                               bool aligned) {
    float v[4];
    if (aligned && base + 3 < n) {
        const float4 q = __ldcs(reinterpret_cast<const float4*>(x + base));
        v[0] = q.x;
        v[1] = q.y;
        v[2] = q.z;
        v[3] = q.w;
    } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] = base + k < n ? x[base + k] : 0.0f;
    }
    unsigned b = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (base + k < n && (double)v[k] <= thr) b |= 1u << k;
    return b;
}

// look-back states of a tile (low two bits of its flag word; the high bits
// hold the call's number, so words of earlier calls never match)
constexpr unsigned long long kTileAgg = 1, kTileIncl = 2;
constexpr int kLookbackSpins = 1 << 20;  // ~0.1-1 s of polling; then the call fails
constexpr int kEdgeSteps = kEdgeTile / (4 * kEdgeThreads);  // coalesced float4 steps per thread
constexpr int kEdgeWords = kEdgeTile / 32;                  // flag words of a tile
constexpr int kWordsPerThread = kEdgeWords / kEdgeThreads;
static_assert(kWordsPerThread == 2, "a thread owns two consecutive flag words");

// Sync-run edges in one pass (single-pass scan with decoupled look-back).
// Each CTA takes the next tile by ticket (so every tile it waits on belongs
// to a CTA that is already running); reads its samples with coalesced
// float4 loads into a shared bitmap of below-threshold flags (bit b of word
// w: sample 32 w + b); each thread then owns two consecutive words (64
// samples), whose edges -- samples whose flag differs from the sample
// before -- it counts; one CTA-wide scan of the counts; the tile's total
// goes to the look-back (warp 0: publish the tile's count, add the counts
// or the inclusive prefix of the tiles before it 32 at a time, publish its
// own inclusive prefix); every thread writes its edges as 2*i + (run start ?
// 1 : 0) in increasing i.  The last tile writes the total.  Each sample is
// read once, and the scan costs one launch instead of three (count, scan of
// the tile counts, write), which matters when it runs beside the
// demodulator and each launch waits for SMs to come free.  A wait that
// outlasts kLookbackSpins sets *err (host-mapped) and takes the missing
// count as 0.
__global__ void __launch_bounds__(kEdgeThreads) edge_pass_kernel(
    const float* __restrict__ x, long long n, double thr, unsigned long long* ticket, unsigned long long base,
    unsigned long long call, unsigned long long* flags, long long* agg, long long* incl, long long ntiles,
    long long* __restrict__ edges, long long cap, long long* __restrict__ total, long long* err) {
    __shared__ unsigned bm[kEdgeWords];
    __shared__ long long s_tile, s_excl;
    __shared__ int warp_tot[kEdgeThreads / 32];
    __shared__ unsigned s_before;  // flag of the sample before the tile
    if (threadIdx.x == 0) s_tile = (long long)(atomicAdd(ticket, 1ull) - base);
    __syncthreads();
    const long long tile = s_tile;
    if (tile < 0 || tile >= ntiles) return;  // more CTAs than tiles: never launched so
    const long long t0 = tile * kEdgeTile;
    const bool aligned = (reinterpret_cast<uintptr_t>(x) & 15) == 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_before = t0 > 0 && t0 - 1 < n && below(x, t0 - 1, thr) ? 1u : 0u;
#pragma unroll 4
    for (int j = 0; j < kEdgeSteps; ++j) {
        const long long b0 = t0 + (long long)j * 4 * kEdgeThreads + 4 * threadIdx.x;
        unsigned f = 0;  // flags of samples b0 .. b0+3 (none past n)
        if (b0 < n) f = four_flags(x, n, b0, thr, aligned);
        // eight lanes' four flags make one word (b0 % 32 == 4 * (lane % 8))
        unsigned v = f << (4 * (lane & 7));
        v |= __shfl_xor_sync(0xffffffffu, v, 1);
        v |= __shfl_xor_sync(0xffffffffu, v, 2);
        v |= __shfl_xor_sync(0xffffffffu, v, 4);
        if ((lane & 7) == 0) bm[j * (kEdgeThreads / 8) + (threadIdx.x >> 3)] = v;
    }
    __syncthreads();
    // this thread's 64 samples: words 2t and 2t+1, and the flag before them
    const int w0 = kWordsPerThread * threadIdx.x;
    const unsigned f0 = bm[w0], f1 = bm[w0 + 1];
    const unsigned pb = w0 ? bm[w0 - 1] >> 31 : s_before;
    const long long s0 = t0 + 32LL * w0;  // first sample of word w0
    unsigned e0 = f0 ^ ((f0 << 1) | pb);
    unsigned e1 = f1 ^ ((f1 << 1) | (f0 >> 31));
    // no edges at or past n (flags there are 0, so a run open at n has no end edge)
    if (s0 + 64 > n) {
        const long long k0 = n - s0, k1 = n - s0 - 32;
        e0 &= k0 <= 0 ? 0u : k0 >= 32 ? 0xffffffffu : (1u << k0) - 1u;
        e1 &= k1 <= 0 ? 0u : k1 >= 32 ? 0xffffffffu : (1u << k1) - 1u;
    }
    const int cnt = __popc(e0) + __popc(e1);
    // CTA-wide exclusive scan of the counts
    int inc = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    int before = 0, tile_count = 0;
#pragma unroll
    for (int w = 0; w < kEdgeThreads / 32; ++w) {
        before += w < warp ? warp_tot[w] : 0;
        tile_count += warp_tot[w];
    }
    if (warp == 0) {
        volatile unsigned long long* vf = flags;
        volatile long long* va = agg;
        volatile long long* vi = incl;
        const long long count = tile_count;
        long long excl = 0;
        if (tile > 0) {
            if (lane == 0) {
                va[tile] = count;
                __threadfence();
                vf[tile] = (call << 2) | kTileAgg;
            }
            // the warp looks back 32 tiles at a time (lane l: tile p - l) and
            // stops at the nearest one whose inclusive prefix is out; tiles
            // before 0 count as an inclusive prefix of 0
            bool timed_out = false;
            for (long long p = tile - 1;; p -= 32) {
                const long long q = p - lane;
                unsigned long long f = (call << 2) | kTileIncl;
                if (q >= 0) {
                    f = vf[q];
                    for (int spins = 0; (f >> 2) != call && spins < kLookbackSpins; ++spins) {
                        __nanosleep(64);
                        f = vf[q];
                    }
                }
                if (__any_sync(0xffffffffu, (f >> 2) != call)) {
                    timed_out = true;
                    break;
                }
                __threadfence();
                const unsigned inc_mask = __ballot_sync(0xffffffffu, (f & 3ull) == kTileIncl);
                const int stop = inc_mask ? __ffs(inc_mask) - 1 : 32;
                long long v = 0;
                if (lane < stop && q >= 0) v = va[q];
                if (lane == stop && q >= 0) v = vi[q];
#pragma unroll
                for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                excl += v;
                if (inc_mask) break;
            }
            if (timed_out && lane == 0) *reinterpret_cast<volatile long long*>(err) = 1;
        }
        if (lane == 0) {
            vi[tile] = excl + count;
            __threadfence();
            vf[tile] = (call << 2) | kTileIncl;
            if (tile == ntiles - 1) *total = excl + count;
            s_excl = excl;
        }
    }
    __syncthreads();
    long long k = s_excl + before + inc - cnt;
    for (unsigned e = e0; e; e &= e - 1) {
        const int b = __ffs(e) - 1;
        if (k < cap) edges[k] = 2 * (s0 + b) + ((f0 >> b) & 1u);
        ++k;
    }
    for (unsigned e = e1; e; e &= e - 1) {
        const int b = __ffs(e) - 1;
        if (k < cap) edges[k] = 2 * (s0 + 32 + b) + ((f1 >> b) & 1u);
        ++k;
    }
}

// Pair edges 2r (start) and 2r+1 (end) into runs, with the interior mean of
// long runs; the run count is total / 2 (an odd total leaves a run open at
// the end), read on the device, and runs beyond `cap` are not written.  A
// warp takes 32 consecutive runs, one per lane, so the outputs -- host-mapped
// pinned memory, read by the host after a stream synchronisation without a
// copy-engine transfer -- are written coalesced; the warp then averages its
// long runs one at a time.  Block 0 writes the edge count to *count_out.
__global__ void run_pair_kernel(const long long* __restrict__ edges, const long long* __restrict__ total,
                                long long cap, const float* __restrict__ x, long long min_long, long long trim_lo,
                                long long trim_hi, long long* rs, long long* rl, double* rm, long long* count_out) {
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    const long long tot = *total;
    const long long nruns = min(tot / 2, cap);
    for (long long r0 = (((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; r0 < nruns;
         r0 += nwarps * 32) {
        const long long r = r0 + lane;
        const bool valid = r < nruns;
        long long s = 0, len = 0;
        if (valid) {
            s = edges[2 * r] >> 1;
            len = (edges[2 * r + 1] >> 1) - s;
        }
        double mean = nan("");
        unsigned longs = __ballot_sync(0xffffffffu, valid && len > min_long);
        while (longs) {
            const int l = __ffs(longs) - 1;
            longs &= longs - 1;
            const long long ls = __shfl_sync(0xffffffffu, s, l), ll = __shfl_sync(0xffffffffu, len, l);
            const long long lo = ls + trim_lo, hi = ls + ll - trim_hi;
            double acc = 0;
            for (long long i = lo + lane; i < hi; i += 32) acc += (double)x[i];
#pragma unroll
            for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == l && hi > lo) mean = acc / (double)(hi - lo);
        }
        if (valid) {
            rs[r] = s;
            rl[r] = len;
            rm[r] = mean;
        }
    }
    if (count_out && blockIdx.x == 0 && threadIdx.x == 0) *count_out = tot;
}

// --------------------------------------------------------- per-line helpers

// calczc (utils.py:812-841) over x[0, n): first crossing of `target` within
// count+1 samples from int(start); edge 0 decides rising/falling from
// x[int(start)].  Comparisons and the interpolation in FP64.
__device__ bool calczc(const float* x, long long n, double start_offset, double target, int edge, double count,
                       double& out) {
    const long long s = (long long)start_offset;
    if (s < 0 || s >= n) return false;
    const long long icount = (long long)(count + 1);
    if (edge == 0) edge = (double)x[s] < target ? 1 : -1;
    const long long end = min(s + icount, n);
    long long loc = -1;
    if (edge == 1) {
        for (long long i = s + 1; i < end; ++i)
            if ((double)x[i - 1] < target && (double)x[i] >= target) {
                loc = i;
                break;
            }
    } else {
        for (long long i = s + 1; i < end; ++i)
            if ((double)x[i - 1] > target && (double)x[i] <= target) {
                loc = i;
                break;
            }
    }
    if (loc < 0) return false;
    const double a = (double)x[loc - 1] - target, b = (double)x[loc] - target;
    const double y = (b - a != 0) ? -a / (-a + b) : 0.0;
    out = (double)(loc - 1) + y;
    return true;
}

// A line's window of a sample array staged in shared memory: x[i] from the
// window when i lies in [base, end), else from global memory.
struct WinView {
    const float* g;
    const float* s;
    long long base, end;
    __device__ __forceinline__ float operator[](long long i) const { return (i >= base && i < end) ? s[i - base] : g[i]; }
};

// np.median of a float32 slice (even length: float32 mean of the middle two)
template <class X>
__device__ double median_f32(const X& x, long long lo, long long hi, long long n) {
    lo = max(lo, 0LL);
    hi = min(hi, n);
    float v[128];
    int m = 0;
    for (long long i = lo; i < hi && m < 128; ++i) {
        const float t = x[i];
        int k = m++;
        while (k > 0 && v[k - 1] > t) {
            v[k] = v[k - 1];
            --k;
        }
        v[k] = t;
    }
    if (m == 0) return nan("");
    if (m & 1) return (double)v[m / 2];
    return (double)((v[m / 2 - 1] + v[m / 2]) * 0.5f);
}

// Warp-cooperative forms (every lane returns the same result).

// calczc with 32 samples tested per step and the first crossing by ballot
template <class X>
__device__ bool warp_calczc(const X& x, long long n, double start_offset, double target, int edge, double count,
                            double& out) {
    const int lane = threadIdx.x & 31;
    const long long s = (long long)start_offset;
    if (s < 0 || s >= n) return false;
    const long long icount = (long long)(count + 1);
    if (edge == 0) edge = (double)x[s] < target ? 1 : -1;
    const long long end = min(s + icount, n);
    for (long long c0 = s + 1; c0 < end; c0 += 32) {
        const long long i = c0 + lane;
        bool hit = false;
        if (i < end) {
            const double a = (double)x[i - 1], b = (double)x[i];
            hit = edge == 1 ? (a < target && b >= target) : (a > target && b <= target);
        }
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (m) {
            const long long loc = c0 + __ffs(m) - 1;
            const double a = (double)x[loc - 1] - target, b = (double)x[loc] - target;
            out = (double)(loc - 1) + ((b - a != 0) ? -a / (-a + b) : 0.0);
            return true;
        }
    }
    return false;
}

template <class X>
__device__ void warp_minmax(const X& x, long long lo, long long hi, long long n, float& mn, float& mx) {
    const int lane = threadIdx.x & 31;
    lo = max(lo, 0LL);
    hi = min(hi, n);
    mn = INFINITY;
    mx = -INFINITY;
    for (long long i = lo + lane; i < hi; i += 32) {
        const float v = x[i];
        mn = fminf(mn, v);
        mx = fmaxf(mx, v);
    }
    for (int o = 16; o; o >>= 1) {
        mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
}

// np.median of a float32 slice of up to 64 samples: the warp sorts them
// (bitonic network over elements e = lane and e = lane + 32, unused ones
// +inf) and reads the middle one or two; longer slices fall back to one
// lane.  The middle values do not depend on how ties are ordered.
template <class X>
__device__ double warp_median_f32(const X& x, long long lo, long long hi, long long n) {
    const int lane = threadIdx.x & 31;
    lo = max(lo, 0LL);
    hi = min(hi, n);
    const int m = (int)max(hi - lo, 0LL);
    if (m == 0) return nan("");
    if (m > 64) {
        double r = 0;
        if (lane == 0) r = median_f32(x, lo, hi, n);
        return __shfl_sync(0xffffffffu, r, 0);
    }
    float v0 = lane < m ? x[lo + lane] : INFINITY;
    float v1 = lane + 32 < m ? x[lo + 32 + lane] : INFINITY;
#pragma unroll
    for (int k = 2; k <= 64; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j == 32) {
                // partners lane and lane + 32 in the same lane; ascending (k = 64)
                const float a = fminf(v0, v1), b = fmaxf(v0, v1);
                v0 = a;
                v1 = b;
            } else {
                const float p0 = __shfl_xor_sync(0xffffffffu, v0, j);
                const float p1 = __shfl_xor_sync(0xffffffffu, v1, j);
                const bool lower = (lane & j) == 0;  // this element is the pair's first
                const bool up0 = (lane & k) == 0, up1 = ((lane + 32) & k) == 0;
                v0 = (lower == up0) ? fminf(v0, p0) : fmaxf(v0, p0);
                v1 = (lower == up1) ? fminf(v1, p1) : fmaxf(v1, p1);
            }
        }
    }
    auto at = [&](int e) {
        const float a = __shfl_sync(0xffffffffu, v0, e & 31);
        const float b = __shfl_sync(0xffffffffu, v1, e & 31);
        return e < 32 ? a : b;
    };
    const float va = at((m - 1) / 2), vb = at(m / 2);
    if (m & 1) return (double)va;
    return (double)((va + vb) * 0.5f);
}

// get_linelen (core.py:1655-1672) with linecount + lineoffset = lc
__device__ double line_len(const double* ll, int line, int lc, double linelen) {
    double length;
    if (line >= lc) length = ll[line] - ll[line - 1];
    else if (line > 0) length = (ll[line + 1] - ll[line - 1]) / 2;
    else length = ll[line + 1] - ll[line];
    return length <= 0 ? linelen : length;
}

// second differences above 4 samples mark both later lines bad
__device__ void deriv_error_block(const double* ll, unsigned char* bad, int nl) {
    const int j = threadIdx.x;
    bool b1 = false;
    if (j + 2 < nl) b1 = fabs((ll[j + 2] - ll[j + 1]) - (ll[j + 1] - ll[j])) > 4;
    __syncthreads();
    if (b1) {
        bad[j + 1] = 1;
        bad[j + 2] = 1;
    }
    __syncthreads();
}

// fix_badlines' interpolation over good neighbours; reads ll, writes out
__device__ void fix_badlines_block(const double* ll, const unsigned char* bad, double* out, int nl, int firstcheck) {
    const int l = threadIdx.x;
    if (l < nl) {
        double v = ll[l];
        if (bad[l]) {
            int pg = l - 1;
            while (pg >= 0 && bad[pg]) --pg;
            int ng = l + 1;
            while (ng < nl && bad[ng]) ++ng;
            if (pg >= firstcheck && ng < nl) {
                const double gap = (ll[ng] - ll[pg]) / (double)(ng - pg);
                v = (gap * (double)(l - pg)) + ll[pg];
            }
        }
        out[l] = v;
    }
    __syncthreads();
}

// block-wide sort of up to 512 doubles in shared memory (NaN-free keys)
__device__ void bitonic512(double* k) {
    for (int size = 2; size <= 512; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = threadIdx.x; t < 256; t += blockDim.x) {
                const int i = 2 * t - (t & (stride - 1));
                const int jx = i + stride;
                const bool up = (i & size) == 0;
                const double a = k[i], b = k[jx];
                if ((a > b) == up) {
                    k[i] = b;
                    k[jx] = a;
                }
            }
            __syncthreads();
        }
    }
}

// median of the first `cnt` entries of a sorted array (np.median)
__device__ __forceinline__ double sorted_median(const double* k, int cnt) {
    if (cnt & 1) return k[cnt / 2];
    return (k[cnt / 2 - 1] + k[cnt / 2]) / 2.0;
}

struct LineParams {
    ldg_lines_args a;
    int system;
    double freq, linelen, linefreq0, samplesperline;
    double half_sync, lo_ok, hi_ok, hz_ire, fsc_mhz, pilot_mhz;
    struct BurstRec* rec;  // nfields x kBurstLines
    double* ll2;           // nfields x kMaxL (NTSC linelocs2)
    double* adjs;          // nfields x kBurstLines (NaN: none)
    int* field14;          // per field
};

// One line's colour-burst zero crossings as clb_findbursts uses them: the
// seed-independent part of zc_cycles, (bstart + zcs - s_rem) / zcburstdiv,
// for all 16 slots (unused slots hold zcs = 0), and the rising flags.
struct BurstRec {
    double cyc[kZc];
    int count, rising, valid, pad;
};

// compute_line_bursts up to the phase update: the zero crossings of the
// line's colour burst (they do not depend on the phase seed)
__device__ void burst_record(const LineParams& P, const double* ll, int line, int lc, const float* burst,
                             const float* demod, long long n, BurstRec& r) {
    r.valid = 0;
    r.count = 0;
    r.rising = 0;
    const long long s = (long long)ll[line];
    const double s_rem = ll[line] - (double)s;
    const double lfreq = P.samplesperline * line_len(ll, line, lc, P.linelen);
    const double fsc_inv = 1 / P.fsc_mhz;
    const long long bstart = (long long)(21 * fsc_inv * lfreq);
    const long long bend = (long long)(28 * fsc_inv * lfreq);
    long long lo = s + bstart, hi = min(s + bend, n);
    if (lo < 0 || hi <= lo) return;
    const int m = (int)min(hi - lo, 128LL);
    float ba[128];
    double acc = 0;
    for (int k = 0; k < m; ++k) acc += (double)burst[lo + k];
    const float mean_f = (float)(acc / m);
    for (int k = 0; k < m; ++k) ba[k] = burst[lo + k] - mean_f;
    double m2 = 0;
    for (int k = 0; k < m; ++k) m2 += (double)ba[k];
    m2 /= m;
    double ss = 0;
    for (int k = 0; k < m; ++k) {
        const double d = (double)ba[k] - m2;
        ss += d * d;
    }
    const double threshold = sqrt(ss / m);
    double accd = 0;
    for (int k = 0; k < m; ++k) accd += (double)demod[lo + k];
    const float mean_d = (float)(accd / m);
    float mx = 0;
    for (int k = 0; k < m; ++k) mx = fmaxf(mx, fabsf(demod[lo + k] - mean_d));
    if ((double)mx > 30 * P.hz_ire) return;
    r.valid = 1;
    const double zcburstdiv = (lfreq * fsc_inv) / 2;
    float zcs[kZc];
    for (int k = 0; k < kZc; ++k) zcs[k] = 0.0f;
    int c = 0;
    long long j = 0;
    const long long end = m - 1;
    while (j < end && c < kZc) {
        if ((double)fabsf(ba[j]) > threshold) {
            double zc;
            if (!calczc(ba, m, (double)j, 0.0, 0, 16, zc)) break;
            if (ba[j] < 0) r.rising |= 1 << c;
            zcs[c] = (float)zc;
            ++c;
            j = (long long)zc + 1;
        } else {
            ++j;
        }
    }
    r.count = c;
    for (int k = 0; k < kZc; ++k) r.cyc[k] = ((double)bstart + (double)zcs[k] - s_rem) / zcburstdiv;
}

// FieldPAL.get_burstlevel (core.py:3095-3104, numpy slice semantics at
// the window's end): the RMS of demod over 2.4 us from 5.5 us into line
// l_adj, less its mean, times sqrt(2); NaN for the reference's None (a
// sample above 30 IRE) or an empty slice.  lc = linecount + lineoffset of
// the moment (get_linelen's last-line rule).
__device__ double pal_burstlevel(const LineParams& P, const double* ll, int l_adj, int lc, const float* demod,
                                 long long n, double hz_ire) {
    const double begin = ll[l_adj] + 5.5 * (P.samplesperline * line_len(ll, l_adj, lc, P.linelen));
    const double length = 2.4 * (P.samplesperline * P.linelen);
    const long long lo = (long long)begin;
    const long long hi = min((long long)(begin + length + 1.0), n);
    if (lo < 0 || hi <= lo) return nan("");
    const long long m = hi - lo;
    double acc = 0;  // float32 samples near 7 MHz: this double sum is exact
    for (long long k = 0; k < m; ++k) acc += (double)demod[lo + k];
    const float mean_f = (float)(acc / (double)m);
    float mx = -INFINITY;
    double s1 = 0;
    for (long long k = 0; k < m; ++k) {
        const float v = demod[lo + k] - mean_f;
        mx = fmaxf(mx, v);
        s1 += (double)v;
    }
    if ((double)mx > 30 * hz_ire) return nan("");
    const double mu = s1 / (double)m;
    double ss = 0;
    for (long long k = 0; k < m; ++k) {
        const double d = (double)(demod[lo + k] - mean_f) - mu;
        ss += d * d;
    }
    return sqrt(ss / (double)m) * 1.4142135623730951;
}

// _angle_mean_phase / phase_distance helpers (core.py:3085-3093)
__device__ __forceinline__ double phase_distance(double x, double c) {
    double d = (x - floor(x)) - c;
    if (d < -0.5) d += 1;
    else if (d > 0.5) d -= 1;
    return d;
}

// one refine_linelocs_pilot pass over ll (shared), in place
__device__ void pilot_pass(const LineParams& P, double* ll, const float* pilot, long long n, double* zcs,
                           double* plen, unsigned char* ok, double* red) {
    const int l = threadIdx.x;
    double zc = 0;
    bool good = false;
    if (l < kPilotLines) {
        double adjfreq = P.freq;
        if (l > 1) adjfreq /= (ll[l] - ll[l - 1]) / P.linelen;
        plen[l] = (adjfreq / P.pilot_mhz) / 2;
        const double b0 = ll[l];
        const long long st = (long long)(b0 + 0.0);
        long long sp = (long long)(b0 + 6 * P.linefreq0 + 0.0 + 1);
        sp = min(sp, n);
        const double lsoffset = ll[l] - (double)st;
        if (st >= 0 && sp > st) {
            const float* seg = pilot + st;
            const long long m = sp - st;
            long long peak = 0;
            float best = -1.0f;
            for (long long k = 0; k < m; ++k) {
                const float v = fabsf(seg[k]);
                if (v > best) {
                    best = v;
                    peak = k;
                }
            }
            double zb;
            if (calczc(seg, m, (double)peak, 0.0, 0, 16, zb)) {
                zc = (zb - lsoffset) / plen[l];
                good = true;
            }
        }
        zcs[l] = zc;
        ok[l] = good;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // a line without a crossing repeats the previous line's value
        double last = 0;
        for (int k = 0; k < kPilotLines; ++k) {
            if (!ok[k]) zcs[k] = last;
            last = zcs[k];
        }
    }
    __syncthreads();
    // mean phase of the fractional parts
    double cs = 0, sn = 0;
    if (l < kPilotLines) {
        const double x = zcs[l];
        const double x2 = x - (double)(int)x;
        const double th = x2 * 3.14159265358979323846 * 2;
        cs = cos(th);
        sn = sin(th);
    }
    red[2 * l] = cs;
    red[2 * l + 1] = sn;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0;
        for (int k = 0; k < kPilotLines; ++k) {
            a += red[2 * k];
            b += red[2 * k + 1];
        }
        double am = atan2(b / kPilotLines, a / kPilotLines) / (3.14159265358979323846 * 2);
        if (am < 0) am = 1 + am;
        red[0] = am;
    }
    __syncthreads();
    const double am = red[0];
    if (l < kPilotLines) ll[l] += phase_distance(zcs[l], am) * plen[l];
    __syncthreads();
}

__global__ void __launch_bounds__(kLineThreads) lines_hsync_kernel(const __grid_constant__ LineParams P) {
    const int f = P.a.first_field + blockIdx.x;
    const ldg_lines_args& a = P.a;
    const long long base = a.startloc[f];
    const long long n = min((long long)a.wlen[f], (long long)(a.capture_len - base));
    const float* d05 = a.d05 + base;
    const int nl = a.proclines;
    __shared__ double ll1[kMaxL], ll[kMaxL], tmp[kMaxL];
    __shared__ unsigned char bad[kMaxL], okf[kMaxL];
    __shared__ double red[2 * kLineThreads];
    const int i = threadIdx.x;
    if (i < nl) {
        ll1[i] = a.linelocs1[(long long)f * kMaxL + i];
        bad[i] = a.linebad1[(long long)f * kMaxL + i];
    }
    __syncthreads();
    // refine_linelocs_hsync: one warp per line; each line's samples (from just
    // before its search start to past its porch) staged in shared memory by
    // one burst of independent loads, so the searches below do not wait on
    // one global load after another
    {
        const int lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
        __shared__ float win[kLineThreads / 32][kHsWin];
        for (int li = threadIdx.x >> 5; li < nl; li += nwarps) {
            bool b = bad[li];
            double v2 = ll1[li];
            if ((li >= 3 && li <= 6) || (P.system == 1 && li >= 1 && li <= 2)) {
                b = true;
            } else {
                const double l1 = ll1[li] - P.freq;
                const long long wb = max((long long)l1 - 64, 0LL);
                const long long we = min(wb + kHsWin, n);
                float* w = win[threadIdx.x >> 5];
                __syncwarp();
                for (long long i = wb + lane; i < we; i += 32) w[i - wb] = d05[i];
                __syncwarp();
                const WinView x{d05, w, wb, we};
                double zc;
                if (warp_calczc(x, n, l1, P.half_sync, 0, P.freq * 2, zc) && !b) {
                    v2 = zc;
                    float mn, mx;
                    warp_minmax(x, (long long)(zc - (P.freq * 0.75)), (long long)(zc + (P.freq * 8)), n, mn, mx);
                    if ((double)mn < P.lo_ok || (double)mx > P.hi_ok) {
                        b = true;
                    } else {
                        const double porch =
                            warp_median_f32(x, (long long)(zc + (P.freq * 8)), (long long)(zc + (P.freq * 9)), n);
                        const double sync =
                            warp_median_f32(x, (long long)(zc + (P.freq * 1)), (long long)(zc + (P.freq * 2.5)), n);
                        double zc2;
                        if (warp_calczc(x, n, l1, (porch + sync) / 2, 0, 400, zc2) && fabs(zc2 - zc) < (P.freq / 2))
                            v2 = zc2;
                        else
                            b = true;
                    }
                } else {
                    b = true;
                }
            }
            if (b) v2 = ll1[li];
            if (lane == 0) {
                ll[li] = v2;
                bad[li] = b;
            }
        }
    }
    __syncthreads();
    deriv_error_block(ll, bad, nl);
    if (P.system == 0) {
        // NTSC: linelocs2 out, burst zero crossings per line
        if (i < nl) P.ll2[(long long)f * kMaxL + i] = ll[i];
        if (i < nl && a.linelocs2) a.linelocs2[(long long)f * kMaxL + i] = ll[i];
        if (i < nl) a.linebad[(long long)f * kMaxL + i] = bad[i];
        if (i < kBurstLines && i < nl)
            burst_record(P, ll, i, a.linecount[f], a.burst + base, a.demod + base, n,
                         P.rec[(long long)f * kBurstLines + i]);
        return;
    }
    // PAL: two pilot passes, then fix_badlines (no backup, lines from 0)
    pilot_pass(P, ll, a.pilot + base, n, tmp, ll1, okf, red);
    pilot_pass(P, ll, a.pilot + base, n, tmp, ll1, okf, red);
    deriv_error_block(ll, bad, nl);
    fix_badlines_block(ll, bad, tmp, nl, 0);
    if (i < nl) {
        a.linelocs[(long long)f * kMaxL + i] = tmp[i];
        a.linebad[(long long)f * kMaxL + i] = bad[i];
    }
    __syncthreads();
    // inputs of the 8-field sequence (FieldPAL.process, core.py:3212-3236):
    // calc_burstmedian runs while the field's line count and offset are still
    // compute_linelocs' (263 / 262 and 0), determine_field_number after they
    // become 312 / 313 and 2 / 3
    {
        const bool isf = a.isfirst[f] != 0;
        const int lc_med = isf ? 263 : 262;
        const int off = isf ? 2 : 3;
        const int lc_seq = (isf ? 312 : 313) + off;
        const float* demod = a.demod + base;
        double lvl = INFINITY;
        if (i >= 11 && i < 313) {
            const double b = pal_burstlevel(P, tmp, i, lc_med, demod, n, P.hz_ire);
            if (!isnan(b)) lvl = b;
        }
        for (int k = i; k < 512; k += blockDim.x) red[k] = k == i ? lvl : INFINITY;
        const int cnt = __syncthreads_count(lvl != INFINITY);
        bitonic512(red);
        if (i == 0) {
            double* out = P.adjs + (long long)f * kBurstLines;
            out[0] = pal_burstlevel(P, tmp, 6 + off, lc_seq, demod, n, P.hz_ire);
            out[1] = cnt ? sorted_median(red, cnt) / P.hz_ire : 0.0;
        }
        if (i < 4)
            burst_record(P, tmp, 7 + 4 * i + off, lc_seq, a.burst + base, demod, n,
                         P.rec[(long long)f * kBurstLines + i]);
    }
}

// np.median of 16 doubles (mean of the two middle ones): Batcher's
// odd-even merge sort network (63 compare-exchanges, the values stay in
// registers)
#define LDG_CS(a, b)                 \
    {                                \
        const double x_ = v[a];      \
        const double y_ = v[b];      \
        if (x_ > y_) {               \
            v[a] = y_;               \
            v[b] = x_;               \
        }                            \
    }
__device__ __forceinline__ double median16(double* v) {
    LDG_CS(0, 1) LDG_CS(2, 3) LDG_CS(4, 5) LDG_CS(6, 7)
    LDG_CS(8, 9) LDG_CS(10, 11) LDG_CS(12, 13) LDG_CS(14, 15)
    LDG_CS(0, 2) LDG_CS(1, 3) LDG_CS(4, 6) LDG_CS(5, 7)
    LDG_CS(8, 10) LDG_CS(9, 11) LDG_CS(12, 14) LDG_CS(13, 15)
    LDG_CS(1, 2) LDG_CS(5, 6) LDG_CS(9, 10) LDG_CS(13, 14)
    LDG_CS(0, 4) LDG_CS(1, 5) LDG_CS(2, 6) LDG_CS(3, 7)
    LDG_CS(8, 12) LDG_CS(9, 13) LDG_CS(10, 14) LDG_CS(11, 15)
    LDG_CS(2, 4) LDG_CS(3, 5) LDG_CS(10, 12) LDG_CS(11, 13)
    LDG_CS(1, 2) LDG_CS(3, 4) LDG_CS(5, 6) LDG_CS(9, 10)
    LDG_CS(11, 12) LDG_CS(13, 14) LDG_CS(0, 8) LDG_CS(1, 9)
    LDG_CS(2, 10) LDG_CS(3, 11) LDG_CS(4, 12) LDG_CS(5, 13)
    LDG_CS(6, 14) LDG_CS(7, 15) LDG_CS(4, 8) LDG_CS(5, 9)
    LDG_CS(6, 10) LDG_CS(7, 11) LDG_CS(2, 4) LDG_CS(3, 5)
    LDG_CS(6, 8) LDG_CS(7, 9) LDG_CS(10, 12) LDG_CS(11, 13)
    LDG_CS(1, 2) LDG_CS(3, 4) LDG_CS(5, 6) LDG_CS(7, 8)
    LDG_CS(9, 10) LDG_CS(11, 12) LDG_CS(13, 14)
    return (v[kZc / 2 - 1] + v[kZc / 2]) / 2.0;
}
#undef LDG_CS

// (key, index) pairs in a strict total order
__device__ __forceinline__ bool pair_less(double ka, int ia, double kb, int ib) {
    return ka < kb || (ka == kb && ia < ib);
}

// ascending bitonic sort of one (key, index) pair per lane across a warp
__device__ __forceinline__ void warp_sort_pairs(double& key, int& idx) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const double ok = __shfl_xor_sync(0xffffffffu, key, j);
            const int oi = __shfl_xor_sync(0xffffffffu, idx, j);
            const bool up = (lane & k) == 0;
            const bool lower = (lane & j) == 0;
            const bool partner_less = pair_less(ok, oi, key, idx);
            // ascending block: the lower lane keeps the smaller pair
            const bool take = lower == up ? partner_less : !partner_less;
            if (take) {
                key = ok;
                idx = oi;
            }
        }
    }
}

// number of pairs in a sorted run of 32 that order before (key, idx)
__device__ __forceinline__ int run_rank(const double* rk, const int* ri, double key, int idx) {
    int lo = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1)
        if (pair_less(rk[lo + step - 1], ri[lo + step - 1], key, idx)) lo += step;
    return lo + (pair_less(rk[lo], ri[lo], key, idx) ? 1 : 0);
}

// ---- NTSC burst phase of every field (compute_burst_offsets, core.py:3360-3388)
//
// Each field's lines start clb_findbursts' phase update from the previous
// field's phase_adjust_median, so the fields form a chain.  The seed enters
// only through the first pass's rounding int(cyc + .5) of every slot: for
// all seeds that leave those roundings as they are, the first pass ends at
// the same phase (the median of the rounded deviations, which moves with
// the seed), so the second pass, the line's adjustment, its rising count
// and the field's median are the same up to the last bits of the FP64
// arithmetic.  So the chain runs as
//   round 1  every field of the range at once, seeded with 0 (the range's
//            first field with its true seed): its median;
//   rounds 2 .. kBurstRounds  every field at once seeded with the round
//            before's median of the field before it (each round carries the
//            true seeds at least one field further, and a seed a few
//            thousandths of a cycle off already decides most fields); the
//            last round keeps adjustments, field-1/4 flag, median, and the
//            interval of seeds that gives the same roundings (with a
//            margin of 1e-9 cycles, also around the second pass's
//            roundings); a field with a valid line without zero crossings
//            (its adjustment is the seed itself) has none;
//   verify   one CTA walking the range in order with the true seeds: a
//            field whose true seed is the last round's seed or lies in its
//            interval keeps that round's results, any other is computed
//            again from its true seed.
// The integer results (rising counts, field-1/4 flags) are those of the
// fields in order; the adjustments and medians agree with them to the
// last bits (kept within 1e-9 of the host restatement by the tests).

constexpr int kBurstWarps = kBurstThreads / 32;
constexpr double kBurstMargin = 1e-9;

struct BurstSmem {
    double rkey[kBurstWarps][32];
    int ridx[kBurstWarps][32];
    double med2[2];
    double lo[kBurstWarps], hi[kBurstWarps];
    double pam, flo, fhi, seed;
    int xonly, next;
};

// The cell of x that int(x + .5) (truncation toward zero) maps to rnd:
// [r - .5, r + .5) for r >= 1, (-1.5, .5) for r = 0, (r - 1.5, r - .5] for r <= -1.
__device__ __forceinline__ void round_cell(int rnd, double& lo, double& hi) {
    lo = rnd >= 1 ? rnd - .5 : rnd - 1.5;
    hi = rnd >= 1 ? rnd + .5 : (rnd == 0 ? .5 : rnd - .5);
}

// One field's burst phase update from seed `prev` (the previous field's
// phase_adjust_median; 0 without one), lines in parallel: two passes of
// clb_findbursts' phase update per line, the field's median from per-warp
// sorted runs (a value's rank is the sum of its positions in the runs), its
// rising count.  All kBurstThreads threads call it; `cur` is the calling
// thread's line record.  Writes the lines' adjustments to adjs_f (NaN: none)
// and the field-1/4 flag to *field14_f when given; leaves the median times 2
// in sm.pam and, with `interval`, the seeds giving the same roundings in
// (sm.flo, sm.fhi) and sm.xonly set when the result depends on the seed
// otherwise.  Ends with the CTA in step.
__device__ void burst_field(const BurstRec& cur, double prev, double* adjs_f, int* field14_f, bool interval,
                            BurstSmem& sm) {
    const int l = threadIdx.x, lane = l & 31, warp = l >> 5;
    const bool line = l < kBurstLines;
    double adj = INFINITY;
    bool ok = false, rising = false, xo = false;
    double plo = -INFINITY, phi = INFINITY;
    if (line && cur.valid) {
        double pa = -prev;
        int rising_count = 0;
        for (int pass = 0; pass < 2; ++pass) {
            rising_count = 0;
            if (cur.count) {
                double dev[kZc];
                int odd = 0;
#pragma unroll
                for (int k = 0; k < kZc; ++k) {
                    const double cyc = cur.cyc[k] + pa;
                    const int rnd = (int)(cyc + .5);
                    if (rnd % 2 != 0) odd |= 1 << k;
                    dev[k] = (double)rnd - cyc;
                    if (interval) {
                        double clo, chi;
                        round_cell(rnd, clo, chi);
                        if (pass == 0) {
                            // seeds s with cur.cyc[k] - s in the cell
                            plo = fmax(plo, cur.cyc[k] - chi);
                            phi = fmin(phi, cur.cyc[k] - clo);
                        } else if (!(fmin(cyc - clo, chi - cyc) > kBurstMargin)) {
                            xo = true;
                        }
                    }
                }
                pa += median16(dev);
                rising_count = __popc((unsigned)(cur.rising ^ odd) & 0xffffu);
            } else {
                xo = true;  // no crossings: the line's adjustment is the seed itself
            }
        }
        rising = (double)rising_count > ((double)cur.count / 2);
        adj = (-pa) / 2;
        ok = true;
    }
    if (line && adjs_f) adjs_f[l] = ok ? adj : nan("");
    double sk = adj;
    int si = l;
    warp_sort_pairs(sk, si);
    sm.rkey[warp][lane] = sk;
    sm.ridx[warp][lane] = si;
    if (interval) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            plo = fmax(plo, __shfl_xor_sync(0xffffffffu, plo, o));
            phi = fmin(phi, __shfl_xor_sync(0xffffffffu, phi, o));
        }
        if (lane == 0) {
            sm.lo[warp] = plo;
            sm.hi[warp] = phi;
        }
    }
    const int cnt = __syncthreads_count(ok);
    const int rsum = __syncthreads_count(ok && !(l % 2) && rising);
    const int xany = __syncthreads_or(xo);
    if (ok) {
        int r = 0;
#pragma unroll
        for (int w = 0; w < kBurstWarps; ++w) r += run_rank(sm.rkey[w], sm.ridx[w], adj, l);
        if (cnt & 1) {
            if (r == cnt / 2) sm.med2[0] = sm.med2[1] = adj;
        } else {
            if (r == cnt / 2 - 1) sm.med2[0] = adj;
            if (r == cnt / 2) sm.med2[1] = adj;
        }
    }
    __syncthreads();
    if (l == 0) {
        // np.median of an empty list is NaN, which the reference then carries forward
        const double med = cnt ? (sm.med2[0] + sm.med2[1]) / 2.0 : nan("");
        sm.pam = med * 2;
        if (field14_f) *field14_f = rsum > (cnt / 4);
        if (interval) {
            double a = -INFINITY, b = INFINITY;
            for (int w = 0; w < kBurstWarps; ++w) {
                a = fmax(a, sm.lo[w]);
                b = fmin(b, sm.hi[w]);
            }
            sm.flo = a;
            sm.fhi = b;
            sm.xonly = xany || isnan(prev);
        }
    }
    __syncthreads();
}

// The true seed of the range's first field: the field before it (a later
// range continues from the previous range's output) or the caller's.
__device__ __forceinline__ double range_seed(const LineParams& P) {
    const ldg_lines_args& a = P.a;
    return a.first_field > 0 ? a.phase_adjust[a.first_field - 1]
                             : (a.prev_phase_adjust_dev ? *a.prev_phase_adjust_dev : a.prev_phase_adjust);
}

constexpr int kBurstRounds = 4;  // rounds before the verification walk

struct BurstSpec {
    double* out1;   // the medians x 2 per field of the odd rounds
    double* out2;   // ... of the even rounds
    double* seed2;  // the last round's seed per field
    double* lo;     // the last round's interval of seeds with the same roundings
    double* hi;
    int* xonly;     // the last round's result depends on the seed otherwise
};

// Round `round` (1 .. kBurstRounds): one CTA per field of the range, seeded
// with 0 (round 1) or with the previous round's median of the field before.
__global__ void __launch_bounds__(kBurstThreads) burst_round_kernel(const __grid_constant__ LineParams P, int round, const __grid_constant__ BurstSpec B) {
    __shared__ BurstSmem sm;
    const ldg_lines_args& a = P.a;
    const int f = a.first_field + blockIdx.x;
    double seed = 0.0;
    if (a.has_prev[f]) {
        if (f == a.first_field) seed = range_seed(P);
        else if (round > 1) seed = (round & 1 ? B.out2 : B.out1)[f - 1];
    }
    BurstRec cur;
    cur.valid = 0;
    if (threadIdx.x < kBurstLines) cur = P.rec[(long long)f * kBurstLines + threadIdx.x];
    if (round < kBurstRounds) {
        burst_field(cur, seed, nullptr, nullptr, false, sm);
        if (threadIdx.x == 0) (round & 1 ? B.out1 : B.out2)[f] = sm.pam;
    } else {
        burst_field(cur, seed, P.adjs + (long long)f * kBurstLines, P.field14 + f, true, sm);
        if (threadIdx.x == 0) {
            a.phase_adjust[f] = sm.pam;
            B.seed2[f] = seed;
            B.lo[f] = sm.flo;
            B.hi[f] = sm.fhi;
            B.xonly[f] = sm.xonly;
        }
    }
}

// The fields of the range in order with their true seeds: the CTA stages
// the last round's seeds, intervals, flags and medians of up to kBurstScan
// fields in shared memory, thread 0 walks over the fields that round got
// right; a field it did not is computed again by the whole CTA.
constexpr int kBurstScan = 512;

__global__ void __launch_bounds__(kBurstThreads) burst_verify_kernel(const __grid_constant__ LineParams P, const __grid_constant__ BurstSpec B) {
    __shared__ BurstSmem sm;
    __shared__ double s_seed2[kBurstScan], s_lo[kBurstScan], s_hi[kBurstScan], s_pam[kBurstScan];
    __shared__ unsigned char s_flags[kBurstScan];  // bit 0: has a previous field; bit 1: no interval
    const ldg_lines_args& a = P.a;
    const int f1 = a.first_field + a.count;
    if (threadIdx.x == 0) sm.seed = range_seed(P);  // the result of the field before the range
    int f = a.first_field;
    while (f < f1) {
        const int n = min(kBurstScan, f1 - f);
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            s_seed2[i] = B.seed2[f + i];
            s_lo[i] = B.lo[f + i];
            s_hi[i] = B.hi[f + i];
            s_pam[i] = a.phase_adjust[f + i];
            s_flags[i] = (unsigned char)((a.has_prev[f + i] ? 1 : 0) | (B.xonly[f + i] ? 2 : 0));
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double prev = sm.seed;  // the result of field f - 1
            int g = 0;
            for (; g < n; ++g) {
                const double p = (s_flags[g] & 1) ? prev : 0.0;
                const bool same = __double_as_longlong(p) == __double_as_longlong(s_seed2[g]);
                const bool inside = !(s_flags[g] & 2) && p > s_lo[g] + kBurstMargin && p < s_hi[g] - kBurstMargin;
                if (!same && !inside) {
                    prev = p;  // field g's seed
                    break;
                }
                prev = s_pam[g];
            }
            sm.next = f + g;
            sm.seed = prev;
        }
        __syncthreads();
        const int g = sm.next;
        if (g < f + n) {
            BurstRec cur;
            cur.valid = 0;
            if (threadIdx.x < kBurstLines) cur = P.rec[(long long)g * kBurstLines + threadIdx.x];
            burst_field(cur, sm.seed, P.adjs + (long long)g * kBurstLines, P.field14 + g, false, sm);
            if (threadIdx.x == 0) {
                a.phase_adjust[g] = sm.pam;
                sm.seed = sm.pam;
            }
            f = g + 1;
        } else {
            f = g;
        }
        __syncthreads();
    }
}

// PAL 8-field sequence (determine_field_number, core.py:3128-3203), fields in
// order.  Lane j follows line 7 + 4j: its burst phase starts from the
// previous field's (0 when there is none, when that line had no result or
// when that field decided its ID before measuring phases), two passes of
// clb_findbursts' phase update, rising or not.  The field's ID comes from
// line 6's burst level against the field's median (present / absent / out of
// both ranges) and the majority of rising lines, or is the previous ID + 1
// when that evidence is missing or split.
__global__ void __launch_bounds__(32) pal_sequence_kernel(const __grid_constant__ LineParams P) {
    const ldg_lines_args& a = P.a;
    const int f0 = a.first_field, f1 = a.first_field + a.count;
    const int j = threadIdx.x;
    double seed = nan("");
    int prev_id;
    if (f0 > 0) {
        if (j < 4) seed = a.phase_adjust[(long long)(f0 - 1) * 4 + j];
        prev_id = a.field_phase[f0 - 1];
    } else {
        if (j < 4) seed = a.prev_pal_adjust_dev ? a.prev_pal_adjust_dev[j] : a.prev_pal_adjust[j];
        prev_id = a.prev_field_phase_dev ? *a.prev_field_phase_dev : a.prev_field_phase;
    }
    for (int f = f0; f < f1; ++f) {
        const bool has_prev = a.has_prev[f] != 0;
        const int following = has_prev ? (prev_id + 1 == 9 ? 1 : prev_id + 1) : 1;
        const double b6 = P.adjs[(long long)f * kBurstLines + 0];
        const double bm = P.adjs[(long long)f * kBurstLines + 1];
        int hasburst = -1;
        if (!isnan(b6)) {
            const double b = b6 / P.hz_ire;
            if (b >= bm * 0.8 && b <= bm * 1.2) hasburst = 1;
            else if (b < bm * 0.2) hasburst = 0;
        }
        double out = nan("");
        int id = following;
        if (hasburst >= 0) {  // warp-uniform
            const bool isf = a.isfirst[f] != 0;
            const int m4 = isf ? (hasburst ? 3 : 1) : (hasburst ? 2 : 4);
            bool valid = false, rising = false;
            if (j < 4) {
                const BurstRec r = P.rec[(long long)f * kBurstLines + j];
                if (r.valid) {
                    double pa = -((has_prev && !isnan(seed)) ? seed : 0.0);
                    int rising_count = 0;
                    for (int pass = 0; pass < 2; ++pass) {
                        rising_count = 0;
                        if (r.count) {
                            double dev[kZc];
                            int odd = 0;
#pragma unroll
                            for (int k = 0; k < kZc; ++k) {
                                const double cyc = r.cyc[k] + pa;
                                const int rnd = (int)(cyc + .5);
                                if (rnd % 2 != 0) odd |= 1 << k;
                                dev[k] = (double)rnd - cyc;
                            }
                            pa += median16(dev);
                            rising_count = __popc((unsigned)(r.rising ^ odd) & 0xffffu);
                        }
                    }
                    rising = (double)rising_count > ((double)r.count / 2);
                    out = -pa;
                    valid = true;
                }
            }
            const int count = __popc(__ballot_sync(0xffffffffu, valid));
            const int rcount = __popc(__ballot_sync(0xffffffffu, valid && rising));
            if (count != 0 && rcount * 2 != count) {
                bool firstfour = rcount * 2 > count;
                if (m4 == 2) firstfour = !firstfour;
                id = m4 + (firstfour ? 0 : 4);
            }
        }
        if (j < 4) a.phase_adjust[(long long)f * 4 + j] = out;
        if (j == 0) a.field_phase[f] = id;
        seed = out;
        prev_id = id;
    }
}

// NTSC: refine_linelocs_burst's application, fix_badlines, subcarrier shift
__global__ void __launch_bounds__(512) burst_apply_kernel(const __grid_constant__ LineParams P, double shift) {
    const int f = P.a.first_field + blockIdx.x;
    const ldg_lines_args& a = P.a;
    const int nl = a.proclines;
    const int lc = a.linecount[f];
    __shared__ double ll2[kMaxL], adj_ll[kMaxL], out[kMaxL], adjs[kBurstLines];
    __shared__ unsigned char bad[kMaxL], has[kBurstLines];
    __shared__ double keys[512];
    __shared__ int nadj;
    const int l = threadIdx.x;
    if (l == 0) nadj = 0;
    if (l < nl) {
        ll2[l] = P.ll2[(long long)f * kMaxL + l];
        bad[l] = a.linebad[(long long)f * kMaxL + l];
    }
    double an = nan("");
    if (l < kBurstLines) an = P.adjs[(long long)f * kBurstLines + l];
    __syncthreads();
    if (l >= 1 && l < kBurstLines && l < nl && isnan(an)) bad[l] = 1;
    __syncthreads();
    double adj = nan("");
    if (l < kBurstLines && l < nl) {
        has[l] = 0;
        if (!(isnan(ll2[l]) || bad[l]) && !isnan(an)) {
            const double lfreq = P.samplesperline * line_len(ll2, l, lc, P.linelen);
            adj = an * lfreq * (1 / P.fsc_mhz);
            has[l] = 1;
            atomicAdd(&nadj, 1);
        }
        adjs[l] = adj;
    }
    keys[l] = isnan(adj) ? INFINITY : adj;
    if (l < nl) adj_ll[l] = ll2[l];
    __syncthreads();
    bitonic512(keys);
    if (l == 0) {
        const int cnt = nadj;
        if (cnt) {
            const double med = sorted_median(keys, cnt);
            double lastvalid = med;
            for (int k = 0; k < kBurstLines && k < nl; ++k) {
                if (has[k] && adjs[k] - med >= -2 && adjs[k] - med <= 2) {
                    adj_ll[k] += adjs[k];
                    lastvalid = adjs[k];
                } else {
                    adj_ll[k] += lastvalid;
                }
            }
            const bool first = a.isfirst[f] != 0, f14 = P.field14[f] != 0;
            a.field_phase[f] = first ? (f14 ? 1 : 3) : (f14 ? 4 : 2);
        } else {
            a.field_phase[f] = 1;
        }
    }
    __syncthreads();
    // fix_badlines(linelocs3, linelocs2): deriv error, NaN from backup, interpolate (from line 1)
    deriv_error_block(adj_ll, bad, nl);
    if (l < nl && isnan(adj_ll[l])) adj_ll[l] = ll2[l];
    __syncthreads();
    fix_badlines_block(adj_ll, bad, out, nl, 1);
    if (l < nl) {
        a.linelocs[(long long)f * kMaxL + l] = out[l] - shift;
        a.linebad[(long long)f * kMaxL + l] = bad[l];
    }
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

extern "C" {

int ldg_sync_runs(ldg_ctx* c, const float* d05, int64_t n, double threshold, int64_t min_long, int64_t trim_lo,
                  int64_t trim_hi, int64_t* run_start, int64_t* run_len, double* run_mean, int64_t cap,
                  int64_t* nruns, void* stream) {
    if (!c || !d05 || !run_start || !run_len || !run_mean || !nruns)
        return ldg::lines_fail(LDG_ERR_ARG, "ldg_sync_runs: NULL argument");
    if (n < 2 || cap < 1 || trim_lo < 0 || trim_hi < 0) return ldg::lines_fail(LDG_ERR_ARG, "ldg_sync_runs: bad size");
    std::lock_guard<std::mutex> lk(ldg::ctx_mutex(c));
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(ldg::ctx_device(c));
    cudaStream_t st = (cudaStream_t)stream;
    const long long ntiles = (n + kEdgeTile - 1) / kEdgeTile;
    const long long ecap = 2 * cap + 2;
    const size_t b_tot = 256, b_edges = align256(ecap * sizeof(long long));
    const size_t b_runs = align256(cap * sizeof(long long));
    const size_t need = b_tot + b_edges + 2 * b_runs + align256(cap * sizeof(double));
    void* scratch = nullptr;
    auto done = [&](int rc) {
        if (prev >= 0) cudaSetDevice(prev);
        return rc;
    };
    if (ldg::ctx_lines_scratch(c, need, &scratch) != LDG_OK) return done(LDG_ERR_CUDA);
    char* p = static_cast<char*>(scratch);
    long long* total = reinterpret_cast<long long*>(p);
    long long* edges = reinterpret_cast<long long*>(p + b_tot);
    long long* rs = reinterpret_cast<long long*>(p + b_tot + b_edges);
    long long* rl = rs + b_runs / sizeof(long long);
    double* rm = reinterpret_cast<double*>(rl + b_runs / sizeof(long long));
    auto cuda_fail = [&](const char* what) {
        ldg::ctx_scan_invalidate(c);
        return done(ldg::lines_fail(LDG_ERR_CUDA, std::string("ldg_sync_runs: ") + what + ": " +
                                                      cudaGetErrorString(cudaGetLastError())));
    };
    // the look-back state (tickets, per-tile flags and counts) and the
    // host-mapped words: [0] the edge count, [1] the look-back error flag
    ldg::ScanState ss;
    long long *hw = nullptr, *dw = nullptr;
    if (ldg::ctx_scan_state(c, ntiles, st, &ss) != LDG_OK || ldg::ctx_host_word(c, &hw, &dw) != LDG_OK)
        return cuda_fail("scan state");
    volatile long long* vhw = hw;
    vhw[0] = -1;
    vhw[1] = 0;
    edge_pass_kernel<<<(unsigned)ntiles, kEdgeThreads, 0, st>>>(d05, n, threshold, ss.ticket, ss.base, ss.call,
                                                                ss.flags, ss.agg, ss.incl, ntiles, edges, ecap,
                                                                total, dw + 1);
    // runs straight into the caller's pinned (mapped) buffers when they are:
    // the host then waits for the stream only (no copy-engine transfer, which
    // would queue behind bulk copies of an end-to-end pipeline)
    void* drs = ldg::device_view(run_start);
    void* drl = ldg::device_view(run_len);
    void* drm = ldg::device_view(run_mean);
    const bool mapped = drs && drl && drm;
    if (mapped) {
        run_pair_kernel<<<4 * 148, 256, 0, st>>>(edges, total, cap, d05, min_long, trim_lo, trim_hi,
                                                 static_cast<long long*>(drs), static_cast<long long*>(drl),
                                                 static_cast<double*>(drm), dw);
    } else {
        run_pair_kernel<<<4 * 148, 256, 0, st>>>(edges, total, cap, d05, min_long, trim_lo, trim_hi, rs, rl, rm,
                                                 dw);
    }
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) return cuda_fail("scan");
    if (vhw[1] != 0) {
        ldg::ctx_scan_invalidate(c);
        return done(ldg::lines_fail(LDG_ERR_CUDA, "ldg_sync_runs: a tile's look-back wait timed out"));
    }
    const long long nedges = vhw[0];
    if (nedges < 0) return cuda_fail("run count not written");
    const long long nr = nedges / 2;
    *nruns = nr;
    if (nr > cap || nedges > ecap) return done(ldg::lines_fail(LDG_ERR_RANGE, "ldg_sync_runs: more runs than cap"));
    if (!mapped && nr > 0) {
        if (cudaMemcpyAsync(run_start, rs, nr * sizeof(long long), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaMemcpyAsync(run_len, rl, nr * sizeof(long long), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaMemcpyAsync(run_mean, rm, nr * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess)
            return cuda_fail("D2H");
        if (cudaStreamSynchronize(st) != cudaSuccess) return cuda_fail("run copy");
    }
    return done(LDG_OK);
}

int64_t ldg_lines_scratch_bytes(int32_t nfields) {
    if (nfields < 0) return -1;
    return (int64_t)(align256((size_t)nfields * kBurstLines * sizeof(BurstRec)) +
                     align256((size_t)nfields * kMaxL * sizeof(double)) +
                     align256((size_t)nfields * kBurstLines * sizeof(double)) +
                     align256((size_t)nfields * sizeof(int)) + 5 * align256((size_t)nfields * sizeof(double)) +
                     align256((size_t)nfields * sizeof(int)));
}

}  // extern "C"

extern "C" int ldg_lines_refine(ldg_ctx* c, const ldg_lines_args* a) {
    if (!c || !a) return ldg::lines_fail(LDG_ERR_ARG, "ldg_lines_refine: NULL argument");
    if (a->nfields < 0 || a->proclines < 8 || a->proclines > kMaxL || (a->k.system != 0 && a->k.system != 1))
        return ldg::lines_fail(LDG_ERR_ARG, "ldg_lines_refine: bad size or system");
    if (a->nfields == 0) return LDG_OK;
    if (!a->d05 || !a->startloc || !a->wlen || !a->isfirst || !a->linecount || !a->has_prev || !a->linelocs1 ||
        !a->linebad1 || !a->linelocs || !a->linebad || !a->scratch ||
        !a->demod || !a->burst || !a->phase_adjust || !a->field_phase || (a->k.system == 1 && !a->pilot))
        return ldg::lines_fail(LDG_ERR_ARG, "ldg_lines_refine: NULL buffer");
    if (a->k.system == 0 && a->proclines < kBurstLines)
        return ldg::lines_fail(LDG_ERR_ARG, "ldg_lines_refine: NTSC needs proclines >= 266");
    if (a->k.system == 1 && a->proclines < kPilotLines)
        return ldg::lines_fail(LDG_ERR_ARG, "ldg_lines_refine: PAL needs proclines >= 323");
    if (a->first_field < 0 || a->first_field >= a->nfields || a->count < 0 ||
        a->first_field + a->count > a->nfields || a->stages < 0 || a->stages > 7)
        return ldg::lines_fail(LDG_ERR_ARG, "ldg_lines_refine: bad field range or stages");
    LineParams P;
    P.a = *a;
    if (P.a.count == 0) P.a.count = a->nfields - a->first_field;
    P.system = a->k.system;
    P.freq = a->k.freq;
    P.linelen = a->k.linelen;
    P.linefreq0 = a->k.linefreq0;
    P.samplesperline = a->k.samplesperline;
    P.half_sync = a->k.half_sync;
    P.lo_ok = a->k.lo_ok;
    P.hi_ok = a->k.hi_ok;
    P.hz_ire = a->k.hz_ire;
    P.fsc_mhz = a->k.fsc_mhz;
    P.pilot_mhz = a->k.pilot_mhz;
    char* s = static_cast<char*>(a->scratch);
    const size_t nf = (size_t)a->nfields;
    P.rec = reinterpret_cast<BurstRec*>(s);
    s += align256(nf * kBurstLines * sizeof(BurstRec));
    P.ll2 = reinterpret_cast<double*>(s);
    s += align256(nf * kMaxL * sizeof(double));
    P.adjs = reinterpret_cast<double*>(s);
    s += align256(nf * kBurstLines * sizeof(double));
    P.field14 = reinterpret_cast<int*>(s);
    s += align256(nf * sizeof(int));
    BurstSpec B;
    B.out1 = reinterpret_cast<double*>(s);
    s += align256(nf * sizeof(double));
    B.out2 = reinterpret_cast<double*>(s);
    s += align256(nf * sizeof(double));
    B.seed2 = reinterpret_cast<double*>(s);
    s += align256(nf * sizeof(double));
    B.lo = reinterpret_cast<double*>(s);
    s += align256(nf * sizeof(double));
    B.hi = reinterpret_cast<double*>(s);
    s += align256(nf * sizeof(double));
    B.xonly = reinterpret_cast<int*>(s);
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(ldg::ctx_device(c));
    cudaStream_t st = (cudaStream_t)a->stream;
    const int stages = a->stages ? a->stages : 7;
    if (stages & 1) lines_hsync_kernel<<<P.a.count, kLineThreads, 0, st>>>(P);
    if (P.system == 1 && (stages & 2)) pal_sequence_kernel<<<1, 32, 0, st>>>(P);
    if (P.system == 0) {
        if (stages & 2) {
            for (int r = 1; r <= kBurstRounds; ++r)
                burst_round_kernel<<<P.a.count, kBurstThreads, 0, st>>>(P, r, B);
            burst_verify_kernel<<<1, kBurstThreads, 0, st>>>(P, B);
        }
        const double shift = (117.25 / 360) / P.fsc_mhz * P.freq;
        if (stages & 4) burst_apply_kernel<<<P.a.count, 512, 0, st>>>(P, shift);
    }
    cudaError_t e = cudaGetLastError();
    if (prev >= 0) cudaSetDevice(prev);
    if (e != cudaSuccess) return ldg::lines_fail(LDG_ERR_CUDA, std::string("ldg_lines_refine: ") + cudaGetErrorString(e));
    return LDG_OK;
}
