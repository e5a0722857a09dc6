// Analog audio to 16-bit output, a batch of fields per launch (restates
// downscale_audio and its helpers, lddecode/core.py:1423-1580, and
// dsa_rescale_and_clip, lddecode/utils.py:1328-1332).
//
// One CTA per field.  Every FP64 operation is an explicitly rounded
// intrinsic in the reference's order (numpy evaluates each operation on its
// own, with no fused multiply-adds), and each run of stage-1 audio is summed
// in float32 in index order as the reference's compiled mean does, so the
// int16 output is the reference's bit for bit.
#include "ldg_audio.cuh"

namespace ldg {

namespace {

constexpr int kAudioThreads = 256;

__device__ __forceinline__ int16_t rescale_clip_neg(double x) {
    // -min(max(int(round(x * 32767 / 371081)), -32766), 32766)
    double v = rint(__ddiv_rn(__dmul_rn(x, 32767.0), 371081.0));
    v = fmin(fmax(v, -32766.0), 32766.0);
    return (int16_t)(-(int)v);
}

__global__ void __launch_bounds__(kAudioThreads) audio_downscale_kernel(const __grid_constant__ AudioBatch b,
                                                                       AudioConsts c, int* muted) {
    const AudioField& f = b.f[blockIdx.x];
    __shared__ double locs[kAudioMaxTicks], swow[kAudioMaxTicks];
    __shared__ int any_jump, any_mute;
    const int t = threadIdx.x;
    const int nt = f.nticks;
    if (t == 0) {
        any_jump = 0;
        any_mute = 0;
    }
    __syncthreads();
    const double* li = f.ll;
    const int nl = f.nlines;
    // _downscale_audio_compute_locs_and_swow (core.py:1455-1488): the line
    // position of every tick, interpolated between line locations
    for (int i = t; i < nt; i += kAudioThreads) {
        const double ar = __dadd_rn(f.timeoffset, __dmul_rn((double)i, f.soundgap));
        const double linenum = __dadd_rn(__ddiv_rn(__dmul_rn(ar, 1000000.0), c.line_period), 1.0);
        double cur, nxt;
        if (linenum < 0) {
            cur = (double)(long long)__dadd_rn(li[0], __dmul_rn(c.linelen, linenum));
            nxt = __dadd_rn(cur, c.linelen);
        } else if ((double)nl > __dadd_rn(linenum, 2.0)) {
            const long long k = (long long)linenum;
            cur = li[k];
            nxt = li[k + 1];
        } else {
            cur = li[nl - 2];
            nxt = __dadd_rn(li[nl - 2], c.linelen);
        }
        const double span = __dadd_rn(nxt, -cur);
        const double sl = __dadd_rn(cur, __dmul_rn(span, __dadd_rn(linenum, -floor(linenum))));
        double sw = __ddiv_rn(span, c.linelen);
        sw = __dadd_rn(__dadd_rn(sw, -1.0), 1.0);
        swow[i] = sw;
        locs[i] = __ddiv_rn(sl, c.scale);
    }
    __syncthreads();
    for (int i = t; i + 1 < nt; i += kAudioThreads)
        if (fabs(__dadd_rn(swow[i + 1], -swow[i])) > 0.015) any_jump = 1;
    __syncthreads();
    if (any_jump && t == 0) {
        // a jump of more than 1.5 % keeps the previous (already clamped)
        // factor, from the first jump of the unclamped factors on
        int j0 = 0;
        while (j0 + 1 < nt && !(fabs(__dadd_rn(swow[j0 + 1], -swow[j0])) > 0.015)) ++j0;
        for (int i = j0 + 1; i < nt; ++i)
            if (fabs(__dadd_rn(swow[i], -swow[i - 1])) > 0.015) swow[i] = swow[i - 1];
    }
    __syncthreads();
    // _downscale_audio_to_output (core.py:1493-1533)
    const int n = nt - 1;
    for (int i = t; i < n; i += kAudioThreads) {
        const long long s = (long long)locs[i], e = (long long)locs[i + 1];
        // the slice audio[s:e] with numpy's bounds: a negative bound counts
        // from the end of the buffer, then clamps at 0; an empty slice (which
        // makes the reference's mean divide by zero and raise) is muted
        const long long s0 = s < 0 ? max(s + (long long)f.len, 0LL) : s;
        const long long e0 = e < 0 ? max(e + (long long)f.len, 0LL) : e;
        int16_t ol = 0, orr = 0;
        if (e > s && e < f.len && e0 > s0) {
            // summed in index order; eight samples per channel loaded ahead
            // of their adds (one memory latency per eight, not per sample)
            float suml = 0.0f, sumr = 0.0f;
            long long k = s0;
            for (; k + 8 <= e0; k += 8) {
                float xl[8], xr[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    xl[u] = __ldg(f.al + k + u);
                    xr[u] = __ldg(f.ar + k + u);
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    suml = __fadd_rn(suml, xl[u]);
                    sumr = __fadd_rn(sumr, xr[u]);
                }
            }
            for (; k < e0; ++k) {
                suml = __fadd_rn(suml, __ldg(f.al + k));
                sumr = __fadd_rn(sumr, __ldg(f.ar + k));
            }
            const double len = (double)(e0 - s0);
            const double w = swow[i];
            ol = rescale_clip_neg(__dadd_rn(__dmul_rn(__ddiv_rn((double)suml, len), w), -c.lfreq));
            orr = rescale_clip_neg(__dadd_rn(__dmul_rn(__ddiv_rn((double)sumr, len), w), -c.rfreq));
        } else {
            any_mute = 1;
        }
        f.out[2 * i] = ol;
        f.out[2 * i + 1] = orr;
    }
    __syncthreads();
    if (t == 0 && muted) muted[blockIdx.x] = any_mute;
}

}  // namespace

cudaError_t launch_audio_downscale(const AudioField* fields, int nfields, AudioConsts c, int* muted,
                                   cudaStream_t stream) {
    for (int off = 0; off < nfields; off += kAudioBatch) {
        const int n = nfields - off < kAudioBatch ? nfields - off : kAudioBatch;
        AudioBatch b;
        for (int i = 0; i < n; ++i) b.f[i] = fields[off + i];
        audio_downscale_kernel<<<n, kAudioThreads, 0, stream>>>(b, c, muted ? muted + off : nullptr);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace ldg
