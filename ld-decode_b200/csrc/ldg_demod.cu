// Fused per-block RF demodulator: one 1024-thread CTA per 32768-sample
// overlap-save block, persistent over blocks.
//
// Per block, in shared memory (a 16384-point complex working set S):
//   X = R2C(x)                                   (input spectrum, bins 0..N/2)
//   rfhpf  = C2R(X * Frfhpf)                     -> sliced, float32
//   efm    = C2R(X * Fefm/2)                     -> int16 (truncated)
//   audio  = 2 x (1024-bin sub-band * filt1 -> iFFT -> FM discriminator)
//   z      = analytic signal of X * RFVideo * MTF^m, computed as its even and
//            odd samples with two 16384-point inverse FFTs
//   demod_raw = arg(z[n] conj z[n-1]) * fs / 2pi, in [0, fs)
//   D      = R2C(clip(demod_raw, 1.5 MHz, 0.75 fs))
//   demod / demod_05 / demod_burst [/ demod_pilot] = C2R(D * F) with rolls
// X and the even-sample half of z are parked in a per-CTA global scratch
// (256 KB per CTA; with one CTA per SM it stays in L2) between the steps
// that need them.  This restates RFDecode.demodblock_cpu
// (lddecode/core.py:755-879) and unwrap_hilbert (lddecode/utils.py:898-926).
#include "ldg_demod.cuh"
#include "ldg_fft.cuh"

namespace ldg {

namespace {

constexpr float kTwoPi = 6.28318530717958647692f;

struct Smem {
    float2* S;       // padded(16384)
    float2* A;       // 2 x padded(1024): audio sub-bands
    Twiddles tw;
};

__device__ __forceinline__ float fm_disc(float2 a, float2 b, float k) {
    // arg(a * conj(b)) wrapped to [0, 2pi), times k = rate / 2pi
    const float re = fmaf(a.x, b.x, a.y * b.y);
    const float im = fmaf(a.y, b.x, -a.x * b.y);
    float d = atan2f(im, re);
    if (d < 0.0f) d += kTwoPi;
    return d * k;
}

// x (N real samples) -> S[m] = (x[2m], x[2m+1])
__device__ void load_block(const DemodParams& p, int blk, float2* S) {
    if (p.in_kind == 0) {
        const int16_t* src = static_cast<const int16_t*>(p.in) + (long long)blk * p.in_stride;
        if ((reinterpret_cast<uintptr_t>(src) & 15) == 0) {
            const int4* s4 = reinterpret_cast<const int4*>(src);
            for (int i = threadIdx.x; i < kN / 8; i += kThreads) {
                const int4 v = __ldg(s4 + i);
                const int w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const float lo = (float)(int16_t)(w[c] & 0xffff);
                    const float hi = (float)(int16_t)(((unsigned)w[c]) >> 16);
                    S[pad(4 * i + c)] = make_float2(lo, hi);
                }
            }
        } else {
            for (int m = threadIdx.x; m < kM; m += kThreads)
                S[pad(m)] = make_float2((float)src[2 * m], (float)src[2 * m + 1]);
        }
    } else {
        const float* src = static_cast<const float*>(p.in) + (long long)blk * p.in_stride;
        for (int m = threadIdx.x; m < kM; m += kThreads)
            S[pad(m)] = make_float2(src[2 * m], src[2 * m + 1]);
    }
}

// S = FFT_M(x[2m] + i x[2m+1])  ->  X[k], k = 0..M, with X[0], X[M] packed in S[0]
__device__ void r2c_post(float2* S, const Twiddles& tw) {
    for (int k = threadIdx.x; k <= kM / 2; k += kThreads) {
        if (k == 0) {
            const float2 z = S[0];
            S[0] = make_float2(z.x + z.y, z.x - z.y);
        } else {
            const float2 zk = S[pad(k)], zm = S[pad(kM - k)];
            const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
            const float2 o = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
            const float2 t = cmul(tw.w<false>(k), o);
            S[pad(k)] = cadd(e, t);
            if (k != kM / 2) S[pad(kM - k)] = cconj(csub(e, t));
        }
    }
}

// S holds H[k], k = 0..M (H[0], H[M] packed) of a real signal; turn it into
// the M-point complex spectrum whose inverse FFT is (x[2m], x[2m+1]) * M.
__device__ void c2r_pre(float2* S, const Twiddles& tw) {
    for (int k = threadIdx.x; k <= kM / 2; k += kThreads) {
        if (k == 0) {
            const float2 h = S[0];
            S[0] = make_float2(0.5f * (h.x + h.y), 0.5f * (h.x - h.y));
        } else {
            const float2 hk = S[pad(k)], hm = S[pad(kM - k)];
            const float2 e = make_float2(0.5f * (hk.x + hm.x), 0.5f * (hk.y - hm.y));
            const float2 d = make_float2(0.5f * (hk.x - hm.x), 0.5f * (hk.y + hm.y));
            const float2 o = cmul(d, tw.w<true>(k));
            S[pad(k)] = make_float2(e.x - o.y, e.y + o.x);
            if (k != kM / 2) S[pad(kM - k)] = make_float2(e.x + o.y, o.x - e.y);
        }
    }
}

// S[k] = src[k] * F[k] for the packed half spectrum (src may alias S).
__device__ __forceinline__ float2 mul_half(float2 x, const float2* F, int k) {
    if (k == 0) return make_float2(x.x * __ldg(&F[0].x), x.y * __ldg(&F[kM].x));
    return cmul(x, __ldg(F + k));
}

// Store real samples [start, start+len) (rolled) of the C2R result in S.
__device__ void write_real(const float2* S, float* out, const OutSlice& s, int roll) {
    const float scale = 1.0f / kM;
    for (int i = threadIdx.x; i < s.len; i += kThreads) {
        const int n = (s.start + i + roll) & (kN - 1);
        const float2 v = S[pad(n >> 1)];
        out[i] = ((n & 1) ? v.y : v.x) * scale;
    }
}

__device__ void write_efm(const float2* S, int16_t* out, const OutSlice& s) {
    const float scale = 1.0f / kM;
    for (int i = threadIdx.x; i < s.len; i += kThreads) {
        const int n = (s.start + i) & (kN - 1);
        const float2 v = S[pad(n >> 1)];
        float x = ((n & 1) ? v.y : v.x) * scale;
        x = fminf(fmaxf(x, -32768.0f), 32767.0f);
        out[i] = (int16_t)__float2int_rz(x);
    }
}

// Real-output transform of the half spectrum already in S (times F):
// multiply, C2R, inverse FFT.  src == nullptr: take X from S itself.
__device__ void real_output(float2* S, const float2* src, const float2* F, const Twiddles& tw,
                            float2* park) {
    for (int k = threadIdx.x; k < kM; k += kThreads) {
        const float2 x = src ? src[k] : S[pad(k)];
        if (park) park[k] = x;
        S[pad(k)] = mul_half(x, F, k);
    }
    __syncthreads();
    c2r_pre(S, tw);
    __syncthreads();
    fft16k<true>(S, tw);
}

__device__ void audio_stage1(const DemodParams& p, Smem& sm, int blk) {
    constexpr int stride = padded(1024);
    const float2* S = sm.S;
    for (int idx = threadIdx.x; idx < 2 * 1024; idx += kThreads) {
        const int ch = idx >> 10, k = idx & 1023;
        float2 v = make_float2(0.f, 0.f);
        if (k <= 512) {
            const int lb = ch ? p.a_lowbin[1] : p.a_lowbin[0];
            const float2* f1 = ch ? p.a_filt1[1] : p.a_filt1[0];
            float2 xb = (k < 512) ? S[pad(lb + k)] : cconj(S[pad(lb + 512)]);
            v = cmul(xb, __ldg(f1 + k));
        }
        sm.A[ch * stride + pad(k)] = v;
    }
    __syncthreads();
    fft1k_x2<true>(sm.A, sm.tw);
    const float kk = p.a_rate / kTwoPi;
    for (int idx = threadIdx.x; idx < 2 * 1024; idx += kThreads) {
        const int ch = idx >> 10, n = idx & 1023;
        const int i = n - p.s_audio.start;
        float* oa = ch ? p.o_audio[1] : p.o_audio[0];
        if (i < 0 || i >= p.s_audio.len || oa == nullptr) continue;
        const float2* Ab = sm.A + ch * stride;
        const float d = (n == 0) ? 0.0f : fm_disc(Ab[pad(n)], Ab[pad(n - 1)], kk);
        oa[(long long)blk * p.s_audio.len + i] = d + (ch ? p.a_low[1] : p.a_low[0]);
    }
}

}  // namespace

__global__ void __launch_bounds__(kThreads, 1) demod_kernel(const DemodParams p) {
    extern __shared__ float2 smem[];
    Smem sm;
    sm.S = smem;
    sm.A = smem + padded(kM);
    float2* twh = sm.A + 2 * padded(1024);
    float2* twl = twh + kTwHi;
    for (int i = threadIdx.x; i < kTwHi; i += kThreads) twh[i] = p.tw_hi[i];
    for (int i = threadIdx.x; i < kTwLo; i += kThreads) twl[i] = p.tw_lo[i];
    sm.tw.hi = twh;
    sm.tw.lo = twl;
    float2* S = sm.S;
    const Twiddles& tw = sm.tw;
    float2* parkX = p.scratch + (size_t)blockIdx.x * 2 * kM;
    float2* parkZ = parkX + kM;
    const float kfs = p.fs_hz / kTwoPi;
    const float clip_lo = 1500000.0f, clip_hi = p.fs_hz * 0.75f;
    __syncthreads();

    for (int blk = blockIdx.x; blk < p.nblocks; blk += gridDim.x) {
        // ---- input spectrum X
        load_block(p, blk, S);
        __syncthreads();
        fft16k<false>(S, tw);
        r2c_post(S, tw);
        __syncthreads();

        if (p.audio) {
            audio_stage1(p, sm, blk);
        }

        // ---- rfhpf (from X in S; park X)
        if (p.o_rfhpf) {
            real_output(S, nullptr, p.f_rfhpf, tw, parkX);
            write_real(S, p.o_rfhpf + (long long)blk * p.s_rfhpf.len, p.s_rfhpf, 0);
        } else {
            for (int k = threadIdx.x; k < kM; k += kThreads) parkX[k] = S[pad(k)];
        }
        __syncthreads();

        // ---- EFM
        if (p.o_efm) {
            real_output(S, parkX, p.f_efm, tw, nullptr);
            write_efm(S, p.o_efm + (long long)blk * p.s_efm.len, p.s_efm);
            __syncthreads();
        }

        // ---- analytic signal, even samples
        for (int k = threadIdx.x; k < kM; k += kThreads) {
            const float2 x = parkX[k];
            float2 y;
            if (k == 0) {
                const float2 a = cscale(__ldg(p.f_g), x.x);
                const float2 b = cscale(__ldg(p.f_g + kM), x.y);
                y = cadd(a, b);
            } else {
                y = cmul(x, __ldg(p.f_g + k));
            }
            S[pad(k)] = y;
        }
        __syncthreads();
        fft16k<true>(S, tw);
        // park z_even, then build the odd-sample spectrum in place
        for (int k = threadIdx.x; k < kM; k += kThreads) {
            parkZ[k] = S[pad(k)];
            const float2 x = parkX[k];
            float2 y;
            if (k == 0) {
                const float2 a = cscale(__ldg(p.f_g), x.x);
                const float2 b = cscale(__ldg(p.f_g + kM), x.y);
                y = csub(a, b);
            } else {
                y = cmul(cmul(x, __ldg(p.f_g + k)), tw.w<true>(k));
            }
            S[pad(k)] = y;
        }
        __syncthreads();
        fft16k<true>(S, tw);

        // ---- FM discriminator: demod[2m] from (z_e[m], z_o[m-1]), demod[2m+1] from
        // (z_o[m], z_e[m]).  X is no longer needed, so its parking slot takes the
        // clipped demod (pairs) until every thread has read its neighbours.
        {
            float* oraw = p.o_raw ? p.o_raw + (long long)blk * p.s_video.len : nullptr;
            for (int m = threadIdx.x; m < kM; m += kThreads) {
                const float2 ze = parkZ[m];
                const float2 zo = S[pad(m)];
                const float de = (m == 0) ? 0.0f : fm_disc(ze, S[pad(m - 1)], kfs);
                const float dodd = fm_disc(zo, ze, kfs);
                if (oraw) {
                    const int i0 = 2 * m - p.s_video.start;
                    if (i0 >= 0 && i0 < p.s_video.len) oraw[i0] = de;
                    if (i0 + 1 >= 0 && i0 + 1 < p.s_video.len) oraw[i0 + 1] = dodd;
                }
                parkX[m] = make_float2(fminf(fmaxf(de, clip_lo), clip_hi),
                                       fminf(fmaxf(dodd, clip_lo), clip_hi));
            }
            __syncthreads();
            for (int m = threadIdx.x; m < kM; m += kThreads) S[pad(m)] = parkX[m];
            __syncthreads();
        }

        // ---- spectrum of the clipped demod, then the video outputs
        fft16k<false>(S, tw);
        r2c_post(S, tw);
        __syncthreads();
        bool first = true;
#pragma unroll
        for (int o = 0; o < OUT_NVIDEO; ++o) {
            if (p.o_video[o] == nullptr) continue;
            real_output(S, first ? nullptr : parkX, p.f_video[o], tw, first ? parkX : nullptr);
            write_real(S, p.o_video[o] + (long long)blk * p.s_video.len, p.s_video, p.roll[o]);
            __syncthreads();
            first = false;
        }
        __syncthreads();
    }
}

cudaError_t launch_demod(const DemodParams& p, int grid, cudaStream_t stream) {
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(demod_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)kSmemBytes);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    if (p.nblocks <= 0) return cudaSuccess;
    demod_kernel<<<grid, kThreads, kSmemBytes, stream>>>(p);
    return cudaGetLastError();
}

}  // namespace ldg
