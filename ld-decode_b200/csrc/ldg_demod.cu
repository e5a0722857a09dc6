// Fused per-block RF demodulator: one 1024-thread CTA per 32768-sample
// overlap-save block, persistent over blocks.
//
// Per block, in shared memory (a 16384-point complex working set S):
//   X = R2C(x)                         input spectrum, bins 0..N/2 (first FFT
//                                      pass reads the int16 block directly)
//   rfhpf  = C2R(X * Frfhpf)           -> float32 (last pass stores directly)
//   efm    = C2R(X * Fefm/2)           -> int16 (truncated)
//   audio  = 2 x (1024-bin sub-band * filt1 -> iFFT -> FM discriminator)
//   z      = analytic signal of X * RFVideo * MTF^m, as its even and odd
//            samples: two 16384-point inverse FFTs whose first pass reads
//            X * G (resp. X * G * W^-k) from the parked spectrum
//   demod_raw = arg(z[n] conj z[n-1]) * fs / 2pi, in [0, fs)
//   D      = R2C(clip(demod_raw, 1.5 MHz, 0.75 fs))
//   demod / demod_05 / demod_burst [/ demod_pilot] = C2R(D * F) with rolls
// The real-FFT pre/post-processing is fused with parking the spectrum and
// with the filter products; spectra and the even half of z are parked in a
// per-CTA global scratch (256 KB per CTA, L2 resident).  This restates
// RFDecode.demodblock_cpu (lddecode/core.py:755-879) and unwrap_hilbert
// (lddecode/utils.py:898-926).
#include "ldg_attr.cuh"
#include "ldg_demod.cuh"
#include "ldg_fft.cuh"
#include "ldg_fft_ip.cuh"

namespace ldg {

namespace {

constexpr float kTwoPi = 6.28318530717958647692f;
constexpr float kInvM = 1.0f / kM;

// arctan t for t in [0, 1]: the minimax polynomial of Abramowitz & Stegun,
// Handbook of Mathematical Functions, 4.4.49 (after Hastings): arctan t / t
// = 1 + a2 t^2 + ... + a16 t^16 with |error| <= 2e-8; in float32 Horner
// form within 1.6 ulp of arctan.
__device__ __forceinline__ float atan01(float t) {
    const float t2 = t * t;
    float p = 0.0028662257f;
    p = fmaf(p, t2, -0.0161657367f);
    p = fmaf(p, t2, 0.0429096138f);
    p = fmaf(p, t2, -0.0752896400f);
    p = fmaf(p, t2, 0.1065626393f);
    p = fmaf(p, t2, -0.1420889944f);
    p = fmaf(p, t2, 0.1999355085f);
    p = fmaf(p, t2, -0.3333314528f);
    p = fmaf(p, t2, 1.0f);
    return t * p;
}

// arg(re + i im) in [0, 2 pi): the octant's arctan of min/max, reflected
__device__ __forceinline__ float arg_2pi(float im, float re) {
    constexpr float kPi = 3.14159265358979323846f, kHalfPi = 1.57079632679489661923f;
    const float ax = fabsf(re), ay = fabsf(im);
    const float mx = fmaxf(ax, ay), mn = fminf(ax, ay);
    float r = atan01(mx > 0.0f ? mn / mx : 0.0f);
    if (ay > ax) r = kHalfPi - r;
    if (re < 0.0f) r = kPi - r;
    return im < 0.0f ? kTwoPi - r : r;
}

__device__ __forceinline__ float fm_disc(float2 a, float2 b, float k) {
    // arg(a * conj(b)) wrapped to [0, 2pi), times k = rate / 2pi
    const float re = fmaf(a.x, b.x, a.y * b.y);
    const float im = fmaf(a.y, b.x, -a.x * b.y);
    return arg_2pi(im, re) * k;
}

// ---- first-pass loaders

struct InLoader16 {  // x[2m], x[2m+1] from int16 samples
    const int16_t* x;
    __device__ float2 operator()(int, int m) const {
        const int w = __ldcs(reinterpret_cast<const int*>(x) + m);  // read once: streaming
        return make_float2((float)(int16_t)(w & 0xffff), (float)(int16_t)(((unsigned)w) >> 16));
    }
};

struct InLoader32 {  // float32 samples
    const float* x;
    __device__ float2 operator()(int, int m) const { return __ldg(reinterpret_cast<const float2*>(x) + m); }
};

struct ParkLoader {
    const float2* p;
    __device__ float2 operator()(int, int m) const { return p[m]; }
};

// X[k] * G[k] from the parked spectrum (X[0], X[M] packed in element 0);
// `odd` selects the odd-sample spectrum (G * W^-k, and X0 G0 - XM GM at 0).
struct AnalyticLoader {
    const float2* X;
    const float2* G;
    const float2* Godd;
    bool odd;
    __device__ float2 operator()(int, int k) const {
        const float2 x = X[k];
        if (k == 0) {
            const float2 a = cscale(__ldg(G), x.x);
            const float2 b = cscale(__ldg(G + kM), x.y);
            return odd ? csub(a, b) : cadd(a, b);
        }
        return cmul(x, __ldg((odd ? Godd : G) + k));
    }
};

// ---- last-pass storers (z[m] = M * (x[2m] + i x[2m+1]))

// Real output: sample n of the block goes to out[i], i = (n - roll - start) mod N, if i < len.
struct RealStorer {
    float* out;
    int start, len, roll;
    __device__ void operator()(int, int m, float2 v) const {
        const int i0 = (2 * m - roll - start) & (kN - 1);
        const int i1 = (i0 + 1) & (kN - 1);
        // streaming stores: outputs are not re-read here, keep L2 for the parked spectra
        if (((i0 & 1) == 0) && i0 + 1 < len && ((reinterpret_cast<uintptr_t>(out + i0) & 7) == 0)) {
            __stcs(reinterpret_cast<float2*>(out + i0), make_float2(v.x * kInvM, v.y * kInvM));
        } else {
            if (i0 < len) __stcs(out + i0, v.x * kInvM);
            if (i1 < len) __stcs(out + i1, v.y * kInvM);
        }
    }
};

__device__ __forceinline__ int16_t to_efm(float x) {
    x = fminf(fmaxf(x * kInvM, -32768.0f), 32767.0f);
    return (int16_t)__float2int_rz(x);
}

struct EfmStorer {
    int16_t* out;
    int start, len;
    __device__ void operator()(int, int m, float2 v) const {
        const int i0 = (2 * m - start) & (kN - 1);
        const int i1 = (i0 + 1) & (kN - 1);
        const short a = (short)to_efm(v.x), b = (short)to_efm(v.y);
        if (((i0 & 1) == 0) && i0 + 1 < len && ((reinterpret_cast<uintptr_t>(out + i0) & 3) == 0)) {
            // both samples in one aligned 32-bit store (little-endian: a first)
            __stcs(reinterpret_cast<int*>(out + i0), (int)(((unsigned)(unsigned short)b << 16) | (unsigned short)a));
        } else {
            if (i0 < len) __stcs(reinterpret_cast<short*>(out) + i0, a);
            if (i1 < len) __stcs(reinterpret_cast<short*>(out) + i1, b);
        }
    }
};

struct ParkStorer {
    float2* p;
    __device__ void operator()(int, int m, float2 v) const { p[m] = v; }
};

// ---- real-FFT pre/post-processing, fused with parking and filter products

// C2R pre-processing of the pair (H[k], H[M-k]) into the M-point complex
// spectrum whose inverse FFT is M * (x[2m] + i x[2m+1]).
__device__ __forceinline__ void c2r_pair(float2* S, int k, float2 hk, float2 hm, float2 wk) {
    const float2 e = make_float2(0.5f * (hk.x + hm.x), 0.5f * (hk.y - hm.y));
    const float2 d = make_float2(0.5f * (hk.x - hm.x), 0.5f * (hk.y + hm.y));
    const float2 o = cmul(d, cconj(wk));
    S[pad(k)] = make_float2(e.x - o.y, e.y + o.x);
    if (k != kM / 2) S[pad(kM - k)] = make_float2(e.x + o.y, o.x - e.y);
}

__device__ __forceinline__ void c2r_dc(float2* S, float x0, float xm, const float2* F) {
    const float h0 = x0 * __ldg(&F[0].x), hm = xm * __ldg(&F[kM].x);
    S[0] = make_float2(0.5f * (h0 + hm), 0.5f * (h0 - hm));
}

struct AudioTaps {
    float2* A;             // two padded 1024-point sets
    int lowbin[2];
    const float2* filt1[2];
};

// Post-processing of one bin pair (k, M-k), 0 < k <= M/2, from Z[k], Z[M-k]
// (S), the real-FFT twiddle wk and, if F is given, the filter bins.
__device__ __forceinline__ void post_pair(float2* S, float2* park, const AudioTaps* au, int k, float2 zk, float2 zm,
                                          float2 wk, const float2* F, float2 fk, float2 fm) {
    const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    const float2 o = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
    const float2 tt = cmul(wk, o);
    const float2 xk = cadd(e, tt);
    const float2 xm = cconj(csub(e, tt));
    park[k] = xk;
    if (k != kM / 2) park[kM - k] = xm;
    if (au) {
#pragma unroll
        for (int ch = 0; ch < 2; ++ch) {
            const int rel = k - au->lowbin[ch];
            if (rel >= 0 && rel <= 512) {
                const float2 xb = rel < 512 ? xk : cconj(xk);
                au->A[ch * padded(1024) + pad(rel)] = cmul(xb, __ldg(au->filt1[ch] + rel));
            }
        }
    }
    if (F) c2r_pair(S, k, cmul(xk, fk), cmul(xm, fm), wk);
}

// S holds Z = FFT_M(x[2m] + i x[2m+1]).  Computes X[k] for k = 0..M, parks
// it, taps the audio sub-bands and, if F is given, leaves the C2R input of
// X * F in S.  Thread t handles k = t + kThreads i; two bins per step with all
// their loads issued before the arithmetic (latency of the global twiddle
// and filter loads overlapped).
__device__ void post_r2c(float2* S, const Tables& t, float2* park, const float2* F, const AudioTaps* au) {
    const int t0 = threadIdx.x;
    const float2 zero = make_float2(0.f, 0.f);
#pragma unroll 1
    for (int i = 0; i < kM / 2 / kThreads; i += 2) {
        const int ka = t0 + i * kThreads, kb = ka + kThreads;  // kb > 0; ka == 0 only for thread 0
        const float2 zka = S[pad(ka)];
        const float2 zma = ka ? S[pad(kM - ka)] : zero;
        const float2 zkb = S[pad(kb)], zmb = S[pad(kM - kb)];
        const float2 wa = __ldg(t.t32 + ka), wb = __ldg(t.t32 + kb);
        float2 fka = zero, fma = zero, fkb = zero, fmb = zero;
        if (F) {
            fka = __ldg(F + ka);
            fma = __ldg(F + kM - ka);
            fkb = __ldg(F + kb);
            fmb = __ldg(F + kM - kb);
        }
        if (ka == 0) {
            const float x0 = zka.x + zka.y, xm = zka.x - zka.y;
            park[0] = make_float2(x0, xm);
            if (F) c2r_dc(S, x0, xm, F);
        } else {
            post_pair(S, park, au, ka, zka, zma, wa, F, fka, fma);
        }
        post_pair(S, park, au, kb, zkb, zmb, wb, F, fkb, fmb);
    }
    if (t0 == 0) {  // k = M/2
        const int k = kM / 2;
        const float2 z = S[pad(k)];
        post_pair(S, park, au, k, z, z, __ldg(t.t32 + k), F, F ? __ldg(F + k) : zero, F ? __ldg(F + k) : zero);
    }
}

// Is the bin pair (k, M - k) inside the band [klo, khi] where the filter's
// float32 bins are not zero?  (Outside it X * F is zero and so is the C2R
// input; for a band-limited filter such as the EFM one most pairs are.)
__device__ __forceinline__ bool pair_live(int k, int klo, int khi) {
    const int m = k == 0 ? kM : kM - k;
    return (k >= klo && k <= khi) || (m >= klo && m <= khi);
}

// C2R input of X * F in S, X from the parked spectrum; two bins per step,
// loads first.  Pairs outside F's band [klo, khi] are written as zeros
// without their loads.
__device__ void pre_c2r(float2* S, const Tables& t, const float2* park, const float2* F, int klo = 0,
                        int khi = kM) {
    const int t0 = threadIdx.x;
    const float2 zero = make_float2(0.f, 0.f);
#pragma unroll 1
    for (int i = 0; i < kM / 2 / kThreads; i += 2) {
        const int ka = t0 + i * kThreads, kb = ka + kThreads;
        if (!pair_live(ka, klo, khi) && !pair_live(kb, klo, khi)) {
            S[pad(ka)] = zero;
            if (ka) S[pad(kM - ka)] = zero;
            S[pad(kb)] = zero;
            S[pad(kM - kb)] = zero;
            continue;
        }
        const float2 xka = park[ka], xkb = park[kb], xmb = park[kM - kb];
        const float2 xma = ka ? park[kM - ka] : xka;
        const float2 fka = __ldg(F + ka), fma = __ldg(F + kM - ka), fkb = __ldg(F + kb), fmb = __ldg(F + kM - kb);
        const float2 wa = __ldg(t.t32 + ka), wb = __ldg(t.t32 + kb);
        if (ka == 0) {
            c2r_dc(S, xka.x, xka.y, F);
        } else {
            c2r_pair(S, ka, cmul(xka, fka), cmul(xma, fma), wa);
        }
        c2r_pair(S, kb, cmul(xkb, fkb), cmul(xmb, fmb), wb);
    }
    if (t0 == 0) {
        const int k = kM / 2;
        if (pair_live(k, klo, khi)) {
            const float2 x = park[k];
            c2r_pair(S, k, cmul(x, __ldg(F + k)), cmul(x, __ldg(F + k)), __ldg(t.t32 + k));
        } else {
            S[pad(k)] = zero;
        }
    }
}

__device__ void audio_stage(const DemodParams& p, float2* A, const Tables& t, int blk) {
    constexpr int stride = padded(1024);
    fft1k_x2<true>(A, t);
    const float kk = p.a_rate / kTwoPi;
    for (int idx = threadIdx.x; idx < 2 * 1024; idx += kThreads) {
        const int ch = idx >> 10, n = idx & 1023;
        const int i = n - p.s_audio.start;
        float* oa = ch ? p.o_audio[1] : p.o_audio[0];
        if (i < 0 || i >= p.s_audio.len || oa == nullptr) continue;
        const float2* Ab = A + ch * stride;
        const float d = (n == 0) ? 0.0f : fm_disc(Ab[pad(n)], Ab[pad(n - 1)], kk);
        __stcs(oa + (long long)blk * p.s_audio.len + i, d + (ch ? p.a_low[1] : p.a_low[0]));
    }
}

// PAL_V4300D_NotchFilter (lddecode/core.py:774-798) on the parked input
// spectrum: in bins [lo, hi), every bin whose magnitude exceeds the band's
// mean + 3 std (FP64, population std) is zeroed with its two neighbours; the
// mirrored negative-frequency bins are implicit in the half spectrum.  One
// warp; the decisions use the magnitudes before any bin is zeroed.  At most
// 1024 bins (checked on the host).
__device__ void notch_park(float2* park, int lo, int hi) {
    if (threadIdx.x >= 32) return;
    const int lane = threadIdx.x;
    const int n = hi - lo;
    auto mag = [&](int i) {
        const float2 x = park[lo + i];
        return sqrt((double)x.x * (double)x.x + (double)x.y * (double)x.y);
    };
    double s = 0.0;
    for (int i = lane; i < n; i += 32) s += mag(i);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    const double mean = s / (double)n;
    double q = 0.0;
    for (int i = lane; i < n; i += 32) {
        const double d = mag(i) - mean;
        q += d * d;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
    const double m = mean + sqrt(q / (double)n) * 3.0;
    unsigned flags = 0;
    for (int i = lane, j = 0; i < n; i += 32, ++j)
        if (mag(i) > m) flags |= 1u << j;
    __syncwarp();
    for (int i = lane, j = 0; i < n; i += 32, ++j) {
        if ((flags >> j) & 1u) {
            const float2 z = make_float2(0.f, 0.f);
            park[lo + i - 1] = z;
            park[lo + i] = z;
            park[lo + i + 1] = z;
        }
    }
}

// Invalidate this CTA's scratch (parkX and parkZ, kScratchPerCta bytes,
// 128-byte aligned) in L2 without write-back: discard.global.L2 per 128-byte
// line.  Every thread of the CTA is past its last scratch access.
__device__ __forceinline__ void discard_scratch(float2* base) {
    char* b = reinterpret_cast<char*>(base);
    constexpr int kLines = (int)(kScratchPerCta / 128);
    for (int l = threadIdx.x; l < kLines; l += kThreads)
        asm volatile("discard.global.L2 [%0], 128;" ::"l"(b + (size_t)l * 128) : "memory");
}

// FM discriminator: demod[2m] from (z_e[m], z_o[m-1]), demod[2m+1] from
// (z_o[m], z_e[m]) -- the even samples parked (parkZ), the odd ones in S,
// both in natural order; the clipped pairs replace X in the parking slot.
__device__ __forceinline__ void discriminate(const DemodParams& p, int blk, const float2* S, float2* parkX,
                                             const float2* parkZ) {
    {
        const float kfs = p.fs_hz / kTwoPi;
        const float clip_hi = p.fs_hz * 0.75f;
        float* oraw = p.o_raw ? p.o_raw + (long long)blk * p.s_video.len : nullptr;
        const int vs = p.s_video.start, vl = p.s_video.len;
        auto disc_store = [&](int m, float de, float dodd) {
            if (oraw) {
                const int i0 = 2 * m - vs;
                if (i0 >= 0 && i0 + 1 < vl && ((reinterpret_cast<uintptr_t>(oraw + i0) & 7) == 0)) {
                    __stcs(reinterpret_cast<float2*>(oraw + i0), make_float2(de, dodd));
                } else {
                    if (i0 >= 0 && i0 < vl) __stcs(oraw + i0, de);
                    if (i0 + 1 >= 0 && i0 + 1 < vl) __stcs(oraw + i0 + 1, dodd);
                }
            }
            parkX[m] = make_float2(fminf(fmaxf(de, 1500000.0f), clip_hi), fminf(fmaxf(dodd, 1500000.0f), clip_hi));
        };
        // two samples per step, the parked (L2) loads first
#pragma unroll 2
        for (int m = threadIdx.x; m < kM; m += 2 * kThreads) {
            const int mb = m + kThreads;
            const float2 zea = parkZ[m], zeb = parkZ[mb];
            const float2 zoa = S[pad(m)], zob = S[pad(mb)];
            const float2 zpa = m ? S[pad(m - 1)] : zoa, zpb = S[pad(mb - 1)];
            const float dea = (m == 0) ? 0.0f : fm_disc(zea, zpa, kfs);
            const float doa = fm_disc(zoa, zea, kfs);
            const float deb = fm_disc(zeb, zpb, kfs);
            const float dob = fm_disc(zob, zeb, kfs);
            disc_store(m, dea, doa);
            disc_store(mb, deb, dob);
        }
    }
}

// One block: every requested output of block `blk` of p.  parkX/parkZ: this
// CTA's scratch (kScratchPerCta).  Ends with the CTA's threads in step.
__device__ __forceinline__ void demod_block(const DemodParams& p, int blk, float2* S, float2* A, const Tables& t,
                                            float2* parkX, float2* parkZ) {
    // ---- input spectrum X (first pass reads the block), parked; audio taps; rfhpf input
    if (p.in_kind == 0) {
        fft16k<false>(S, t, InLoader16{static_cast<const int16_t*>(p.in) + (long long)blk * p.in_stride});
    } else {
        fft16k<false>(S, t, InLoader32{static_cast<const float*>(p.in) + (long long)blk * p.in_stride});
    }
    if (p.audio) {
        for (int idx = threadIdx.x; idx < 2 * 511; idx += kThreads) {
            const int ch = idx / 511, k = 513 + idx % 511;
            A[ch * padded(1024) + pad(k)] = make_float2(0.f, 0.f);
        }
    }
    {
        AudioTaps au{A, {p.a_lowbin[0], p.a_lowbin[1]}, {p.a_filt1[0], p.a_filt1[1]}};
        post_r2c(S, t, parkX, p.o_rfhpf ? p.f_rfhpf : nullptr, p.audio ? &au : nullptr);
    }
    __syncthreads();
    // rfhpf (already in S) and the audio taps use the spectrum before the
    // notch, as the reference does (its notch band lies far from the audio bands)
    if (p.notch_hi > p.notch_lo) {
        notch_park(parkX, p.notch_lo, p.notch_hi);
        __syncthreads();
    }
    if (p.audio) audio_stage(p, A, t, blk);

    // ---- rfhpf
    if (p.o_rfhpf) {
        fft16k<true>(S, t, SmemIO(),
                     RealStorer{p.o_rfhpf + (long long)blk * p.s_rfhpf.len, p.s_rfhpf.start, p.s_rfhpf.len, 0});
    }

    // ---- EFM
    if (p.o_efm) {
        pre_c2r(S, t, parkX, p.f_efm, p.efm_klo, p.efm_khi);
        __syncthreads();
        fft16k<true>(S, t, SmemIO(), EfmStorer{p.o_efm + (long long)blk * p.s_efm.len, p.s_efm.start, p.s_efm.len});
    }

    // ---- analytic signal: even samples (parked), then odd samples (in S)
    fft16k<true>(S, t, AnalyticLoader{parkX, p.f_g, p.f_godd, false}, ParkStorer{parkZ});
    fft16k<true>(S, t, AnalyticLoader{parkX, p.f_g, p.f_godd, true});

    discriminate(p, blk, S, parkX, parkZ);
    __syncthreads();

    // ---- spectrum D of the clipped demod, then the video outputs
    fft16k<false>(S, t, ParkLoader{parkX});
    int first = -1;
#pragma unroll
    for (int o = 0; o < OUT_NVIDEO; ++o)
        if (first < 0 && p.o_video[o]) first = o;
    post_r2c(S, t, parkX, first >= 0 ? p.f_video[first] : nullptr, nullptr);
    __syncthreads();
#pragma unroll
    for (int o = 0; o < OUT_NVIDEO; ++o) {
        if (p.o_video[o] == nullptr) continue;
        if (o != first) {
            pre_c2r(S, t, parkX, p.f_video[o]);
            __syncthreads();
        }
        fft16k<true>(S, t, SmemIO(),
                     RealStorer{p.o_video[o] + (long long)blk * p.s_video.len, p.s_video.start, p.s_video.len,
                                p.roll[o]});
    }
    __syncthreads();
    // the parked spectra are dead: drop their L2 lines without writing them
    // back (the next block on this scratch writes before it reads)
    discard_scratch(parkX);
}

struct CtaSmem {
    float2* S;
    float2* A;
    Tables t;       // Stockham pass tables (t.s3 / t.s4 only for the Stockham variant) and the 1024-point ones
    ip::Twiddles tw;  // in-place stage tables (in-place variant)
};

// Carves the dynamic shared memory -- working set, audio bands, 1024-point
// tables, then the 16384-point tables of the variant -- and loads the tables.
template <int V>
__device__ __forceinline__ CtaSmem cta_setup(float2* smem, const float2* tw16, const float2* tw32) {
    CtaSmem c;
    c.S = smem;
    c.A = smem + padded(kM);
    float2* s2 = c.A + 2 * padded(1024);
    float2* s4a = s2 + kS2;
    float2* rest = s4a + kS4a;
    load_1k_tables(s2, s4a, tw16);
    c.t.t16 = tw16;
    c.t.t32 = tw32;
    c.t.s2 = s2;
    c.t.s4a = s4a;
    if (V == kVariantStockham) {
        float2* s3 = rest;
        float2* s4 = s3 + kS3;
        load_pass_tables(s3, s4, tw16);
        c.t.s3 = s3;
        c.t.s4 = s4;
        c.tw = {nullptr, nullptr, nullptr};
    } else {
        float2* t1 = rest;
        float2* t2 = t1 + ip::kT1;
        float2* t3 = t2 + ip::kT2;
        ip::load_stage_tables(t1, t2, t3, tw16);
        c.tw = {t1, t2, t3};
        c.t.s3 = nullptr;
        c.t.s4 = nullptr;
    }
    __syncthreads();
    return c;
}

// ---- the in-place variant: spectra in position order (ldg_fft_ip.cuh)

// X[k] * G[k] at positions p .. p+3 (k = bin_of(p)) from the parked spectrum
// (position order, X[0] and X[M] packed at position 0) and G at positions;
// `odd` as AnalyticLoader.
struct AnalyticLoaderIp {
    const float2* X;
    const float2* Gpos;
    const float2* G;  // natural order: G[0], G[M]
    bool odd;
    __device__ void quad(int p, float2 (&v)[4]) const {
        const float4 x01 = *reinterpret_cast<const float4*>(X + p);
        const float4 x23 = *reinterpret_cast<const float4*>(X + p + 2);
        const float4 g01 = __ldg(reinterpret_cast<const float4*>(Gpos + p));
        const float4 g23 = __ldg(reinterpret_cast<const float4*>(Gpos + p + 2));
        v[0] = cmul(make_float2(x01.x, x01.y), make_float2(g01.x, g01.y));
        v[1] = cmul(make_float2(x01.z, x01.w), make_float2(g01.z, g01.w));
        v[2] = cmul(make_float2(x23.x, x23.y), make_float2(g23.x, g23.y));
        v[3] = cmul(make_float2(x23.z, x23.w), make_float2(g23.z, g23.w));
        if (p == 0) {
            const float2 a = cscale(__ldg(G), x01.x);
            const float2 b = cscale(__ldg(G + kM), x01.y);
            v[0] = odd ? csub(a, b) : cadd(a, b);
        }
    }
};

// C2R pre-processing of one bin pair at positions p (bin k) and q (bin M-k)
// (c2r_pair in position order; p == q for k = M/2).
__device__ __forceinline__ void c2r_pair_ip(float2* S, int p, int q, float2 hk, float2 hm, float2 wk) {
    const float2 e = make_float2(0.5f * (hk.x + hm.x), 0.5f * (hk.y - hm.y));
    const float2 d = make_float2(0.5f * (hk.x - hm.x), 0.5f * (hk.y + hm.y));
    const float2 o = cmul(d, cconj(wk));
    S[pad(p)] = make_float2(e.x - o.y, e.y + o.x);
    if (q != p) S[pad(q)] = make_float2(e.x + o.y, o.x - e.y);
}

// post_pair in position order: X[k], X[M-k] of the pair at (p, q) from
// Z[k] = S[p], Z[M-k] = S[q]; parked at p and q; the audio taps use the
// pair's bin at or below M/2; with F, the C2R input of X * F left at p, q.
__device__ __forceinline__ void post_pair_ip(float2* S, float2* park, const AudioTaps* au, int p, int q, float2 zk,
                                             float2 zm, float2 wk, bool hasF, float4 f) {
    const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    const float2 o = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
    const float2 tt = cmul(wk, o);
    const float2 xk = cadd(e, tt);
    const float2 xm = cconj(csub(e, tt));
    park[p] = xk;
    if (q != p) park[q] = xm;
    if (au) {
        const int k = ip::bin_of(p);
        const bool low = k <= kM / 2;
        const int kk = low ? k : kM - k;
        const float2 xkk = low ? xk : xm;
#pragma unroll
        for (int ch = 0; ch < 2; ++ch) {
            const int rel = kk - au->lowbin[ch];
            if (rel >= 0 && rel <= 512) {
                const float2 xb = rel < 512 ? xkk : cconj(xkk);
                au->A[ch * padded(1024) + pad(rel)] = cmul(xb, __ldg(au->filt1[ch] + rel));
            }
        }
    }
    if (hasF) c2r_pair_ip(S, p, q, cmul(xk, make_float2(f.x, f.y)), cmul(xm, make_float2(f.z, f.w)), wk);
}

// post_r2c in position order: S holds Z at positions; parks X (position
// order), taps the audio bands and, with FP, leaves the C2R input of X * F
// in S.  Thread t takes pairs u = t + kThreads i, two per step, loads first.
__device__ void post_r2c_ip(float2* S, const float2* twp, float2* park, const float4* FP, const AudioTaps* au) {
    const int t0 = threadIdx.x;
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll 1
    for (int i = 0; i < 8; i += 2) {
        const int ua = t0 + i * kThreads, ub = ua + kThreads;
        const int pa = ip::pair_pos(ua), pb = ip::pair_pos(ub);
        const int qa = ip::partner_pos(pa), qb = ip::partner_pos(pb);
        const float2 zka = S[pad(pa)], zma = S[pad(qa)];
        const float2 zkb = S[pad(pb)], zmb = S[pad(qb)];
        const float2 wa = __ldg(twp + ua), wb = __ldg(twp + ub);
        float4 fa = zero4, fb = zero4;
        if (FP) {
            fa = __ldg(FP + ua);
            fb = __ldg(FP + ub);
        }
        if (pa != 0) post_pair_ip(S, park, au, pa, qa, zka, zma, wa, FP != nullptr, fa);
        if (pb != 0) {
            post_pair_ip(S, park, au, pb, qb, zkb, zmb, wb, FP != nullptr, fb);
        } else {  // bins 0 and M
            const float x0 = zkb.x + zkb.y, xm = zkb.x - zkb.y;
            park[0] = make_float2(x0, xm);
            if (FP) {
                const float h0 = x0 * fb.x, hm = xm * fb.z;
                S[0] = make_float2(0.5f * (h0 + hm), 0.5f * (h0 - hm));
            }
        }
    }
    if (t0 == 0) {  // u = M/2: position 2, bin M/2, its own partner
        const int u = kM / 2;
        const float2 z = S[pad(2)];
        post_pair_ip(S, park, au, 2, 2, z, z, __ldg(twp + u), FP != nullptr, FP ? __ldg(FP + u) : zero4);
    }
}

// pre_c2r in position order: the C2R input of X * F in S, X from the parked
// spectrum (position order).
__device__ void pre_c2r_ip(float2* S, const float2* twp, const float2* park, const float4* FP, int klo = 0,
                           int khi = kM) {
    const int t0 = threadIdx.x;
    const float2 zero = make_float2(0.f, 0.f);
#pragma unroll 1
    for (int i = 0; i < 8; i += 2) {
        const int ua = t0 + i * kThreads, ub = ua + kThreads;
        const int pa = ip::pair_pos(ua), pb = ip::pair_pos(ub);
        const int qa = ip::partner_pos(pa), qb = ip::partner_pos(pb);
        if (!pair_live(ip::bin_of(pa), klo, khi) && !pair_live(ip::bin_of(pb), klo, khi)) {
            // pa is never position 0 (ua < 7680); pb is for the pair of bins 0 and M
            S[pad(pa)] = zero;
            if (qa != pa) S[pad(qa)] = zero;
            S[pad(pb)] = zero;
            if (pb != 0 && qb != pb) S[pad(qb)] = zero;
            continue;
        }
        const float2 xka = park[pa], xma = park[qa], xkb = park[pb], xmb = park[qb];
        const float4 fa = __ldg(FP + ua), fb = __ldg(FP + ub);
        const float2 wa = __ldg(twp + ua), wb = __ldg(twp + ub);
        c2r_pair_ip(S, pa, qa, cmul(xka, make_float2(fa.x, fa.y)), cmul(xma, make_float2(fa.z, fa.w)), wa);
        if (pb != 0) {
            c2r_pair_ip(S, pb, qb, cmul(xkb, make_float2(fb.x, fb.y)), cmul(xmb, make_float2(fb.z, fb.w)), wb);
        } else {
            const float h0 = xkb.x * fb.x, hm = xkb.y * fb.z;
            S[0] = make_float2(0.5f * (h0 + hm), 0.5f * (h0 - hm));
        }
    }
    if (t0 == 0) {
        const int u = kM / 2;
        if (pair_live(kM / 2, klo, khi)) {
            const float2 x = park[2];
            const float4 f = __ldg(FP + u);
            c2r_pair_ip(S, 2, 2, cmul(x, make_float2(f.x, f.y)), cmul(x, make_float2(f.z, f.w)), __ldg(twp + u));
        } else {
            S[pad(2)] = zero;
        }
    }
}

// notch_park on the position-order parked spectrum.
__device__ void notch_park_ip(float2* park, int lo, int hi) {
    if (threadIdx.x >= 32) return;
    const int lane = threadIdx.x;
    const int n = hi - lo;
    auto mag = [&](int i) {
        const float2 x = park[ip::pos_of(lo + i)];
        return sqrt((double)x.x * (double)x.x + (double)x.y * (double)x.y);
    };
    double s = 0.0;
    for (int i = lane; i < n; i += 32) s += mag(i);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    const double mean = s / (double)n;
    double q = 0.0;
    for (int i = lane; i < n; i += 32) {
        const double d = mag(i) - mean;
        q += d * d;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
    const double m = mean + sqrt(q / (double)n) * 3.0;
    unsigned flags = 0;
    for (int i = lane, j = 0; i < n; i += 32, ++j)
        if (mag(i) > m) flags |= 1u << j;
    __syncwarp();
    for (int i = lane, j = 0; i < n; i += 32, ++j) {
        if ((flags >> j) & 1u) {
            const float2 z = make_float2(0.f, 0.f);
            park[ip::pos_of(lo + i - 1)] = z;
            park[ip::pos_of(lo + i)] = z;
            park[ip::pos_of(lo + i + 1)] = z;
        }
    }
}

// demod_block with the in-place transforms: the same outputs from the same
// steps, spectra in position order.
__device__ __forceinline__ void demod_block_ip(const DemodParams& p, int blk, float2* S, float2* A, const Tables& t,
                                               const ip::Twiddles& tw, float2* parkX, float2* parkZ) {
    if (p.in_kind == 0) {
        ip::fft16k_fwd(S, tw, InLoader16{static_cast<const int16_t*>(p.in) + (long long)blk * p.in_stride});
    } else {
        ip::fft16k_fwd(S, tw, InLoader32{static_cast<const float*>(p.in) + (long long)blk * p.in_stride});
    }
    if (p.audio) {
        for (int idx = threadIdx.x; idx < 2 * 511; idx += kThreads) {
            const int ch = idx / 511, k = 513 + idx % 511;
            A[ch * padded(1024) + pad(k)] = make_float2(0.f, 0.f);
        }
    }
    post_r2c_ip(S, p.tw_pair, parkX, p.o_rfhpf ? p.fp_rfhpf : nullptr, nullptr);
    __syncthreads();
    if (p.audio) {
        // the audio bands' bins, gathered from the parked spectrum (before the
        // notch, as the taps in post_r2c of the Stockham form): one L2 load per
        // thread instead of a band test in every bin pair's post-processing
        for (int idx = threadIdx.x; idx < 2 * 513; idx += kThreads) {
            const int ch = idx >= 513, rel = idx - 513 * ch;
            const float2 x = parkX[ip::pos_of(p.a_lowbin[ch] + rel)];
            A[ch * padded(1024) + pad(rel)] = cmul(rel < 512 ? x : cconj(x), __ldg(p.a_filt1[ch] + rel));
        }
        __syncthreads();
    }
    if (p.notch_hi > p.notch_lo) {
        notch_park_ip(parkX, p.notch_lo, p.notch_hi);
        __syncthreads();
    }
    if (p.audio) audio_stage(p, A, t, blk);

    if (p.o_rfhpf) {
        ip::fft16k_inv(S, tw, SmemIO(),
                       RealStorer{p.o_rfhpf + (long long)blk * p.s_rfhpf.len, p.s_rfhpf.start, p.s_rfhpf.len, 0});
    }
    if (p.o_efm) {
        pre_c2r_ip(S, p.tw_pair, parkX, p.fp_efm, p.efm_klo, p.efm_khi);
        __syncthreads();
        ip::fft16k_inv(S, tw, SmemIO(),
                       EfmStorer{p.o_efm + (long long)blk * p.s_efm.len, p.s_efm.start, p.s_efm.len});
    }

    ip::fft16k_inv(S, tw, AnalyticLoaderIp{parkX, p.g_pos, p.f_g, false}, ParkStorer{parkZ});
    ip::fft16k_inv(S, tw, AnalyticLoaderIp{parkX, p.godd_pos, p.f_g, true});

    discriminate(p, blk, S, parkX, parkZ);
    __syncthreads();

    ip::fft16k_fwd(S, tw, ParkLoader{parkX});
    int first = -1;
#pragma unroll
    for (int o = 0; o < OUT_NVIDEO; ++o)
        if (first < 0 && p.o_video[o]) first = o;
    post_r2c_ip(S, p.tw_pair, parkX, first >= 0 ? p.fp_video[first] : nullptr, nullptr);
    __syncthreads();
#pragma unroll
    for (int o = 0; o < OUT_NVIDEO; ++o) {
        if (p.o_video[o] == nullptr) continue;
        if (o != first) {
            pre_c2r_ip(S, p.tw_pair, parkX, p.fp_video[o]);
            __syncthreads();
        }
        ip::fft16k_inv(S, tw, SmemIO(),
                       RealStorer{p.o_video[o] + (long long)blk * p.s_video.len, p.s_video.start, p.s_video.len,
                                  p.roll[o]});
    }
    __syncthreads();
    discard_scratch(parkX);
}

template <int V>
__device__ __forceinline__ void run_block(const DemodParams& p, int blk, const CtaSmem& c, float2* parkX,
                                          float2* parkZ) {
    if (V == kVariantStockham) {
        demod_block(p, blk, c.S, c.A, c.t, parkX, parkZ);
    } else {
        demod_block_ip(p, blk, c.S, c.A, c.t, c.tw, parkX, parkZ);
    }
}

}  // namespace

namespace {

template <int V>
__device__ __forceinline__ void demod_body(const DemodParams& p, float2* smem) {
    const CtaSmem c = cta_setup<V>(smem, p.tw16, p.tw32);

    __shared__ int s_got;
    const bool per_block = p.slot_lock != nullptr;
    const int slot = per_block ? (int)(blockIdx.x % (unsigned)p.nslots) : (int)blockIdx.x;
    if (per_block) {
        if (threadIdx.x == 0) {
            int got = 0;
            for (int tries = 0; tries < (1 << 22); ++tries) {
                if (atomicCAS(p.slot_lock + slot, 0, 1) == 0) {
                    got = 1;
                    break;
                }
                __nanosleep(256);
            }
            if (!got) atomicOr(p.error, kDemodErrSlotWait);
            __threadfence();
            s_got = got;
        }
        __syncthreads();
        if (!s_got) return;
    }
    int blk = per_block ? (int)blockIdx.x * p.blocks_per_cta : (int)blockIdx.x;
    const int blk_end = per_block ? min(blk + p.blocks_per_cta, p.nblocks) : p.nblocks;
    const int blk_step = per_block ? 1 : (int)gridDim.x;
    float2* parkX = p.scratch + (size_t)slot * 2 * kM;
    float2* parkZ = parkX + kM;
    for (; blk < blk_end; blk += blk_step) run_block<V>(p, blk, c, parkX, parkZ);
    if (per_block) {
        // every thread is done with the slot's scratch before it is handed on
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            atomicExch(p.slot_lock + slot, 0);
        }
    }
}

// Persistent CTAs over a device work queue of blocks of many captures: each
// CTA pops `grab` consecutive global block indices at a time from *head,
// finds the capture that holds each (binary search over first_block), keeps
// that capture's parameters in shared memory, and demodulates the block.
template <int V>
__device__ __forceinline__ void queue_body(const QueueParams& q, float2* smem) {
    const CtaSmem c = cta_setup<V>(smem, q.tw16, q.tw32);
    __shared__ DemodParams sp;
    __shared__ long long s_pop;
    __shared__ int s_item;
    float2* parkX = q.scratch + (size_t)blockIdx.x * 2 * kM;
    float2* parkZ = parkX + kM;
    int cur = -1;
    for (;;) {
        if (threadIdx.x == 0) s_pop = (long long)atomicAdd(q.head, (unsigned long long)q.grab);
        __syncthreads();
        const long long g0 = s_pop;
        if (g0 >= q.total) break;
        const long long g1 = min(g0 + (long long)q.grab, q.total);
        for (long long g = g0; g < g1; ++g) {
            if (threadIdx.x == 0) {
                int lo = 0, hi = q.nitems - 1;  // last item whose first block is <= g
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (q.first_block[mid] <= g) lo = mid; else hi = mid - 1;
                }
                s_item = lo;
            }
            __syncthreads();
            const int it = s_item;
            if (it != cur) {
                const int* src = reinterpret_cast<const int*>(q.items + it);
                int* dst = reinterpret_cast<int*>(&sp);
                for (int w = threadIdx.x; w < (int)(sizeof(DemodParams) / sizeof(int)); w += kThreads) dst[w] = src[w];
                cur = it;
                __syncthreads();
            }
            run_block<V>(sp, (int)(g - q.first_block[it]), c, parkX, parkZ);
        }
    }
}

}  // namespace

// The demodulator with the Stockham transforms (natural-order spectra).
__global__ void __launch_bounds__(kThreads, 1) demod_kernel(const __grid_constant__ DemodParams p) {
    extern __shared__ float2 smem[];
    demod_body<kVariantStockham>(p, smem);
}

// The demodulator with the in-place transforms (position-order spectra).
__global__ void __launch_bounds__(kThreads, 1) demod_ip_kernel(const __grid_constant__ DemodParams p) {
    extern __shared__ float2 smem[];
    demod_body<kVariantInPlace>(p, smem);
}

__global__ void __launch_bounds__(kThreads, 1) demod_queue_kernel(const __grid_constant__ QueueParams q) {
    extern __shared__ float2 smem[];
    queue_body<kVariantStockham>(q, smem);
}

__global__ void __launch_bounds__(kThreads, 1) demod_queue_ip_kernel(const __grid_constant__ QueueParams q) {
    extern __shared__ float2 smem[];
    queue_body<kVariantInPlace>(q, smem);
}

// ---- analog audio stage 2 (RFDecode.runfilter_audio_phase2, core.py:884-915)

namespace {

// raw[j] = x[j] - carrier (float32), zero where a left-channel spike is
// within 8 samples or beyond the segment (the transform's zero padding)
struct Audio2Loader {
    const float* x;
    float cf;
    int n;
    const unsigned* mask;
    __device__ float val(int j) const {
        if (j >= n || ((mask[j >> 5] >> (j & 31)) & 1u)) return 0.0f;
        return __ldg(x + j) - cf;
    }
    __device__ float2 operator()(int, int m) const { return make_float2(val(2 * m), val(2 * m + 1)); }
};

struct Audio2Storer {
    float* out;
    double cf;
    int n;
    __device__ void operator()(int, int m, float2 v) const {
        const int j = 2 * m;
        if (j < n) out[j] = (float)((double)(v.x * kInvM) + cf);
        if (j + 1 < n) out[j + 1] = (float)((double)(v.y * kInvM) + cf);
    }
};

// Input spectrum from Z (as post_r2c), times the filter, into the C2R input
// (no parking).
__device__ void audio2_filter(float2* S, const Tables& t, const float2* F) {
    for (int k = threadIdx.x; k <= kM / 2; k += kThreads) {
        if (k == 0) {
            const float2 z = S[0];
            c2r_dc(S, z.x + z.y, z.x - z.y, F);
            continue;
        }
        const float2 zk = S[pad(k)], zm = S[pad(kM - k)];
        const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        const float2 o = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
        const float2 wk = __ldg(t.t32 + k);
        const float2 tt = cmul(wk, o);
        const float2 xk = cadd(e, tt);
        const float2 xm = cconj(csub(e, tt));
        c2r_pair(S, k, cmul(xk, __ldg(F + k)), cmul(xm, __ldg(F + kM - k)), wk);
    }
}

}  // namespace

// One CTA per (segment, channel): the left channel's spikes (findpeaks,
// utils.py:1207-1216: samples above 500 kHz from the carrier rising above
// the segment's last value) mark +-8 samples that are zeroed in both
// channels; then R2C, the stage-2 filter, C2R, carrier added back.
__global__ void __launch_bounds__(kThreads, 1) audio2_kernel(const __grid_constant__ Audio2Params p) {
    extern __shared__ float2 smem[];
    const CtaSmem c = cta_setup<kVariantStockham>(smem, p.tw16, p.tw32);
    const Audio2Seg sg = p.segs[blockIdx.x];
    const int ch = blockIdx.y;
    const int n = sg.len;
    unsigned* mask = reinterpret_cast<unsigned*>(c.A);  // kN bits in the audio-band area
    for (int w = threadIdx.x; w < kN / 32; w += kThreads) mask[w] = 0u;
    __syncthreads();
    const float cfl = p.cf32[0];
    auto a2 = [&](int i) {
        const float v = __ldg(sg.left + i) - cfl;
        return v < 500000.0f ? 0.0f : v;
    };
    const float last = a2(n - 1);
    for (int i = threadIdx.x; i < n - 1; i += kThreads) {
        const float ai = a2(i);
        if (ai > last && a2(i + 1) > ai) {
            const int l = i - 1;
            const int lo = max(0, l - 8), hi = min(l + 8, n);
            for (int j = lo; j < hi; ++j) atomicOr(mask + (j >> 5), 1u << (j & 31));
        }
    }
    __syncthreads();
    const float* x = ch ? sg.right : sg.left;
    fft16k<false>(c.S, c.t, Audio2Loader{x, p.cf32[ch], n, mask});
    audio2_filter(c.S, c.t, p.filt[ch]);
    __syncthreads();
    fft16k<true>(c.S, c.t, SmemIO(), Audio2Storer{ch ? sg.out_right : sg.out_left, p.cf[ch], n});
}

// ---- demodblock's fftdata (RFDecode.demodblock_cpu, core.py:758-761)

// The real block ifft(X).real of a full N-bin spectrum (complex128), one CTA
// per block: its Hermitian part (X[k] + conj(X[N-k])) / 2 on the
// non-negative bins, the C2R pre-processing and one inverse 16384-point
// transform.
__global__ void __launch_bounds__(kThreads, 1) spectrum_block_kernel(const __grid_constant__ SpectrumParams p) {
    extern __shared__ float2 smem[];
    const CtaSmem c = cta_setup<kVariantStockham>(smem, p.tw16, p.tw32);
    const double2* X = p.spectra + (long long)blockIdx.x * kN;
    auto herm = [&](int k) {  // bins 0 < k < N/2
        const double2 a = X[k], b = X[kN - k];
        return make_float2((float)(0.5 * (a.x + b.x)), (float)(0.5 * (a.y - b.y)));
    };
    for (int k = threadIdx.x; k <= kM / 2; k += kThreads) {
        if (k == 0) {
            // bins 0 and N/2: their real parts (the imaginary parts leave ifft(X).real alone)
            const double h0 = X[0].x, hm = X[kM].x;
            c.S[0] = make_float2((float)(0.5 * (h0 + hm)), (float)(0.5 * (h0 - hm)));
            continue;
        }
        c2r_pair(c.S, k, herm(k), herm(kM - k), __ldg(c.t.t32 + k));
    }
    __syncthreads();
    fft16k<true>(c.S, c.t, SmemIO(), RealStorer{p.out + (long long)blockIdx.x * kN, 0, kN, 0});
}

cudaError_t launch_spectrum_blocks(const SpectrumParams& p, int nblocks, cudaStream_t stream) {
    static SmemAttr attr;
    cudaError_t e = attr.ensure(spectrum_block_kernel, kSmemBytes);
    if (e != cudaSuccess) return e;
    if (nblocks <= 0) return cudaSuccess;
    spectrum_block_kernel<<<nblocks, kThreads, kSmemBytes, stream>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_audio2(const Audio2Params& p, int nsegs, cudaStream_t stream) {
    static SmemAttr attr;
    cudaError_t e = attr.ensure(audio2_kernel, kSmemBytes);
    if (e != cudaSuccess) return e;
    if (nsegs <= 0) return cudaSuccess;
    audio2_kernel<<<dim3((unsigned)nsegs, 2), kThreads, kSmemBytes, stream>>>(p);
    return cudaGetLastError();
}

cudaError_t prepare_demod_queue() {
    static SmemAttr attr, attr_ip;
    cudaError_t e = attr.ensure(demod_queue_kernel, kSmemBytes);
    if (e != cudaSuccess) return e;
    return attr_ip.ensure(demod_queue_ip_kernel, kSmemBytesIp);
}

cudaError_t launch_demod_queue(const QueueParams& q, int grid, cudaStream_t stream) {
    cudaError_t e = prepare_demod_queue();
    if (e != cudaSuccess) return e;
    if (q.total <= 0 || grid <= 0) return cudaSuccess;
    if (q.variant == kVariantInPlace) {
        demod_queue_ip_kernel<<<grid, kThreads, kSmemBytesIp, stream>>>(q);
    } else {
        demod_queue_kernel<<<grid, kThreads, kSmemBytes, stream>>>(q);
    }
    return cudaGetLastError();
}

cudaError_t launch_demod(const DemodParams& p, int grid, cudaStream_t stream) {
    static SmemAttr attr, attr_ip;
    cudaError_t e = attr.ensure(demod_kernel, kSmemBytes);
    if (e != cudaSuccess) return e;
    e = attr_ip.ensure(demod_ip_kernel, kSmemBytesIp);
    if (e != cudaSuccess) return e;
    if (p.nblocks <= 0) return cudaSuccess;
    if (p.variant == kVariantInPlace) {
        if (!p.tw_pair || !p.g_pos || !p.godd_pos) return cudaErrorInvalidValue;
        demod_ip_kernel<<<grid, kThreads, kSmemBytesIp, stream>>>(p);
    } else {
        demod_kernel<<<grid, kThreads, kSmemBytes, stream>>>(p);
    }
    return cudaGetLastError();
}

}  // namespace ldg
