// In-shared-memory complex FFT building blocks for the RF demodulator.
//
// One 1024-thread CTA owns one 16384-point complex working set S (float2)
// in shared memory and transforms it with four Stockham autosort passes of
// radix 16, 16, 16 and 4.  Each thread loads its 16 points into registers,
// applies the inter-pass twiddles, runs the small DFTs fully in registers
// and writes the results back in natural order; one barrier separates the
// loads of a pass from its stores, so a single buffer suffices (no
// ping-pong) and each thread holds 16 complex values across it (64
// registers per thread is the budget at 1024 threads).  Shared memory is
// padded by one float2 per 16 (pad(i) = i + i/16), which makes the
// stride-16 stores of the first pass bank-conflict free.
//
// Twiddles W_N^k = exp(-2 pi i k / N), N = 32768, come from two small
// tables built on the host in FP64 and stored as FP32:
// W_N^k = hi[k >> 7] * lo[k & 127].
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ldg {

constexpr int kN = 32768;          // real block length
constexpr int kM = kN / 2;         // complex FFT length
constexpr int kThreads = 1024;     // threads per demod CTA
constexpr int kTwHi = kN / 128;    // 256 coarse twiddles
constexpr int kTwLo = 128;         // 128 fine twiddles

__device__ __forceinline__ int pad(int i) { return i + (i >> 4); }
__host__ __device__ constexpr int padded(int n) { return n + (n >> 4); }

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

// Twiddle tables in shared memory.
struct Twiddles {
    const float2* hi;  // hi[a] = W_N^(128 a), a < 256
    const float2* lo;  // lo[b] = W_N^b, b < 128
    // W_N^k for 0 <= k < N; conj() of it for the inverse direction.
    template <bool INV>
    __device__ __forceinline__ float2 w(int k) const {
        float2 t = cmul(hi[(k >> 7) & (kTwHi - 1)], lo[k & (kTwLo - 1)]);
        return INV ? cconj(t) : t;
    }
};

// cos/sin(2 pi m / 32) for m = 0..15
__device__ __forceinline__ float c32(int m) {
    constexpr float c[16] = {1.0f, 0.9807852804032304f, 0.9238795325112867f, 0.8314696123025452f,
                             0.7071067811865476f, 0.5555702330196023f, 0.38268343236508984f,
                             0.19509032201612833f, 0.0f, -0.1950903220161282f, -0.3826834323650897f,
                             -0.555570233019602f, -0.7071067811865475f, -0.8314696123025453f,
                             -0.9238795325112867f, -0.9807852804032304f};
    return c[m];
}
__device__ __forceinline__ float s32(int m) {
    constexpr float s[16] = {0.0f, 0.19509032201612825f, 0.3826834323650898f, 0.5555702330196022f,
                             0.7071067811865475f, 0.8314696123025452f, 0.9238795325112867f,
                             0.9807852804032304f, 1.0f, 0.9807852804032304f, 0.9238795325112867f,
                             0.8314696123025455f, 0.7071067811865476f, 0.5555702330196022f,
                             0.3826834323650899f, 0.1950903220161286f};
    return s[m];
}

// v * W_32^m (forward: exp(-2 pi i m/32); inverse: exp(+2 pi i m/32)), m < 16,
// with the trivial rotations done exactly.
template <bool INV>
__device__ __forceinline__ float2 rot32(float2 v, int m) {
    if (m == 0) return v;
    if (m == 8) return INV ? make_float2(-v.y, v.x) : make_float2(v.y, -v.x);
    const float c = c32(m);
    const float s = INV ? s32(m) : -s32(m);
    return make_float2(fmaf(v.x, c, -v.y * s), fmaf(v.x, s, v.y * c));
}

__host__ __device__ constexpr int ilog2(int r) { return r <= 1 ? 0 : 1 + ilog2(r >> 1); }
__host__ __device__ constexpr int bitrev(int i, int bits) {
    int o = 0;
    for (int b = 0; b < bits; ++b) o |= ((i >> b) & 1) << (bits - 1 - b);
    return o;
}

// R-point DFT in registers, decimation in frequency; on return v[i] holds
// output bin bitrev(i).  R is 4, 16 or 32.
template <int R, bool INV>
__device__ __forceinline__ void dft_dif(float2 (&v)[R]) {
#pragma unroll
    for (int span = R / 2; span >= 1; span >>= 1) {
#pragma unroll
        for (int st = 0; st < R; st += 2 * span) {
#pragma unroll
            for (int j = 0; j < span; ++j) {
                const float2 a = v[st + j];
                const float2 b = v[st + j + span];
                v[st + j] = cadd(a, b);
                v[st + j + span] = rot32<INV>(csub(a, b), j * (32 / (2 * span)));
            }
        }
    }
}

// One Stockham pass of radix R over NB independent padded M-point working
// sets laid out back to back (set b starts at S + b * padded(M)) in shared
// memory.  Ns = product of the radices of the earlier passes.  The pass
// twiddle W_{Ns R}^{k r} is read as W_N^{k r N/(Ns R)}.  All threads of the
// CTA must call it; it starts with the loads (callers sync before) and ends
// with a barrier.
template <int R, int M, int NB, bool INV>
__device__ __forceinline__ void stockham_pass(float2* S, int Ns, const Twiddles& tw) {
    constexpr int B = M / R;                       // butterflies per set
    constexpr int BT = B * NB;                     // butterflies per pass
    constexpr int PER = (BT + kThreads - 1) / kThreads;
    static_assert(BT % kThreads == 0 || BT < kThreads, "butterfly count");
    constexpr int bits = ilog2(R);
    constexpr int stride = padded(M);
    float2 v[PER][R];
    const int scale = kN / (Ns * R);
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int jt = threadIdx.x + q * kThreads;
        if (jt < BT) {
            const int b = jt / B, j = jt - b * B;
            const float2* Sb = S + b * stride;
#pragma unroll
            for (int r = 0; r < R; ++r) v[q][r] = Sb[pad(j + r * B)];
            const int k = j % Ns;
            if (Ns > 1) {
#pragma unroll
                for (int r = 1; r < R; ++r) v[q][r] = cmul(v[q][r], tw.w<INV>((k * r * scale) & (kN - 1)));
            }
            dft_dif<R, INV>(v[q]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int jt = threadIdx.x + q * kThreads;
        if (jt < BT) {
            const int b = jt / B, j = jt - b * B;
            float2* Sb = S + b * stride;
            const int k = j % Ns;
            const int d = (j / Ns) * Ns * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) Sb[pad(d + r * Ns)] = v[q][bitrev(r, bits)];
        }
    }
    __syncthreads();
}

// Unnormalised 16384-point complex FFT of the padded working set S.
// The radix-4 pass runs 4 butterflies per thread (16 values, as the others).
// Forward uses exp(-2 pi i nk/M); inverse exp(+2 pi i nk/M).
template <bool INV>
__device__ __noinline__ void fft16k(float2* S, const Twiddles& tw) {
    stockham_pass<16, kM, 1, INV>(S, 1, tw);
    stockham_pass<16, kM, 1, INV>(S, 16, tw);
    stockham_pass<16, kM, 1, INV>(S, 256, tw);
    stockham_pass<4, kM, 1, INV>(S, 4096, tw);
}

// Two independent unnormalised 1024-point complex FFTs (the analog-audio
// sub-bands), sets at S and S + padded(1024).
template <bool INV>
__device__ __forceinline__ void fft1k_x2(float2* S, const Twiddles& tw) {
    stockham_pass<16, 1024, 2, INV>(S, 1, tw);
    stockham_pass<16, 1024, 2, INV>(S, 16, tw);
    stockham_pass<4, 1024, 2, INV>(S, 256, tw);
}

}  // namespace ldg
