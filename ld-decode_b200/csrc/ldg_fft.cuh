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
// The first pass can take its inputs from a loader functor (global memory,
// with a filter product fused in) and the last pass can hand its outputs to
// a storer functor (straight to global memory), which saves a shared-memory
// round trip at each end.
//
// Twiddles come from a table built on the host in FP64 and stored as FP32,
// T16[i] = exp(-2 pi i i/16384), copied into small per-pass shared tables
// at kernel start; a radix-16 butterfly reads W^k, W^2k, W^4k, W^8k and
// forms the other eleven by at most three complex products.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace ldg {

constexpr int kN = 32768;          // real block length
constexpr int kM = kN / 2;         // complex FFT length
constexpr int kThreads = 1024;     // threads per demod CTA
constexpr int kT16 = 16384;        // entries of the pass twiddle table
constexpr int kT32 = kM / 2 + 1;   // entries of the real-FFT twiddle table W_N^k, k <= M/2

__device__ __forceinline__ int pad(int i) { return i + (i >> 4); }
__host__ __device__ constexpr int padded(int n) { return n + (n >> 4); }

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

struct Tables {
    const float2* t16;  // global: W_16384^i, i < 16384
    const float2* t32;  // global: W_32768^k, k <= 8192 (real-FFT pre/post-processing)
    // shared-memory pass tables, laid out so a warp reads consecutive entries
    const float2* s2;   // [4][16]:   W_256^(k 2^r)  (pass Ns = 16, radix 16)
    const float2* s3;   // [4][256]:  W_4096^(k 2^r) (pass Ns = 256, radix 16)
    const float2* s4;   // [4096]:    W_16384^k      (pass Ns = 4096, radix 4)
    const float2* s4a;  // [256]:     W_1024^k       (1024-point pass Ns = 256, radix 4)
};

constexpr int kS2 = 4 * 16, kS3 = 4 * 256, kS4 = 4096, kS4a = 256;  // float2 entries of the shared tables

// Fill the 1024-point tables (s2, s4a) from the global W_16384 table (all threads).
__device__ __forceinline__ void load_1k_tables(float2* s2, float2* s4a, const float2* t16) {
    for (int i = threadIdx.x; i < kS2; i += blockDim.x) {
        const int r = i >> 4, k = i & 15;
        s2[i] = __ldg(t16 + ((k << r) * 64 & 16383));
    }
    for (int i = threadIdx.x; i < kS4a; i += blockDim.x) s4a[i] = __ldg(t16 + 16 * i);
}

// Fill the 16384-point Stockham pass tables from the global W_16384 table (all threads).
__device__ __forceinline__ void load_pass_tables(float2* s3, float2* s4, const float2* t16) {
    for (int i = threadIdx.x; i < kS4; i += blockDim.x) s4[i] = __ldg(t16 + i);
    for (int i = threadIdx.x; i < kS3; i += blockDim.x) {
        const int r = i >> 8, k = i & 255;
        s3[i] = __ldg(t16 + ((k << r) * 4 & 16383));
    }
}

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
// output bin bitrev(i).  R is 4 or 16.
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

template <bool INV>
__device__ __forceinline__ float2 sw(const float2* tab, int i) {
    const float2 w = tab[i];
    return INV ? cconj(w) : w;
}

// Multiply v[r] by the pass twiddle W_{Ns R}^(k r), r = 1..R-1, from the
// shared tables (radix 16: W^k, W^2k, W^4k, W^8k read, the rest formed by at
// most three complex products; radix 4: W^k read, W^2k, W^3k formed).
template <int R, int M, int Ns, bool INV>
__device__ __forceinline__ void apply_twiddles(float2 (&v)[R], const Tables& t, int k) {
    if constexpr (R == 4) {
        static_assert((M == 16384 && Ns == 4096) || (M == 1024 && Ns == 256), "radix-4 pass");
        const float2 w1 = M == 16384 ? sw<INV>(t.s4, k) : sw<INV>(t.s4a, k);
        const float2 w2 = cmul(w1, w1);
        const float2 w3 = cmul(w2, w1);
        v[1] = cmul(v[1], w1);
        v[2] = cmul(v[2], w2);
        v[3] = cmul(v[3], w3);
    } else {
        static_assert(Ns == 16 || (Ns == 256 && M == 16384), "radix-16 pass");
        const float2* tab = Ns == 16 ? t.s2 : t.s3;
        const float2 w1 = sw<INV>(tab, k), w2 = sw<INV>(tab, Ns + k);
        const float2 w4 = sw<INV>(tab, 2 * Ns + k), w8 = sw<INV>(tab, 3 * Ns + k);
        const float2 w3 = cmul(w2, w1), w5 = cmul(w4, w1), w6 = cmul(w4, w2), w7 = cmul(w4, w3);
        v[1] = cmul(v[1], w1);
        v[2] = cmul(v[2], w2);
        v[3] = cmul(v[3], w3);
        v[4] = cmul(v[4], w4);
        v[5] = cmul(v[5], w5);
        v[6] = cmul(v[6], w6);
        v[7] = cmul(v[7], w7);
        v[8] = cmul(v[8], w8);
        v[9] = cmul(v[9], cmul(w8, w1));
        v[10] = cmul(v[10], cmul(w8, w2));
        v[11] = cmul(v[11], cmul(w8, w3));
        v[12] = cmul(v[12], cmul(w8, w4));
        v[13] = cmul(v[13], cmul(w8, w5));
        v[14] = cmul(v[14], cmul(w8, w6));
        v[15] = cmul(v[15], cmul(w8, w7));
    }
}

// Loader / storer placeholder: read / write the shared working set.
struct SmemIO {};

// One Stockham pass of radix R over NB independent padded M-point working
// sets laid out back to back (set b starts at S + b * padded(M)).
// Ns = product of the radices of the earlier passes (a template constant,
// so the index arithmetic reduces to shifts and masks).  `ld(b, idx)` supplies
// the inputs when LD is not SmemIO; `st(b, idx, value)` consumes the outputs
// when ST is not SmemIO.  All threads of the CTA must call it; it starts
// with the loads (callers sync before) and ends with a barrier.  Kept out
// of line so each pass gets the whole 64-register budget (inlined into the
// demod kernel, live state around the passes made the allocator spill).
template <int R, int M, int NB, int Ns, bool INV, class LD, class ST>
__device__ __noinline__ void stockham_pass(float2* S, const Tables t, const LD ld, const ST st) {
    constexpr int B = M / R;                       // butterflies per set
    constexpr int BT = B * NB;                     // butterflies per pass
    constexpr int PER = (BT + kThreads - 1) / kThreads;
    static_assert(BT % kThreads == 0 || BT < kThreads, "butterfly count");
    static_assert(B % 16 == 0 && (Ns == 1 || Ns % 16 == 0) && (Ns > 1 || R == 16), "padding offsets");
    constexpr int bits = ilog2(R);
    constexpr int stride = padded(M);
    constexpr bool from_smem = std::is_same<LD, SmemIO>::value;
    constexpr bool to_smem = std::is_same<ST, SmemIO>::value;
    float2 v[PER][R];
    if constexpr (BT < kThreads) {
        // a pass with fewer butterflies than threads (the 1024-point audio
        // sets): the idle threads only keep the barrier count; this also
        // keeps the working threads' code within the register budget
        if (threadIdx.x >= BT) {
            if constexpr (from_smem && to_smem) __syncthreads();
            __syncthreads();
            return;
        }
    }
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int jt = threadIdx.x + q * kThreads;
        if (BT >= kThreads || jt < BT) {
            const int b = jt / B, j = jt - b * B;
            // pad(j + r B) = pad(j) + r padded(B) because B is a multiple of 16:
            // one base register, compile-time offsets
            const float2* Sb = S + b * stride + pad(j);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if constexpr (from_smem) {
                    v[q][r] = Sb[r * padded(B)];
                } else {
                    v[q][r] = ld(b, j + r * B);
                }
            }
            if constexpr (Ns > 1) apply_twiddles<R, M, Ns, INV>(v[q], t, j % Ns);
            dft_dif<R, INV>(v[q]);
        }
    }
    // loads from shared memory must all complete before any thread stores
    if constexpr (from_smem && to_smem) __syncthreads();
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int jt = threadIdx.x + q * kThreads;
        if (jt < BT) {
            const int b = jt / B, j = jt - b * B;
            const int k = j % Ns;
            const int d = (j / Ns) * Ns * R + k;
            // pad(d + r Ns) = pad(d) + r padded(Ns) for Ns a multiple of 16; for
            // Ns = 1, d = 16 j and pad(d + r) = pad(d) + r
            float2* Sb = S + b * stride + pad(d);
            constexpr int step = Ns >= 16 ? padded(Ns) : Ns;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if constexpr (to_smem) {
                    Sb[r * step] = v[q][bitrev(r, bits)];
                } else {
                    st(b, d + r * Ns, v[q][bitrev(r, bits)]);
                }
            }
        }
    }
    __syncthreads();
}

// Unnormalised 16384-point complex FFT of the padded working set S.
// Forward uses exp(-2 pi i nk/M); inverse exp(+2 pi i nk/M).  The first
// pass reads through `ld` and the last pass writes through `st` unless they
// are SmemIO.  Callers must __syncthreads() before when S was just written.
template <bool INV, class LD = SmemIO, class ST = SmemIO>
__device__ __forceinline__ void fft16k(float2* S, const Tables& t, const LD& ld = LD(), const ST& st = ST()) {
    const SmemIO s;
    stockham_pass<16, kM, 1, 1, INV>(S, t, ld, s);
    stockham_pass<16, kM, 1, 16, INV>(S, t, s, s);
    stockham_pass<16, kM, 1, 256, INV>(S, t, s, s);
    stockham_pass<4, kM, 1, 4096, INV>(S, t, s, st);
}

// Two independent unnormalised 1024-point complex FFTs (the analog-audio
// sub-bands), sets at S and S + padded(1024).
template <bool INV>
__device__ __forceinline__ void fft1k_x2(float2* S, const Tables& t) {
    const SmemIO s;
    stockham_pass<16, 1024, 2, 1, INV>(S, t, s, s);
    stockham_pass<16, 1024, 2, 16, INV>(S, t, s, s);
    stockham_pass<4, 1024, 2, 256, INV>(S, t, s, s);
}

}  // namespace ldg
