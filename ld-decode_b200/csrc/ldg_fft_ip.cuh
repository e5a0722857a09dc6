// In-place 16384-point complex FFT of a padded shared-memory working set,
// the second decomposition of the demodulator's transforms (the first is
// the Stockham form of ldg_fft.cuh).
//
// Cooley-Tukey in place, radices 16, 16, 16, 4: each thread loads its 16
// points of a butterfly group, transforms them in registers and stores them
// back to the same 16 addresses, so a stage needs no barrier between its
// loads and its stores -- one barrier per stage, and the warps of a stage
// run their loads, arithmetic and stores out of step with each other.  The
// price is the order of the spectrum: the forward transform (decimation in
// frequency: butterfly, then twiddle) takes its input in natural order and
// leaves bin k at position pos_of(k), the four radix digits of k reversed;
// the inverse (decimation in time: twiddle, then butterfly, the stages in
// the opposite order) takes its input at those positions and leaves its
// output in natural order.  Spectra therefore stay in position order
// between a forward and an inverse transform (the parked spectra, the
// filters' bin-pair tables), and only time-domain data is in natural order.
//
// Stage s works on groups of R points at stride L inside blocks of R*L
// points: L = 1024, 64, 4 (radix 16) and L = 1 (radix 4, four groups per
// thread).  Only the L = 1024 stage mixes the whole set.  The threads of an
// L = 64 stage work on the 1024-point block t / 64 (two warps), those of an
// L = 4 stage on the 64-point block t / 4 and the radix-4 stage gives each
// thread four groups of that same 64-point block, so between the stages
// nearer the radix-4 end a barrier over the four warps of the 1024-point
// block's pair (L = 64 <-> L = 4) or over the warp (L = 4 <-> radix 4)
// orders every access; only L = 1024 needs the whole CTA.  The padding pad(i) = i + i/16 of ldg_fft.cuh makes every stage's
// loads and stores, and the position-order passes over bin pairs, free of
// bank conflicts.  Twiddles W_(RL)^(j q) come from per-stage shared tables
// holding W^j, W^2j, W^4j, W^8j (FP64-made, stored FP32); the other eleven
// are at most three complex products away, as in ldg_fft.cuh.
#pragma once
#include "ldg_fft.cuh"

namespace ldg {
namespace ip {

// bin of position p, and position of bin k (M = 16384 = 16*16*16*4)
__host__ __device__ __forceinline__ constexpr int bin_of(int p) {
    return (p >> 10) | (((p >> 6) & 15) << 4) | (((p >> 2) & 15) << 8) | ((p & 3) << 12);
}
__host__ __device__ __forceinline__ constexpr int pos_of(int k) {
    return ((k & 15) << 10) | (((k >> 4) & 15) << 6) | (((k >> 8) & 15) << 2) | (k >> 12);
}

// The bin pairs (k, M - k) of a real transform's half-length spectrum, one
// position of each pair in a fixed order u = 0 .. M/2: positions whose
// partner pos_of(M - bin_of(p)) comes later.  u < 7680: [1024, 8704);
// then [64, 544), [4, 34) and 0 (bins 0 / M), 1 (4096, partner 3), 2 (M/2).
constexpr int kPairs = kM / 2 + 1;
__host__ __device__ __forceinline__ constexpr int pair_pos(int u) {
    return u < 7680 ? 1024 + u : u < 8160 ? 64 + (u - 7680) : u < 8190 ? 4 + (u - 8160) : u - 8190;
}
__host__ __device__ __forceinline__ constexpr int partner_pos(int p) { return pos_of((kM - bin_of(p)) & (kM - 1)); }

// shared twiddle tables: [4][1024] W_16384^(j 2^r); [4][64] W_1024^(j 2^r); [4][4] W_64^(j 2^r)
constexpr int kT1 = 4 * 1024, kT2 = 4 * 64, kT3 = 4 * 4;

struct Twiddles {
    const float2* t1;
    const float2* t2;
    const float2* t3;
};

// Fill the stage tables from the global W_16384^i table (all threads).
__device__ __forceinline__ void load_stage_tables(float2* t1, float2* t2, float2* t3, const float2* t16) {
    for (int i = threadIdx.x; i < kT1; i += blockDim.x) {
        const int r = i >> 10, j = i & 1023;
        t1[i] = __ldg(t16 + ((j << r) & 16383));
    }
    for (int i = threadIdx.x; i < kT2; i += blockDim.x) {
        const int r = i >> 6, j = i & 63;
        t2[i] = __ldg(t16 + (((j << r) * 16) & 16383));
    }
    for (int i = threadIdx.x; i < kT3; i += blockDim.x) {
        const int r = i >> 2, j = i & 3;
        t3[i] = __ldg(t16 + (((j << r) * 256) & 16383));
    }
}

// The group's twiddles W^(j q), q = 1..15, from W^j, W^2j, W^4j, W^8j
// (conjugated for the inverse) by at most three complex products, each
// handed to mul(q, W^(j q)) as soon as it is formed, so that only W^j,
// W^2j, W^4j, W^8j and W^3j stay live beside the 16 points.
template <bool INV, class M>
__device__ __forceinline__ void apply_twiddles(const float2* tab, int stride, int j, M&& mul) {
    float2 w1 = tab[j], w2 = tab[stride + j], w4 = tab[2 * stride + j], w8 = tab[3 * stride + j];
    if (INV) {
        w1 = cconj(w1);
        w2 = cconj(w2);
        w4 = cconj(w4);
        w8 = cconj(w8);
    }
    mul(1, w1);
    mul(2, w2);
    mul(4, w4);
    mul(8, w8);
    const float2 w3 = cmul(w2, w1);
    mul(3, w3);
    {
        const float2 w5 = cmul(w4, w1);
        mul(5, w5);
        mul(13, cmul(w8, w5));
    }
    {
        const float2 w6 = cmul(w4, w2);
        mul(6, w6);
        mul(14, cmul(w8, w6));
    }
    {
        const float2 w7 = cmul(w4, w3);
        mul(7, w7);
        mul(15, cmul(w8, w7));
    }
    mul(9, cmul(w8, w1));
    mul(10, cmul(w8, w2));
    mul(11, cmul(w8, w3));
    mul(12, cmul(w8, w4));
}

// How far the barrier at the end of a stage reaches.
enum Sync { kSyncCta = 0, kSyncQuad = 1, kSyncWarp = 2 };

template <int SY>
__device__ __forceinline__ void stage_sync() {
    if constexpr (SY == kSyncCta) {
        __syncthreads();
    } else if constexpr (SY == kSyncQuad) {
        // named barriers 1..8: the four warps of threads [128 q, 128 q + 128)
        asm volatile("bar.sync %0, 128;" ::"r"(1 + (threadIdx.x >> 7)) : "memory");
    } else {
        __syncwarp();
    }
}

// One radix-16 stage at stride L (1024, 64 or 4).  Forward: load, butterfly,
// twiddle the outputs, store; inverse: load, twiddle the inputs, butterfly,
// store.  LD (first forward stage, L = 1024) supplies the natural-order
// input ld(0, n); ST (last inverse stage, L = 1024) takes the natural-order
// output st(0, n, v) instead of shared memory.  Ends with a barrier of reach SY.
template <int L, bool INV, int SY, class LD, class ST>
__device__ __noinline__ void stage16(float2* S, const Twiddles tw, const LD ld, const ST st) {
    static_assert(L == 1024 || L == 64 || L == 4, "stride");
    constexpr bool from_smem = std::is_same<LD, SmemIO>::value;
    constexpr bool to_smem = std::is_same<ST, SmemIO>::value;
    const int t = threadIdx.x;
    int base, j;
    if (L == 1024) {
        base = 0;
        j = t;
    } else if (L == 64) {
        base = (t >> 6) << 10;
        j = t & 63;
    } else {
        base = (t >> 2) << 6;
        j = t & 3;
    }
    float2* Sb = S + pad(base + j);
    // pad(base + j + L r) = pad(base + j) + off(r)
    auto off = [](int r) { return L >= 16 ? r * padded(L) : 4 * r + (r >> 2); };
    float2 v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) {
        if constexpr (from_smem) {
            v[r] = Sb[off(r)];
        } else {
            v[r] = ld(0, j + L * r);
        }
    }
    // the twiddles are formed next to their use (forward: after the
    // butterfly), so they are not live across it
    const float2* tab = L == 1024 ? tw.t1 : L == 64 ? tw.t2 : tw.t3;
    constexpr int stride = L == 1024 ? 1024 : L == 64 ? 64 : 4;
    if (INV) apply_twiddles<INV>(tab, stride, j, [&](int q, float2 w) { v[q] = cmul(v[q], w); });
    dft_dif<16, INV>(v);  // v[i] = Y[bitrev(i)]
    if (!INV) {
        // v[i] holds bin bitrev(i): it takes W^(j bitrev(i))
        apply_twiddles<INV>(tab, stride, j, [&](int q, float2 w) {
            const int i = bitrev(q, 4);
            v[i] = cmul(v[i], w);
        });
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int q = bitrev(i, 4);
        if constexpr (to_smem) {
            Sb[off(q)] = v[i];
        } else {
            st(0, j + L * q, v[i]);
        }
    }
    stage_sync<SY>();
}

// The radix-4 stage (L = 1): groups 4g .. 4g+3, no twiddles.  From shared
// memory thread t takes g = 16 (t / 4) + 4 (t % 4) + i, i < 4: the four
// groups of its L = 4 stage's 64-point block that sit at 4 (t % 4) + i (a
// half warp's accesses then cover all 32 banks once), so a barrier over
// the warp orders it against that stage.  With a loader (LD, first inverse
// stage: the position-order input ld.quad(p, v4) for the four points at
// positions p .. p+3, from global memory) thread t takes g = t + 1024 i, so
// that a warp reads one contiguous kilobyte per step; that order needs the
// whole CTA's barrier (SY is then kSyncCta).  Ends with a barrier of reach SY.
template <bool INV, int SY, class LD>
__device__ __noinline__ void stage4(float2* S, const LD ld) {
    constexpr bool from_smem = std::is_same<LD, SmemIO>::value;
    static_assert(from_smem || SY == kSyncCta, "the loader order spans the CTA");
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int g = from_smem ? 16 * (threadIdx.x >> 2) + 4 * (threadIdx.x & 3) + i : threadIdx.x + kThreads * i;
        float2* Sb = S + pad(4 * g);  // pad(4g + r) = pad(4g) + r
        float2 v[4];
        if constexpr (from_smem) {
#pragma unroll
            for (int r = 0; r < 4; ++r) v[r] = Sb[r];
        } else {
            ld.quad(4 * g, v);
        }
        dft_dif<4, INV>(v);
#pragma unroll
        for (int q = 0; q < 4; ++q) Sb[bitrev(q, 2)] = v[q];
    }
    stage_sync<SY>();
}

// Forward (exp(-2 pi i nk/M)): natural-order input (through `ld` unless
// SmemIO), bin k left at S[pad(pos_of(k))].  Callers sync before when S was
// just written.
template <class LD = SmemIO>
__device__ __forceinline__ void fft16k_fwd(float2* S, const Twiddles& tw, const LD& ld = LD()) {
    const SmemIO s;
    stage16<1024, false, kSyncCta>(S, tw, ld, s);
    stage16<64, false, kSyncQuad>(S, tw, s, s);
    stage16<4, false, kSyncWarp>(S, tw, s, s);
    stage4<false, kSyncCta>(S, s);
}

// Inverse (exp(+2 pi i nk/M), unnormalised): bin k taken from position
// pos_of(k) (S, or `ld.quad` when LD is not SmemIO), natural-order output
// (S, or `st` when ST is not SmemIO).  Callers sync before when S was just
// written.
template <class LD = SmemIO, class ST = SmemIO>
__device__ __forceinline__ void fft16k_inv(float2* S, const Twiddles& tw, const LD& ld = LD(), const ST& st = ST()) {
    const SmemIO s;
    stage4<true, std::is_same<LD, SmemIO>::value ? kSyncWarp : kSyncCta>(S, ld);
    stage16<4, true, kSyncQuad>(S, tw, s, s);
    stage16<64, true, kSyncCta>(S, tw, s, s);
    stage16<1024, true, kSyncCta>(S, tw, s, st);
}

}  // namespace ip
}  // namespace ldg
