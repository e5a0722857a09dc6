// Parameters of the fused per-block RF demodulator kernel.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ldg {

// Real-output spectra applied to the demodulated block (order fixed).
enum VideoOut { OUT_DEMOD = 0, OUT_05, OUT_BURST, OUT_PILOT, OUT_NVIDEO };

struct OutSlice {
    int start;  // first sample of the N-point block that is stored
    int len;    // samples stored per block (0: output not requested)
    int roll;   // value at n is taken from sample (n + roll) mod N
};

struct DemodParams {
    // input: block b's first sample is in + b * in_stride (elements)
    const void* in;
    int in_kind;          // 0 int16, 1 float32
    long long in_stride;
    int nblocks;

    float fs_hz;          // input sample rate
    // half spectra, bins 0..N/2 (float2[N/2+1]); G = RFVideo * MTF^m
    const float2* f_rfhpf;
    const float2* f_g;      // RFVideo * MTF^m
    const float2* f_godd;   // G * W_N^-k (odd-sample spectrum of the analytic signal)
    const float2* f_video[OUT_NVIDEO];
    const float2* f_efm;

    // outputs (nullptr: not requested); block b writes at ptr + b * len
    float* o_raw;         // demod_raw
    float* o_video[OUT_NVIDEO];
    float* o_rfhpf;
    int16_t* o_efm;
    OutSlice s_video;     // raw/demod/05/burst/pilot share start/len
    int roll[OUT_NVIDEO];
    OutSlice s_rfhpf;
    OutSlice s_efm;

    // analog audio (two channels)
    int audio;            // 0/1
    int a_lowbin[2];
    const float2* a_filt1[2];  // 513 weights per channel (bins 0..512)
    float a_rate;         // sample rate of the decimated band (a1_freq)
    float a_low[2];       // low_freq added back per channel
    float* o_audio[2];
    OutSlice s_audio;     // over the 1024-sample band output

    // per-CTA global scratch (2 * N/2 float2 per CTA), L2 resident
    float2* scratch;
    const float2* tw16;     // W_16384^i, i < 16384
    const float2* tw32;     // W_32768^k, k <= 8192

    // Scheduling.  slot_lock == nullptr: persistent CTAs, CTA i takes blocks
    // i, i + grid, ... with scratch slot i.  Otherwise CTA i works through
    // blocks [i * blocks_per_cta, (i + 1) * blocks_per_cta), so kernels of
    // other streams get SMs between CTAs; it works in scratch slot
    // i % nslots, which it holds under slot_lock[slot] (0 free, 1 held).  A wait for
    // a slot gives up after a bounded number of tries, sets *error and skips
    // the block (never seen in practice: nslots exceeds the resident CTAs).
    int* slot_lock;
    int nslots;
    int* error;
    int blocks_per_cta;   // per-slot mode: consecutive blocks a CTA works through

    // PAL_V4300D_NotchFilter: bins [notch_lo, notch_hi) searched (0, 0: off)
    int notch_lo, notch_hi;

    // FFT decomposition: kVariantStockham (natural-order spectra, ldg_fft.cuh)
    // or kVariantInPlace (position-order spectra, ldg_fft_ip.cuh), which
    // reads the filters through the tables below
    int variant;
    const float4* fp_rfhpf;          // bin-pair tables: pair u -> (F[k], F[M-k]), k = bin_of(pair_pos(u))
    const float4* fp_video[OUT_NVIDEO];
    const float4* fp_efm;
    const float2* g_pos;             // G at positions: g_pos[p] = G[bin_of(p)], p < M
    const float2* godd_pos;
    const float2* tw_pair;           // W_N^k of pair u
    // bins [efm_klo, efm_khi] outside which the EFM filter's float32 bins are
    // zero (its C2R input is zero there)
    int efm_klo, efm_khi;
};

enum { kVariantStockham = 0, kVariantInPlace = 1, kNumVariants = 2 };

constexpr int kDemodErrSlotWait = 1;

// A device work queue over the blocks of many captures (each with its own
// parameters: system, filters, outputs).  Block g of the queue is block
// g - first_block[i] of item i, first_block[i] <= g < first_block[i + 1].
struct QueueParams {
    const DemodParams* items;      // device array, nitems (scratch/slot fields unused)
    const long long* first_block;  // device array, nitems + 1 (prefix sums)
    int nitems;
    int grab;                      // consecutive blocks taken per pop
    long long total;               // first_block[nitems]
    unsigned long long* head;      // next unclaimed block; 0 at launch
    float2* scratch;               // kScratchPerCta per CTA of the launch
    const float2* tw16;
    const float2* tw32;
    int variant;                   // FFT decomposition for every item (as DemodParams.variant)
};

// Dynamic shared memory the kernels need: the padded working set, the two
// padded audio bands, the 1024-point tables (4 x 16 and 256 entries), then
// the 16384-point tables of the decomposition (Stockham: 4 x 256 and 4096;
// in place: 4 x 1024, 4 x 64 and 4 x 4).
constexpr int kSmemFloat2Common = (16384 + 1024) + 2 * (1024 + 64) + 4 * 16 + 256;
constexpr int kSmemFloat2 = kSmemFloat2Common + 4 * 256 + 4096;
constexpr int kSmemFloat2Ip = kSmemFloat2Common + 4 * 1024 + 4 * 64 + 4 * 4;
constexpr size_t kSmemBytes = size_t(kSmemFloat2) * 8;
constexpr size_t kSmemBytesIp = size_t(kSmemFloat2Ip) * 8;
constexpr size_t kScratchPerCta = size_t(2) * 16384 * 8;

// Analog audio stage 2 (one transform of up to kN stage-1 samples per
// segment and channel).
struct Audio2Seg {
    const float* left;
    const float* right;
    int len;              // 2 .. kN
    float* out_left;
    float* out_right;
};

struct Audio2Params {
    const Audio2Seg* segs;
    float cf32[2];        // carriers as float32 (the reference subtracts them from float32 audio)
    double cf[2];         // carriers added back in FP64
    const float2* filt[2];  // half spectra of the stage-2 filters (bins 0..kN/2)
    const float2* tw16;
    const float2* tw32;
};

// Real blocks from full spectra (demodblock's fftdata): out[b * N + n] = ifft(X_b).real[n].
struct SpectrumParams {
    const double2* spectra;  // nblocks x N complex128
    float* out;              // nblocks x N float32
    const float2* tw16;
    const float2* tw32;
};

cudaError_t launch_demod(const DemodParams& p, int grid, cudaStream_t stream);
cudaError_t launch_spectrum_blocks(const SpectrumParams& p, int nblocks, cudaStream_t stream);
cudaError_t launch_audio2(const Audio2Params& p, int nsegs, cudaStream_t stream);
// Sets the queue kernel's shared-memory size (call before a stream capture).
cudaError_t prepare_demod_queue();
cudaError_t launch_demod_queue(const QueueParams& q, int grid, cudaStream_t stream);

}  // namespace ldg
