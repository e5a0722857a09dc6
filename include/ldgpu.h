/*
 * ldgpu -- C ABI of the B200 (sm_100a) LaserDisc RF demodulator and
 * time-base corrector.
 *
 * This is the drop-in boundary under the reference decoder's Python API:
 *   RFDecode.demodblock(data, mtf_level, fftdata, cut)   lddecode/core.py:747-879
 *   Field.downscale(lineinfo, linesout, outwidth, ...)   lddecode/core.py:2626-2722
 *     (computewow_scaled core.py:2591-2623, scale_field utils.py:127-183,
 *      hz_to_output_array utils.py:1061-1075)
 * A host wrapper (the ldgpu Python package, through ctypes) designs the
 * filters in FP64 exactly as the reference does and calls these entry
 * points; everything below runs on the GPU.
 *
 * Conventions: every function returns LDG_OK (0) or a negative LDG_ERR_*
 * code and then ldg_last_error() describes the failure (thread-local text).
 * No C++ exception crosses this boundary.  All buffers are owned by the
 * caller.  Data pointers may point to host memory (pageable or pinned) or
 * to device memory of the context's GPU; host buffers are staged through
 * the context, which makes the call synchronous.  A context is not safe
 * for concurrent use from several threads -- the reference creates one
 * RFDecode per worker thread (core.py:1165), and so does the wrapper.
 */
#ifndef LDGPU_H
#define LDGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LDG_ABI_VERSION 3

#define LDG_OK 0
#define LDG_ERR_ARG (-1)         /* invalid argument or size */
#define LDG_ERR_CUDA (-2)        /* CUDA runtime error */
#define LDG_ERR_STATE (-3)       /* a required filter / table was not set */
#define LDG_ERR_UNSUPPORTED (-4) /* valid in the reference, not on this path */
#define LDG_ERR_RANGE (-5)       /* a TBC tap fell outside the field buffer */

typedef struct ldg_ctx ldg_ctx;

/* television system (reference SysParams_NTSC / SysParams_PAL) */
enum { LDG_NTSC = 0, LDG_PAL = 1 };

/* filter slots, each a half spectrum of N/2+1 complex bins (bins 0..N/2)
 * given as interleaved (re, im) doubles; see ldg_set_filter */
enum {
    LDG_F_RFHPF = 0,   /* Frfhpf                   (core.py:553-554, 769) */
    LDG_F_VIDEO_G = 1, /* RFVideo * MTF^mtf         (core.py:800-803)      */
    LDG_F_DEMOD = 2,   /* FVideo                    (core.py:643-653, 811) */
    LDG_F_05 = 3,      /* FVideo05                  (core.py:658-662, 813) */
    LDG_F_BURST = 4,   /* FVideoBurst               (core.py:664-668, 816) */
    LDG_F_PILOT = 5,   /* FVideoPilot, PAL          (core.py:670-679, 820) */
    LDG_F_EFM = 6,     /* Fefm                      (core.py:422-465, 848) */
    LDG_F_VIDEO_G_ODD = 7, /* RFVideo * MTF^mtf * exp(+2 pi i k/N): the
                              odd-sample half of the analytic inverse FFT */
    LDG_F_AUDIO2_LEFT = 8,  /* audio2_filter, left  (core.py:722-737, 908) */
    LDG_F_AUDIO2_RIGHT = 9, /* audio2_filter, right */
    LDG_NFILTERS = 10
};

/* input sample type of ldg_demod_args.in */
enum { LDG_IN_INT16 = 0, LDG_IN_FLOAT32 = 1 };

/* Which samples of each N-point block an output keeps: samples
 * [start, start+len) of the block, sample n taken from (n + roll) mod N.
 * len == 0 disables the output. */
typedef struct {
    int32_t start;
    int32_t len;
    int32_t roll;
} ldg_slice;

/* One batch of overlap-save blocks: block b reads N samples starting at
 * in + b * in_stride and writes len samples at out + b * len for every
 * requested output (NULL: not computed). */
typedef struct {
    const void* in;
    int32_t in_kind;   /* LDG_IN_INT16 or LDG_IN_FLOAT32 */
    int64_t in_stride; /* samples between consecutive block starts */
    int64_t nblocks;

    float* out_demod;  /* video["demod"]       */
    float* out_raw;    /* video["demod_raw"]   */
    float* out_05;     /* video["demod_05"]    */
    float* out_burst;  /* video["demod_burst"] */
    float* out_pilot;  /* video["demod_pilot"] (PAL) */
    float* out_rfhpf;  /* rfhpf                */
    int16_t* out_efm;  /* efm                  */
    float* out_audio_left;
    float* out_audio_right;

    ldg_slice video;   /* shared by demod/raw/05/burst/pilot (roll ignored) */
    int32_t roll_05;   /* F05_offset (core.py:814)          */
    int32_t roll_burst;/* FVideoBurst_offset (core.py:817)  */
    ldg_slice rfhpf;   /* start = blockcut - video_rot (core.py:770-772) */
    ldg_slice efm;
    ldg_slice audio;   /* over the 1024-sample stage-1 audio output */
    void* stream;      /* cudaStream_t, or NULL for the context's stream */
} ldg_demod_args;

/* One field for the analog audio downscale (the audio of Field.downscale,
 * downscale_audio core.py:1423-1580).  The host computes the field's output
 * clock as the reference does: ticks at timeoffset + i * soundgap, i <
 * nticks, with freq < 0 meaning line-locked (core.py:1445-1452). */
typedef struct {
    const float* audio_left;   /* field-local stage-1 audio (device), demod sample s <-> audio s / scale */
    const float* audio_right;
    int64_t audio_len;
    const double* linelocs;    /* FP64 line locations, field-local demod samples (device) */
    int32_t nlines;            /* >= 2 */
    int32_t nticks;            /* output samples + 1, in [1, 2048] */
    double timeoffset;         /* time of the first tick (s) */
    double soundgap;           /* 1 / output rate (s) */
    int16_t* out;              /* 2 * (nticks - 1) interleaved L/R (device) */
} ldg_audio_field;

typedef struct {
    double line_period;        /* SysParams line_period (us) */
    double linelen;            /* RFDecode.linelen */
    double scale;              /* Filters audio_fdiv: demod samples per audio sample */
    double lfreq, rfreq;       /* SysParams audio_lfreq / audio_rfreq (Hz) */
} ldg_audio_params;

/* One field for the time-base corrector. */
typedef struct {
    const float* buf;        /* field demod samples (field-local index 0) */
    int64_t buf_len;         /* < 2^31 */
    const double* linelocs;  /* FP64 line locations, field-local samples */
    int32_t nlines;          /* len(linelocs), <= 513 */
    int32_t lineoffset;      /* Field.lineoffset */
    int32_t outwidth;        /* output samples per line */
    int32_t linesout;        /* output lines */
    int32_t outlinecount;    /* Field.outlinecount (wow statistics span) */
    int32_t coord_f32;       /* 1: round coordinates to float32 as utils.py:160 */
    double inlinelen;        /* RFDecode.linelen */
    double outlinelen;       /* SysParams outlinelen */
    double ire0, hz_ire, vsync_ire, out_scale, output_zero; /* hz_to_output */
    float* out_f32;          /* linesout*outwidth float32 (may be NULL) */
    uint16_t* out_u16;       /* linesout*outwidth uint16 (may be NULL) */
    double wow_smoothing;    /* Field.wow_level_adjust_smoothing: 0 off, else the level-adjust
                                IIR of utils.py:141-149 with alpha = 1 / (smoothing * outwidth) */
    int32_t wow_interp;      /* Field.wow_interpolation_method (core.py:2602-2613): 0 or
                                LDG_WOW_LINEAR, LDG_WOW_QUADRATIC (k = 2, scipy's default
                                knots), LDG_WOW_CUBIC (k = 3, natural ends); the spline
                                forms need nlines >= 4 */
    int32_t pad1;
} ldg_tbc_field;

enum { LDG_WOW_LINEAR = 1, LDG_WOW_QUADRATIC = 2, LDG_WOW_CUBIC = 3 };

int ldg_abi_version(void);
const char* ldg_last_error(void);

/* Number of visible CUDA devices (0 when none). */
int ldg_device_count(int32_t* count);

/* Create a context on `device` for `system` (LDG_NTSC/LDG_PAL), block
 * length `blocklen` (only 32768, the reference BLOCKSIZE core.py:66, is
 * supported) and input rate fs_hz.  Replaces the device side of
 * RFDecode.__init__ (core.py:284-402). */
int ldg_ctx_create(ldg_ctx** out, int32_t device, int32_t system, int32_t blocklen, double fs_hz);
void ldg_ctx_destroy(ldg_ctx* ctx);

/* Upload one FP64 half spectrum (nbins = blocklen/2+1 complex bins as
 * 2*nbins doubles) into filter slot `which`; stored as float32.  Replaces
 * the per-call use of self.Filters[...] in demodblock_cpu (core.py:769-851). */
int ldg_set_filter(ldg_ctx* ctx, int32_t which, const double* reim, int64_t nbins);

/* Analog audio stage-1 band of channel 0 (left) / 1 (right): FFT bins
 * [lowbin, lowbin+nbins/2] times filt1 (nbins complex, only the first
 * nbins/2+1 are nonzero), decimated rate a1_freq, offset low_freq
 * (core.py:706-721, 854-875).  Only nbins == 1024 is supported. */
int ldg_set_audio(ldg_ctx* ctx, int32_t channel, int32_t lowbin, int32_t nbins, const double* filt1_reim,
                  double a1_freq, double low_freq);

/* Windowed-sinc TBC table, rows x taps float32 (65537 x 16; utils.py:77-78). */
int ldg_set_sinc_lut(ldg_ctx* ctx, const float* lut, int32_t rows, int32_t taps);

/* Demodulate a batch of blocks (RFDecode.demodblock, core.py:747-879). */
int ldg_demod_blocks(ldg_ctx* ctx, const ldg_demod_args* args);

/* Resample a batch of fields (Field.downscale's video part,
 * core.py:2691-2713). */
int ldg_tbc_fields(ldg_ctx* ctx, const ldg_tbc_field* fields, int32_t nfields, void* stream);

/* Analog audio of a batch of fields to 16-bit output (downscale_audio,
 * core.py:1423-1580; rescale utils.py:1328-1332): per output sample the
 * mean of the stage-1 audio run between two ticks' line-interpolated
 * positions, times the line-length wow factor (jumps over 1.5 % keep the
 * previous factor), minus the carrier, scaled, rounded, clipped, negated.
 * A sample whose run falls outside the field's audio is 0 and sets
 * muted[i] (the reference logs "Analog audio processing error, muting
 * samples").  Device buffers; enqueued on `stream` without waiting.  No
 * counterpart for a batch in the reference. */
int ldg_audio_downscale(ldg_ctx* ctx, const ldg_audio_field* fields, int32_t nfields, const ldg_audio_params* params,
                        int32_t* muted, void* stream);

/* ldg_tbc_fields for device-resident buffers without waiting: enqueues on
 * `stream` and returns (the descriptors go through one of four pinned
 * workspaces, reused once their launch has completed).  Taps outside a
 * field buffer are reported later by ldg_tbc_status.  Calls on one context
 * must use one stream.  No counterpart in the reference. */
int ldg_tbc_fields_async(ldg_ctx* ctx, const ldg_tbc_field* fields, int32_t nfields, void* stream);

/* Sticky TBC error bits since the last call (cleared by reading);
 * LDG_ERR_RANGE / LDG_ERR_ARG as ldg_tbc_fields would have returned.
 * Synchronous.  No counterpart in the reference. */
int ldg_tbc_status(ldg_ctx* ctx, int32_t* flags);

/* Wait for all work queued on the context's stream. */
int ldg_synchronize(ldg_ctx* ctx);

/* Sticky error bits of the context's demodulator launches since the last
 * call (cleared by reading): LDG_ERR_CUDA with flags = 1 when a block gave up
 * waiting for its scratch slot and was skipped.  Synchronous.  No
 * counterpart in the reference. */
int ldg_demod_status(ldg_ctx* ctx, int32_t* flags);

/* PAL_V4300D_NotchFilter (core.py:329, 774-798): search bins [lo, hi) of
 * each block's spectrum (the reference uses int(N * 8.42 / MHz) ..
 * int(1 + N * 8.6 / MHz)); bins above the band's mean + 3 std are zeroed
 * with their neighbours before the video, EFM and audio filters (rfhpf uses
 * the spectrum before).  0, 0 turns it off (the default). */
int ldg_set_notch(ldg_ctx* ctx, int32_t lo, int32_t hi);

/* FFT decomposition of the demodulator -- no counterpart in the reference
 * (its transforms are scipy's).  Both compute every output from the same
 * float32 spectra and filters, to the same accuracy; they differ in the
 * order of the float32 roundings and in speed:
 *   LDG_VARIANT_STOCKHAM  16384-point Stockham passes of radix 16, 16, 16, 4
 *                         (two barriers per pass), spectra in bin order;
 *   LDG_VARIANT_IN_PLACE  in-place Cooley-Tukey stages of the same radices
 *                         (one barrier per stage), spectra in digit-reversed
 *                         position order between the transforms.
 * The default is LDG_VARIANT_STOCKHAM; ldgpu.batch.autotune times both. */
enum { LDG_VARIANT_STOCKHAM = 0, LDG_VARIANT_IN_PLACE = 1 };
int ldg_set_demod_variant(ldg_ctx* ctx, int32_t variant);
int ldg_get_demod_variant(ldg_ctx* ctx, int32_t* variant);

/* ldg_demod_blocks' schedule (no counterpart in the reference): each CTA
 * demodulates `blocks_per_cta` consecutive blocks (1..64) in one scratch
 * slot; 0 (the default) takes 2 for batches of at least 16 blocks per SM
 * and 1 below.  Outputs do not depend on it. */
int ldg_set_demod_schedule(ldg_ctx* ctx, int32_t blocks_per_cta);

/* Device scratch the demodulator uses for a batch of `nblocks` blocks
 * (bytes; parked spectra, one slot per resident CTA). */
int ldg_demod_scratch_bytes(ldg_ctx* ctx, int64_t nblocks, int64_t* bytes);

/* Allocation-free form of ldg_demod_blocks -- no counterpart in the
 * reference.  For callers that cannot call cudaMalloc while decoding (a
 * process whose device memory belongs to another allocator's pool, or a
 * capture loop that cannot afford cudaMalloc's device-wide synchronisation):
 * it calls no cudaMalloc/cudaFree and no allocating library routine.  All
 * buffers must be device memory (host buffers are rejected: staging them
 * would allocate).  The demodulator's scratch is a static device array of
 * 32 CTA slots x 256 KB (8 MB) that every GPU loading the library keeps
 * until exit; `ctas` is the number of CTA slots to use (0: min(nblocks,
 * 32)), and ctas > 32 is rejected with LDG_ERR_ARG.  Every call looks up
 * the array's device address on the context's device (cudaGetSymbolAddress,
 * which allocates nothing; the first lookup on a device sets the array up
 * there, so make the first call before any stream capture), so no address
 * outlives a device reset.  Calls share the array:
 * calls that overlap on the GPU race and must be serialised by the caller;
 * nothing in it needs clearing between calls.  The filters and tables still
 * come from `ctx`, which is created (and allocates) beforehand.  Enqueues
 * on args->stream (or the context's stream) and returns without waiting. */
int ldg_demod_blocks_noalloc(ldg_ctx* ctx, const ldg_demod_args* args, int32_t ctas);

/* demodblock's fftdata (RFDecode.demodblock_cpu, core.py:758-761: the
 * spectrum takes precedence over the samples): out[b*N + n] =
 * ifft(X_b).real[n] for `nblocks` full N-bin complex128 spectra X_b
 * (interleaved re, im; the FFT of a real block, as DemodCache passes it),
 * as float32 blocks for ldg_demod_blocks (LDG_IN_FLOAT32).  Both buffers
 * device memory; enqueued on `stream` (NULL: the context's) without
 * waiting.  A spectrum that is not Hermitian enters through its real
 * inverse, i.e. through its Hermitian part. */
int ldg_blocks_from_spectra(ldg_ctx* ctx, const double* spectra, int64_t nblocks, float* out, void* stream);

/* ---- Analog audio stage 2 (RFDecode.audio_phase2, core.py:884-950) ---- */

/* One transform of stage-1 audio: `len` (2 .. blocklen) samples per channel
 * from `left` / `right` (device), results to out_left / out_right (device). */
typedef struct {
    const float* left;
    const float* right;
    int64_t len;
    float* out_left;
    float* out_right;
} ldg_audio2_segment;

/* RFDecode.runfilter_audio_phase2 (core.py:884-915) for `n` segments in one
 * launch: carrier removed (center_left / center_right, SysParams
 * audio_lfreq / audio_rfreq), samples within 8 of each left-channel spike
 * above 500 kHz zeroed in both channels (findpeaks, utils.py:1207-1216),
 * the stage-2 filter (LDG_F_AUDIO2_*) applied by a blocklen-point transform
 * with zero padding, carrier added back; float32 results.  The caller
 * stitches longer inputs as audio_phase2 does (core.py:917-950).
 * `segs` is a host array; enqueued on `stream` without waiting. */
int ldg_audio_phase2(ldg_ctx* ctx, const ldg_audio2_segment* segs, int32_t n, double center_left,
                     double center_right, void* stream);

/* ---- Mixed batches: many captures in one launch (no reference counterpart;
 * the reference demodulates one capture's blocks at a time in
 * DemodCache.worker, core.py:1165-1200) ---- */

typedef struct ldg_queue ldg_queue;

/* One capture of a mixed batch: the context of its configuration (system,
 * filters, MTF, audio bands) and its blocks and outputs as for
 * ldg_demod_blocks, all buffers device memory (args.stream is ignored). */
typedef struct {
    ldg_ctx* ctx;
    ldg_demod_args args;
} ldg_work_item;

/* A device work queue on `device`: a persistent demodulator launch whose
 * CTAs pop blocks of all submitted captures (NTSC and PAL mixed) until the
 * queue is empty.  Every block's outputs are bit-identical to those of
 * ldg_demod_blocks on its capture. */
int ldg_queue_create(ldg_queue** out, int32_t device);
void ldg_queue_destroy(ldg_queue* q);

/* Replace the queue's captures (validated as ldg_demod_blocks validates a
 * device batch).  Waits for the queue's previous run.  A run reads each
 * item's context filters as they are then, so contexts must outlive the
 * runs that use them. */
int ldg_queue_submit(ldg_queue* q, const ldg_work_item* items, int32_t n);

/* Scheduling: `grab` consecutive blocks per pop (1..64), `ctas` persistent
 * CTAs (0: one per SM; at most 4 x SMs).  Default 1, 0. */
int ldg_queue_set_schedule(ldg_queue* q, int32_t grab, int32_t ctas);

/* FFT decomposition of the queue's launch (as ldg_set_demod_variant):
 * -1 (the default) takes the first submitted item's context's. */
int ldg_queue_set_variant(ldg_queue* q, int32_t variant);

/* Blocks submitted and the CTAs a run launches. */
int ldg_queue_info(ldg_queue* q, int64_t* total_blocks, int32_t* grid);

/* Demodulate every submitted block: reset of the queue head plus one
 * persistent launch, enqueued on `stream` (NULL: the queue's own stream)
 * without waiting.  use_graph != 0: the two are captured once into a CUDA
 * graph (re-captured after a submit or schedule change) and the graph is
 * launched.  Runs of one queue must not overlap on the GPU (they share its
 * head and scratch): order them on one stream. */
int ldg_queue_run(ldg_queue* q, void* stream, int32_t use_graph);

/* ---- Copies by the SMs (no counterpart in the reference) ---- */

/* dst[0, nbytes) = src[0, nbytes) by a kernel on `stream` (the current
 * device), each buffer device memory or pinned host memory (read or written
 * through its mapping over PCIe).  For small transfers that the host waits
 * on while bulk copies occupy the copy engines: a cudaMemcpyAsync would
 * queue behind them, the kernel does not.  Pageable host memory is rejected
 * (LDG_ERR_ARG). */
int ldg_copy_async(void* dst, const void* src, int64_t nbytes, void* stream);

/* ---- Ingest ---- */

/* .lds captures (DomesdayDuplicator: four 10-bit samples in 5 bytes, most
 * significant bits first) to the signed 16-bit samples of the reference's
 * loader, load_packed_data_4_40 / unpack_data_4_40 (utils.py:371-410):
 * out[i] = (v - 512) << 6, v the 10-bit value of sample first + i of
 * `packed` (its sample 0 starts at byte 0).  `packed` (4-byte aligned, at
 * least ((first + n - 1) / 4 + 1) * 5 bytes) and `out` (8-byte aligned) are
 * device memory on the current device; enqueued on `stream`. */
int ldg_unpack_lds(const uint8_t* packed, int64_t nbytes, int64_t first, int64_t n, int16_t* out, void* stream);

/* ---- RF TBC (Field.rf_tbc, core.py:2724-2752) ---- */

typedef struct {
    const int16_t* input;    /* the field read's raw samples, Field.data["input"] (field-local sample 0) */
    int64_t len;
    const double* linelocs;  /* FP64 line locations, field-local */
    int32_t nlines;
    int32_t startline;       /* Field.lineoffset (NTSC), 1 (PAL) */
    int32_t linecount;       /* output lines */
    int32_t linelen;         /* int(round(inlinelen)) output samples per line */
    double delay;            /* rf.delays["video_white"] */
    int16_t* out;            /* linecount * linelen int16 */
} ldg_rftbc_field;

/* Field.rf_tbc for nfields fields: line l of the output is the cubic
 * scaler (utils.py:37-70) over input[linelocs[l] - delay, linelocs[l+1] -
 * delay] to linelen samples, rounded half to even, int16; FP64 without
 * fused multiply-adds, bit-identical to the reference.  `fields` is a host
 * array; all buffers device memory.  Enqueued on `stream` without waiting; a
 * tap outside a field's read is reported by ldg_tbc_status (LDG_ERR_RANGE)
 * and gives 0. */
int ldg_rf_tbc(ldg_ctx* ctx, const ldg_rftbc_field* fields, int32_t nfields, void* stream);

/* ---- Dropout detection (Field.dropout_detect, core.py:2829-2983) ---- */

/* One field: its read (field-local sample 0 of each array), device memory. */
typedef struct {
    const float* demod;      /* video["demod"]     */
    const float* demod_05;   /* video["demod_05"]  */
    const float* demod_raw;  /* video["demod_raw"] */
    const float* rfhpf;      /* rfhpf              */
    int64_t len;             /* samples in the read */
    const double* linelocs;  /* FP64 line locations, field-local */
    int32_t nlines;
    int32_t lineoffset, linecount, isfirst;
    int32_t hsync_len;       /* int(Field.LT["hsync"][1]) */
    int32_t pad;
} ldg_dropout_field;

typedef struct {
    int32_t system;          /* LDG_NTSC / LDG_PAL */
    int32_t video_rot;       /* rf.delays["video_rot"] (> 0) */
    int32_t outlinelen;      /* SysParams outlinelen */
    int32_t err_cap;         /* error samples kept per field */
    int32_t out_cap;         /* dropouts kept per field */
    int32_t pad;
    double freq_mhz;         /* rf.freq */
    double freq_hz_half;     /* rf.freq_hz_half */
    double ire0, hz_ire;     /* DecoderParams */
    double vsync_ire;        /* SysParams */
} ldg_dropout_params;

/* Field.dropout_detect for nfields fields in one launch: the per-sample
 * error mask (dropout_detect_demod, core.py:2829-2887; the rfhpf standard
 * deviation in FP64 over the field read), the merge of the error samples
 * into spans (build_errlist, 2889-2908) and the spans as TBC line ranges
 * (dropout_errlist_to_tbc, 2910-2960).  `fields` is a host array; every
 * buffer is device memory.  Device outputs: drops[(f * out_cap + j) * 3 +
 * {0, 1, 2}] = dropOuts fieldLine / startx / endx of dropout j of field f
 * (core.py:2978-2983, 4536-4542); counts[2 f] = its dropouts, or -1 more than
 * out_cap, -2 line locations out of order, -3 a vertical-sync line past the
 * line locations (the reference raises IndexError); counts[2 f + 1] = error
 * samples, or -1 more than err_cap (no dropouts listed then); rfstd (may be
 * NULL) = the rfhpf standard deviation per field.  Enqueued on `stream`
 * without waiting. */
int ldg_dropouts(ldg_ctx* ctx, const ldg_dropout_params* p, const ldg_dropout_field* fields, int32_t nfields,
                 int32_t* drops, int32_t* counts, double* rfstd, void* stream);

/* ---- AC3-RF (2.88 MHz QPSK) demodulation, lddecode/ac3rf.py ---- */

typedef struct ldg_ac3 ldg_ac3;
typedef struct ldg_ac3_dpll ldg_ac3_dpll;

/* Text of the last failing ldg_ac3_* call on this thread. */
const char* ldg_ac3_last_error(void);

/* Front-end filters of Ac3RfDemodulator (ac3rf.py:315-357): the half-band
 * taps (19 before and between the mixer, 23 for the last /2), the RRC
 * matched filter, and the NCO cos/sin tables of 2^lut_bits entries with the
 * accumulator step per 10 MHz sample.  float32 taps as the reference's
 * _FirDecimStage uses them; zero taps are skipped as it does. */
int ldg_ac3_create(ldg_ac3** out, int32_t device, const float* hb19, int32_t n19, const float* hb23, int32_t n23,
                   const float* rrc, int32_t nrrc, int32_t lut_bits, const float* cos_lut, const float* sin_lut,
                   int32_t phase_step);
void ldg_ac3_destroy(ldg_ac3* ac3);

/* Baseband I/Q at fs/16 (2.5 MHz for 40 MSPS) of a raw RF stream that
 * starts at absolute sample 0 (filter history zero before it); `in` holds
 * the absolute samples [in_first, in_first + nsamples) and must reach back
 * over the filters' history of the requested outputs (1134 samples before
 * 16 * out_first, unless in_first == 0).  Final outputs
 * [out_first, out_first+out_count), with out_first+out_count <=
 * ceil((in_first+nsamples)/16).  Equal to feeding the same samples, in any
 * chunking, through the reference's pre-mix stages, mixer and post-mix
 * stages (ac3rf.py:372-392). */
int ldg_ac3_frontend(ldg_ac3* ac3, const void* in, int32_t in_kind, int64_t in_first, int64_t nsamples,
                     int64_t out_first, int64_t out_count, float* out_i, float* out_q, void* stream);

/* Symbol-timing DPLL of AC3_DPLL (ac3rf.py:200-299), host code, streaming:
 * state carries across calls.  Writes at most n symbols (values 0..3). */
int ldg_ac3_dpll_create(ldg_ac3_dpll** out, double final_fs);
void ldg_ac3_dpll_destroy(ldg_ac3_dpll* dpll);
int ldg_ac3_dpll_reclock(ldg_ac3_dpll* dpll, const float* in_i, const float* in_q, int64_t n, uint8_t* out,
                         int64_t* nout);

/* ---- Line locations of every field of a capture (batched) ------------------
 *
 * The reference finds a field's line locations in Field.process()
 * (core.py:1636-1653, FieldNTSC.process 3477-3495, FieldPAL.process
 * 3209-3239) one field at a time, each from the previous one.  Batched here
 * in three steps: ldg_sync_runs (GPU) finds the sync-level runs of demod_05
 * over the whole capture; ldg_field_chain (host) walks the fields and
 * computes the pulse-level line locations; ldg_lines_refine (GPU) does the
 * per-line H-sync, colour-burst (NTSC) and pilot (PAL) refinement of all
 * fields and writes their final FP64 line locations, ready for
 * ldg_tbc_fields.  No counterpart in the reference as one call; the
 * per-field results equal Field.process()'s. */

#define LDG_CHAIN_MAX_LINES 336

enum {
    LDG_CHAIN_STOP_END = 0,     /* the next field's read runs past the capture */
    LDG_CHAIN_STOP_FULL = 1,    /* max_plans fields planned */
    LDG_CHAIN_STOP_PREV = 2,    /* the next field's result depends on the previous field's refined lines */
    LDG_CHAIN_STOP_LEVELS = 3,  /* the next field needs the reference's level re-calibration */
    LDG_CHAIN_STOP_ERROR = 4    /* the next field has no line to fill gaps from (the reference raises) */
};

typedef struct ldg_chain_params {
    int32_t system;             /* 0 NTSC, 1 PAL */
    int32_t num_pulses;         /* SysParams numPulses */
    int32_t field_lines[2];
    int32_t outlinecount;       /* frame_lines // 2 + 1 */
    int32_t proclines;          /* outlinecount + 10 (+3 PAL) */
    double freq;                /* MHz */
    double freq_hz;
    double linelen;             /* rf.linelen */
    double inlinelen;
    double linefreq0;           /* rf.samplesperline * rf.linelen (usectoinpx factor) */
    double hsync_pulse_us, eq_pulse_us, vsync_pulse_us;
    double first_field_h[2];
    double hsync_tolerance;
    double ire0, hz_ire, vsync_ire;
    int64_t max_pulse_len;      /* findpulses max_len (5000) */
    int64_t blocklen, blockcut, blockcut_end, readlen;
    int64_t nblocks;            /* demodulated blocks of the capture */
} ldg_chain_params;

typedef struct ldg_chain_state {
    double start;               /* LDdecode's read position of the next field */
    int32_t prev_valid;         /* the previous field was valid (Field.prevfield set) */
    int32_t prev_isfirst;
    int64_t prev_startloc;
    int32_t fields_written;
    /* What getLine0 (core.py:2156-2239) reads of the previous field's refined
     * line locations, when the caller has it (the chain clears it after each
     * field): prev_known = 1 gives its line at linecount as a sample
     * position of the next field's read (line0loc_prev) -- exactly when
     * prev_line0 == prev_line0_hi, else only that it lies in [prev_line0,
     * prev_line0_hi], which suffices when every line 0 that range allows
     * assigns the pulses to the same line slots -- and its sync confidence;
     * prev_skip is skip_check() >= 50 (1 / 0) or -1 for unknown.  Without
     * what a field needs the chain stops before it (LDG_CHAIN_STOP_PREV). */
    int32_t prev_known;
    double prev_line0;
    double prev_line0_hi;
    int32_t prev_skip;
    int32_t prev_conf;
    /* Set by the chain after each valid field: the capture-wide sample
     * position of that field's pulse-level line at linecount (PAL: 312 /
     * 313) and its sync confidence.  When a field needs what prev_known
     * gives and the caller has not given it, the chain first retries the
     * field with line0loc_prev known only to lie within
     * LDG_CHAIN_PREV_MARGIN samples of this estimate (the refined line
     * locations move a line by a few samples at most) and skip_check
     * unknown; it stops only if that does not decide the field. */
    double prev_est;
    int32_t prev_est_valid;
    int32_t prev_est_conf;
} ldg_chain_state;

#define LDG_CHAIN_PREV_MARGIN 32.0

typedef struct ldg_field_plan {
    double start;
    int64_t readloc, first_block, nblocks, startloc, length;  /* the field's read window (fieldread) */
    int32_t valid, isfirst, linecount, proclines, has_prev, sync_confidence;
    int32_t hsync_len;                        /* int(Field.LT["hsync"][1]) (dropout detection) */
    int32_t prev_range;                       /* 1: planned from the previous field's estimate (prev_est) */
    double nextfieldoffset;
    double linelocs1[LDG_CHAIN_MAX_LINES];   /* pulse-level line locations (field-local samples) */
    uint8_t linebad[LDG_CHAIN_MAX_LINES];
} ldg_field_plan;

/* Runs of demod_05 <= threshold over a capture-wide output array `d05`
 * (device, n samples), sorted: run_start/run_len (host arrays of capacity
 * `cap`) and, for runs longer than min_long samples, the FP64 mean of
 * d05[start + trim_lo, start + len - trim_hi) (NaN otherwise).  A run still
 * open at the end of the array is not reported.  LDG_ERR_RANGE if more
 * than `cap` runs (*nruns then holds the count needed).  Two kernels (a
 * single-pass scan and the run pairing; pinned run arrays are written by
 * the second directly); calls on one context are serialised and each
 * synchronises `stream`; LDG_ERR_CUDA (the next call starts afresh) if a
 * tile of the scan waited for its predecessors' counts past its bound. */
int ldg_sync_runs(ldg_ctx* ctx, const float* d05, int64_t n, double threshold, int64_t min_long, int64_t trim_lo,
                  int64_t trim_hi, int64_t* run_start, int64_t* run_len, double* run_mean, int64_t cap,
                  int64_t* nruns, void* stream);

/* Host: walk fields from state_in through the runs, writing one plan per
 * field read (valid or not) until a stop condition (*stop, LDG_CHAIN_STOP_*);
 * state_out continues the walk.  Pure host code (no GPU). */
int ldg_field_chain(const ldg_chain_params* params, const int64_t* run_start, const int64_t* run_len,
                    const double* run_mean, int64_t nruns, const ldg_chain_state* state_in,
                    ldg_chain_state* state_out, ldg_field_plan* plans, int32_t max_plans, int32_t* nplans,
                    int32_t* stop);
const char* ldg_chain_last_error(void);

/* ldg_field_chain in `nthreads` pieces on host threads.  The read chain
 * locks onto the signal (a field read is placed from the next vertical
 * blanking interval on, whatever came before), so piece t > 0 starts from
 * a guessed position at its first block and the previous piece, which runs
 * margin_blocks past its end, is joined to it at the first chain state both
 * reached (same read position and previous-field flags); the joined plans
 * are re-walked from the true state.  The result equals ldg_field_chain's;
 * where no common state is found the rest is walked sequentially.  Pieces
 * shorter than min_seg_blocks: sequential. */
int ldg_field_chain_mt(const ldg_chain_params* params, const int64_t* run_start, const int64_t* run_len,
                       const double* run_mean, int64_t nruns, const ldg_chain_state* state_in,
                       ldg_chain_state* state_out, ldg_field_plan* plans, int32_t max_plans, int32_t* nplans,
                       int32_t* stop, int32_t nthreads, int64_t margin_blocks, int64_t min_seg_blocks);

typedef struct ldg_lines_consts {
    int32_t system;             /* 0 NTSC, 1 PAL */
    int32_t pad;
    double freq;                /* MHz */
    double linelen;             /* rf.linelen */
    double linefreq0;           /* rf.samplesperline * rf.linelen */
    double samplesperline;      /* rf.samplesperline */
    double half_sync;           /* iretohz(vsync_ire / 2) */
    double lo_ok, hi_ok;        /* iretohz(-55), iretohz(30) */
    double hz_ire;
    double fsc_mhz, pilot_mhz;
} ldg_lines_consts;

typedef struct ldg_lines_args {
    ldg_lines_consts k;
    const float* d05;           /* capture-wide outputs (device) */
    const float* demod;
    const float* burst;         /* demod_burst (NTSC) */
    const float* pilot;         /* demod_pilot (PAL) */
    int64_t capture_len;        /* samples in each capture-wide array */
    int32_t nfields;            /* valid fields, in chain order */
    int32_t proclines;
    const int64_t* startloc;    /* per field (device) */
    const int64_t* wlen;
    const int32_t* isfirst;
    const int32_t* linecount;   /* 262/263 as compute_linelocs sets it */
    const int32_t* has_prev;    /* the previous field in the chain is this list's previous entry */
    const double* linelocs1;    /* nfields x LDG_CHAIN_MAX_LINES */
    const uint8_t* linebad1;
    double prev_phase_adjust;   /* NTSC: phase_adjust_median of the field before the first one */
    double* linelocs;           /* out: final line locations, nfields x LDG_CHAIN_MAX_LINES */
    uint8_t* linebad;           /* out */
    double* phase_adjust;       /* out, NTSC: per-field phase_adjust_median */
    int32_t* field_phase;       /* out, NTSC: fieldPhaseID */
    void* scratch;              /* ldg_lines_scratch_bytes(nfields) bytes of device memory */
    void* stream;
    const double* prev_phase_adjust_dev;  /* if set: device copy of prev_phase_adjust (read in stream order) */
    int32_t first_field;        /* work on fields [first_field, first_field + count) of the nfields */
    int32_t count;              /* 0: to the end */
    int32_t stages;             /* bits: 1 H-sync (PAL: all of PAL's line locations), 2 NTSC burst chain /
                                   PAL 8-field sequence, 4 NTSC apply; 0: all */
    int32_t pad2;
    /* PAL 8-field sequence (determine_field_number, core.py:3095-3203): the
     * field before the first one -- the burst phase adjusts of its lines 7,
     * 11, 15, 19 (NaN: none) and its field phase ID (0: no such field) --
     * taken from the device copies when set (read in stream order).  PAL
     * phase_adjust holds nfields x 4 such adjusts, field_phase the IDs. */
    double prev_pal_adjust[4];
    const double* prev_pal_adjust_dev;
    const int32_t* prev_field_phase_dev;
    int32_t prev_field_phase;
    int32_t pad3;
    double* linelocs2;          /* NTSC, optional out: the H-sync-refined line locations (Field.linelocs2),
                                   nfields x LDG_CHAIN_MAX_LINES */
} ldg_lines_args;

int64_t ldg_lines_scratch_bytes(int32_t nfields);

/* sizeof of an ABI struct by its type name (binding checks), -1 if unknown. */
int64_t ldg_abi_sizeof(const char* name);

/* GPU refinement of all fields' line locations: refine_linelocs_hsync,
 * compute_deriv_error, NTSC refine_linelocs_burst + fix_badlines + the
 * 117.25-degree subcarrier shift, PAL refine_linelocs_pilot x2 +
 * fix_badlines.  All pointers device memory; asynchronous on `stream`.
 * A call may do some stages for a range of the fields (the scratch layout is
 * that of all nfields): stage 1 for all fields, then stages 2 and 4 range by
 * range in order lets the fields of a finished range go on (e.g. to the TBC
 * on another stream) while the NTSC burst chain, which walks the fields one
 * after another, continues.  A range's burst chain starts from the previous
 * field's phase_adjust output when first_field > 0. */
int ldg_lines_refine(ldg_ctx* ctx, const ldg_lines_args* args);

/* ---- EFM phase-locked loop (efm_pll.EFM_PLL, efm_pll.py:80-244) ----
 * Host code (the loop is serial and edge-driven): T-values from the int16
 * EFM output of the demodulator, bit-identical to the reference's.  One PLL
 * per decoded stream; its state carries from call to call (field to field,
 * as LDdecode.writeout feeds it, core.py:3918-3925).  A PLL is not safe for
 * concurrent use; different PLLs may run on different threads. */
typedef struct ldg_efm_pll ldg_efm_pll;

/* EFM_PLL() (efm_pll.py:100-122). */
int ldg_efm_pll_create(ldg_efm_pll** out);
int ldg_efm_pll_destroy(ldg_efm_pll* pll);

/* EFM_PLL.process(inputBuffer) (efm_pll.py:124-167, pushEdge 169-240):
 * `in` n int16 samples (host memory); the T-values of this call go to
 * out[0 .. *out_count).  out_cap >= n is required, as the reference sizes
 * its result buffer to the input (the count is far smaller: at most one
 * T-value per three loop periods of ~9.3 samples). */
int ldg_efm_pll_process(ldg_efm_pll* pll, const int16_t* in, int64_t n, int8_t* out, int64_t out_cap,
                        int64_t* out_count);

/* The loop state, for tests: dstate = {delta, currentPeriod, phaseAdjust,
 * refClockTime}, istate = {zcPreviousInput, frequencyHysteresis, tCounter}. */
int ldg_efm_pll_state(const ldg_efm_pll* pll, double* dstate, int32_t* istate);

/* One zero crossing of an EFM sample array, as EFM_PLL.process detects it
 * (efm_pll.py:148-151): sample `pos` has a sign (negative / not negative)
 * other than the sample before it; `prev` and `cur` are the two values, from
 * which the PLL's interpolated fraction -prev / (cur - prev) follows. */
typedef struct ldg_efm_edge {
    int32_t pos;
    int16_t prev;
    int16_t cur;
} ldg_efm_edge;

/* GPU: the zero crossings of efm[0, n) (device int16, e.g. the demodulator's
 * efm output over a range of blocks): every i with sign(efm[i-1]) !=
 * sign(efm[i]); for i = 0 the sample before is efm[-1] when has_before,
 * else 0 (no crossing at 0 for a non-negative efm[0]).  Written in
 * increasing position to `edges` (device, at most `cap`), each pos =
 * pos_offset + i (pos_offset + n must fit int32); their number to *count
 * (device or host-mapped pinned memory, may be NULL), by the GPU in stream
 * order, so the host can read it after a synchronisation without a copy.
 * More than cap crossings: *count holds the number found, cap are written.
 * `scratch`: ldg_efm_edges_scratch_bytes(n) bytes of device memory, not
 * shared with a call in flight on another stream.  Runs on the current
 * device.  No counterpart in the reference as one call. */
int64_t ldg_efm_edges_scratch_bytes(int64_t n);
int ldg_efm_edges(const int16_t* efm, int64_t n, int32_t has_before, int64_t pos_offset, ldg_efm_edge* edges,
                  int64_t cap, int64_t* count, void* scratch, void* stream);

/* GPU: the EFM slice Field.downscale hands to the PLL for each of n fields,
 * efm[int(linelocs[1]) : int(linelocs[end_line])] (core.py:2704-2707, with
 * end_line = linecount + 1 and positions made capture-wide by the field's
 * startloc): bounds[2i], bounds[2i+1] = that range of efm, samples[2i],
 * samples[2i+1] = its first and last sample.  linelocs[i] is the device
 * address of field i's FP64 line locations.  The input and output arrays
 * may be device memory or pinned host memory (read and written by the
 * kernel in stream order).  No counterpart in the reference as one call. */
int ldg_efm_field_slices(const int64_t* startloc, const uint64_t* linelocs, const int32_t* end_line, int32_t n,
                         const int16_t* efm, int64_t efm_len, int64_t* bounds, int16_t* samples, void* stream);

/* EFM_PLL.process over the samples [lo, hi) of an array whose zero
 * crossings are `edges` (sorted by position, host memory; those inside
 * (lo, hi) are used, the sample at lo is tested against the PLL's previous
 * sample as the reference's loop does), with first = sample lo and last =
 * sample hi - 1: the same T-values and loop state as ldg_efm_pll_process
 * on those samples (out_cap >= hi - lo, as there).  LDdecode feeds the PLL
 * one field's slice after another (core.py:3918-3925); the slices of
 * consecutive fields may overlap or leave gaps, and each call takes one. */
int ldg_efm_pll_process_edges(ldg_efm_pll* pll, const ldg_efm_edge* edges, int64_t nedges, int64_t lo, int64_t hi,
                              int16_t first, int16_t last, int8_t* out, int64_t out_cap, int64_t* out_count);

#ifdef __cplusplus
}
#endif

#endif /* LDGPU_H */
