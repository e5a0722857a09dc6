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

#define LDG_ABI_VERSION 1

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
    LDG_NFILTERS = 8
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

/* One field for the time-base corrector. */
typedef struct {
    const float* buf;        /* field demod samples (field-local index 0) */
    int64_t buf_len;
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
} ldg_tbc_field;

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

/* Wait for all work queued on the context's stream. */
int ldg_synchronize(ldg_ctx* ctx);

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
 * 32)), and ctas > 32 is rejected with LDG_ERR_ARG.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress), so
 * make that first call before any stream capture.  Calls share the array:
 * calls that overlap on the GPU race and must be serialised by the caller;
 * nothing in it needs clearing between calls.  The filters and tables still
 * come from `ctx`, which is created (and allocates) beforehand.  Enqueues
 * on args->stream (or the context's stream) and returns without waiting. */
int ldg_demod_blocks_noalloc(ldg_ctx* ctx, const ldg_demod_args* args, int32_t ctas);

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

#ifdef __cplusplus
}
#endif

#endif /* LDGPU_H */
