// C ABI of the ldgpu demodulator / TBC (declared in include/ldgpu.h).
//
// A context owns the device copies of one RFDecode configuration: filter
// half spectra (float32), twiddle tables, the sinc table, the demodulator's
// parked-spectrum scratch and a staging arena for callers that pass host
// buffers.  Device buffers passed in are used in place and the call only
// enqueues work; host buffers make the call copy in, run and copy out
// synchronously (the plain, one-block-at-a-time form the reference's
// DemodCache workers use).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "ldg_copy.cuh"
#include "ldg_demod.cuh"
#include "ldg_fft_ip.cuh"
#include "ldg_dropouts.cuh"
#include "ldg_fft.cuh"
#include "ldg_noalloc.h"
#include "ldg_scan.cuh"
#include "ldg_audio.cuh"
#include "ldg_tbc.cuh"
#include "ldgpu.h"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define LDG_CK(call)                                                                          \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return fail(LDG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

bool is_device_ptr(const void* p) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Restores the caller's current device on scope exit.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace

struct ldg_ctx {
    int device = 0;
    int system = LDG_NTSC;
    int blocklen = ldg::kN;
    double fs_hz = 40e6;
    int sms = 148;
    cudaStream_t stream = nullptr;
    float2* d_filter[LDG_NFILTERS] = {};
    float2* d_audio[2] = {};
    int a_lowbin[2] = {0, 0};
    double a_rate[2] = {0, 0};
    double a_low[2] = {0, 0};
    float2* d_tw16 = nullptr;  // W_16384^i
    float2* d_tw32 = nullptr;  // W_32768^k, k <= 8192
    // in-place variant: per filter the bin-pair table (ip::kPairs float4) and,
    // for the RFVideo filters, the position-order table (kM float2); W_N^k per pair
    float4* d_fpair[LDG_NFILTERS] = {};
    int fband[LDG_NFILTERS][2] = {};  // first and last bin whose float32 value is not zero
    float2* d_fpos[LDG_NFILTERS] = {};
    float2* d_twpair = nullptr;
    int variant = ldg::kVariantStockham;
    int blocks_per_cta = 0;  // ldg_demod_blocks: consecutive blocks per CTA (0: 2 for large batches, else 1)
    float* d_lut = nullptr;
    float2* d_scratch = nullptr;
    size_t scratch_bytes = 0;
    char* d_stage = nullptr;
    size_t stage_bytes = 0;
    ldg::TbcField* d_fields = nullptr;
    int fields_cap = 0;
    double* d_seg = nullptr;
    size_t seg_cap = 0;
    double* d_ll = nullptr;
    size_t ll_cap = 0;
    int* d_status = nullptr;
    void* d_lines = nullptr;  // sync-run scan scratch (ldg_sync_runs)
    int* d_slots = nullptr;   // demod scratch-slot locks (nslots) and the error word after them
    int nslots = 0;
    // ldg_tbc_fields_async workspaces, used in turn; a workspace is reused once
    // the launch that last used it has completed
    struct TbcWs {
        ldg::TbcField* d_fields = nullptr;
        ldg::TbcField* h_fields = nullptr;  // pinned
        int cap = 0;
        double* d_seg = nullptr;
        size_t seg_cap = 0;
        cudaEvent_t done = nullptr;
        bool used = false;
    } tws[4];
    int tws_next = 0;
    size_t lines_cap = 0;
    // ldg_dropouts: device field descriptors and error lists; reused once the
    // launch that last used them has completed
    ldg::DropField* d_drop_fields = nullptr;
    size_t drop_fields_cap = 0;
    int* d_drop_errs = nullptr;
    size_t drop_errs_cap = 0;
    cudaEvent_t drop_done = nullptr;
    bool drop_used = false;
    int notch_lo = 0, notch_hi = 0;      // PAL_V4300D_NotchFilter search band (bins), 0 0: off
    ldg::Audio2Seg* d_a2 = nullptr;      // ldg_audio_phase2 segments; reused once the last launch is done
    size_t a2_cap = 0;
    cudaEvent_t a2_done = nullptr;
    bool a2_used = false;
    long long* h_word = nullptr;         // pinned, mapped: results the host reads right after a kernel
    // ldg_sync_runs' single-pass scan: [0] ticket counter, then flags, counts
    // and prefixes of scan_cap tiles; scan_base = tickets handed out so far
    unsigned long long* d_scan = nullptr;
    long long scan_cap = 0;
    unsigned long long scan_base = 0, scan_call = 0;
    bool scan_dirty = false;
    ldg::RfTbcField* d_rftbc = nullptr;  // ldg_rf_tbc descriptors, same reuse rule
    size_t rftbc_cap = 0;
    cudaEvent_t rftbc_done = nullptr;
    bool rftbc_used = false;
    std::mutex mu;
};

namespace {

// The FFT decomposition and the in-place variant's filter layouts (ctx->mu held).
void variant_tables(const ldg_ctx* c, ldg::DemodParams* p) {
    p->variant = c->variant;
    p->fp_rfhpf = c->d_fpair[LDG_F_RFHPF];
    const int fslot[4] = {LDG_F_DEMOD, LDG_F_05, LDG_F_BURST, LDG_F_PILOT};
    for (int o = 0; o < 4; ++o) p->fp_video[o] = c->d_fpair[fslot[o]];
    p->fp_efm = c->d_fpair[LDG_F_EFM];
    p->g_pos = c->d_fpos[LDG_F_VIDEO_G];
    p->godd_pos = c->d_fpos[LDG_F_VIDEO_G_ODD];
    p->tw_pair = c->d_twpair;
    p->efm_klo = c->fband[LDG_F_EFM][0];
    p->efm_khi = c->fband[LDG_F_EFM][1];
}

int grow(void** p, size_t* cap, size_t need) {
    if (need <= *cap) return LDG_OK;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    size_t sz = need + need / 4;
    LDG_CK(cudaMalloc(p, sz));
    *cap = sz;
    return LDG_OK;
}

bool slice_ok(const ldg_slice& s, int n) {
    return s.len >= 0 && s.start >= 0 && (s.len == 0 || (long long)s.start + s.len <= n) &&
           s.roll >= 0 && s.roll < n;
}

long long tbc_nwow(const ldg_tbc_field& f) {
    return (long long)(f.outlinecount + f.lineoffset + 1) * (long long)f.outlinelen;
}

// Argument checks shared by ldg_tbc_fields and ldg_tbc_fields_async.
int check_tbc_field(const ldg_tbc_field& f, const std::string& who) {
    if (!f.buf || !f.linelocs) return fail(LDG_ERR_ARG, who + ": NULL buffer");
    if (f.nlines < 2 || f.nlines > 513) return fail(LDG_ERR_ARG, who + ": nlines must be in [2, 513]");
    if (f.outwidth <= 0 || f.linesout <= 0 || f.outlinecount <= 0 || f.lineoffset < 0 || f.buf_len <= 0 ||
        f.buf_len >= (1ll << 31))
        return fail(LDG_ERR_ARG, who + ": bad field geometry");
    if (!(f.inlinelen > 0) || !(f.outlinelen > 0) || !(f.hz_ire != 0))
        return fail(LDG_ERR_ARG, who + ": bad line length or level");
    if (f.outlinelen != (double)(int)f.outlinelen) return fail(LDG_ERR_ARG, who + ": outlinelen must be an integer");
    if (!(f.wow_smoothing >= 0) || !(f.wow_smoothing * f.outwidth >= 1 || f.wow_smoothing == 0))
        return fail(LDG_ERR_ARG, who + ": wow_smoothing must be 0 or at least 1 / outwidth");
    if (f.wow_interp < 0 || f.wow_interp > LDG_WOW_CUBIC)
        return fail(LDG_ERR_ARG, who + ": wow_interp must be 0 or one of LDG_WOW_*");
    if (f.wow_interp >= LDG_WOW_QUADRATIC) {
        if (f.nlines < 4) return fail(LDG_ERR_ARG, who + ": quadratic / cubic wow interpolation needs nlines >= 4");
        const long long last = (long long)f.outwidth * (f.lineoffset + 1) + (long long)f.linesout * f.outwidth;
        if (last > tbc_nwow(f) || tbc_nwow(f) >= (1ll << 31))
            return fail(LDG_ERR_ARG, who + ": output pixels beyond the wow array");
    }
    return LDG_OK;
}

// Doubles of spline scratch a field needs: its pieces, median and
// threshold, and with smoothing the IIR state every 32 output pixels.
size_t tbc_spline_doubles(const ldg_tbc_field& f) {
    if (f.wow_interp < LDG_WOW_QUADRATIC) return 0;
    const size_t nout = (size_t)f.linesout * f.outwidth;
    return (size_t)ldg::kSplStride * f.nlines + 2 + (f.wow_smoothing > 0 ? (nout + 31) / 32 : 0);
}

// Device descriptor of one field: geometry, levels and scratch pointers
// (segment scratch at seg + sego in three arrays of seg_total, spline
// scratch at spl).
void fill_tbc_field(const ldg_tbc_field& f, ldg::TbcField& d, double* seg, size_t seg_total, size_t sego,
                    double* spl, int* status) {
    d.buf_len = f.buf_len;
    d.nlines = f.nlines;
    d.lineoffset = f.lineoffset;
    d.outwidth = f.outwidth;
    d.linesout = f.linesout;
    d.nwow = tbc_nwow(f);
    d.coord_f32 = f.coord_f32;
    d.inlinelen = f.inlinelen;
    d.outscale = f.inlinelen / f.outlinelen;
    d.inv_inl = 1.0 / f.inlinelen;
    d.u16_scale = f.out_scale / f.hz_ire;
    d.u16_offset = f.output_zero - f.vsync_ire * f.out_scale - f.ire0 * d.u16_scale;
    d.seg_level = seg + sego;
    d.seg_start = seg + seg_total + sego;
    d.seg_lo = reinterpret_cast<long long*>(seg + 2 * seg_total + sego);
    d.smooth_b = f.wow_smoothing > 0 ? 1.0 - 1.0 / (f.wow_smoothing * (double)f.outwidth) : 0.0;
    d.smooth_a = f.wow_smoothing > 0 ? 1.0 / (f.wow_smoothing * (double)f.outwidth) : 0.0;
    d.status = status;
    d.spline_k = f.wow_interp >= LDG_WOW_QUADRATIC ? f.wow_interp : 1;
    d.npieces = d.spline_k == 3 ? f.nlines - 1 : (d.spline_k == 2 ? f.nlines - 2 : 0);
    if (d.spline_k >= 2) {
        d.spl = spl;
        d.stat = spl + (size_t)ldg::kSplStride * f.nlines;
        d.ybefore = f.wow_smoothing > 0 ? d.stat + 2 : nullptr;
    } else {
        d.spl = d.stat = d.ybefore = nullptr;
    }
}

}  // namespace

extern "C" {

int ldg_abi_version(void) { return LDG_ABI_VERSION; }

const char* ldg_last_error(void) { return g_err.c_str(); }

int ldg_device_count(int32_t* count) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    if (count) *count = n;
    return LDG_OK;
}

int ldg_ctx_create(ldg_ctx** out, int32_t device, int32_t system, int32_t blocklen, double fs_hz) {
    if (!out) return fail(LDG_ERR_ARG, "ldg_ctx_create: out is NULL");
    *out = nullptr;
    if (system != LDG_NTSC && system != LDG_PAL) return fail(LDG_ERR_ARG, "ldg_ctx_create: system must be NTSC or PAL");
    if (blocklen != ldg::kN)
        return fail(LDG_ERR_UNSUPPORTED, "ldg_ctx_create: only blocklen 32768 (the reference BLOCKSIZE) is supported");
    if (!(fs_hz > 0)) return fail(LDG_ERR_ARG, "ldg_ctx_create: fs_hz must be positive");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(LDG_ERR_CUDA, "ldg_ctx_create: no CUDA device");
    }
    if (device < 0 || device >= ndev) return fail(LDG_ERR_ARG, "ldg_ctx_create: bad device index");
    DeviceGuard g(device);
    ldg_ctx* c = new ldg_ctx();
    c->device = device;
    c->system = system;
    c->blocklen = blocklen;
    c->fs_hz = fs_hz;
    cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return fail(LDG_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
    }
    // twiddle tables in FP64, stored FP32
    const double two_pi = 6.283185307179586476925286766559;
    std::vector<float2> t16(ldg::kT16), t32(ldg::kT32);
    for (int i = 0; i < ldg::kT16; ++i) {
        const double ang = -two_pi * (double)i / ldg::kT16;
        t16[i] = make_float2((float)std::cos(ang), (float)std::sin(ang));
    }
    for (int k = 0; k < ldg::kT32; ++k) {
        const double ang = -two_pi * (double)k / ldg::kN;
        t32[k] = make_float2((float)std::cos(ang), (float)std::sin(ang));
    }
    std::vector<float2> twp(ldg::ip::kPairs);
    for (int u = 0; u < ldg::ip::kPairs; ++u) {
        const int k = ldg::ip::bin_of(ldg::ip::pair_pos(u));
        const double ang = -two_pi * (double)k / ldg::kN;
        twp[u] = make_float2((float)std::cos(ang), (float)std::sin(ang));
    }
    if (cudaMalloc(&c->d_tw16, t16.size() * sizeof(float2)) != cudaSuccess ||
        cudaMemcpy(c->d_tw16, t16.data(), t16.size() * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMalloc(&c->d_tw32, t32.size() * sizeof(float2)) != cudaSuccess ||
        cudaMemcpy(c->d_tw32, t32.data(), t32.size() * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMalloc(&c->d_twpair, twp.size() * sizeof(float2)) != cudaSuccess ||
        cudaMemcpy(c->d_twpair, twp.data(), twp.size() * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMalloc(&c->d_status, sizeof(int)) != cudaSuccess || cudaMemset(c->d_status, 0, sizeof(int)) != cudaSuccess) {
        const std::string msg = cudaGetErrorString(cudaGetLastError());
        ldg_ctx_destroy(c);
        return fail(LDG_ERR_CUDA, "ldg_ctx_create: " + msg);
    }
    *out = c;
    return LDG_OK;
}

void ldg_ctx_destroy(ldg_ctx* c) {
    if (!c) return;
    DeviceGuard g(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto& f : c->d_filter) cudaFree(f);
    for (auto& f : c->d_fpair) cudaFree(f);
    for (auto& f : c->d_fpos) cudaFree(f);
    cudaFree(c->d_twpair);
    for (auto& a : c->d_audio) cudaFree(a);
    cudaFree(c->d_tw16);
    cudaFree(c->d_tw32);
    cudaFree(c->d_lut);
    cudaFree(c->d_scratch);
    cudaFree(c->d_stage);
    cudaFree(c->d_fields);
    cudaFree(c->d_seg);
    cudaFree(c->d_ll);
    cudaFree(c->d_status);
    cudaFree(c->d_lines);
    cudaFree(c->d_slots);
    if (c->drop_used) cudaEventSynchronize(c->drop_done);
    if (c->rftbc_used) cudaEventSynchronize(c->rftbc_done);
    if (c->h_word) cudaFreeHost(c->h_word);
    cudaFree(c->d_scan);
    if (c->a2_used) cudaEventSynchronize(c->a2_done);
    cudaFree(c->d_a2);
    if (c->a2_done) cudaEventDestroy(c->a2_done);
    cudaFree(c->d_rftbc);
    if (c->rftbc_done) cudaEventDestroy(c->rftbc_done);
    cudaFree(c->d_drop_fields);
    cudaFree(c->d_drop_errs);
    if (c->drop_done) cudaEventDestroy(c->drop_done);
    for (auto& w : c->tws) {
        if (w.used) cudaEventSynchronize(w.done);
        cudaFree(w.d_fields);
        cudaFreeHost(w.h_fields);
        cudaFree(w.d_seg);
        if (w.done) cudaEventDestroy(w.done);
    }
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

int ldg_set_filter(ldg_ctx* c, int32_t which, const double* reim, int64_t nbins) {
    if (!c || !reim) return fail(LDG_ERR_ARG, "ldg_set_filter: NULL argument");
    if (which < 0 || which >= LDG_NFILTERS) return fail(LDG_ERR_ARG, "ldg_set_filter: bad filter slot");
    if (nbins != ldg::kM + 1) return fail(LDG_ERR_ARG, "ldg_set_filter: nbins must be blocklen/2+1");
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    std::vector<float2> h(nbins);
    for (int64_t k = 0; k < nbins; ++k) h[k] = make_float2((float)reim[2 * k], (float)reim[2 * k + 1]);
    int klo = (int)nbins, khi = -1;
    for (int k = 0; k < (int)nbins; ++k)
        if (h[k].x != 0.f || h[k].y != 0.f) {
            klo = std::min(klo, k);
            khi = k;
        }
    // the in-place variant's layouts of the same float32 values: per bin pair
    // u the bins k = bin_of(pair_pos(u)) and M - k (M itself for k = 0), and
    // for the RFVideo filters every bin at its position
    std::vector<float4> fp(ldg::ip::kPairs);
    for (int u = 0; u < ldg::ip::kPairs; ++u) {
        const int k = ldg::ip::bin_of(ldg::ip::pair_pos(u));
        const int m = k == 0 ? ldg::kM : ldg::kM - k;
        fp[u] = make_float4(h[k].x, h[k].y, h[m].x, h[m].y);
    }
    const bool pos = which == LDG_F_VIDEO_G || which == LDG_F_VIDEO_G_ODD;
    std::vector<float2> fq(pos ? ldg::kM : 0);
    for (int p = 0; p < (int)fq.size(); ++p) fq[p] = h[ldg::ip::bin_of(p)];
    if (!c->d_filter[which]) LDG_CK(cudaMalloc(&c->d_filter[which], nbins * sizeof(float2)));
    if (!c->d_fpair[which]) LDG_CK(cudaMalloc(&c->d_fpair[which], fp.size() * sizeof(float4)));
    if (pos && !c->d_fpos[which]) LDG_CK(cudaMalloc(&c->d_fpos[which], fq.size() * sizeof(float2)));
    LDG_CK(cudaStreamSynchronize(c->stream));
    LDG_CK(cudaMemcpy(c->d_filter[which], h.data(), nbins * sizeof(float2), cudaMemcpyHostToDevice));
    LDG_CK(cudaMemcpy(c->d_fpair[which], fp.data(), fp.size() * sizeof(float4), cudaMemcpyHostToDevice));
    if (pos) LDG_CK(cudaMemcpy(c->d_fpos[which], fq.data(), fq.size() * sizeof(float2), cudaMemcpyHostToDevice));
    c->fband[which][0] = klo;
    c->fband[which][1] = khi;
    return LDG_OK;
}

int ldg_set_demod_variant(ldg_ctx* c, int32_t variant) {
    if (!c) return fail(LDG_ERR_ARG, "ldg_set_demod_variant: NULL context");
    if (variant < 0 || variant >= ldg::kNumVariants)
        return fail(LDG_ERR_ARG, "ldg_set_demod_variant: variant must be LDG_VARIANT_STOCKHAM or LDG_VARIANT_IN_PLACE");
    std::lock_guard<std::mutex> lk(c->mu);
    c->variant = variant;
    return LDG_OK;
}

int ldg_set_demod_schedule(ldg_ctx* c, int32_t blocks_per_cta) {
    if (!c) return fail(LDG_ERR_ARG, "ldg_set_demod_schedule: NULL context");
    if (blocks_per_cta < 0 || blocks_per_cta > 64)
        return fail(LDG_ERR_ARG, "ldg_set_demod_schedule: blocks_per_cta must be in [0, 64]");
    std::lock_guard<std::mutex> lk(c->mu);
    c->blocks_per_cta = blocks_per_cta;
    return LDG_OK;
}

int ldg_get_demod_variant(ldg_ctx* c, int32_t* variant) {
    if (!c || !variant) return fail(LDG_ERR_ARG, "ldg_get_demod_variant: NULL argument");
    std::lock_guard<std::mutex> lk(c->mu);
    *variant = c->variant;
    return LDG_OK;
}

int ldg_set_audio(ldg_ctx* c, int32_t ch, int32_t lowbin, int32_t nbins, const double* filt1, double a1_freq,
                  double low_freq) {
    if (!c || !filt1) return fail(LDG_ERR_ARG, "ldg_set_audio: NULL argument");
    if (ch < 0 || ch > 1) return fail(LDG_ERR_ARG, "ldg_set_audio: channel must be 0 or 1");
    if (nbins != 1024) return fail(LDG_ERR_UNSUPPORTED, "ldg_set_audio: only 1024-bin audio bands are supported");
    if (lowbin < 1 || lowbin + nbins / 2 > ldg::kM / 2)
        return fail(LDG_ERR_ARG, "ldg_set_audio: band outside the spectrum");
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    std::vector<float2> h(nbins / 2 + 1);
    for (int k = 0; k <= nbins / 2; ++k) h[k] = make_float2((float)filt1[2 * k], (float)filt1[2 * k + 1]);
    if (!c->d_audio[ch]) LDG_CK(cudaMalloc(&c->d_audio[ch], h.size() * sizeof(float2)));
    LDG_CK(cudaStreamSynchronize(c->stream));
    LDG_CK(cudaMemcpy(c->d_audio[ch], h.data(), h.size() * sizeof(float2), cudaMemcpyHostToDevice));
    c->a_lowbin[ch] = lowbin;
    c->a_rate[ch] = a1_freq;
    c->a_low[ch] = low_freq;
    return LDG_OK;
}

int ldg_set_sinc_lut(ldg_ctx* c, const float* lut, int32_t rows, int32_t taps) {
    if (!c || !lut) return fail(LDG_ERR_ARG, "ldg_set_sinc_lut: NULL argument");
    if (rows != 65537 || taps != 16) return fail(LDG_ERR_UNSUPPORTED, "ldg_set_sinc_lut: table must be 65537 x 16");
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    // device layout for the gather: per phase p < 65536 and tap pair k < 8
    // one float4 (w[p][2k], w[p][2k+1], w[p+1][2k] - w[p][2k],
    // w[p+1][2k+1] - w[p][2k+1]), the differences rounded to float32 as the
    // kernel's own subtraction would be; one 16-byte load per lane and pixel
    std::vector<float> h((size_t)ldg::kLutPhases * 32);
    for (int ph = 0; ph < ldg::kLutPhases; ++ph) {
        const float* a = lut + (size_t)ph * 16;
        const float* b = a + 16;
        float* o = h.data() + (size_t)ph * 32;
        for (int k = 0; k < 8; ++k) {
            o[4 * k + 0] = a[2 * k];
            o[4 * k + 1] = a[2 * k + 1];
            o[4 * k + 2] = b[2 * k] - a[2 * k];
            o[4 * k + 3] = b[2 * k + 1] - a[2 * k + 1];
        }
    }
    const size_t bytes = h.size() * sizeof(float);
    if (!c->d_lut) LDG_CK(cudaMalloc(&c->d_lut, bytes));
    LDG_CK(cudaStreamSynchronize(c->stream));
    LDG_CK(cudaMemcpy(c->d_lut, h.data(), bytes, cudaMemcpyHostToDevice));
    return LDG_OK;
}

int ldg_set_notch(ldg_ctx* c, int32_t lo, int32_t hi) {
    if (!c) return fail(LDG_ERR_ARG, "ldg_set_notch: NULL context");
    if (!(lo == 0 && hi == 0) && !(lo >= 2 && hi > lo && hi <= ldg::kM - 2 && hi - lo <= 1024))
        return fail(LDG_ERR_ARG, "ldg_set_notch: the band must satisfy 2 <= lo < hi <= blocklen/2 - 2, at most 1024 bins");
    std::lock_guard<std::mutex> lk(c->mu);
    c->notch_lo = lo;
    c->notch_hi = hi;
    return LDG_OK;
}

int ldg_demod_scratch_bytes(ldg_ctx* c, int64_t nblocks, int64_t* bytes) {
    if (!c || !bytes) return fail(LDG_ERR_ARG, "ldg_demod_scratch_bytes: NULL argument");
    const long long grid = nblocks < c->sms ? nblocks : c->sms;
    *bytes = (int64_t)(grid * ldg::kScratchPerCta);
    return LDG_OK;
}

int ldg_demod_blocks(ldg_ctx* c, const ldg_demod_args* a) {
    if (!c || !a) return fail(LDG_ERR_ARG, "ldg_demod_blocks: NULL argument");
    if (!a->in) return fail(LDG_ERR_ARG, "demodblock called without raw or FFT data");
    if (a->in_kind != LDG_IN_INT16 && a->in_kind != LDG_IN_FLOAT32)
        return fail(LDG_ERR_ARG, "ldg_demod_blocks: in_kind must be LDG_IN_INT16 or LDG_IN_FLOAT32");
    if (a->nblocks < 0 || a->in_stride < 0) return fail(LDG_ERR_ARG, "ldg_demod_blocks: negative size");
    if (a->nblocks > (1LL << 30)) return fail(LDG_ERR_ARG, "ldg_demod_blocks: too many blocks");
    const int N = ldg::kN;
    if (!slice_ok(a->video, N) || !slice_ok(a->rfhpf, N) || !slice_ok(a->efm, N) || !slice_ok(a->audio, 1024))
        return fail(LDG_ERR_ARG, "ldg_demod_blocks: output slice outside the block");
    if (a->roll_05 < 0 || a->roll_05 >= N || a->roll_burst < 0 || a->roll_burst >= N)
        return fail(LDG_ERR_ARG, "ldg_demod_blocks: roll outside the block");
    std::lock_guard<std::mutex> lk(c->mu);
    if (!c->d_filter[LDG_F_VIDEO_G] || !c->d_filter[LDG_F_VIDEO_G_ODD])
        return fail(LDG_ERR_STATE, "ldg_demod_blocks: RFVideo filter not set");
    const bool want_video[4] = {a->out_demod != nullptr, a->out_05 != nullptr, a->out_burst != nullptr,
                                a->out_pilot != nullptr};
    const int fslot[4] = {LDG_F_DEMOD, LDG_F_05, LDG_F_BURST, LDG_F_PILOT};
    for (int o = 0; o < 4; ++o)
        if (want_video[o] && !c->d_filter[fslot[o]]) return fail(LDG_ERR_STATE, "ldg_demod_blocks: video filter not set");
    if (a->out_rfhpf && !c->d_filter[LDG_F_RFHPF]) return fail(LDG_ERR_STATE, "ldg_demod_blocks: rfhpf filter not set");
    if (a->out_efm && !c->d_filter[LDG_F_EFM]) return fail(LDG_ERR_STATE, "ldg_demod_blocks: EFM filter not set");
    const bool audio = a->out_audio_left || a->out_audio_right;
    if (audio && (!c->d_audio[0] || !c->d_audio[1])) return fail(LDG_ERR_STATE, "ldg_demod_blocks: audio bands not set");
    if (a->nblocks == 0) return LDG_OK;

    DeviceGuard g(c->device);
    cudaStream_t st = a->stream ? (cudaStream_t)a->stream : c->stream;
    const long long nb = a->nblocks;
    // one CTA per block; scratch slots for twice the SMs' worth of resident CTAs
    const int nslots = 2 * c->sms;
    // two blocks per CTA amortise its set-up on large batches, unless set
    const int per_cta = c->blocks_per_cta ? c->blocks_per_cta : (nb >= 16 * c->sms ? 2 : 1);
    const int grid = (int)((nb + per_cta - 1) / per_cta);
    int rc = grow((void**)&c->d_scratch, &c->scratch_bytes, (size_t)nslots * ldg::kScratchPerCta);
    if (rc) return rc;
    if (!c->d_slots) {
        LDG_CK(cudaMalloc(&c->d_slots, (nslots + 1) * sizeof(int)));
        LDG_CK(cudaMemset(c->d_slots, 0, (nslots + 1) * sizeof(int)));
        c->nslots = nslots;
    }

    // host/device placement of every buffer; host ones go through the arena
    const size_t esz = a->in_kind == LDG_IN_INT16 ? 2 : 4;
    const size_t in_elems = (size_t)((nb - 1) * a->in_stride + N);
    struct Buf { void* user; size_t bytes; size_t off; bool host; };
    Buf bufs[10];
    int nbuf = 0;
    auto add = [&](void* p, size_t bytes) -> int {
        const int i = nbuf++;
        bufs[i].user = p;
        bufs[i].bytes = bytes;
        bufs[i].host = p && !is_device_ptr(p);
        bufs[i].off = 0;
        return i;
    };
    const int i_in = add(const_cast<void*>(a->in), in_elems * esz);
    float* vids[4] = {a->out_demod, a->out_05, a->out_burst, a->out_pilot};
    int i_vid[4];
    for (int o = 0; o < 4; ++o) i_vid[o] = add(vids[o], (size_t)nb * a->video.len * 4);
    const int i_raw = add(a->out_raw, (size_t)nb * a->video.len * 4);
    const int i_hp = add(a->out_rfhpf, (size_t)nb * a->rfhpf.len * 4);
    const int i_efm = add(a->out_efm, (size_t)nb * a->efm.len * 2);
    const int i_al = add(a->out_audio_left, (size_t)nb * a->audio.len * 4);
    const int i_ar = add(a->out_audio_right, (size_t)nb * a->audio.len * 4);
    size_t stage = 0;
    bool any_host = false;
    for (int i = 0; i < nbuf; ++i) {
        if (bufs[i].host && bufs[i].bytes) {
            bufs[i].off = stage;
            stage += (bufs[i].bytes + 255) & ~size_t(255);
            any_host = true;
        }
    }
    if (stage) {
        rc = grow((void**)&c->d_stage, &c->stage_bytes, stage);
        if (rc) return rc;
    }
    auto dev = [&](int i) -> void* {
        if (!bufs[i].user) return nullptr;
        return bufs[i].host ? (void*)(c->d_stage + bufs[i].off) : bufs[i].user;
    };
    // the kernel reads samples in pairs: 4-byte (int16) / 8-byte (float32) aligned block starts
    if ((a->in_stride & 1) != 0 || (reinterpret_cast<uintptr_t>(dev(i_in)) & (esz == 2 ? 3 : 7)) != 0)
        return fail(LDG_ERR_ARG, "ldg_demod_blocks: input blocks must start on an even sample of an aligned buffer");
    if (bufs[i_in].host) LDG_CK(cudaMemcpyAsync(dev(i_in), a->in, bufs[i_in].bytes, cudaMemcpyHostToDevice, st));

    ldg::DemodParams p;
    memset(&p, 0, sizeof(p));
    p.in = dev(i_in);
    p.in_kind = a->in_kind;
    p.in_stride = a->in_stride;
    p.nblocks = (int)nb;
    p.fs_hz = (float)c->fs_hz;
    p.f_rfhpf = c->d_filter[LDG_F_RFHPF];
    p.f_g = c->d_filter[LDG_F_VIDEO_G];
    p.f_godd = c->d_filter[LDG_F_VIDEO_G_ODD];
    for (int o = 0; o < 4; ++o) {
        p.f_video[o] = c->d_filter[fslot[o]];
        p.o_video[o] = (float*)dev(i_vid[o]);
    }
    p.f_efm = c->d_filter[LDG_F_EFM];
    p.o_raw = (float*)dev(i_raw);
    p.o_rfhpf = a->rfhpf.len ? (float*)dev(i_hp) : nullptr;
    p.o_efm = a->efm.len ? (int16_t*)dev(i_efm) : nullptr;
    p.s_video = {a->video.start, a->video.len, 0};
    if (a->video.len == 0)
        for (int o = 0; o < 4; ++o) p.o_video[o] = nullptr;
    if (a->video.len == 0) p.o_raw = nullptr;
    p.roll[ldg::OUT_DEMOD] = 0;
    p.roll[ldg::OUT_05] = a->roll_05;
    p.roll[ldg::OUT_BURST] = a->roll_burst;
    p.roll[ldg::OUT_PILOT] = 0;
    p.s_rfhpf = {a->rfhpf.start, a->rfhpf.len, 0};
    p.s_efm = {a->efm.start, a->efm.len, 0};
    p.audio = audio && a->audio.len > 0;
    for (int ch = 0; ch < 2; ++ch) {
        p.a_lowbin[ch] = c->a_lowbin[ch];
        p.a_filt1[ch] = c->d_audio[ch];
        p.a_low[ch] = (float)c->a_low[ch];
    }
    p.a_rate = (float)c->a_rate[0];
    p.o_audio[0] = (float*)dev(i_al);
    p.o_audio[1] = (float*)dev(i_ar);
    p.s_audio = {a->audio.start, a->audio.len, 0};
    p.scratch = c->d_scratch;
    p.tw16 = c->d_tw16;
    p.tw32 = c->d_tw32;
    LDG_CK(cudaMemsetAsync(c->d_slots, 0, c->nslots * sizeof(int), st));
    p.slot_lock = c->d_slots;
    p.nslots = c->nslots;
    p.error = c->d_slots + c->nslots;
    p.blocks_per_cta = per_cta;
    p.notch_lo = c->notch_lo;
    p.notch_hi = c->notch_hi;
    variant_tables(c, &p);

    cudaError_t e = ldg::launch_demod(p, grid, st);
    if (e != cudaSuccess) return fail(LDG_ERR_CUDA, std::string("demod launch: ") + cudaGetErrorString(e));
    if (any_host) {
        for (int i = 1; i < nbuf; ++i)
            if (bufs[i].host && bufs[i].bytes)
                LDG_CK(cudaMemcpyAsync(bufs[i].user, dev(i), bufs[i].bytes, cudaMemcpyDeviceToHost, st));
        LDG_CK(cudaStreamSynchronize(st));
    }
    return LDG_OK;
}

int ldg_tbc_fields(ldg_ctx* c, const ldg_tbc_field* fields, int32_t nfields, void* stream) {
    if (!c || (!fields && nfields)) return fail(LDG_ERR_ARG, "ldg_tbc_fields: NULL argument");
    if (nfields < 0) return fail(LDG_ERR_ARG, "ldg_tbc_fields: negative field count");
    if (nfields == 0) return LDG_OK;
    std::lock_guard<std::mutex> lk(c->mu);
    if (!c->d_lut) return fail(LDG_ERR_STATE, "ldg_tbc_fields: sinc table not set");
    size_t ll_total = 0, seg_total = 0, spl_total = 0;
    long long max_nout = 0;
    for (int i = 0; i < nfields; ++i) {
        const ldg_tbc_field& f = fields[i];
        const int rc = check_tbc_field(f, "ldg_tbc_fields");
        if (rc) return rc;
        ll_total += f.nlines;
        seg_total += f.nlines - 1;
        spl_total += tbc_spline_doubles(f);
        if ((long long)f.linesout * f.outwidth > max_nout) max_nout = (long long)f.linesout * f.outwidth;
    }
    DeviceGuard g(c->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    int rc = grow((void**)&c->d_ll, &c->ll_cap, ll_total * sizeof(double));
    if (rc) return rc;
    rc = grow((void**)&c->d_seg, &c->seg_cap, (3 * seg_total + spl_total) * sizeof(double));
    if (rc) return rc;
    if (nfields > c->fields_cap) {
        cudaFree(c->d_fields);
        c->d_fields = nullptr;
        c->fields_cap = 0;
        LDG_CK(cudaMalloc(&c->d_fields, nfields * sizeof(ldg::TbcField)));
        c->fields_cap = nfields;
    }
    // staging for host buffers / outputs
    std::vector<ldg::TbcField> h(nfields);
    std::vector<double> lls(ll_total);
    size_t stage = 0;
    struct Host { size_t buf_off, f32_off, u16_off; bool buf, f32, u16; };
    std::vector<Host> hs(nfields);
    for (int i = 0; i < nfields; ++i) {
        const ldg_tbc_field& f = fields[i];
        const size_t nout = (size_t)f.linesout * f.outwidth;
        Host& x = hs[i];
        x.buf = !is_device_ptr(f.buf);
        x.f32 = f.out_f32 && !is_device_ptr(f.out_f32);
        x.u16 = f.out_u16 && !is_device_ptr(f.out_u16);
        auto take = [&](size_t bytes) { size_t o = stage; stage += (bytes + 255) & ~size_t(255); return o; };
        x.buf_off = x.buf ? take((size_t)f.buf_len * 4) : 0;
        x.f32_off = x.f32 ? take(nout * 4) : 0;
        x.u16_off = x.u16 ? take(nout * 2) : 0;
    }
    bool any_host = stage > 0;
    if (stage) {
        rc = grow((void**)&c->d_stage, &c->stage_bytes, stage);
        if (rc) return rc;
    }
    size_t llo = 0, sego = 0, splo = 0;
    bool any_spline = false;
    for (int i = 0; i < nfields; ++i) {
        const ldg_tbc_field& f = fields[i];
        ldg::TbcField& d = h[i];
        const Host& x = hs[i];
        const bool ll_dev = is_device_ptr(f.linelocs);
        if (!ll_dev) memcpy(lls.data() + llo, f.linelocs, f.nlines * sizeof(double));
        d.buf = x.buf ? (const float*)(c->d_stage + x.buf_off) : f.buf;
        if (x.buf) LDG_CK(cudaMemcpyAsync((void*)d.buf, f.buf, (size_t)f.buf_len * 4, cudaMemcpyHostToDevice, st));
        d.linelocs = ll_dev ? f.linelocs : c->d_ll + llo;
        fill_tbc_field(f, d, c->d_seg, seg_total, sego, c->d_seg + 3 * seg_total + splo, c->d_status);
        any_spline |= d.spline_k >= 2;
        d.out_f32 = x.f32 ? (float*)(c->d_stage + x.f32_off) : f.out_f32;
        d.out_u16 = x.u16 ? (uint16_t*)(c->d_stage + x.u16_off) : f.out_u16;
        llo += f.nlines;
        sego += f.nlines - 1;
        splo += tbc_spline_doubles(f);
    }
    // linelocs given in host memory: one copy for all of them (device ones were copied above)
    {
        size_t o = 0;
        for (int i = 0; i < nfields; ++i) {
            if (!is_device_ptr(fields[i].linelocs))
                LDG_CK(cudaMemcpyAsync(c->d_ll + o, lls.data() + o, fields[i].nlines * sizeof(double),
                                       cudaMemcpyHostToDevice, st));
            o += fields[i].nlines;
        }
    }
    LDG_CK(cudaMemcpyAsync(c->d_fields, h.data(), nfields * sizeof(ldg::TbcField), cudaMemcpyHostToDevice, st));
    cudaError_t e = ldg::launch_tbc(c->d_fields, nfields, max_nout, c->d_lut, 15.0, any_spline, st);
    if (e != cudaSuccess) return fail(LDG_ERR_CUDA, std::string("tbc launch: ") + cudaGetErrorString(e));
    if (any_host) {
        for (int i = 0; i < nfields; ++i) {
            const size_t nout = (size_t)fields[i].linesout * fields[i].outwidth;
            if (hs[i].f32) LDG_CK(cudaMemcpyAsync(fields[i].out_f32, h[i].out_f32, nout * 4, cudaMemcpyDeviceToHost, st));
            if (hs[i].u16) LDG_CK(cudaMemcpyAsync(fields[i].out_u16, h[i].out_u16, nout * 2, cudaMemcpyDeviceToHost, st));
        }
    }
    // the host copies of h/lls must stay alive until the async copies are done
    LDG_CK(cudaStreamSynchronize(st));
    int status = 0;
    LDG_CK(cudaMemcpy(&status, c->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (status) {
        LDG_CK(cudaMemset(c->d_status, 0, sizeof(int)));
        if (status & ldg::LDG_TBC_BAD_LINES) return fail(LDG_ERR_ARG, "ldg_tbc_fields: too many lines for the wow statistics");
        return fail(LDG_ERR_RANGE, "ldg_tbc_fields: a resampling tap fell outside the field buffer (those pixels are 0)");
    }
    (void)any_host;
    return LDG_OK;
}

int ldg_tbc_fields_async(ldg_ctx* c, const ldg_tbc_field* fields, int32_t nfields, void* stream) {
    if (!c || (!fields && nfields)) return fail(LDG_ERR_ARG, "ldg_tbc_fields_async: NULL argument");
    if (nfields < 0) return fail(LDG_ERR_ARG, "ldg_tbc_fields_async: negative field count");
    if (nfields == 0) return LDG_OK;
    std::lock_guard<std::mutex> lk(c->mu);
    if (!c->d_lut) return fail(LDG_ERR_STATE, "ldg_tbc_fields_async: sinc table not set");
    size_t seg_total = 0, spl_total = 0;
    long long max_nout = 0;
    for (int i = 0; i < nfields; ++i) {
        const ldg_tbc_field& f = fields[i];
        const int rc = check_tbc_field(f, "ldg_tbc_fields_async");
        if (rc) return rc;
        if (!f.out_f32 && !f.out_u16) return fail(LDG_ERR_ARG, "ldg_tbc_fields_async: no output");
        seg_total += f.nlines - 1;
        spl_total += tbc_spline_doubles(f);
        if ((long long)f.linesout * f.outwidth > max_nout) max_nout = (long long)f.linesout * f.outwidth;
    }
    DeviceGuard g(c->device);
    // every buffer must already be device memory (checked on the first field's
    // pointers; the batched callers allocate all fields alike)
    const ldg_tbc_field& f0 = fields[0];
    if (!is_device_ptr(f0.buf) || !is_device_ptr(f0.linelocs) || (f0.out_f32 && !is_device_ptr(f0.out_f32)) ||
        (f0.out_u16 && !is_device_ptr(f0.out_u16)))
        return fail(LDG_ERR_ARG, "ldg_tbc_fields_async: buffers must be device memory");
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    auto& w = c->tws[c->tws_next];
    c->tws_next = (c->tws_next + 1) % 4;
    if (w.used) LDG_CK(cudaEventSynchronize(w.done));
    if (!w.done) LDG_CK(cudaEventCreateWithFlags(&w.done, cudaEventDisableTiming));
    if (nfields > w.cap) {
        cudaFree(w.d_fields);
        cudaFreeHost(w.h_fields);
        w.d_fields = nullptr;
        w.h_fields = nullptr;
        w.cap = 0;
        LDG_CK(cudaMalloc(&w.d_fields, nfields * sizeof(ldg::TbcField)));
        LDG_CK(cudaMallocHost(&w.h_fields, nfields * sizeof(ldg::TbcField)));
        w.cap = nfields;
    }
    int rc = grow((void**)&w.d_seg, &w.seg_cap, (3 * seg_total + spl_total) * sizeof(double));
    if (rc) return rc;
    size_t sego = 0, splo = 0;
    bool any_spline = false;
    for (int i = 0; i < nfields; ++i) {
        const ldg_tbc_field& f = fields[i];
        ldg::TbcField& d = w.h_fields[i];
        d.buf = f.buf;
        d.linelocs = f.linelocs;
        fill_tbc_field(f, d, w.d_seg, seg_total, sego, w.d_seg + 3 * seg_total + splo, c->d_status);
        any_spline |= d.spline_k >= 2;
        d.out_f32 = f.out_f32;
        d.out_u16 = f.out_u16;
        sego += f.nlines - 1;
        splo += tbc_spline_doubles(f);
    }
    // descriptors read by SMs from the pinned workspace: a copy-engine transfer
    // would queue behind bulk output copies on the same engines
    void* hf = ldg::device_view(w.h_fields);
    if (hf) {
        LDG_CK(ldg::sm_copy(w.d_fields, hf, nfields * sizeof(ldg::TbcField), st));
    } else {
        LDG_CK(cudaMemcpyAsync(w.d_fields, w.h_fields, nfields * sizeof(ldg::TbcField), cudaMemcpyHostToDevice, st));
    }
    cudaError_t e = ldg::launch_tbc(w.d_fields, nfields, max_nout, c->d_lut, 15.0, any_spline, st);
    if (e != cudaSuccess) return fail(LDG_ERR_CUDA, std::string("tbc launch: ") + cudaGetErrorString(e));
    LDG_CK(cudaEventRecord(w.done, st));
    w.used = true;
    return LDG_OK;
}

int ldg_blocks_from_spectra(ldg_ctx* c, const double* spectra, int64_t nblocks, float* out, void* stream) {
    if (!c || (nblocks && (!spectra || !out))) return fail(LDG_ERR_ARG, "ldg_blocks_from_spectra: NULL argument");
    if (nblocks < 0 || nblocks > (1LL << 24)) return fail(LDG_ERR_ARG, "ldg_blocks_from_spectra: bad block count");
    if (nblocks == 0) return LDG_OK;
    if (!is_device_ptr(spectra) || !is_device_ptr(out))
        return fail(LDG_ERR_ARG, "ldg_blocks_from_spectra: buffers must be device memory");
    if ((reinterpret_cast<uintptr_t>(spectra) & 15) || (reinterpret_cast<uintptr_t>(out) & 7))
        return fail(LDG_ERR_ARG, "ldg_blocks_from_spectra: spectra must be 16-byte and out 8-byte aligned");
    DeviceGuard g(c->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    ldg::SpectrumParams p;
    p.spectra = reinterpret_cast<const double2*>(spectra);
    p.out = out;
    p.tw16 = c->d_tw16;
    p.tw32 = c->d_tw32;
    const cudaError_t e = ldg::launch_spectrum_blocks(p, (int)nblocks, st);
    if (e != cudaSuccess) return fail(LDG_ERR_CUDA, std::string("spectrum launch: ") + cudaGetErrorString(e));
    return LDG_OK;
}

int ldg_audio_phase2(ldg_ctx* c, const ldg_audio2_segment* segs, int32_t n, double center_left,
                     double center_right, void* stream) {
    if (!c || (!segs && n)) return fail(LDG_ERR_ARG, "ldg_audio_phase2: NULL argument");
    if (n < 0) return fail(LDG_ERR_ARG, "ldg_audio_phase2: negative segment count");
    for (int i = 0; i < n; ++i) {
        const ldg_audio2_segment& g = segs[i];
        if (!g.left || !g.right || !g.out_left || !g.out_right) return fail(LDG_ERR_ARG, "ldg_audio_phase2: NULL buffer");
        if (g.len < 2 || g.len > ldg::kN)
            return fail(LDG_ERR_ARG, "ldg_audio_phase2: a segment holds 2 .. blocklen samples");
    }
    if (n == 0) return LDG_OK;
    if (!is_device_ptr(segs[0].left) || !is_device_ptr(segs[0].out_left))
        return fail(LDG_ERR_ARG, "ldg_audio_phase2: buffers must be device memory");
    std::lock_guard<std::mutex> lk(c->mu);
    if (!c->d_filter[LDG_F_AUDIO2_LEFT] || !c->d_filter[LDG_F_AUDIO2_RIGHT])
        return fail(LDG_ERR_STATE, "ldg_audio_phase2: stage-2 audio filters not set");
    DeviceGuard g(c->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    if (!c->a2_done) LDG_CK(cudaEventCreateWithFlags(&c->a2_done, cudaEventDisableTiming));
    if (c->a2_used) LDG_CK(cudaEventSynchronize(c->a2_done));
    int rc = grow((void**)&c->d_a2, &c->a2_cap, (size_t)n * sizeof(ldg::Audio2Seg));
    if (rc) return rc;
    std::vector<ldg::Audio2Seg> h(n);
    for (int i = 0; i < n; ++i)
        h[i] = {segs[i].left, segs[i].right, (int)segs[i].len, segs[i].out_left, segs[i].out_right};
    LDG_CK(cudaMemcpyAsync(c->d_a2, h.data(), h.size() * sizeof(ldg::Audio2Seg), cudaMemcpyHostToDevice, st));
    ldg::Audio2Params p;
    memset(&p, 0, sizeof(p));
    p.segs = c->d_a2;
    p.cf32[0] = (float)center_left;
    p.cf32[1] = (float)center_right;
    p.cf[0] = center_left;
    p.cf[1] = center_right;
    p.filt[0] = c->d_filter[LDG_F_AUDIO2_LEFT];
    p.filt[1] = c->d_filter[LDG_F_AUDIO2_RIGHT];
    p.tw16 = c->d_tw16;
    p.tw32 = c->d_tw32;
    cudaError_t e = ldg::launch_audio2(p, n, st);
    if (e != cudaSuccess) return fail(LDG_ERR_CUDA, std::string("audio2 launch: ") + cudaGetErrorString(e));
    LDG_CK(cudaEventRecord(c->a2_done, st));
    c->a2_used = true;
    return LDG_OK;
}

int ldg_audio_downscale(ldg_ctx* c, const ldg_audio_field* fields, int32_t nfields, const ldg_audio_params* p,
                        int32_t* muted, void* stream) {
    if (!c || !p || (!fields && nfields)) return fail(LDG_ERR_ARG, "ldg_audio_downscale: NULL argument");
    if (nfields < 0) return fail(LDG_ERR_ARG, "ldg_audio_downscale: negative field count");
    if (!(p->line_period > 0) || !(p->linelen > 0) || !(p->scale > 0))
        return fail(LDG_ERR_ARG, "ldg_audio_downscale: line period, line length and scale must be positive");
    for (int i = 0; i < nfields; ++i) {
        const ldg_audio_field& f = fields[i];
        if (!f.audio_left || !f.audio_right || !f.linelocs || (f.nticks > 1 && !f.out))
            return fail(LDG_ERR_ARG, "ldg_audio_downscale: NULL buffer");
        if (f.audio_len <= 0 || f.nlines < 2) return fail(LDG_ERR_ARG, "ldg_audio_downscale: bad field geometry");
        if (f.nticks < 1 || f.nticks > ldg::kAudioMaxTicks)
            return fail(LDG_ERR_UNSUPPORTED, "ldg_audio_downscale: 1 .. 2048 ticks per field are supported");
        if (!(f.soundgap > 0)) return fail(LDG_ERR_ARG, "ldg_audio_downscale: soundgap must be positive");
    }
    if (nfields == 0) return LDG_OK;
    if (!is_device_ptr(fields[0].audio_left) || !is_device_ptr(fields[0].linelocs) ||
        (fields[0].out && !is_device_ptr(fields[0].out)) || (muted && !is_device_ptr(muted)))
        return fail(LDG_ERR_ARG, "ldg_audio_downscale: buffers must be device memory");
    DeviceGuard g(c->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    // the descriptors go in the launches' parameters: no device buffer, no wait
    std::vector<ldg::AudioField> h(nfields);
    for (int i = 0; i < nfields; ++i) {
        const ldg_audio_field& f = fields[i];
        h[i] = {f.audio_left, f.audio_right, f.audio_len, f.linelocs, f.nlines, f.nticks, f.timeoffset, f.soundgap,
                f.out};
    }
    const ldg::AudioConsts k{p->line_period, p->linelen, p->scale, p->lfreq, p->rfreq};
    cudaError_t e = ldg::launch_audio_downscale(h.data(), nfields, k, muted, st);
    if (e != cudaSuccess) return fail(LDG_ERR_CUDA, std::string("audio launch: ") + cudaGetErrorString(e));
    return LDG_OK;
}

int ldg_rf_tbc(ldg_ctx* c, const ldg_rftbc_field* fields, int32_t nfields, void* stream) {
    if (!c || (!fields && nfields)) return fail(LDG_ERR_ARG, "ldg_rf_tbc: NULL argument");
    if (nfields < 0) return fail(LDG_ERR_ARG, "ldg_rf_tbc: negative field count");
    int max_lines = 0;
    for (int i = 0; i < nfields; ++i) {
        const ldg_rftbc_field& f = fields[i];
        if (!f.input || !f.linelocs || !f.out) return fail(LDG_ERR_ARG, "ldg_rf_tbc: NULL buffer");
        if (f.len <= 0 || f.linelen <= 0 || f.linecount <= 0 || f.startline < 0)
            return fail(LDG_ERR_ARG, "ldg_rf_tbc: bad field geometry");
        if (f.startline + f.linecount >= f.nlines)
            return fail(LDG_ERR_ARG, "ldg_rf_tbc: lines startline .. startline + linecount must exist");
        if (f.linecount > max_lines) max_lines = f.linecount;
    }
    if (nfields == 0) return LDG_OK;
    if (!is_device_ptr(fields[0].input) || !is_device_ptr(fields[0].linelocs) || !is_device_ptr(fields[0].out))
        return fail(LDG_ERR_ARG, "ldg_rf_tbc: buffers must be device memory");
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    if (!c->rftbc_done) LDG_CK(cudaEventCreateWithFlags(&c->rftbc_done, cudaEventDisableTiming));
    if (c->rftbc_used) LDG_CK(cudaEventSynchronize(c->rftbc_done));
    int rc = grow((void**)&c->d_rftbc, &c->rftbc_cap, (size_t)nfields * sizeof(ldg::RfTbcField));
    if (rc) return rc;
    std::vector<ldg::RfTbcField> h(nfields);
    for (int i = 0; i < nfields; ++i) {
        const ldg_rftbc_field& f = fields[i];
        h[i] = {f.input, f.len, f.linelocs, f.nlines, f.startline, f.linecount, f.linelen, f.delay, f.out,
                c->d_status};
    }
    LDG_CK(cudaMemcpyAsync(c->d_rftbc, h.data(), h.size() * sizeof(ldg::RfTbcField), cudaMemcpyHostToDevice, st));
    cudaError_t e = ldg::launch_rf_tbc(c->d_rftbc, nfields, max_lines, st);
    if (e != cudaSuccess) return fail(LDG_ERR_CUDA, std::string("rf_tbc launch: ") + cudaGetErrorString(e));
    LDG_CK(cudaEventRecord(c->rftbc_done, st));
    c->rftbc_used = true;
    return LDG_OK;
}

int ldg_dropouts(ldg_ctx* c, const ldg_dropout_params* p, const ldg_dropout_field* fields, int32_t nfields,
                 int32_t* drops, int32_t* counts, double* rfstd, void* stream) {
    if (!c || !p || (!fields && nfields) || (nfields && (!drops || !counts)))
        return fail(LDG_ERR_ARG, "ldg_dropouts: NULL argument");
    if (nfields < 0) return fail(LDG_ERR_ARG, "ldg_dropouts: negative field count");
    if (p->system != LDG_NTSC && p->system != LDG_PAL) return fail(LDG_ERR_ARG, "ldg_dropouts: bad system");
    if (p->video_rot <= 0) return fail(LDG_ERR_ARG, "ldg_dropouts: video_rot must be positive");
    if (p->err_cap <= 0 || p->out_cap <= 0 || p->outlinelen <= 0)
        return fail(LDG_ERR_ARG, "ldg_dropouts: caps and outlinelen must be positive");
    if (!(p->hz_ire != 0) || !(p->freq_mhz > 0)) return fail(LDG_ERR_ARG, "ldg_dropouts: bad levels or rate");
    for (int i = 0; i < nfields; ++i) {
        const ldg_dropout_field& f = fields[i];
        if (!f.demod || !f.demod_05 || !f.demod_raw || !f.rfhpf || !f.linelocs)
            return fail(LDG_ERR_ARG, "ldg_dropouts: NULL buffer");
        if (f.len <= 0 || f.len > (1LL << 31) - 1) return fail(LDG_ERR_ARG, "ldg_dropouts: bad field length");
        if (f.nlines < 2 || f.nlines > ldg::kMaxDropRegions + 1)
            return fail(LDG_ERR_ARG, "ldg_dropouts: nlines must be in [2, 513]");
        if (f.lineoffset < 0 || f.linecount <= 0 || f.lineoffset + f.linecount + 1 >= f.nlines)
            return fail(LDG_ERR_ARG, "ldg_dropouts: lines lineoffset .. lineoffset + linecount + 1 must exist");
        if (f.hsync_len < 0) return fail(LDG_ERR_ARG, "ldg_dropouts: negative hsync length");
    }
    if (nfields == 0) return LDG_OK;
    const ldg_dropout_field& f0 = fields[0];
    if (!is_device_ptr(f0.demod) || !is_device_ptr(f0.linelocs) || !is_device_ptr(drops) || !is_device_ptr(counts))
        return fail(LDG_ERR_ARG, "ldg_dropouts: buffers must be device memory");
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    if (!c->drop_done) LDG_CK(cudaEventCreateWithFlags(&c->drop_done, cudaEventDisableTiming));
    if (c->drop_used) LDG_CK(cudaEventSynchronize(c->drop_done));
    int rc = grow((void**)&c->d_drop_fields, &c->drop_fields_cap, (size_t)nfields * sizeof(ldg::DropField));
    if (rc) return rc;
    rc = grow((void**)&c->d_drop_errs, &c->drop_errs_cap, (size_t)nfields * p->err_cap * sizeof(int));
    if (rc) return rc;
    std::vector<ldg::DropField> h(nfields);
    for (int i = 0; i < nfields; ++i) {
        const ldg_dropout_field& f = fields[i];
        h[i] = {f.demod, f.demod_05, f.demod_raw, f.rfhpf, f.len, f.linelocs, f.nlines, f.lineoffset, f.linecount,
                f.isfirst, f.hsync_len};
    }
    // pageable source: the copy has taken the data when the call returns
    LDG_CK(cudaMemcpyAsync(c->d_drop_fields, h.data(), h.size() * sizeof(ldg::DropField), cudaMemcpyHostToDevice, st));
    const bool pal = p->system == LDG_PAL;
    auto hz = [&](double ire) { return (float)(p->ire0 + p->hz_ire * ire); };
    ldg::DropConsts k;
    k.system = p->system;
    k.video_rot = p->video_rot;
    k.outlinelen = p->outlinelen;
    k.err_cap = p->err_cap;
    k.out_cap = p->out_cap;
    k.freq_mhz = p->freq_mhz;
    k.fhalf = p->freq_hz_half;
    // core.py:2846-2867: iretohz with DecoderParams, stored in float32 arrays
    k.vmin = hz(pal ? -70 : -50);
    k.vmax = hz(pal ? 150 : 160);
    k.vmin05 = hz(-30);
    k.vmax05 = hz(115);
    k.smin = hz(pal ? p->vsync_ire - 60 : p->vsync_ire - 35);
    k.smin05 = hz(p->vsync_ire - 10);
    cudaError_t e = ldg::launch_dropouts(c->d_drop_fields, nfields, k, c->d_drop_errs, drops, counts, rfstd, st);
    if (e != cudaSuccess) return fail(LDG_ERR_CUDA, std::string("dropout launch: ") + cudaGetErrorString(e));
    LDG_CK(cudaEventRecord(c->drop_done, st));
    c->drop_used = true;
    return LDG_OK;
}

int ldg_tbc_status(ldg_ctx* c, int32_t* flags) {
    if (!c || !flags) return fail(LDG_ERR_ARG, "ldg_tbc_status: NULL argument");
    DeviceGuard g(c->device);
    int status = 0;
    LDG_CK(cudaMemcpy(&status, c->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (status) LDG_CK(cudaMemset(c->d_status, 0, sizeof(int)));
    *flags = status;
    if (status & ldg::LDG_TBC_BAD_LINES) return fail(LDG_ERR_ARG, "TBC: too many lines for the wow statistics");
    if (status) return fail(LDG_ERR_RANGE, "TBC: a resampling tap fell outside the field buffer (those pixels are 0)");
    return LDG_OK;
}

int ldg_synchronize(ldg_ctx* c) {
    if (!c) return fail(LDG_ERR_ARG, "ldg_synchronize: NULL context");
    DeviceGuard g(c->device);
    LDG_CK(cudaStreamSynchronize(c->stream));
    return LDG_OK;
}

int ldg_demod_status(ldg_ctx* c, int32_t* flags) {
    if (!c || !flags) return fail(LDG_ERR_ARG, "ldg_demod_status: NULL argument");
    *flags = 0;
    if (!c->d_slots) return LDG_OK;
    DeviceGuard g(c->device);
    int v = 0;
    LDG_CK(cudaMemcpy(&v, c->d_slots + c->nslots, sizeof(int), cudaMemcpyDeviceToHost));
    if (v) LDG_CK(cudaMemset(c->d_slots + c->nslots, 0, sizeof(int)));
    *flags = v;
    if (v) return fail(LDG_ERR_CUDA, "demod: a block gave up waiting for a scratch slot and was skipped");
    return LDG_OK;
}

}  // extern "C"

namespace ldg {

int api_fail(int code, const std::string& msg) { return fail(code, msg); }

int lines_fail(int code, const std::string& msg) { return fail(code, msg); }

int ctx_device(const ldg_ctx* c) { return c->device; }

std::mutex& ctx_mutex(ldg_ctx* c) { return c->mu; }

cudaStream_t ctx_stream(const ldg_ctx* c) { return c->stream; }

int ctx_host_word(ldg_ctx* c, long long** host, long long** dev) {
    if (!c->h_word) {
        void* p = nullptr;
        LDG_CK(cudaHostAlloc(&p, 256, cudaHostAllocMapped));
        c->h_word = static_cast<long long*>(p);
    }
    void* d = nullptr;
    LDG_CK(cudaHostGetDevicePointer(&d, c->h_word, 0));
    *host = c->h_word;
    *dev = static_cast<long long*>(d);
    return LDG_OK;
}

int ctx_scan_state(ldg_ctx* c, long long ntiles, cudaStream_t st, ScanState* out) {
    if (!c->d_scan || ntiles > c->scan_cap || c->scan_dirty) {
        // a fresh state: tickets from 0, flags 0 (call numbers start at 1,
        // so no flag of a new call matches them)
        const long long cap = std::max<long long>(ntiles + ntiles / 4, 4096);
        if (c->d_scan) cudaFree(c->d_scan);
        c->d_scan = nullptr;
        c->scan_cap = 0;
        void* p = nullptr;
        LDG_CK(cudaMalloc(&p, (size_t)(1 + 3 * cap) * sizeof(unsigned long long)));
        c->d_scan = static_cast<unsigned long long*>(p);
        LDG_CK(cudaMemsetAsync(p, 0, (size_t)(1 + 3 * cap) * sizeof(unsigned long long), st));
        c->scan_cap = cap;
        c->scan_base = 0;
        c->scan_dirty = false;
    }
    out->ticket = c->d_scan;
    out->flags = c->d_scan + 1;
    out->agg = reinterpret_cast<long long*>(c->d_scan + 1 + c->scan_cap);
    out->incl = out->agg + c->scan_cap;
    out->base = c->scan_base;
    out->call = ++c->scan_call;
    c->scan_base += (unsigned long long)ntiles;
    return LDG_OK;
}

void ctx_scan_invalidate(ldg_ctx* c) { c->scan_dirty = true; }

int ctx_lines_scratch(ldg_ctx* c, size_t need, void** out) {
    int rc = grow(&c->d_lines, &c->lines_cap, need);
    *out = c->d_lines;
    return rc;
}

void* noalloc_stream(ldg_ctx* c, const ldg_demod_args* a) { return a->stream ? a->stream : (void*)c->stream; }

// Validates a batch whose buffers are all device memory and fills the
// kernel parameters from it and the context's filters (scheduling fields
// left zero).  `who` names the entry point in error messages.
int device_params(ldg_ctx* c, const ldg_demod_args* a, const std::string& who, DemodParams* p) {
    if (!c || !a) return fail(LDG_ERR_ARG, who + ": NULL argument");
    if (!a->in) return fail(LDG_ERR_ARG, "demodblock called without raw or FFT data");
    if (a->in_kind != LDG_IN_INT16 && a->in_kind != LDG_IN_FLOAT32)
        return fail(LDG_ERR_ARG, who + ": in_kind must be LDG_IN_INT16 or LDG_IN_FLOAT32");
    if (a->nblocks < 0 || a->in_stride < 0 || a->nblocks > (1LL << 30))
        return fail(LDG_ERR_ARG, who + ": bad block count or stride");
    const int N = kN;
    if (!slice_ok(a->video, N) || !slice_ok(a->rfhpf, N) || !slice_ok(a->efm, N) || !slice_ok(a->audio, 1024))
        return fail(LDG_ERR_ARG, who + ": output slice outside the block");
    if (a->roll_05 < 0 || a->roll_05 >= N || a->roll_burst < 0 || a->roll_burst >= N)
        return fail(LDG_ERR_ARG, who + ": roll outside the block");
    const void* ptrs[10] = {a->in, a->out_demod, a->out_raw, a->out_05, a->out_burst, a->out_pilot,
                            a->out_rfhpf, a->out_efm, a->out_audio_left, a->out_audio_right};
    for (const void* q : ptrs)
        if (q && !is_device_ptr(q)) return fail(LDG_ERR_ARG, who + ": all buffers must be device memory (no host staging)");
    std::lock_guard<std::mutex> lk(c->mu);
    if (!c->d_filter[LDG_F_VIDEO_G] || !c->d_filter[LDG_F_VIDEO_G_ODD])
        return fail(LDG_ERR_STATE, who + ": RFVideo filter not set");
    const int fslot[4] = {LDG_F_DEMOD, LDG_F_05, LDG_F_BURST, LDG_F_PILOT};
    float* vids[4] = {a->out_demod, a->out_05, a->out_burst, a->out_pilot};
    for (int o = 0; o < 4; ++o)
        if (vids[o] && !c->d_filter[fslot[o]]) return fail(LDG_ERR_STATE, who + ": video filter not set");
    if (a->out_rfhpf && !c->d_filter[LDG_F_RFHPF]) return fail(LDG_ERR_STATE, who + ": rfhpf filter not set");
    if (a->out_efm && !c->d_filter[LDG_F_EFM]) return fail(LDG_ERR_STATE, who + ": EFM filter not set");
    const bool audio = a->out_audio_left || a->out_audio_right;
    if (audio && (!c->d_audio[0] || !c->d_audio[1])) return fail(LDG_ERR_STATE, who + ": audio bands not set");
    const size_t esz = a->in_kind == LDG_IN_INT16 ? 2 : 4;
    if ((a->in_stride & 1) != 0 || (reinterpret_cast<uintptr_t>(a->in) & (esz == 2 ? 3 : 7)) != 0)
        return fail(LDG_ERR_ARG, who + ": input blocks must start on an even sample of an aligned buffer");

    memset(p, 0, sizeof(*p));
    p->in = a->in;
    p->in_kind = a->in_kind;
    p->in_stride = a->in_stride;
    p->nblocks = (int)a->nblocks;
    p->fs_hz = (float)c->fs_hz;
    p->f_rfhpf = c->d_filter[LDG_F_RFHPF];
    p->f_g = c->d_filter[LDG_F_VIDEO_G];
    p->f_godd = c->d_filter[LDG_F_VIDEO_G_ODD];
    for (int o = 0; o < 4; ++o) {
        p->f_video[o] = c->d_filter[fslot[o]];
        p->o_video[o] = a->video.len ? vids[o] : nullptr;
    }
    p->f_efm = c->d_filter[LDG_F_EFM];
    p->o_raw = a->video.len ? a->out_raw : nullptr;
    p->o_rfhpf = a->rfhpf.len ? a->out_rfhpf : nullptr;
    p->o_efm = a->efm.len ? a->out_efm : nullptr;
    p->s_video = {a->video.start, a->video.len, 0};
    p->roll[OUT_DEMOD] = 0;
    p->roll[OUT_05] = a->roll_05;
    p->roll[OUT_BURST] = a->roll_burst;
    p->roll[OUT_PILOT] = 0;
    p->s_rfhpf = {a->rfhpf.start, a->rfhpf.len, 0};
    p->s_efm = {a->efm.start, a->efm.len, 0};
    p->audio = audio && a->audio.len > 0;
    for (int ch = 0; ch < 2; ++ch) {
        p->a_lowbin[ch] = c->a_lowbin[ch];
        p->a_filt1[ch] = c->d_audio[ch];
        p->a_low[ch] = (float)c->a_low[ch];
    }
    p->a_rate = (float)c->a_rate[0];
    p->o_audio[0] = a->out_audio_left;
    p->o_audio[1] = a->out_audio_right;
    p->s_audio = {a->audio.start, a->audio.len, 0};
    p->tw16 = c->d_tw16;
    p->tw32 = c->d_tw32;
    p->notch_lo = c->notch_lo;
    p->notch_hi = c->notch_hi;
    variant_tables(c, p);
    return LDG_OK;
}

int noalloc_prepare(ldg_ctx* c, const ldg_demod_args* a, int ctas, int max_slots, DemodParams* p, int* grid,
                    int* device) {
    *grid = 0;
    if (ctas < 0 || ctas > max_slots)
        return fail(LDG_ERR_ARG, "ldg_demod_blocks_noalloc: ctas = " + std::to_string(ctas) +
                                     " exceeds the static scratch (" + std::to_string(max_slots) +
                                     " CTA slots of 256 KB); use 0 < ctas <= " + std::to_string(max_slots));
    const int rc = device_params(c, a, "ldg_demod_blocks_noalloc", p);
    if (rc) return rc;
    *device = c->device;
    if (a->nblocks == 0) return LDG_OK;
    const long long nb = a->nblocks;
    const int cap = ctas ? ctas : max_slots;
    *grid = (int)(nb < cap ? nb : cap);
    return LDG_OK;
}

}  // namespace ldg
