// AC3-RF front end on the GPU and the symbol-timing DPLL on the host.
//
// Restates lddecode/ac3rf.py: Ac3RfDemodulator.demodulate_to_symbols
// (ac3rf.py:372-396) -- two real half-band /2 stages (ac3rf.py:99-151), a
// 2.88 MHz mix with a 14-bit phase-accumulator NCO (ac3rf.py:352-357,
// 382-392), two complex half-band /2 stages and a root-raised-cosine matched
// filter (ac3rf.py:154-167, 343-349) -- and AC3_DPLL.reclock_symbols
// (ac3rf.py:232-299).
//
// The reference streams blocks through FIR stages that carry their history
// (zeros at the start) and decimation phase; every stage is a causal FIR, so
// output j of a stage is sum_k h[k] u[phi + D j - k] over its whole input
// history with u[i < 0] = 0, independent of how the input was chunked.  The
// GPU computes each stage that way over shared-memory tiles: one CTA makes
// kTile final (fs/16) samples from the input window it depends on.
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "ldg_ac3.h"
#include "ldg_attr.cuh"

namespace ldg {

namespace {

constexpr int kTile = 512;      // final samples per CTA
constexpr int kAc3Threads = 256;

struct Ac3Params {
    const void* in;             // absolute samples [in_first, in_first + nsamples)
    int in_kind;                // 0 int16, 1 float32
    long long in_first;
    long long nsamples;
    long long out_first;
    long long out_count;
    float* out_i;
    float* out_q;
    Ac3Taps taps;
};

__device__ __forceinline__ float tap_sum(const float* u, long long ulo, long long pos, const float* val,
                                         const int* off, int n) {
    // sum_k val[k] * u[pos - off[k]] in the reference's order; u[i] = 0 for i < 0
    float acc = 0.0f;
    for (int k = 0; k < n; ++k) {
        const long long i = pos - off[k];
        const float x = i < 0 ? 0.0f : u[i - ulo];
        acc = (k == 0) ? val[0] * x : fmaf(val[k], x, acc);
    }
    return acc;
}

__global__ void __launch_bounds__(kAc3Threads) ac3_frontend_kernel(const __grid_constant__ Ac3Params p) {
    extern __shared__ float sm[];
    const Ac3Taps& t = p.taps;
    const long long J = p.out_first + (long long)blockIdx.x * kTile;
    const long long Jend = min(J + (long long)kTile, p.out_first + p.out_count);
    if (J >= Jend) return;
    // index ranges of every stage this tile needs (inclusive lo, exclusive hi)
    const long long lo5 = J, hi5 = Jend;
    const long long lo4 = lo5 - (t.n_rrc - 1), hi4 = hi5;
    const long long lo3 = 2 * lo4 - (t.n_hb23 - 1), hi3 = 2 * (hi4 - 1) + 1;
    const long long lo2 = 2 * lo3 - (t.n_hb19 - 1), hi2 = 2 * (hi3 - 1) + 1;
    const long long lo1 = 2 * lo2 - (t.n_hb19 - 1), hi1 = 2 * (hi2 - 1) + 1;
    const long long lo0 = 2 * lo1 - (t.n_hb19 - 1), hi0 = 2 * (hi1 - 1) + 1;
    const int n0 = (int)(hi0 - lo0), n1 = (int)(hi1 - lo1), n2 = (int)(hi2 - lo2);
    const int n3 = (int)(hi3 - lo3), n4 = (int)(hi4 - lo4);
    float* u0 = sm;                 // input
    float* u1 = u0 + n0;            // stage 1
    float* u2 = u1 + n1;            // stage 2 (real), then mixed I in place
    float* q2 = u2 + n2;            // mixed Q
    float* i3 = q2 + n2;
    float* q3 = i3 + n3;
    float* i4 = q3 + n3;
    float* q4 = i4 + n4;
    for (int k = threadIdx.x; k < n0; k += blockDim.x) {
        const long long gi = lo0 + k - p.in_first;  // the host checked gi >= 0 wherever lo0 + k >= 0
        float v = 0.0f;
        if (lo0 + k >= 0 && gi >= 0 && gi < p.nsamples)
            v = p.in_kind == 0 ? (float)static_cast<const int16_t*>(p.in)[gi] : static_cast<const float*>(p.in)[gi];
        u0[k] = v;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n1; k += blockDim.x) {
        const long long j = lo1 + k;
        u1[k] = j < 0 ? 0.0f : tap_sum(u0, lo0, 2 * j, t.hb19_val, t.hb19_off, t.n_hb19_nz);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n2; k += blockDim.x) {
        const long long j = lo2 + k;
        float v = j < 0 ? 0.0f : tap_sum(u1, lo1, 2 * j, t.hb19_val, t.hb19_off, t.n_hb19_nz);
        // NCO: phase = (step * j) mod 2^bits, cos/sin tables
        const unsigned mask = (1u << t.lut_bits) - 1u;
        const unsigned ph = j < 0 ? 0u : (unsigned)(((unsigned long long)(j & mask) * (unsigned)t.phase_step) & mask);
        u2[k] = v * t.cos_lut[ph];
        q2[k] = v * t.sin_lut[ph];
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n3; k += blockDim.x) {
        const long long j = lo3 + k;
        i3[k] = j < 0 ? 0.0f : tap_sum(u2, lo2, 2 * j, t.hb19_val, t.hb19_off, t.n_hb19_nz);
        q3[k] = j < 0 ? 0.0f : tap_sum(q2, lo2, 2 * j, t.hb19_val, t.hb19_off, t.n_hb19_nz);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n4; k += blockDim.x) {
        const long long j = lo4 + k;
        i4[k] = j < 0 ? 0.0f : tap_sum(i3, lo3, 2 * j, t.hb23_val, t.hb23_off, t.n_hb23_nz);
        q4[k] = j < 0 ? 0.0f : tap_sum(q3, lo3, 2 * j, t.hb23_val, t.hb23_off, t.n_hb23_nz);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < (int)(hi5 - lo5); k += blockDim.x) {
        const long long j = lo5 + k;
        p.out_i[j - p.out_first] = tap_sum(i4, lo4, j, t.rrc_val, t.rrc_off, t.n_rrc_nz);
        p.out_q[j - p.out_first] = tap_sum(q4, lo4, j, t.rrc_val, t.rrc_off, t.n_rrc_nz);
    }
}

size_t tile_smem(const Ac3Taps& t) {
    const long long n4 = kTile + t.n_rrc - 1;
    const long long n3 = 2 * n4 - 1 + t.n_hb23 - 1;
    const long long n2 = 2 * n3 - 1 + t.n_hb19 - 1;
    const long long n1 = 2 * n2 - 1 + t.n_hb19 - 1;
    const long long n0 = 2 * n1 - 1 + t.n_hb19 - 1;
    return (size_t)(n0 + n1 + 2 * n2 + 2 * n3 + 2 * n4) * sizeof(float);
}

}  // namespace

long long ac3_history(const Ac3Taps& t) {
    // input samples before 16 * j that final output j depends on
    return 16LL * (t.n_rrc - 1) + 8LL * (t.n_hb23 - 1) + 7LL * (t.n_hb19 - 1);
}

cudaError_t launch_ac3_frontend(const void* in, int in_kind, long long in_first, long long nsamples,
                                long long out_first, long long out_count, float* out_i, float* out_q,
                                const Ac3Taps& taps, cudaStream_t stream) {
    if (out_count <= 0) return cudaSuccess;
    Ac3Params p;
    p.in = in;
    p.in_kind = in_kind;
    p.in_first = in_first;
    p.nsamples = nsamples;
    p.out_first = out_first;
    p.out_count = out_count;
    p.out_i = out_i;
    p.out_q = out_q;
    p.taps = taps;
    const size_t smem = tile_smem(taps);
    static SmemAttr attr;
    cudaError_t e = attr.ensure(ac3_frontend_kernel, smem);
    if (e != cudaSuccess) return e;
    const unsigned grid = (unsigned)((out_count + kTile - 1) / kTile);
    ac3_frontend_kernel<<<grid, kAc3Threads, smem, stream>>>(p);
    return cudaGetLastError();
}

size_t ac3_tile_smem(const Ac3Taps& t) { return tile_smem(t); }

// ---- symbol-timing DPLL (host, ac3rf.py:200-299)

Ac3Dpll::Ac3Dpll(double fs) {
    symbol_distance = (int)std::nearbyint(fs / kSymbolRate);
    nominal_add = (int)((double)(1 << kCounterBits) * kSymbolRate / fs);
    prev_i.assign(symbol_distance, 0.0f);
    prev_q.assign(symbol_distance, 0.0f);
    const double pi = 3.14159265358979323846;
    const double omega = 2 * pi * 1800, zeta = 0.6, ts = 1.0 / kSymbolRate, gain = 0.3;
    g1 = (1 - std::exp(-2 * zeta * omega * ts)) / gain;
    g2 = (1 + std::exp(-2 * omega * zeta * ts) -
          2 * std::exp(-omega * zeta * ts) * std::cos(omega * ts * std::sqrt(1 - zeta * zeta))) /
         gain;
}

long long Ac3Dpll::reclock(const float* in_i, const float* in_q, long long n, uint8_t* out) {
    const int mask = (1 << kCounterBits) - 1;
    const int sd = symbol_distance;
    long long count = 0;
    for (long long i = 0; i < n; ++i) {
        float di, dq;
        if (i >= sd) {
            di = in_i[i - sd];
            dq = in_q[i - sd];
        } else {
            di = prev_i[i];
            dq = prev_q[i];
        }
        const float re = in_i[i] * di + in_q[i] * dq;
        const float im = in_q[i] * di - in_i[i] * dq;
        int cur;
        if (std::fabs(re) >= std::fabs(im))
            cur = re >= 0 ? 0 : 3;
        else
            cur = im >= 0 ? 1 : 2;
        if (cur != prev_symbol) {
            toggle_position = clk_counter;
            number_of_toggles += 1;
        }
        prev_symbol = cur;
        const int new_counter = (clk_counter + nominal_add + filter_out) & mask;
        filter_out = 0;
        if (new_counter < clk_counter) {
            out[count++] = (uint8_t)prev_symbol;
            const int error = number_of_toggles == 1 ? -(toggle_position - (1 << (kCounterBits - 1))) : 0;
            int es = (error_sum + error) & ((1 << kErrorSumBits) - 1);
            if (es >= (1 << (kErrorSumBits - 1))) es -= 1 << kErrorSumBits;
            error_sum = es;
            filter_out = (int)(error * g1 + error_sum * g2);  // truncation toward zero, as int()
            number_of_toggles = 0;
        }
        clk_counter = new_counter;
    }
    // keep the last symbol_distance samples (of previous tail + this input) for the next call
    if (n >= sd) {
        for (int k = 0; k < sd; ++k) {
            prev_i[k] = in_i[n - sd + k];
            prev_q[k] = in_q[n - sd + k];
        }
    } else {
        std::vector<float> ti(prev_i.begin() + n, prev_i.end()), tq(prev_q.begin() + n, prev_q.end());
        ti.insert(ti.end(), in_i, in_i + n);
        tq.insert(tq.end(), in_q, in_q + n);
        prev_i.swap(ti);
        prev_q.swap(tq);
    }
    return count;
}

}  // namespace ldg

// ---- C ABI

#include "ldgpu.h"

namespace {
thread_local std::string g_ac3_err;
int ac3_fail(int code, const std::string& m) {
    g_ac3_err = m;
    return code;
}
}  // namespace

struct ldg_ac3 {
    int device = 0;
    ldg::Ac3Taps taps{};
    std::vector<void*> allocs;
    std::mutex mu;
};

struct ldg_ac3_dpll {
    ldg::Ac3Dpll d;
    explicit ldg_ac3_dpll(double fs) : d(fs) {}
};

extern "C" {

const char* ldg_ac3_last_error(void) { return g_ac3_err.c_str(); }

void ldg_ac3_destroy(ldg_ac3* a) {
    if (!a) return;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(a->device);
    for (void* p : a->allocs) cudaFree(p);
    if (prev >= 0) cudaSetDevice(prev);
    delete a;
}

int ldg_ac3_create(ldg_ac3** out, int32_t device, const float* hb19, int32_t n19, const float* hb23, int32_t n23,
                   const float* rrc, int32_t nrrc, int32_t lut_bits, const float* cos_lut, const float* sin_lut,
                   int32_t phase_step) {
    if (!out || !hb19 || !hb23 || !rrc || !cos_lut || !sin_lut) return ac3_fail(LDG_ERR_ARG, "ldg_ac3_create: NULL argument");
    *out = nullptr;
    if (n19 < 3 || n23 < 3 || nrrc < 1 || n19 > 255 || n23 > 255 || nrrc > 1023 || lut_bits < 4 || lut_bits > 20)
        return ac3_fail(LDG_ERR_ARG, "ldg_ac3_create: bad filter length or NCO table size");
    int prev = -1;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return ac3_fail(LDG_ERR_CUDA, "ldg_ac3_create: bad device");
    }
    ldg_ac3* a = new ldg_ac3();
    a->device = device;
    auto upload = [&](const void* src, size_t bytes) -> void* {
        void* d = nullptr;
        if (cudaMalloc(&d, bytes) != cudaSuccess) return nullptr;
        a->allocs.push_back(d);
        if (cudaMemcpy(d, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
        return d;
    };
    bool ok = true;
    auto nz = [&](const float* h, int n, const float** val, const int** off, int* nnz) {
        std::vector<float> v;
        std::vector<int> o;
        for (int k = 0; k < n; ++k)
            if (h[k] != 0.0f) {
                v.push_back(h[k]);
                o.push_back(k);
            }
        *nnz = (int)v.size();
        *val = static_cast<const float*>(upload(v.data(), v.size() * sizeof(float)));
        *off = static_cast<const int*>(upload(o.data(), o.size() * sizeof(int)));
        ok = ok && *val && *off && *nnz > 0;
    };
    ldg::Ac3Taps& t = a->taps;
    t.n_hb19 = n19;
    t.n_hb23 = n23;
    t.n_rrc = nrrc;
    nz(hb19, n19, &t.hb19_val, &t.hb19_off, &t.n_hb19_nz);
    nz(hb23, n23, &t.hb23_val, &t.hb23_off, &t.n_hb23_nz);
    nz(rrc, nrrc, &t.rrc_val, &t.rrc_off, &t.n_rrc_nz);
    const size_t lut_bytes = (size_t(1) << lut_bits) * sizeof(float);
    t.cos_lut = static_cast<const float*>(upload(cos_lut, lut_bytes));
    t.sin_lut = static_cast<const float*>(upload(sin_lut, lut_bytes));
    t.lut_bits = lut_bits;
    t.phase_step = phase_step;
    ok = ok && t.cos_lut && t.sin_lut;
    if (prev >= 0) cudaSetDevice(prev);
    if (!ok || ldg::ac3_tile_smem(t) > 227 * 1024) {
        const std::string msg = cudaGetErrorString(cudaGetLastError());
        ldg_ac3_destroy(a);
        return ac3_fail(LDG_ERR_CUDA, "ldg_ac3_create: " + msg);
    }
    *out = a;
    return LDG_OK;
}

int ldg_ac3_frontend(ldg_ac3* a, const void* in, int32_t in_kind, int64_t in_first, int64_t nsamples,
                     int64_t out_first, int64_t out_count, float* out_i, float* out_q, void* stream) {
    if (!a || !in || !out_i || !out_q) return ac3_fail(LDG_ERR_ARG, "ldg_ac3_frontend: NULL argument");
    if (in_kind != LDG_IN_INT16 && in_kind != LDG_IN_FLOAT32) return ac3_fail(LDG_ERR_ARG, "ldg_ac3_frontend: bad in_kind");
    if (nsamples < 0 || in_first < 0 || out_first < 0 || out_count < 0)
        return ac3_fail(LDG_ERR_ARG, "ldg_ac3_frontend: negative size");
    // after n inputs the reference has produced ceil(n/16) outputs
    const long long avail = (in_first + nsamples + 15) / 16;
    if (out_first + out_count > avail)
        return ac3_fail(LDG_ERR_ARG, "ldg_ac3_frontend: outputs beyond the input (at most ceil(end/16))");
    if (out_count && in_first > 0 && 16 * out_first - ldg::ac3_history(a->taps) < in_first)
        return ac3_fail(LDG_ERR_ARG, "ldg_ac3_frontend: the input window does not cover the filters' history");
    if (out_count == 0) return LDG_OK;
    std::lock_guard<std::mutex> lk(a->mu);
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(a->device);
    auto is_dev = [](const void* p) {
        cudaPointerAttributes at;
        if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
    };
    const size_t esz = in_kind == LDG_IN_INT16 ? 2 : 4;
    const bool hin = !is_dev(in), hi = !is_dev(out_i), hq = !is_dev(out_q);
    cudaStream_t st = (cudaStream_t)stream;
    void *din = const_cast<void*>(in), *dio = out_i, *dqo = out_q;
    std::vector<void*> tmp;
    auto fail_cuda = [&](const char* what) {
        for (void* p : tmp) cudaFree(p);
        if (prev >= 0) cudaSetDevice(prev);
        return ac3_fail(LDG_ERR_CUDA, std::string("ldg_ac3_frontend: ") + what + ": " +
                                          cudaGetErrorString(cudaGetLastError()));
    };
    if (hin) {
        if (cudaMalloc(&din, nsamples * esz) != cudaSuccess) return fail_cuda("cudaMalloc");
        tmp.push_back(din);
        if (cudaMemcpyAsync(din, in, nsamples * esz, cudaMemcpyHostToDevice, st) != cudaSuccess) return fail_cuda("H2D");
    }
    if (hi) {
        if (cudaMalloc(&dio, out_count * 4) != cudaSuccess) return fail_cuda("cudaMalloc");
        tmp.push_back(dio);
    }
    if (hq) {
        if (cudaMalloc(&dqo, out_count * 4) != cudaSuccess) return fail_cuda("cudaMalloc");
        tmp.push_back(dqo);
    }
    if (ldg::launch_ac3_frontend(din, in_kind, in_first, nsamples, out_first, out_count, (float*)dio, (float*)dqo,
                                 a->taps, st) != cudaSuccess)
        return fail_cuda("launch");
    if (hi && cudaMemcpyAsync(out_i, dio, out_count * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess) return fail_cuda("D2H");
    if (hq && cudaMemcpyAsync(out_q, dqo, out_count * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess) return fail_cuda("D2H");
    if (!tmp.empty()) {
        if (cudaStreamSynchronize(st) != cudaSuccess) return fail_cuda("sync");
        for (void* p : tmp) cudaFree(p);
    }
    if (prev >= 0) cudaSetDevice(prev);
    return LDG_OK;
}

int ldg_ac3_dpll_create(ldg_ac3_dpll** out, double final_fs) {
    if (!out) return ac3_fail(LDG_ERR_ARG, "ldg_ac3_dpll_create: NULL argument");
    if (!(final_fs >= 2 * ldg::kSymbolRate) || final_fs > 1e9)
        return ac3_fail(LDG_ERR_ARG, "ldg_ac3_dpll_create: sample rate must be >= 2 x 288 kHz");
    *out = new ldg_ac3_dpll(final_fs);
    return LDG_OK;
}

void ldg_ac3_dpll_destroy(ldg_ac3_dpll* d) { delete d; }

int ldg_ac3_dpll_reclock(ldg_ac3_dpll* d, const float* in_i, const float* in_q, int64_t n, uint8_t* out,
                         int64_t* nout) {
    if (!d || (!in_i && n) || (!in_q && n) || (!out && n) || !nout)
        return ac3_fail(LDG_ERR_ARG, "ldg_ac3_dpll_reclock: NULL argument");
    if (n < 0) return ac3_fail(LDG_ERR_ARG, "ldg_ac3_dpll_reclock: negative length");
    *nout = d->d.reclock(in_i, in_q, n, out);
    return LDG_OK;
}

}  // extern "C"
