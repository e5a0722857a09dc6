// AC3-RF front end (GPU) and symbol-timing DPLL (host) internals.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

namespace ldg {

// Filter taps of the front end, device pointers; only non-zero taps are
// stored (value + index), in ascending index order like the reference.
struct Ac3Taps {
    const float* hb19_val;
    const int* hb19_off;
    int n_hb19, n_hb19_nz;      // full length, non-zero count
    const float* hb23_val;
    const int* hb23_off;
    int n_hb23, n_hb23_nz;
    const float* rrc_val;
    const int* rrc_off;
    int n_rrc, n_rrc_nz;
    const float* cos_lut;
    const float* sin_lut;
    int lut_bits;
    int phase_step;
};

cudaError_t launch_ac3_frontend(const void* in, int in_kind, long long in_first, long long nsamples,
                                long long out_first, long long out_count, float* out_i, float* out_q,
                                const Ac3Taps& taps, cudaStream_t stream);
long long ac3_history(const Ac3Taps& t);
size_t ac3_tile_smem(const Ac3Taps& t);

constexpr double kSymbolRate = 288e3;
constexpr int kCounterBits = 10;
constexpr int kErrorSumBits = 15;

struct Ac3Dpll {
    int symbol_distance = 0;
    int nominal_add = 0;
    std::vector<float> prev_i, prev_q;
    int prev_symbol = 0;
    int error_sum = 0;
    int filter_out = 0;
    int clk_counter = 0;
    int toggle_position = 0;
    int number_of_toggles = 0;
    double g1 = 0, g2 = 0;
    explicit Ac3Dpll(double fs);
    long long reclock(const float* in_i, const float* in_q, long long n, uint8_t* out);
};

}  // namespace ldg
