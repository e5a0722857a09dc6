// Dropout detection kernel (Field.dropout_detect, lddecode/core.py:2829-2983).
#pragma once
#include <cuda_runtime.h>

namespace ldg {

constexpr int kDropThreads = 512;
constexpr int kMaxDropRegions = 512;  // sync areas: lines 1 .. nlines-1, nlines <= 513

struct DropField {
    const float* demod;
    const float* d05;
    const float* raw;
    const float* rfhpf;
    long long len;
    const double* ll;
    int nlines, lineoffset, linecount, isfirst, hsync_len;
};

struct DropConsts {
    int system, video_rot, outlinelen, err_cap, out_cap;
    double freq_mhz, fhalf;
    float vmin, vmax, vmin05, vmax05, smin, smin05;  // float32 limits (Hz)
};

cudaError_t launch_dropouts(const DropField* fields, int nfields, const DropConsts& k, int* errs, int* drops,
                            int* counts, double* rfstd, cudaStream_t stream);

}  // namespace ldg
