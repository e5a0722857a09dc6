// Device-side descriptors of the analog audio downscale.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ldg {

constexpr int kAudioMaxTicks = 2048;  // output samples + 1 per field

struct AudioField {
    const float* al;
    const float* ar;
    long long len;
    const double* ll;
    int nlines;
    int nticks;
    double timeoffset, soundgap;
    int16_t* out;
};

struct AudioConsts {
    double line_period, linelen, scale, lfreq, rfreq;
};

cudaError_t launch_audio_downscale(const AudioField* dfields, int nfields, AudioConsts c, int* muted,
                                   cudaStream_t stream);

}  // namespace ldg
