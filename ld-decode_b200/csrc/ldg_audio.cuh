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

// Up to kAudioBatch field descriptors travel in the kernel's parameters
// (8 KB), so a launch needs no device descriptor buffer and the host never
// waits for an earlier launch.
constexpr int kAudioBatch = 128;
struct AudioBatch {
    AudioField f[kAudioBatch];
};

// fields: host array of n descriptors (any n; launched kAudioBatch at a time)
cudaError_t launch_audio_downscale(const AudioField* fields, int nfields, AudioConsts c, int* muted,
                                   cudaStream_t stream);

}  // namespace ldg
