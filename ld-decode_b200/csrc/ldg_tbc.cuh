// Device-side descriptor of one field for the TBC kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ldg {

enum { LDG_TBC_BAD_LINES = 1, LDG_TBC_OUT_OF_RANGE = 2 };

struct TbcField {
    const float* buf;
    long long buf_len;
    const double* linelocs;
    int nlines;
    int lineoffset;
    int outwidth;
    int linesout;
    long long nwow;      // pixels in the wow statistics: (outlinecount+lineoffset+1)*outlinelen
    int coord_f32;
    double inlinelen;
    double outscale;     // inlinelen / outlinelen
    double inv_inl;      // 1.0 / inlinelen (the degree-1 spline basis weight)
    double u16_scale;    // out_scale / hz_ire
    double u16_offset;   // output_zero - vsync_ire*out_scale - ire0*u16_scale
    double* seg_level;   // nlines-1 level-adjust factors (device scratch)
    double smooth_b;     // 1 - alpha of the level-adjust IIR, 0: off
    double* seg_start;   // with the IIR: the smoothed level just before segment j
    long long* seg_lo;   // first wow pixel of segment j
    int* status;         // LDG_TBC_* bits
    float* out_f32;
    uint16_t* out_u16;
    // quadratic / cubic wow interpolation (spline_k 2 / 3; 1: the linear
    // segments above)
    int spline_k;
    int npieces;         // polynomial pieces: nlines - 1 (cubic), nlines - 2 (quadratic)
    double* spl;         // kSplStride doubles per piece: left edge, anchor, c0..c3 (scratch)
    double* stat;        // median, outlier threshold of the wow factors (scratch)
    double* ybefore;     // with the IIR: smoothed level just before output pixel 32*m (scratch)
    double smooth_a;     // alpha of the level-adjust IIR
};

constexpr int kSplStride = 6;
constexpr int kLutPhases = 65536;  // sinc table phases (rows 0..65536, the last a copy)

// lut: the sinc table interleaved for the gather (kLutPhases x 8 float4:
// two taps of phase p and their differences to phase p + 1).
cudaError_t launch_tbc(const TbcField* dfields, int nfields, long long max_nout, const float* lut,
                       double threshold_mult, bool any_spline, cudaStream_t stream);

struct RfTbcField {
    const int16_t* in;   // raw samples of the field read (field-local sample 0)
    long long len;
    const double* ll;
    int nlines;
    int startline;       // lineoffset (NTSC) or 1 (PAL)
    int nout;            // output lines (linecount)
    int linelen;         // output samples per line
    double delay;        // video_white delay (samples)
    int16_t* out;
    int* status;         // LDG_TBC_OUT_OF_RANGE when a tap leaves the read
};

cudaError_t launch_rf_tbc(const RfTbcField* dfields, int nfields, int max_lines, cudaStream_t stream);

}  // namespace ldg
