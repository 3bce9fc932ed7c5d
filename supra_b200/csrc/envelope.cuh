// Parameter blocks and device helpers shared by the envelope / IQ / fused scan kernels.
#pragma once

#include "common.cuh"

namespace sb {

constexpr int kIqMaxTaps = 128;

// Frequency-compounding IQ demodulator (Beamformer/IQDemodulator.cu:215-345), filters by value.
struct IqArgs {
    int nS, nL, nOut, stride;
    int numFilters, bpN, lpN;
    float scale;                       // 1 / sum(weights)
    float weights[8];
    float fOverFs[8];                  // reference frequency / sampling frequency
    float bank[8 * (kIqMaxTaps + 1)];  // band-pass k at [k * (bpN + 1)], one zero tap appended
    float lp[kIqMaxTaps + 1];          // decimation low-pass, one zero tap appended
};

struct IqComplexArgs {
    int nS, nL, nOut, dec, taps, half;
    double fOverFs;
    float lp[kIqMaxTaps + 1];
};

// thrustLogcompress::operator() (Beamformer/LogCompressor.cu:36-40):
// log10(|x| * inScale + 1) * k, k = gain * outMax / log10(10^(DR/20) + 1).
__device__ __forceinline__ float logCompress(float x, float inScale, float k) {
    return __fmul_rn(log10f(__fadd_rn(__fmul_rn(fabsf(x), inScale), 1.0f)), k);
}

int launchLog(const void* in, int inDt, void* out, int outDt, size_t n, float inScale, float k, cudaStream_t st);
void logConstants(double dynamicRange, double gain, double inMax, int inDt, float& inScale, float& k);

}  // namespace sb

struct sb_hilbert_plan {
    uint32_t N;
    float* dTaps;  // N Hilbert taps (Hamming window)
    // The nonzero taps sit at j0, j0 + 2, ..., j0 + 2 (nz - 1) (odd offsets from the centre); dNz holds
    // them padded with zeros to a multiple of four. nz = 0: no such pattern (generic kernel only).
    int j0, nz;
    float* dNz;
};

namespace sb {
// Envelope of a float / int16 image [nS][nL] into a float image; with `logc` its log compression
// (inScale, k) instead, for the env -> log -> scan chain.
int launchHilbert(const sb_hilbert_plan* p, const void* in, int inDt, float* out, int nS, int nL, bool logc,
                  float inScale, float k, cudaStream_t st);
}  // namespace sb
