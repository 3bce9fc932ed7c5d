// Delay-and-sum plan and the device-side geometry shared by the DAS, raw-delay, batched and
// adjoint kernels.
#pragma once

#include <vector>

#include "common.cuh"

namespace sb {

// One receive scanline in "DT space" (positions in units of c*dt, delays in samples), the form
// RxBeamformerCuda::convertToDtSpace produces (Beamformer/RxBeamformerCuda.cu:58-107).
struct LineDT {
    float x, z;              // scanline origin (lateral, elevation)
    float dirX, dirY, dirZ;  // direction (lateral, depth, elevation)
    float maxDistX, maxDistY;
    float txWeight[4];       // (float) txWeights
    float initialDelay[4];   // samples
    uint16_t firstX[4], firstY[4], lastX[4], lastY[4], txIdx[4];
    int32_t highest;         // index of the highest-weight transmit
    int32_t activeMask;      // bit k set when txWeights[k] > 0
};

struct WindowLut {
    float v[64];
};

}  // namespace sb

struct sb_das_plan {
    uint32_t numElements, layoutX, layoutY, numChannels, numSamples, numTx, numRx, rxLayoutX, rxLayoutY, numDepths;
    double fs;
    bool is3D;
    bool hasChannelMap;
    // geometry as given (mm), on the device
    float* dXeMM = nullptr;
    float* dYeMM = nullptr;
    float* dDepthMM = nullptr;
    sb_scanline_rx* dLinesMM = nullptr;
    int32_t* dE2C = nullptr;
    // DT-space copies for the current speed of sound
    float* dXe = nullptr;
    float* dYe = nullptr;
    float* dDepth = nullptr;
    sb::LineDT* dLines = nullptr;
    double cachedC = -1.0;
    // host copies used for launch planning
    std::vector<sb_scanline_rx>* hLines = nullptr;
    std::vector<float>* hXeMM = nullptr;
    std::vector<float>* hDepthMM = nullptr;
    int32_t maxApertureX = 0, maxApertureY = 0;  // largest (last - first) over lines and transmits
    // device scratch of the adjoint (per-pixel factors, recomputed forward), grown on demand and kept
    // with the plan so that repeated calls allocate nothing
    void* adjScratch = nullptr;
    size_t adjScratchBytes = 0;
    // work items (scanline, depth segment) of the single-frame pack path of sb_das_run and its work
    // counter, built on the first call
    void* packItems = nullptr;
    uint32_t packItemCount = 0;
    uint32_t* packCounter = nullptr;
};

namespace sb {
// Makes the DT-space buffers of `plan` current for speed of sound c (mm/s), stream-ordered.
int ensureDtSpace(sb_das_plan* plan, double c_mm_s, cudaStream_t stream);
WindowLut makeLut(int windowType, float windowParameter);
}  // namespace sb
