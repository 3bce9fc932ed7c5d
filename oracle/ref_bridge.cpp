// ================================================================================================
// Reference checker bridge — test infrastructure only (built into oracle/_ref/, never shipped).
//
// Compiled together with the reference's own sources (SupraLib/Beamformer/WindowFunction.cpp,
// SupraLib/ContainerFactory.cpp, SupraLib/utilities/Logging.cpp, and the header-only
// FirFilterFactory.h / RxSampleBeamformerDelayAndSum.h / RxBeamformerCommon.h) in the reference's
// CPU configuration (no HAVE_CUDA). It exposes a C interface so that tests can compare the oracle's
// restatement with what the reference's code computes:
//   - FirFilterFactory::createFilter coefficients,
//   - WindowFunction LUTs and WindowFunctionGpu::get,
//   - the per-sample reducers sampleBeamform2D / sampleBeamform3D of the four sample beamformers
//     (DelayAndSum, DelayAndStdDev, CoherenceFactorDelayAndSum, TestSignal), called exactly as the
//     kernels rxBeamformingDTSPACEKernel / rxBeamformingDTSPACE3DKernel call them
//     (RxBeamformerCuda.cu:238-323 and :119-228, one (line, depth) at a time),
//   - the mock metadata reader RxBeamformerParameters::readMetaDataForMock and the JSON writer
//     writeMetaDataForMock (Beamformer/RxBeamformerParameters.cpp:93-450, with the vendored jsoncpp).
// ================================================================================================
#include <math.h>    // brings the float overloads of abs() into the global namespace
#include <stdlib.h>
#include <cmath>
#include <cstdint>
#include <vector>

namespace supra {
// The reference defines squ only for CUDA compilation (SupraLib/utilities/cudaUtility.h:100-105);
// same definition for the host.
template <typename T> constexpr inline T squ(const T& x) { return x * x; }
}  // namespace supra

#include "Container.h"
#include "utilities/FirFilterFactory.h"
#include "WindowFunction.h"
#include "USImageProperties.h"
#include "USTransducer.h"
#include "RxBeamformerCommon.h"
#include "RxSampleBeamformerDelayAndSum.h"
#include "RxSampleBeamformerDelayAndStdDev.h"
#include "RxSampleBeamformerCoherenceFactorDelayAndSum.h"
#include "RxSampleBeamformerTestSignal.h"
#include "RxBeamformerParameters.h"
#include "USRawData.h"

#include <cstring>
#include <fstream>
#include <iomanip>

#include "supra_b200.h"

using namespace supra;

extern "C" {

int ref_fir(uint32_t length, int type, int window, double fs, double f, double bw, float* out) {
    auto filt = FirFilterFactory::createFilter<float>(length, static_cast<FirFilterFactory::FilterType>(type),
                                                      static_cast<FirFilterFactory::FilterWindow>(window), fs, f, bw);
    for (uint32_t i = 0; i < length; i++) out[i] = filt->get()[i];
    return 0;
}

int ref_window_lut(int type, float param, uint32_t n, float* out) {
    WindowFunction w(static_cast<WindowType>(type), param, n);
    for (uint32_t i = 0; i < n; i++) out[i] = w.getDirect(i);
    return 0;
}

float ref_window_get(int type, float param, uint32_t n, float rel) {
    WindowFunction w(static_cast<WindowType>(type), param, n);
    return w.getGpu()->get(rel);
}

}  // extern "C"

// One frame through the reference's per-sample reducers of SampleBeamformer. The geometry conversion
// is the first call of RxBeamformerCuda::convertToDtSpace (RxBeamformerCuda.cu:58-107).
template <class SampleBeamformer>
int refDas(const sb_geometry* g, const float* rf, float* out, double fNumber, double speedOfSoundMMperS,
           int windowType, float windowParameter, int interpolateTransmits, int32_t additionalOffset) {
    typedef float LocationType;
    double dt = 1.0 / g->sampling_frequency_hz;
    double factor = 1 / 1.0 / (speedOfSoundMMperS * dt);
    double factorTime = 1 / 1.0 / dt;
    std::vector<ScanlineRxParameters3D> lines(g->num_rx);
    for (uint32_t i = 0; i < g->num_rx; i++) {
        static_assert(sizeof(ScanlineRxParameters3D) == sizeof(sb_scanline_rx), "layout");
        std::memcpy(&lines[i], &g->scanlines[i], sizeof(sb_scanline_rx));
        ScanlineRxParameters3D p = lines[i];
        p.position = p.position * factor;
        for (size_t k = 0; k < 4; k++) p.txParameters[k].initialDelay *= factorTime;
        p.maxElementDistance = p.maxElementDistance * factor;
        lines[i] = p;
    }
    std::vector<LocationType> xs(g->num_elements), ys(g->num_elements), ds(g->num_depths);
    for (uint32_t i = 0; i < g->num_depths; i++) ds[i] = static_cast<LocationType>(g->depths_mm[i] * factor);
    for (uint32_t i = 0; i < g->num_elements; i++) {
        xs[i] = static_cast<LocationType>(g->element_x_mm[i] * factor);
        ys[i] = static_cast<LocationType>(g->element_y_mm[i] * factor);
    }
    WindowFunction win(static_cast<WindowType>(windowType), windowParameter, 64);
    const WindowFunctionGpu* wg = win.getGpu();
    std::vector<float> functionShared(64);
    for (int i = 0; i < 64; i++) functionShared[i] = win.getDirect(i);
    LocationType speedOfSound = static_cast<LocationType>(speedOfSoundMMperS);
    LocationType dtf = static_cast<LocationType>(dt);
    LocationType F = static_cast<LocationType>(fNumber);
    bool is3D = g->rx_layout[0] > 1 && g->rx_layout[1] > 1;
    vec2T<uint32_t> elementLayout{g->element_layout[0], g->element_layout[1]};
    // scanlines are independent (as the kernel's threads are): spread over the host cores
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t sl = 0; sl < static_cast<int64_t>(g->num_rx); sl++) {
        const uint32_t scanlineIdx = static_cast<uint32_t>(sl);
        for (uint32_t r = 0; r < g->num_depths; r++) {
            LocationType d = ds[r];
            ScanlineRxParameters3D scanline = lines[scanlineIdx];
            LocationType scanline_x = scanline.position.x;
            LocationType scanline_z = scanline.position.z;
            LocationType dirX = scanline.direction.x;
            LocationType dirY = scanline.direction.y;
            LocationType dirZ = scanline.direction.z;
            LocationType aDT;
            LocationType invMax2D = 0;
            vec2f invMax3D{0, 0};
            if (is3D) {
                aDT = squ(computeAperture_D(F, d * dtf * speedOfSound) / speedOfSound / dtf);
                vec2f maxElementDistance = static_cast<vec2f>(scanline.maxElementDistance);
                invMax3D = vec2f{1.0f, 1.0f} / min(vec2f{sqrtf(aDT), sqrtf(aDT)}, maxElementDistance);
            } else {
                aDT = computeAperture_D(F, d * dtf * speedOfSound) / speedOfSound / dtf;
                LocationType maxElementDistance = static_cast<LocationType>(scanline.maxElementDistance.x);
                invMax2D = 1 / min(aDT, maxElementDistance);
            }
            float sInterp = 0.0f;
            int highestWeightIndex = 0;
            if (!interpolateTransmits) {
                float highestWeight = scanline.txWeights[0];
                for (int k = 1; k < 4; k++) {
                    if (scanline.txWeights[k] > highestWeight) {
                        highestWeight = scanline.txWeights[k];
                        highestWeightIndex = k;
                    }
                }
            }
            bool invalid = false;
            for (int k = (interpolateTransmits ? 0 : highestWeightIndex);
                 (interpolateTransmits && k < 4) || (!interpolateTransmits && k == highestWeightIndex); k++) {
                if (scanline.txWeights[k] > 0.0) {
                    ScanlineRxParameters3D::TransmitParameters txParams = scanline.txParameters[k];
                    if (txParams.txScanlineIdx >= g->num_tx) { invalid = true; break; }
                    float sLocal;
                    if (is3D) {
                        sLocal = SampleBeamformer::template sampleBeamform3D<true, false, float, float, LocationType>(
                            txParams, rf, elementLayout, g->num_channels, g->num_samples, xs.data(), ys.data(),
                            scanline_x, scanline_z, dirX, dirY, dirZ, aDT, d, invMax3D, speedOfSound, dtf,
                            additionalOffset, wg, functionShared.data(), nullptr);
                    } else {
                        sLocal = SampleBeamformer::template sampleBeamform2D<true, false, float, float, LocationType>(
                            txParams, rf, g->num_elements, g->num_channels, g->num_samples, xs.data(), scanline_x,
                            dirX, dirY, dirZ, aDT, d, invMax2D, speedOfSound, dtf, additionalOffset, wg, nullptr);
                    }
                    if (interpolateTransmits) sInterp += static_cast<float>(scanline.txWeights[k]) * sLocal;
                    else sInterp += sLocal;
                }
            }
            if (!invalid) out[scanlineIdx + static_cast<size_t>(r) * g->num_rx] = clampCast<float>(sInterp);
        }
    }
    return 0;
}

extern "C" {

int ref_das(const sb_geometry* g, const float* rf, float* out, double fNumber, double speedOfSoundMMperS,
            int windowType, float windowParameter, int interpolateTransmits, int32_t additionalOffset) {
    return refDas<RxSampleBeamformerDelayAndSum>(g, rf, out, fNumber, speedOfSoundMMperS, windowType, windowParameter,
                                                 interpolateTransmits, additionalOffset);
}

// The reference's JSON mock metadata for a geometry (writeMetaDataForMock).
int ref_mock_write_json(const char* filename, const sb_geometry* g, double depth, double speedOfSoundMMperS) {
    std::vector<ScanlineRxParameters3D> lines(g->num_rx);
    std::memcpy(lines.data(), g->scanlines, g->num_rx * sizeof(sb_scanline_rx));
    std::vector<float> depths(g->depths_mm, g->depths_mm + g->num_depths);
    std::vector<float> xs(g->element_x_mm, g->element_x_mm + g->num_elements);
    std::vector<float> ys(g->element_y_mm, g->element_y_mm + g->num_elements);
    auto params = std::make_shared<RxBeamformerParameters>(g->num_rx, vec2s{g->rx_layout[0], g->rx_layout[1]},
                                                           speedOfSoundMMperS, depths, lines, xs, ys, g->num_depths);
    auto props = std::make_shared<USImageProperties>(vec2s{g->num_tx, 1}, g->num_depths, USImageProperties::ImageType::BMode,
                                                     USImageProperties::ImageState::Raw,
                                                     USImageProperties::TransducerType::Linear, depth);
    auto raw = std::make_shared<USRawData>(g->num_tx, g->num_elements, vec2s{g->element_layout[0], g->element_layout[1]},
                                           g->num_channels, g->num_samples, g->sampling_frequency_hz, nullptr, params,
                                           props, 0, 0);
    params->writeMetaDataForMock(filename, raw);
    return 0;
}

// An ASCII mock file in the layout readMetaDataForMockAscii reads, scanlines written with the
// reference's operator<< (SupraLib/USImageProperties.cpp:38-59).
int ref_mock_write_ascii(const char* filename, const sb_geometry* g, double depth, double speedOfSoundMMperS) {
    std::ofstream f(filename);
    f << "rawDataMockMetadata v 1\n";
    f << g->num_elements << " " << g->element_layout[0] << " " << g->element_layout[1] << " " << g->num_channels << " "
      << g->num_samples << " " << g->num_tx << " " << g->rx_layout[0] << " " << g->rx_layout[1] << " "
      << std::setprecision(17) << depth << " " << g->sampling_frequency_hz << " " << g->num_depths << " "
      << speedOfSoundMMperS << "\n";
    for (uint32_t i = 0; i < g->num_rx; i++) {
        ScanlineRxParameters3D p;
        std::memcpy(&p, &g->scanlines[i], sizeof(p));
        f << p << "\n";
    }
    f << std::setprecision(9);
    for (uint32_t i = 0; i < g->num_depths; i++) f << g->depths_mm[i] << " ";
    f << "\n";
    for (uint32_t i = 0; i < g->num_elements; i++) f << g->element_x_mm[i] << " ";
    f << "\n";
    for (uint32_t i = 0; i < g->num_elements; i++) f << g->element_y_mm[i] << " ";
    f << "\n";
    return f.good() ? 0 : -1;
}

// readMetaDataForMock of the reference: sizes[9] = numElements, elementLayout x/y, numReceivedChannels,
// numSamples, numTxScanlines, scanlineLayout x/y, rxNumDepths; vals[3] = depth, samplingFrequency,
// speedOfSoundMMperS; arrays filled up to their capacities. Returns -1 on a reader exception.
int ref_mock_read(const char* filename, uint64_t* sizes, double* vals, sb_scanline_rx* lines, float* depths, float* xs,
                  float* ys, uint64_t capLines, uint64_t capDepths, uint64_t capElems) {
    std::shared_ptr<USRawData> raw;
    try {
        raw = RxBeamformerParameters::readMetaDataForMock(filename);
    } catch (...) {
        return -1;
    }
    auto p = raw->getRxBeamformerParameters();
    sizes[0] = raw->getNumElements();
    sizes[1] = raw->getElementLayout().x;
    sizes[2] = raw->getElementLayout().y;
    sizes[3] = raw->getNumReceivedChannels();
    sizes[4] = raw->getNumSamples();
    sizes[5] = raw->getNumScanlines();
    sizes[6] = p->getRxScanlineLayout().x;
    sizes[7] = p->getRxScanlineLayout().y;
    sizes[8] = p->getRxNumDepths();
    vals[0] = raw->getImageProperties()->getDepth();
    vals[1] = raw->getSamplingFrequency();
    vals[2] = p->getSpeedOfSoundMMperS();
    const auto& L = p->getRxScanlines();
    for (size_t i = 0; i < L.size() && i < capLines; i++) std::memcpy(&lines[i], &L[i], sizeof(sb_scanline_rx));
    const auto& D = p->getRxDepths();
    for (size_t i = 0; i < D.size() && i < capDepths; i++) depths[i] = D[i];
    const auto& X = p->getRxElementXs();
    const auto& Y = p->getRxElementYs();
    for (size_t i = 0; i < X.size() && i < capElems; i++) {
        xs[i] = X[i];
        ys[i] = Y[i];
    }
    return 0;
}

// beamformer: the order of RxBeamformerCuda::RxSampleBeamformer (RxBeamformerCuda.h:31-36).
int ref_das_bf(const sb_geometry* g, const float* rf, float* out, double fNumber, double speedOfSoundMMperS,
               int windowType, float windowParameter, int interpolateTransmits, int32_t additionalOffset, int beamformer) {
    switch (beamformer) {
    case 0:
        return refDas<RxSampleBeamformerDelayAndSum>(g, rf, out, fNumber, speedOfSoundMMperS, windowType,
                                                     windowParameter, interpolateTransmits, additionalOffset);
    case 1:
        return refDas<RxSampleBeamformerDelayAndStdDev>(g, rf, out, fNumber, speedOfSoundMMperS, windowType,
                                                        windowParameter, interpolateTransmits, additionalOffset);
    case 2:
        return refDas<RxSampleBeamformerCoherenceFactorDelayAndSum>(g, rf, out, fNumber, speedOfSoundMMperS, windowType,
                                                                    windowParameter, interpolateTransmits, additionalOffset);
    case 3:
        return refDas<RxSampleBeamformerTestSignal>(g, rf, out, fNumber, speedOfSoundMMperS, windowType, windowParameter,
                                                    interpolateTransmits, additionalOffset);
    default:
        return -1;
    }
}

}  // extern "C"
