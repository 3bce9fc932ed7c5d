// ================================================================================================
// Reference GPU checker bridge — test infrastructure only (built into oracle/_ref/, never shipped).
//
// Compiled by nvcc together with the reference's own CUDA sources (SupraLib/Beamformer/
// RxBeamformerCuda.cu, RawDelay.cu, HilbertFirEnvelope.cu, IQDemodulator.cu, LogCompressor.cu) and
// the host sources they need, WITHOUT --use_fast_math and with -fmad=false:
// every float operation of the reference's kernels is then a separately rounded IEEE operation, the
// semantics the library's kernels and the CPU oracle follow. Each entry takes host arrays, runs the
// reference's classes on the GPU exactly as its nodes call them, and copies the result back, so the
// tests compare the library's kernels with the reference's kernels on the same inputs.
// ================================================================================================
#include <functional>
#include <cstring>
#include <memory>
#include <vector>

#include "Container.h"
#include "ContainerFactory.h"
#include "USImage.h"
#include "USImageProperties.h"
#include "USRawData.h"
#include "RxBeamformerParameters.h"
#include "RxBeamformerCuda.h"
#include "RawDelay.h"
#include "HilbertFirEnvelope.h"
#include "IQDemodulator.h"
#include "LogCompressor.h"

#include "supra_b200.h"

using namespace supra;

namespace {

template <typename T>
void toHost(const std::shared_ptr<const Container<T>>& c, T* out) {
    Container<T> h(LocationHost, *c, true);
    std::memcpy(out, h.get(), h.size() * sizeof(T));
}

std::shared_ptr<RxBeamformerParameters> paramsOf(const sb_geometry* g, double speedOfSoundMMperS) {
    std::vector<ScanlineRxParameters3D> lines(g->num_rx);
    std::memcpy(lines.data(), g->scanlines, g->num_rx * sizeof(sb_scanline_rx));
    std::vector<float> depths(g->depths_mm, g->depths_mm + g->num_depths);
    std::vector<float> xs(g->element_x_mm, g->element_x_mm + g->num_elements);
    std::vector<float> ys(g->element_y_mm, g->element_y_mm + g->num_elements);
    return std::make_shared<RxBeamformerParameters>(g->num_rx, vec2s{g->rx_layout[0], g->rx_layout[1]},
                                                    speedOfSoundMMperS, depths, lines, xs, ys, g->num_depths);
}

// USRawData of one frame [tx][channel][sample] (host data copied to the GPU), raw or raw-delayed.
template <typename T>
std::shared_ptr<USRawData> rawDataOf(const sb_geometry* g, const T* data, size_t numel, double depth,
                                     std::shared_ptr<RxBeamformerParameters> params, uint32_t numTx,
                                     uint32_t numChannels, uint32_t numSamples, bool delayed) {
    auto c = std::make_shared<Container<T>>(LocationGpu, ContainerFactory::getNextStream(), data, data + numel);
    auto props = std::make_shared<USImageProperties>(vec2s{numTx, 1}, numSamples, USImageProperties::ImageType::BMode,
                                                     delayed ? USImageProperties::ImageState::RawDelayed
                                                             : USImageProperties::ImageState::Raw,
                                                     USImageProperties::TransducerType::Linear, depth);
    return std::make_shared<USRawData>(numTx, g->num_elements, vec2s{g->element_layout[0], g->element_layout[1]},
                                       numChannels, numSamples, g->sampling_frequency_hz, c, params, props, 0, 0);
}

}  // namespace

extern "C" {

// RxBeamformerCuda::performRxBeamforming (sample beamformer 0..3), int16 channel data, float image.
int refg_das(const sb_geometry* g, const int16_t* rf, float* out, double fNumber, double c, int windowType,
             float windowParameter, int interpTx, int32_t offset, int beamformer, double depth) {
    auto params = paramsOf(g, c);
    auto raw = rawDataOf<int16_t>(g, rf, static_cast<size_t>(g->num_tx) * g->num_channels * g->num_samples, depth,
                                  params, g->num_tx, g->num_channels, g->num_samples, false);
    RxBeamformerCuda bf(*params);
    auto img = bf.performRxBeamforming<int16_t, float>(static_cast<RxBeamformerCuda::RxSampleBeamformer>(beamformer), raw, fNumber, c,
                                       static_cast<WindowType>(windowType), windowParameter, interpTx != 0, offset);
    toHost<float>(img->getData<float>(), out);
    return 0;
}

// RawDelay::performDelay, int16 channel data, float [scanline][channel][depth].
int refg_rawdelay(const sb_geometry* g, const int16_t* rf, float* out, double fNumber, double c, int windowType,
                  float windowParameter, double depth) {
    auto params = paramsOf(g, c);
    auto raw = rawDataOf<int16_t>(g, rf, static_cast<size_t>(g->num_tx) * g->num_channels * g->num_samples, depth,
                                  params, g->num_tx, g->num_channels, g->num_samples, false);
    RawDelay rd(*params);
    auto d = rd.performDelay<int16_t, float>(raw, fNumber, c, static_cast<WindowType>(windowType), windowParameter);
    toHost<float>(d->getData<float>(), out);
    return 0;
}

// HilbertFirEnvelope::demodulate, float image [sample][scanline].
int refg_hilbert(const float* in, float* out, uint32_t numRx, uint32_t numSamples, uint32_t filterLength) {
    auto c = std::make_shared<const Container<float>>(LocationGpu, ContainerFactory::getNextStream(), in,
                                                      in + static_cast<size_t>(numRx) * numSamples);
    HilbertFirEnvelope h(filterLength);
    toHost<float>(h.demodulate<float, float>(c, static_cast<int>(numRx), static_cast<int>(numSamples)), out);
    return 0;
}

// LogCompressor::compress, float image -> float (out_uint8 = 0) or uint8.
int refg_logcompress(const float* in, void* out, uint32_t numRx, uint32_t numSamples, double dynamicRange,
                     double gain, double inMax, int out_uint8) {
    auto c = std::make_shared<const Container<float>>(LocationGpu, ContainerFactory::getNextStream(), in,
                                                      in + static_cast<size_t>(numRx) * numSamples);
    LogCompressor lc;
    const vec3s size{numRx, numSamples, 1};
    if (out_uint8) toHost<uint8_t>(lc.compress<float, uint8_t>(c, size, dynamicRange, gain, inMax), static_cast<uint8_t*>(out));
    else toHost<float>(lc.compress<float, float>(c, size, dynamicRange, gain, inMax), static_cast<float*>(out));
    return 0;
}

// IQDemodulator::demodulateMagnitudeFrequencyCompounding, float image -> float [samples/dec][scanline].
int refg_iq(const float* in, float* out, uint32_t numRx, uint32_t numSamples, double fs, double referenceFrequency,
            double cutoff, uint32_t lowpassLength, uint32_t bandpassLength, uint32_t decimation, uint32_t numFilters,
            const double* frequencies, const double* bandwidths, const double* weights) {
    auto c = std::make_shared<const Container<float>>(LocationGpu, ContainerFactory::getNextStream(), in,
                                                      in + static_cast<size_t>(numRx) * numSamples);
    IQDemodulator iq(fs, referenceFrequency, cutoff, lowpassLength, bandpassLength);
    std::vector<double> f(frequencies, frequencies + numFilters), b(bandwidths, bandwidths + numFilters),
        w(weights, weights + numFilters);
    toHost<float>(iq.demodulateMagnitudeFrequencyCompounding<float, float>(c, static_cast<int>(numRx),
                                                                           static_cast<int>(numSamples), decimation, f, b, w),
                  out);
    return 0;
}

}  // extern "C"
