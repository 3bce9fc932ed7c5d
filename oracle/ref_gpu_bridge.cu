// ================================================================================================
// Reference GPU checker bridge — test infrastructure only (built into oracle/_ref/, never shipped).
//
// Compiled by nvcc together with the reference's own CUDA sources (SupraLib/Beamformer/
// RxBeamformerCuda.cu, RawDelay.cu, HilbertFirEnvelope.cu, IQDemodulator.cu, LogCompressor.cu,
// ScanConverter.cu, RxBeamformerMV.cu, RxBeamformerMVpcg.cu, TemporalFilter.cu, HilbertEnvelope.cu)
// and the host sources they need, as a release build (NDEBUG), WITHOUT --use_fast_math and with
// -fmad=false:
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
#include "RxBeamformerMV.h"
#include "RxBeamformerMVpcg.h"
#include "TemporalFilter.h"
#include "HilbertEnvelope.h"
#include <cublas_v2.h>
#include <queue>

// The scan converter keeps its tables in private members; the checker reads them directly. Every
// header the class declaration needs is included above, so only ScanConverter itself is affected.
#define private public
#include "ScanConverter.h"
#undef private

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

// ---------------------------------------------------------------- scan converter
// ScanConverter::updateInternals on the scanlines [lx * ly] (x fastest) of a record of num_samples
// samples over `depth` mm, image resolution `resolution` mm; the handle keeps the converter and its
// image properties.
struct RefScan {
    ScanConverter sc;
    std::shared_ptr<USImageProperties> props;
};

void* refg_scan_create(const sb_scanline_rx* lines, uint32_t lx, uint32_t ly, uint32_t numSamples, double depth,
                       double resolution) {
    auto info = std::make_shared<std::vector<std::vector<ScanlineRxParameters3D>>>(
        lx, std::vector<ScanlineRxParameters3D>(ly));
    for (uint32_t y = 0; y < ly; y++)
        for (uint32_t x = 0; x < lx; x++)
            std::memcpy(&(*info)[x][y], &lines[x + y * lx], sizeof(sb_scanline_rx));
    RefScan* h = new RefScan();
    h->props = std::make_shared<USImageProperties>(vec2s{lx, ly}, numSamples, USImageProperties::ImageType::BMode,
                                                   USImageProperties::ImageState::EnvDetected,
                                                   USImageProperties::TransducerType::Linear, depth);
    h->props->setImageResolution(resolution);
    h->props->setScanlineInfo(info);
    h->sc.updateInternals(h->props);
    return h;
}

void refg_scan_size(void* h, uint32_t* size3) {
    vec3s s = static_cast<RefScan*>(h)->sc.getImageSize();
    size3[0] = static_cast<uint32_t>(s.x);
    size3[1] = static_cast<uint32_t>(s.y);
    size3[2] = static_cast<uint32_t>(s.z);
}

// The mask, sample-index and weight tables (host arrays of the image's voxel count).
int refg_scan_tables(void* hv, uint8_t* mask, uint32_t* sampleIdx, float* wX, float* wY, float* wZ) {
    RefScan* h = static_cast<RefScan*>(hv);
    toHost<uint8_t>(h->sc.m_mask, mask);
    toHost<uint32_t>(h->sc.m_sampleIdx, sampleIdx);
    toHost<float>(h->sc.m_weightX, wX);
    toHost<float>(h->sc.m_weightY, wY);
    if (!h->sc.m_is2D) toHost<float>(h->sc.m_weightZ, wZ);
    return 0;
}

// ScanConverter::convert of a float image [num_samples][lx * ly] to uint8 (out_uint8) or float.
int refg_scan_convert(void* hv, const float* in, void* out, int out_uint8) {
    RefScan* h = static_cast<RefScan*>(hv);
    const size_t n = static_cast<size_t>(h->props->getNumScanlines()) * h->props->getNumSamples();
    auto c = std::make_shared<Container<float>>(LocationGpu, ContainerFactory::getNextStream(), in, in + n);
    vec2s layout = h->props->getScanlineLayout();
    auto img = std::make_shared<USImage>(vec3s{layout.x * layout.y, h->props->getNumSamples(), 1}, c, h->props, 0, 0);
    if (out_uint8) toHost<uint8_t>(h->sc.convert<float, uint8_t>(img), static_cast<uint8_t*>(out));
    else toHost<float>(h->sc.convert<float, float>(img), static_cast<float*>(out));
    return 0;
}

void refg_scan_destroy(void* h) { delete static_cast<RefScan*>(h); }

// ---------------------------------------------------------------- minimum variance
// Raw-delayed data [scanline][channel][sample] as the MV nodes receive it (RawDelay output).
std::shared_ptr<USRawData> delayedOf(const float* raw, uint32_t numRx, uint32_t numCh, uint32_t numS) {
    auto c = std::make_shared<Container<float>>(LocationGpu, ContainerFactory::getNextStream(), raw,
                                                raw + static_cast<size_t>(numRx) * numCh * numS);
    auto props = std::make_shared<USImageProperties>(vec2s{numRx, 1}, numS, USImageProperties::ImageType::BMode,
                                                     USImageProperties::ImageState::RawDelayed,
                                                     USImageProperties::TransducerType::Linear, 1.0);
    return std::make_shared<USRawData>(numRx, numCh, vec2s{numCh, 1}, numCh, numS, 40e6, c, nullptr, props, 0, 0);
}

// RxBeamformerMV::performRxBeamforming (cuBLAS batched LU), float image [sample][scanline].
int refg_mv(const float* raw, float* out, uint32_t numRx, uint32_t numCh, uint32_t numS, uint32_t subArraySize,
            uint32_t temporalSmoothing, double scalingPower) {
    auto rd = delayedOf(raw, numRx, numCh, numS);
    cublasHandle_t h;
    if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) return -1;
    cublasSetStream(h, rd->getData<float>()->getStream());
    auto img = RxBeamformerMV::performRxBeamforming<float, float>(rd, subArraySize, temporalSmoothing, h, scalingPower,
                                                                  false);
    toHost<float>(img->getData<float>(), out);
    cublasDestroy(h);
    return 0;
}

// RxBeamformerMVpcg::performRxBeamforming (Jacobi PCG per system), float image [sample][scanline].
int refg_mvpcg(const float* raw, float* out, uint32_t numRx, uint32_t numCh, uint32_t numS, uint32_t subArraySize,
               uint32_t temporalSmoothing, uint32_t maxIterationsOverride, double convergenceThreshold,
               double scalingPower) {
    auto rd = delayedOf(raw, numRx, numCh, numS);
    auto img = RxBeamformerMVpcg::performRxBeamforming<float, float>(rd, subArraySize, temporalSmoothing,
                                                                     maxIterationsOverride, convergenceThreshold,
                                                                     scalingPower, false);
    toHost<float>(img->getData<float>(), out);
    return 0;
}

// ---------------------------------------------------------------- temporal filter, FFT envelope
// TemporalFilter::filter over `n` float images of numel elements (oldest first), weights per image.
int refg_temporal(const float* const* images, uint32_t n, const double* weights, uint32_t width, uint32_t height,
                  float* out) {
    const size_t numel = static_cast<size_t>(width) * height;
    std::queue<std::shared_ptr<const ContainerBase>> q;
    auto stream = ContainerFactory::getNextStream();
    for (uint32_t i = 0; i < n; i++)
        q.push(std::make_shared<Container<float>>(LocationGpu, stream, images[i], images[i] + numel));
    TemporalFilter tf;
    toHost<float>(tf.filter<float, float>(q, vec3s{width, height, 1}, std::vector<double>(weights, weights + n)), out);
    return 0;
}

// HilbertEnvelope::computeHilbertEnvelope (cuFFT C2C), float image [sample][scanline].
int refg_fft_env(const float* in, float* out, uint32_t numRx, uint32_t numSamples) {
    auto c = std::make_shared<const Container<float>>(LocationGpu, ContainerFactory::getNextStream(), in,
                                                      in + static_cast<size_t>(numRx) * numSamples);
    HilbertEnvelope h;
    toHost<float>(h.computeHilbertEnvelope<float, float>(c, static_cast<int>(numRx), static_cast<int>(numSamples), 1),
                  out);
    return 0;
}

// ---------------------------------------------------------------- device time of the reference's calls
// Each timer builds its inputs on the GPU once, makes two warm-up calls, then records CUDA events on the
// input container's stream around `iters` back-to-back calls, five times, and returns the smallest
// mean time per call in ms (the reference's calls do host work between launches, so single samples
// vary with the host). A call is what the reference's node runs per frame: its kernels plus the pooled
// allocation of its output (the pool reuses buffers, so no cudaMalloc in the timed calls).
}  // extern "C"

namespace {
template <typename F>
float timeCalls(cudaStream_t st, int iters, F&& f) {
    f();
    f();
    cudaStreamSynchronize(st);
    cudaDeviceSynchronize();
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best = 1e30f;
    for (int rep = 0; rep < 5; rep++) {
        cudaEventRecord(a, st);
        for (int i = 0; i < iters; i++) f();
        cudaEventRecord(b, st);
        cudaEventSynchronize(b);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, a, b);
        best = ms / iters < best ? ms / iters : best;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return best;
}
}  // namespace

extern "C" {

float refg_time_das(const sb_geometry* g, const int16_t* rf, double fNumber, double c, int windowType, int beamformer,
                    double depth, int iters) {
    auto params = paramsOf(g, c);
    auto raw = rawDataOf<int16_t>(g, rf, static_cast<size_t>(g->num_tx) * g->num_channels * g->num_samples, depth,
                                  params, g->num_tx, g->num_channels, g->num_samples, false);
    RxBeamformerCuda bf(*params);
    return timeCalls(raw->getData<int16_t>()->getStream(), iters, [&]() {
        bf.performRxBeamforming<int16_t, float>(static_cast<RxBeamformerCuda::RxSampleBeamformer>(beamformer), raw,
                                                fNumber, c, static_cast<WindowType>(windowType), 0.0f, false, 0);
    });
}

float refg_time_rawdelay(const sb_geometry* g, const int16_t* rf, double fNumber, double c, int windowType,
                         double depth, int iters) {
    auto params = paramsOf(g, c);
    auto raw = rawDataOf<int16_t>(g, rf, static_cast<size_t>(g->num_tx) * g->num_channels * g->num_samples, depth,
                                  params, g->num_tx, g->num_channels, g->num_samples, false);
    RawDelay rd(*params);
    return timeCalls(raw->getData<int16_t>()->getStream(), iters, [&]() {
        rd.performDelay<int16_t, float>(raw, fNumber, c, static_cast<WindowType>(windowType), 0.0f);
    });
}

float refg_time_hilbert(const float* in, uint32_t numRx, uint32_t numSamples, uint32_t filterLength, int iters) {
    auto c = std::make_shared<const Container<float>>(LocationGpu, ContainerFactory::getNextStream(), in,
                                                      in + static_cast<size_t>(numRx) * numSamples);
    HilbertFirEnvelope h(filterLength);
    return timeCalls(c->getStream(), iters,
                     [&]() { h.demodulate<float, float>(c, static_cast<int>(numRx), static_cast<int>(numSamples)); });
}

float refg_time_logcompress(const float* in, uint32_t numRx, uint32_t numSamples, double dynamicRange, double gain,
                            double inMax, int iters) {
    auto c = std::make_shared<const Container<float>>(LocationGpu, ContainerFactory::getNextStream(), in,
                                                      in + static_cast<size_t>(numRx) * numSamples);
    LogCompressor lc;
    const vec3s size{numRx, numSamples, 1};
    return timeCalls(c->getStream(), iters, [&]() { lc.compress<float, uint8_t>(c, size, dynamicRange, gain, inMax); });
}

float refg_time_iq(const float* in, uint32_t numRx, uint32_t numSamples, double fs, double referenceFrequency,
                   double cutoff, uint32_t lowpassLength, uint32_t bandpassLength, uint32_t decimation,
                   uint32_t numFilters, const double* frequencies, const double* bandwidths, const double* weights,
                   int iters) {
    auto c = std::make_shared<const Container<float>>(LocationGpu, ContainerFactory::getNextStream(), in,
                                                      in + static_cast<size_t>(numRx) * numSamples);
    IQDemodulator iq(fs, referenceFrequency, cutoff, lowpassLength, bandpassLength);
    std::vector<double> f(frequencies, frequencies + numFilters), b(bandwidths, bandwidths + numFilters),
        w(weights, weights + numFilters);
    return timeCalls(c->getStream(), iters, [&]() {
        iq.demodulateMagnitudeFrequencyCompounding<float, float>(c, static_cast<int>(numRx), static_cast<int>(numSamples),
                                                                 decimation, f, b, w);
    });
}

float refg_time_scan(void* hv, const float* in, int iters) {
    RefScan* h = static_cast<RefScan*>(hv);
    const size_t n = static_cast<size_t>(h->props->getNumScanlines()) * h->props->getNumSamples();
    auto c = std::make_shared<Container<float>>(LocationGpu, ContainerFactory::getNextStream(), in, in + n);
    vec2s layout = h->props->getScanlineLayout();
    auto img = std::make_shared<USImage>(vec3s{layout.x * layout.y, h->props->getNumSamples(), 1}, c, h->props, 0, 0);
    return timeCalls(c->getStream(), iters, [&]() { h->sc.convert<float, uint8_t>(img); });
}

float refg_time_mv(const float* raw, uint32_t numRx, uint32_t numCh, uint32_t numS, uint32_t subArraySize,
                   uint32_t temporalSmoothing, double scalingPower, int iters) {
    auto rd = delayedOf(raw, numRx, numCh, numS);
    cublasHandle_t h;
    if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) return -1.0f;
    cudaStream_t st = rd->getData<float>()->getStream();
    cublasSetStream(h, st);
    const float ms = timeCalls(st, iters, [&]() {
        RxBeamformerMV::performRxBeamforming<float, float>(rd, subArraySize, temporalSmoothing, h, scalingPower, false);
    });
    cublasDestroy(h);
    return ms;
}

float refg_time_mvpcg(const float* raw, uint32_t numRx, uint32_t numCh, uint32_t numS, uint32_t subArraySize,
                      uint32_t temporalSmoothing, double convergenceThreshold, double scalingPower, int iters) {
    auto rd = delayedOf(raw, numRx, numCh, numS);
    return timeCalls(rd->getData<float>()->getStream(), iters, [&]() {
        RxBeamformerMVpcg::performRxBeamforming<float, float>(rd, subArraySize, temporalSmoothing, 0,
                                                              convergenceThreshold, scalingPower, false);
    });
}

float refg_time_fft_env(const float* in, uint32_t numRx, uint32_t numSamples, int iters) {
    auto c = std::make_shared<const Container<float>>(LocationGpu, ContainerFactory::getNextStream(), in,
                                                      in + static_cast<size_t>(numRx) * numSamples);
    HilbertEnvelope h;
    return timeCalls(c->getStream(), iters, [&]() {
        h.computeHilbertEnvelope<float, float>(c, static_cast<int>(numRx), static_cast<int>(numSamples), 1);
    });
}

float refg_time_temporal(const float* image, uint32_t n, uint32_t width, uint32_t height, int iters) {
    const size_t numel = static_cast<size_t>(width) * height;
    std::queue<std::shared_ptr<const ContainerBase>> q;
    auto stream = ContainerFactory::getNextStream();
    for (uint32_t i = 0; i < n; i++) q.push(std::make_shared<Container<float>>(LocationGpu, stream, image, image + numel));
    TemporalFilter tf;
    std::vector<double> w(n, 1.0);
    return timeCalls(stream, iters, [&]() { tf.filter<float, float>(q, vec3s{width, height, 1}, w); });
}

}  // extern "C"
