// ================================================================================================
// supra_b200 ORACLE — test infrastructure only.
//
// A CPU restatement of SUPRA's receive-processing kernels, written to follow the reference's
// arithmetic step by step (same float/double types per operation, same loop order, same
// reductions) so that the CUDA path can be checked against it. It is loaded only by tests/,
// __graft_entry__.smoke() and bench.py's CPU baseline / reference arm; the product never links it.
//
// Citations are paths inside the reference project (src/SupraLib = "SL/", src/SupraLib/Beamformer
// = "BF/"). Compiled with -O2 -ffp-contract=off and without -ffast-math so that every float
// operation is a separately rounded IEEE operation. The reference is built with --use_fast_math
// (SL/CMakeLists.txt:65); the tolerances in tests/ absorb that difference.
//
// Pinning: FIR coefficients, window LUTs, the per-sample DAS functions and the 2D scan-conversion
// helpers are checked bit-for-bit against the reference's own sources compiled in oracle/_ref
// (see oracle/ref_bridge.cpp, oracle/Makefile); tests/test_oracle_pin.py holds those checks.
// ================================================================================================
#include "supra_b200.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ------------------------------------------------------------------------------------------ utils
template <typename T> inline T squ(const T& x) { return x * x; }

// clampCast: clamp to the target's [min,max] then static_cast (truncation). SL/utilities/cudaUtility.h:111-147.
// The reference evaluates it in device code, where max/min of floats are fmaxf/fminf: a NaN input
// becomes the lower bound (e.g. the 0/0 of a zero-weight aperture at depth 0 is written as -FLT_MAX).
inline float clampToFloat(float x) { return std::fmin(std::fmax(x, -FLT_MAX), FLT_MAX); }
inline int16_t clampToInt16(float x) { return static_cast<int16_t>(std::fmin(std::fmax(x, -32767.0f), 32767.0f)); }
inline uint8_t clampToUint8(float x) { return static_cast<uint8_t>(std::fmin(std::fmax(x, 0.0f), 255.0f)); }
inline uint16_t clampToUint16(float x) { return static_cast<uint16_t>(std::fmin(std::fmax(x, 0.0f), 65535.0f)); }

inline void storeClamped(void* out, int dtype, size_t idx, float v) {
    switch (dtype) {
    case SB_FLOAT32: static_cast<float*>(out)[idx] = clampToFloat(v); break;
    case SB_INT16: static_cast<int16_t*>(out)[idx] = clampToInt16(v); break;
    case SB_UINT8: static_cast<uint8_t*>(out)[idx] = clampToUint8(v); break;
    case SB_UINT16: static_cast<uint16_t*>(out)[idx] = clampToUint16(v); break;
    default: break;
    }
}

inline float loadAsFloat(const void* p, int dtype, size_t idx) {
    switch (dtype) {
    case SB_INT16: return static_cast<float>(static_cast<const int16_t*>(p)[idx]);
    case SB_UINT8: return static_cast<float>(static_cast<const uint8_t*>(p)[idx]);
    default: return static_cast<const float*>(p)[idx];
    }
}

// ------------------------------------------------------------------------------------ window LUT
// WindowFunction::windowFunction<float>, BF/WindowFunction.h:121-138 (T = float).
float windowValue(int type, float relativeIndex, float windowParameter) {
    switch (type) {
    case SB_WINDOW_RECTANGULAR: return 1.0f;
    case SB_WINDOW_HANN:
        return (1 - windowParameter) *
                   (0.5f - 0.5f * std::cos(2 * static_cast<float>(M_PI) * ((relativeIndex + 1) * 0.5f))) +
               windowParameter;
    case SB_WINDOW_HAMMING:
        return (1 - windowParameter) *
                   (0.54f - 0.46f * std::cos(2 * static_cast<float>(M_PI) * ((relativeIndex + 1) * 0.5f))) +
               windowParameter;
    case SB_WINDOW_GAUSS:
        return static_cast<float>(1.0 / (windowParameter * std::sqrt(2.0 * M_PI)) *
                                  std::exp((-1.0 / 2.0) * (relativeIndex / windowParameter) *
                                           (relativeIndex / windowParameter)));
    default: return 0;
    }
}

// WindowFunction::WindowFunction, BF/WindowFunction.cpp:18-49: sample, then normalise to the max.
std::vector<float> windowLut(int type, float param, size_t n) {
    std::vector<float> data(n);
    float maxValue = std::numeric_limits<float>::min();
    for (size_t i = 0; i < n; i++) {
        float rel = (static_cast<float>(i) / (n - 1)) * 2 - 1;
        float v = windowValue(type, rel, param);
        data[i] = v;
        maxValue = std::max(maxValue, v);
    }
    for (size_t i = 0; i < n; i++) data[i] /= maxValue;
    return data;
}

// WindowFunctionGpu::get, BF/WindowFunction.h:58-64 (nearest LUT entry).
struct Window {
    std::vector<float> lut;
    float scale;
    Window(int type, float param, size_t n = 64) : lut(windowLut(type, param, n)), scale(static_cast<float>(n - 1) * 0.5f) {}
    float get(float relativeIndex) const {
        // the reference runs this on the GPU, where min/max of floats are fminf/fmaxf (a NaN
        // argument yields the other operand)
        float c = std::fmin(std::fmax(relativeIndex, -1.0f), 1.0f);
        uint32_t idx = static_cast<uint32_t>(std::round(scale * (c + 1.0f)));
        return lut[idx];
    }
};

// ------------------------------------------------------------------------------------- FIR design
// FirFilterFactory, SL/utilities/FirFilterFactory.h:58-230, ElementType = float.
float bessel0(float x) {  // :216-228, T = float
    float sum = 0.0f;
    static const int factorial[9] = {1, 2, 6, 24, 120, 720, 5040, 40320, 362880};
    for (int k = 1; k < 10; k++) {
        float xPower = std::pow(x / 2.0f, static_cast<float>(k));
        sum += std::pow(xPower / static_cast<float>(factorial[k - 1]), 2.0f);
    }
    return 1.0f + sum;
}
double bessel0d(double x) {  // same, T = double
    double sum = 0.0;
    static const int factorial[9] = {1, 2, 6, 24, 120, 720, 5040, 40320, 362880};
    for (int k = 1; k < 10; k++) {
        double xPower = std::pow(x / 2.0, static_cast<double>(k));
        sum += std::pow(xPower / static_cast<double>(factorial[k - 1]), 2.0);
    }
    return 1.0 + sum;
}

std::vector<float> firDesign(size_t length, int type, int window, double fs, double frequency, double bandwidth) {
    // createFilterNoWindow :76-158
    float omega = static_cast<float>(2 * M_PI * frequency / fs);
    float omegaBandwidth = static_cast<float>(2 * M_PI * bandwidth / fs);
    int halfWidth = (static_cast<int>(length) - 1) / 2;
    std::vector<float> f(length);
    for (size_t kk = 0; kk < length; kk++) {
        int n = static_cast<int>(kk);
        float v;
        switch (type) {
        case 3: {  // Hilbert :98-110
            int k = n - halfWidth;
            v = (k % 2 == 0) ? 0.0f : static_cast<float>(2.0 / (M_PI * k));
            break;
        }
        case 1:  // high-pass :112-121
            if (n == halfWidth) v = static_cast<float>(1 - omega / M_PI);
            else v = static_cast<float>(-omega / M_PI * std::sin(omega * (n - halfWidth)) / (omega * (n - halfWidth)));
            break;
        case 2:  // band-pass :123-134 (cos(omega*n - halfWidth) as written, quirk Q6)
            if (n == halfWidth) v = static_cast<float>(2.0 * omegaBandwidth / M_PI);
            else
                v = static_cast<float>(2.0 * std::cos(omega * n - halfWidth) * omegaBandwidth / M_PI *
                                       std::sin(omegaBandwidth * (n - halfWidth)) /
                                       (omegaBandwidth * (n - halfWidth)));
            break;
        case 0:
        default:  // low-pass :136-146
            if (n == halfWidth) v = static_cast<float>(omega / M_PI);
            else v = static_cast<float>(omega / M_PI * std::sin(omega * (n - halfWidth)) / (omega * (n - halfWidth)));
            break;
        }
        f[kk] = v;
    }
    // applyWindowToFilter :161-197
    size_t maxN = length - 1;
    float beta = 4.0f;
    for (size_t kk = 0; kk < length; kk++) {
        int n = static_cast<int>(kk);
        float w;
        switch (window) {
        case 1: w = static_cast<float>(0.50 - 0.50 * std::cos(2 * M_PI * n / maxN)); break;
        case 2: w = static_cast<float>(0.54 - 0.46 * std::cos(2 * M_PI * n / maxN)); break;
        case 3: {
            double argument = beta * std::sqrt(1.0 - std::pow(2 * (static_cast<float>(n) - maxN / 2) / maxN, 2.0));
            w = static_cast<float>(bessel0d(argument) / bessel0(beta));
            break;
        }
        default: w = 1.0f; break;
        }
        f[kk] *= w;
    }
    // normalizeGain :199-214 (band-pass only)
    if (type == 2) {
        float gainR = 0, gainI = 0;
        for (int k = 0; k < static_cast<int>(length); k++) {
            gainR += f[k] * std::cos(omega * static_cast<float>(k));
            gainI += f[k] * std::sin(omega * static_cast<float>(k));
        }
        float gain = std::sqrt(gainR * gainR + gainI * gainI);
        for (size_t k = 0; k < length; k++) f[k] /= gain;
    }
    return f;
}

// ---------------------------------------------------------------------------- geometry in DT space
// RxBeamformerCuda::convertToDtSpace, BF/RxBeamformerCuda.cu:58-107, first call (m_lastSeenDt == 0):
// positions, depths and element positions scaled by 1/(c dt) in double, initial delays by 1/dt.
struct LineDT {
    float x, z, dirX, dirY, dirZ;
    float maxDistX, maxDistY;
    double txWeights[4];
    uint16_t firstX[4], firstY[4], lastX[4], lastY[4], txIdx[4];
    float initialDelay[4];
};

struct GeomDT {
    std::vector<float> xe, ye, depths;
    std::vector<LineDT> lines;
    float c, dt;
};

GeomDT toDtSpace(const sb_geometry* g, double speedOfSoundMMperS) {
    GeomDT r;
    double dt = 1.0 / g->sampling_frequency_hz;
    double oldFactor = 1, oldFactorTime = 1;
    double factor = 1 / oldFactor / (speedOfSoundMMperS * dt);
    double factorTime = 1 / oldFactorTime / dt;
    r.xe.resize(g->num_elements);
    r.ye.resize(g->num_elements);
    for (uint32_t i = 0; i < g->num_elements; i++) {
        r.xe[i] = static_cast<float>(g->element_x_mm[i] * factor);
        r.ye[i] = static_cast<float>(g->element_y_mm[i] * factor);
    }
    r.depths.resize(g->num_depths);
    for (uint32_t i = 0; i < g->num_depths; i++) r.depths[i] = static_cast<float>(g->depths_mm[i] * factor);
    r.lines.resize(g->num_rx);
    for (uint32_t l = 0; l < g->num_rx; l++) {
        const sb_scanline_rx& s = g->scanlines[l];
        LineDT& o = r.lines[l];
        // kernel-side casts (RxBeamformerCuda.cu:167-175, 264-270): double -> float
        o.x = static_cast<float>(s.position[0] * factor);
        o.z = static_cast<float>(s.position[2] * factor);
        o.dirX = static_cast<float>(s.direction[0]);
        o.dirY = static_cast<float>(s.direction[1]);
        o.dirZ = static_cast<float>(s.direction[2]);
        o.maxDistX = static_cast<float>(s.max_element_distance[0] * factor);
        o.maxDistY = static_cast<float>(s.max_element_distance[1] * factor);
        for (int k = 0; k < 4; k++) {
            o.txWeights[k] = s.tx_weights[k];
            o.firstX[k] = s.tx[k].first_active_element[0];
            o.firstY[k] = s.tx[k].first_active_element[1];
            o.lastX[k] = s.tx[k].last_active_element[0];
            o.lastY[k] = s.tx[k].last_active_element[1];
            o.txIdx[k] = s.tx[k].tx_scanline_idx;
            o.initialDelay[k] = static_cast<float>(s.tx[k].initial_delay_s * factorTime);
        }
    }
    r.c = static_cast<float>(speedOfSoundMMperS);
    r.dt = static_cast<float>(dt);
    return r;
}

// Highest-weight transmit (RxBeamformerCuda.cu:274-287): the comparison promotes the float
// running maximum to double.
int highestWeightIndex(const LineDT& s) {
    int idx = 0;
    float hw = static_cast<float>(s.txWeights[0]);
    for (int k = 1; k < 4; k++) {
        if (s.txWeights[k] > hw) {
            hw = static_cast<float>(s.txWeights[k]);
            idx = k;
        }
    }
    return idx;
}

inline int32_t channelOf(const sb_geometry* g, uint32_t elem) {
    if (g->element_to_channel) return g->element_to_channel[elem];
    return static_cast<int32_t>(elem % g->num_channels);
}

// ------------------------------------------------------------------------------------------- DAS
// Acc = float: reference semantics. Acc = double: the same discrete decisions (aperture, LUT index,
// sample index) with delay fraction, interpolation and sums in double, for error statements.
template <typename Acc>
Acc sampleBeamform2D(const sb_geometry* g, const GeomDT& G, const Window& win, const float* rf, const LineDT& s,
                     int k, float aDT, float depth, float invMaxElementDistance, int32_t additionalOffset,
                     const float* apod) {
    // RxSampleBeamformerDelayAndSum::sampleBeamform2D, BF/RxSampleBeamformerDelayAndSum.h:123-208
    Acc sample = 0;
    Acc weightAcum = 0;
    int numAdds = 0;
    float initialDelay = s.initialDelay[k];
    uint32_t txScanlineIdx = s.txIdx[k];
    uint32_t numTimesteps = g->num_samples;
    uint32_t numReceivedChannels = g->num_channels;
    for (int32_t e = s.firstX[k]; e < s.lastX[k]; e++) {
        int32_t ch = channelOf(g, static_cast<uint32_t>(e));
        if (ch < 0) continue;  // ElementChannelMapNotConnected
        uint32_t channelIdx = static_cast<uint32_t>(ch);
        float x_elem = G.xe[e];
        if (std::fabs(x_elem - s.x) <= aDT) {
            float w = win.get((x_elem - s.x) * invMaxElementDistance);
            Acc weight = apod ? static_cast<Acc>(w) * static_cast<Acc>(apod[e]) : static_cast<Acc>(w);
            weightAcum += weight;
            numAdds++;
            // computeDelayDTSPACE_D, BF/RxBeamformerCommon.h:27-33
            float a = s.x + s.dirX * depth;
            float dx = x_elem - a;
            float dy = s.dirY * depth;
            float delayf = initialDelay + (std::sqrt(dx * dx + dy * dy) + depth) + static_cast<float>(additionalOffset);
            int32_t delay = static_cast<int32_t>(std::floor(delayf));
            Acc frac;
            if (sizeof(Acc) == sizeof(float)) {
                frac = delayf - static_cast<float>(delay);
            } else {
                double dd = static_cast<double>(initialDelay) +
                            (std::sqrt(static_cast<double>(dx) * dx + static_cast<double>(dy) * dy) + depth) +
                            additionalOffset;
                frac = static_cast<Acc>(dd - delay);
            }
            size_t base = static_cast<size_t>(channelIdx) * numTimesteps +
                          static_cast<size_t>(txScanlineIdx) * numReceivedChannels * numTimesteps;
            // signed delay compared against an unsigned bound (quirk Q9: negative delays skipped)
            if (static_cast<uint32_t>(delay) < numTimesteps - 1) {
                sample += weight * ((Acc(1) - frac) * static_cast<Acc>(rf[base + delay]) +
                                    frac * static_cast<Acc>(rf[base + delay + 1]));
            } else if (static_cast<uint32_t>(delay) < numTimesteps && frac == 0) {
                sample += weight * static_cast<Acc>(rf[base + delay]);
            }
        }
    }
    if (numAdds > 0) return sample / weightAcum * static_cast<Acc>(numAdds);
    return 0;
}

template <typename Acc>
Acc sampleBeamform3D(const sb_geometry* g, const GeomDT& G, const Window& win, const float* rf, const LineDT& s,
                     int k, float aDT, float depth, float invMaxX, float invMaxY, int32_t additionalOffset) {
    // RxSampleBeamformerDelayAndSum::sampleBeamform3D, BF/RxSampleBeamformerDelayAndSum.h:26-120
    Acc sample = 0;
    Acc weightAcum = 0;
    int numAdds = 0;
    float initialDelay = s.initialDelay[k];
    uint32_t txScanlineIdx = s.txIdx[k];
    uint32_t numTimesteps = g->num_samples;
    uint32_t numReceivedChannels = g->num_channels;
    for (uint32_t ex = s.firstX[k]; ex < s.lastX[k]; ex++) {
        for (uint32_t ey = s.firstY[k]; ey < s.lastY[k]; ey++) {
            uint32_t elemIdx = ex + ey * g->element_layout[0];
            int32_t ch = channelOf(g, elemIdx);
            if (ch < 0) continue;
            uint32_t channelIdx = static_cast<uint32_t>(ch);
            float x_elem = G.xe[elemIdx];
            float z_elem = G.ye[elemIdx];
            float ddx = x_elem - s.x, ddz = z_elem - s.z;
            if ((squ(ddx) + squ(ddz)) <= aDT) {
                // computeWindow3DShared, BF/RxBeamformerCommon.h:55-61
                float wx = win.get(ddx * invMaxX);
                float wz = win.get(ddz * invMaxY);
                float w = std::sqrt(wx * wz);
                Acc weight = static_cast<Acc>(w);
                weightAcum += weight;
                numAdds++;
                // computeDelayDTSPACE3D_D, BF/RxBeamformerCommon.h:35-42
                float ax = x_elem - (s.x + s.dirX * depth);
                float az = z_elem - (s.z + s.dirZ * depth);
                float ay = s.dirY * depth;
                float delayf = initialDelay + (std::sqrt(squ(ax) + squ(az) + squ(ay)) + depth) +
                               static_cast<float>(additionalOffset);
                // float -> uint32 conversion: negative values saturate to 0 on the GPU
                float fl = std::floor(delayf);
                uint32_t delay = fl <= 0.0f ? 0u : static_cast<uint32_t>(fl);
                Acc frac;
                if (sizeof(Acc) == sizeof(float)) {
                    frac = delayf - static_cast<float>(delay);
                } else {
                    double dd = static_cast<double>(initialDelay) +
                                (std::sqrt(static_cast<double>(ax) * ax + static_cast<double>(az) * az +
                                           static_cast<double>(ay) * ay) + depth) + additionalOffset;
                    frac = static_cast<Acc>(dd - delay);
                }
                size_t base = static_cast<size_t>(channelIdx) * numTimesteps +
                              static_cast<size_t>(txScanlineIdx) * numReceivedChannels * numTimesteps;
                if (delay < numTimesteps - 1) {
                    sample += weight * ((Acc(1) - frac) * static_cast<Acc>(rf[base + delay]) +
                                        frac * static_cast<Acc>(rf[base + delay + 1]));
                } else if (delay < numTimesteps && frac == 0) {
                    sample += weight * static_cast<Acc>(rf[base + delay]);
                }
            }
        }
    }
    if (numAdds > 0) return sample / weightAcum * static_cast<Acc>(numAdds);
    return 0;
}

template <typename Acc>
void dasFrame(const sb_geometry* g, const float* rf, Acc* out, double fNumber, double c, int windowType,
              float windowParameter, int interpolateTransmits, int32_t additionalOffset, const float* apod,
              int nthreads) {
    GeomDT G = toDtSpace(g, c);
    Window win(windowType, windowParameter, 64);
    bool is3D = g->rx_layout[0] > 1 && g->rx_layout[1] > 1;
    const float F = static_cast<float>(fNumber);
    const float speedOfSound = G.c, dt = G.dt;
    const int nD = static_cast<int>(g->num_depths), nRx = static_cast<int>(g->num_rx);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int line = 0; line < nRx; line++) {
        const LineDT& s = G.lines[line];
        for (int r = 0; r < nD; r++) {
            float d = G.depths[r];
            // computeAperture_D(F, d*dt*c)/c/dt, RxBeamformerCuda.cu:166 (3D, squared) / :263 (2D)
            float aDT = ((d * dt) * speedOfSound) / (2 * F) / speedOfSound / dt;
            Acc sInterp = 0;
            int hw = highestWeightIndex(s);
            bool invalid = false;
            for (int k = 0; k < 4; k++) {
                if (!interpolateTransmits && k != hw) continue;
                if (!(s.txWeights[k] > 0.0)) continue;
                if (s.txIdx[k] >= g->num_tx) { invalid = true; break; }
                Acc sLocal;
                if (is3D) {
                    float aDT2 = squ(aDT);
                    float sq = std::sqrt(aDT2);
                    float invX = 1.0f / std::min(sq, s.maxDistX);
                    float invY = 1.0f / std::min(sq, s.maxDistY);
                    sLocal = sampleBeamform3D<Acc>(g, G, win, rf, s, k, aDT2, d, invX, invY, additionalOffset);
                } else {
                    float inv = 1 / std::min(aDT, s.maxDistX);
                    sLocal = sampleBeamform2D<Acc>(g, G, win, rf, s, k, aDT, d, inv, additionalOffset, apod);
                }
                if (interpolateTransmits) sInterp += static_cast<Acc>(static_cast<float>(s.txWeights[k])) * sLocal;
                else sInterp += sLocal;
            }
            if (!invalid) {
                // clampCast<float> of the output (RxBeamformerCuda.cu:321); the FP64 variant keeps NaN
                if (sizeof(Acc) == sizeof(float)) out[static_cast<size_t>(r) * nRx + line] = clampToFloat(static_cast<float>(sInterp));
                else out[static_cast<size_t>(r) * nRx + line] = sInterp;
            }
        }
    }
}

// --------------------------------------------------------------------------------- DAS variants
// The other sample beamformers of RxBeamformerCuda::performRxBeamforming (BF/RxBeamformerCuda.cu:
// 567-591), called by the same kernels in place of the delay-and-sum reducer. Float semantics only.
enum { kBfDelayAndSum = 0, kBfDelayAndStdDev = 1, kBfCoherenceFactor = 2, kBfTestSignal = 3 };

// Interpolated sample of one element (the two cases of the reference's reducers). Returns false when
// the delay falls outside the record; `value` is then left as it was (the variants keep the previous
// element's value).
inline bool delayedSample2D(const float* rf, size_t base, uint32_t numTimesteps, float delayfIn, float weight,
                            bool weighted, float& value) {
    int32_t delay = static_cast<int32_t>(std::floor(delayfIn));
    float delayf = delayfIn - static_cast<float>(delay);
    if (static_cast<uint32_t>(delay) < numTimesteps - 1) {
        float v = (1.0f - delayf) * rf[base + delay] + delayf * rf[base + delay + 1];
        value = weighted ? weight * v : v;
        return true;
    } else if (static_cast<uint32_t>(delay) < numTimesteps && delayf == 0.0f) {
        value = weighted ? weight * rf[base + delay] : rf[base + delay];
        return true;
    }
    return false;
}

inline bool delayedSample3D(const float* rf, size_t base, uint32_t numTimesteps, float delayfIn, float weight,
                            bool weighted, float& value) {
    float fl = std::floor(delayfIn);
    uint32_t delay = fl <= 0.0f ? 0u : static_cast<uint32_t>(fl);  // float -> uint32 saturates on the GPU
    float delayf = delayfIn - static_cast<float>(delay);
    if (delay < numTimesteps - 1) {
        float v = (1.0f - delayf) * rf[base + delay] + delayf * rf[base + delay + 1];
        value = weighted ? weight * v : v;
        return true;
    } else if (delay < numTimesteps && delayf == 0.0f) {
        value = weighted ? weight * rf[base + delay] : rf[base + delay];
        return true;
    }
    return false;
}

// RxSampleBeamformerDelayAndStdDev::sampleBeamform2D (BF/RxSampleBeamformerDelayAndStdDev.h:146-248) and
// RxSampleBeamformerCoherenceFactorDelayAndSum::sampleBeamform2D (BF/RxSampleBeamformerCoherenceFactor
// DelayAndSum.h:139-235): the DAS result, then a second pass over the aperture.
float variant2D(int bf, const sb_geometry* g, const GeomDT& G, const Window& win, const float* rf, const LineDT& s,
                int k, float aDT, float depth, float invMax, int32_t additionalOffset) {
    float das = sampleBeamform2D<float>(g, G, win, rf, s, k, aDT, depth, invMax, additionalOffset, nullptr);
    float value = 0.0f, acc = 0.0f, acc2 = 0.0f, weightAcum = 0.0f;
    int numAdds = 0;
    const float initialDelay = s.initialDelay[k];
    const uint32_t nS = g->num_samples, nCh = g->num_channels;
    for (int32_t e = s.firstX[k]; e < s.lastX[k]; e++) {
        int32_t ch = channelOf(g, static_cast<uint32_t>(e));
        if (ch < 0) continue;
        float x_elem = G.xe[e];
        if (std::fabs(x_elem - s.x) <= aDT) {
            float weight = 0.0f;
            if (bf == kBfDelayAndStdDev) {
                weight = win.get((x_elem - s.x) * invMax);
                weightAcum += weight;
            }
            numAdds++;
            float a = s.x + s.dirX * depth;
            float dx = x_elem - a;
            float dy = s.dirY * depth;
            float delayf = initialDelay + (std::sqrt(dx * dx + dy * dy) + depth) + static_cast<float>(additionalOffset);
            size_t base = static_cast<size_t>(ch) * nS + static_cast<size_t>(s.txIdx[k]) * nCh * nS;
            delayedSample2D(rf, base, nS, delayf, weight, bf == kBfDelayAndStdDev, value);
            if (bf == kBfDelayAndStdDev) {
                acc += squ(value - das);
            } else {
                acc += value;
                acc2 += squ(value);
            }
        }
    }
    if (numAdds == 0) return 0.0f;
    if (bf == kBfDelayAndStdDev) return std::sqrt(acc) / weightAcum * static_cast<float>(numAdds);
    return squ(acc) / acc2 / static_cast<float>(numAdds) * das;
}

// The 3D reducers of the same classes (DelayAndStdDev.h:34-144, CoherenceFactorDelayAndSum.h:30-137).
float variant3D(int bf, const sb_geometry* g, const GeomDT& G, const Window& win, const float* rf, const LineDT& s,
                int k, float aDT, float depth, float invMaxX, float invMaxY, int32_t additionalOffset) {
    float das = sampleBeamform3D<float>(g, G, win, rf, s, k, aDT, depth, invMaxX, invMaxY, additionalOffset);
    float value = 0.0f, acc = 0.0f, acc2 = 0.0f, weightAcum = 0.0f;
    int numAdds = 0;
    const float initialDelay = s.initialDelay[k];
    const uint32_t nS = g->num_samples, nCh = g->num_channels;
    for (uint32_t ex = s.firstX[k]; ex < s.lastX[k]; ex++) {
        for (uint32_t ey = s.firstY[k]; ey < s.lastY[k]; ey++) {
            uint32_t elemIdx = ex + ey * g->element_layout[0];
            int32_t ch = channelOf(g, elemIdx);
            if (ch < 0) continue;
            float x_elem = G.xe[elemIdx];
            float z_elem = G.ye[elemIdx];
            if ((squ(x_elem - s.x) + squ(z_elem - s.z)) <= aDT) {
                float weight = 0.0f;
                if (bf == kBfDelayAndStdDev) {
                    float wx = win.get((x_elem - s.x) * invMaxX);
                    float wz = win.get((z_elem - s.z) * invMaxY);
                    weight = std::sqrt(wx * wz);
                    weightAcum += weight;
                }
                numAdds++;
                float ax = x_elem - (s.x + s.dirX * depth);
                float az = z_elem - (s.z + s.dirZ * depth);
                float ay = s.dirY * depth;
                float delayf = initialDelay + (std::sqrt(squ(ax) + squ(az) + squ(ay)) + depth) +
                               static_cast<float>(additionalOffset);
                size_t base = static_cast<size_t>(ch) * nS + static_cast<size_t>(s.txIdx[k]) * nCh * nS;
                delayedSample3D(rf, base, nS, delayf, weight, bf == kBfDelayAndStdDev, value);
                if (bf == kBfDelayAndStdDev) {
                    acc += squ(value - das);
                } else {
                    acc += value;
                    acc2 += squ(value);
                }
            }
        }
    }
    if (numAdds == 0) return 0.0f;
    if (bf == kBfDelayAndStdDev) return std::sqrt(acc) / weightAcum * static_cast<float>(numAdds);
    return squ(acc) / acc2 / static_cast<float>(numAdds) * das;
}

// RxSampleBeamformerTestSignal (BF/RxSampleBeamformerTestSignal.h:24-133): 2 mm cylinders every 6 mm
// at 30 mm depth, along the elevation axis (and, in 3D, along x), value 1000 inside.
float testSignal(const LineDT& s, float depth, float dt, float speedOfSound, bool is3D) {
    const float spacing = 6.0f, diameter = 2.0f, cDepth = 30.0f;
    float px = s.x + s.dirX * depth, py = s.dirY * depth, pz = is3D ? s.z + s.dirZ * depth : s.dirZ * depth;
    px = px * dt * speedOfSound;
    py = py * dt * speedOfSound;
    pz = pz * dt * speedOfSound;
    float sample = 0.0f;
    for (int n = -3; n <= 3; n++) {
        float dx = px - static_cast<float>(n) * spacing, dy = py - cDepth, dz = 0.0f - 0.0f;
        if (std::sqrt(dx * dx + dy * dy + dz * dz) <= diameter) sample = 1000.0f;
    }
    if (is3D) {
        for (int n = -3; n <= 3; n++) {
            float dx = 0.0f - 0.0f, dy = py - cDepth, dz = pz - static_cast<float>(n) * spacing;
            if (std::sqrt(dx * dx + dy * dy + dz * dz) <= diameter) sample = 1000.0f;
        }
    }
    return sample;
}

void dasFrameBf(const sb_geometry* g, const float* rf, float* out, double fNumber, double c, int windowType,
                float windowParameter, int interpolateTransmits, int32_t additionalOffset, int bf, int nthreads) {
    GeomDT G = toDtSpace(g, c);
    Window win(windowType, windowParameter, 64);
    bool is3D = g->rx_layout[0] > 1 && g->rx_layout[1] > 1;
    const float F = static_cast<float>(fNumber);
    const float speedOfSound = G.c, dt = G.dt;
    const int nD = static_cast<int>(g->num_depths), nRx = static_cast<int>(g->num_rx);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int line = 0; line < nRx; line++) {
        const LineDT& s = G.lines[line];
        for (int r = 0; r < nD; r++) {
            float d = G.depths[r];
            float aDT = ((d * dt) * speedOfSound) / (2 * F) / speedOfSound / dt;
            float sInterp = 0;
            int hw = highestWeightIndex(s);
            bool invalid = false;
            for (int k = 0; k < 4; k++) {
                if (!interpolateTransmits && k != hw) continue;
                if (!(s.txWeights[k] > 0.0)) continue;
                if (s.txIdx[k] >= g->num_tx) { invalid = true; break; }
                float sLocal;
                if (bf == kBfTestSignal) {
                    sLocal = testSignal(s, d, dt, speedOfSound, is3D);
                } else if (is3D) {
                    float aDT2 = squ(aDT);
                    float sq = std::sqrt(aDT2);
                    float invX = 1.0f / std::min(sq, s.maxDistX);
                    float invY = 1.0f / std::min(sq, s.maxDistY);
                    sLocal = bf == kBfDelayAndSum ? sampleBeamform3D<float>(g, G, win, rf, s, k, aDT2, d, invX, invY, additionalOffset)
                                                  : variant3D(bf, g, G, win, rf, s, k, aDT2, d, invX, invY, additionalOffset);
                } else {
                    float inv = 1 / std::min(aDT, s.maxDistX);
                    sLocal = bf == kBfDelayAndSum ? sampleBeamform2D<float>(g, G, win, rf, s, k, aDT, d, inv, additionalOffset, nullptr)
                                                  : variant2D(bf, g, G, win, rf, s, k, aDT, d, inv, additionalOffset);
                }
                if (interpolateTransmits) sInterp += static_cast<float>(s.txWeights[k]) * sLocal;
                else sInterp += sLocal;
            }
            if (!invalid) out[static_cast<size_t>(r) * nRx + line] = clampToFloat(sInterp);
        }
    }
}

// ------------------------------------------------------------------------------------- raw delay
// RawDelay::sampleDelay2D + rxDelayDTSPACEKernel, BF/RawDelay.cu:221-312 and :406-468.
void rawDelayFrame(const sb_geometry* g, const float* rf, float* out, double fNumber, double c, int windowType,
                   float windowParameter, int nthreads) {
    GeomDT G = toDtSpace(g, c);
    Window win(windowType, windowParameter, 64);
    const float F = static_cast<float>(fNumber);
    const int nD = static_cast<int>(g->num_depths), nRx = static_cast<int>(g->num_rx);
    const uint32_t nCh = g->num_channels, nS = g->num_samples;
    std::fill(out, out + static_cast<size_t>(nRx) * nCh * nD, 0.0f);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int line = 0; line < nRx; line++) {
        const LineDT& s = G.lines[line];
        int k = highestWeightIndex(s);
        if (!(s.txWeights[k] > 0.0)) continue;
        if (s.txIdx[k] >= g->num_tx) continue;
        for (int r = 0; r < nD; r++) {
            float d = G.depths[r];
            float aDT = ((d * G.dt) * G.c) / (2 * F) / G.c / G.dt;
            float invMax = 1 / std::min(aDT, s.maxDistX);
            float weightAcum = 0.0f;
            int numAdds = 0;
            for (int32_t e = s.firstX[k]; e < s.lastX[k]; e++) {
                float x_elem = G.xe[e];
                if (std::fabs(x_elem - s.x) <= aDT) {
                    weightAcum += win.get((x_elem - s.x) * invMax);
                    numAdds++;
                }
            }
            float weightingScale = 1.0f;
            if (numAdds > 0) weightingScale = 1.0f / weightAcum * numAdds;
            int32_t local = 0;
            for (int32_t e = s.firstX[k]; e < s.lastX[k]; e++, local++) {
                float sample = 0.0f;
                uint32_t ch = static_cast<uint32_t>(e) % nCh;
                float x_elem = G.xe[e];
                if (std::fabs(x_elem - s.x) <= aDT) {
                    float weight = win.get((x_elem - s.x) * invMax);
                    float a = s.x + s.dirX * d;
                    float dx = x_elem - a;
                    float dy = s.dirY * d;
                    float delayf = s.initialDelay[k] + (std::sqrt(dx * dx + dy * dy) + d);
                    int32_t delay = static_cast<int32_t>(std::floor(delayf));
                    delayf -= delay;
                    size_t base = static_cast<size_t>(ch) * nS + static_cast<size_t>(s.txIdx[k]) * nCh * nS;
                    if (static_cast<uint32_t>(delay) < nS - 1) {
                        sample = weight * ((1.0f - delayf) * rf[base + delay] + delayf * rf[base + delay + 1]);
                    } else if (static_cast<uint32_t>(delay) < nS && delayf == 0.0f) {
                        sample = weight * rf[base + delay];
                    }
                }
                if (static_cast<uint32_t>(local) < nCh)
                    out[static_cast<size_t>(r) + static_cast<size_t>(local) * nD + static_cast<size_t>(line) * nCh * nD] =
                        clampToFloat(sample * weightingScale);
            }
        }
    }
}

}  // namespace

// ================================================================================================
extern "C" {

int orc_window_lut(int type, float param, uint32_t n, float* out) {
    if (n < 2 || !out) return -1;
    auto v = windowLut(type, param, n);
    std::copy(v.begin(), v.end(), out);
    return 0;
}

int orc_fir(uint32_t length, int type, int window, double fs, double f, double bw, float* out) {
    if (length < 1 || !out) return -1;
    auto v = firDesign(length, type, window, fs, f, bw);
    std::copy(v.begin(), v.end(), out);
    return 0;
}

// Window weight of a relative position, for pinning WindowFunctionGpu::get.
float orc_window_get(int type, float param, uint32_t n, float rel) {
    Window w(type, param, n);
    return w.get(rel);
}

// DT-space conversion outputs (for pinning the geometry arithmetic).
int orc_dt_space(const sb_geometry* g, double c, float* xe, float* ye, float* depths, float* line_xz) {
    GeomDT G = toDtSpace(g, c);
    std::copy(G.xe.begin(), G.xe.end(), xe);
    std::copy(G.ye.begin(), G.ye.end(), ye);
    std::copy(G.depths.begin(), G.depths.end(), depths);
    for (size_t i = 0; i < G.lines.size(); i++) {
        line_xz[4 * i + 0] = G.lines[i].x;
        line_xz[4 * i + 1] = G.lines[i].z;
        line_xz[4 * i + 2] = G.lines[i].maxDistX;
        line_xz[4 * i + 3] = G.lines[i].initialDelay[0];
    }
    return 0;
}

// DAS over one frame. rf is FP32 [num_tx][num_channels][num_samples] (int16 data converted exactly).
// precision 32: reference float semantics into out_f32. precision 64: double accumulation into out_f64.
int orc_das(const sb_geometry* g, const float* rf, float* out_f32, double* out_f64, double fNumber, double c,
            int windowType, float windowParameter, int interpolateTransmits, int32_t additionalOffset,
            const float* apod, int precision, int nthreads) {
    if (!g || !rf) return -1;
    if (nthreads <= 0) nthreads = 1;
    if (precision == 64) {
        if (!out_f64) return -1;
        dasFrame<double>(g, rf, out_f64, fNumber, c, windowType, windowParameter, interpolateTransmits,
                         additionalOffset, apod, nthreads);
    } else {
        if (!out_f32) return -1;
        dasFrame<float>(g, rf, out_f32, fNumber, c, windowType, windowParameter, interpolateTransmits,
                        additionalOffset, apod, nthreads);
    }
    return 0;
}

// DAS with another sample beamformer (0 DelayAndSum, 1 DelayAndStdDev, 2 CoherenceFactorDelayAndSum,
// 3 TestSignal: the order of RxBeamformerCuda::RxSampleBeamformer, BF/RxBeamformerCuda.h:31-36).
int orc_das_bf(const sb_geometry* g, const float* rf, float* out, double fNumber, double c, int windowType,
               float windowParameter, int interpolateTransmits, int32_t additionalOffset, int beamformer, int nthreads) {
    if (!g || !rf || !out || beamformer < 0 || beamformer > 3) return -1;
    dasFrameBf(g, rf, out, fNumber, c, windowType, windowParameter, interpolateTransmits, additionalOffset, beamformer,
               nthreads <= 0 ? 1 : nthreads);
    return 0;
}

// TemporalFilter::filter + temporalFilterKernel (BF/TemporalFilter.cu:22-46, WorkType float): per element
// sum += w_k * x_k, sumWeights += w_k over the images in order, then sum / sumWeights, clampCast to
// out_dtype (SB_FLOAT32 or SB_INT16; out holds that type). Images are given as float.
int orc_temporal_filter(const float* const* images, uint32_t n, const double* weights, uint64_t numel, void* out,
                        int out_dtype) {
    if (!images || !out || n == 0) return -1;
    for (uint64_t i = 0; i < numel; i++) {
        float sum = 0.0f, sumWeights = 0.0f;
        for (uint32_t k = 0; k < n; k++) {
            float w = static_cast<float>(weights ? weights[k] : 1.0);
            sum += w * images[k][i];
            sumWeights += w;
        }
        sum /= sumWeights;
        storeClamped(out, out_dtype, i, sum);
    }
    return 0;
}

// FP64 reference gradient of the apodised 2D DAS (extension without a reference counterpart): the
// transpose of sampleBeamform2D<double> with apodisation (same discrete decisions: aperture, window
// index, sample index), highest-weight transmit. For a pixel with upstream g, W_e = w_e a_e,
// D = sum W_e, n active elements, v_e = lerp(rf, tau_e), s = n / D sum W_e v_e:
//   grad_rf[delta] += g n / D W_e (1 - frac), grad_rf[delta + 1] += g n / D W_e frac,
//   grad_apod[e] += g w_e (n v_e - s) / D,
//   grad_c += g n / D sum_e W_e (rf[delta + 1] - rf[delta]) * (-(path_e) / c), path = dist + depth (DT units).
// Single-threaded (the scatter is not partitioned). grad_rf has rf's shape.
int orc_das_adjoint64(const sb_geometry* g, const float* rf, const float* apod, const double* gout, double* grad_rf,
                      double* grad_apod, double* grad_c, double fNumber, double c, int windowType,
                      float windowParameter) {
    if (!g || !rf || !gout) return -1;
    GeomDT G = toDtSpace(g, c);
    Window win(windowType, windowParameter, 64);
    const float F = static_cast<float>(fNumber);
    const float speedOfSound = G.c, dt = G.dt;
    const uint32_t nS = g->num_samples, nCh = g->num_channels;
    if (grad_rf) std::fill(grad_rf, grad_rf + static_cast<size_t>(g->num_tx) * nCh * nS, 0.0);
    if (grad_apod) std::fill(grad_apod, grad_apod + g->num_elements, 0.0);
    double gc = 0.0;
    for (uint32_t line = 0; line < g->num_rx; line++) {
        const LineDT& s = G.lines[line];
        const int k = highestWeightIndex(s);
        if (!(s.txWeights[k] > 0.0) || s.txIdx[k] >= g->num_tx) continue;
        for (uint32_t r = 0; r < g->num_depths; r++) {
            const float d = G.depths[r];
            const float aDT = ((d * dt) * speedOfSound) / (2 * F) / speedOfSound / dt;
            const float inv = 1 / std::min(aDT, s.maxDistX);
            const double gp = gout[static_cast<size_t>(r) * g->num_rx + line];
            if (gp == 0.0) continue;
            struct Term { uint32_t e; size_t base; int32_t delay; double w, W, frac, v, slope, path; int kind; };
            std::vector<Term> terms;
            double D = 0.0, num = 0.0;
            int n = 0;
            for (int32_t e = s.firstX[k]; e < s.lastX[k]; e++) {
                int32_t ch = channelOf(g, static_cast<uint32_t>(e));
                if (ch < 0) continue;
                float x_elem = G.xe[e];
                if (!(std::fabs(x_elem - s.x) <= aDT)) continue;
                Term t{};
                t.e = static_cast<uint32_t>(e);
                t.w = win.get((x_elem - s.x) * inv);
                t.W = apod ? t.w * static_cast<double>(apod[e]) : t.w;
                D += t.W;
                n++;
                float a = s.x + s.dirX * d;
                float dx = x_elem - a;
                float dy = s.dirY * d;
                float delayf = s.initialDelay[k] + (std::sqrt(dx * dx + dy * dy) + d);
                t.delay = static_cast<int32_t>(std::floor(delayf));
                t.path = std::sqrt(static_cast<double>(dx) * dx + static_cast<double>(dy) * dy) + d;
                double dd = static_cast<double>(s.initialDelay[k]) + t.path;
                t.frac = dd - t.delay;
                t.base = static_cast<size_t>(ch) * nS + static_cast<size_t>(s.txIdx[k]) * nCh * nS;
                t.kind = 0;
                if (static_cast<uint32_t>(t.delay) < nS - 1) {
                    double v0 = rf[t.base + t.delay], v1 = rf[t.base + t.delay + 1];
                    t.v = (1 - t.frac) * v0 + t.frac * v1;
                    t.slope = v1 - v0;
                    t.kind = 1;
                } else if (static_cast<uint32_t>(t.delay) < nS && static_cast<float>(delayf - static_cast<float>(t.delay)) == 0.0f) {
                    t.v = rf[t.base + t.delay];
                    t.kind = 2;
                }
                num += t.W * t.v;
                terms.push_back(t);
            }
            if (n == 0 || gp == 0.0 || !(D != 0.0)) continue;
            const double sv = num / D * n;
            if (!std::isfinite(sv)) continue;
            const double G1 = gp * n / D;
            for (const Term& t : terms) {
                if (t.kind == 1) {
                    if (grad_rf) {
                        grad_rf[t.base + t.delay] += G1 * t.W * (1 - t.frac);
                        grad_rf[t.base + t.delay + 1] += G1 * t.W * t.frac;
                    }
                    gc += G1 * t.W * t.slope * (-t.path / c);
                } else if (t.kind == 2 && grad_rf) {
                    grad_rf[t.base + t.delay] += G1 * t.W;
                }
                if (grad_apod) grad_apod[t.e] += gp * t.w * (n * t.v - sv) / D;
            }
        }
    }
    if (grad_c) *grad_c = gc;
    return 0;
}

int orc_rawdelay(const sb_geometry* g, const float* rf, float* out, double fNumber, double c, int windowType,
                 float windowParameter, int nthreads) {
    if (!g || !rf || !out) return -1;
    rawDelayFrame(g, rf, out, fNumber, c, windowType, windowParameter, nthreads > 0 ? nthreads : 1);
    return 0;
}

// HilbertFirEnvelope: kernelFilterDemodulation, BF/HilbertFirEnvelope.cu:28-61, filter from
// FirFilterFactory(Hilbert, Hamming) :75-81. Even lengths read filter[N] in the reference (Q3): 0 here.
int orc_hilbert_env(const float* in, float* out, uint32_t numScanlines, uint32_t numSamples, uint32_t filterLength,
                    int nthreads) {
    std::vector<float> h = firDesign(filterLength, 3, 2, 2.0, 0.0, 0.0);
    h.push_back(0.0f);
    const int nS = static_cast<int>(numSamples), nL = static_cast<int>(numScanlines), N = static_cast<int>(filterLength);
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1)
    for (int s = 0; s < nS; s++) {
        for (int l = 0; l < nL; l++) {
            float acc = 0;
            int start = s - N / 2, end = s + N / 2, fe = 0;
            for (int cs = start; cs <= end; cs++, fe++) {
                if (cs >= 0 && cs < nS) acc += in[l + static_cast<size_t>(cs) * nL] * h[fe];
            }
            float v = in[l + static_cast<size_t>(s) * nL];
            out[l + static_cast<size_t>(s) * nL] = std::sqrt(squ(v) + squ(acc));
        }
    }
    return 0;
}

// LogCompressor: thrustLogcompress, BF/LogCompressor.cu:22-64 (WorkType float).
int orc_logcompress(const void* in, int inDtype, void* out, int outDtype, size_t n, double dynamicRange,
                    double gain, double inMax) {
    double dr = std::pow(10, (dynamicRange / 20));
    double inMaxT = inDtype == SB_INT16 ? static_cast<double>(static_cast<int16_t>(inMax))
                  : inDtype == SB_UINT8 ? static_cast<double>(static_cast<uint8_t>(inMax))
                                        : static_cast<double>(static_cast<float>(inMax));
    double outMax = outDtype == SB_UINT8 ? 255.0 : 255.0;
    float inScale = static_cast<float>(dr / inMaxT);
    float scaleOverDen = static_cast<float>(gain * outMax / std::log10(dr + 1));
    for (size_t i = 0; i < n; i++) {
        float a = loadAsFloat(in, inDtype, i);
        float val = std::log10(std::fabs(a) * inScale + 1.0f) * scaleOverDen;
        storeClamped(out, outDtype, i, val);
    }
    return 0;
}

// IQDemodulator::demodulateMagnitudeFrequencyCompounding, BF/IQDemodulator.cu:215-345: the filter
// bank kernel (:68-137, bank offset 1, I phase 0, Q phase 3/4) then the strided low-pass (:142-175).
int orc_iq_magnitude(const float* in, float* out, uint32_t numScanlines, uint32_t numSamples, uint32_t decimation,
                     double fs, double cutoff, uint32_t lpLength, uint32_t bpLength, uint32_t numFilters,
                     const double* refFreqs, const double* bandwidths, const double* weights, int nthreads) {
    if (numFilters < 1 || numFilters > 8) return -1;
    std::vector<std::vector<float>> bank(numFilters);
    float weightAcum = 0;
    std::vector<float> w(numFilters), fOverFs(numFilters);
    for (uint32_t k = 0; k < numFilters; k++) {
        if (refFreqs[k] > 0 && bandwidths[k] > 0) bank[k] = firDesign(bpLength, 2, 3, fs, refFreqs[k], bandwidths[k]);
        else bank[k].assign(bpLength, 0.0f);
        bank[k].push_back(0.0f);  // Q3: tap N reads as 0
        w[k] = static_cast<float>(weights[k]);
        weightAcum += static_cast<float>(weights[k]);
        fOverFs[k] = static_cast<float>(refFreqs[k] / fs);
    }
    float scale = 1 / weightAcum;
    std::vector<float> lp = firDesign(lpLength, 0, 2, fs, cutoff, 0.0);
    lp.push_back(0.0f);
    const int nS = static_cast<int>(numSamples), nL = static_cast<int>(numScanlines);
    const int bpN = static_cast<int>(bpLength), lpN = static_cast<int>(lpLength);
    std::vector<float> band(static_cast<size_t>(nS) * nL);
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1)
    for (int s = 0; s < nS; s++) {
        for (int l = 0; l < nL; l++) {
            float acc[8] = {0};
            float signalValue = in[l + static_cast<size_t>(s) * nL];
            acc[0] = signalValue;
            int start = s - bpN / 2, end = s + bpN / 2, fe = 0;
            for (int cs = start; cs <= end; cs++, fe++) {
                if (cs >= 0 && cs < nS) {
                    float sample = in[l + static_cast<size_t>(cs) * nL];
                    for (uint32_t f = 1; f < numFilters; f++) acc[f] += sample * bank[f][fe];
                }
            }
            float accumulator = 0;
            for (uint32_t f = 0; f < numFilters; f++) {
                float sv = acc[f];
                float ph = s * fOverFs[f];
                float phI = ph + 0.0f / 1.0f;
                float phQ = ph + 3.0f / 4.0f;
                phI = phI - std::trunc(phI);
                phQ = phQ - std::trunc(phQ);
                float rI = std::cos(phI * 2.0f * static_cast<float>(M_PI));
                float rQ = std::cos(phQ * 2.0f * static_cast<float>(M_PI));
                float dI = sv * rI, dQ = sv * rQ;
                accumulator += w[f] * std::sqrt(squ(dI) + squ(dQ));
            }
            band[l + static_cast<size_t>(s) * nL] = scale * accumulator;
        }
    }
    int nOut = decimation > 1 ? nS / static_cast<int>(decimation) : nS;
    int stride = static_cast<int>(std::max(decimation, 1u));
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1)
    for (int so = 0; so < nOut; so++) {
        int si = so * stride;
        if (si >= nS) continue;
        for (int l = 0; l < nL; l++) {
            float acc = 0;
            int start = si - lpN / 2, end = si + lpN / 2, fe = 0;
            for (int cs = start; cs <= end; cs++, fe++)
                if (cs >= 0 && cs < nS) acc += band[l + static_cast<size_t>(cs) * nL] * lp[fe];
            out[l + static_cast<size_t>(so) * nL] = clampToFloat(acc);
        }
    }
    return 0;
}

// Complex baseband IQ (extension, no reference counterpart), FP64: x[n] exp(-j 2 pi f n / fs), then a
// Hamming low-pass of lpLength taps centred on the output sample (taps -N/2..N/2, tap N = 0), every
// decimation-th sample. out interleaved complex, [numSamples/decimation][numScanlines].
int orc_iq_complex(const float* in, double* out, uint32_t numScanlines, uint32_t numSamples, double fs, double fmix,
                   double cutoff, uint32_t lpLength, uint32_t decimation, int nthreads) {
    std::vector<float> lpf = firDesign(lpLength, 0, 2, fs, cutoff, 0.0);
    std::vector<double> lp(lpf.begin(), lpf.end());
    lp.push_back(0.0);
    const int nS = static_cast<int>(numSamples), nL = static_cast<int>(numScanlines), N = static_cast<int>(lpLength);
    int dec = static_cast<int>(std::max(decimation, 1u));
    int nOut = nS / dec;
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1)
    for (int so = 0; so < nOut; so++) {
        int si = so * dec;
        for (int l = 0; l < nL; l++) {
            double re = 0, im = 0;
            int start = si - N / 2, end = si + N / 2, fe = 0;
            for (int cs = start; cs <= end; cs++, fe++) {
                if (cs >= 0 && cs < nS) {
                    double x = in[l + static_cast<size_t>(cs) * nL];
                    double ph = 2.0 * M_PI * fmix / fs * cs;
                    re += lp[fe] * x * std::cos(ph);
                    im -= lp[fe] * x * std::sin(ph);
                }
            }
            out[2 * (l + static_cast<size_t>(so) * nL) + 0] = re;
            out[2 * (l + static_cast<size_t>(so) * nL) + 1] = im;
        }
    }
    return 0;
}

}  // extern "C"
