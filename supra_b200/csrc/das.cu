// Delay-and-sum receive beamforming (2D and 3D) and the raw-delay stage, per frame.
//
// Semantics follow RxBeamformerCuda / RxSampleBeamformerDelayAndSum (Beamformer/RxBeamformerCuda.cu:119-323,
// Beamformer/RxSampleBeamformerDelayAndSum.h:26-208) and RawDelay (Beamformer/RawDelay.cu:221-468).
// The discrete decisions of the reference — aperture membership, the nearest window-LUT entry, the
// sample index — are evaluated with the same IEEE float operations in the same order (explicit
// _rn intrinsics, so nothing is contracted into FMAs), which keeps them bit-identical to the CPU
// restatement of the reference.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "batch_pack.cuh"
#include "das.cuh"
#include "das_core.cuh"
#include "design.h"

namespace sb {

WindowLut makeLut(int windowType, float windowParameter) {
    WindowLut w;
    std::vector<float> v = windowLut(windowType, windowParameter, 64);
    for (int i = 0; i < 64; i++) w.v[i] = v[i];
    return w;
}

namespace {

// convertToDtSpace (RxBeamformerCuda.cu:58-107), first-call form: mm -> units of c*dt in double,
// then rounded to float as the kernels read them.
__global__ void dtConvertKernel(const float* xeMM, const float* yeMM, uint32_t nE, const float* dMM, uint32_t nD,
                                const sb_scanline_rx* lines, uint32_t nRx, double factor, double factorTime,
                                float* xe, float* ye, float* d, LineDT* out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nE) {
        xe[i] = static_cast<float>(static_cast<double>(xeMM[i]) * factor);
        ye[i] = static_cast<float>(static_cast<double>(yeMM[i]) * factor);
    }
    if (i < nD) d[i] = static_cast<float>(static_cast<double>(dMM[i]) * factor);
    if (i < nRx) {
        const sb_scanline_rx& s = lines[i];
        LineDT o;
        o.x = static_cast<float>(s.position[0] * factor);
        o.z = static_cast<float>(s.position[2] * factor);
        o.dirX = static_cast<float>(s.direction[0]);
        o.dirY = static_cast<float>(s.direction[1]);
        o.dirZ = static_cast<float>(s.direction[2]);
        o.maxDistX = static_cast<float>(s.max_element_distance[0] * factor);
        o.maxDistY = static_cast<float>(s.max_element_distance[1] * factor);
        int hi = 0;
        float hw = static_cast<float>(s.tx_weights[0]);
        int mask = 0;
        for (int k = 0; k < 4; k++) {
            o.txWeight[k] = static_cast<float>(s.tx_weights[k]);
            o.initialDelay[k] = static_cast<float>(s.tx[k].initial_delay_s * factorTime);
            o.firstX[k] = s.tx[k].first_active_element[0];
            o.firstY[k] = s.tx[k].first_active_element[1];
            o.lastX[k] = s.tx[k].last_active_element[0];
            o.lastY[k] = s.tx[k].last_active_element[1];
            o.txIdx[k] = s.tx[k].tx_scanline_idx;
            if (s.tx_weights[k] > 0.0) mask |= 1 << k;
            if (k > 0 && s.tx_weights[k] > static_cast<double>(hw)) {  // double vs promoted float, as the reference
                hw = static_cast<float>(s.tx_weights[k]);
                hi = k;
            }
        }
        o.highest = hi;
        o.activeMask = mask;
        out[i] = o;
    }
}

struct DasArgs {
    const void* rf;
    void* out;
    const float* xe;
    const float* ye;
    const float* depth;
    const LineDT* lines;
    const int32_t* e2c;
    const float* apod;
    uint32_t nE, layoutX, nCh, nS, nTx, nRx, nD;
    float c, dt, F, offset;
    int interpTx;
    WindowLut lut;
};

// WindowFunctionGpu::get (Beamformer/WindowFunction.h:58-64): nearest of 64 entries.
__device__ __forceinline__ float lutGet(const float* lut, float rel) {
    float cl = fminf(fmaxf(rel, -1.0f), 1.0f);
    uint32_t idx = static_cast<uint32_t>(roundf(__fmul_rn(31.5f, __fadd_rn(cl, 1.0f))));
    return lut[idx];
}

// computeAperture_D(F, d*dt*c)/c/dt (Beamformer/RxBeamformerCommon.h:21-25, RxBeamformerCuda.cu:263)
__device__ __forceinline__ float apertureDT(float d, float dt, float c, float F) {
    return __fdiv_rn(__fdiv_rn(__fdiv_rn(__fmul_rn(__fmul_rn(d, dt), c), __fmul_rn(2.0f, F)), c), dt);
}

template <typename RF>
__device__ __forceinline__ float sample2D(const DasArgs& a, const LineDT& s, int k, const float* lut, float aDT,
                                          float depth, float invMax) {
    float sample = 0.0f, weightAcum = 0.0f;
    int numAdds = 0;
    const float iD = s.initialDelay[k];
    const RF* tx = static_cast<const RF*>(a.rf) + static_cast<size_t>(s.txIdx[k]) * a.nCh * a.nS;
    const float xz = __fadd_rn(s.x, __fmul_rn(s.dirX, depth));
    const float dy = __fmul_rn(s.dirY, depth);
    const float dy2 = __fmul_rn(dy, dy);
    for (int e = s.firstX[k]; e < s.lastX[k]; e++) {
        int ch = a.e2c ? __ldg(a.e2c + e) : static_cast<int>(static_cast<uint32_t>(e) % a.nCh);
        if (ch < 0) continue;
        const float xel = __ldg(a.xe + e);
        const float dx = __fsub_rn(xel, s.x);
        if (fabsf(dx) <= aDT) {
            float w = lutGet(lut, __fmul_rn(dx, invMax));
            if (a.apod) w = __fmul_rn(w, __ldg(a.apod + e));
            weightAcum = __fadd_rn(weightAcum, w);
            numAdds++;
            const float ex = __fsub_rn(xel, xz);
            const float dist = __fsqrt_rn(__fadd_rn(__fmul_rn(ex, ex), dy2));
            const float delayf = __fadd_rn(__fadd_rn(iD, __fadd_rn(dist, depth)), a.offset);
            const int32_t delay = static_cast<int32_t>(floorf(delayf));
            const float frac = __fsub_rn(delayf, static_cast<float>(delay));
            const RF* p = tx + static_cast<size_t>(ch) * a.nS;
            if (static_cast<uint32_t>(delay) < a.nS - 1) {
                const float v0 = toFloat(p[delay]), v1 = toFloat(p[delay + 1]);
                const float v = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, frac), v0), __fmul_rn(frac, v1));
                sample = __fadd_rn(sample, __fmul_rn(w, v));
            } else if (static_cast<uint32_t>(delay) < a.nS && frac == 0.0f) {
                sample = __fadd_rn(sample, __fmul_rn(w, toFloat(p[delay])));
            }
        }
    }
    return numAdds > 0 ? __fmul_rn(__fdiv_rn(sample, weightAcum), static_cast<float>(numAdds)) : 0.0f;
}

template <typename RF>
__device__ __forceinline__ float sample3D(const DasArgs& a, const LineDT& s, int k, const float* lut, float aDT2,
                                          float depth, float invX, float invY) {
    float sample = 0.0f, weightAcum = 0.0f;
    int numAdds = 0;
    const float iD = s.initialDelay[k];
    const RF* tx = static_cast<const RF*>(a.rf) + static_cast<size_t>(s.txIdx[k]) * a.nCh * a.nS;
    const float px = __fadd_rn(s.x, __fmul_rn(s.dirX, depth));
    const float pz = __fadd_rn(s.z, __fmul_rn(s.dirZ, depth));
    const float ay = __fmul_rn(s.dirY, depth);
    const float ay2 = __fmul_rn(ay, ay);
    for (uint32_t ex = s.firstX[k]; ex < s.lastX[k]; ex++) {
        for (uint32_t ey = s.firstY[k]; ey < s.lastY[k]; ey++) {
            const uint32_t e = ex + ey * a.layoutX;
            int ch = a.e2c ? __ldg(a.e2c + e) : static_cast<int>(e % a.nCh);
            if (ch < 0) continue;
            const float xel = __ldg(a.xe + e), zel = __ldg(a.ye + e);
            const float dx = __fsub_rn(xel, s.x), dz = __fsub_rn(zel, s.z);
            if (__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dz, dz)) <= aDT2) {
                const float w = __fsqrt_rn(__fmul_rn(lutGet(lut, __fmul_rn(dx, invX)), lutGet(lut, __fmul_rn(dz, invY))));
                weightAcum = __fadd_rn(weightAcum, w);
                numAdds++;
                const float qx = __fsub_rn(xel, px), qz = __fsub_rn(zel, pz);
                const float q = __fadd_rn(__fadd_rn(__fmul_rn(qx, qx), __fmul_rn(qz, qz)), ay2);
                const float delayf = __fadd_rn(__fadd_rn(iD, __fadd_rn(__fsqrt_rn(q), depth)), a.offset);
                const uint32_t delay = static_cast<uint32_t>(floorf(delayf));  // saturates at 0 like the reference
                const float frac = __fsub_rn(delayf, static_cast<float>(delay));
                const RF* p = tx + static_cast<size_t>(ch) * a.nS;
                if (delay < a.nS - 1) {
                    const float v0 = toFloat(p[delay]), v1 = toFloat(p[delay + 1]);
                    const float v = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, frac), v0), __fmul_rn(frac, v1));
                    sample = __fadd_rn(sample, __fmul_rn(w, v));
                } else if (delay < a.nS && frac == 0.0f) {
                    sample = __fadd_rn(sample, __fmul_rn(w, toFloat(p[delay])));
                }
            }
        }
    }
    return numAdds > 0 ? __fmul_rn(__fdiv_rn(sample, weightAcum), static_cast<float>(numAdds)) : 0.0f;
}

// One thread per (scanline, depth); block = 256 consecutive depths of one scanline.
template <typename RF, typename OUT, bool IS3D>
__global__ void __launch_bounds__(256) dasKernel(DasArgs a) {
    __shared__ float lut[64];
    if (threadIdx.x < 64) lut[threadIdx.x] = a.lut.v[threadIdx.x];
    __syncthreads();
    const uint32_t line = blockIdx.y;
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nD) return;
    const LineDT s = a.lines[line];
    const float d = __ldg(a.depth + r);
    float aDT = apertureDT(d, a.dt, a.c, a.F);
    float invX = 0.0f, invY = 0.0f;
    if (IS3D) {
        aDT = __fmul_rn(aDT, aDT);
        const float sq = __fsqrt_rn(aDT);
        invX = __fdiv_rn(1.0f, fminf(sq, s.maxDistX));
        invY = __fdiv_rn(1.0f, fminf(sq, s.maxDistY));
    } else {
        invX = __fdiv_rn(1.0f, fminf(aDT, s.maxDistX));
    }
    float acc = 0.0f;
    for (int k = 0; k < 4; k++) {
        if (!a.interpTx && k != s.highest) continue;
        if (!((s.activeMask >> k) & 1)) continue;
        const float v = IS3D ? sample3D<RF>(a, s, k, lut, aDT, d, invX, invY) : sample2D<RF>(a, s, k, lut, aDT, d, invX);
        acc = a.interpTx ? __fadd_rn(acc, __fmul_rn(s.txWeight[k], v)) : __fadd_rn(acc, v);
    }
    static_cast<OUT*>(a.out)[line + static_cast<size_t>(r) * a.nRx] = clampCast<OUT>(acc);
}

// ---------------------------------------------------------------------------------------------
// The other sample beamformers of RxBeamformerCuda::performRxBeamforming (Beamformer/RxBeamformerCuda.cu:
// 567-591), run by the same per-(scanline, depth) structure as dasKernel:
//  - DelayAndStdDev (Beamformer/RxSampleBeamformerDelayAndStdDev.h): the DAS value s, then
//    sqrt(sum_e (v_e - s)^2) / sum w * n with v_e = w_e * lerp_e (a second pass over the aperture);
//  - CoherenceFactorDelayAndSum (...CoherenceFactorDelayAndSum.h): (sum u_e)^2 / sum u_e^2 / n * s
//    with u_e = lerp_e unweighted, accumulated in the DAS pass itself (same elements, same delays);
//  - TestSignal (...TestSignal.h): 1000 inside 2 mm cylinders every 6 mm at 30 mm depth, else 0.
// In both reducers an element whose delay falls outside the record keeps the previous element's
// value (the reference's `value` is not reset per element). Every operation is the reference's, in
// its order, as separately rounded IEEE operations.
template <typename RF, int BF>
__device__ __forceinline__ float variant2D(const DasArgs& a, const LineDT& s, int k, const float* lut, float aDT,
                                           float depth, float invMax) {
    const float iD = s.initialDelay[k];
    const RF* tx = static_cast<const RF*>(a.rf) + static_cast<size_t>(s.txIdx[k]) * a.nCh * a.nS;
    const float xz = __fadd_rn(s.x, __fmul_rn(s.dirX, depth));
    const float dy = __fmul_rn(s.dirY, depth);
    const float dy2 = __fmul_rn(dy, dy);
    float sample = 0.0f, weightAcum = 0.0f, value = 0.0f, cs = 0.0f, energy = 0.0f;
    int numAdds = 0;
    for (int pass = 0; pass < (BF == SB_BF_DELAY_AND_STDDEV ? 2 : 1); pass++) {
        const float mean = pass == 0 ? 0.0f
                                     : (numAdds > 0 ? __fmul_rn(__fdiv_rn(sample, weightAcum), static_cast<float>(numAdds)) : 0.0f);
        if (pass == 1) {
            weightAcum = 0.0f;
            numAdds = 0;
            value = 0.0f;
        }
        for (int e = s.firstX[k]; e < s.lastX[k]; e++) {
            const int ch = a.e2c ? __ldg(a.e2c + e) : static_cast<int>(static_cast<uint32_t>(e) % a.nCh);
            if (ch < 0) continue;
            const float xel = __ldg(a.xe + e);
            const float dx = __fsub_rn(xel, s.x);
            if (!(fabsf(dx) <= aDT)) continue;
            const float w = lutGet(lut, __fmul_rn(dx, invMax));
            weightAcum = __fadd_rn(weightAcum, w);
            numAdds++;
            const float ex = __fsub_rn(xel, xz);
            const float dist = __fsqrt_rn(__fadd_rn(__fmul_rn(ex, ex), dy2));
            const float delayf = __fadd_rn(__fadd_rn(iD, __fadd_rn(dist, depth)), a.offset);
            const int32_t delay = static_cast<int32_t>(floorf(delayf));
            const float frac = __fsub_rn(delayf, static_cast<float>(delay));
            const RF* p = tx + static_cast<size_t>(ch) * a.nS;
            if (static_cast<uint32_t>(delay) < a.nS - 1) {
                const float v0 = toFloat(p[delay]), v1 = toFloat(p[delay + 1]);
                const float v = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, frac), v0), __fmul_rn(frac, v1));
                if (pass == 0) sample = __fadd_rn(sample, __fmul_rn(w, v));
                value = BF == SB_BF_DELAY_AND_STDDEV ? __fmul_rn(w, v) : v;
            } else if (static_cast<uint32_t>(delay) < a.nS && frac == 0.0f) {
                const float v0 = toFloat(p[delay]);
                if (pass == 0) sample = __fadd_rn(sample, __fmul_rn(w, v0));
                value = BF == SB_BF_DELAY_AND_STDDEV ? __fmul_rn(w, v0) : v0;
            }
            if (BF == SB_BF_COHERENCE_FACTOR_DAS) {
                cs = __fadd_rn(cs, value);
                energy = __fadd_rn(energy, __fmul_rn(value, value));
            } else if (pass == 1) {
                const float t = __fsub_rn(value, mean);
                cs = __fadd_rn(cs, __fmul_rn(t, t));
            }
        }
    }
    if (numAdds == 0) return 0.0f;
    if (BF == SB_BF_DELAY_AND_STDDEV) return __fmul_rn(__fdiv_rn(__fsqrt_rn(cs), weightAcum), static_cast<float>(numAdds));
    const float das = __fmul_rn(__fdiv_rn(sample, weightAcum), static_cast<float>(numAdds));
    return __fmul_rn(__fdiv_rn(__fdiv_rn(__fmul_rn(cs, cs), energy), static_cast<float>(numAdds)), das);
}

template <typename RF, int BF>
__device__ __forceinline__ float variant3D(const DasArgs& a, const LineDT& s, int k, const float* lut, float aDT2,
                                           float depth, float invX, float invY) {
    const float iD = s.initialDelay[k];
    const RF* tx = static_cast<const RF*>(a.rf) + static_cast<size_t>(s.txIdx[k]) * a.nCh * a.nS;
    const float px = __fadd_rn(s.x, __fmul_rn(s.dirX, depth));
    const float pz = __fadd_rn(s.z, __fmul_rn(s.dirZ, depth));
    const float ay = __fmul_rn(s.dirY, depth);
    const float ay2 = __fmul_rn(ay, ay);
    float sample = 0.0f, weightAcum = 0.0f, value = 0.0f, cs = 0.0f, energy = 0.0f;
    int numAdds = 0;
    for (int pass = 0; pass < (BF == SB_BF_DELAY_AND_STDDEV ? 2 : 1); pass++) {
        const float mean = pass == 0 ? 0.0f
                                     : (numAdds > 0 ? __fmul_rn(__fdiv_rn(sample, weightAcum), static_cast<float>(numAdds)) : 0.0f);
        if (pass == 1) {
            weightAcum = 0.0f;
            numAdds = 0;
            value = 0.0f;
        }
        for (uint32_t ex = s.firstX[k]; ex < s.lastX[k]; ex++) {
            for (uint32_t ey = s.firstY[k]; ey < s.lastY[k]; ey++) {
                const uint32_t e = ex + ey * a.layoutX;
                const int ch = a.e2c ? __ldg(a.e2c + e) : static_cast<int>(e % a.nCh);
                if (ch < 0) continue;
                const float xel = __ldg(a.xe + e), zel = __ldg(a.ye + e);
                const float dx = __fsub_rn(xel, s.x), dz = __fsub_rn(zel, s.z);
                if (!(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dz, dz)) <= aDT2)) continue;
                const float w = __fsqrt_rn(__fmul_rn(lutGet(lut, __fmul_rn(dx, invX)), lutGet(lut, __fmul_rn(dz, invY))));
                weightAcum = __fadd_rn(weightAcum, w);
                numAdds++;
                const float qx = __fsub_rn(xel, px), qz = __fsub_rn(zel, pz);
                const float q = __fadd_rn(__fadd_rn(__fmul_rn(qx, qx), __fmul_rn(qz, qz)), ay2);
                const float delayf = __fadd_rn(__fadd_rn(iD, __fadd_rn(__fsqrt_rn(q), depth)), a.offset);
                const uint32_t delay = static_cast<uint32_t>(floorf(delayf));  // saturates at 0 like the reference
                const float frac = __fsub_rn(delayf, static_cast<float>(delay));
                const RF* p = tx + static_cast<size_t>(ch) * a.nS;
                if (delay < a.nS - 1) {
                    const float v0 = toFloat(p[delay]), v1 = toFloat(p[delay + 1]);
                    const float v = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, frac), v0), __fmul_rn(frac, v1));
                    if (pass == 0) sample = __fadd_rn(sample, __fmul_rn(w, v));
                    value = BF == SB_BF_DELAY_AND_STDDEV ? __fmul_rn(w, v) : v;
                } else if (delay < a.nS && frac == 0.0f) {
                    const float v0 = toFloat(p[delay]);
                    if (pass == 0) sample = __fadd_rn(sample, __fmul_rn(w, v0));
                    value = BF == SB_BF_DELAY_AND_STDDEV ? __fmul_rn(w, v0) : v0;
                }
                if (BF == SB_BF_COHERENCE_FACTOR_DAS) {
                    cs = __fadd_rn(cs, value);
                    energy = __fadd_rn(energy, __fmul_rn(value, value));
                } else if (pass == 1) {
                    const float t = __fsub_rn(value, mean);
                    cs = __fadd_rn(cs, __fmul_rn(t, t));
                }
            }
        }
    }
    if (numAdds == 0) return 0.0f;
    if (BF == SB_BF_DELAY_AND_STDDEV) return __fmul_rn(__fdiv_rn(__fsqrt_rn(cs), weightAcum), static_cast<float>(numAdds));
    const float das = __fmul_rn(__fdiv_rn(sample, weightAcum), static_cast<float>(numAdds));
    return __fmul_rn(__fdiv_rn(__fdiv_rn(__fmul_rn(cs, cs), energy), static_cast<float>(numAdds)), das);
}

// RxSampleBeamformerTestSignal::sampleBeamform2D / 3D: the point back in mm (times dt times c), then
// the distance to each cylinder axis in the plane normal to it.
__device__ __forceinline__ float testSignal(const LineDT& s, float depth, float dt, float c, bool is3D) {
    float px = __fadd_rn(s.x, __fmul_rn(s.dirX, depth));
    float py = __fmul_rn(s.dirY, depth);
    float pz = is3D ? __fadd_rn(s.z, __fmul_rn(s.dirZ, depth)) : __fmul_rn(s.dirZ, depth);
    px = __fmul_rn(__fmul_rn(px, dt), c);
    py = __fmul_rn(__fmul_rn(py, dt), c);
    pz = __fmul_rn(__fmul_rn(pz, dt), c);
    const float dy = __fsub_rn(py, 30.0f);
    const float dy2 = __fmul_rn(dy, dy);
    float sample = 0.0f;
    for (int n = -3; n <= 3; n++) {  // cylinders along the elevation axis
        const float dx = __fsub_rn(px, static_cast<float>(n) * 6.0f);
        if (__fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), dy2), 0.0f)) <= 2.0f) sample = 1000.0f;
    }
    if (is3D) {
        for (int n = -3; n <= 3; n++) {  // cylinders along x
            const float dz = __fsub_rn(pz, static_cast<float>(n) * 6.0f);
            if (__fsqrt_rn(__fadd_rn(__fadd_rn(0.0f, dy2), __fmul_rn(dz, dz))) <= 2.0f) sample = 1000.0f;
        }
    }
    return sample;
}

template <typename RF, typename OUT, bool IS3D, int BF>
__global__ void __launch_bounds__(256) dasVariantKernel(DasArgs a) {
    __shared__ float lut[64];
    if (threadIdx.x < 64) lut[threadIdx.x] = a.lut.v[threadIdx.x];
    __syncthreads();
    const uint32_t line = blockIdx.y;
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nD) return;
    const LineDT s = a.lines[line];
    const float d = __ldg(a.depth + r);
    float aDT = apertureDT(d, a.dt, a.c, a.F);
    float invX = 0.0f, invY = 0.0f;
    if (IS3D) {
        aDT = __fmul_rn(aDT, aDT);
        const float sq = __fsqrt_rn(aDT);
        invX = __fdiv_rn(1.0f, fminf(sq, s.maxDistX));
        invY = __fdiv_rn(1.0f, fminf(sq, s.maxDistY));
    } else {
        invX = __fdiv_rn(1.0f, fminf(aDT, s.maxDistX));
    }
    float acc = 0.0f;
    for (int k = 0; k < 4; k++) {
        if (!a.interpTx && k != s.highest) continue;
        if (!((s.activeMask >> k) & 1)) continue;
        float v;
        if (BF == SB_BF_TEST_SIGNAL) v = testSignal(s, d, a.dt, a.c, IS3D);
        else if (IS3D) v = variant3D<RF, BF>(a, s, k, lut, aDT, d, invX, invY);
        else v = variant2D<RF, BF>(a, s, k, lut, aDT, d, invX);
        acc = a.interpTx ? __fadd_rn(acc, __fmul_rn(s.txWeight[k], v)) : __fadd_rn(acc, v);
    }
    static_cast<OUT*>(a.out)[line + static_cast<size_t>(r) * a.nRx] = clampCast<OUT>(acc);
}

// DelayAndStdDev / CoherenceFactorDelayAndSum, 2D, highest-weight transmit (the common case of
// dasVariantKernel): the scanline's elements (position, offset from the scanline, channel row offset or
// -1 for an unmapped element) sit in a shared-memory table, padded to a multiple of four with unmapped
// entries. Each pass takes elements four at a time: aperture test, weight and running weight sum in
// element order, delays, then the eight gathers together, then the reducer's updates in element order,
// so the arithmetic and its order are those of variant2D (bit-identical).
// Elements outside the aperture change nothing in the reference's loop, so a pass may start at any
// multiple of four at or below the first element inside it and stop after the last (j0, j1: a range
// covering the aperture). DX2 (unsteered scanline): the table's w field holds dx * dx, the product the
// general form computes per depth. OFS: a nonzero sample offset is added. INTERIOR (checked by the
// caller for the warp): every element of [j0, j1) has its delay in [0, nS - 1).
constexpr int kVarUnroll = 4;

template <typename RF, int BF, int PASS, bool DX2, bool OFS, bool INTERIOR>
__device__ __forceinline__ void variantPass(const float4* el, int j0, int j1, const float* lut, const RF* tx, uint32_t nS,
                                            float aDT, float invMax, float xz, float dy2, float depth, float iD,
                                            float offset, float mean, float& sample, float& weightAcum, int& numAdds,
                                            float& value, float& cs, float& energy) {
    for (int j = j0; j < j1; j += kVarUnroll) {
        float w[kVarUnroll], frac[kVarUnroll], v0[kVarUnroll], v1[kVarUnroll];
        int32_t idx[kVarUnroll];
        bool inAp[kVarUnroll], one[kVarUnroll], two[kVarUnroll];
#pragma unroll
        for (int u = 0; u < kVarUnroll; u++) {
            const float4 e = el[j + u];
            const int chOff = __float_as_int(e.z);
            inAp[u] = chOff >= 0 && fabsf(e.y) <= aDT;
            w[u] = 0.0f;
            if (inAp[u]) {
                w[u] = lutGet(lut, __fmul_rn(e.y, invMax));
                weightAcum = __fadd_rn(weightAcum, w[u]);
                numAdds++;
            }
            float ex2;
            if constexpr (DX2) {
                ex2 = e.w;
            } else {
                const float ex = __fsub_rn(e.x, xz);
                ex2 = __fmul_rn(ex, ex);
            }
            const float dist = __fsqrt_rn(__fadd_rn(ex2, dy2));
            const float dl = __fadd_rn(iD, __fadd_rn(dist, depth));
            const float delayf = OFS ? __fadd_rn(dl, offset) : dl;
            const int32_t delay = static_cast<int32_t>(floorf(delayf));
            frac[u] = __fsub_rn(delayf, static_cast<float>(delay));
            if constexpr (INTERIOR) {
                two[u] = inAp[u];
                one[u] = inAp[u];
            } else {
                two[u] = inAp[u] && static_cast<uint32_t>(delay) < nS - 1;
                one[u] = two[u] || (inAp[u] && static_cast<uint32_t>(delay) < nS && frac[u] == 0.0f);
            }
            idx[u] = static_cast<int32_t>(static_cast<uint32_t>(chOff) + static_cast<uint32_t>(delay));  // used when one[u]
        }
#pragma unroll
        for (int u = 0; u < kVarUnroll; u++) {
            v0[u] = one[u] ? toFloat(__ldg(tx + idx[u])) : 0.0f;
            v1[u] = two[u] ? toFloat(__ldg(tx + idx[u] + 1)) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < kVarUnroll; u++) {
            if (one[u]) {
                const float v = two[u] ? __fadd_rn(__fmul_rn(__fsub_rn(1.0f, frac[u]), v0[u]), __fmul_rn(frac[u], v1[u]))
                                       : v0[u];
                if (PASS == 0) sample = __fadd_rn(sample, __fmul_rn(w[u], v));
                value = BF == SB_BF_DELAY_AND_STDDEV ? __fmul_rn(w[u], v) : v;
            }
            if (inAp[u]) {  // an element whose sample lies outside the record reuses the previous value
                if (BF == SB_BF_COHERENCE_FACTOR_DAS) {
                    cs = __fadd_rn(cs, value);
                    energy = __fadd_rn(energy, __fmul_rn(value, value));
                } else if (PASS == 1) {
                    const float t = __fsub_rn(value, mean);
                    cs = __fadd_rn(cs, __fmul_rn(t, t));
                }
            }
        }
    }
}

template <typename RF, typename OUT, int BF>
__global__ void __launch_bounds__(256) dasVariantTableKernel(DasArgs a) {
    __shared__ float lut[64];
    __shared__ float4 el[kMaxApertureElems];
    const int tid = threadIdx.x;
    if (tid < 64) lut[tid] = a.lut.v[tid];
    const uint32_t line = blockIdx.y;
    const LineDT s = a.lines[line];
    const int k = s.highest;
    const bool active = (s.activeMask >> k) & 1;
    const int n = active ? max(static_cast<int>(s.lastX[k]) - static_cast<int>(s.firstX[k]), 0) : 0;  // <= 256 (host)
    const int nPad = (n + kVarUnroll - 1) / kVarUnroll * kVarUnroll;
    const bool dx2 = s.dirX == 0.0f;
    for (int j = tid; j < nPad; j += 256) {
        float4 r = make_float4(0.0f, 0.0f, __int_as_float(-1), 0.0f);
        if (j < n) {
            const int e = s.firstX[k] + j;
            const int ch = a.e2c ? __ldg(a.e2c + e) : static_cast<int>(static_cast<uint32_t>(e) % a.nCh);
            const float xel = __ldg(a.xe + e);
            const float dx = __fsub_rn(xel, s.x);
            r = make_float4(xel, dx, __int_as_float(ch < 0 ? -1 : ch * static_cast<int>(a.nS)), __fmul_rn(dx, dx));
        }
        el[j] = r;
    }
    __syncthreads();
    // ordered by dx (the usual linear probe): the aperture is a contiguous range
    int unsortedMine = 0;
    for (int j = tid + 1; j < n; j += 256)
        if (!(el[j].y >= el[j - 1].y)) unsortedMine = 1;
    const bool sortedX = !__syncthreads_or(unsortedMine);
    const uint32_t r = blockIdx.x * blockDim.x + tid;
    if (r >= a.nD) return;
    float acc = 0.0f;
    if (active) {
        const float d = __ldg(a.depth + r);
        const float aDT = apertureDT(d, a.dt, a.c, a.F);
        const float invMax = __fdiv_rn(1.0f, fminf(aDT, s.maxDistX));
        const RF* tx = static_cast<const RF*>(a.rf) + static_cast<size_t>(s.txIdx[k]) * a.nCh * a.nS;
        const float xz = __fadd_rn(s.x, __fmul_rn(s.dirX, d));
        const float dy = __fmul_rn(s.dirY, d);
        const float dy2 = __fmul_rn(dy, dy);
        const float iD = s.initialDelay[k];
        float sample = 0.0f, weightAcum = 0.0f, value = 0.0f, cs = 0.0f, energy = 0.0f;
        int numAdds = 0;
        // the aperture's range: binary searches on dx, the first element rounded down to a group of four
        int j0 = 0, j1 = nPad;
        if (sortedX) {
            int lo = 0, hi = n;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (el[mid].y < -aDT) lo = mid + 1;
                else hi = mid;
            }
            j0 = lo & ~(kVarUnroll - 1);
            hi = n;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (el[mid].y <= aDT) lo = mid + 1;
                else hi = mid;
            }
            j1 = lo;
        }
        // every delay of the range inside [0, nS - 1)? delays grow with dx^2 (largest at an end of the
        // range) and are at least iD + depth; for unsteered lines without an offset, voted over the warp
        bool interior = false;
        const bool ofs = a.offset != 0.0f;
        if (sortedX && dx2 && !ofs && j1 > j0) {
            const int jl = max(j0, 0), jr = min(j1, n) - 1;
            const float e2 = fmaxf(el[jl].w, el[jr].w);
            const float lo = __fadd_rn(iD, __fadd_rn(__fsqrt_rn(dy2), d));
            const float hi = __fadd_rn(iD, __fadd_rn(__fsqrt_rn(__fadd_rn(e2, dy2)), d));
            interior = lo >= 0.0f && hi < static_cast<float>(a.nS - 1);
        }
        interior = __all_sync(__activemask(), interior);
#define SB_VPASS(PS, DXX, OF, IN, MEAN)                                                                          \
    variantPass<RF, BF, PS, DXX, OF, IN>(el, j0, j1, lut, tx, a.nS, aDT, invMax, xz, dy2, d, iD, a.offset, MEAN,  \
                                         sample, weightAcum, numAdds, value, cs, energy)
#define SB_VPASS_ALL(PS, MEAN)                                                                                   \
    do {                                                                                                         \
        if (interior) SB_VPASS(PS, true, false, true, MEAN);                                                     \
        else if (dx2 && !ofs) SB_VPASS(PS, true, false, false, MEAN);                                            \
        else SB_VPASS(PS, false, true, false, MEAN);                                                             \
    } while (0)
        SB_VPASS_ALL(0, 0.0f);
        float v = 0.0f;
        if (BF == SB_BF_DELAY_AND_STDDEV) {
            const float mean = numAdds > 0 ? __fmul_rn(__fdiv_rn(sample, weightAcum), static_cast<float>(numAdds)) : 0.0f;
            weightAcum = 0.0f;
            numAdds = 0;
            value = 0.0f;
            SB_VPASS_ALL(1, mean);
            if (numAdds > 0) v = __fmul_rn(__fdiv_rn(__fsqrt_rn(cs), weightAcum), static_cast<float>(numAdds));
#undef SB_VPASS_ALL
#undef SB_VPASS
        } else if (numAdds > 0) {
            const float das = __fmul_rn(__fdiv_rn(sample, weightAcum), static_cast<float>(numAdds));
            v = __fmul_rn(__fdiv_rn(__fdiv_rn(__fmul_rn(cs, cs), energy), static_cast<float>(numAdds)), das);
        }
        acc = __fadd_rn(acc, v);
    }
    static_cast<OUT*>(a.out)[line + static_cast<size_t>(r) * a.nRx] = clampCast<OUT>(acc);
}

// 3D delay-and-sum with a per-scanline element table in shared memory (highest-weight transmit).
// The table keeps the reference's summation order (x outer, y inner, RxSampleBeamformerDelayAndSum.h:
// 55-57), each element's position, channel row offset and offsets from the scanline. Once the aperture
// covers maxElementDistance in both directions and every element of the table (depths where
// sqrt(aDT^2) >= maxDistX, maxDistY and aDT^2 >= max(dx^2 + dz^2)), the window weights no longer
// depend on depth: they and their running sum are computed once per scanline in the same order, so
// results stay bit-identical to sample3D. The loop takes elements four at a time: delays and
// weights of all four, then their gathers, then the four additions in element order (an element the
// reference skips adds nothing). The table is padded to a multiple of four (see das3dAccum for the
// padding entries). Six CTAs per SM (40 registers, 56 bytes of spill stores): the
// gathers' latency is hidden by occupancy and the four-element groups (2% faster than five CTAs at 48
// registers on c2); eight-element groups run slower at 64 registers and four CTAs.
constexpr int kMax3DElems = 1024;
constexpr int k3DUnroll = 4;

template <typename RF> __device__ __forceinline__ float ldSample(const RF* p);
template <> __device__ __forceinline__ float ldSample<int16_t>(const int16_t* p) {
    return static_cast<float>(__ldg(p));  // the conversion unit has room here (the ALU pipes do not)
}
template <> __device__ __forceinline__ float ldSample<float>(const float* p) { return __ldg(p); }

// elA[j] = (x, z, deep weight, channel row offset as int bits), elB[j] = (dx, dz, dx^2 + dz^2, 0).
// STRAIGHT (a scanline with dirX = dirZ = 0): the element's offsets from the scanline do not depend on
// depth, so elA[j].x holds dx^2 + dz^2, the same float operations the general form performs per
// depth. OFS: a nonzero sample offset is added (x + 0 is x, so a zero offset is skipped).
// INTERIOR (STRAIGHT only, checked by the caller for the whole warp): every element's delay lies in
// [0, nS - 1), so the record-edge cases drop out. Padding elements then have r2 = 0, deep weight 0 and
// row 0 (an in-range gather whose term is +-0, which leaves the sum unchanged) and no aperture.
template <typename RF, bool DEEP, bool STRAIGHT, bool OFS, bool INTERIOR, bool NEWTON>
__device__ __forceinline__ void das3dAccum(const float4* elA, const float4* elB, const float* lut, int nPad,
                                           const RF* tx, uint32_t nS, float px, float pz, float ay2, float iD,
                                           float d, float offset, float aDT2, float invX, float invY,
                                           float& sample, float& weightAcum, int& numAdds) {
    for (int j = 0; j < nPad; j += k3DUnroll) {
        float w[k3DUnroll], frac[k3DUnroll], v0[k3DUnroll], v1[k3DUnroll];
        int idx[k3DUnroll];
        bool one[k3DUnroll], two[k3DUnroll];
#pragma unroll
        for (int u = 0; u < k3DUnroll; u++) {
            const float4 A = elA[j + u];
            bool inR = true;
            if (DEEP) {
                w[u] = A.z;
            } else {
                const float4 B = elB[j + u];
                inR = B.z <= aDT2;
                w[u] = __fsqrt_rn(__fmul_rn(lutGet(lut, __fmul_rn(B.x, invX)), lutGet(lut, __fmul_rn(B.y, invY))));
                if (inR) {
                    weightAcum = __fadd_rn(weightAcum, w[u]);
                    numAdds++;
                }
            }
            float q;
            if constexpr (STRAIGHT) {
                q = __fadd_rn(A.x, ay2);
            } else {
                const float qx = __fsub_rn(A.x, px), qz = __fsub_rn(A.y, pz);
                q = __fadd_rn(__fadd_rn(__fmul_rn(qx, qx), __fmul_rn(qz, qz)), ay2);
            }
            const float dl = __fadd_rn(iD, __fadd_rn(NEWTON ? sqrtNewton(q) : __fsqrt_rn(q), d));
            const float delayf = OFS ? __fadd_rn(dl, offset) : dl;
            // floor as unsigned, saturating at 0 for negative (and NaN) positions like the reference's
            // conversion; positions >= 2^23 give an index >= 2^23, beyond every record
            const float t = __fadd_rd(fmaxf(delayf, 0.0f), 8388608.0f);
            const uint32_t delay = __float_as_uint(t) - 0x4B000000u;
            frac[u] = __fsub_rn(delayf, __fsub_rn(t, 8388608.0f));
            if constexpr (INTERIOR) {
                two[u] = inR;
                one[u] = inR;
            } else {
                two[u] = inR && delay < nS - 1;
                one[u] = two[u] || (inR && delay < nS && frac[u] == 0.0f);
            }
            idx[u] = static_cast<int>(static_cast<uint32_t>(__float_as_int(A.w)) + delay);  // used when one[u]
        }
#pragma unroll
        for (int u = 0; u < k3DUnroll; u++) {
            v0[u] = one[u] ? ldSample<RF>(tx + idx[u]) : 0.0f;
            v1[u] = two[u] ? ldSample<RF>(tx + idx[u] + 1) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < k3DUnroll; u++) {
            // at the last sample (frac == 0) this is 1 * v0 + 0 * 0 = v0, the reference's single read
            const float v = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, frac[u]), v0[u]), __fmul_rn(frac[u], v1[u]));
            if (one[u]) sample = __fadd_rn(sample, __fmul_rn(w[u], v));
        }
    }
}

template <typename RF, typename OUT>
__global__ void __launch_bounds__(256, 6) das3dTableKernel(DasArgs a, int cap) {
    __shared__ float lut[64];
    __shared__ int nEl, maxR2Bits;
    __shared__ float sumDeep;
    extern __shared__ float4 table3D[];
    float4* elA = table3D;
    float4* elB = table3D + cap;
    const int tid = threadIdx.x;
    if (tid < 64) lut[tid] = a.lut.v[tid];
    if (tid == 0) maxR2Bits = 0;
    __syncthreads();
    const uint32_t line = blockIdx.y;
    const LineDT s = a.lines[line];
    const int k = s.highest;
    const bool active = (s.activeMask >> k) & 1;
    const int nx = active ? max(static_cast<int>(s.lastX[k]) - static_cast<int>(s.firstX[k]), 0) : 0;
    const int ny = active ? max(static_cast<int>(s.lastY[k]) - static_cast<int>(s.firstY[k]), 0) : 0;
    const int n0 = min(nx * ny, cap);  // nx * ny <= maxApertureX * maxApertureY <= cap for every line
    const float invXd = __fdiv_rn(1.0f, s.maxDistX), invYd = __fdiv_rn(1.0f, s.maxDistY);
    const bool mapped = a.e2c != nullptr;
    const bool straight = s.dirX == 0.0f && s.dirZ == 0.0f;
    for (int j = tid; j < n0; j += 256) {
        const uint32_t ex = s.firstX[k] + j / ny, ey = s.firstY[k] + j % ny;
        const uint32_t e = ex + ey * a.layoutX;
        const int ch = mapped ? __ldg(a.e2c + e) : static_cast<int>(e % a.nCh);
        const float xel = __ldg(a.xe + e), zel = __ldg(a.ye + e);
        const float dx = __fsub_rn(xel, s.x), dz = __fsub_rn(zel, s.z);
        const float r2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dz, dz));
        const float wDeep = __fsqrt_rn(__fmul_rn(lutGet(lut, __fmul_rn(dx, invXd)), lutGet(lut, __fmul_rn(dz, invYd))));
        // unmapped elements (ch < 0) are removed below; the row offset keeps them recognisable
        const int chOff = ch < 0 ? -1 : ch * static_cast<int>(a.nS);
        elA[j] = make_float4(straight ? r2 : xel, zel, wDeep, __int_as_float(chOff));
        elB[j] = make_float4(dx, dz, r2, 0.0f);
        if (!mapped && r2 == r2) atomicMax(&maxR2Bits, __float_as_int(r2));
    }
    __syncthreads();
    if (mapped) {
        // channel map: drop unmapped elements in order, then the sums over the remaining ones
        if (tid == 0) {
            int m = 0;
            float sum = 0.0f, mr = 0.0f;
            for (int j = 0; j < n0; j++) {
                const float4 A = elA[j], B = elB[j];
                if (__float_as_int(A.w) < 0) continue;
                elA[m] = A;
                elB[m] = B;
                m++;
                sum = __fadd_rn(sum, A.z);
                mr = fmaxf(mr, B.z);
            }
            nEl = m;
            sumDeep = sum;
            maxR2Bits = __float_as_int(mr);
        }
        __syncthreads();
    }
    const int n = mapped ? nEl : n0;
    const int nPad = (n + k3DUnroll - 1) / k3DUnroll * k3DUnroll;  // <= cap (cap is a multiple of 4)
    for (int j = n + tid; j < nPad; j += 256) {
        // general form: an element at infinity (delay beyond every record); unsteered: r2 = 0, deep
        // weight 0, row 0 (see das3dAccum)
        elA[j] = make_float4(straight ? 0.0f : INFINITY, 0.0f, 0.0f, __int_as_float(0));
        elB[j] = make_float4(0.0f, 0.0f, INFINITY, 0.0f);
    }
    __syncthreads();
    if (!mapped && tid == 0) {
        // the deep weights' running sum in element order, overlapped with the other warps' loops
        float sum = 0.0f;
        for (int j = 0; j < n; j++) sum = __fadd_rn(sum, elA[j].z);
        sumDeep = sum;
    }
    const float maxR2 = __int_as_float(maxR2Bits);
    const uint32_t r = blockIdx.x * blockDim.x + tid;
    const bool inRange = r < a.nD;
    float sample = 0.0f, weightAcum = 0.0f;
    int numAdds = 0;
    bool deep = false;
    if (active && inRange) {
        const float d = __ldg(a.depth + r);
        const float aDT = apertureDT(d, a.dt, a.c, a.F);
        const float aDT2 = __fmul_rn(aDT, aDT);
        const float sq = __fsqrt_rn(aDT2);
        const float invX = __fdiv_rn(1.0f, fminf(sq, s.maxDistX));
        const float invY = __fdiv_rn(1.0f, fminf(sq, s.maxDistY));
        deep = sq >= s.maxDistX && sq >= s.maxDistY && aDT2 >= maxR2;
        const RF* tx = static_cast<const RF*>(a.rf) + static_cast<size_t>(s.txIdx[k]) * a.nCh * a.nS;
        const float px = __fadd_rn(s.x, __fmul_rn(s.dirX, d));
        const float pz = __fadd_rn(s.z, __fmul_rn(s.dirZ, d));
        const float ay = __fmul_rn(s.dirY, d);
        const float ay2 = __fmul_rn(ay, ay);
#define SB_3D(DP, ST, OF, IN, NW)                                                                              \
    das3dAccum<RF, DP, ST, OF, IN, NW>(elA, elB, lut, nPad, tx, a.nS, px, pz, ay2, s.initialDelay[k], d, a.offset, \
                                       aDT2, invX, invY, sample, weightAcum, numAdds)
        const bool ofs = a.offset != 0.0f;
        if (straight && !ofs) {
            // delays grow with q = r2 + ay2 (monotone float operations), so the element with the largest
            // r2 and q = ay2 bound every delay of this depth (the padding's r2 = 0 included)
            const float iD = s.initialDelay[k];
            const float lo = __fadd_rn(iD, __fadd_rn(__fsqrt_rn(ay2), d));
            const float hi = __fadd_rn(iD, __fadd_rn(__fsqrt_rn(__fadd_rn(maxR2, ay2)), d));
            // every q = r2 + ay2 of this depth (r2 >= 0 from the table, sums of non-negative floats are
            // monotone) lies in [ay2, maxR2 + ay2]: inside [2^-102, FLT_MAX], where the Newton square root
            // is the IEEE one, unless ay2 is 0 or tiny (the first depths) or the sum overflows. The
            // interior loop takes the Newton root; a warp with any other depth takes the general loop.
            const bool newton = ay2 >= 0x1p-102f && __fadd_rn(maxR2, ay2) <= FLT_MAX;
            const bool interior =
                __all_sync(__activemask(), lo >= 0.0f && hi < static_cast<float>(a.nS - 1) && newton);
            if (interior) {
                if (deep) SB_3D(true, true, false, true, true);
                else SB_3D(false, true, false, true, true);
            } else {
                if (deep) SB_3D(true, true, false, false, false);
                else SB_3D(false, true, false, false, false);
            }
        } else if (deep) {
            SB_3D(true, false, true, false, false);
        } else {
            SB_3D(false, false, true, false, false);
        }
#undef SB_3D
    }
    __syncthreads();  // sumDeep
    if (!inRange) return;
    float acc = 0.0f;
    if (active) {
        if (deep) {
            weightAcum = sumDeep;
            numAdds = n;
        }
        const float v = numAdds > 0 ? __fmul_rn(__fdiv_rn(sample, weightAcum), static_cast<float>(numAdds)) : 0.0f;
        acc = __fadd_rn(acc, v);
    }
    static_cast<OUT*>(a.out)[line + static_cast<size_t>(r) * a.nRx] = clampCast<OUT>(acc);
}

// RawDelay (Beamformer/RawDelay.cu:221-312 with the kernel :406-468): highest-weight transmit only,
// out [line][local element][depth], normalised by numAdds / sum(w); unused slots written as 0.
template <typename RF, typename OUT>
__global__ void __launch_bounds__(256) rawDelayKernel(DasArgs a) {
    __shared__ float lut[64];
    if (threadIdx.x < 64) lut[threadIdx.x] = a.lut.v[threadIdx.x];
    __syncthreads();
    const uint32_t line = blockIdx.y;
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nD) return;
    const LineDT s = a.lines[line];
    OUT* out = static_cast<OUT*>(a.out) + static_cast<size_t>(line) * a.nCh * a.nD + r;
    const int k = s.highest;
    int written = 0;
    if ((s.activeMask >> k) & 1) {
        const float d = __ldg(a.depth + r);
        const float aDT = apertureDT(d, a.dt, a.c, a.F);
        const float invMax = __fdiv_rn(1.0f, fminf(aDT, s.maxDistX));
        float weightAcum = 0.0f;
        int numAdds = 0;
        for (int e = s.firstX[k]; e < s.lastX[k]; e++) {
            const float dx = __fsub_rn(__ldg(a.xe + e), s.x);
            if (fabsf(dx) <= aDT) {
                weightAcum = __fadd_rn(weightAcum, lutGet(lut, __fmul_rn(dx, invMax)));
                numAdds++;
            }
        }
        const float scale = numAdds > 0 ? __fmul_rn(__fdiv_rn(1.0f, weightAcum), static_cast<float>(numAdds)) : 1.0f;
        const RF* tx = static_cast<const RF*>(a.rf) + static_cast<size_t>(s.txIdx[k]) * a.nCh * a.nS;
        const float xz = __fadd_rn(s.x, __fmul_rn(s.dirX, d));
        const float dy = __fmul_rn(s.dirY, d);
        const float dy2 = __fmul_rn(dy, dy);
        for (int e = s.firstX[k]; e < s.lastX[k] && written < static_cast<int>(a.nCh); e++, written++) {
            float sample = 0.0f;
            const float xel = __ldg(a.xe + e);
            const float dx = __fsub_rn(xel, s.x);
            if (fabsf(dx) <= aDT) {
                const float w = lutGet(lut, __fmul_rn(dx, invMax));
                const float ex = __fsub_rn(xel, xz);
                const float delayf = __fadd_rn(s.initialDelay[k], __fadd_rn(__fsqrt_rn(__fadd_rn(__fmul_rn(ex, ex), dy2)), d));
                const int32_t delay = static_cast<int32_t>(floorf(delayf));
                const float frac = __fsub_rn(delayf, static_cast<float>(delay));
                const RF* p = tx + static_cast<size_t>(static_cast<uint32_t>(e) % a.nCh) * a.nS;
                if (static_cast<uint32_t>(delay) < a.nS - 1) {
                    sample = __fmul_rn(w, __fadd_rn(__fmul_rn(__fsub_rn(1.0f, frac), toFloat(p[delay])),
                                                    __fmul_rn(frac, toFloat(p[delay + 1]))));
                } else if (static_cast<uint32_t>(delay) < a.nS && frac == 0.0f) {
                    sample = __fmul_rn(w, toFloat(p[delay]));
                }
            }
            out[static_cast<size_t>(written) * a.nD] = clampCast<OUT>(__fmul_rn(sample, scale));
        }
    }
    for (int j = written; j < static_cast<int>(a.nCh); j++) out[static_cast<size_t>(j) * a.nD] = clampCast<OUT>(0.0f);
}

// RawDelay with the scanline's elements in a shared-memory table (apertures up to
// kMaxApertureElems elements): the weight sum over the whole aperture first, then the written slots
// four elements at a time (delays and weights of all four, their gathers together, then the four
// stores), in rawDelayKernel's arithmetic (bit-identical).
template <typename RF, typename OUT>
__global__ void __launch_bounds__(256) rawDelayTableKernel(DasArgs a) {
    __shared__ float lut[64];
    __shared__ float4 el[kMaxApertureElems];  // (x, dx, channel row offset as int bits, 0)
    const int tid = threadIdx.x;
    if (tid < 64) lut[tid] = a.lut.v[tid];
    const uint32_t line = blockIdx.y;
    const LineDT s = a.lines[line];
    const int k = s.highest;
    const bool active = (s.activeMask >> k) & 1;
    const int n = active ? max(static_cast<int>(s.lastX[k]) - static_cast<int>(s.firstX[k]), 0) : 0;  // <= 256 (host)
    const int nw = min(n, static_cast<int>(a.nCh));                          // slots written
    const int nPad = (nw + kVarUnroll - 1) / kVarUnroll * kVarUnroll;        // <= 256
    for (int j = tid; j < max(n, nPad); j += 256) {
        float4 r = make_float4(0.0f, INFINITY, __int_as_float(0), 0.0f);     // padding: outside every aperture
        if (j < n) {
            const int e = s.firstX[k] + j;
            const float xel = __ldg(a.xe + e);
            r = make_float4(xel, __fsub_rn(xel, s.x), __int_as_float(static_cast<int>((static_cast<uint32_t>(e) % a.nCh) * a.nS)), 0.0f);
        }
        el[j] = r;
    }
    __syncthreads();
    const uint32_t r = blockIdx.x * blockDim.x + tid;
    if (r >= a.nD) return;
    OUT* out = static_cast<OUT*>(a.out) + static_cast<size_t>(line) * a.nCh * a.nD + r;
    int written = 0;
    if (active) {
        const float d = __ldg(a.depth + r);
        const float aDT = apertureDT(d, a.dt, a.c, a.F);
        const float invMax = __fdiv_rn(1.0f, fminf(aDT, s.maxDistX));
        float weightAcum = 0.0f;
        int numAdds = 0;
        for (int j = 0; j < n; j++) {
            const float dx = el[j].y;
            if (fabsf(dx) <= aDT) {
                weightAcum = __fadd_rn(weightAcum, lutGet(lut, __fmul_rn(dx, invMax)));
                numAdds++;
            }
        }
        const float scale = numAdds > 0 ? __fmul_rn(__fdiv_rn(1.0f, weightAcum), static_cast<float>(numAdds)) : 1.0f;
        const RF* tx = static_cast<const RF*>(a.rf) + static_cast<size_t>(s.txIdx[k]) * a.nCh * a.nS;
        const float xz = __fadd_rn(s.x, __fmul_rn(s.dirX, d));
        const float dy = __fmul_rn(s.dirY, d);
        const float dy2 = __fmul_rn(dy, dy);
        const float iD = s.initialDelay[k];
        for (int j0 = 0; j0 < nPad; j0 += kVarUnroll) {
            float w[kVarUnroll], frac[kVarUnroll], v0[kVarUnroll], v1[kVarUnroll];
            int32_t idx[kVarUnroll];
            bool one[kVarUnroll], two[kVarUnroll];
#pragma unroll
            for (int u = 0; u < kVarUnroll; u++) {
                const float4 e = el[j0 + u];
                const bool inAp = fabsf(e.y) <= aDT;
                w[u] = inAp ? lutGet(lut, __fmul_rn(e.y, invMax)) : 0.0f;
                const float ex = __fsub_rn(e.x, xz);
                const float delayf = __fadd_rn(iD, __fadd_rn(__fsqrt_rn(__fadd_rn(__fmul_rn(ex, ex), dy2)), d));
                const int32_t delay = static_cast<int32_t>(floorf(delayf));
                frac[u] = __fsub_rn(delayf, static_cast<float>(delay));
                two[u] = inAp && static_cast<uint32_t>(delay) < a.nS - 1;
                one[u] = two[u] || (inAp && static_cast<uint32_t>(delay) < a.nS && frac[u] == 0.0f);
                idx[u] = static_cast<int32_t>(static_cast<uint32_t>(__float_as_int(e.z)) + static_cast<uint32_t>(delay));
            }
#pragma unroll
            for (int u = 0; u < kVarUnroll; u++) {
                v0[u] = one[u] ? toFloat(__ldg(tx + idx[u])) : 0.0f;
                v1[u] = two[u] ? toFloat(__ldg(tx + idx[u] + 1)) : 0.0f;
            }
#pragma unroll
            for (int u = 0; u < kVarUnroll; u++) {
                float sample = 0.0f;
                if (two[u])
                    sample = __fmul_rn(w[u], __fadd_rn(__fmul_rn(__fsub_rn(1.0f, frac[u]), v0[u]), __fmul_rn(frac[u], v1[u])));
                else if (one[u])
                    sample = __fmul_rn(w[u], v0[u]);
                if (j0 + u < nw) out[static_cast<size_t>(j0 + u) * a.nD] = clampCast<OUT>(__fmul_rn(sample, scale));
            }
        }
        written = nw;
    }
    for (int j = written; j < static_cast<int>(a.nCh); j++) out[static_cast<size_t>(j) * a.nD] = clampCast<OUT>(0.0f);
}

// Staged per-frame 2D DAS: one CTA per (scanline, chunksPerCta chunks of NT depths).
template <typename RF, typename OUT, int NT>
__global__ void __launch_bounds__(NT) dasStagedKernel(FrameDesc f, WindowLut lut, void* out, uint32_t maxW,
                                                      uint32_t chunksPerCta, int* errFlag) {
    extern __shared__ __align__(128) unsigned char smraw[];
    CtaState& st = *reinterpret_cast<CtaState*>(smraw);
    RF* smemRF = reinterpret_cast<RF*>(smraw + ((sizeof(CtaState) + 127) & ~size_t(127)));
    const int tid = threadIdx.x;
    const uint32_t line = blockIdx.y;
    if (tid < 64) st.lut[tid] = lut.v[tid];
    if (tid == 0) {
        mbarInit(&st.bar[0], 1);
        mbarInit(&st.bar[1], 1);
        mbarInitFence();
        st.phase[0] = st.phase[1] = 0;
    }
    __syncthreads();
    const LineK s = reduceLine(f.lines[line]);
    OUT* o = static_cast<OUT*>(out);
    const bool ok = setupLine<NT>(st, f, s);
    const bool useOffset = f.offset != 0.0f;
    for (uint32_t c = 0; c < chunksPerCta; c++) {
        const uint32_t r0 = (blockIdx.x * chunksPerCta + c) * NT;
        if (r0 >= f.nD) break;
        const uint32_t r = r0 + tid;
        if (!ok) {  // no active transmit: the reference writes clampCast(0)
            if (r < f.nD) o[line + static_cast<size_t>(r) * f.nRx] = clampCast<OUT>(0.0f);
            continue;
        }
        planChunk<RF, NT>(st, smemRF, 0, f, s, r0, maxW, maxW, useOffset);
        if (!waitChunk(st, 0)) {
            if (tid == 0) atomicExch(errFlag, 1);
            return;
        }
        if (r < f.nD) o[line + static_cast<size_t>(r) * f.nRx] = clampCast<OUT>(dasDepth<RF>(st, smemRF, 0, maxW, f, s, r, useOffset));
        __syncthreads();
    }
}

int checkWindow(int windowType, float windowParameter) {
    SB_REQUIRE(windowType >= 0 && windowType <= 3, "window type %d not in [0,3]", windowType);
    SB_REQUIRE(!(windowType == SB_WINDOW_GAUSS && windowParameter == 0.0f), "Gauss window needs a non-zero parameter");
    return SB_OK;
}

int fillArgs(sb_das_plan* p, DasArgs& a, const void* rf, void* out, double fNumber, double c, int windowType,
             float windowParameter, int interpTx, int32_t offset, cudaStream_t st) {
    SB_REQUIRE(fNumber > 0.0, "f-number must be > 0");
    SB_REQUIRE(c > 0.0, "speed of sound must be > 0");
    int e = checkWindow(windowType, windowParameter);
    if (e != SB_OK) return e;
    e = ensureDtSpace(p, c, st);
    if (e != SB_OK) return e;
    a.rf = rf;
    a.out = out;
    a.xe = p->dXe;
    a.ye = p->dYe;
    a.depth = p->dDepth;
    a.lines = p->dLines;
    a.e2c = p->dE2C;
    a.apod = nullptr;
    a.nE = p->numElements;
    a.layoutX = p->layoutX;
    a.nCh = p->numChannels;
    a.nS = p->numSamples;
    a.nTx = p->numTx;
    a.nRx = p->numRx;
    a.nD = p->numDepths;
    a.c = static_cast<float>(c);
    a.dt = static_cast<float>(1.0 / p->fs);
    a.F = static_cast<float>(fNumber);
    a.offset = static_cast<float>(offset);
    a.interpTx = interpTx ? 1 : 0;
    a.lut = makeLut(windowType, windowParameter);
    return SB_OK;
}

constexpr int kStagedThreads = 256;
constexpr size_t kStagedSmemBudget = 72 * 1024;

uint32_t stagedMaxW(uint32_t nCh, size_t rfSize) {
    const size_t state = (sizeof(CtaState) + 127) & ~size_t(127);
    if (kStagedSmemBudget <= state) return 0;
    size_t w = (kStagedSmemBudget - state) / (nCh * rfSize);
    w &= ~size_t(7);
    return static_cast<uint32_t>(std::min<size_t>(w, 4096));
}

FrameDesc frameOf(const sb_das_plan* p, const DasArgs& a) {
    FrameDesc f;
    f.rf = a.rf;
    f.lines = a.lines;
    f.xe = a.xe;
    f.depth = a.depth;
    f.e2c = a.e2c;
    f.nCh = a.nCh;
    f.nS = a.nS;
    f.nTx = a.nTx;
    f.nRx = a.nRx;
    f.nD = a.nD;
    f.c = a.c;
    f.dt = a.dt;
    f.F = a.F;
    f.offset = a.offset;
    return f;
}

// Single-frame path (2D, int16 channel data, float image, highest-weight transmit): the frame-pack
// kernel with one frame, in the reference's exact arithmetic (MODE 1). Items are (scanline, 128-depth
// segment), deepest segments first (they hold the most aperture elements), so a single frame still
// spreads over every SM.
constexpr int kSinglePackThreads = 128;

int launchSinglePackKernel(const DasArgs& a, const PackItem* items, uint32_t nItems, uint32_t* counter,
                           cudaStream_t st);

int launchSinglePack(sb_das_plan* p, const DasArgs& a, cudaStream_t st) {
    if (!p->packItems) {
        std::vector<PackItem> items;
        const uint32_t nSeg = (p->numDepths + kSinglePackRows - 1) / kSinglePackRows;
        for (uint32_t it = 0; it < nSeg * p->numRx; it++) items.push_back(singleItem(it, p->numRx, p->numDepths));
        void* di = nullptr;
        uint32_t* dc = nullptr;
        cudaError_t e = cudaMalloc(&di, items.size() * sizeof(PackItem));
        if (e == cudaSuccess) e = cudaMalloc(&dc, sizeof(uint32_t));
        if (e == cudaSuccess) e = cudaMemcpy(di, items.data(), items.size() * sizeof(PackItem), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaFree(di);
            cudaFree(dc);
            return cudaFail(e, "sb_das_run: work items");
        }
        p->packItems = di;
        p->packCounter = dc;
        p->packItemCount = static_cast<uint32_t>(items.size());
    }
    return launchSinglePackKernel(a, static_cast<const PackItem*>(p->packItems), p->packItemCount, p->packCounter, st);
}

// The single-frame pack kernel over `nItems` items: from the table `items`, or, when it is null, the
// items singleItem() derives from the item index. `counter` is the work counter (reset here).
int launchSinglePackKernel(const DasArgs& a, const PackItem* items, uint32_t nItems, uint32_t* counter,
                           cudaStream_t st) {
    PackArgs pa;
    std::memset(&pa, 0, sizeof(pa));
    pa.items = items;
    pa.nItems = nItems;
    pa.counter = counter;
    pa.dec = 1;
    pa.lut = a.lut;
    PackDev& d = pa.single;
    d.lines = a.lines;
    d.xe = a.xe;
    d.depth = a.depth;
    d.e2c = a.e2c;
    d.nCh = a.nCh;
    d.nS = a.nS;
    d.nRx = a.nRx;
    d.nD = a.nD;
    d.c = a.c;
    d.dt = a.dt;
    d.F = a.F;
    d.offset = a.offset;
    d.nf = 1;
    d.rf[0] = static_cast<const int16_t*>(a.rf);
    d.rfOut[0] = static_cast<float*>(a.out);
    SB_CUDA(cudaMemsetAsync(counter, 0, sizeof(uint32_t), st));
    const unsigned grid = static_cast<unsigned>(std::min<size_t>(static_cast<size_t>(smCount()) * 8, (nItems + 1)));
    batchPackKernel<1, kSinglePackThreads, 8, 1><<<grid, kSinglePackThreads, 0, st>>>(pa);
    SB_CHECK_LAUNCH("batchPackKernel");
    return SB_OK;
}

int launchStaged(const sb_das_plan* p, const DasArgs& a, int rfDt, int outDt, cudaStream_t st) {
    const size_t rfSize = rfDt == SB_INT16 ? 2 : 4;
    const uint32_t maxW = stagedMaxW(p->numChannels, rfSize);
    const size_t shm = ((sizeof(CtaState) + 127) & ~size_t(127)) + static_cast<size_t>(maxW) * p->numChannels * rfSize;
    const uint32_t nChunks = (p->numDepths + kStagedThreads - 1) / kStagedThreads;
    // enough CTAs to fill the GPU (about 3 resident per SM), fewer setups per scanline otherwise
    uint32_t per = 1;
    while (per < nChunks && static_cast<size_t>(p->numRx) * ((nChunks + per * 2 - 1) / (per * 2)) >= static_cast<size_t>(smCount()) * 6)
        per *= 2;
    dim3 grid((nChunks + per - 1) / per, p->numRx);
    FrameDesc f = frameOf(p, a);
    int* err = deviceErrorFlag();
    if (!err) return fail(SB_ERR_NO_MEMORY, "error flag allocation failed");
#define SB_STAGED(RFT, OUTT)                                                                                           \
    do {                                                                                                               \
        auto kern = dasStagedKernel<RFT, OUTT, kStagedThreads>;                                                        \
        SB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(shm)));       \
        kern<<<grid, kStagedThreads, shm, st>>>(f, a.lut, a.out, maxW, per, err);                                      \
    } while (0)
    if (rfDt == SB_INT16 && outDt == SB_FLOAT32) SB_STAGED(int16_t, float);
    else if (rfDt == SB_INT16) SB_STAGED(int16_t, int16_t);
    else if (outDt == SB_FLOAT32) SB_STAGED(float, float);
    else SB_STAGED(float, int16_t);
#undef SB_STAGED
    SB_CHECK_LAUNCH("dasStagedKernel");
    return SB_OK;
}

}  // namespace

int ensureDtSpace(sb_das_plan* p, double c, cudaStream_t st) {
    if (p->cachedC == c) return SB_OK;
    const double dt = 1.0 / p->fs;
    const double factor = 1 / 1.0 / (c * dt);
    const double factorTime = 1 / 1.0 / dt;
    uint32_t n = std::max(std::max(p->numElements, p->numDepths), p->numRx);
    dtConvertKernel<<<(n + 255) / 256, 256, 0, st>>>(p->dXeMM, p->dYeMM, p->numElements, p->dDepthMM, p->numDepths,
                                                     p->dLinesMM, p->numRx, factor, factorTime, p->dXe, p->dYe,
                                                     p->dDepth, p->dLines);
    SB_CHECK_LAUNCH("dtConvertKernel");
    p->cachedC = c;
    return SB_OK;
}

}  // namespace sb

using namespace sb;

extern "C" {

int sb_das_plan_create(const sb_geometry* g, sb_das_plan** out) {
    SB_REQUIRE(g && out, "sb_das_plan_create: null argument");
    *out = nullptr;
    SB_REQUIRE(g->num_elements > 0 && g->num_channels > 0 && g->num_samples > 1 && g->num_tx > 0 && g->num_depths > 0,
               "sb_das_plan_create: empty geometry");
    SB_REQUIRE(g->num_rx == g->rx_layout[0] * g->rx_layout[1] && g->num_rx > 0, "num_rx != rx_layout product");
    SB_REQUIRE(g->element_layout[0] * g->element_layout[1] == g->num_elements, "element_layout != num_elements");
    SB_REQUIRE(g->sampling_frequency_hz > 0, "sampling frequency must be > 0");
    SB_REQUIRE(g->element_x_mm && g->element_y_mm && g->depths_mm && g->scanlines, "null geometry array");
    bool is3D = g->rx_layout[0] > 1 && g->rx_layout[1] > 1;
    int32_t maxAx = 0, maxAy = 0;
    for (uint32_t i = 0; i < g->num_rx; i++) {
        const sb_scanline_rx& s = g->scanlines[i];
        for (int k = 0; k < 4; k++) {
            if (!(s.tx_weights[k] > 0.0)) continue;
            SB_REQUIRE(s.tx[k].tx_scanline_idx < g->num_tx, "scanline %u: transmit index %u >= num_tx %u", i,
                       s.tx[k].tx_scanline_idx, g->num_tx);
            SB_REQUIRE(s.tx[k].last_active_element[0] <= g->element_layout[0] &&
                           s.tx[k].last_active_element[1] <= g->element_layout[1],
                       "scanline %u: aperture beyond the element layout", i);
            maxAx = std::max(maxAx, static_cast<int32_t>(s.tx[k].last_active_element[0]) - s.tx[k].first_active_element[0]);
            maxAy = std::max(maxAy, static_cast<int32_t>(s.tx[k].last_active_element[1]) - s.tx[k].first_active_element[1]);
        }
    }
    if (g->element_to_channel)
        for (uint32_t e = 0; e < g->num_elements; e++)
            SB_REQUIRE(g->element_to_channel[e] < static_cast<int32_t>(g->num_channels), "element %u maps to channel %d",
                       e, g->element_to_channel[e]);
    sb_das_plan* p = new sb_das_plan();
    p->numElements = g->num_elements;
    p->layoutX = g->element_layout[0];
    p->layoutY = g->element_layout[1];
    p->numChannels = g->num_channels;
    p->numSamples = g->num_samples;
    p->numTx = g->num_tx;
    p->numRx = g->num_rx;
    p->rxLayoutX = g->rx_layout[0];
    p->rxLayoutY = g->rx_layout[1];
    p->numDepths = g->num_depths;
    p->fs = g->sampling_frequency_hz;
    p->is3D = is3D;
    p->hasChannelMap = g->element_to_channel != nullptr;
    p->maxApertureX = maxAx;
    p->maxApertureY = maxAy;
    p->hLines = new std::vector<sb_scanline_rx>(g->scanlines, g->scanlines + g->num_rx);
    p->hXeMM = new std::vector<float>(g->element_x_mm, g->element_x_mm + g->num_elements);
    p->hDepthMM = new std::vector<float>(g->depths_mm, g->depths_mm + g->num_depths);
    auto cleanup = [&](int code) {
        sb_das_plan_destroy(p);
        return code;
    };
    size_t nE = g->num_elements, nD = g->num_depths, nRx = g->num_rx;
    cudaError_t e = cudaSuccess;
    e = cudaMalloc(&p->dXeMM, nE * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&p->dYeMM, nE * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&p->dDepthMM, nD * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&p->dLinesMM, nRx * sizeof(sb_scanline_rx));
    if (e == cudaSuccess) e = cudaMalloc(&p->dXe, nE * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&p->dYe, nE * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&p->dDepth, nD * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&p->dLines, nRx * sizeof(LineDT));
    if (e == cudaSuccess && g->element_to_channel) e = cudaMalloc(&p->dE2C, nE * sizeof(int32_t));
    if (e != cudaSuccess) return cleanup(cudaFail(e, "sb_das_plan_create: cudaMalloc"));
    e = cudaMemcpy(p->dXeMM, g->element_x_mm, nE * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->dYeMM, g->element_y_mm, nE * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->dDepthMM, g->depths_mm, nD * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->dLinesMM, g->scanlines, nRx * sizeof(sb_scanline_rx), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && g->element_to_channel)
        e = cudaMemcpy(p->dE2C, g->element_to_channel, nE * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cleanup(cudaFail(e, "sb_das_plan_create: cudaMemcpy"));
    *out = p;
    return SB_OK;
}

int sb_das_plan_destroy(sb_das_plan* p) {
    if (!p) return SB_OK;
    cudaFree(p->dXeMM);
    cudaFree(p->dYeMM);
    cudaFree(p->dDepthMM);
    cudaFree(p->dLinesMM);
    cudaFree(p->dE2C);
    cudaFree(p->dXe);
    cudaFree(p->dYe);
    cudaFree(p->dDepth);
    cudaFree(p->dLines);
    cudaFree(p->adjScratch);
    cudaFree(p->packItems);
    cudaFree(p->packCounter);
    delete p->hLines;
    delete p->hXeMM;
    delete p->hDepthMM;
    delete p;
    return SB_OK;
}

int sb_das_run(const sb_das_plan* plan, const void* rf, int rf_dtype, void* out, int out_dtype, double f_number,
               double speed_of_sound_mm_s, int window_type, float window_parameter, int interpolate_transmits,
               int32_t additional_offset, sb_stream stream) {
    SB_REQUIRE(plan && rf && out, "sb_das_run: null argument");
    SB_REQUIRE(rf_dtype == SB_INT16 || rf_dtype == SB_FLOAT32, "sb_das_run: rf dtype %d unsupported", rf_dtype);
    SB_REQUIRE(out_dtype == SB_FLOAT32 || out_dtype == SB_INT16, "sb_das_run: out dtype %d unsupported", out_dtype);
    sb_das_plan* p = const_cast<sb_das_plan*>(plan);
    cudaStream_t st = S(stream);
    DasArgs a;
    int err = fillArgs(p, a, rf, out, f_number, speed_of_sound_mm_s, window_type, window_parameter,
                       interpolate_transmits, additional_offset, st);
    if (err != SB_OK) return err;
    const size_t rfSize = rf_dtype == SB_INT16 ? 2 : 4;
    const bool staged = !p->is3D && !interpolate_transmits && p->maxApertureX <= kMaxApertureElems &&
                        (p->numSamples * rfSize) % 16 == 0 && (reinterpret_cast<uintptr_t>(rf) % 16) == 0 &&
                        stagedMaxW(p->numChannels, rfSize) >= 64;
    // the frame-pack kernel with one frame (exact arithmetic) where its conditions hold
    if (!p->is3D && !interpolate_transmits && rf_dtype == SB_INT16 && out_dtype == SB_FLOAT32 &&
        p->maxApertureX <= kMaxApertureElems && p->numSamples >= 2)
        return launchSinglePack(p, a, st);
    if (staged) return launchStaged(p, a, rf_dtype, out_dtype, st);
    dim3 grid((p->numDepths + 255) / 256, p->numRx);
    const bool table3D = p->is3D && !interpolate_transmits &&
                         static_cast<int64_t>(p->maxApertureX) * p->maxApertureY <= kMax3DElems &&
                         static_cast<int64_t>(p->numChannels) * p->numSamples <= INT32_MAX;
    const int cap3D = table3D ? (p->maxApertureX * p->maxApertureY + k3DUnroll - 1) / k3DUnroll * k3DUnroll : 0;
    const size_t smem3D = 2 * sizeof(float4) * static_cast<size_t>(cap3D);  // <= 32 KB: no opt-in needed
#define SB_DAS_LAUNCH(RFT, OUTT)                                                        \
    do {                                                                                \
        if (table3D) das3dTableKernel<RFT, OUTT><<<grid, 256, smem3D, st>>>(a, cap3D); \
        else if (p->is3D) dasKernel<RFT, OUTT, true><<<grid, 256, 0, st>>>(a);         \
        else dasKernel<RFT, OUTT, false><<<grid, 256, 0, st>>>(a);                     \
    } while (0)
    if (rf_dtype == SB_INT16 && out_dtype == SB_FLOAT32) SB_DAS_LAUNCH(int16_t, float);
    else if (rf_dtype == SB_INT16) SB_DAS_LAUNCH(int16_t, int16_t);
    else if (out_dtype == SB_FLOAT32) SB_DAS_LAUNCH(float, float);
    else SB_DAS_LAUNCH(float, int16_t);
#undef SB_DAS_LAUNCH
    SB_CHECK_LAUNCH("dasKernel");
    return SB_OK;
}

int sb_das_run_beamformer(const sb_das_plan* plan, int sample_beamformer, const void* rf, int rf_dtype, void* out,
                          int out_dtype, double f_number, double speed_of_sound_mm_s, int window_type,
                          float window_parameter, int interpolate_transmits, int32_t additional_offset, sb_stream stream) {
    SB_REQUIRE(sample_beamformer >= SB_BF_DELAY_AND_SUM && sample_beamformer <= SB_BF_TEST_SIGNAL,
               "sb_das_run_beamformer: sample beamformer %d not in [0, 3]", sample_beamformer);
    if (sample_beamformer == SB_BF_DELAY_AND_SUM)
        return sb_das_run(plan, rf, rf_dtype, out, out_dtype, f_number, speed_of_sound_mm_s, window_type,
                          window_parameter, interpolate_transmits, additional_offset, stream);
    SB_REQUIRE(plan && rf && out, "sb_das_run_beamformer: null argument");
    SB_REQUIRE(rf_dtype == SB_INT16 || rf_dtype == SB_FLOAT32, "sb_das_run_beamformer: rf dtype %d unsupported", rf_dtype);
    SB_REQUIRE(out_dtype == SB_FLOAT32 || out_dtype == SB_INT16, "sb_das_run_beamformer: out dtype %d unsupported", out_dtype);
    sb_das_plan* p = const_cast<sb_das_plan*>(plan);
    cudaStream_t st = S(stream);
    DasArgs a;
    int err = fillArgs(p, a, rf, out, f_number, speed_of_sound_mm_s, window_type, window_parameter,
                       interpolate_transmits, additional_offset, st);
    if (err != SB_OK) return err;
    dim3 grid((p->numDepths + 255) / 256, p->numRx);
    // 2D, highest-weight transmit, aperture within the element table: the table kernel
    const bool table = !p->is3D && !interpolate_transmits && p->maxApertureX <= kMaxApertureElems &&
                       static_cast<int64_t>(p->numChannels) * p->numSamples <= INT32_MAX;
#define SB_BF_LAUNCH(RFT, OUTT, BFV)                                                                     \
    do {                                                                                                 \
        if (table && BFV != SB_BF_TEST_SIGNAL) dasVariantTableKernel<RFT, OUTT, BFV><<<grid, 256, 0, st>>>(a); \
        else if (p->is3D) dasVariantKernel<RFT, OUTT, true, BFV><<<grid, 256, 0, st>>>(a);               \
        else dasVariantKernel<RFT, OUTT, false, BFV><<<grid, 256, 0, st>>>(a);                           \
    } while (0)
#define SB_BF_TYPES(BFV)                                                                \
    do {                                                                                \
        if (rf_dtype == SB_INT16 && out_dtype == SB_FLOAT32) SB_BF_LAUNCH(int16_t, float, BFV); \
        else if (rf_dtype == SB_INT16) SB_BF_LAUNCH(int16_t, int16_t, BFV);             \
        else if (out_dtype == SB_FLOAT32) SB_BF_LAUNCH(float, float, BFV);              \
        else SB_BF_LAUNCH(float, int16_t, BFV);                                         \
    } while (0)
    if (sample_beamformer == SB_BF_DELAY_AND_STDDEV) SB_BF_TYPES(SB_BF_DELAY_AND_STDDEV);
    else if (sample_beamformer == SB_BF_COHERENCE_FACTOR_DAS) SB_BF_TYPES(SB_BF_COHERENCE_FACTOR_DAS);
    else SB_BF_TYPES(SB_BF_TEST_SIGNAL);
#undef SB_BF_TYPES
#undef SB_BF_LAUNCH
    SB_CHECK_LAUNCH("dasVariantKernel");
    return SB_OK;
}

int sb_rawdelay_run(const sb_das_plan* plan, const void* rf, int rf_dtype, void* out, int out_dtype, double f_number,
                    double speed_of_sound_mm_s, int window_type, float window_parameter, sb_stream stream) {
    SB_REQUIRE(plan && rf && out, "sb_rawdelay_run: null argument");
    SB_REQUIRE(rf_dtype == SB_INT16 || rf_dtype == SB_FLOAT32, "sb_rawdelay_run: rf dtype %d unsupported", rf_dtype);
    SB_REQUIRE(out_dtype == SB_FLOAT32 || out_dtype == SB_INT16, "sb_rawdelay_run: out dtype %d unsupported", out_dtype);
    sb_das_plan* p = const_cast<sb_das_plan*>(plan);
    if (p->is3D) return fail(SB_ERR_UNSUPPORTED, "sb_rawdelay_run: 3D raw delay is not implemented");
    cudaStream_t st = S(stream);
    DasArgs a;
    int err = fillArgs(p, a, rf, out, f_number, speed_of_sound_mm_s, window_type, window_parameter, 0, 0, st);
    if (err != SB_OK) return err;
    dim3 grid((p->numDepths + 255) / 256, p->numRx);
    // apertures within the element table: the table kernel
    const bool table = p->maxApertureX <= kMaxApertureElems && static_cast<int64_t>(p->numChannels) * p->numSamples <= INT32_MAX;
#define SB_RD(RFT, OUTT)                                                                 \
    do {                                                                                 \
        if (table) rawDelayTableKernel<RFT, OUTT><<<grid, 256, 0, st>>>(a);              \
        else rawDelayKernel<RFT, OUTT><<<grid, 256, 0, st>>>(a);                         \
    } while (0)
    if (rf_dtype == SB_INT16 && out_dtype == SB_FLOAT32) SB_RD(int16_t, float);
    else if (rf_dtype == SB_INT16) SB_RD(int16_t, int16_t);
    else if (out_dtype == SB_FLOAT32) SB_RD(float, float);
    else SB_RD(float, int16_t);
#undef SB_RD
    SB_CHECK_LAUNCH("rawDelayKernel");
    return SB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- allocation-free variant
// sb_das_run_static: the per-frame DAS without any device allocation. Its scratch (the geometry as
// given, the geometry in DT space, the wait-failure flag) lives in one statically reserved device
// array; the launch is the same dtConvertKernel + DAS kernels as sb_das_run.
namespace sb {
namespace {

constexpr size_t r256(size_t n) { return (n + 255) & ~size_t(255); }
constexpr uint32_t kSE = SB_DAS_STATIC_MAX_ELEMENTS, kSD = SB_DAS_STATIC_MAX_DEPTHS, kSL = SB_DAS_STATIC_MAX_SCANLINES;
constexpr size_t kOffXeMM = 0;
constexpr size_t kOffYeMM = kOffXeMM + r256(kSE * sizeof(float));
constexpr size_t kOffDepthMM = kOffYeMM + r256(kSE * sizeof(float));
constexpr size_t kOffLinesMM = kOffDepthMM + r256(kSD * sizeof(float));
constexpr size_t kOffE2C = kOffLinesMM + r256(kSL * sizeof(sb_scanline_rx));
constexpr size_t kOffXe = kOffE2C + r256(kSE * sizeof(int32_t));
constexpr size_t kOffYe = kOffXe + r256(kSE * sizeof(float));
constexpr size_t kOffDepth = kOffYe + r256(kSE * sizeof(float));
constexpr size_t kOffLines = kOffDepth + r256(kSD * sizeof(float));
constexpr size_t kOffErr = kOffLines + r256(kSL * sizeof(LineDT));
constexpr size_t kOffCounter = kOffErr + 256;
constexpr size_t kStaticScratchBytes = kOffCounter + 256;

}  // namespace
}  // namespace sb

// Device scratch of sb_das_run_static. In host code this name is only a stand-in for the device
// array: its device address comes from cudaGetSymbolAddress (staticScratchBase).
static __device__ __align__(256) unsigned char g_dasStaticScratch[sb::kStaticScratchBytes];

namespace sb {
namespace {

std::mutex g_staticMutex;
unsigned char* g_staticBase[64] = {nullptr};

// Device address of the scratch array on the current device, looked up once per device (the first
// call of sb_das_run_static on that device). A device reset after that call is not supported: the
// cached address would be stale.
int staticScratchBase(unsigned char** base) {
    int dev = 0;
    SB_CUDA(cudaGetDevice(&dev));
    SB_REQUIRE(dev >= 0 && dev < 64, "sb_das_run_static: device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_staticMutex);
    if (!g_staticBase[dev]) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_dasStaticScratch);
        if (e != cudaSuccess || !ptr) return cudaFail(e, "sb_das_run_static: cudaGetSymbolAddress");
        g_staticBase[dev] = static_cast<unsigned char*>(ptr);
    }
    *base = g_staticBase[dev];
    return SB_OK;
}

}  // namespace

// The wait-failure flag of sb_das_run_static's staged kernel on the current device, or null before
// the first call there. sb_check_device_errors reads and clears it with the library's own flag.
int* staticWaitFlag() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(g_staticMutex);
    return g_staticBase[dev] ? reinterpret_cast<int*>(g_staticBase[dev] + kOffErr) : nullptr;
}

}  // namespace sb

extern "C" int sb_das_run_static(const sb_geometry* g, const void* rf, int rf_dtype, void* out, int out_dtype,
                                 double f_number, double speed_of_sound_mm_s, int window_type, float window_parameter,
                                 int interpolate_transmits, int32_t additional_offset, sb_stream stream) {
    using namespace sb;
    SB_REQUIRE(g && rf && out, "sb_das_run_static: null argument");
    SB_REQUIRE(rf_dtype == SB_INT16 || rf_dtype == SB_FLOAT32, "sb_das_run_static: rf dtype %d unsupported", rf_dtype);
    SB_REQUIRE(out_dtype == SB_FLOAT32 || out_dtype == SB_INT16, "sb_das_run_static: out dtype %d unsupported", out_dtype);
    SB_REQUIRE(g->num_elements > 0 && g->num_channels > 0 && g->num_samples > 1 && g->num_tx > 0 && g->num_depths > 0,
               "sb_das_run_static: empty geometry");
    SB_REQUIRE(g->num_elements <= kSE && g->num_depths <= kSD && g->num_rx <= kSL,
               "sb_das_run_static: geometry (%u elements, %u depths, %u scanlines) exceeds the static limits "
               "(%u, %u, %u)", g->num_elements, g->num_depths, g->num_rx, kSE, kSD, kSL);
    SB_REQUIRE(g->num_rx == g->rx_layout[0] * g->rx_layout[1] && g->num_rx > 0, "num_rx != rx_layout product");
    SB_REQUIRE(g->element_layout[0] * g->element_layout[1] == g->num_elements, "element_layout != num_elements");
    SB_REQUIRE(g->sampling_frequency_hz > 0, "sampling frequency must be > 0");
    SB_REQUIRE(g->element_x_mm && g->element_y_mm && g->depths_mm && g->scanlines, "null geometry array");
    SB_REQUIRE(f_number > 0.0 && speed_of_sound_mm_s > 0.0, "f-number and speed of sound must be > 0");
    int err = checkWindow(window_type, window_parameter);
    if (err != SB_OK) return err;
    int32_t maxAx = 0;
    for (uint32_t i = 0; i < g->num_rx; i++) {
        const sb_scanline_rx& s = g->scanlines[i];
        for (int k = 0; k < 4; k++) {
            if (!(s.tx_weights[k] > 0.0)) continue;
            SB_REQUIRE(s.tx[k].tx_scanline_idx < g->num_tx, "scanline %u: transmit index %u >= num_tx %u", i,
                       s.tx[k].tx_scanline_idx, g->num_tx);
            SB_REQUIRE(s.tx[k].last_active_element[0] <= g->element_layout[0] &&
                           s.tx[k].last_active_element[1] <= g->element_layout[1],
                       "scanline %u: aperture beyond the element layout", i);
            maxAx = std::max(maxAx, static_cast<int32_t>(s.tx[k].last_active_element[0]) - s.tx[k].first_active_element[0]);
        }
    }
    if (g->element_to_channel)
        for (uint32_t e = 0; e < g->num_elements; e++)
            SB_REQUIRE(g->element_to_channel[e] < static_cast<int32_t>(g->num_channels), "element %u maps to channel %d",
                       e, g->element_to_channel[e]);
    unsigned char* base = nullptr;
    err = staticScratchBase(&base);
    if (err != SB_OK) return err;
    cudaStream_t st = S(stream);
    float* xeMM = reinterpret_cast<float*>(base + kOffXeMM);
    float* yeMM = reinterpret_cast<float*>(base + kOffYeMM);
    float* dMM = reinterpret_cast<float*>(base + kOffDepthMM);
    sb_scanline_rx* linesMM = reinterpret_cast<sb_scanline_rx*>(base + kOffLinesMM);
    int32_t* e2c = reinterpret_cast<int32_t*>(base + kOffE2C);
    float* xe = reinterpret_cast<float*>(base + kOffXe);
    float* ye = reinterpret_cast<float*>(base + kOffYe);
    float* dDT = reinterpret_cast<float*>(base + kOffDepth);
    LineDT* lines = reinterpret_cast<LineDT*>(base + kOffLines);
    // the wait-failure flag keeps its value across calls (zero when the module loads) until
    // sb_check_device_errors reads and clears it
    int* flag = reinterpret_cast<int*>(base + kOffErr);
    uint32_t* counter = reinterpret_cast<uint32_t*>(base + kOffCounter);
    const size_t nE = g->num_elements, nD = g->num_depths, nRx = g->num_rx;
    SB_CUDA(cudaMemcpyAsync(xeMM, g->element_x_mm, nE * sizeof(float), cudaMemcpyHostToDevice, st));
    SB_CUDA(cudaMemcpyAsync(yeMM, g->element_y_mm, nE * sizeof(float), cudaMemcpyHostToDevice, st));
    SB_CUDA(cudaMemcpyAsync(dMM, g->depths_mm, nD * sizeof(float), cudaMemcpyHostToDevice, st));
    SB_CUDA(cudaMemcpyAsync(linesMM, g->scanlines, nRx * sizeof(sb_scanline_rx), cudaMemcpyHostToDevice, st));
    if (g->element_to_channel)
        SB_CUDA(cudaMemcpyAsync(e2c, g->element_to_channel, nE * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    const double dt = 1.0 / g->sampling_frequency_hz;
    const double factor = 1 / 1.0 / (speed_of_sound_mm_s * dt);
    const double factorTime = 1 / 1.0 / dt;
    const uint32_t n = std::max(std::max(g->num_elements, g->num_depths), g->num_rx);
    dtConvertKernel<<<(n + 255) / 256, 256, 0, st>>>(xeMM, yeMM, g->num_elements, dMM, g->num_depths, linesMM,
                                                     g->num_rx, factor, factorTime, xe, ye, dDT, lines);
    SB_CHECK_LAUNCH("sb_das_run_static: dtConvertKernel");
    DasArgs a;
    a.rf = rf;
    a.out = out;
    a.xe = xe;
    a.ye = ye;
    a.depth = dDT;
    a.lines = lines;
    a.e2c = g->element_to_channel ? e2c : nullptr;
    a.apod = nullptr;
    a.nE = g->num_elements;
    a.layoutX = g->element_layout[0];
    a.nCh = g->num_channels;
    a.nS = g->num_samples;
    a.nTx = g->num_tx;
    a.nRx = g->num_rx;
    a.nD = g->num_depths;
    a.c = static_cast<float>(speed_of_sound_mm_s);
    a.dt = static_cast<float>(dt);
    a.F = static_cast<float>(f_number);
    a.offset = static_cast<float>(additional_offset);
    a.interpTx = interpolate_transmits ? 1 : 0;
    a.lut = makeLut(window_type, window_parameter);
    const bool is3D = g->rx_layout[0] > 1 && g->rx_layout[1] > 1;
    // 2D int16 -> float with the highest-weight transmit: the single-frame pack kernel of sb_das_run
    // (the reference's exact arithmetic), its work items derived from the item index, its work counter
    // in the scratch area
    if (!is3D && !interpolate_transmits && rf_dtype == SB_INT16 && out_dtype == SB_FLOAT32 &&
        maxAx <= kMaxApertureElems && g->num_samples >= 2) {
        const uint32_t nItems = (g->num_depths + kSinglePackRows - 1) / kSinglePackRows * g->num_rx;
        return launchSinglePackKernel(a, nullptr, nItems, counter, st);
    }
    const size_t rfSize = rf_dtype == SB_INT16 ? 2 : 4;
    const uint32_t maxW = stagedMaxW(g->num_channels, rfSize);
    const bool staged = !is3D && !interpolate_transmits && maxAx <= kMaxApertureElems && (g->num_samples * rfSize) % 16 == 0 &&
                        (reinterpret_cast<uintptr_t>(rf) % 16) == 0 && maxW >= 64;
    if (staged) {
        const size_t shm = ((sizeof(CtaState) + 127) & ~size_t(127)) + static_cast<size_t>(maxW) * g->num_channels * rfSize;
        const uint32_t nChunks = (g->num_depths + kStagedThreads - 1) / kStagedThreads;
        dim3 grid(nChunks, g->num_rx);
        FrameDesc f = frameOf(nullptr, a);
#define SB_STATIC_STAGED(RFT, OUTT)                                                                                    \
    do {                                                                                                               \
        auto kern = dasStagedKernel<RFT, OUTT, kStagedThreads>;                                                        \
        SB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(shm)));       \
        kern<<<grid, kStagedThreads, shm, st>>>(f, a.lut, a.out, maxW, 1u, flag);                                      \
    } while (0)
        if (rf_dtype == SB_INT16 && out_dtype == SB_FLOAT32) SB_STATIC_STAGED(int16_t, float);
        else if (rf_dtype == SB_INT16) SB_STATIC_STAGED(int16_t, int16_t);
        else if (out_dtype == SB_FLOAT32) SB_STATIC_STAGED(float, float);
        else SB_STATIC_STAGED(float, int16_t);
#undef SB_STATIC_STAGED
        SB_CHECK_LAUNCH("sb_das_run_static: dasStagedKernel");
        return SB_OK;
    }
    dim3 grid((g->num_depths + 255) / 256, g->num_rx);
#define SB_STATIC_GENERIC(RFT, OUTT)                                                   \
    do {                                                                               \
        if (is3D) dasKernel<RFT, OUTT, true><<<grid, 256, 0, st>>>(a);                \
        else dasKernel<RFT, OUTT, false><<<grid, 256, 0, st>>>(a);                    \
    } while (0)
    if (rf_dtype == SB_INT16 && out_dtype == SB_FLOAT32) SB_STATIC_GENERIC(int16_t, float);
    else if (rf_dtype == SB_INT16) SB_STATIC_GENERIC(int16_t, int16_t);
    else if (out_dtype == SB_FLOAT32) SB_STATIC_GENERIC(float, float);
    else SB_STATIC_GENERIC(float, int16_t);
#undef SB_STATIC_GENERIC
    SB_CHECK_LAUNCH("sb_das_run_static: dasKernel");
    return SB_OK;
}

// ------------------------------------------------------------------------------------------------
// Differentiable 2D DAS (extension without a reference counterpart): forward with per-element
// apodisation and its adjoint. The forward is the generic kernel above with w_e -> w_e * apod[e]
// (sample2D), so the two share every discrete decision (aperture, window index, sample index).
//
// For one pixel with upstream gradient g, weights W_e = w_e a_e, D = sum_e W_e, n active elements,
// v_e = lerp(rf_e, tau_e) and s = n / D * sum_e W_e v_e:
//   ds/drf[delta_e]     = n / D * W_e (1 - frac_e),  ds/drf[delta_e + 1] = n / D * W_e frac_e
//   ds/da_e             = w_e (n v_e - s) / D
//   ds/dc               = n / D * sum_e W_e (rf[delta_e + 1] - rf[delta_e]) * dtau_e/dc,
//   dtau_e/dc           = -(dist_e + depth) / c   (DT-space path length; the initial delay is in
//                         samples and the aperture and window are ratios, both independent of c)
// A prologue pass recomputes D and n per pixel (the aperture is recomputed, not stored) and forms
// G = g n / D and H = g s / D, with the pixel's aperture and window scale. The main pass gives one
// warp each (scanline, element) pair; its lanes walk the depths in order, so the channel samples it
// touches advance with the delays: they are accumulated in a small ring in shared memory and
// written to HBM once, in order, as they become final.
namespace sb {
namespace {

struct AdjArgs {
    DasArgs a;
    const float* fwd;      // [frames][nD][nRx] forward output
    const float* gout;     // [frames][nD][nRx]
    float4* gh;            // [frames][nRx][nD] scratch: (G, H, aperture aDT, 1 / min(aDT, maxDist))
    float* gradRf;         // [frames][nTx][nCh][nS] or null
    float* gradApod;       // [nE] or null
    float* gradC;          // [1] or null
    size_t rfFrameStride, outFrameStride;
    int exclusiveRows;     // every (transmit, channel) row has one writer: whole rows are stored
};

__global__ void __launch_bounds__(256) adjPixelKernel(AdjArgs p) {
    __shared__ float lut[64];
    const DasArgs& a = p.a;
    if (threadIdx.x < 64) lut[threadIdx.x] = a.lut.v[threadIdx.x];
    __syncthreads();
    const uint32_t line = blockIdx.y, frame = blockIdx.z;
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nD) return;
    const LineDT s = a.lines[line];
    const int k = s.highest;
    float4 gh = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if ((s.activeMask >> k) & 1) {
        const float d = __ldg(a.depth + r);
        const float aDT = apertureDT(d, a.dt, a.c, a.F);
        const float invMax = __fdiv_rn(1.0f, fminf(aDT, s.maxDistX));
        gh.z = aDT;
        gh.w = invMax;
        float D = 0.0f;
        int n = 0;
        for (int e = s.firstX[k]; e < s.lastX[k]; e++) {
            const int ch = a.e2c ? __ldg(a.e2c + e) : static_cast<int>(static_cast<uint32_t>(e) % a.nCh);
            if (ch < 0) continue;
            const float dx = __fsub_rn(__ldg(a.xe + e), s.x);
            if (fabsf(dx) <= aDT) {
                float w = lutGet(lut, __fmul_rn(dx, invMax));
                if (a.apod) w = __fmul_rn(w, __ldg(a.apod + e));
                D = __fadd_rn(D, w);
                n++;
            }
        }
        const size_t o = static_cast<size_t>(frame) * p.outFrameStride + static_cast<size_t>(r) * a.nRx + line;
        const float g = __ldg(p.gout + o);
        const float sv = __ldg(p.fwd + o);
        // pixels whose forward value is not finite (weight sum 0: the reference writes 0/0, clamped to
        // -FLT_MAX) and pixels without gradient contribute nothing
        if (n > 0 && g != 0.0f && D != 0.0f && fabsf(sv) < FLT_MAX) {
            gh.x = g * static_cast<float>(n) / D;
            gh.y = g * sv / D;
        }
    }
    p.gh[(static_cast<size_t>(frame) * a.nRx + line) * a.nD + r] = gh;
}

// blockIdx.x: group of warps over the aperture elements of scanline blockIdx.y, frame blockIdx.z.
// A warp walks the depths of its (scanline, element) in chunks of 32. Delays grow with depth, so the
// channel samples a chunk touches lie just ahead of those already final: the warp accumulates them
// in a ring of kAdjRing floats in shared memory and, after each chunk, writes out every sample below
// the next chunk's first delay (whole rows in order, zeros included, when rows are exclusive).
constexpr int kAdjRing = 128;

__global__ void __launch_bounds__(256) adjElemKernel(AdjArgs p) {
    __shared__ float ringAll[8][kAdjRing];
    __shared__ float lut[64];
    const DasArgs& a = p.a;
    if (threadIdx.x < 64) lut[threadIdx.x] = a.lut.v[threadIdx.x];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int warps = blockDim.x >> 5;
    const uint32_t line = blockIdx.y, frame = blockIdx.z;
    const LineDT s = a.lines[line];
    const int k = s.highest;
    if (!((s.activeMask >> k) & 1)) return;
    const int slot = blockIdx.x * warps + warp;
    const int e = s.firstX[k] + slot;
    if (e >= s.lastX[k]) {
        // exclusive rows: slots past the aperture zero the rows of the channels it does not reach
        if (p.exclusiveRows && p.gradRf && slot < static_cast<int>(a.nCh)) {
            const uint32_t chz = static_cast<uint32_t>(e) % a.nCh;
            float* dz = p.gradRf + static_cast<size_t>(frame) * p.rfFrameStride +
                        (static_cast<size_t>(s.txIdx[k]) * a.nCh + chz) * a.nS;
            for (uint32_t t = lane; t < a.nS; t += 32) dz[t] = 0.0f;
        }
        return;
    }
    const int ch = a.e2c ? __ldg(a.e2c + e) : static_cast<int>(static_cast<uint32_t>(e) % a.nCh);
    if (ch < 0) return;
    float* ring = ringAll[warp];
    const bool wantRf = p.gradRf != nullptr;
    for (int i = lane; i < kAdjRing; i += 32) ring[i] = 0.0f;
    __syncwarp();
    const float xel = __ldg(a.xe + e);
    const float dx = __fsub_rn(xel, s.x);
    const float apodE = a.apod ? __ldg(a.apod + e) : 1.0f;
    const float iD = s.initialDelay[k];
    const float* rf = static_cast<const float*>(a.rf) + static_cast<size_t>(frame) * p.rfFrameStride +
                      (static_cast<size_t>(s.txIdx[k]) * a.nCh + ch) * a.nS;
    float* dst = wantRf ? p.gradRf + static_cast<size_t>(frame) * p.rfFrameStride +
                              (static_cast<size_t>(s.txIdx[k]) * a.nCh + ch) * a.nS
                        : nullptr;
    const float4* gh = p.gh + (static_cast<size_t>(frame) * a.nRx + line) * a.nD;
    const int nS = static_cast<int>(a.nS);
    float gA = 0.0f, gC = 0.0f;
    int flushed = 0;  // samples below `flushed` are final and written out
    // contribution c to sample t: into the ring while it is within reach, else directly to HBM
    auto add = [&](int t, float c) {
        if (t >= flushed && t < flushed + kAdjRing) atomicAdd(&ring[t & (kAdjRing - 1)], c);
        else atomicAdd(dst + t, c);
    };
    // writes samples [flushed, upTo) from the ring (all of them, zeros included, when rows are exclusive)
    auto flush = [&](int upTo) {
        upTo = min(upTo, nS);
        if (upTo <= flushed) return;
        __syncwarp();
        for (int t = flushed + lane; t < upTo; t += 32) {
            float* rs = &ring[t & (kAdjRing - 1)];
            const float v = *rs;
            *rs = 0.0f;
            if (p.exclusiveRows) dst[t] = v;
            else if (v != 0.0f) atomicAdd(dst + t, v);
        }
        __syncwarp();
        flushed = upTo;
    };
    for (uint32_t r0 = 0; r0 < a.nD; r0 += 32) {
        const uint32_t r = r0 + lane;
        if (r < a.nD) {
            const float4 GH = gh[r];  // per-pixel factors and the aperture, from the prologue
            const float aDT = GH.z;
            if (fabsf(dx) <= aDT && (GH.x != 0.0f || GH.y != 0.0f)) {
                const float d = __ldg(a.depth + r);
                const float w = lutGet(lut, __fmul_rn(dx, GH.w));
                const float W = __fmul_rn(w, apodE);
                const float xz = __fadd_rn(s.x, __fmul_rn(s.dirX, d));
                const float dy = __fmul_rn(s.dirY, d);
                const float ex = __fsub_rn(xel, xz);
                const float dist = __fsqrt_rn(__fadd_rn(__fmul_rn(ex, ex), __fmul_rn(dy, dy)));
                const float path = __fadd_rn(dist, d);
                const float delayf = __fadd_rn(__fadd_rn(iD, path), a.offset);
                const int32_t delay = static_cast<int32_t>(floorf(delayf));
                const float frac = __fsub_rn(delayf, static_cast<float>(delay));
                float v = 0.0f;
                const float GW = GH.x * W;
                if (static_cast<uint32_t>(delay) < a.nS - 1) {
                    const float v0 = __ldg(rf + delay), v1 = __ldg(rf + delay + 1);
                    v = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, frac), v0), __fmul_rn(frac, v1));
                    gC += GW * (v1 - v0) * path;
                    if (wantRf) {
                        add(delay, GW * (1.0f - frac));
                        add(delay + 1, GW * frac);
                    }
                } else if (static_cast<uint32_t>(delay) < a.nS && frac == 0.0f) {
                    v = __ldg(rf + delay);
                    if (wantRf) add(delay, GW);
                }
                gA += w * (GH.x * v - GH.y);
            }
        }
        if (wantRf) {
            // the next chunk's delays start at its first depth's delay (less one sample of slack for
            // float rounding): everything below is final
            int safe = nS;
            const uint32_t rn = r0 + 32;
            if (rn < a.nD) {
                const float d = __ldg(a.depth + rn);
                const float xz = __fadd_rn(s.x, __fmul_rn(s.dirX, d));
                const float dy = __fmul_rn(s.dirY, d);
                const float ex = __fsub_rn(xel, xz);
                const float t = __fadd_rn(__fadd_rn(iD, __fadd_rn(__fsqrt_rn(__fadd_rn(__fmul_rn(ex, ex), __fmul_rn(dy, dy))), d)),
                                          a.offset);
                safe = t > -1e9f ? static_cast<int>(floorf(fminf(t, 1e9f))) - 2 : 0;
            }
            flush(safe);
        }
    }
    if (wantRf) flush(nS);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        gA += __shfl_xor_sync(0xffffffffu, gA, o);
        gC += __shfl_xor_sync(0xffffffffu, gC, o);
    }
    if (lane == 0) {
        if (p.gradApod) atomicAdd(p.gradApod + e, gA);
        if (p.gradC) atomicAdd(p.gradC, -gC / a.c);
    }
}

// True when every (transmit, channel) row of grad_rf has at most one writer: each transmit is the
// highest-weight transmit of one scanline only, there is no channel map, and no aperture spans more
// than num_channels elements (consecutive elements map to distinct channels). The kernel then stores
// whole rows, including the zero rows of channels an aperture does not reach; only the rows of
// transmits that no scanline uses are left to zero here.
bool exclusiveGradRows(const sb_das_plan* p, std::vector<uint8_t>& txUsed) {
    if (p->hasChannelMap || !p->hLines) return false;
    txUsed.assign(p->numTx, 0);
    for (const sb_scanline_rx& s : *p->hLines) {
        int hi = 0;
        float hw = static_cast<float>(s.tx_weights[0]);
        for (int k = 1; k < 4; k++)
            if (s.tx_weights[k] > static_cast<double>(hw)) {
                hw = static_cast<float>(s.tx_weights[k]);
                hi = k;
            }
        if (!(s.tx_weights[hi] > 0.0)) continue;
        const uint32_t tx = s.tx[hi].tx_scanline_idx;
        const int n = static_cast<int>(s.tx[hi].last_active_element[0]) - static_cast<int>(s.tx[hi].first_active_element[0]);
        if (tx >= p->numTx || txUsed[tx] || n > static_cast<int>(p->numChannels)) return false;
        txUsed[tx] = 1;
    }
    return true;
}

int adjointCheck(const sb_das_plan* plan, uint32_t frames) {
    SB_REQUIRE(plan, "null plan");
    SB_REQUIRE(frames >= 1, "num_frames must be >= 1");
    if (plan->is3D) return fail(SB_ERR_UNSUPPORTED, "the differentiable DAS is 2D only");
    return SB_OK;
}

}  // namespace
}  // namespace sb

int sb_das_forward_apod(const sb_das_plan* plan, const float* rf, const float* apod, float* out, uint32_t num_frames,
                        double f_number, double speed_of_sound_mm_s, int window_type, float window_parameter,
                        sb_stream stream) {
    using namespace sb;
    int err = adjointCheck(plan, num_frames);
    if (err != SB_OK) return err;
    SB_REQUIRE(rf && out, "sb_das_forward_apod: null argument");
    sb_das_plan* p = const_cast<sb_das_plan*>(plan);
    cudaStream_t st = S(stream);
    DasArgs a;
    err = fillArgs(p, a, rf, out, f_number, speed_of_sound_mm_s, window_type, window_parameter, 0, 0, st);
    if (err != SB_OK) return err;
    a.apod = apod;
    const size_t rfStride = static_cast<size_t>(p->numTx) * p->numChannels * p->numSamples;
    const size_t outStride = static_cast<size_t>(p->numDepths) * p->numRx;
    dim3 grid((p->numDepths + 255) / 256, p->numRx);
    for (uint32_t f = 0; f < num_frames; f++) {
        a.rf = rf + f * rfStride;
        a.out = out + f * outStride;
        dasKernel<float, float, false><<<grid, 256, 0, st>>>(a);
    }
    SB_CHECK_LAUNCH("sb_das_forward_apod");
    return SB_OK;
}

int sb_das_adjoint(const sb_das_plan* plan, const float* rf, const float* apod, const float* forward_out,
                   const float* grad_out, float* grad_rf, float* grad_apod, float* grad_c, uint32_t num_frames,
                   double f_number, double speed_of_sound_mm_s, int window_type, float window_parameter,
                   sb_stream stream) {
    using namespace sb;
    int err = adjointCheck(plan, num_frames);
    if (err != SB_OK) return err;
    SB_REQUIRE(rf && grad_out, "sb_das_adjoint: null argument");
    sb_das_plan* p = const_cast<sb_das_plan*>(plan);
    cudaStream_t st = S(stream);
    const size_t rfStride = static_cast<size_t>(p->numTx) * p->numChannels * p->numSamples;
    const size_t outStride = static_cast<size_t>(p->numDepths) * p->numRx;
    // scratch: the forward output when not given, and the per-pixel (G, H)
    const size_t ghBytes = static_cast<size_t>(num_frames) * outStride * sizeof(float4);
    const size_t fwdBytes = forward_out ? 0 : static_cast<size_t>(num_frames) * outStride * sizeof(float);
    if (p->adjScratchBytes < ghBytes + fwdBytes) {
        // growing the cached scratch synchronises once (cudaFree); later calls reuse it
        cudaFree(p->adjScratch);
        p->adjScratch = nullptr;
        p->adjScratchBytes = 0;
        SB_CUDA(cudaMalloc(&p->adjScratch, ghBytes + fwdBytes));
        p->adjScratchBytes = ghBytes + fwdBytes;
    }
    void* scratch = p->adjScratch;
    float4* gh = static_cast<float4*>(scratch);
    const float* fwd = forward_out;
    int rc = SB_OK;
    if (!fwd) {
        float* tmp = reinterpret_cast<float*>(static_cast<char*>(scratch) + ghBytes);
        rc = sb_das_forward_apod(plan, rf, apod, tmp, num_frames, f_number, speed_of_sound_mm_s, window_type,
                                 window_parameter, stream);
        fwd = tmp;
    }
    DasArgs a;
    std::vector<uint8_t> txUsed;
    const bool exclusive = exclusiveGradRows(p, txUsed);
    if (rc == SB_OK)
        rc = fillArgs(p, a, rf, nullptr, f_number, speed_of_sound_mm_s, window_type, window_parameter, 0, 0, st);
    if (rc == SB_OK) {
        a.apod = apod;
        if (grad_rf) {
            // exclusive rows: only transmits that no scanline uses need zeros; otherwise reductions
            // into a zeroed buffer
            const size_t txBytes = static_cast<size_t>(p->numChannels) * p->numSamples * sizeof(float);
            for (uint32_t f = 0; f < num_frames && rc == SB_OK; f++) {
                float* base = grad_rf + f * rfStride;
                if (!exclusive) {
                    if (cudaMemsetAsync(base, 0, rfStride * sizeof(float), st) != cudaSuccess)
                        rc = cudaFail(cudaGetLastError(), "cudaMemsetAsync");
                    continue;
                }
                for (uint32_t tx = 0; tx < p->numTx && rc == SB_OK; tx++)
                    if (!txUsed[tx] && cudaMemsetAsync(reinterpret_cast<char*>(base) + tx * txBytes, 0, txBytes, st) != cudaSuccess)
                        rc = cudaFail(cudaGetLastError(), "cudaMemsetAsync");
            }
        }
        if (rc == SB_OK && grad_apod && cudaMemsetAsync(grad_apod, 0, p->numElements * sizeof(float), st) != cudaSuccess)
            rc = cudaFail(cudaGetLastError(), "cudaMemsetAsync");
        if (rc == SB_OK && grad_c && cudaMemsetAsync(grad_c, 0, sizeof(float), st) != cudaSuccess)
            rc = cudaFail(cudaGetLastError(), "cudaMemsetAsync");
    }
    if (rc == SB_OK) {
        AdjArgs q;
        q.a = a;
        q.fwd = fwd;
        q.gout = grad_out;
        q.gh = gh;
        q.gradRf = grad_rf;
        q.gradApod = grad_apod;
        q.gradC = grad_c;
        q.rfFrameStride = rfStride;
        q.outFrameStride = outStride;
        q.exclusiveRows = exclusive ? 1 : 0;
        adjPixelKernel<<<dim3((p->numDepths + 255) / 256, p->numRx, num_frames), 256, 0, st>>>(q);
        const int w = 8;
        const uint32_t slots = exclusive && grad_rf ? std::max<uint32_t>(p->maxApertureX, p->numChannels)
                                                    : static_cast<uint32_t>(std::max(p->maxApertureX, 1));
        const uint32_t groups = (slots + w - 1) / w;
        adjElemKernel<<<dim3(groups, p->numRx, num_frames), 32 * w, 0, st>>>(q);
        cudaError_t le = cudaGetLastError();
        if (le != cudaSuccess) rc = cudaFail(le, "adjElemKernel");
    }
    return rc;
}
