// Staged 2D delay-and-sum core shared by the per-frame and the batched (persistent) kernels.
//
// A CTA owns one receive scanline at a time and walks its depths in chunks of NT (one depth per
// thread). Per scanline it builds, in shared memory, the table of the aperture elements of the
// highest-weight transmit {x_e, x_e - x_line, deep weight, shared-memory row}. Per chunk it bounds
// the channel-sample window the chunk's delays fall in, stages rows [s0, s0 + W) of every channel
// of that transmit into shared memory with TMA bulk copies (one per channel, completion counted on
// an mbarrier), and then every thread sums its depth over the elements from shared memory.
//
// The aperture test, the nearest window-LUT entry and the sample index are computed with the same
// IEEE float operations, in the same order, as RxSampleBeamformerDelayAndSum::sampleBeamform2D
// (Beamformer/RxSampleBeamformerDelayAndSum.h:123-208), so results are bit-identical to the
// per-frame reference semantics. Once the aperture reaches maxElementDistance the window weight no
// longer depends on depth ("deep" depths): weights and their running sum are precomputed per line
// (sum in element order, as the reference accumulates it).
#pragma once

#include <cfloat>
#include <climits>

#include "das.cuh"
#include "tma.cuh"

namespace sb {

constexpr int kMaxApertureElems = 256;   // elements per aperture handled by the staged kernels
constexpr uint32_t kWaitLimit = 1u << 22; // mbarrier polls before a staged load is declared lost

struct __align__(16) ElemRec {
    float xel;    // element x (units of c dt)
    float dx;     // xel - line x, exact
    float wDeep;  // window weight once the aperture covers maxElementDistance
    int ch;       // channel of the element
};

struct FrameDesc {
    const void* rf;  // [nTx][nCh][nS]
    const LineDT* lines;
    const float* xe;
    const float* depth;
    const int32_t* e2c;
    uint32_t nCh, nS, nTx, nRx, nD;
    float c, dt, F, offset;
};

// The scanline reduced to its highest-weight transmit, in registers.
struct LineK {
    float x, dirX, dirY, maxDistX, iD;
    uint32_t txIdx;
    int first, last;
    int valid;
};

template <typename T> __device__ __forceinline__ T pick4(const T* a, int k) {
    return k == 0 ? a[0] : k == 1 ? a[1] : k == 2 ? a[2] : a[3];
}

__device__ __forceinline__ LineK reduceLine(const LineDT& s) {
    LineK l;
    const int k = s.highest;
    l.x = s.x;
    l.dirX = s.dirX;
    l.dirY = s.dirY;
    l.maxDistX = s.maxDistX;
    l.iD = pick4(s.initialDelay, k);
    l.txIdx = pick4(s.txIdx, k);
    l.first = pick4(s.firstX, k);
    l.last = pick4(s.lastX, k);
    l.valid = (s.activeMask >> k) & 1;
    return l;
}

// Per-CTA shared state (the staged samples follow it in dynamic shared memory).
struct CtaState {
    uint64_t bar[2];
    int n;            // aperture elements in the table
    float sumDeep;    // sum of deep weights (element order)
    int cntDeep;
    int deepOk;       // every element lies within maxElementDistance
    int wmin, wmax;   // window bounds being reduced
    int s0[2], W[2];  // staged window [s0, s0 + W) per stage
    int staged[2];    // 1 if the stage holds the window
    uint32_t phase[2];
    float lut[64];
    ElemRec el[kMaxApertureElems];
};

__device__ __forceinline__ float lutIndexWeight(const float* lut, float rel) {
    const float cl = fminf(fmaxf(rel, -1.0f), 1.0f);
    return lut[static_cast<uint32_t>(roundf(__fmul_rn(31.5f, __fadd_rn(cl, 1.0f))))];
}

__device__ __forceinline__ float apertureDTf(float d, float dt, float c, float F) {
    return __fdiv_rn(__fdiv_rn(__fdiv_rn(__fmul_rn(__fmul_rn(d, dt), c), __fmul_rn(2.0f, F)), c), dt);
}

// delay in samples, the reference's operation order (RxBeamformerCommon.h:27-33 + the sums of
// RxSampleBeamformerDelayAndSum.h:174-175)
__device__ __forceinline__ float delayOf(float xel, float xz, float dy2, float depth, float iD, float offset, bool useOffset) {
    const float ex = __fsub_rn(xel, xz);
    const float t = __fadd_rn(iD, __fadd_rn(__fsqrt_rn(__fadd_rn(__fmul_rn(ex, ex), dy2)), depth));
    return useOffset ? __fadd_rn(t, offset) : t;
}

// Builds the element table of `line` (all threads participate). Returns false when the aperture
// exceeds the table (caller uses the unstaged path).
template <int NT>
__device__ bool setupLine(CtaState& st, const FrameDesc& f, const LineK& s) {
    const int tid = threadIdx.x;
    const int n = max(s.last - s.first, 0);
    if (!s.valid || n > kMaxApertureElems) return false;
    const int first = s.first;
    const float invDeep = __fdiv_rn(1.0f, s.maxDistX);
    for (int j = tid; j < n; j += NT) {
        const int e = first + j;
        const int ch = f.e2c ? __ldg(f.e2c + e) : static_cast<int>(static_cast<uint32_t>(e) % f.nCh);
        const float xel = __ldg(f.xe + e);
        ElemRec r;
        r.xel = xel;
        r.dx = __fsub_rn(xel, s.x);
        r.wDeep = lutIndexWeight(st.lut, __fmul_rn(r.dx, invDeep));
        r.ch = ch;
        st.el[j] = r;
    }
    __syncthreads();
    if (tid == 0) {
        // drop unconnected elements (keep order) and sum the deep weights in element order
        int m = 0;
        float sum = 0.0f;
        int ok = 1;
        for (int j = 0; j < n; j++) {
            ElemRec r = st.el[j];
            if (r.ch < 0) continue;
            st.el[m++] = r;
            sum = __fadd_rn(sum, r.wDeep);
            if (!(fabsf(r.dx) <= s.maxDistX)) ok = 0;
        }
        st.n = m;
        st.sumDeep = sum;
        st.cntDeep = m;
        st.deepOk = ok;
    }
    __syncthreads();
    return true;
}

// Bounds the samples the chunk [r0, r0 + NT) can touch and starts staging them into stage `b`
// (all threads participate; the copies complete asynchronously on bar[b]).
template <typename RF, int NT>
__device__ void planChunk(CtaState& st, RF* smemRF, int b, const FrameDesc& f, const LineK& s, uint32_t r0, uint32_t maxW,
                          uint32_t rowPitch, bool useOffset) {
    const int tid = threadIdx.x;
    const uint32_t rEnd = min(r0 + NT, f.nD) - 1;
    const float dFirst = __ldg(f.depth + r0), dLast = __ldg(f.depth + rEnd);
    const float aLast = apertureDTf(dLast, f.dt, f.c, f.F);
    const float iD = s.iD;
    if (tid == 0) {
        st.wmin = INT_MAX;
        st.wmax = INT_MIN;
    }
    __syncthreads();
    const float xz0 = __fadd_rn(s.x, __fmul_rn(s.dirX, dFirst)), xz1 = __fadd_rn(s.x, __fmul_rn(s.dirX, dLast));
    const float dy0 = __fmul_rn(s.dirY, dFirst), dy1 = __fmul_rn(s.dirY, dLast);
    const float dy20 = __fmul_rn(dy0, dy0), dy21 = __fmul_rn(dy1, dy1);
    int lo = INT_MAX, hi = INT_MIN;
    for (int j = tid; j < st.n; j += NT) {
        const ElemRec r = st.el[j];
        if (fabsf(r.dx) <= aLast) {
            const float a = delayOf(r.xel, xz0, dy20, dFirst, iD, f.offset, useOffset);
            const float c = delayOf(r.xel, xz1, dy21, dLast, iD, f.offset, useOffset);
            lo = min(lo, static_cast<int>(fmaxf(fminf(floorf(fminf(a, c)), 1e9f), -1e9f)));
            hi = max(hi, static_cast<int>(fmaxf(fminf(floorf(fmaxf(a, c)), 1e9f), -1e9f)));
        }
    }
    if (lo != INT_MAX) atomicMin(&st.wmin, lo);
    if (hi != INT_MIN) atomicMax(&st.wmax, hi);
    __syncthreads();
    if (tid == 0) {
        int s0 = st.wmin == INT_MAX ? 0 : st.wmin - 2;
        int s1 = st.wmax == INT_MIN ? 0 : st.wmax + 3;  // slack for float non-monotonicity, +1 for the lerp
        s0 = max(s0, 0);
        s1 = min(s1, static_cast<int>(f.nS));
        s0 &= ~7;
        s1 = min((s1 + 7) & ~7, static_cast<int>(f.nS));
        const int W = s1 - s0;
        const bool ok = W > 0 && static_cast<uint32_t>(W) <= maxW;
        st.s0[b] = s0;
        st.W[b] = ok ? W : 0;
        st.staged[b] = ok ? 1 : 0;
        if (ok) mbarArriveExpectTx(&st.bar[b], static_cast<uint32_t>(W) * f.nCh * sizeof(RF));
    }
    __syncthreads();
    if (!st.staged[b]) return;
    const RF* tx = static_cast<const RF*>(f.rf) + static_cast<size_t>(s.txIdx) * f.nCh * f.nS;
    const uint32_t bytes = static_cast<uint32_t>(st.W[b]) * sizeof(RF);
    RF* dst = smemRF + static_cast<size_t>(b) * f.nCh * rowPitch;
    for (uint32_t ch = tid; ch < f.nCh; ch += NT) {
        fenceProxyAsyncShared();
        bulkCopyG2S(dst + ch * rowPitch, tx + static_cast<size_t>(ch) * f.nS + st.s0[b], bytes, &st.bar[b]);
    }
}

// Waits for stage b (bounded). All threads call it; returns false if the copies never completed.
// The result is the same in every thread of the CTA (false if any thread's wait gave up), so the
// CTA returns, or goes on to its next barrier, as a whole.
__device__ __forceinline__ bool waitChunk(CtaState& st, int b) {
    int done = 1;
    if (st.staged[b]) done = mbarWaitBounded(&st.bar[b], st.phase[b], kWaitLimit) ? 1 : 0;
    done = __syncthreads_and(done);
    if (threadIdx.x == 0 && st.staged[b]) st.phase[b] ^= 1u;
    return done != 0;
}

template <typename RF>
__device__ __forceinline__ float rdGlobal(const RF* p) {
    return toFloat(__ldg(p));
}

// int16 -> float without the conversion unit: 1.5*2^23 + v is exact for |v| < 2^22.
__device__ __forceinline__ float s16ToFloat(int v) { return __fsub_rn(__int_as_float(0x4B400000 + v), 12582912.0f); }
template <typename RF> __device__ __forceinline__ float smemToFloat(RF v);
template <> __device__ __forceinline__ float smemToFloat<int16_t>(int16_t v) { return s16ToFloat(static_cast<int>(v)); }
template <> __device__ __forceinline__ float smemToFloat<float>(float v) { return v; }

// floor() of a sample position as int and float without the conversion unit. Valid (exact) for
// x in [0, 2^23); negative x yields a negative index (skipped by the reference's unsigned test)
// and x >= 2^23 an index >= 2^23 (beyond any record).
__device__ __forceinline__ int floorIdx(float x, float& fl) {
    const float t = __fadd_rd(fmaxf(x, -1.0f), 8388608.0f);
    fl = __fsub_rn(t, 8388608.0f);
    return __float_as_int(t) - 0x4B000000;
}

// One depth of the chunk: the reference's per-sample reduction over the element table.
template <typename RF>
__device__ __forceinline__ float dasDepth(const CtaState& st, const RF* smemRF, int b, uint32_t rowPitch,
                                          const FrameDesc& f, const LineK& s, uint32_t r, bool useOffset) {
    const float d = __ldg(f.depth + r);
    const float aDT = apertureDTf(d, f.dt, f.c, f.F);
    const float iD = s.iD;
    const float xz = __fadd_rn(s.x, __fmul_rn(s.dirX, d));
    const float dyy = __fmul_rn(s.dirY, d);
    const float dy2 = __fmul_rn(dyy, dyy);
    const int s0 = st.s0[b];
    const uint32_t wm1 = st.staged[b] ? static_cast<uint32_t>(st.W[b] - 1) : 0u;
    smemRF += static_cast<size_t>(b) * f.nCh * rowPitch;
    const RF* tx = static_cast<const RF*>(f.rf) + static_cast<size_t>(s.txIdx) * f.nCh * f.nS;
    const bool deep = st.deepOk && aDT >= s.maxDistX;
    const float invMax = __fdiv_rn(1.0f, fminf(aDT, s.maxDistX));
    float sample = 0.0f, wsum = 0.0f;
    int cnt = 0;
    const int n = st.n;
#pragma unroll 4
    for (int j = 0; j < n; j++) {
        const ElemRec e = st.el[j];
        float w;
        if (deep) {
            w = e.wDeep;
        } else {
            if (!(fabsf(e.dx) <= aDT)) continue;
            w = lutIndexWeight(st.lut, __fmul_rn(e.dx, invMax));
            wsum = __fadd_rn(wsum, w);
            cnt++;
        }
        const float delayf = delayOf(e.xel, xz, dy2, d, iD, f.offset, useOffset);
        float fl;
        const int32_t delay = floorIdx(delayf, fl);
        const float frac = __fsub_rn(delayf, fl);
        const uint32_t rel = static_cast<uint32_t>(delay - s0);
        float v0, v1;
        if (rel < wm1) {  // staged: delay in [s0, s0 + W - 2], inside [0, nS - 2]
            const RF* p = smemRF + static_cast<uint32_t>(e.ch) * rowPitch + rel;
            v0 = toFloat(p[0]);
            v1 = smemToFloat<RF>(p[1]);
        } else if (static_cast<uint32_t>(delay) < f.nS - 1) {
            const RF* p = tx + static_cast<size_t>(e.ch) * f.nS + delay;
            v0 = rdGlobal(p);
            v1 = rdGlobal(p + 1);
        } else if (static_cast<uint32_t>(delay) < f.nS && frac == 0.0f) {
            v0 = rdGlobal(tx + static_cast<size_t>(e.ch) * f.nS + delay);
            v1 = 0.0f;
        } else {
            continue;
        }
        const float v = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, frac), v0), __fmul_rn(frac, v1));
        sample = __fadd_rn(sample, __fmul_rn(w, v));
    }
    if (deep) {
        wsum = st.sumDeep;
        cnt = st.cntDeep;
    }
    return cnt > 0 ? __fmul_rn(__fdiv_rn(sample, wsum), static_cast<float>(cnt)) : 0.0f;
}

}  // namespace sb
