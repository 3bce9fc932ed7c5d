// Warp-specialised staged DAS pipeline (used by the batched kernel).
//
// Warp 0 is the producer: it takes work items (whole scanlines) from the queue, builds the element
// table of each scanline into one of two line slots, and for every chunk of NC*32 depths bounds the
// channel-sample window and issues the TMA bulk copies into one of S shared-memory stages (full
// barrier: bytes landed; empty barrier: every consumer warp released the stage). Warps 1..NC are
// consumers: one depth per thread per chunk, the reference's per-sample reduction over the element
// table (das_core.cuh), results into the scanline buffer; after a scanline's last chunk they run
// the epilogue (complex IQ) behind a consumer-only named barrier and release the line slot. No
// CTA-wide barrier is taken in the steady state, so warps with more aperture elements do not stall
// the others.
#pragma once

#include "das_core.cuh"

namespace sb {

constexpr int kStages = 3;

struct StageMeta {
    int s0, W, staged;
    int slot;         // line slot the chunk belongs to
    uint32_t r0;      // first depth of the chunk
    int flags;        // bit 0: last chunk of its line, bit 1: end of work
};

struct LineSlot {
    FrameDesc f;
    LineK s;
    uint32_t frame, line;
    int n, cntDeep, deepOk, valid;
    float sumDeep;
    ElemRec el[kMaxApertureElems];
};

struct WsState {
    uint64_t full[kStages], empty[kStages], slotFree[2];
    StageMeta meta[kStages];
    float lut[64];
    LineSlot slot[2];
};

__device__ __forceinline__ void mbarArrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smemAddr(bar)) : "memory");
}

__device__ __forceinline__ void consumerBarrier(int nthreads) {
    asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}

// Producer warp: builds the element table of `sl` for scanline s (lanes over elements; lane 0
// compacts unconnected elements and sums the deep weights in element order).
__device__ __forceinline__ void producerSetupLine(LineSlot& sl, const float* lut, int lane) {
    const LineK& s = sl.s;
    const FrameDesc& f = sl.f;
    const int n = max(s.last - s.first, 0);
    sl.valid = s.valid && n <= kMaxApertureElems;
    if (!sl.valid) {
        __syncwarp();
        return;
    }
    const float invDeep = __fdiv_rn(1.0f, s.maxDistX);
    for (int j = lane; j < n; j += 32) {
        const int e = s.first + j;
        const int ch = f.e2c ? __ldg(f.e2c + e) : static_cast<int>(static_cast<uint32_t>(e) % f.nCh);
        const float xel = __ldg(f.xe + e);
        ElemRec r;
        r.xel = xel;
        r.dx = __fsub_rn(xel, s.x);
        r.wDeep = lutIndexWeight(lut, __fmul_rn(r.dx, invDeep));
        r.ch = ch;
        sl.el[j] = r;
    }
    __syncwarp();
    if (lane == 0) {
        int m = 0, ok = 1;
        float sum = 0.0f;
        for (int j = 0; j < n; j++) {
            const ElemRec r = sl.el[j];
            if (r.ch < 0) continue;
            sl.el[m++] = r;
            sum = __fadd_rn(sum, r.wDeep);
            if (!(fabsf(r.dx) <= s.maxDistX)) ok = 0;
        }
        sl.n = m;
        sl.sumDeep = sum;
        sl.cntDeep = m;
        sl.deepOk = ok;
    }
    __syncwarp();
}

// Producer warp: window of chunk [r0, r0 + CH) of the line in `sl` (warp reduction), meta, copies.
template <int CH>
__device__ __forceinline__ void producerIssueChunk(WsState& st, int16_t* stages, int stage, int slotIdx, uint32_t r0,
                                                   bool last, uint32_t maxW, int lane) {
    const LineSlot& sl = st.slot[slotIdx];
    const FrameDesc& f = sl.f;
    const LineK& s = sl.s;
    const uint32_t rEnd = min(r0 + CH, f.nD) - 1;
    const float dFirst = __ldg(f.depth + r0), dLast = __ldg(f.depth + rEnd);
    const float aLast = apertureDTf(dLast, f.dt, f.c, f.F);
    const bool useOffset = f.offset != 0.0f;
    const float xz0 = __fadd_rn(s.x, __fmul_rn(s.dirX, dFirst)), xz1 = __fadd_rn(s.x, __fmul_rn(s.dirX, dLast));
    const float dy0 = __fmul_rn(s.dirY, dFirst), dy1 = __fmul_rn(s.dirY, dLast);
    const float dy20 = __fmul_rn(dy0, dy0), dy21 = __fmul_rn(dy1, dy1);
    int lo = INT_MAX, hi = INT_MIN;
    if (sl.valid) {
        for (int j = lane; j < sl.n; j += 32) {
            const ElemRec r = sl.el[j];
            if (fabsf(r.dx) <= aLast) {
                const float a = delayOf(r.xel, xz0, dy20, dFirst, s.iD, f.offset, useOffset);
                const float c = delayOf(r.xel, xz1, dy21, dLast, s.iD, f.offset, useOffset);
                lo = min(lo, static_cast<int>(fmaxf(fminf(floorf(fminf(a, c)), 1e9f), -1e9f)));
                hi = max(hi, static_cast<int>(fmaxf(fminf(floorf(fmaxf(a, c)), 1e9f), -1e9f)));
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    int s0 = lo == INT_MAX ? 0 : lo - 2;
    int s1 = hi == INT_MIN ? 0 : hi + 3;  // slack for float non-monotonicity, +1 for the lerp
    s0 = max(s0, 0);
    s1 = min(s1, static_cast<int>(f.nS));
    s0 &= ~7;
    s1 = min((s1 + 7) & ~7, static_cast<int>(f.nS));
    const int W = s1 - s0;
    const bool staged = sl.valid && W > 0 && static_cast<uint32_t>(W) <= maxW;
    if (lane == 0) {
        StageMeta m;
        m.s0 = s0;
        m.W = staged ? W : 0;
        m.staged = staged ? 1 : 0;
        m.slot = slotIdx;
        m.r0 = r0;
        m.flags = last ? 1 : 0;
        st.meta[stage] = m;
        if (staged) mbarArriveExpectTx(&st.full[stage], static_cast<uint32_t>(W) * f.nCh * sizeof(int16_t));
        else mbarArrive(&st.full[stage]);
    }
    __syncwarp();
    if (!staged) return;
    const int16_t* tx = static_cast<const int16_t*>(f.rf) + static_cast<size_t>(s.txIdx) * f.nCh * f.nS + s0;
    int16_t* dst = stages + static_cast<size_t>(stage) * f.nCh * maxW;
    const uint32_t bytes = static_cast<uint32_t>(W) * sizeof(int16_t);
    for (uint32_t ch = lane; ch < f.nCh; ch += 32) {
        fenceProxyAsyncShared();
        bulkCopyG2S(dst + ch * maxW, tx + static_cast<size_t>(ch) * f.nS, bytes, &st.full[stage]);
    }
}

// Consumer: one depth, deep (window weights depth-independent) and shallow loops split.
template <bool USE_OFFSET>
__device__ __forceinline__ float consumerDepth(const LineSlot& sl, const float* lut, const StageMeta& m,
                                               const int16_t* stage, uint32_t rowPitch, uint32_t r) {
    const FrameDesc& f = sl.f;
    const LineK& s = sl.s;
    const float d = __ldg(f.depth + r);
    const float aDT = apertureDTf(d, f.dt, f.c, f.F);
    const float xz = __fadd_rn(s.x, __fmul_rn(s.dirX, d));
    const float dyy = __fmul_rn(s.dirY, d);
    const float dy2 = __fmul_rn(dyy, dyy);
    const int s0 = m.s0;
    const uint32_t wm1 = m.staged ? static_cast<uint32_t>(m.W - 1) : 0u;
    const int16_t* tx = static_cast<const int16_t*>(f.rf) + static_cast<size_t>(s.txIdx) * f.nCh * f.nS;
    const int n = sl.n;
    float sample = 0.0f;
    auto addElement = [&](const ElemRec& e, float w) {
        float t = __fadd_rn(s.iD, __fadd_rn(__fsqrt_rn(__fadd_rn(__fmul_rn(__fsub_rn(e.xel, xz), __fsub_rn(e.xel, xz)), dy2)), d));
        const float delayf = USE_OFFSET ? __fadd_rn(t, f.offset) : t;
        float fl;
        const int32_t delay = floorIdx(delayf, fl);
        const float frac = __fsub_rn(delayf, fl);
        const uint32_t rel = static_cast<uint32_t>(delay - s0);
        float v0, v1;
        if (rel < wm1) {
            const int16_t* p = stage + static_cast<uint32_t>(e.ch) * rowPitch + rel;
            v0 = toFloat(p[0]);
            v1 = s16ToFloat(p[1]);
        } else if (static_cast<uint32_t>(delay) < f.nS - 1) {
            const int16_t* p = tx + static_cast<size_t>(e.ch) * f.nS + delay;
            v0 = rdGlobal(p);
            v1 = rdGlobal(p + 1);
        } else if (static_cast<uint32_t>(delay) < f.nS && frac == 0.0f) {
            v0 = rdGlobal(tx + static_cast<size_t>(e.ch) * f.nS + delay);
            v1 = 0.0f;
        } else {
            return;
        }
        sample = __fadd_rn(sample, __fmul_rn(w, __fadd_rn(__fmul_rn(__fsub_rn(1.0f, frac), v0), __fmul_rn(frac, v1))));
    };
    if (sl.deepOk && aDT >= s.maxDistX) {
#pragma unroll 4
        for (int j = 0; j < n; j++) {
            const ElemRec e = sl.el[j];
            addElement(e, e.wDeep);
        }
        return sl.cntDeep > 0 ? __fmul_rn(__fdiv_rn(sample, sl.sumDeep), static_cast<float>(sl.cntDeep)) : 0.0f;
    }
    const float invMax = __fdiv_rn(1.0f, fminf(aDT, s.maxDistX));
    float wsum = 0.0f;
    int cnt = 0;
#pragma unroll 2
    for (int j = 0; j < n; j++) {
        const ElemRec e = sl.el[j];
        if (!(fabsf(e.dx) <= aDT)) continue;
        const float w = lutIndexWeight(lut, __fmul_rn(e.dx, invMax));
        wsum = __fadd_rn(wsum, w);
        cnt++;
        addElement(e, w);
    }
    return cnt > 0 ? __fmul_rn(__fdiv_rn(sample, wsum), static_cast<float>(cnt)) : 0.0f;
}

}  // namespace sb
