// Shared-geometry batched DAS + complex IQ: frames of the same probe are processed together.
//
// Frames acquired with one probe share every delay, aperture decision and window weight; only the
// channel data differs. A work item is (frame pack, scanline, depth segment): the CTA builds the
// scanline's element table once, then every thread evaluates, for its depth, each element's delay,
// sample index, interpolation fraction and weight ONCE and applies them to the FP frames of the pack
// (gather + lerp + accumulate per frame). This turns the per-(pixel, element) geometry work — the
// dominant cost of the per-frame reduction — into an amortised term, leaving the per-frame cost at a
// gather and four flops. Channel samples are read through L1/L2 (each transmit's rows are used by
// exactly one scanline, so they cross HBM once).
//
// Depth segments of SEG depths (multiple of the decimation) are beamformed with a halo of `half`
// depths on both sides so that the low-pass of the IQ stage sees all its taps; the beamformed
// depths go to a two-block ring in shared memory and the IQ outputs whose taps are complete are
// written after each block. The arithmetic per (depth, element, frame) is the reference's.
#pragma once

#include "das_core.cuh"
#include "envelope.cuh"

namespace sb {

constexpr int kMaxPack = 8;

struct PackDev {
    const LineDT* lines;
    const float* xe;
    const float* depth;
    const int32_t* e2c;
    uint32_t nCh, nS, nRx, nD;
    float c, dt, F, offset;
    int nf;
    const int16_t* rf[kMaxPack];
    float2* iq[kMaxPack];
    float* rfOut[kMaxPack];
};

struct PackItem {
    uint32_t pack, line, seg0, seg1;  // IQ outputs for samples [seg0, seg1) (multiples of dec)
};

struct PackArgs {
    const PackDev* packs;
    const PackItem* items;
    uint32_t nItems;
    uint32_t* counter;
    const float2* rot;
    int taps, half, dec;
    WindowLut lut;
    float lp[kIqMaxTaps + 1];
};

__device__ __forceinline__ int floorDiv(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

template <int FP>
struct PackAcc {
    float v[FP];
};

// Sum of one depth over the element table for the FP frames of the pack (the reference's
// sampleBeamform2D per frame, with the per-element geometry shared).
template <int FP, bool DEEP, bool USE_OFFSET>
__device__ __forceinline__ void packDepth(const ElemRec* el, int n, const float* lut, const PackDev& P, const LineK& s,
                                          const int16_t* const (&tb)[FP], int nf, float d, float aDT, float invMax,
                                          float& wsum, int& cnt, PackAcc<FP>& acc) {
    const float xz = __fadd_rn(s.x, __fmul_rn(s.dirX, d));
    const float dyy = __fmul_rn(s.dirY, d);
    const float dy2 = __fmul_rn(dyy, dyy);
    const uint32_t nS = P.nS;
#pragma unroll 2
    for (int j = 0; j < n; j++) {
        const ElemRec e = el[j];
        float w;
        if (DEEP) {
            w = e.wDeep;
        } else {
            if (!(fabsf(e.dx) <= aDT)) continue;
            w = lutIndexWeight(lut, __fmul_rn(e.dx, invMax));
            wsum = __fadd_rn(wsum, w);
            cnt++;
        }
        const float ex = __fsub_rn(e.xel, xz);
        float t = __fadd_rn(s.iD, __fadd_rn(__fsqrt_rn(__fadd_rn(__fmul_rn(ex, ex), dy2)), d));
        const float delayf = USE_OFFSET ? __fadd_rn(t, P.offset) : t;
        float fl;
        const int32_t delay = floorIdx(delayf, fl);
        const float frac = __fsub_rn(delayf, fl);
        const size_t off = static_cast<size_t>(e.ch) * nS + static_cast<uint32_t>(delay);
        if (static_cast<uint32_t>(delay) < nS - 1) {
            const float om = __fsub_rn(1.0f, frac);
#pragma unroll
            for (int f = 0; f < FP; f++) {
                if (f < nf) {
                    const int16_t* p = tb[f] + off;
                    const float v0 = static_cast<float>(__ldg(p));
                    const float v1 = s16ToFloat(__ldg(p + 1));
                    acc.v[f] = __fadd_rn(acc.v[f], __fmul_rn(w, __fadd_rn(__fmul_rn(om, v0), __fmul_rn(frac, v1))));
                }
            }
        } else if (static_cast<uint32_t>(delay) < nS && frac == 0.0f) {
#pragma unroll
            for (int f = 0; f < FP; f++) {
                if (f < nf) {
                    const float v0 = static_cast<float>(__ldg(tb[f] + off));
                    // the reference adds weight * RF[delay]; (1 - 0) * v0 + 0 * v1 with v1 = 0 is the same value
                    acc.v[f] = __fadd_rn(acc.v[f], __fmul_rn(w, __fadd_rn(__fmul_rn(1.0f, v0), 0.0f)));
                }
            }
        }
    }
}

template <int FP, int NT>
__global__ void __launch_bounds__(NT) batchPackKernel(PackArgs a) {
    __shared__ ElemRec el[kMaxApertureElems];
    __shared__ float lut[64];
    __shared__ float ring[2][FP][NT];
    __shared__ uint32_t itemIdx;
    __shared__ int nEl, cntDeep, deepOk;
    __shared__ float sumDeep;
    const int tid = threadIdx.x;
    if (tid < 64) lut[tid] = a.lut.v[tid];
    __syncthreads();
    for (;;) {
        if (tid == 0) itemIdx = atomicAdd(a.counter, 1u);
        __syncthreads();
        const uint32_t it = itemIdx;
        if (it >= a.nItems) return;
        const PackItem pi = a.items[it];
        const PackDev& P = a.packs[pi.pack];
        const LineK s = reduceLine(P.lines[pi.line]);
        const int nf = P.nf;
        // element table (as setupLine, all threads)
        const int n0 = max(s.last - s.first, 0);
        const bool valid = s.valid && n0 <= kMaxApertureElems;
        if (valid) {
            const float invDeep = __fdiv_rn(1.0f, s.maxDistX);
            for (int j = tid; j < n0; j += NT) {
                const int e = s.first + j;
                const int ch = P.e2c ? __ldg(P.e2c + e) : static_cast<int>(static_cast<uint32_t>(e) % P.nCh);
                const float xel = __ldg(P.xe + e);
                ElemRec r;
                r.xel = xel;
                r.dx = __fsub_rn(xel, s.x);
                r.wDeep = lutIndexWeight(lut, __fmul_rn(r.dx, invDeep));
                r.ch = ch;
                el[j] = r;
            }
        }
        __syncthreads();
        if (tid == 0) {
            int m = 0, ok = 1;
            float sum = 0.0f;
            if (valid) {
                for (int j = 0; j < n0; j++) {
                    const ElemRec r = el[j];
                    if (r.ch < 0) continue;
                    el[m++] = r;
                    sum = __fadd_rn(sum, r.wDeep);
                    if (!(fabsf(r.dx) <= s.maxDistX)) ok = 0;
                }
            }
            nEl = m;
            sumDeep = sum;
            cntDeep = m;
            deepOk = ok;
        }
        __syncthreads();
        const int n = nEl;
        const int16_t* tb[FP];
#pragma unroll
        for (int f = 0; f < FP; f++)
            tb[f] = (f < nf) ? P.rf[f] + static_cast<size_t>(s.txIdx) * P.nCh * P.nS : P.rf[0];
        const int nD = static_cast<int>(P.nD);
        const int rStart = max(0, static_cast<int>(pi.seg0) - a.half);
        const int rEnd = min(nD, static_cast<int>(pi.seg1) + a.half + 1);
        const int so0 = static_cast<int>(pi.seg0) / a.dec;
        const int so1 = min(static_cast<int>(pi.seg1) / a.dec, nD / a.dec);
        const int nBlocks = (rEnd - rStart + NT - 1) / NT;
        int soNext = so0;
        for (int k = 0; k < nBlocks; k++) {
            const int r = rStart + k * NT + tid;
            const int slot = k & 1;
            PackAcc<FP> acc;
#pragma unroll
            for (int f = 0; f < FP; f++) acc.v[f] = 0.0f;
            if (r < rEnd && valid) {
                const float d = __ldg(P.depth + r);
                const float aDT = apertureDTf(d, P.dt, P.c, P.F);
                const bool useOffset = P.offset != 0.0f;
                float wsum = 0.0f;
                int cnt = 0;
                if (deepOk && aDT >= s.maxDistX) {
                    if (useOffset) packDepth<FP, true, true>(el, n, lut, P, s, tb, nf, d, aDT, 0.0f, wsum, cnt, acc);
                    else packDepth<FP, true, false>(el, n, lut, P, s, tb, nf, d, aDT, 0.0f, wsum, cnt, acc);
                    wsum = sumDeep;
                    cnt = cntDeep;
                } else {
                    const float invMax = __fdiv_rn(1.0f, fminf(aDT, s.maxDistX));
                    if (useOffset) packDepth<FP, false, true>(el, n, lut, P, s, tb, nf, d, aDT, invMax, wsum, cnt, acc);
                    else packDepth<FP, false, false>(el, n, lut, P, s, tb, nf, d, aDT, invMax, wsum, cnt, acc);
                }
#pragma unroll
                for (int f = 0; f < FP; f++) {
                    const float v = cnt > 0 ? __fmul_rn(__fdiv_rn(acc.v[f], wsum), static_cast<float>(cnt)) : 0.0f;
                    acc.v[f] = clampCast<float>(v);
                }
            }
#pragma unroll
            for (int f = 0; f < FP; f++) {
                ring[slot][f][tid] = acc.v[f];
                if (f < nf && r < rEnd && r >= static_cast<int>(pi.seg0) && r < static_cast<int>(pi.seg1) && P.rfOut[f])
                    P.rfOut[f][pi.line + static_cast<size_t>(r) * P.nRx] = acc.v[f];
            }
            __syncthreads();
            // outputs whose last tap lies in this block (all remaining ones after the last block)
            const int blockLast = rStart + (k + 1) * NT - 1;
            const int soEnd = (k + 1 == nBlocks) ? so1 : min(so1, floorDiv(blockLast - a.half, a.dec) + 1);
            const int cntOut = max(0, soEnd - soNext) * nf;
            for (int idx = tid; idx < cntOut; idx += NT) {
                const int so = soNext + idx / nf;
                const int f = idx % nf;
                float re = 0.0f, im = 0.0f;
                const int base = so * a.dec - a.half;
                for (int j = 0; j < a.taps; j++) {
                    const int nn = base + j;
                    if (nn >= 0 && nn < nD) {
                        const int rel = nn - rStart;
                        const float x = ring[(rel / NT) & 1][f][rel % NT] * a.lp[j];
                        const float2 w = __ldg(a.rot + nn);
                        re = fmaf(x, w.x, re);
                        im = fmaf(x, w.y, im);
                    }
                }
                P.iq[f][pi.line + static_cast<size_t>(so) * P.nRx] = make_float2(re, im);
            }
            soNext = max(soNext, soEnd);
            __syncthreads();
        }
    }
}

}  // namespace sb
