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
// Depth segments (multiples of the decimation) are beamformed with a halo of `half` depths on both
// sides so that the low-pass of the IQ stage sees all its taps; the host cuts each scanline so that an
// item's depths (halo included, at most kPackRows) fill whole blocks of the CTA's threads. The
// beamformed depths of the whole item stay in shared memory and the IQ outputs are computed once the
// item is complete, so the CTA meets one barrier per item instead of two per depth block. A partial
// pack (fewer frames than slots) runs the loops of a narrower pack. The aperture test,
// window-LUT entry and sample index are the reference's bit for bit; the per-frame accumulation is
// contracted into FMAs (w(1-f) and w f computed once per element), so sums differ from the per-frame
// kernel by float rounding only (~1e-7 relative).
#pragma once

#include "das_core.cuh"
#include "envelope.cuh"

namespace sb {

constexpr int kMaxPack = 8;
constexpr int kPackRows = 1152;  // beamformed depths per work item, low-pass halo included (9 blocks of 128)

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
    PackDev single;  // MODE 1: the one frame (no pack table)
};

__device__ __forceinline__ int floorDiv(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

// Depths per work item of the single-frame path (MODE 1).
constexpr uint32_t kSinglePackRows = 128;

// MODE 1 work item `it` without an item table: (scanline, 128-depth segment), deepest segments first
// and scanlines inner, the order the planned single-frame path writes into its table.
__host__ __device__ __forceinline__ PackItem singleItem(uint32_t it, uint32_t nRx, uint32_t nD) {
    const uint32_t nSeg = (nD + kSinglePackRows - 1) / kSinglePackRows;
    const uint32_t k = nSeg - 1 - it / nRx;
    const uint32_t seg1 = (k + 1) * kSinglePackRows < nD ? (k + 1) * kSinglePackRows : nD;
    return PackItem{0u, it % nRx, k * kSinglePackRows, seg1};
}

template <int FP>
struct PackAcc {
    float v[FP];
};

// Sum of one depth over the element table for the first K frames of the pack (the reference's
// sampleBeamform2D per frame, with the per-element geometry shared).
template <int FP, int K, bool DEEP, bool USE_OFFSET, bool EXACT>
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
        // The reference's three cases (RxSampleBeamformerDelayAndSum.h:178-188). Fast path when every
        // lane of the warp has an interior sample (the common case); otherwise a branch-free form:
        // last sample with zero fraction -> lerp(nS - 2, nS - 1) with weights (0, 1) = RF[nS - 1];
        // no sample -> weight 0 on an in-range index.
        const bool interior = static_cast<uint32_t>(delay) < nS - 1;
        if constexpr (EXACT) {
            // the reference's arithmetic: sample += w * ((1 - f) * x[i] + f * x[i + 1]); the last sample
            // with zero fraction as (i = nS - 2, f = 1), which gives w * x[nS - 1] exactly; no sample as w = 0
            const bool lastOne = !interior && static_cast<uint32_t>(delay) < nS && frac == 0.0f;
            const uint32_t idx = interior ? static_cast<uint32_t>(delay) : (lastOne ? nS - 2 : 0u);
            const float wE = (interior || lastOne) ? w : 0.0f;
            const float fE = interior ? frac : (lastOne ? 1.0f : 0.0f);
            const uint32_t off = static_cast<uint32_t>(e.ch) + idx;
#pragma unroll
            for (int f = 0; f < K; f++) {
                const int16_t* p = tb[f] + off;
                const float v0 = static_cast<float>(__ldg(p));
                const float v1 = s16ToFloat(__ldg(p + 1));
                acc.v[f] = __fadd_rn(acc.v[f],
                                     __fmul_rn(wE, __fadd_rn(__fmul_rn(__fsub_rn(1.0f, fE), v0), __fmul_rn(fE, v1))));
            }
            continue;
        }
        uint32_t idx;
        float wA, wB;
        if (__all_sync(__activemask(), interior)) {  // vote among the lanes present here (the loop and the depth range diverge)
            idx = static_cast<uint32_t>(delay);
            wB = __fmul_rn(w, frac);
            wA = __fmul_rn(w, __fsub_rn(1.0f, frac));
        } else {
            const bool lastOne = !interior && static_cast<uint32_t>(delay) < nS && frac == 0.0f;
            idx = interior ? static_cast<uint32_t>(delay) : (lastOne ? nS - 2 : 0u);
            wB = interior ? __fmul_rn(w, frac) : (lastOne ? w : 0.0f);
            wA = interior ? __fmul_rn(w, __fsub_rn(1.0f, frac)) : 0.0f;
        }
        const uint32_t off = static_cast<uint32_t>(e.ch) + idx;  // e.ch holds the row offset
        // every slot of a partial pack points at valid data (frame 0): no per-frame predicate; the sums
        // of empty slots are never written
#pragma unroll
        for (int f = 0; f < K; f++) {
            const int16_t* p = tb[f] + off;
            const float v0 = static_cast<float>(__ldg(p));
            const float v1 = s16ToFloat(__ldg(p + 1));
            acc.v[f] = fmaf(wB, v1, fmaf(wA, v0, acc.v[f]));
        }
    }
}

// Sum over the contiguous element range [j0, j1) for the first K frames, software-pipelined: the
// gathers of element j+1 are in flight while element j is accumulated and element j+2's geometry is
// computed. DEEP: every element is active with its precomputed weight. Otherwise the range is the set
// of elements inside the aperture (contiguous when the table is ordered by x) and each weight is the
// window-LUT entry of dx / min(aDT, maxElementDistance), summed into wsum in element order (the
// reference's order).
//
// INTERIOR: every element's delay lies in [0, nS - 1) (checked by the caller), so the record-edge cases
// drop out. DX2: the scanline is not steered laterally (dirX == 0), so x_e - x_line(d) = dx for every
// depth and the table's first field holds dx * dx (the same float product the general form computes).
template <int FP, int K, bool USE_OFFSET, bool DEEP, bool EXACT, bool INTERIOR, bool DX2>
__device__ __forceinline__ void packDepthPipelined(const ElemRec* el, int j0, int j1, const float* lut, const PackDev& P,
                                                   const LineK& s, const int16_t* const (&tb)[FP], float d,
                                                   float invMax, float& wsum, PackAcc<FP>& acc) {
    if (j1 <= j0) return;
    const float xz = __fadd_rn(s.x, __fmul_rn(s.dirX, d));
    const float dyy = __fmul_rn(s.dirY, d);
    const float dy2 = __fmul_rn(dyy, dyy);
    const uint32_t nS = P.nS;
    struct G {
        uint32_t off;
        float wA, wB;
    };
    // geometry of element j; `count` adds its window weight to wsum (false for the clamped look-ahead
    // past the range, which repeats the last element so that every address stays valid without a branch)
    auto geom = [&](int j, bool count) -> G {
        const ElemRec e = el[j];
        float w;
        if (DEEP) {
            w = e.wDeep;
        } else {
            w = lutIndexWeight(lut, __fmul_rn(e.dx, invMax));
            const float ws = __fadd_rn(wsum, w);
            wsum = count ? ws : wsum;
        }
        float ex2;
        if constexpr (DX2) {
            ex2 = e.xel;
        } else {
            const float ex = __fsub_rn(e.xel, xz);
            ex2 = __fmul_rn(ex, ex);
        }
        float t = __fadd_rn(s.iD, __fadd_rn(__fsqrt_rn(__fadd_rn(ex2, dy2)), d));
        const float delayf = USE_OFFSET ? __fadd_rn(t, P.offset) : t;
        float fl;
        const int32_t delay = floorIdx(delayf, fl);
        const float frac = __fsub_rn(delayf, fl);
        G g;
        if constexpr (INTERIOR) {
            if constexpr (EXACT) {
                g.wA = w;
                g.wB = frac;
            } else {
                g.wB = __fmul_rn(w, frac);
                g.wA = __fmul_rn(w, __fsub_rn(1.0f, frac));
            }
            g.off = static_cast<uint32_t>(e.ch) + static_cast<uint32_t>(delay);
            return g;
        }
        const bool interior = static_cast<uint32_t>(delay) < nS - 1;
        const bool lastOne = !interior && static_cast<uint32_t>(delay) < nS && frac == 0.0f;
        const uint32_t idx = interior ? static_cast<uint32_t>(delay) : (lastOne ? nS - 2 : 0u);
        if constexpr (EXACT) {  // (weight, fraction) for the reference's arithmetic, see packDepth
            g.wA = (interior || lastOne) ? w : 0.0f;
            g.wB = interior ? frac : (lastOne ? 1.0f : 0.0f);
        } else {
            g.wB = interior ? __fmul_rn(w, frac) : (lastOne ? w : 0.0f);
            g.wA = interior ? __fmul_rn(w, __fsub_rn(1.0f, frac)) : 0.0f;
        }
        g.off = static_cast<uint32_t>(e.ch) + idx;  // e.ch holds the row offset
        return g;
    };
    if constexpr (K >= 6) {
        // wide packs: one element's gathers in flight while the next element's geometry is computed
        // (two sample registers per frame instead of four, so 6 and 8 frames fit the register budget)
        // The gathers of element j + kPrefetchAhead are announced to L2 at element j's delay index
        // (neighbouring elements' delays differ by a few samples): a prefetch holds no register, and the
        // one-element look-ahead alone leaves the DRAM latency of these gathers exposed (-9% on a batch of
        // 64 frames of 64/128/192-element probes).
        constexpr int kPrefetchAhead = 2;
        // the frames' sums in pairs: one packed FMA (two IEEE fused multiply-adds) per pair of frames,
        // the same rounding as one fmaf per frame
        static_assert(K % 2 == 0, "wide loops take pairs of frames");
        float2 acc2[K / 2];
#pragma unroll
        for (int f = 0; f < K; f += 2) acc2[f / 2] = make_float2(acc.v[f], acc.v[f + 1]);
        G g = geom(j0, true);
        for (int j = j0; j < j1; j++) {
            int16_t a[K], b[K];
            const uint32_t o2 = g.off << 1;  // byte offset in the transmit's rows (< 4 GB)
#pragma unroll
            for (int f = 0; f < K; f++) {
                const char* pb = reinterpret_cast<const char*>(tb[f]) + o2;
                a[f] = __ldg(reinterpret_cast<const int16_t*>(pb));
                b[f] = __ldg(reinterpret_cast<const int16_t*>(pb + 2));
            }
            if (j + kPrefetchAhead < j1) {
                // row offset of element j + kPrefetchAhead plus element j's sample index (< nS - 1):
                // an address inside that channel's row
                const uint32_t offp = static_cast<uint32_t>(el[j + kPrefetchAhead].ch) +
                                      (g.off - static_cast<uint32_t>(el[j].ch));
#pragma unroll
                for (int f = 0; f < K; f++)
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(reinterpret_cast<const char*>(tb[f]) + (offp << 1)));
            }
            const G gn = geom(min(j + 1, j1 - 1), j + 1 < j1);
            const float2 wA2 = make_float2(g.wA, g.wA), wB2 = make_float2(g.wB, g.wB);
#pragma unroll
            for (int f = 0; f < K; f += 2) {
                // int16 -> float: a by the conversion unit, b as (1.5 * 2^23 + b) - 1.5 * 2^23 (exact),
                // both subtractions of a pair in one packed add
                const float2 va = make_float2(static_cast<float>(a[f]), static_cast<float>(a[f + 1]));
                const float2 vb = __fadd2_rn(make_float2(__int_as_float(0x4B400000 + b[f]), __int_as_float(0x4B400000 + b[f + 1])),
                                             make_float2(-12582912.0f, -12582912.0f));
                acc2[f / 2] = __ffma2_rn(wB2, vb, __ffma2_rn(wA2, va, acc2[f / 2]));
            }
            g = gn;
        }
#pragma unroll
        for (int f = 0; f < K; f += 2) {
            acc.v[f] = acc2[f / 2].x;
            acc.v[f + 1] = acc2[f / 2].y;
        }
        return;
    }
    int16_t a0[K], b0[K], a1[K], b1[K];
    G g0 = geom(j0, true);
    G g1 = geom(min(j0 + 1, j1 - 1), j0 + 1 < j1);
    // all slots load valid addresses (empty pack slots alias frame 0, the step past the last element
    // repeats it), so the loads carry no predicate
#pragma unroll
    for (int f = 0; f < K; f++) {
        a0[f] = __ldg(tb[f] + g0.off);
        b0[f] = __ldg(tb[f] + g0.off + 1);
    }
    for (int j = j0; j < j1; j++) {
#pragma unroll
        for (int f = 0; f < K; f++) {
            a1[f] = __ldg(tb[f] + g1.off);
            b1[f] = __ldg(tb[f] + g1.off + 1);
        }
        const G g2 = geom(min(j + 2, j1 - 1), j + 2 < j1);
#pragma unroll
        for (int f = 0; f < K; f++) {
            if constexpr (EXACT)
                acc.v[f] = __fadd_rn(acc.v[f], __fmul_rn(g0.wA, __fadd_rn(__fmul_rn(__fsub_rn(1.0f, g0.wB),
                                                                                    static_cast<float>(a0[f])),
                                                                          __fmul_rn(g0.wB, s16ToFloat(b0[f])))));
            else
                acc.v[f] = fmaf(g0.wB, s16ToFloat(b0[f]), fmaf(g0.wA, static_cast<float>(a0[f]), acc.v[f]));
            a0[f] = a1[f];
            b0[f] = b1[f];
        }
        g0 = g1;
        g1 = g2;
    }
}

// [j0, j1): the elements with |dx| <= aDT in a table ordered by dx (binary searches).
__device__ __forceinline__ void apertureRange(const ElemRec* el, int n, float aDT, int& j0, int& j1) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (el[mid].dx < -aDT) lo = mid + 1;
        else hi = mid;
    }
    j0 = lo;
    hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (el[mid].dx <= aDT) lo = mid + 1;
        else hi = mid;
    }
    j1 = lo;
}

// One beamformed depth for the first K frames of the pack: the deep path (every element active
// with its precomputed weight), the aperture range of an x-ordered table, or the element-by-element
// aperture test; then the reference's normalisation (sum / weight sum * count) and clamped cast.
// dx2: the table's first field holds dx * dx (unsteered line); otherwise the element's x.
template <int FP, int K, bool EXACT>
__device__ __forceinline__ void packRow(const ElemRec* el, int n, const float* lut, const PackDev& P, const LineK& s,
                                        const int16_t* const (&tb)[FP], int nf, float d, int deepOk, int sortedX,
                                        float sumDeep, int cntDeep, bool dx2, PackAcc<FP>& acc) {
    const float aDT = apertureDTf(d, P.dt, P.c, P.F);
    const bool useOffset = P.offset != 0.0f;
    float wsum = 0.0f;
    int cnt = 0;
    const bool deep = deepOk && aDT >= s.maxDistX && n > 0;
    if (deep || sortedX) {
        float invMax = 0.0f;
        int j0 = 0, j1 = n;
        if (!deep) {
            invMax = __fdiv_rn(1.0f, fminf(aDT, s.maxDistX));
            apertureRange(el, n, aDT, j0, j1);
        }
        // Every delay of the range inside [0, nS - 1)? Delays grow with |dx| (the table is ordered by dx, so
        // the largest |dx| is at an end of the range) and each is at least iD + d (+ offset): bounding the
        // two ends bounds all, with the same float operations the loop uses. For unsteered lines only
        // (dx2 holds dx * dx); voted over the warp so that its lanes take the same loop.
        bool inRange = false;
        if (dx2 && j1 > j0) {
            const float dyy = __fmul_rn(s.dirY, d);
            const float dy2 = __fmul_rn(dyy, dyy);
            const float lo = useOffset ? __fadd_rn(__fadd_rn(s.iD, d), P.offset) : __fadd_rn(s.iD, d);
            const float e2 = fmaxf(el[j0].xel, el[j1 - 1].xel);
            const float t = __fadd_rn(s.iD, __fadd_rn(__fsqrt_rn(__fadd_rn(e2, dy2)), d));
            const float hi = useOffset ? __fadd_rn(t, P.offset) : t;
            inRange = lo >= 0.0f && hi < static_cast<float>(P.nS - 1);
        }
        inRange = __all_sync(__activemask(), inRange);
#define SB_PACK_ROW(OFS, DP)                                                                                          \
    do {                                                                                                              \
        if (inRange) packDepthPipelined<FP, K, OFS, DP, EXACT, true, true>(el, j0, j1, lut, P, s, tb, d, invMax, wsum, acc); \
        else if (dx2) packDepthPipelined<FP, K, OFS, DP, EXACT, false, true>(el, j0, j1, lut, P, s, tb, d, invMax, wsum, acc); \
        else packDepthPipelined<FP, K, OFS, DP, EXACT, false, false>(el, j0, j1, lut, P, s, tb, d, invMax, wsum, acc); \
    } while (0)
        if (deep) {
            if (useOffset) SB_PACK_ROW(true, true);
            else SB_PACK_ROW(false, true);
            wsum = sumDeep;
            cnt = cntDeep;
        } else {
            if (useOffset) SB_PACK_ROW(true, false);
            else SB_PACK_ROW(false, false);
            cnt = j1 - j0;
        }
#undef SB_PACK_ROW
    } else {
        const float invMax = __fdiv_rn(1.0f, fminf(aDT, s.maxDistX));
        if (useOffset) packDepth<FP, K, false, true, EXACT>(el, n, lut, P, s, tb, nf, d, aDT, invMax, wsum, cnt, acc);
        else packDepth<FP, K, false, false, EXACT>(el, n, lut, P, s, tb, nf, d, aDT, invMax, wsum, cnt, acc);
    }
#pragma unroll
    for (int f = 0; f < K; f++) {
        const float v = cnt > 0 ? __fmul_rn(__fdiv_rn(acc.v[f], wsum), static_cast<float>(cnt)) : 0.0f;
        acc.v[f] = clampCast<float>(v);
    }
}

// MODE 0: batched DAS + complex IQ over frame packs (RF contracted into FMAs). MODE 1: one frame,
// DAS only, bit-identical to the reference's arithmetic (sb_das_run's single-frame path): items carry
// no low-pass halo and the RF is written straight to the output image.
template <int FP, int NT, int MINB, int MODE>
__global__ void __launch_bounds__(NT, MINB) batchPackKernel(PackArgs a) {
    constexpr bool EXACT = MODE == 1;
    __shared__ ElemRec el[kMaxApertureElems];
    __shared__ float lut[64];
    constexpr int kHalf = FP >= 4 ? FP / 2 : 1;
    // the item's beamformed depths (segment + low-pass halo), for the IQ epilogue of MODE 0
    // stored by decimation phase (row q of the item at (q mod dec) * segQ + q / dec), so that the
    // epilogue's lanes, dec rows apart, read consecutive words
    constexpr int kSegStride = kPackRows + 32;
    __shared__ float seg[MODE == 0 ? FP : 1][MODE == 0 ? kSegStride : 1];
    __shared__ uint32_t itemIdx;
    __shared__ int rowChunk;  // MODE 0: the item's next 32-row chunk
    __shared__ int nEl, cntDeep, deepOk, sortedX, dx2Line;
    __shared__ float sumDeep;
    const int tid = threadIdx.x;
    if (tid < 64) lut[tid] = a.lut.v[tid];
    __syncthreads();
    for (;;) {
        if (tid == 0) {
            itemIdx = atomicAdd(a.counter, 1u);
            rowChunk = 0;  // the previous item's warps left its row loop before its epilogue barrier
        }
        __syncthreads();
        const uint32_t it = itemIdx;
        if (it >= a.nItems) return;
        const PackItem pi = (MODE == 1 && !a.items) ? singleItem(it, a.single.nRx, a.single.nD) : a.items[it];
        const PackDev& P = MODE == 1 ? a.single : a.packs[pi.pack];
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
                // without a channel map no element drops out: the row offset is final here
                r.ch = P.e2c ? ch : ch * static_cast<int>(P.nS);
                el[j] = r;
            }
        }
        if (!P.e2c) {
            // table in element order as filled: order and deep-aperture tests in parallel, the
            // weight sum in element order by one thread
            int sortedMine = 1, okMine = 1;
            __syncthreads();
            if (valid)
                for (int j = tid; j < n0; j += NT) {
                    if (j > 0 && !(el[j].dx >= el[j - 1].dx)) sortedMine = 0;
                    if (!(fabsf(el[j].dx) <= s.maxDistX)) okMine = 0;
                }
            const int sortedAll = __syncthreads_and(sortedMine);
            const int okAll = __syncthreads_and(okMine);
            // an unsteered line ordered by x keeps dx * dx in place of x (its only use from here on)
            const bool toDx2 = valid && sortedAll && s.dirX == 0.0f;
            if (toDx2)
                for (int j = tid; j < n0; j += NT) el[j].xel = __fmul_rn(el[j].dx, el[j].dx);
            if (tid == 0) {
                float sum = 0.0f;
                const int m = valid ? n0 : 0;
                for (int j = 0; j < m; j++) sum = __fadd_rn(sum, el[j].wDeep);
                nEl = m;
                sumDeep = sum;
                cntDeep = m;
                deepOk = okAll;
                sortedX = sortedAll;
                dx2Line = toDx2 ? 1 : 0;
            }
        }
        __syncthreads();
        if (tid == 0 && P.e2c) {
            int m = 0, ok = 1, sorted = 1;
            float sum = 0.0f;
            if (valid) {
                for (int j = 0; j < n0; j++) {
                    ElemRec r = el[j];
                    if (r.ch < 0) continue;
                    r.ch = r.ch * static_cast<int>(P.nS);  // from here on: the channel's row offset
                    if (m > 0 && !(r.dx >= el[m - 1].dx)) sorted = 0;
                    el[m++] = r;
                    sum = __fadd_rn(sum, r.wDeep);
                    if (!(fabsf(r.dx) <= s.maxDistX)) ok = 0;
                }
            }
            nEl = m;
            sumDeep = sum;
            cntDeep = m;
            deepOk = ok;
            sortedX = sorted;
            dx2Line = 0;
        }
        __syncthreads();
        const int n = nEl;
        const bool dx2 = dx2Line != 0;
        const int16_t* tb[FP];
#pragma unroll
        for (int f = 0; f < FP; f++) {
            // The same for every thread of the CTA; passing it through a warp reduction makes that
            // visible to the compiler, which then keeps the frame bases in uniform registers (one
            // fewer 64-bit register pair per frame in the gather loops: -1.7% on a 64-frame batch).
            const uint64_t u = reinterpret_cast<uint64_t>(P.rf[f < nf ? f : 0] + static_cast<size_t>(s.txIdx) * P.nCh * P.nS);
            const uint32_t lo = __reduce_max_sync(0xffffffffu, static_cast<uint32_t>(u));
            const uint32_t hi = __reduce_max_sync(0xffffffffu, static_cast<uint32_t>(u >> 32));
            tb[f] = reinterpret_cast<const int16_t*>((static_cast<uint64_t>(hi) << 32) | lo);
        }
        const int nD = static_cast<int>(P.nD);
        const int rStart = MODE == 1 ? static_cast<int>(pi.seg0) : max(0, static_cast<int>(pi.seg0) - a.half);
        const int rEnd = MODE == 1 ? min(nD, static_cast<int>(pi.seg1)) : min(nD, static_cast<int>(pi.seg1) + a.half + 1);
        const int so0 = static_cast<int>(pi.seg0) / a.dec;
        const int so1 = min(static_cast<int>(pi.seg1) / a.dec, nD / a.dec);
        const int nBlocks = (rEnd - rStart + NT - 1) / NT;
        const int pd = a.dec <= 32 ? a.dec : 1;
        const int segQ = (kPackRows + 32) / pd;
        auto segAt = [pd, segQ](int q) { return (q % pd) * segQ + q / pd; };
        // frames of a partial pack take the narrower loops (a pack of 4 frames holding 1 or 2; a pack of
        // 8 holding 5 or 6 takes the 6-frame loop)
        constexpr int kSix = FP == 8 ? 6 : FP;
        const int kw = nf > kSix ? FP : nf > kHalf ? kSix : (nf > 1 ? kHalf : 1);
        if constexpr (MODE == 0) {
            // the warps take the item's rows 32 at a time from a CTA counter, deepest chunk first
            // (deeper rows hold wider apertures): a warp that finishes early takes more rows, so the
            // warps reach the item's barrier together
            const int lane = tid & 31;
            const int nChunks = (rEnd - rStart + 31) >> 5;
            for (;;) {
                int c = 0;
                if (lane == 0) c = atomicAdd(&rowChunk, 1);
                c = __shfl_sync(0xffffffffu, c, 0);
                if (c >= nChunks) break;
                const int r = rStart + ((nChunks - 1 - c) << 5) + lane;
                PackAcc<FP> acc;
#pragma unroll
                for (int f = 0; f < FP; f++) acc.v[f] = 0.0f;
                if (r < rEnd && valid) {
                    const float d = __ldg(P.depth + r);
                    if (kw == FP) packRow<FP, FP, EXACT>(el, n, lut, P, s, tb, nf, d, deepOk, sortedX, sumDeep, cntDeep, dx2, acc);
                    else if (FP == 8 && kw == kSix) packRow<FP, kSix, EXACT>(el, n, lut, P, s, tb, nf, d, deepOk, sortedX, sumDeep, cntDeep, dx2, acc);
                    else if (kw == kHalf) packRow<FP, kHalf, EXACT>(el, n, lut, P, s, tb, nf, d, deepOk, sortedX, sumDeep, cntDeep, dx2, acc);
                    else packRow<FP, 1, EXACT>(el, n, lut, P, s, tb, nf, d, deepOk, sortedX, sumDeep, cntDeep, dx2, acc);
                }
                if (r < rEnd) {
#pragma unroll
                    for (int f = 0; f < FP; f++) {
                        seg[f][segAt(r - rStart)] = acc.v[f];
                        if (f < nf && r >= static_cast<int>(pi.seg0) && r < static_cast<int>(pi.seg1) && P.rfOut[f])
                            P.rfOut[f][pi.line + static_cast<size_t>(r) * P.nRx] = acc.v[f];
                    }
                }
            }
        } else {
            // MODE 1: one frame, rows in block order, RF straight to the image
            for (int k = 0; k < nBlocks; k++) {
                const int r = rStart + k * NT + tid;
                PackAcc<FP> acc;
#pragma unroll
                for (int f = 0; f < FP; f++) acc.v[f] = 0.0f;
                if (r < rEnd && valid) {
                    const float d = __ldg(P.depth + r);
                    if (kw == FP) packRow<FP, FP, EXACT>(el, n, lut, P, s, tb, nf, d, deepOk, sortedX, sumDeep, cntDeep, dx2, acc);
                    else if (FP == 8 && kw == kSix) packRow<FP, kSix, EXACT>(el, n, lut, P, s, tb, nf, d, deepOk, sortedX, sumDeep, cntDeep, dx2, acc);
                    else if (kw == kHalf) packRow<FP, kHalf, EXACT>(el, n, lut, P, s, tb, nf, d, deepOk, sortedX, sumDeep, cntDeep, dx2, acc);
                    else packRow<FP, 1, EXACT>(el, n, lut, P, s, tb, nf, d, deepOk, sortedX, sumDeep, cntDeep, dx2, acc);
                }
                if (r < rEnd) P.rfOut[0][pi.line + static_cast<size_t>(r) * P.nRx] = acc.v[0];
            }
        }
        if (MODE == 1) continue;  // the next item's first barrier orders the table's reuse
        // one barrier per item: the segment's RF is complete; its IQ outputs [so0, so1) for every frame
        __syncthreads();
        // one decimated output per thread for all frames of the pack: each tap's low-pass weight and
        // mixer phasor are loaded once for the pack's frames; interior outputs skip the record-edge tests
        const int nso = max(0, so1 - so0);
        for (int o = tid; o < nso; o += NT) {
            const int so = so0 + o;
            const int base = so * a.dec - a.half;
            const bool interior = base >= 0 && base + a.taps <= nD;
            // (re, im) of each frame in one packed FMA per tap: two IEEE fused multiply-adds
            float2 z[FP];
#pragma unroll
            for (int f = 0; f < FP; f++) z[f] = make_float2(0.0f, 0.0f);
            // taps inside the record, in order; the first one's row is at or after rStart
            const int jLo = interior ? 0 : max(0, -base);
            const int jHi = interior ? a.taps : min(a.taps, nD - base);
            int ph = 0, qi = 0;
            if (jLo < jHi) {
                const int q = base + jLo - rStart;
                ph = q % pd;
                qi = q / pd;
            }
            for (int j = jLo; j < jHi; j++) {
                const int nn = base + j;
                const float lpj = a.lp[j];
                const float2 w = __ldg(a.rot + nn);
                const int sq = ph * segQ + qi;
#pragma unroll
                for (int f = 0; f < FP; f++) {
                    if (f < nf) {
                        const float x = __fmul_rn(seg[f][sq], lpj);
                        z[f] = __ffma2_rn(make_float2(x, x), w, z[f]);
                    }
                }
                if (++ph == pd) {
                    ph = 0;
                    qi++;
                }
            }
#pragma unroll
            for (int f = 0; f < FP; f++)
                if (f < nf) P.iq[f][pi.line + static_cast<size_t>(so) * P.nRx] = z[f];
        }
        // the next item's first barrier orders these reads of seg before its writes
    }
}

}  // namespace sb
