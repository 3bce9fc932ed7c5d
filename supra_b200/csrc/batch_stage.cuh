// Shared-memory-staged variant of the frame-pack kernel (batch_pack.cuh).
//
// The register-gather pack kernel is bound by the latency of its scattered 2-byte gathers: a warp
// keeps only a few loads in flight, far from the ~35 KB per SM that HBM needs at full rate. Here the
// channel samples a depth block needs are copied into shared memory ahead of use with cp.async
// (16-byte copies, no registers held while in flight), one block ahead of the computation:
//
//  * delays grow monotonically with depth along a scanline, so for each (frame, element) the samples
//    of a block of B depths lie in the window [floor(tau(first depth)) - 1, floor(tau(last depth)) + 2),
//    about B samples wide; the window start is aligned down to 8 samples (16 bytes);
//  * windows wider than the slot (unusual depth spacing) and elements past the staged count are
//    read from global memory instead, so any geometry stays correct;
//  * two threads share a depth and split the element loop (even / odd elements), so a CTA of 256
//    threads covers B = 128 depths; their partial sums are combined in shared memory.
//
// Per block k: barrier A (block k's copies have landed; block k+1's windows are visible), issue of
// block k+1's copies (they overlap block k's element loop), the element loop over shared memory,
// the windows of block k+2 (a 3-slot table, so no slot in use is overwritten), barrier B (partials),
// combine, barrier C (ring visible), complex-IQ epilogue as in the register kernel. The aperture
// test, window index and sample index are the reference's; sums are FMA-contracted and split in two
// halves, so results differ from the per-frame kernel by float rounding only.
#pragma once

#include "batch_pack.cuh"

namespace sb {

constexpr int kStageThreads = 256;
constexpr int kStageDepths = 128;   // depths per block (two threads per depth)
constexpr int kStageSlot = 144;     // staged samples per (frame, element) and block: 128 + alignment + slack
constexpr int kStageElems = 64;     // staged elements per scanline (larger apertures: rest from global)

template <int FP> constexpr size_t stagedSmemBytes() {
    return 2ull * FP * kStageElems * kStageSlot * sizeof(int16_t);
}

__device__ __forceinline__ void cpAsync16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cpAsyncCommitGroup() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cpAsyncWaitGroup() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Window of element j for depths [r0, r1]: first staged sample (multiple of 8) or -1 if unstaged.
__device__ __forceinline__ int stageWindow(const ElemRec& e, const LineK& s, const PackDev& P, int r0, int r1, bool useOffset) {
    const float d0 = __ldg(P.depth + r0), d1 = __ldg(P.depth + r1);
    const float xz0 = __fadd_rn(s.x, __fmul_rn(s.dirX, d0)), xz1 = __fadd_rn(s.x, __fmul_rn(s.dirX, d1));
    const float y0 = __fmul_rn(s.dirY, d0), y1 = __fmul_rn(s.dirY, d1);
    const float t0 = delayOf(e.xel, xz0, __fmul_rn(y0, y0), d0, s.iD, P.offset, useOffset);
    const float t1 = delayOf(e.xel, xz1, __fmul_rn(y1, y1), d1, s.iD, P.offset, useOffset);
    const float lo = fminf(t0, t1), hi = fmaxf(t0, t1);
    if (!(lo > -1e9f && hi < 1e9f)) return -1;
    int a = static_cast<int>(floorf(lo)) - 1;
    int b = static_cast<int>(floorf(hi)) + 3;  // exclusive: index + 1 of the lerp, one sample of slack
    a = max(a, 0) & ~7;
    b = min(b, static_cast<int>(P.nS));
    if (b <= a || b - a > kStageSlot) return -1;
    return a;
}

template <int FP, int MINB>
__global__ void __launch_bounds__(kStageThreads, MINB) batchPackStagedKernel(PackArgs a) {
    constexpr int NT = kStageThreads, B = kStageDepths;
    extern __shared__ __align__(16) int16_t stage[];  // [2][FP][kStageElems][kStageSlot]
    __shared__ ElemRec el[kMaxApertureElems];
    __shared__ float lut[64];
    __shared__ float ring[2][FP][B];
    __shared__ float part[FP][B];
    __shared__ float wpart[B];
    __shared__ int cpart[B];
    __shared__ int lo[3][kStageElems];  // windows of blocks k, k+1, k+2 (slot = block % 3)
    __shared__ uint32_t itemIdx;
    __shared__ int nEl, cntDeep, deepOk;
    __shared__ float sumDeep;
    const int tid = threadIdx.x;
    const int rr = tid % B, half = tid / B;
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
        const int n = valid ? nEl : 0;
        const int nStaged = min(n, kStageElems);
        const int16_t* tb[FP];
#pragma unroll
        for (int f = 0; f < FP; f++)
            tb[f] = (f < nf) ? P.rf[f] + static_cast<size_t>(s.txIdx) * P.nCh * P.nS : P.rf[0];
        const int nD = static_cast<int>(P.nD);
        const int rStart = max(0, static_cast<int>(pi.seg0) - a.half);
        const int rEnd = min(nD, static_cast<int>(pi.seg1) + a.half + 1);
        const int so0 = static_cast<int>(pi.seg0) / a.dec;
        const int so1 = min(static_cast<int>(pi.seg1) / a.dec, nD / a.dec);
        const int nBlocks = (rEnd - rStart + B - 1) / B;
        const bool useOffset = P.offset != 0.0f;
        const uint32_t nS = P.nS;

        // copies of block kb into stage buffer kb & 1 (windows in lo[kb % 3])
        auto issue = [&](int kb) {
            const int buf = kb & 1, ws = kb % 3;
            const int perElem = kStageSlot / 8;
            const int tasks = nf * nStaged * perElem;
            for (int t = tid; t < tasks; t += NT) {
                const int f = t / (nStaged * perElem);
                const int rem = t - f * nStaged * perElem;
                const int j = rem / perElem, c = rem - j * perElem;
                const int w0 = lo[ws][j];
                if (w0 < 0) continue;
                const int s0 = w0 + c * 8;
                if (s0 + 8 > static_cast<int>(nS)) continue;
                const int16_t* src = tb[0];
#pragma unroll
                for (int q = 0; q < FP; q++)
                    if (q == f) src = tb[q];
                src += static_cast<size_t>(el[j].ch) * nS + s0;
                int16_t* dst = stage + ((static_cast<size_t>(buf) * FP + f) * kStageElems + j) * kStageSlot + c * 8;
                cpAsync16(dst, src);
            }
            cpAsyncCommitGroup();
        };
        auto windows = [&](int kb) {
            if (kb < nBlocks && tid < nStaged) {
                const int r0 = rStart + kb * B;
                lo[kb % 3][tid] = stageWindow(el[tid], s, P, r0, min(r0 + B, rEnd) - 1, useOffset);
            }
        };
        // windows of blocks 0 and 1, block 0's copies
        windows(0);
        windows(1);
        __syncthreads();
        if (nBlocks > 0) issue(0);

        int soNext = so0;
        for (int k = 0; k < nBlocks; k++) {
            const int buf = k & 1, wsl = k % 3;
            cpAsyncWaitGroup<0>();
            __syncthreads();  // A: block k's samples are in shared memory; block k+1's windows are visible
            if (k + 1 < nBlocks) issue(k + 1);  // buffer (k+1) & 1 held block k-1, read before this barrier
            const int r = rStart + k * B + rr;
            PackAcc<FP> acc;
#pragma unroll
            for (int f = 0; f < FP; f++) acc.v[f] = 0.0f;
            float wsum = 0.0f;
            int cnt = 0;
            bool deepHere = false;
            if (r < rEnd && n > 0) {
                const float d = __ldg(P.depth + r);
                const float aDT = apertureDTf(d, P.dt, P.c, P.F);
                deepHere = deepOk && aDT >= s.maxDistX;
                const float invMax = __fdiv_rn(1.0f, fminf(aDT, s.maxDistX));
                const float xz = __fadd_rn(s.x, __fmul_rn(s.dirX, d));
                const float dyy = __fmul_rn(s.dirY, d);
                const float dy2 = __fmul_rn(dyy, dyy);
                const int16_t* sb0 = stage + static_cast<size_t>(buf) * FP * kStageElems * kStageSlot;
#pragma unroll 2
                for (int j = half; j < n; j += 2) {
                    const ElemRec e = el[j];
                    float w;
                    if (deepHere) {
                        w = e.wDeep;
                    } else {
                        if (!(fabsf(e.dx) <= aDT)) continue;
                        w = lutIndexWeight(lut, __fmul_rn(e.dx, invMax));
                        wsum = __fadd_rn(wsum, w);
                        cnt++;
                    }
                    const float delayf = delayOf(e.xel, xz, dy2, d, s.iD, P.offset, useOffset);
                    float fl;
                    const int32_t delay = floorIdx(delayf, fl);
                    const float frac = __fsub_rn(delayf, fl);
                    // the reference's three cases (RxSampleBeamformerDelayAndSum.h:178-188); an element
                    // without a sample still counts in the weight sum and adds nothing
                    const bool interior = static_cast<uint32_t>(delay) < nS - 1;
                    const bool lastOne = !interior && static_cast<uint32_t>(delay) < nS && frac == 0.0f;
                    if (!interior && !lastOne) continue;
                    const uint32_t idx = interior ? static_cast<uint32_t>(delay) : nS - 2;
                    const float wB = interior ? __fmul_rn(w, frac) : w;
                    const float wA = interior ? __fmul_rn(w, __fsub_rn(1.0f, frac)) : 0.0f;
                    const int w0 = j < kStageElems ? lo[wsl][j] : -1;
                    const int rel = static_cast<int>(idx) - w0;
                    if (w0 >= 0 && rel >= 0 && rel + 1 < kStageSlot) {
                        const int16_t* p = sb0 + static_cast<size_t>(j) * kStageSlot + rel;
#pragma unroll
                        for (int f = 0; f < FP; f++) {
                            if (f < nf) {
                                const int16_t* q = p + static_cast<size_t>(f) * kStageElems * kStageSlot;
                                acc.v[f] = fmaf(wB, static_cast<float>(q[1]), fmaf(wA, static_cast<float>(q[0]), acc.v[f]));
                            }
                        }
                    } else {
                        const uint32_t off = static_cast<uint32_t>(e.ch) * nS + idx;
#pragma unroll
                        for (int f = 0; f < FP; f++) {
                            if (f < nf) {
                                const int16_t* q = tb[f] + off;
                                acc.v[f] = fmaf(wB, static_cast<float>(__ldg(q + 1)), fmaf(wA, static_cast<float>(__ldg(q)), acc.v[f]));
                            }
                        }
                    }
                }
            }
            windows(k + 2);  // slot (k+2) % 3 held block k-1's windows, last read before barrier A
            if (half == 1) {
#pragma unroll
                for (int f = 0; f < FP; f++) part[f][rr] = acc.v[f];
                wpart[rr] = wsum;
                cpart[rr] = cnt;
            }
            __syncthreads();  // B: partials visible
            if (half == 0) {
                const float ws = deepHere ? sumDeep : __fadd_rn(wsum, wpart[rr]);
                const int c = deepHere ? cntDeep : cnt + cpart[rr];
#pragma unroll
                for (int f = 0; f < FP; f++) {
                    float v = 0.0f;
                    if (r < rEnd && n > 0 && c > 0) v = __fmul_rn(__fdiv_rn(acc.v[f] + part[f][rr], ws), static_cast<float>(c));
                    v = clampCast<float>(v);
                    ring[buf][f][rr] = v;
                    if (f < nf && r < rEnd && r >= static_cast<int>(pi.seg0) && r < static_cast<int>(pi.seg1) && P.rfOut[f])
                        P.rfOut[f][pi.line + static_cast<size_t>(r) * P.nRx] = v;
                }
            }
            __syncthreads();  // C: the block's RF is in the ring
            const int blockLast = rStart + (k + 1) * B - 1;
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
                        const float x = ring[(rel / B) & 1][f][rel % B] * a.lp[j];
                        const float2 w = __ldg(a.rot + nn);
                        re = fmaf(x, w.x, re);
                        im = fmaf(x, w.y, im);
                    }
                }
                P.iq[f][pi.line + static_cast<size_t>(so) * P.nRx] = make_float2(re, im);
            }
            soNext = max(soNext, soEnd);
        }
        cpAsyncWaitGroup<0>();
        __syncthreads();
    }
}

}  // namespace sb
