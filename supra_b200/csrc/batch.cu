// Batched, persistent, graph-captured DAS + complex IQ over many frames of uneven probes.
//
// One launch processes every (frame, scanline) of the batch. Work items are whole scanlines, sorted
// longest first and handed out through an atomic counter to persistent CTAs (ctas_per_sm per SM).
// A CTA builds the scanline's element table once, then walks its depths in chunks of NT with two
// shared-memory stages: while chunk c is summed, the TMA bulk copies of chunk c+1's channel-sample
// window are in flight. The beamformed scanline stays in shared memory; the epilogue mixes it to
// baseband with exp(-j 2 pi f n / fs), applies the decimating low-pass and writes complex IQ. The
// RF image never goes to HBM (unless per-frame RF outputs are requested).
//
// The DAS arithmetic is the per-frame kernel's (das_core.cuh): bit-identical to the reference's
// sample reducer for the highest-weight transmit. The IQ stage is an extension without a reference
// counterpart (checked against an FP64 oracle).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "das_core.cuh"
#include "das_ws.cuh"
#include "batch_pack.cuh"
#include "batch_stage.cuh"
#include "design.h"
#include "envelope.cuh"

namespace sb {
namespace {

struct BatchFrameDev {
    FrameDesc f;
    float2* iq;     // [nD / dec][nRx]
    float* rfOut;   // optional [nD][nRx]
};

struct BatchItem {
    uint32_t frame;
    uint32_t line;
};

struct BatchArgs {
    const BatchFrameDev* frames;
    const BatchItem* items;
    uint32_t nItems;
    uint32_t* counter;
    int* err;
    const float2* rot;  // exp(-j 2 pi f n / fs), n in [0, maxD)
    uint32_t maxW;      // staged samples per channel row
    uint32_t maxCh;     // channel rows per stage
    uint32_t maxD;      // scanline buffer capacity
    int taps, half, dec;
    WindowLut lut;
    float lp[kIqMaxTaps + 1];
};

__host__ __device__ constexpr size_t align128(size_t x) { return (x + 127) & ~size_t(127); }

// Bounded wait helper for the pipeline: returns false (and flags the error) when it gives up.
__device__ __forceinline__ bool waitOrFlag(uint64_t* bar, uint32_t parity, int* err) {
    if (mbarWaitBounded(bar, parity, kWaitLimit)) return true;
    atomicExch(err, 1);
    return false;
}

// NC consumer warps + 1 producer warp; chunk = NC * 32 depths.
template <int NC>
__global__ void __launch_bounds__((NC + 1) * 32) batchDasIqKernel(BatchArgs a) {
    constexpr int CH = NC * 32;
    extern __shared__ __align__(128) unsigned char smraw[];
    WsState& st = *reinterpret_cast<WsState*>(smraw);
    int16_t* stages = reinterpret_cast<int16_t*>(smraw + align128(sizeof(WsState)));
    float* lineBuf = reinterpret_cast<float*>(smraw + align128(sizeof(WsState)) +
                                              align128(static_cast<size_t>(kStages) * a.maxCh * a.maxW * sizeof(int16_t)));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x < 64) st.lut[threadIdx.x] = a.lut.v[threadIdx.x];
    if (threadIdx.x == 0) {
        for (int i = 0; i < kStages; i++) {
            mbarInit(&st.full[i], 1);
            mbarInit(&st.empty[i], NC);
        }
        mbarInit(&st.slotFree[0], 1);
        mbarInit(&st.slotFree[1], 1);
        mbarInitFence();
    }
    __syncthreads();
    if (warp == 0) {
        // ---------------------------------------------------------------- producer
        uint32_t chunkCount = 0;
        uint32_t slotUse[2] = {0, 0};
        int slotIdx = 0;
        for (;;) {
            uint32_t it = 0;
            if (lane == 0) it = atomicAdd(a.counter, 1u);
            it = __shfl_sync(0xffffffffu, it, 0);
            if (it >= a.nItems) {
                const int stage = chunkCount % kStages;
                if (!waitOrFlag(&st.empty[stage], ((chunkCount / kStages) & 1) ^ 1, a.err)) return;
                if (lane == 0) {
                    st.meta[stage].flags = 2;
                    mbarArrive(&st.full[stage]);
                }
                return;
            }
            if (!waitOrFlag(&st.slotFree[slotIdx], (slotUse[slotIdx] & 1) ^ 1, a.err)) return;
            slotUse[slotIdx]++;
            LineSlot& sl = st.slot[slotIdx];
            const BatchItem bi = a.items[it];
            const BatchFrameDev& fr = a.frames[bi.frame];
            if (lane == 0) {
                sl.f = fr.f;
                sl.frame = bi.frame;
                sl.line = bi.line;
                sl.s = reduceLine(fr.f.lines[bi.line]);
            }
            __syncwarp();
            producerSetupLine(sl, st.lut, lane);
            const uint32_t nD = sl.f.nD;
            const uint32_t nChunks = (nD + CH - 1) / CH;
            for (uint32_t c = 0; c < nChunks; c++) {
                const int stage = chunkCount % kStages;
                if (!waitOrFlag(&st.empty[stage], ((chunkCount / kStages) & 1) ^ 1, a.err)) return;
                producerIssueChunk<CH>(st, stages, stage, slotIdx, c * CH, c + 1 == nChunks, a.maxW, lane);
                chunkCount++;
            }
            slotIdx ^= 1;
        }
    }
    // -------------------------------------------------------------------- consumers
    const int ctid = threadIdx.x - 32;
    uint32_t chunkCount = 0;
    for (;;) {
        const int stage = chunkCount % kStages;
        if (!waitOrFlag(&st.full[stage], (chunkCount / kStages) & 1, a.err)) return;
        const StageMeta m = st.meta[stage];
        if (m.flags & 2) return;
        const LineSlot& sl = st.slot[m.slot];
        const BatchFrameDev& fr = a.frames[sl.frame];
        const uint32_t r = m.r0 + ctid;
        if (r < sl.f.nD) {
            float v = 0.0f;
            if (sl.valid) {
                const int16_t* stg = stages + static_cast<size_t>(stage) * sl.f.nCh * a.maxW;
                v = sl.f.offset != 0.0f ? consumerDepth<true>(sl, st.lut, m, stg, a.maxW, r)
                                        : consumerDepth<false>(sl, st.lut, m, stg, a.maxW, r);
            }
            v = clampCast<float>(v);
            lineBuf[r] = v;
            if (fr.rfOut) fr.rfOut[sl.line + static_cast<size_t>(r) * sl.f.nRx] = v;
        }
        __syncwarp();
        if (lane == 0) mbarArrive(&st.empty[stage]);
        chunkCount++;
        if (m.flags & 1) {
            consumerBarrier(CH);
            // complex baseband IQ of the scanline: taps j = 0 .. taps-1 centred on sample so * dec
            const int nD = static_cast<int>(sl.f.nD);
            const int nOut = nD / a.dec;
            for (int so = ctid; so < nOut; so += CH) {
                float re = 0.0f, im = 0.0f;
                const int base = so * a.dec - a.half;
                for (int j = 0; j < a.taps; j++) {
                    const int n = base + j;
                    if (n >= 0 && n < nD) {
                        const float x = lineBuf[n] * a.lp[j];
                        const float2 w = __ldg(a.rot + n);
                        re = fmaf(x, w.x, re);
                        im = fmaf(x, w.y, im);
                    }
                }
                fr.iq[sl.line + static_cast<size_t>(so) * sl.f.nRx] = make_float2(re, im);
            }
            consumerBarrier(CH);
            if (ctid == 0) mbarArrive(&st.slotFree[m.slot]);
        }
    }
}

size_t batchSmem(uint32_t maxCh, uint32_t maxW, uint32_t maxD) {
    return align128(sizeof(WsState)) + align128(static_cast<size_t>(kStages) * maxCh * maxW * sizeof(int16_t)) +
           align128(static_cast<size_t>(maxD) * sizeof(float));
}

}  // namespace
}  // namespace sb

using namespace sb;

struct PackSet {  // pack and item tables for one (frames per pack, depth tile)
    PackDev* dPacks = nullptr;
    PackItem* dItems = nullptr;
    uint32_t nItems = 0;
};

struct sb_batch_plan {
    std::vector<sb_batch_frame> frames;
    sb_batch_params params;
    PackSet packs[4][2];  // frames per pack 1 (unused), 2, 4, 8 x depth tile 128, 256
    int fp = 8;
    BatchFrameDev* dFrames = nullptr;
    BatchItem* dItems = nullptr;
    float2* dRot = nullptr;
    uint32_t* dCounter = nullptr;
    uint32_t nItems = 0, maxCh = 0, maxD = 0;
    std::vector<BatchFrameDev> hFrames;
    BatchArgs args;
    int nt = 256, ctasPerSm = 2, staged = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graphExec = nullptr;
    int graphNt = 0, graphCtas = 0, graphFp = 0, graphStaged = -1;
    std::string signature;
};

namespace {

uint32_t batchMaxW(uint32_t maxCh, uint32_t maxD, int ctasPerSm) {
    int dev = 0;
    cudaGetDevice(&dev);
    int smemPerSm = 0, smemPerBlock = 0;
    cudaDeviceGetAttribute(&smemPerSm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&smemPerBlock, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (smemPerSm <= 0) smemPerSm = 228 * 1024;
    if (smemPerBlock <= 0) smemPerBlock = 227 * 1024;
    size_t budget = std::min<size_t>(static_cast<size_t>(smemPerSm) / ctasPerSm - 2048, static_cast<size_t>(smemPerBlock));
    size_t fixed = batchSmem(maxCh, 0, maxD) + 256;
    if (budget <= fixed) return 0;
    size_t w = (budget - fixed) / (kStages * static_cast<size_t>(maxCh) * sizeof(int16_t));
    w &= ~size_t(7);
    return static_cast<uint32_t>(std::min<size_t>(w, 4096));
}

int packSlot(int fp) { return fp == 2 ? 1 : fp == 4 ? 2 : fp == 8 ? 3 : -1; }

// Depth segments of one scanline of nD depths for a CTA of nt threads: each item's beamformed depths
// (its IQ outputs' depths plus the low-pass halo of `half` on both sides, clipped to [0, nD)) fill at
// most kPackRows depths, a whole number of nt-depth blocks; segment bounds are multiples of dec.
std::vector<std::pair<uint32_t, uint32_t>> lineSegments(uint32_t nD, int nt, int half, int dec) {
    const uint32_t target = static_cast<uint32_t>((kPackRows / nt) * nt);
    std::vector<std::pair<uint32_t, uint32_t>> segs;
    uint32_t s0 = 0;
    while (s0 < nD) {
        const uint32_t lo = s0 > static_cast<uint32_t>(half) ? s0 - half : 0u;
        // largest s1 (multiple of dec, or nD) with min(nD, s1 + half + 1) - lo <= target
        uint32_t s1 = nD;
        if (nD - lo > target) {
            s1 = lo + target - static_cast<uint32_t>(half) - 1;
            s1 -= s1 % static_cast<uint32_t>(dec);
            if (s1 <= s0) s1 = std::min(nD, s0 + static_cast<uint32_t>(dec));  // degenerate shapes: progress
        }
        segs.push_back({s0, s1});
        s0 = s1;
    }
    return segs;
}

// Groups frames by probe plan into packs of up to fp frames; items (pack, line, depth segment) in
// decreasing order of estimated cost: beamformed depths x receive-aperture elements (window of
// depth / F-number over the element pitch, capped at the plan's largest aperture) x (element geometry +
// per-frame gather work for the pack's loop width), so that the queue ends on the cheapest items.
int buildPacks(sb_batch_plan* p, int fp, int nt) {
    const int slot = packSlot(fp);
    if (slot < 0) return fail(SB_ERR_INVALID_ARG, "sb_batch: frames_per_pack %d not in {1, 2, 4, 8}", fp);
    if (nt != 128 && nt != 256) return fail(SB_ERR_INVALID_ARG, "sb_batch: pack kernel block %d not in {128, 256}", nt);
    PackSet& ps = p->packs[slot][nt == 128 ? 0 : 1];
    if (ps.dPacks) return SB_OK;
    std::vector<PackDev> packs;
    std::vector<const sb_das_plan*> probes, packProbe;
    for (const auto& fr : p->frames)
        if (std::find(probes.begin(), probes.end(), fr.probe) == probes.end()) probes.push_back(fr.probe);
    for (const sb_das_plan* probe : probes) {
        std::vector<size_t> idx;
        for (size_t i = 0; i < p->frames.size(); i++)
            if (p->frames[i].probe == probe) idx.push_back(i);
        for (size_t b = 0; b < idx.size(); b += fp) {
            const BatchFrameDev& f0 = p->hFrames[idx[b]];
            PackDev d;
            std::memset(&d, 0, sizeof(d));
            d.lines = f0.f.lines;
            d.xe = f0.f.xe;
            d.depth = f0.f.depth;
            d.e2c = f0.f.e2c;
            d.nCh = f0.f.nCh;
            d.nS = f0.f.nS;
            d.nRx = f0.f.nRx;
            d.nD = f0.f.nD;
            d.c = f0.f.c;
            d.dt = f0.f.dt;
            d.F = f0.f.F;
            d.offset = f0.f.offset;
            d.nf = static_cast<int>(std::min<size_t>(fp, idx.size() - b));
            for (int k = 0; k < d.nf; k++) {
                const BatchFrameDev& fk = p->hFrames[idx[b + k]];
                d.rf[k] = static_cast<const int16_t*>(fk.f.rf);
                d.iq[k] = fk.iq;
                d.rfOut[k] = fk.rfOut;
            }
            packs.push_back(d);
            packProbe.push_back(probe);
        }
    }
    const int dec = p->args.dec, half = p->args.half;
    const int kHalf = fp >= 4 ? fp / 2 : 1;
    std::vector<PackItem> items;
    std::vector<double> cost;
    for (uint32_t k = 0; k < packs.size(); k++) {
        const sb_das_plan* pr = packProbe[k];
        const int kw = packs[k].nf > kHalf ? fp : (packs[k].nf > 1 ? kHalf : 1);
        const double perElem = 35.0 + 16.0 * kw;  // instructions per element: geometry + per-frame gathers
        // receive-aperture elements per depth, from the element pitch and the F-number
        const std::vector<float>& xe = *pr->hXeMM;
        const std::vector<float>& dep = *pr->hDepthMM;
        const double pitch = pr->layoutX > 1 ? std::fabs(static_cast<double>(xe[pr->layoutX - 1]) - xe[0]) / (pr->layoutX - 1) : 1.0;
        const double maxAp = std::max(1, pr->maxApertureX) * std::max(1, pr->is3D ? pr->maxApertureY : 1);
        const double F = packs[k].F > 0.0f ? packs[k].F : 1.0;
        std::vector<double> prefix(packs[k].nD + 1, 0.0);  // cumulative aperture elements over depths
        for (uint32_t r = 0; r < packs[k].nD; r++) {
            const double w = pitch > 0.0 ? dep[r] / F / pitch + 1.0 : maxAp;
            prefix[r + 1] = prefix[r] + std::min(maxAp, std::max(1.0, w));
        }
        const auto segs = lineSegments(packs[k].nD, nt, half, dec);
        for (uint32_t l = 0; l < packs[k].nRx; l++)
            for (const auto& sg : segs) {
                items.push_back({k, l, sg.first, sg.second});
                const uint32_t lo = sg.first > static_cast<uint32_t>(half) ? sg.first - half : 0u;
                const uint32_t hi = std::min(packs[k].nD, sg.second + static_cast<uint32_t>(half) + 1);
                if (hi - lo > static_cast<uint32_t>(kPackRows))
                    return fail(SB_ERR_UNSUPPORTED, "sb_batch: item of %u depths exceeds %d", hi - lo, kPackRows);
                cost.push_back((prefix[hi] - prefix[lo]) * perElem);
            }
    }
    std::vector<uint32_t> order(items.size());
    for (uint32_t i = 0; i < order.size(); i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return cost[a] > cost[b]; });
    std::vector<PackItem> sorted(items.size());
    for (size_t i = 0; i < order.size(); i++) sorted[i] = items[order[i]];
    items.swap(sorted);
    cudaError_t e = cudaMalloc(&ps.dPacks, packs.size() * sizeof(PackDev));
    if (e == cudaSuccess) e = cudaMalloc(&ps.dItems, items.size() * sizeof(PackItem));
    if (e == cudaSuccess) e = cudaMemcpy(ps.dPacks, packs.data(), packs.size() * sizeof(PackDev), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(ps.dItems, items.data(), items.size() * sizeof(PackItem), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(ps.dPacks);
        cudaFree(ps.dItems);
        ps.dPacks = nullptr;
        ps.dItems = nullptr;
        return cudaFail(e, "sb_batch: pack tables");
    }
    ps.nItems = static_cast<uint32_t>(items.size());
    return SB_OK;
}

void freePacks(sb_batch_plan* p) {
    for (auto& row : p->packs)
        for (auto& ps : row) {
            cudaFree(ps.dPacks);
            cudaFree(ps.dItems);
            ps = PackSet();
        }
}

template <int FP, int MINB> int launchStagedPack(const PackArgs& a, int grid, cudaStream_t st) {
    constexpr size_t shm = stagedSmemBytes<FP>();
    static bool attrSet = false;  // per instantiation; the attribute is per function and device-independent here
    if (!attrSet) {
        SB_CUDA(cudaFuncSetAttribute(batchPackStagedKernel<FP, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(shm)));
        attrSet = true;
    }
    batchPackStagedKernel<FP, MINB><<<grid, kStageThreads, shm, st>>>(a);
    SB_CHECK_LAUNCH("batchPackStagedKernel");
    return SB_OK;
}

int launchBatch(sb_batch_plan* p, int nt, int ctas, int fp, int staged, cudaStream_t st) {
    const int grid = smCount() * ctas;
    if (fp > 1) {
        if (staged ? nt != kStageDepths : (nt != 128 && nt != 256))
            return fail(SB_ERR_INVALID_ARG, "sb_batch: pack kernel block %d not in {128, 256}", nt);
        int e = buildPacks(p, fp, nt);
        if (e != SB_OK) return e;
        const PackSet& ps = p->packs[packSlot(fp)][nt == 128 ? 0 : 1];
        PackArgs a;
        a.packs = ps.dPacks;
        a.items = ps.dItems;
        a.nItems = ps.nItems;
        a.counter = p->dCounter;
        a.rot = p->dRot;
        a.taps = p->args.taps;
        a.half = p->args.half;
        a.dec = p->args.dec;
        a.lut = p->args.lut;
        for (int j = 0; j <= kIqMaxTaps; j++) a.lp[j] = p->args.lp[j];
        SB_CUDA(cudaMemsetAsync(p->dCounter, 0, sizeof(uint32_t), st));
        if (staged) {
            if (nt != kStageDepths || (fp != 2 && fp != 4) || ctas < 1 || ctas > 2 || (fp == 4 && ctas > 1))
                return fail(SB_ERR_INVALID_ARG, "sb_batch: staged packs take depth_tile %d, frames_per_pack 2 (1-2 CTAs/SM) "
                            "or 4 (1 CTA/SM)", kStageDepths);
            if (fp == 4) return launchStagedPack<4, 1>(a, grid, st);
            return ctas == 2 ? launchStagedPack<2, 2>(a, grid, st) : launchStagedPack<2, 1>(a, grid, st);
        }
#define SB_PACK_LAUNCH(FPV, NTV, MB) batchPackKernel<FPV, NTV, MB, 0><<<grid, NTV, 0, st>>>(a)
        if (nt != 128 && nt != 256) return fail(SB_ERR_INVALID_ARG, "sb_batch: pack kernel block %d not in {128, 256}", nt);
        // register budget: `ctas` resident CTAs of nt threads per SM
        const int mb = std::max(1, std::min(ctas, 2048 / nt));
        if (fp == 2) { if (nt == 128) SB_PACK_LAUNCH(2, 128, 8); else SB_PACK_LAUNCH(2, 256, 4); }
        else if (fp == 4) {
            if (nt == 128) { if (mb >= 12) SB_PACK_LAUNCH(4, 128, 12); else SB_PACK_LAUNCH(4, 128, 8); }
            else { if (mb >= 6) SB_PACK_LAUNCH(4, 256, 6); else if (mb >= 5) SB_PACK_LAUNCH(4, 256, 5); else SB_PACK_LAUNCH(4, 256, 4); }
        } else {
            if (nt == 128) SB_PACK_LAUNCH(8, 128, 8);
            else { if (mb >= 5) SB_PACK_LAUNCH(8, 256, 5); else if (mb == 4) SB_PACK_LAUNCH(8, 256, 4); else SB_PACK_LAUNCH(8, 256, 3); }
        }
#undef SB_PACK_LAUNCH
        SB_CHECK_LAUNCH("batchPackKernel");
        return SB_OK;
    }
    BatchArgs a = p->args;
    a.maxW = batchMaxW(p->maxCh, p->maxD, ctas);
    if (a.maxW < 64) return fail(SB_ERR_UNSUPPORTED, "sb_batch: shape (%d CTAs/SM) leaves no room to stage samples", ctas);
    const size_t shm = batchSmem(p->maxCh, a.maxW, p->maxD);
    SB_CUDA(cudaMemsetAsync(p->dCounter, 0, sizeof(uint32_t), st));
#define SB_BATCH_LAUNCH(NCW)                                                                                          \
    do {                                                                                                              \
        SB_CUDA(cudaFuncSetAttribute(batchDasIqKernel<NCW>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(shm))); \
        batchDasIqKernel<NCW><<<grid, (NCW + 1) * 32, shm, st>>>(a);                                                   \
    } while (0)
    switch (nt) {
    case 128: SB_BATCH_LAUNCH(4); break;
    case 256: SB_BATCH_LAUNCH(8); break;
    case 384: SB_BATCH_LAUNCH(12); break;
    case 512: SB_BATCH_LAUNCH(16); break;
    default: return fail(SB_ERR_INVALID_ARG, "sb_batch: depth tile %d not in {128, 256, 384, 512}", nt);
    }
#undef SB_BATCH_LAUNCH
    SB_CHECK_LAUNCH("batchDasIqKernel");
    return SB_OK;
}

void dropGraph(sb_batch_plan* p) {
    if (p->graphExec) cudaGraphExecDestroy(p->graphExec);
    if (p->graph) cudaGraphDestroy(p->graph);
    p->graphExec = nullptr;
    p->graph = nullptr;
}

}  // namespace

extern "C" {

int sb_batch_plan_create(const sb_batch_frame* frames, uint32_t num_frames, const sb_batch_params* params,
                         sb_batch_plan** plan) {
    SB_REQUIRE(frames && params && plan && num_frames > 0, "sb_batch_plan_create: null argument / no frames");
    *plan = nullptr;
    SB_REQUIRE(params->f_number > 0 && params->speed_of_sound_mm_s > 0, "sb_batch_plan_create: bad f-number / c");
    SB_REQUIRE(params->lowpass_length >= 1 && params->lowpass_length < static_cast<uint32_t>(kIqMaxTaps),
               "sb_batch_plan_create: low-pass length must be in [1, %d)", kIqMaxTaps);
    SB_REQUIRE(params->decimation >= 1, "sb_batch_plan_create: decimation must be >= 1");
    SB_REQUIRE(params->window_type >= 0 && params->window_type <= 3, "sb_batch_plan_create: window type");
    SB_REQUIRE(params->depth_tile == 0 || params->depth_tile == 128 || params->depth_tile == 256 ||
                   params->depth_tile == 384 || params->depth_tile == 512,
               "sb_batch_plan_create: depth_tile must be 0, 128, 256, 384 or 512");
    SB_REQUIRE(params->ctas_per_sm >= 0 && params->ctas_per_sm <= 8, "sb_batch_plan_create: ctas_per_sm in [0, 8]");
    SB_REQUIRE(params->frames_per_pack == 0 || params->frames_per_pack == 1 || params->frames_per_pack == 2 ||
                   params->frames_per_pack == 4 || params->frames_per_pack == 8,
               "sb_batch_plan_create: frames_per_pack must be 0, 1, 2, 4 or 8");
    sb_batch_plan* p = new sb_batch_plan();
    p->frames.assign(frames, frames + num_frames);
    p->params = *params;
    auto bad = [&](int code) {
        sb_batch_plan_destroy(p);
        return code;
    };
    double fs0 = 0.0;
    std::vector<BatchItem> items;
    std::vector<uint32_t> itemLen;
    std::ostringstream sig;
    for (uint32_t i = 0; i < num_frames; i++) {
        const sb_batch_frame& fr = frames[i];
        if (!fr.probe || !fr.rf || !fr.iq_out) return bad(fail(SB_ERR_INVALID_ARG, "frame %u: null probe/rf/iq_out", i));
        sb_das_plan* dp = const_cast<sb_das_plan*>(fr.probe);
        if (dp->is3D) return bad(fail(SB_ERR_UNSUPPORTED, "frame %u: batched path is 2D only", i));
        if (dp->maxApertureX > kMaxApertureElems)
            return bad(fail(SB_ERR_UNSUPPORTED, "frame %u: aperture of %d elements > %d", i, dp->maxApertureX, kMaxApertureElems));
        if ((dp->numSamples % 8) != 0 || (reinterpret_cast<uintptr_t>(fr.rf) % 16) != 0)
            return bad(fail(SB_ERR_UNSUPPORTED, "frame %u: samples per channel must be a multiple of 8 and rf 16-byte aligned", i));
        if (i == 0) fs0 = dp->fs;
        if (dp->fs != fs0) return bad(fail(SB_ERR_UNSUPPORTED, "frame %u: all frames must share the sampling frequency", i));
        int e = ensureDtSpace(dp, params->speed_of_sound_mm_s, 0);
        if (e != SB_OK) return bad(e);
        BatchFrameDev d;
        d.f.rf = fr.rf;
        d.f.lines = dp->dLines;
        d.f.xe = dp->dXe;
        d.f.depth = dp->dDepth;
        d.f.e2c = dp->dE2C;
        d.f.nCh = dp->numChannels;
        d.f.nS = dp->numSamples;
        d.f.nTx = dp->numTx;
        d.f.nRx = dp->numRx;
        d.f.nD = dp->numDepths;
        d.f.c = static_cast<float>(params->speed_of_sound_mm_s);
        d.f.dt = static_cast<float>(1.0 / dp->fs);
        d.f.F = static_cast<float>(params->f_number);
        d.f.offset = 0.0f;
        d.iq = static_cast<float2*>(fr.iq_out);
        d.rfOut = nullptr;
        p->hFrames.push_back(d);
        p->maxCh = std::max(p->maxCh, dp->numChannels);
        p->maxD = std::max(p->maxD, dp->numDepths);
        for (uint32_t l = 0; l < dp->numRx; l++) {
            items.push_back({i, l});
            itemLen.push_back(dp->numDepths);
        }
        sig << dp->numChannels << "x" << dp->numSamples << "x" << dp->numRx << "x" << dp->numDepths << ";";
    }
    // longest scanlines first (LPT order for the dynamic queue)
    std::vector<size_t> order(items.size());
    for (size_t i = 0; i < order.size(); i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return itemLen[a] > itemLen[b]; });
    std::vector<BatchItem> sorted(items.size());
    for (size_t i = 0; i < order.size(); i++) sorted[i] = items[order[i]];
    p->nItems = static_cast<uint32_t>(sorted.size());
    // rotation table exp(-j 2 pi f n / fs), phase reduced in double
    std::vector<float2> rot(p->maxD);
    const double fOverFs = params->mixing_frequency_hz / fs0;
    for (uint32_t n = 0; n < p->maxD; n++) {
        double ph = fOverFs * n;
        ph -= std::floor(ph);
        rot[n] = make_float2(static_cast<float>(std::cos(2.0 * M_PI * ph)), static_cast<float>(-std::sin(2.0 * M_PI * ph)));
    }
    cudaError_t e = cudaMalloc(&p->dFrames, p->hFrames.size() * sizeof(BatchFrameDev));
    if (e == cudaSuccess) e = cudaMalloc(&p->dItems, sorted.size() * sizeof(BatchItem));
    if (e == cudaSuccess) e = cudaMalloc(&p->dRot, rot.size() * sizeof(float2));
    if (e == cudaSuccess) e = cudaMalloc(&p->dCounter, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemcpy(p->dFrames, p->hFrames.data(), p->hFrames.size() * sizeof(BatchFrameDev), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->dItems, sorted.data(), sorted.size() * sizeof(BatchItem), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->dRot, rot.data(), rot.size() * sizeof(float2), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return bad(cudaFail(e, "sb_batch_plan_create"));
    int* err = deviceErrorFlag();
    if (!err) return bad(fail(SB_ERR_NO_MEMORY, "sb_batch_plan_create: error flag"));
    BatchArgs& a = p->args;
    a.frames = p->dFrames;
    a.items = p->dItems;
    a.nItems = p->nItems;
    a.counter = p->dCounter;
    a.err = err;
    a.rot = p->dRot;
    a.maxCh = p->maxCh;
    a.maxD = p->maxD;
    a.maxW = 0;
    a.dec = static_cast<int>(params->decimation);
    a.half = static_cast<int>(params->lowpass_length) / 2;
    a.taps = 2 * a.half + 1;
    std::vector<float> lp = firDesign(params->lowpass_length, 0, 2, fs0, params->cutoff_frequency_hz, 0.0);
    for (int j = 0; j <= kIqMaxTaps; j++) a.lp[j] = j < static_cast<int>(params->lowpass_length) ? lp[j] : 0.0f;
    a.lut = makeLut(params->window_type, params->window_parameter);
    p->fp = params->frames_per_pack ? params->frames_per_pack : 8;
    p->nt = params->depth_tile ? params->depth_tile : (p->fp > 1 ? 256 : 384);
    p->ctasPerSm = params->ctas_per_sm ? params->ctas_per_sm : (p->fp > 1 ? 4 : 1);
    p->staged = params->staged ? 1 : 0;
    if (p->staged && (p->fp != 2 && p->fp != 4))
        return bad(fail(SB_ERR_INVALID_ARG, "sb_batch_plan_create: staged packs need frames_per_pack 2 or 4"));
    if (p->staged && !params->depth_tile) p->nt = kStageDepths;
    if (p->staged && !params->ctas_per_sm) p->ctasPerSm = 1;
    sig << "F" << params->f_number << "L" << params->lowpass_length << "D" << params->decimation;
    p->signature = sig.str();
    if (p->fp == 1 && batchMaxW(p->maxCh, p->maxD, p->ctasPerSm) < 64)
        return bad(fail(SB_ERR_UNSUPPORTED, "sb_batch_plan_create: frames too large to stage"));
    *plan = p;
    return SB_OK;
}

int sb_batch_plan_destroy(sb_batch_plan* p) {
    if (!p) return SB_OK;
    dropGraph(p);
    freePacks(p);
    cudaFree(p->dFrames);
    cudaFree(p->dItems);
    cudaFree(p->dRot);
    cudaFree(p->dCounter);
    delete p;
    return SB_OK;
}

int sb_batch_set_rf_outputs(sb_batch_plan* p, float* const* rf_out) {
    SB_REQUIRE(p, "sb_batch_set_rf_outputs: null plan");
    for (size_t i = 0; i < p->hFrames.size(); i++) p->hFrames[i].rfOut = rf_out ? rf_out[i] : nullptr;
    SB_CUDA(cudaMemcpy(p->dFrames, p->hFrames.data(), p->hFrames.size() * sizeof(BatchFrameDev), cudaMemcpyHostToDevice));
    freePacks(p);  // pack tables embed the output pointers
    dropGraph(p);
    return SB_OK;
}

int sb_batch_run(sb_batch_plan* p, int use_graph, sb_stream stream) {
    SB_REQUIRE(p, "sb_batch_run: null plan");
    cudaStream_t st = S(stream);
    if (!use_graph) return launchBatch(p, p->nt, p->ctasPerSm, p->fp, p->staged, st);
    if (p->fp > 1) {
        int e = buildPacks(p, p->fp, p->staged ? kStageDepths : p->nt);  // outside the capture: it allocates
        if (e != SB_OK) return e;
    }
    if (!p->graphExec || p->graphNt != p->nt || p->graphCtas != p->ctasPerSm || p->graphFp != p->fp ||
        p->graphStaged != p->staged) {
        dropGraph(p);
        // capture on a private stream so that the caller's stream may be the legacy default stream
        cudaStream_t cap;
        SB_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        int r = SB_OK;
        if (e == cudaSuccess) r = launchBatch(p, p->nt, p->ctasPerSm, p->fp, p->staged, cap);
        cudaGraph_t g = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(cap, &g);
        cudaStreamDestroy(cap);
        if (e != cudaSuccess) return cudaFail(e, "sb_batch_run: begin capture");
        if (r != SB_OK) {
            if (g) cudaGraphDestroy(g);
            return r;
        }
        if (e2 != cudaSuccess) return cudaFail(e2, "sb_batch_run: end capture");
        p->graph = g;
        SB_CUDA(cudaGraphInstantiate(&p->graphExec, g, 0));
        p->graphNt = p->nt;
        p->graphCtas = p->ctasPerSm;
        p->graphFp = p->fp;
        p->graphStaged = p->staged;
    }
    SB_CUDA(cudaGraphLaunch(p->graphExec, st));
    return SB_OK;
}

int sb_batch_autotune(sb_batch_plan* p, const char* cache_path, int32_t* ctas_per_sm, int32_t* depth_tile,
                      int32_t* frames_per_pack, int32_t* staged, sb_stream stream) {
    SB_REQUIRE(p, "sb_batch_autotune: null plan");
    cudaStream_t st = S(stream);
    auto report = [&]() {
        if (ctas_per_sm) *ctas_per_sm = p->ctasPerSm;
        if (depth_tile) *depth_tile = p->nt;
        if (frames_per_pack) *frames_per_pack = p->fp;
        if (staged) *staged = p->staged;
    };
    // cached choice for this problem signature? (lines: signature ctas tile frames [staged])
    if (cache_path) {
        std::ifstream in(cache_path);
        std::string key, line;
        while (std::getline(in, line)) {
            std::istringstream ls(line);
            int c = 0, t = 0, f = 0, g = 0;
            if (!(ls >> key >> c >> t >> f) || key != p->signature) continue;
            if (!(ls >> g)) g = 0;
            const bool okStaged = g == 1 && t == kStageDepths && ((f == 2 && (c == 1 || c == 2)) || (f == 4 && c == 1));
            const bool okPack = g == 0 && f > 1 && packSlot(f) >= 0 && (t == 128 || t == 256) && c >= 1 && c <= 12;
            const bool okPipe = g == 0 && f == 1 && (t == 128 || t == 256 || t == 384 || t == 512) && c >= 1 && c <= 3 &&
                                batchMaxW(p->maxCh, p->maxD, c) >= 64;
            if (okStaged || okPack || okPipe) {
                p->ctasPerSm = c;
                p->nt = t;
                p->fp = f;
                p->staged = g;
                report();
                return SB_OK;
            }
        }
    }
    // {ctas per SM, depth tile, frames per pack, staged}
    const int shapes[][4] = {{1, 384, 1, 0}, {4, 256, 4, 0}, {5, 256, 4, 0}, {6, 256, 4, 0}, {8, 128, 4, 0},
                             {12, 128, 4, 0}, {3, 256, 8, 0}, {4, 256, 8, 0}, {5, 256, 8, 0}, {8, 128, 8, 0}, {1, 128, 4, 1},
                             {1, 128, 2, 1},  {2, 128, 2, 1}};
    float best = 1e30f;
    int bestC = p->ctasPerSm, bestT = p->nt, bestF = p->fp, bestG = p->staged;
    cudaEvent_t e0, e1;
    SB_CUDA(cudaEventCreate(&e0));
    SB_CUDA(cudaEventCreate(&e1));
    for (const auto& sh : shapes) {
        if (sh[2] == 1 && batchMaxW(p->maxCh, p->maxD, sh[0]) < 64) continue;
        int r = launchBatch(p, sh[1], sh[0], sh[2], sh[3], st);  // warm-up (builds pack tables)
        if (r != SB_OK) continue;
        SB_CUDA(cudaEventRecord(e0, st));
        for (int i = 0; i < 3; i++) {
            r = launchBatch(p, sh[1], sh[0], sh[2], sh[3], st);
            if (r != SB_OK) break;
        }
        SB_CUDA(cudaEventRecord(e1, st));
        SB_CUDA(cudaEventSynchronize(e1));
        if (r != SB_OK) continue;
        float ms = 0;
        SB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) {
            best = ms;
            bestC = sh[0];
            bestT = sh[1];
            bestF = sh[2];
            bestG = sh[3];
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    p->ctasPerSm = bestC;
    p->nt = bestT;
    p->fp = bestF;
    p->staged = bestG;
    report();
    if (cache_path) {
        std::ofstream out(cache_path, std::ios::app);
        if (out) out << p->signature << " " << bestC << " " << bestT << " " << bestF << " " << bestG << "\n";
    }
    return SB_OK;
}

}  // extern "C"
