// Envelope detection (Hilbert FIR), log compression and IQ demodulation.
//   HilbertFirEnvelope   Beamformer/HilbertFirEnvelope.cu:28-104
//   LogCompressor        Beamformer/LogCompressor.cu:22-66
//   IQDemodulator        Beamformer/IQDemodulator.cu:68-345 (frequency-compounded magnitude)
// plus a complex baseband IQ demodulator (extension). Images are [sample][scanline], scanline fastest.
#include <cmath>
#include <vector>

#include "common.cuh"
#include "design.h"
#include "envelope.cuh"

namespace sb {

namespace {

// ----------------------------------------------------------------------------- Hilbert envelope
// One thread per (scanline, sample); the filter (plus one zero tap, see Q3 below) sits in shared
// memory. env = sqrt(x^2 + (sum_j x[s - N/2 + j] h[j])^2), j = 0..2*(N/2) with out-of-range samples
// skipped. For even N the reference reads h[N] one past its buffer; here that tap is 0.
template <typename IN, typename OUT>
__global__ void __launch_bounds__(256) hilbertKernel(const IN* __restrict__ in, OUT* __restrict__ out,
                                                     const float* __restrict__ taps, int nS, int nL, int N) {
    extern __shared__ float h[];
    for (int i = threadIdx.y * blockDim.x + threadIdx.x; i <= N; i += blockDim.x * blockDim.y) h[i] = i < N ? taps[i] : 0.0f;
    __syncthreads();
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y * blockDim.y + threadIdx.y;
    if (l >= nL || s >= nS) return;
    float acc = 0.0f;
    const int start = s - N / 2, end = s + N / 2;
    for (int cs = start, fe = 0; cs <= end; cs++, fe++) {
        if (cs >= 0 && cs < nS) acc = __fadd_rn(acc, __fmul_rn(toFloat(in[l + static_cast<size_t>(cs) * nL]), h[fe]));
    }
    const float v = toFloat(in[l + static_cast<size_t>(s) * nL]);
    out[l + static_cast<size_t>(s) * nL] = static_cast<OUT>(__fsqrt_rn(__fadd_rn(__fmul_rn(v, v), __fmul_rn(acc, acc))));
}

// Tiled envelope: a CTA of 8 warps covers 32 scanlines x 8R samples. The input rows it needs (halo
// included) are staged once into shared memory, one column per scanline, so that each lane reads
// its own scanline's samples as aligned float pairs; each lane then computes R consecutive outputs
// of its scanline, two at a time: products by __fmul_rn (never merged into an FMA), running sums
// by __fadd2_rn (two IEEE round-to-nearest additions per instruction). A packed multiply feeding a
// packed add (__fmul2_rn, then __fadd2_rn, as intrinsics or as mul.rn/add.rn.f32x2 in PTX) was
// measured here to round like a fused multiply-add, so the products stay scalar. Every output sums
// its taps in the reference's order with a separately rounded multiply and add per tap, so results
// are bit-identical to hilbertKernel.
// The Hilbert taps at even offsets from the centre are exactly zero; their terms (finite x times
// +-0) are +-0 and leave the running sum unchanged, since a sum that starts at +0 never becomes -0.
// So a tile whose inputs are all finite sums only the nonzero taps (j0 + 2t); a tile holding an
// infinity or NaN, whose zero-tap terms are NaN, sums every tap. Samples outside the record are
// staged as 0, whose terms are +-0 as well (the reference skips them).
constexpr int kHilTileRowsExtra = 8;  // tap padding to a multiple of four, the pair-alignment shift

__host__ __device__ constexpr int hilTileRows(int R, int H) { return 8 * R + 2 * H + kHilTileRowsExtra; }
// column pitch: even (pairs stay 8-byte aligned) with an odd number of pairs (conflict-free pair reads)
__host__ __device__ constexpr int hilTilePitch(int R, int H) {
    return ((hilTileRows(R, H) + 1) & ~1) + ((((hilTileRows(R, H) + 1) & ~1) / 2) % 2 == 0 ? 2 : 0);
}

// four consecutive scanlines of one sample row as floats (a 16-byte or an 8-byte load)
__device__ __forceinline__ float4 load4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ float4 load4(const int16_t* p) {
    const short4 v = __ldg(reinterpret_cast<const short4*>(p));
    return make_float4(v.x, v.y, v.z, v.w);
}

// vec4: the scanline count is a multiple of 4 and the input aligned to 4 elements
template <typename IN, int R, bool LOGC>
__global__ void __launch_bounds__(256) hilbertTileKernel(const IN* __restrict__ in, float* __restrict__ out,
                                                         const float* __restrict__ taps, const float* __restrict__ nzTaps,
                                                         int nS, int nL, int N, int j0, int nz, float inScale, float k,
                                                         bool vec4) {
    extern __shared__ __align__(16) float hsm[];
    const int H = N / 2;
    const int nzPad = (nz + 3) & ~3;
    const int pitch = hilTilePitch(R, H);
    const int rows = hilTileRows(R, H);
    float* T = hsm;                                  // [32 scanlines][pitch]
    float* hAll = T + 32 * pitch;                    // taps 0 .. 2H (h[N] = 0 for even N)
    float* hNz = hAll + ((2 * H + 1 + 3) & ~3);      // nonzero taps, padded with zeros
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    for (int i = tid; i <= 2 * H; i += 256) hAll[i] = i < N ? taps[i] : 0.0f;
    for (int i = tid; i < nzPad; i += 256) hNz[i] = nzTaps[i];
    const int off = j0 & 1;
    const int l0 = blockIdx.x * 32, s0 = blockIdx.y * 8 * R;
    const int l = l0 + lane;
    // position p of a column holds sample s0 - H - off + p (0 outside the record or the image)
    bool bad = false;
    if (vec4) {
        // 4 scanlines x 1 row per thread and load (16 / 8 bytes), 32 rows per CTA pass, 4 passes in flight
        const int g = tid & 7, ro = tid >> 3;
        for (int p0 = ro; p0 < rows; p0 += 128) {
            float4 v[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int p = p0 + 32 * u, s = s0 - H - off + p;
                v[u] = (p < rows && s >= 0 && s < nS && l0 + 4 * g < nL)
                           ? load4(in + l0 + 4 * g + static_cast<size_t>(s) * nL)
                           : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int p = p0 + 32 * u;
                if (p < rows) {
                    bad |= !(isfinite(v[u].x) && isfinite(v[u].y) && isfinite(v[u].z) && isfinite(v[u].w));
                    T[(4 * g) * pitch + p] = v[u].x;
                    T[(4 * g + 1) * pitch + p] = v[u].y;
                    T[(4 * g + 2) * pitch + p] = v[u].z;
                    T[(4 * g + 3) * pitch + p] = v[u].w;
                }
            }
        }
    } else
    // eight rows per warp in flight: all loads of a batch issue before the first store
    for (int p0 = w; p0 < rows; p0 += 64) {
        float v[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int p = p0 + 8 * u, s = s0 - H - off + p;
            v[u] = (p < rows && s >= 0 && s < nS && l < nL) ? toFloat(in[l + static_cast<size_t>(s) * nL]) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int p = p0 + 8 * u;
            if (p < rows) {
                bad |= !isfinite(v[u]);
                T[lane * pitch + p] = v[u];
            }
        }
    }
    const bool anyBad = __syncthreads_or(bad);
    const float* col = T + lane * pitch;
    const int sw = s0 + R * w;  // this warp's first output sample
    float2 acc[R / 2];
#pragma unroll
    for (int q = 0; q < R / 2; q++) acc[q] = make_float2(0.0f, 0.0f);
    if (!anyBad) {
        // output sw + 2q + e (e = 0, 1), nonzero tap t: position R w + 2q + e + j0 + 2t + off, so pair
        // (2q, 2q + 1) at tap t is pair number kb + q + t of the column
        const float2* P = reinterpret_cast<const float2*>(col);
        const int kb = (R * w + j0 + off) >> 1;
        for (int t = 0; t < nzPad; t += 4) {
            float2 xv[R / 2 + 3];
#pragma unroll
            for (int i = 0; i < R / 2 + 3; i++) xv[i] = P[kb + t + i];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const float hv = hNz[t + u];
#pragma unroll
                for (int q = 0; q < R / 2; q++)
                    acc[q] = __fadd2_rn(acc[q], make_float2(__fmul_rn(xv[q + u].x, hv), __fmul_rn(xv[q + u].y, hv)));
            }
        }
    } else {
        float a1[R];
#pragma unroll
        for (int r = 0; r < R; r++) a1[r] = 0.0f;
        for (int j = 0; j <= 2 * H; j++) {
            const float hv = hAll[j];
#pragma unroll
            for (int r = 0; r < R; r++) a1[r] = __fadd_rn(a1[r], __fmul_rn(col[R * w + r + j + off], hv));
        }
#pragma unroll
        for (int q = 0; q < R / 2; q++) acc[q] = make_float2(a1[2 * q], a1[2 * q + 1]);
    }
    if (l >= nL) return;
#pragma unroll
    for (int q = 0; q < R / 2; q++) {
        const int r = 2 * q;
        const float2 v = make_float2(col[R * w + r + H + off], col[R * w + r + 1 + H + off]);
        const float2 e2 = __fadd2_rn(make_float2(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y)),
                                     make_float2(__fmul_rn(acc[q].x, acc[q].x), __fmul_rn(acc[q].y, acc[q].y)));
        float e0 = __fsqrt_rn(e2.x), e1 = __fsqrt_rn(e2.y);
        if (LOGC) {  // LogCompressor to a float image (clampCast<float>)
            e0 = clampCast<float>(logCompress(e0, inScale, k));
            e1 = clampCast<float>(logCompress(e1, inScale, k));
        }
        if (sw + r < nS) out[l + static_cast<size_t>(sw + r) * nL] = e0;
        if (sw + r + 1 < nS) out[l + static_cast<size_t>(sw + r + 1) * nL] = e1;
    }
}

// Adjoint of the envelope (extension without a reference counterpart): env = sqrt(x^2 + h^2) with
// h = taps (*) x along the samples, so dL/dx[j] = G[j] x[j] / env[j] + sum_s q[s] taps[j - s + N/2]
// with q[s] = G[s] h[s] / env[s] (0 where env = 0). Pass 1 writes the direct term and q, pass 2
// adds the correlation of q with the taps.
__global__ void __launch_bounds__(256) hilbertAdjQKernel(const float* __restrict__ in, const float* __restrict__ genv,
                                                         float* __restrict__ gin, float* __restrict__ q,
                                                         const float* __restrict__ taps, int nS, int nL, int N) {
    extern __shared__ float h[];
    for (int i = threadIdx.y * blockDim.x + threadIdx.x; i <= N; i += blockDim.x * blockDim.y) h[i] = i < N ? taps[i] : 0.0f;
    __syncthreads();
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y * blockDim.y + threadIdx.y;
    if (l >= nL || s >= nS) return;
    float acc = 0.0f;
    const int start = s - N / 2, end = s + N / 2;
    for (int cs = start, fe = 0; cs <= end; cs++, fe++) {
        if (cs >= 0 && cs < nS) acc = __fadd_rn(acc, __fmul_rn(in[l + static_cast<size_t>(cs) * nL], h[fe]));
    }
    const size_t o = l + static_cast<size_t>(s) * nL;
    const float v = in[o];
    const float env = __fsqrt_rn(__fadd_rn(__fmul_rn(v, v), __fmul_rn(acc, acc)));
    const float g = genv[o];
    const bool ok = env > 0.0f;
    gin[o] = ok ? g * v / env : 0.0f;
    q[o] = ok ? g * acc / env : 0.0f;
}

__global__ void __launch_bounds__(256) hilbertAdjCorrKernel(const float* __restrict__ q, float* __restrict__ gin,
                                                            const float* __restrict__ taps, int nS, int nL, int N) {
    extern __shared__ float h[];
    for (int i = threadIdx.y * blockDim.x + threadIdx.x; i <= N; i += blockDim.x * blockDim.y) h[i] = i < N ? taps[i] : 0.0f;
    __syncthreads();
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (l >= nL || j >= nS) return;
    float acc = 0.0f;
    for (int fe = 0; fe <= 2 * (N / 2); fe++) {
        const int s = j + N / 2 - fe;
        if (s >= 0 && s < nS) acc += q[l + static_cast<size_t>(s) * nL] * h[fe];
    }
    gin[l + static_cast<size_t>(j) * nL] += acc;
}

// clampCast of a buffer (element type conversion between nodes).
template <typename IN, typename OUT>
__global__ void convertKernel(const IN* __restrict__ in, OUT* __restrict__ out, size_t n) {
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n; i += stride)
        out[i] = clampCast<OUT>(toFloat(in[i]));
}

// ----------------------------------------------------------------------------- log compression
template <typename IN, typename OUT>
__global__ void logKernel(const IN* __restrict__ in, OUT* __restrict__ out, size_t n, float inScale, float k) {
    size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    for (; i < n; i += stride) out[i] = clampCast<OUT>(logCompress(toFloat(in[i]), inScale, k));
}

// Four elements per thread as one vector load and one vector store, evict-first (the image streams
// through once); the last n % 4 elements by the first thread. Input and output aligned to 4 elements.
template <typename T> struct Vec4;
template <> struct Vec4<float> {
    using type = float4;
    static __device__ __forceinline__ float4 make(float a, float b, float c, float d) { return make_float4(a, b, c, d); }
};
template <> struct Vec4<int16_t> {
    using type = short4;
    static __device__ __forceinline__ short4 make(int16_t a, int16_t b, int16_t c, int16_t d) { return make_short4(a, b, c, d); }
};
template <> struct Vec4<uint8_t> {
    using type = uchar4;
    static __device__ __forceinline__ uchar4 make(uint8_t a, uint8_t b, uint8_t c, uint8_t d) { return make_uchar4(a, b, c, d); }
};

// Grid-stride over groups of four: each thread loads kLogU groups before converting any, so that
// their loads are in flight together (one group per short-lived thread left the kernel waiting on
// load latency at about half its issue rate).
constexpr int kLogU = 4;

template <typename IN, typename OUT>
__global__ void __launch_bounds__(256) logKernel4(const IN* __restrict__ in, OUT* __restrict__ out, size_t n, float inScale,
                                                  float k) {
    using VI = typename Vec4<IN>::type;
    using VO = typename Vec4<OUT>::type;
    const size_t n4 = n / 4;
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    for (size_t g0 = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; g0 < n4; g0 += stride * kLogU) {
        VI v[kLogU];
#pragma unroll
        for (int u = 0; u < kLogU; u++) {
            const size_t g = g0 + u * stride;
            if (g < n4) v[u] = __ldcs(reinterpret_cast<const VI*>(in) + g);
        }
#pragma unroll
        for (int u = 0; u < kLogU; u++) {
            const size_t g = g0 + u * stride;
            if (g < n4)
                __stcs(reinterpret_cast<VO*>(out) + g,
                       Vec4<OUT>::make(clampCast<OUT>(logCompress(toFloat(v[u].x), inScale, k)),
                                       clampCast<OUT>(logCompress(toFloat(v[u].y), inScale, k)),
                                       clampCast<OUT>(logCompress(toFloat(v[u].z), inScale, k)),
                                       clampCast<OUT>(logCompress(toFloat(v[u].w), inScale, k))));
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        for (size_t i = 4 * n4; i < n; i++) out[i] = clampCast<OUT>(logCompress(toFloat(in[i]), inScale, k));
}

// ----------------------------------------------------------------------------- IQ magnitude
// One CTA = 32 scanlines x OT decimated outputs. Phase 1 evaluates the filter-bank magnitude
// (kernelFilterBankDemodulation, IQDemodulator.cu:68-137) for every input sample the low-pass needs
// and keeps it in shared memory; phase 2 applies the decimating low-pass (kernelFilterStrided
// :142-175). No full-resolution intermediate goes to HBM.
constexpr int IQ_LINES = 32;
constexpr int IQ_OT = 32;

// cos(2 pi ph) for a mixer phase ph in [0, 1): the argument folded into [-pi, pi] (ph - 1 is exact
// for ph > 1/2) and evaluated by the hardware approximation, as the reference's production build
// does (--use_fast_math, SupraLib/CMakeLists.txt:65): absolute error about 2^-21.
__device__ __forceinline__ float mixCos(float ph) {
    const float p = ph > 0.5f ? __fsub_rn(ph, 1.0f) : ph;
    return __cosf(__fmul_rn(__fmul_rn(p, 2.0f), static_cast<float>(M_PI)));
}

template <typename IN, typename OUT>
__global__ void __launch_bounds__(256) iqMagnitudeKernel(const IN* __restrict__ in, OUT* __restrict__ out, IqArgs a) {
    extern __shared__ float sm[];
    __shared__ float lps[kIqMaxTaps + 1];               // the low-pass taps
    float* band = sm;                                   // [rows][IQ_LINES]
    const int rows = (IQ_OT - 1) * a.stride + a.lpN + 1;
    const int l0 = blockIdx.x * IQ_LINES;
    const int so0 = blockIdx.y * IQ_OT;
    const int sIn0 = so0 * a.stride - a.lpN / 2;       // first input sample a low-pass tap touches
    const int tid = threadIdx.x;
    for (int idx = tid; idx < rows * IQ_LINES; idx += blockDim.x) {
        const int row = idx / IQ_LINES, li = idx % IQ_LINES;
        const int s = sIn0 + row, l = l0 + li;
        float v = 0.0f;
        if (l < a.nL && s >= 0 && s < a.nS) {
            // filter loops unrolled over the 8 slots (guarded) so the sums stay in registers
            float acc[8];
            const float sv = toFloat(in[l + static_cast<size_t>(s) * a.nL]);
#pragma unroll
            for (int f = 0; f < 8; f++) acc[f] = f < 1 ? sv : 0.0f;
            if (a.numFilters > 1) {
                const int start = s - a.bpN / 2, end = s + a.bpN / 2;
                for (int cs = start, fe = 0; cs <= end; cs++, fe++) {
                    if (cs >= 0 && cs < a.nS) {
                        const float x = toFloat(in[l + static_cast<size_t>(cs) * a.nL]);
#pragma unroll
                        for (int f = 1; f < 8; f++)
                            if (f < a.numFilters) acc[f] = __fadd_rn(acc[f], __fmul_rn(x, a.bank[f * (a.bpN + 1) + fe]));
                    }
                }
            }
            float m = 0.0f;
#pragma unroll
            for (int f = 0; f < 8; f++) {
                if (f >= a.numFilters) break;
                const float ph = __fmul_rn(static_cast<float>(s), a.fOverFs[f]);
                float phI = __fadd_rn(ph, 0.0f);
                float phQ = __fadd_rn(ph, 0.75f);
                phI = __fsub_rn(phI, truncf(phI));
                phQ = __fsub_rn(phQ, truncf(phQ));
                const float dI = __fmul_rn(acc[f], mixCos(phI));
                const float dQ = __fmul_rn(acc[f], mixCos(phQ));
                m = __fadd_rn(m, __fmul_rn(a.weights[f], __fsqrt_rn(__fadd_rn(__fmul_rn(dI, dI), __fmul_rn(dQ, dQ)))));
            }
            v = __fmul_rn(a.scale, m);
        }
        band[row * IQ_LINES + li] = v;
    }
    for (int j = tid; j <= a.lpN; j += blockDim.x) lps[j] = a.lp[j];
    __syncthreads();
    for (int idx = tid; idx < IQ_OT * IQ_LINES; idx += blockDim.x) {
        const int o = idx / IQ_LINES, li = idx % IQ_LINES;
        const int so = so0 + o, l = l0 + li;
        const int si = so * a.stride;
        if (so >= a.nOut || l >= a.nL || si >= a.nS) continue;
        float acc = 0.0f;
        const int start = si - a.lpN / 2, end = si + a.lpN / 2;
        const float* b = band + (start - sIn0) * IQ_LINES + li;
        if (start >= 0 && end < a.nS) {  // the whole window inside the record
            for (int fe = 0; fe <= end - start; fe++) acc = __fadd_rn(acc, __fmul_rn(b[fe * IQ_LINES], lps[fe]));
        } else {
            for (int cs = start, fe = 0; cs <= end; cs++, fe++) {
                if (cs >= 0 && cs < a.nS) acc = __fadd_rn(acc, __fmul_rn(b[fe * IQ_LINES], lps[fe]));
            }
        }
        out[l + static_cast<size_t>(so) * a.nL] = clampCast<OUT>(acc);
    }
}

// One reference frequency (the common case): the filter-bank stage of sample s is
// scale w0 sqrt((x cI)^2 + (x cQ)^2) with mixer values cI, cQ that depend on s only, i.e. |x| G(s) with
// G(s) = scale w0 sqrt(cI^2 + cQ^2) (equal up to the rounding of the products, ~1e-7 relative).
// A CTA of 32 scanlines x 64 decimated outputs forms cI, cQ and G once per input row and |x| G per
// sample (no halo recomputation of the mixer), then each thread sums 4 outputs of two neighbouring
// scanlines, one shared tap value per step for all 8 (fused multiply-adds, as nvcc contracts the reference's
// `accumulator += sample * filterElement` in its default build). A sample with |x| >= 2^63 or not finite, whose squares may overflow, takes the
// reference's expression (so clamped +-FLT_MAX pixels give the same infinities). Samples outside the
// record are staged as 0: their terms leave the sums unchanged, as the reference skips them.
constexpr int IQ1_OT = 64;
constexpr int IQ1_R = 8;  // outputs per thread (256 threads = 16 scanline pairs x 16 groups of 4 outputs)

template <typename IN, typename OUT>
__global__ void __launch_bounds__(256) iqMagnitude1Kernel(const IN* __restrict__ in, OUT* __restrict__ out, IqArgs a) {
    extern __shared__ float sm[];
    __shared__ float lps[kIqMaxTaps + 1];
    const int rows = (IQ1_OT - 1) * a.stride + a.lpN + 1;
    float* band = sm;                     // [rows][IQ_LINES]
    float* gain = sm + rows * IQ_LINES;   // [rows]
    float2* mix = reinterpret_cast<float2*>(gain + rows + (rows & 1));  // [rows] (cI, cQ), 8-byte aligned
    const int l0 = blockIdx.x * IQ_LINES;
    const int so0 = blockIdx.y * IQ1_OT;
    const int sIn0 = so0 * a.stride - a.lpN / 2;
    const int tid = threadIdx.x;
    for (int r = tid; r < rows; r += blockDim.x) {
        const int s = sIn0 + r;
        float gv = 0.0f, cI = 0.0f, cQ = 0.0f;
        if (s >= 0 && s < a.nS) {
            const float ph = __fmul_rn(static_cast<float>(s), a.fOverFs[0]);
            float phI = __fadd_rn(ph, 0.0f);
            float phQ = __fadd_rn(ph, 0.75f);
            phI = __fsub_rn(phI, truncf(phI));
            phQ = __fsub_rn(phQ, truncf(phQ));
            cI = mixCos(phI);
            cQ = mixCos(phQ);
            gv = __fmul_rn(a.scale, __fmul_rn(a.weights[0], __fsqrt_rn(__fadd_rn(__fmul_rn(cI, cI), __fmul_rn(cQ, cQ)))));
        }
        gain[r] = gv;
        mix[r] = make_float2(cI, cQ);
    }
    for (int j = tid; j <= a.lpN; j += blockDim.x) lps[j] = a.lp[j];
    __syncthreads();
    // the tile's samples, eight loads in flight per thread before any is used
    const int total = rows * IQ_LINES;
    constexpr int kU = 8;
    for (int base = tid; base < total; base += 256 * kU) {
        float xs[kU];
#pragma unroll
        for (int u = 0; u < kU; u++) {
            const int idx = base + u * 256;
            const int s = sIn0 + idx / IQ_LINES, l = l0 + idx % IQ_LINES;
            const bool ok = idx < total && l < a.nL && s >= 0 && s < a.nS;
            xs[u] = ok ? toFloat(in[l + static_cast<size_t>(ok ? s : 0) * a.nL]) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < kU; u++) {
            const int idx = base + u * 256;
            if (idx < total) {
                const int row = idx / IQ_LINES;
                const float x = xs[u];  // 0 outside the record and the image
                float v;
                if (fabsf(x) < 9.22337204e18f) {  // 2^63: x^2 stays finite
                    v = __fmul_rn(fabsf(x), gain[row]);
                } else {
                    const float2 c = mix[row];
                    const float dI = __fmul_rn(x, c.x), dQ = __fmul_rn(x, c.y);
                    v = __fmul_rn(a.scale, __fmul_rn(a.weights[0], __fsqrt_rn(__fadd_rn(__fmul_rn(dI, dI), __fmul_rn(dQ, dQ)))));
                }
                band[idx] = v;
            }
        }
    }
    __syncthreads();
    // a thread: two neighbouring scanlines (one 8-byte shared-memory read per row) x IQ1_R / 2 outputs;
    // the pair's two sums in one packed FMA (two IEEE fused multiply-adds)
    constexpr int kR = IQ1_R / 2;
    const int lp = tid % (IQ_LINES / 2), o0 = (tid / (IQ_LINES / 2)) * kR;
    const float2* b = reinterpret_cast<const float2*>(band) + o0 * a.stride * (IQ_LINES / 2) + lp;
    const int step = a.stride * (IQ_LINES / 2);
    const int nTaps = 2 * (a.lpN / 2) + 1;  // the reference's window [si - lpN/2, si + lpN/2]
    float2 acc[kR];
#pragma unroll
    for (int k = 0; k < kR; k++) acc[k] = make_float2(0.0f, 0.0f);
#pragma unroll 2
    for (int j = 0; j < nTaps; j++) {
        const float t = lps[j];
        const float2 t2 = make_float2(t, t);
        const float2* bj = b + j * (IQ_LINES / 2);
#pragma unroll
        for (int k = 0; k < kR; k++) acc[k] = __ffma2_rn(bj[k * step], t2, acc[k]);
    }
    const int l = l0 + 2 * lp;
#pragma unroll
    for (int k = 0; k < kR; k++) {
        const int so = so0 + o0 + k;
        if (so < a.nOut) {
            if (l < a.nL) out[l + static_cast<size_t>(so) * a.nL] = clampCast<OUT>(acc[k].x);
            if (l + 1 < a.nL) out[l + 1 + static_cast<size_t>(so) * a.nL] = clampCast<OUT>(acc[k].y);
        }
    }
}

// Several reference frequencies (frequency compounding): a CTA of 32 scanlines x 32 decimated outputs
// stages its raw samples (band-pass and low-pass halos included, eight loads in flight per thread)
// and the filter bank in shared memory, forms each filter's mixer values once per input row, then
// evaluates the filter-bank magnitude of a group of neighbouring samples per thread from shared memory in
// the reference's order (IQDemodulator.cu:68-137: band-pass sums over the taps in order, contracted
// into fused multiply-adds as nvcc contracts them; the weighted magnitudes summed over the filters in
// order), and the decimating low-pass as in iqMagnitude1Kernel (four outputs per thread).
constexpr int IQB_OT = 32;
constexpr int IQB_R = 4;
// band rows per thread in the band-pass stage: their windows share all raw reads and tap reads (eight
// rows for two filters, four for three or four, two above: the measured best at 16384 x 2048)
__host__ __device__ constexpr int iqbRowsPerThread(int nf) { return nf <= 2 ? 8 : nf <= 4 ? 4 : 2; }

template <typename IN, typename OUT, int NF>
__global__ void __launch_bounds__(256) iqMagnitudeBankKernel(const IN* __restrict__ in, OUT* __restrict__ out, IqArgs a) {
    extern __shared__ float sm[];
    __shared__ float lps[kIqMaxTaps + 1];
    __shared__ __align__(16) float bank[8 * (kIqMaxTaps + 4)];  // filter rows at a 16-byte pitch
    const int rows = (IQB_OT - 1) * a.stride + a.lpN + 1;  // band rows
    const int hb = a.bpN / 2;
    constexpr int RB = iqbRowsPerThread(NF);
    const int rowsX = rows + 2 * hb + RB - 1;               // raw rows (the last group's windows included)
    constexpr int nf = NF;
    float* raw = sm;                                        // [rowsX][IQ_LINES]
    float* band = raw + rowsX * IQ_LINES;                   // [rows][IQ_LINES]
    float2* mix = reinterpret_cast<float2*>(band + rows * IQ_LINES);  // [rows][nf] (cI, cQ); offsets even
    const int l0 = blockIdx.x * IQ_LINES;
    const int so0 = blockIdx.y * IQB_OT;
    const int sIn0 = so0 * a.stride - a.lpN / 2;
    const int sX0 = sIn0 - hb;
    const int tid = threadIdx.x;
    const int bs = (a.bpN + 1 + 3) & ~3;  // bank row pitch (floats)
    for (int j = tid; j < nf * bs; j += blockDim.x) {
        const int f = j / bs, k = j % bs;
        bank[j] = k <= a.bpN ? a.bank[f * (a.bpN + 1) + k] : 0.0f;
    }
    for (int j = tid; j <= a.lpN; j += blockDim.x) lps[j] = a.lp[j];
    for (int k = tid; k < rows * nf; k += blockDim.x) {
        const int r = k / nf, f = k % nf;
        const int s = sIn0 + r;
        const float ph = __fmul_rn(static_cast<float>(s), a.fOverFs[f]);
        float phI = __fadd_rn(ph, 0.0f);
        float phQ = __fadd_rn(ph, 0.75f);
        phI = __fsub_rn(phI, truncf(phI));
        phQ = __fsub_rn(phQ, truncf(phQ));
        mix[k] = make_float2(mixCos(phI), mixCos(phQ));
    }
    const int totalX = rowsX * IQ_LINES;
    constexpr int kU = 8;
    for (int base = tid; base < totalX; base += 256 * kU) {
        float xs[kU];
#pragma unroll
        for (int u = 0; u < kU; u++) {
            const int idx = base + u * 256;
            const int s = sX0 + idx / IQ_LINES, l = l0 + idx % IQ_LINES;
            const bool ok = idx < totalX && l < a.nL && s >= 0 && s < a.nS;
            xs[u] = ok ? toFloat(in[l + static_cast<size_t>(ok ? s : 0) * a.nL]) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < kU; u++)
            if (base + u * 256 < totalX) raw[base + u * 256] = xs[u];
    }
    __syncthreads();
    // RB neighbouring rows per thread: their band-pass windows overlap, so each raw value and each tap
    // is read once for all of them (fused multiply-adds, as nvcc contracts the reference's
    // `accumulators[filter] += sample * filterElement`; every row sums its taps in order). Raw value e
    // of the group meets tap e - h of row h; tp[f][h] holds filter f's tap e - h. Out-of-record samples
    // are staged as 0 and add nothing, as the reference skips them.
    const float* bk = bank + bs;
    const int W = 2 * hb;  // last tap
    const int nGroups = (rows + RB - 1) / RB;
    for (int idx = tid; idx < nGroups * IQ_LINES; idx += blockDim.x) {
        const int row = RB * (idx / IQ_LINES), li = idx % IQ_LINES;
        const float* xr = raw + row * IQ_LINES + li;
        float acc[RB][NF], tp[NF][RB];
#pragma unroll
        for (int h = 0; h < RB; h++) {
            acc[h][0] = xr[(hb + h) * IQ_LINES];
#pragma unroll
            for (int f = 1; f < NF; f++) {
                acc[h][f] = 0.0f;
                tp[f][h] = 0.0f;
            }
        }
        if (W >= RB - 1) {
            // e < RB - 1: rows h <= e have begun
#pragma unroll
            for (int e = 0; e < RB - 1; e++) {
                const float x = xr[e * IQ_LINES];
#pragma unroll
                for (int f = 1; f < NF; f++) {
#pragma unroll
                    for (int k = RB - 1; k > 0; k--) tp[f][k] = tp[f][k - 1];
                    tp[f][0] = bk[(f - 1) * bs + e];
#pragma unroll
                    for (int h = 0; h <= e; h++) acc[h][f] = fmaf(x, tp[f][h], acc[h][f]);
                }
            }
            // every row of the group takes a tap: single steps up to a multiple of four, then four steps
            // per iteration with each filter's four taps in one 16-byte read, then single steps
            auto step = [&](int e, const float (&tv)[NF]) {
                const float x = xr[e * IQ_LINES];
#pragma unroll
                for (int f = 1; f < NF; f++) {
#pragma unroll
                    for (int k = RB - 1; k > 0; k--) tp[f][k] = tp[f][k - 1];
                    tp[f][0] = tv[f];
#pragma unroll
                    for (int h = 0; h < RB; h++) acc[h][f] = fmaf(x, tp[f][h], acc[h][f]);
                }
            };
            int e = RB - 1;
            for (; e <= W && (e & 3); e++) {
                float tv[NF];
#pragma unroll
                for (int f = 1; f < NF; f++) tv[f] = bk[(f - 1) * bs + e];
                step(e, tv);
            }
            for (; e + 3 <= W; e += 4) {
                float4 t4[NF];
#pragma unroll
                for (int f = 1; f < NF; f++) t4[f] = *reinterpret_cast<const float4*>(bk + (f - 1) * bs + e);
                float tv[NF];
#pragma unroll
                for (int f = 1; f < NF; f++) tv[f] = t4[f].x;
                step(e, tv);
#pragma unroll
                for (int f = 1; f < NF; f++) tv[f] = t4[f].y;
                step(e + 1, tv);
#pragma unroll
                for (int f = 1; f < NF; f++) tv[f] = t4[f].z;
                step(e + 2, tv);
#pragma unroll
                for (int f = 1; f < NF; f++) tv[f] = t4[f].w;
                step(e + 3, tv);
            }
            for (; e <= W; e++) {
                float tv[NF];
#pragma unroll
                for (int f = 1; f < NF; f++) tv[f] = bk[(f - 1) * bs + e];
                step(e, tv);
            }
            // e = W + i: rows h > i - 1 still take tap e - h
#pragma unroll
            for (int i = 1; i < RB; i++) {
                const float x = xr[(W + i) * IQ_LINES];
#pragma unroll
                for (int f = 1; f < NF; f++) {
#pragma unroll
                    for (int k = RB - 1; k > 0; k--) tp[f][k] = tp[f][k - 1];
#pragma unroll
                    for (int h = i; h < RB; h++) acc[h][f] = fmaf(x, tp[f][h], acc[h][f]);
                }
            }
        } else {
            // filters shorter than the group: the same sums with the tap range tested per row
            for (int e = 0; e <= W + RB - 1; e++) {
                const float x = xr[e * IQ_LINES];
#pragma unroll
                for (int f = 1; f < NF; f++) {
#pragma unroll
                    for (int h = 0; h < RB; h++) {
                        const int fe = e - h;
                        if (fe >= 0 && fe <= W) acc[h][f] = fmaf(x, bk[(f - 1) * bs + fe], acc[h][f]);
                    }
                }
            }
        }
#pragma unroll
        for (int h = 0; h < RB; h++) {
            const int rr = row + h;
            const int s = sIn0 + rr, l = l0 + li;
            if (rr >= rows) break;
            float v = 0.0f;
            if (l < a.nL && s >= 0 && s < a.nS) {
                float m = 0.0f;
#pragma unroll
                for (int f = 0; f < NF; f++) {
                    const float av = acc[h][f];
                    const float2 c = mix[rr * nf + f];
                    const float dI = __fmul_rn(av, c.x), dQ = __fmul_rn(av, c.y);
                    m = __fadd_rn(m, __fmul_rn(a.weights[f], __fsqrt_rn(__fadd_rn(__fmul_rn(dI, dI), __fmul_rn(dQ, dQ)))));
                }
                v = __fmul_rn(a.scale, m);
            }
            band[rr * IQ_LINES + li] = v;
        }
    }
    __syncthreads();
    const int li = tid % IQ_LINES, o0 = (tid / IQ_LINES) * IQB_R;
    const float* b = band + o0 * a.stride * IQ_LINES + li;
    const int step = a.stride * IQ_LINES;
    const int nTaps = 2 * (a.lpN / 2) + 1;
    float acc[IQB_R];
#pragma unroll
    for (int k = 0; k < IQB_R; k++) acc[k] = 0.0f;
#pragma unroll 2
    for (int j = 0; j < nTaps; j++) {
        const float t = lps[j];
        const float* bj = b + j * IQ_LINES;
#pragma unroll
        for (int k = 0; k < IQB_R; k++) acc[k] = fmaf(bj[k * step], t, acc[k]);
    }
    const int l = l0 + li;
#pragma unroll
    for (int k = 0; k < IQB_R; k++) {
        const int so = so0 + o0 + k;
        if (so < a.nOut && l < a.nL) out[l + static_cast<size_t>(so) * a.nL] = clampCast<OUT>(acc[k]);
    }
}

// ----------------------------------------------------------------------------- complex IQ
template <typename IN>
__global__ void __launch_bounds__(256) iqComplexKernel(const IN* __restrict__ in, float2* __restrict__ out,
                                                       IqComplexArgs a) {
    extern __shared__ float sm[];
    const int rows = (IQ_OT - 1) * a.dec + a.taps;
    float* xs = sm;                         // [rows][IQ_LINES]
    float2* rot = reinterpret_cast<float2*>(xs + rows * IQ_LINES);  // [rows]
    const int l0 = blockIdx.x * IQ_LINES;
    const int so0 = blockIdx.y * IQ_OT;
    const int s0 = so0 * a.dec - a.half;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) {
        const int n = s0 + r;
        double ph = static_cast<double>(a.fOverFs) * n;
        ph -= floor(ph);
        float sn, cs;
        sincospif(static_cast<float>(2.0 * ph), &sn, &cs);
        rot[r] = make_float2(cs, -sn);
    }
    for (int idx = threadIdx.x; idx < rows * IQ_LINES; idx += blockDim.x) {
        const int r = idx / IQ_LINES, li = idx % IQ_LINES;
        const int s = s0 + r, l = l0 + li;
        xs[idx] = (l < a.nL && s >= 0 && s < a.nS) ? toFloat(in[l + static_cast<size_t>(s) * a.nL]) : 0.0f;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < IQ_OT * IQ_LINES; idx += blockDim.x) {
        const int o = idx / IQ_LINES, li = idx % IQ_LINES;
        const int so = so0 + o, l = l0 + li;
        if (so >= a.nOut || l >= a.nL) continue;
        float re = 0.0f, im = 0.0f;
        const int rb = o * a.dec;
        for (int j = 0; j < a.taps; j++) {
            const float x = xs[(rb + j) * IQ_LINES + li] * a.lp[j];
            const float2 w = rot[rb + j];
            re = fmaf(x, w.x, re);
            im = fmaf(x, w.y, im);
        }
        out[l + static_cast<size_t>(so) * a.nL] = make_float2(re, im);
    }
}

}  // namespace

int launchLog(const void* in, int inDt, void* out, int outDt, size_t n, float inScale, float k, cudaStream_t st) {
    if (n == 0) return SB_OK;
    const size_t inB = inDt == SB_FLOAT32 ? 4 : inDt == SB_INT16 ? 2 : 1;
    const size_t outB = outDt == SB_FLOAT32 ? 4 : 1;
    const bool vec = reinterpret_cast<uintptr_t>(in) % (4 * inB) == 0 && reinterpret_cast<uintptr_t>(out) % (4 * outB) == 0 &&
                     (n / 4 + 255) / 256 <= 0x7fffffffu;
    int blocks = static_cast<int>(std::min<size_t>((n + 255) / 256, static_cast<size_t>(smCount()) * 16));
    if (blocks < 1) blocks = 1;
    // four resident CTAs per SM (55-57 registers), each thread kLogU groups of four per step
    const unsigned blocks4 = static_cast<unsigned>(std::max<size_t>(
        std::min<size_t>((n / 4 + 256 * kLogU - 1) / (256 * kLogU), static_cast<size_t>(smCount()) * 4), 1));
#define SB_LOG(INT, OUTT)                                                                                                  \
    do {                                                                                                                   \
        if (vec) logKernel4<INT, OUTT><<<blocks4, 256, 0, st>>>(static_cast<const INT*>(in), static_cast<OUTT*>(out), n, inScale, k); \
        else logKernel<INT, OUTT><<<blocks, 256, 0, st>>>(static_cast<const INT*>(in), static_cast<OUTT*>(out), n, inScale, k);       \
    } while (0)
    if (inDt == SB_FLOAT32 && outDt == SB_UINT8) SB_LOG(float, uint8_t);
    else if (inDt == SB_FLOAT32 && outDt == SB_FLOAT32) SB_LOG(float, float);
    else if (inDt == SB_INT16 && outDt == SB_UINT8) SB_LOG(int16_t, uint8_t);
    else if (inDt == SB_INT16 && outDt == SB_FLOAT32) SB_LOG(int16_t, float);
    else if (inDt == SB_UINT8 && outDt == SB_UINT8) SB_LOG(uint8_t, uint8_t);
    else if (inDt == SB_UINT8 && outDt == SB_FLOAT32) SB_LOG(uint8_t, float);
    else return fail(SB_ERR_UNSUPPORTED, "log compression %d -> %d unsupported", inDt, outDt);
#undef SB_LOG
    SB_CHECK_LAUNCH("logKernel");
    return SB_OK;
}

int launchHilbert(const sb_hilbert_plan* p, const void* in, int inDt, float* out, int nS, int nL, bool logc,
                  float inScale, float k, cudaStream_t st) {
    const int N = static_cast<int>(p->N), H = N / 2;
    const int tiles16 = ((nL + 31) / 32) * ((nS + 127) / 128);
    const int R = tiles16 >= 2 * smCount() ? 16 : 4;
    const int nzPad = (p->nz + 3) & ~3;
    const size_t shm = (static_cast<size_t>(32) * hilTilePitch(R, H) + ((2 * H + 1 + 3) & ~3) + nzPad) * sizeof(float);
    if (p->nz > 0 && shm <= 48 * 1024 && (inDt == SB_FLOAT32 || inDt == SB_INT16)) {
        const dim3 grid((nL + 31) / 32, (nS + 8 * R - 1) / (8 * R));
        const size_t eb = inDt == SB_FLOAT32 ? 4 : 2;
        const bool vec4 = nL % 4 == 0 && reinterpret_cast<uintptr_t>(in) % (4 * eb) == 0;
#define SB_HT(INT, RR, LG)                                                                                           \
    hilbertTileKernel<INT, RR, LG><<<grid, 256, shm, st>>>(static_cast<const INT*>(in), out, p->dTaps, p->dNz, nS, nL, \
                                                           N, p->j0, p->nz, inScale, k, vec4)
        if (inDt == SB_FLOAT32) {
            if (R == 16) { if (logc) SB_HT(float, 16, true); else SB_HT(float, 16, false); }
            else { if (logc) SB_HT(float, 4, true); else SB_HT(float, 4, false); }
        } else {
            if (R == 16) { if (logc) SB_HT(int16_t, 16, true); else SB_HT(int16_t, 16, false); }
            else { if (logc) SB_HT(int16_t, 4, true); else SB_HT(int16_t, 4, false); }
        }
#undef SB_HT
        SB_CHECK_LAUNCH("hilbertTileKernel");
        return SB_OK;
    }
    // other filters (no zero-tap pattern, or longer than the tile allows): one thread per output
    dim3 block(32, 8);
    dim3 grid((nL + 31) / 32, (nS + 7) / 8);
    const size_t shm1 = (p->N + 1) * sizeof(float);
    if (inDt == SB_FLOAT32)
        hilbertKernel<float, float><<<grid, block, shm1, st>>>(static_cast<const float*>(in), out, p->dTaps, nS, nL, N);
    else if (inDt == SB_INT16)
        hilbertKernel<int16_t, float><<<grid, block, shm1, st>>>(static_cast<const int16_t*>(in), out, p->dTaps, nS, nL, N);
    else
        return fail(SB_ERR_UNSUPPORTED, "sb_hilbert_env_run: input dtype %d unsupported", inDt);
    SB_CHECK_LAUNCH("hilbertKernel");
    if (logc) return launchLog(out, SB_FLOAT32, out, SB_FLOAT32, static_cast<size_t>(nS) * nL, inScale, k, st);
    return SB_OK;
}

// LogCompressor constants (LogCompressor.cu:22-34, :44-64): inScale = 10^(DR/20) / inMax and
// k = gain * outMax / log10(10^(DR/20) + 1), both rounded to float from double.
void logConstants(double dynamicRange, double gain, double inMax, int inDt, float& inScale, float& k) {
    double dr = std::pow(10, (dynamicRange / 20));
    double inMaxT = inDt == SB_INT16   ? static_cast<double>(static_cast<int16_t>(inMax))
                    : inDt == SB_UINT8 ? static_cast<double>(static_cast<uint8_t>(inMax))
                                       : static_cast<double>(static_cast<float>(inMax));
    inScale = static_cast<float>(dr / inMaxT);
    k = static_cast<float>(gain * 255.0 / std::log10(dr + 1));
}

}  // namespace sb

using namespace sb;

struct sb_iq_plan {
    sb::IqArgs args;  // filters embedded by value
};

extern "C" {

int sb_hilbert_plan_create(uint32_t filter_length, sb_hilbert_plan** plan) {
    SB_REQUIRE(plan && filter_length >= 1 && filter_length <= 1024, "sb_hilbert_plan_create: filter length %u", filter_length);
    *plan = nullptr;
    std::vector<float> taps = firDesign(filter_length, 3, 2, 2.0, 0.0, 0.0);
    sb_hilbert_plan* p = new sb_hilbert_plan{filter_length, nullptr, 0, 0, nullptr};
    // nonzero taps among j = 0 .. 2 (N / 2) (tap N of an even-length filter is 0): j0, j0 + 2, ...?
    std::vector<int> nzIdx;
    for (int j = 0; j <= 2 * static_cast<int>(filter_length / 2); j++)
        if (j < static_cast<int>(filter_length) && taps[j] != 0.0f) nzIdx.push_back(j);
    bool stride2 = !nzIdx.empty();
    for (size_t t = 1; t < nzIdx.size(); t++) stride2 = stride2 && nzIdx[t] == nzIdx[0] + 2 * static_cast<int>(t);
    std::vector<float> nzTaps;
    if (stride2) {
        p->j0 = nzIdx[0];
        p->nz = static_cast<int>(nzIdx.size());
        for (int j : nzIdx) nzTaps.push_back(taps[j]);
        while (nzTaps.size() % 4) nzTaps.push_back(0.0f);
    }
    cudaError_t e = cudaMalloc(&p->dTaps, filter_length * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(p->dTaps, taps.data(), filter_length * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !nzTaps.empty()) e = cudaMalloc(&p->dNz, nzTaps.size() * sizeof(float));
    if (e == cudaSuccess && !nzTaps.empty())
        e = cudaMemcpy(p->dNz, nzTaps.data(), nzTaps.size() * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(p->dTaps);
        cudaFree(p->dNz);
        delete p;
        return cudaFail(e, "sb_hilbert_plan_create");
    }
    *plan = p;
    return SB_OK;
}

int sb_hilbert_plan_destroy(sb_hilbert_plan* p) {
    if (!p) return SB_OK;
    cudaFree(p->dTaps);
    cudaFree(p->dNz);
    delete p;
    return SB_OK;
}

int sb_hilbert_env_run(const sb_hilbert_plan* p, const void* in, int in_dtype, void* out, int out_dtype,
                       uint32_t num_scanlines, uint32_t num_samples, sb_stream stream) {
    SB_REQUIRE(p && in && out, "sb_hilbert_env_run: null argument");
    SB_REQUIRE(num_scanlines > 0 && num_samples > 0, "sb_hilbert_env_run: empty image");
    SB_REQUIRE(num_scanlines <= INT32_MAX && num_samples <= INT32_MAX, "sb_hilbert_env_run: image too large");
    if (!((in_dtype == SB_FLOAT32 || in_dtype == SB_INT16) && out_dtype == SB_FLOAT32))
        return fail(SB_ERR_UNSUPPORTED, "sb_hilbert_env_run: %d -> %d unsupported", in_dtype, out_dtype);
    return launchHilbert(p, in, in_dtype, static_cast<float*>(out), static_cast<int>(num_samples),
                         static_cast<int>(num_scanlines), false, 0.0f, 0.0f, S(stream));
}

int sb_hilbert_env_adjoint(const sb_hilbert_plan* p, const float* in, const float* grad_env, float* grad_in,
                           uint32_t num_scanlines, uint32_t num_samples, sb_stream stream) {
    SB_REQUIRE(p && in && grad_env && grad_in, "sb_hilbert_env_adjoint: null argument");
    SB_REQUIRE(num_scanlines > 0 && num_samples > 0, "sb_hilbert_env_adjoint: empty image");
    cudaStream_t st = S(stream);
    dim3 block(32, 8);
    dim3 grid((num_scanlines + 31) / 32, (num_samples + 7) / 8);
    size_t shm = (p->N + 1) * sizeof(float);
    int nS = static_cast<int>(num_samples), nL = static_cast<int>(num_scanlines), N = static_cast<int>(p->N);
    float* q = nullptr;
    SB_CUDA(cudaMallocAsync(&q, static_cast<size_t>(nS) * nL * sizeof(float), st));
    hilbertAdjQKernel<<<grid, block, shm, st>>>(in, grad_env, grad_in, q, p->dTaps, nS, nL, N);
    hilbertAdjCorrKernel<<<grid, block, shm, st>>>(q, grad_in, p->dTaps, nS, nL, N);
    cudaError_t e = cudaGetLastError();
    cudaFreeAsync(q, st);
    if (e != cudaSuccess) return cudaFail(e, "sb_hilbert_env_adjoint");
    return SB_OK;
}

int sb_convert_run(const void* in, int in_dtype, void* out, int out_dtype, size_t n, sb_stream stream) {
    SB_REQUIRE(in && out, "sb_convert_run: null argument");
    if (n == 0) return SB_OK;
    cudaStream_t st = S(stream);
    const int threads = 256;
    const int blocks = static_cast<int>(std::min<size_t>((n + threads - 1) / threads, 148u * 16u));
#define SB_CONVERT(IT, OT) convertKernel<IT, OT><<<blocks, threads, 0, st>>>(static_cast<const IT*>(in), static_cast<OT*>(out), n)
    if (in_dtype == SB_FLOAT32 && out_dtype == SB_FLOAT32) SB_CONVERT(float, float);
    else if (in_dtype == SB_FLOAT32 && out_dtype == SB_INT16) SB_CONVERT(float, int16_t);
    else if (in_dtype == SB_FLOAT32 && out_dtype == SB_UINT8) SB_CONVERT(float, uint8_t);
    else if (in_dtype == SB_FLOAT32 && out_dtype == SB_UINT16) SB_CONVERT(float, uint16_t);
    else if (in_dtype == SB_INT16 && out_dtype == SB_FLOAT32) SB_CONVERT(int16_t, float);
    else if (in_dtype == SB_INT16 && out_dtype == SB_UINT8) SB_CONVERT(int16_t, uint8_t);
    else return fail(SB_ERR_UNSUPPORTED, "sb_convert_run: %d -> %d unsupported", in_dtype, out_dtype);
#undef SB_CONVERT
    SB_CHECK_LAUNCH("convertKernel");
    return SB_OK;
}

int sb_logcompress_run(const void* in, int in_dtype, void* out, int out_dtype, size_t num_values,
                       double dynamic_range_db, double gain, double in_max, sb_stream stream) {
    SB_REQUIRE(in && out, "sb_logcompress_run: null argument");
    SB_REQUIRE(in_max > 0 && dynamic_range_db > 0, "sb_logcompress_run: inMax and dynamic range must be > 0");
    if (num_values == 0) return SB_OK;
    float inScale, k;
    logConstants(dynamic_range_db, gain, in_max, in_dtype, inScale, k);
    return launchLog(in, in_dtype, out, out_dtype, num_values, inScale, k, S(stream));
}

int sb_iq_plan_create(double fs, double cutoff, uint32_t lpLen, uint32_t bpLen, uint32_t numFilters,
                      const double* refFreqs, const double* bandwidths, const double* weights, sb_iq_plan** plan) {
    SB_REQUIRE(plan && refFreqs && bandwidths && weights, "sb_iq_plan_create: null argument");
    SB_REQUIRE(numFilters >= 1 && numFilters <= 8, "sb_iq_plan_create: 1..8 filters, got %u", numFilters);
    SB_REQUIRE(lpLen >= 1 && lpLen <= kIqMaxTaps - 1 && bpLen >= 1 && bpLen <= kIqMaxTaps - 1,
               "sb_iq_plan_create: filter lengths must be in [1, %d]", kIqMaxTaps - 1);
    SB_REQUIRE(fs > 0 && cutoff > 0, "sb_iq_plan_create: frequencies must be > 0");
    sb_iq_plan* p = new sb_iq_plan();
    IqArgs& a = p->args;
    a.numFilters = static_cast<int>(numFilters);
    a.bpN = static_cast<int>(bpLen);
    a.lpN = static_cast<int>(lpLen);
    float weightAcum = 0;
    for (uint32_t k = 0; k < numFilters; k++) {
        std::vector<float> bp = (refFreqs[k] > 0 && bandwidths[k] > 0) ? firDesign(bpLen, 2, 3, fs, refFreqs[k], bandwidths[k])
                                                                       : std::vector<float>(bpLen, 0.0f);
        for (uint32_t j = 0; j <= bpLen; j++) a.bank[k * (bpLen + 1) + j] = j < bpLen ? bp[j] : 0.0f;
        a.weights[k] = static_cast<float>(weights[k]);
        weightAcum += static_cast<float>(weights[k]);
        a.fOverFs[k] = static_cast<float>(refFreqs[k] / fs);
    }
    a.scale = 1 / weightAcum;
    std::vector<float> lp = firDesign(lpLen, 0, 2, fs, cutoff, 0.0);
    for (uint32_t j = 0; j <= lpLen; j++) a.lp[j] = j < lpLen ? lp[j] : 0.0f;
    *plan = p;
    return SB_OK;
}

int sb_iq_plan_destroy(sb_iq_plan* p) {
    delete p;
    return SB_OK;
}

int sb_iq_magnitude_run(const sb_iq_plan* p, const void* in, int in_dtype, void* out, int out_dtype,
                        uint32_t num_scanlines, uint32_t num_samples, uint32_t decimation, sb_stream stream) {
    SB_REQUIRE(p && in && out, "sb_iq_magnitude_run: null argument");
    SB_REQUIRE(num_scanlines > 0 && num_samples > 0, "sb_iq_magnitude_run: empty image");
    IqArgs a = p->args;
    a.nS = static_cast<int>(num_samples);
    a.nL = static_cast<int>(num_scanlines);
    a.stride = static_cast<int>(std::max(decimation, 1u));
    a.nOut = decimation > 1 ? a.nS / static_cast<int>(decimation) : a.nS;
    if (a.nOut == 0) return SB_OK;
    cudaStream_t st = S(stream);
    const int rows1 = (IQ1_OT - 1) * a.stride + a.lpN + 1;
    const size_t shm1 = (static_cast<size_t>(rows1) * (IQ_LINES + 1) + (rows1 & 1) + 2 * static_cast<size_t>(rows1)) * sizeof(float);
    if (a.numFilters == 1 && shm1 <= 100 * 1024) {
        dim3 grid1((a.nL + IQ_LINES - 1) / IQ_LINES, (a.nOut + IQ1_OT - 1) / IQ1_OT);
        SB_REQUIRE(grid1.y <= 65535u, "sb_iq_magnitude_run: %d outputs exceed the grid", a.nOut);
#define SB_IQ1(INT, OUTT)                                                                                         \
    do {                                                                                                          \
        SB_CUDA(cudaFuncSetAttribute(iqMagnitude1Kernel<INT, OUTT>, cudaFuncAttributeMaxDynamicSharedMemorySize,  \
                                     static_cast<int>(shm1)));                                                    \
        iqMagnitude1Kernel<INT, OUTT><<<grid1, 256, shm1, st>>>(static_cast<const INT*>(in), static_cast<OUTT*>(out), a); \
        SB_CHECK_LAUNCH("iqMagnitude1Kernel");                                                                    \
        return SB_OK;                                                                                             \
    } while (0)
        if (in_dtype == SB_FLOAT32 && out_dtype == SB_FLOAT32) SB_IQ1(float, float);
        if (in_dtype == SB_INT16 && out_dtype == SB_FLOAT32) SB_IQ1(int16_t, float);
        if (in_dtype == SB_FLOAT32 && out_dtype == SB_INT16) SB_IQ1(float, int16_t);
        if (in_dtype == SB_INT16 && out_dtype == SB_INT16) SB_IQ1(int16_t, int16_t);
#undef SB_IQ1
        return fail(SB_ERR_UNSUPPORTED, "sb_iq_magnitude_run: %d -> %d unsupported", in_dtype, out_dtype);
    }
    const int rowsB = (IQB_OT - 1) * a.stride + a.lpN + 1;
    const int rowsBX = rowsB + 2 * (a.bpN / 2) + iqbRowsPerThread(static_cast<int>(a.numFilters)) - 1;
    const size_t shmB = (static_cast<size_t>(rowsBX + rowsB) * IQ_LINES + 2 * static_cast<size_t>(rowsB) * a.numFilters) * sizeof(float);
    if (a.numFilters > 1 && shmB <= 150 * 1024) {
        dim3 gridB((a.nL + IQ_LINES - 1) / IQ_LINES, (a.nOut + IQB_OT - 1) / IQB_OT);
        SB_REQUIRE(gridB.y <= 65535u, "sb_iq_magnitude_run: %d outputs exceed the grid", a.nOut);
#define SB_IQBN(INT, OUTT, NF)                                                                                       \
    do {                                                                                                             \
        SB_CUDA(cudaFuncSetAttribute(iqMagnitudeBankKernel<INT, OUTT, NF>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                     static_cast<int>(shmB)));                                                       \
        iqMagnitudeBankKernel<INT, OUTT, NF><<<gridB, 256, shmB, st>>>(static_cast<const INT*>(in), static_cast<OUTT*>(out), a); \
    } while (0)
#define SB_IQB(INT, OUTT)                                                                                            \
    do {                                                                                                             \
        switch (a.numFilters) {                                                                                      \
            case 2: SB_IQBN(INT, OUTT, 2); break;                                                                    \
            case 3: SB_IQBN(INT, OUTT, 3); break;                                                                    \
            case 4: SB_IQBN(INT, OUTT, 4); break;                                                                    \
            case 5: SB_IQBN(INT, OUTT, 5); break;                                                                    \
            case 6: SB_IQBN(INT, OUTT, 6); break;                                                                    \
            case 7: SB_IQBN(INT, OUTT, 7); break;                                                                    \
            default: SB_IQBN(INT, OUTT, 8); break;                                                                   \
        }                                                                                                            \
        SB_CHECK_LAUNCH("iqMagnitudeBankKernel");                                                                    \
        return SB_OK;                                                                                                \
    } while (0)
        if (in_dtype == SB_FLOAT32 && out_dtype == SB_FLOAT32) SB_IQB(float, float);
        if (in_dtype == SB_INT16 && out_dtype == SB_FLOAT32) SB_IQB(int16_t, float);
        if (in_dtype == SB_FLOAT32 && out_dtype == SB_INT16) SB_IQB(float, int16_t);
        if (in_dtype == SB_INT16 && out_dtype == SB_INT16) SB_IQB(int16_t, int16_t);
#undef SB_IQB
#undef SB_IQBN
        return fail(SB_ERR_UNSUPPORTED, "sb_iq_magnitude_run: %d -> %d unsupported", in_dtype, out_dtype);
    }
    const int rows = (IQ_OT - 1) * a.stride + a.lpN + 1;
    size_t shm = static_cast<size_t>(rows) * IQ_LINES * sizeof(float);
    SB_REQUIRE(shm <= 200 * 1024, "sb_iq_magnitude_run: decimation %u too large", decimation);
    dim3 grid((a.nL + IQ_LINES - 1) / IQ_LINES, (a.nOut + IQ_OT - 1) / IQ_OT);
#define SB_IQM(INT, OUTT)                                                                                      \
    do {                                                                                                       \
        SB_CUDA(cudaFuncSetAttribute(iqMagnitudeKernel<INT, OUTT>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                     static_cast<int>(shm)));                                                  \
        iqMagnitudeKernel<INT, OUTT><<<grid, 256, shm, st>>>(static_cast<const INT*>(in), static_cast<OUTT*>(out), a); \
        SB_CHECK_LAUNCH("iqMagnitudeKernel");                                                                  \
        return SB_OK;                                                                                          \
    } while (0)
    if (in_dtype == SB_FLOAT32 && out_dtype == SB_FLOAT32) SB_IQM(float, float);
    if (in_dtype == SB_INT16 && out_dtype == SB_FLOAT32) SB_IQM(int16_t, float);
    if (in_dtype == SB_FLOAT32 && out_dtype == SB_INT16) SB_IQM(float, int16_t);
    if (in_dtype == SB_INT16 && out_dtype == SB_INT16) SB_IQM(int16_t, int16_t);
#undef SB_IQM
    return fail(SB_ERR_UNSUPPORTED, "sb_iq_magnitude_run: %d -> %d unsupported", in_dtype, out_dtype);
}

int sb_iq_complex_run(const void* in, int in_dtype, void* out, uint32_t num_scanlines, uint32_t num_samples, double fs,
                      double fmix, double cutoff, uint32_t lpLen, uint32_t decimation, sb_stream stream) {
    SB_REQUIRE(in && out, "sb_iq_complex_run: null argument");
    SB_REQUIRE(fs > 0 && cutoff > 0 && lpLen >= 1 && lpLen < kIqMaxTaps, "sb_iq_complex_run: bad filter parameters");
    SB_REQUIRE(in_dtype == SB_FLOAT32 || in_dtype == SB_INT16, "sb_iq_complex_run: dtype %d", in_dtype);
    IqComplexArgs a;
    a.nS = static_cast<int>(num_samples);
    a.nL = static_cast<int>(num_scanlines);
    a.dec = static_cast<int>(std::max(decimation, 1u));
    a.nOut = a.nS / a.dec;
    a.fOverFs = fmix / fs;
    std::vector<float> lp = firDesign(lpLen, 0, 2, fs, cutoff, 0.0);
    // taps j = 0 .. 2*(N/2) centred on the output sample (the reference's FIR loop form); for even N
    // the last one is 0
    a.half = static_cast<int>(lpLen) / 2;
    a.taps = 2 * a.half + 1;
    for (int j = 0; j < a.taps; j++) a.lp[j] = j < static_cast<int>(lpLen) ? lp[j] : 0.0f;
    if (a.nOut == 0 || a.nL == 0) return SB_OK;
    const int rows = (IQ_OT - 1) * a.dec + a.taps;
    size_t shm = static_cast<size_t>(rows) * IQ_LINES * sizeof(float) + static_cast<size_t>(rows) * sizeof(float2);
    SB_REQUIRE(shm <= 200 * 1024, "sb_iq_complex_run: decimation %u too large", decimation);
    cudaStream_t st = S(stream);
    dim3 grid((a.nL + IQ_LINES - 1) / IQ_LINES, (a.nOut + IQ_OT - 1) / IQ_OT);
    if (in_dtype == SB_FLOAT32) {
        SB_CUDA(cudaFuncSetAttribute(iqComplexKernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(shm)));
        iqComplexKernel<float><<<grid, 256, shm, st>>>(static_cast<const float*>(in), static_cast<float2*>(out), a);
    } else {
        SB_CUDA(cudaFuncSetAttribute(iqComplexKernel<int16_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(shm)));
        iqComplexKernel<int16_t><<<grid, 256, shm, st>>>(static_cast<const int16_t*>(in), static_cast<float2*>(out), a);
    }
    SB_CHECK_LAUNCH("iqComplexKernel");
    return SB_OK;
}

}  // extern "C"
