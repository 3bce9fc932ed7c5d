// Envelope of the analytic signal along the samples of each scanline (HilbertEnvelope,
// Beamformer/HilbertEnvelope.cu:27-207): the reference takes the FFT of each line, doubles the positive
// frequencies, zeroes the negative ones (DC and, for even lengths, the Nyquist bin kept), inverts and
// writes |.| / N, i.e. env = |x + i h| with h the circular discrete Hilbert transform of the line.
//
// B200 design: h is computed directly as the circular convolution h[n] = sum_m k[(n - m) mod N] x[m]
// with k[n] = (2/N) sum_{j=1..J} sin(2 pi j n / N) (J = N/2 - 1 for even N, (N - 1)/2 for odd N), which
// is exact for every length N (no power-of-two or mixed-radix restriction) and needs no FFT library.
// It is an FP32 FMA-bound circulant product: a CTA of 64 threads computes 32 samples x 32 scanlines,
// each thread a 4 x 4 register tile; x tiles are staged in shared memory and the k values a thread
// needs slide by one per input sample, so each step is one shared-memory float4 of x, one k and 16
// FMAs. Sums are blocked per 32-sample chunk (chunk sum added to the total) to keep the FP32 error of
// the N-term sums small. The output is clampCast(sqrt(x^2 + h^2)).
// Long lines leave too few tiles to fill the GPU (2048 x 128: 256 CTAs of 2 warps), so the input
// range of each output tile is split over the 8 CTAs of a thread-block cluster (CTA r sums chunks
// r, r + 8, ...); rank 0 adds the 8 partial tiles from distributed shared memory in rank order (a
// deterministic reduction, no scratch memory) and writes the envelope.
// Power-of-two lengths (64 .. 16384) take an FFT path instead: a CTA packs two real scanlines x, y as
// z = x + i y, transforms z in shared memory (radix-2, decimation in time from a bit-reversed load),
// multiplies by -i sgn(k) (DC and Nyquist bins zeroed) and transforms back (decimation in frequency,
// bit-reversed result): since the Hilbert transform is linear and real for real input, the result
// over N is h_x + i h_y. O(N log N) instead of the circulant product's 2 N^2 flops per scanline.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "common.cuh"

struct sb_analytic_plan {
    uint32_t n = 0;
    float* dK = nullptr;    // k[0..N)
    float2* dTw = nullptr;  // per FFT stage s (h = 2^(s-1) entries at offset h - 1): exp(-2 pi i j / 2^s), j < h
};

namespace sb {
namespace {

constexpr int kAT = 32;   // samples and scanlines per CTA tile, and samples per staged chunk
constexpr int kAThreads = 64;

constexpr int kASplit = 8;  // CTAs per cluster sharing one output tile

// Lengths of the FFT path: powers of two from 64 to 16384 (the transform, 8 N bytes, fits a CTA's
// shared memory).
inline bool fftLength(uint32_t N) { return N >= 64 && N <= 16384 && (N & (N - 1)) == 0; }

__device__ __forceinline__ float4 load4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ float4 load4(const int16_t* p) {
    const short4 v = __ldg(reinterpret_cast<const short4*>(p));
    return make_float4(v.x, v.y, v.z, v.w);
}

// The 4 x 4 partial sums of this thread over the chunks m0 = first, first + step, ... (x tiles staged
// in xs, kernel values in ks).
template <typename IN>
__device__ __forceinline__ void analyticPartial(const IN* __restrict__ in, const float* __restrict__ kern, int N, int nL,
                                                int n0, int l0, int first, int step, float (&xs)[kAT][kAT],
                                                float (&ks)[2 * kAT], float (&tot)[4][4]) {
    const int tid = threadIdx.x;
    const int ty = tid / 8, tx = tid % 8;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) tot[i][j] = 0.0f;
    // the next chunk's x tile (4 groups of 4 scanlines per thread) and kernel value are fetched into
    // registers while the current chunk is summed
    float4 px[4];
    float pk = 0.0f;
    const bool vec = nL % 4 == 0 && reinterpret_cast<uintptr_t>(in) % (4 * sizeof(IN)) == 0;
    auto fetch = [&](int m0) {
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int e = tid + kAThreads * u, mm = e >> 3, c = (e & 7) * 4;
            const int m = m0 + mm, l = l0 + c;
            float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if (m < N) {
                const IN* row = in + static_cast<size_t>(m) * nL;
                if (vec && l + 3 < nL) {
                    v = load4(row + l);
                } else {
                    if (l < nL) v.x = toFloat(row[l]);
                    if (l + 1 < nL) v.y = toFloat(row[l + 1]);
                    if (l + 2 < nL) v.z = toFloat(row[l + 2]);
                    if (l + 3 < nL) v.w = toFloat(row[l + 3]);
                }
            }
            px[u] = v;
        }
        if (tid < 2 * kAT - 1) {
            int d = n0 - m0 + tid - (kAT - 1);  // in (-2N, N)
            d %= N;
            if (d < 0) d += N;
            pk = __ldg(kern + d);
        }
    };
    if (first < N) fetch(first);
    for (int m0 = first; m0 < N; m0 += step) {
        __syncthreads();  // the previous chunk's reads are done
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int e = tid + kAThreads * u;
            *reinterpret_cast<float4*>(&xs[e >> 3][(e & 7) * 4]) = px[u];
        }
        if (tid < 2 * kAT - 1) ks[tid] = pk;
        __syncthreads();
        if (m0 + step < N) fetch(m0 + step);
        float acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) acc[i][j] = 0.0f;
        // sample s = ty*4 + i of the tile at input mm uses ks[s - mm + kAT - 1]
        float kw[4];
#pragma unroll
        for (int i = 0; i < 4; i++) kw[i] = ks[ty * 4 + i + kAT - 1];
#pragma unroll 4
        for (int mm = 0; mm < kAT; mm++) {
            const float4 xv = *reinterpret_cast<const float4*>(&xs[mm][tx * 4]);
#pragma unroll
            for (int i = 0; i < 4; i++) {
                acc[i][0] = fmaf(kw[i], xv.x, acc[i][0]);
                acc[i][1] = fmaf(kw[i], xv.y, acc[i][1]);
                acc[i][2] = fmaf(kw[i], xv.z, acc[i][2]);
                acc[i][3] = fmaf(kw[i], xv.w, acc[i][3]);
            }
            // slide: at mm + 1 sample i needs the value sample i - 1 used at mm
            if (mm + 1 < kAT) {
#pragma unroll
                for (int i = 3; i > 0; i--) kw[i] = kw[i - 1];
                kw[0] = ks[ty * 4 - (mm + 1) + kAT - 1];
            }
        }
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) tot[i][j] += acc[i][j];
    }
}

template <typename IN, typename OUT>
__device__ __forceinline__ void analyticStore(const IN* __restrict__ in, OUT* __restrict__ out, int N, int nL, int n0,
                                              int l0, const float (&h)[4][4]) {
    const int ty = threadIdx.x / 8, tx = threadIdx.x % 8;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int n = n0 + ty * 4 + i;
        if (n >= N) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int l = l0 + tx * 4 + j;
            if (l >= nL) continue;
            const size_t o = static_cast<size_t>(n) * nL + l;
            const float x = toFloat(in[o]);
            out[o] = clampCast<OUT>(sqrtf(fmaf(x, x, h[i][j] * h[i][j])));
        }
    }
}

// Cluster of kASplit CTAs along z per output tile.
template <typename IN, typename OUT>
__global__ void __cluster_dims__(1, 1, kASplit) __launch_bounds__(kAThreads)
    analyticEnvClusterKernel(const IN* __restrict__ in, OUT* __restrict__ out, const float* __restrict__ kern, int N,
                             int nL) {
    namespace cg = cooperative_groups;
    __shared__ __align__(16) float xs[kAT][kAT];
    __shared__ float ks[2 * kAT];
    __shared__ float part[kAThreads][16];  // this CTA's partial tile, per thread
    cg::cluster_group cluster = cg::this_cluster();
    const unsigned rank = cluster.block_rank();
    const int n0 = blockIdx.y * kAT, l0 = blockIdx.x * kAT;
    float tot[4][4];
    analyticPartial<IN>(in, kern, N, nL, n0, l0, static_cast<int>(rank) * kAT, kASplit * kAT, xs, ks, tot);
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) part[threadIdx.x][i * 4 + j] = tot[i][j];
    cluster.sync();  // every partial tile is in its CTA's shared memory
    if (rank == 0) {
        float h[4][4];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) h[i][j] = tot[i][j];
        for (unsigned r = 1; r < kASplit; r++) {
            const float* rp = cluster.map_shared_rank(&part[threadIdx.x][0], r);
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) h[i][j] += rp[i * 4 + j];
        }
        analyticStore<IN, OUT>(in, out, N, nL, n0, l0, h);
    }
    cluster.sync();  // the other CTAs keep their shared memory until rank 0 has read it
}

template <typename IN, typename OUT>
__global__ void __launch_bounds__(kAThreads) analyticEnvKernel(const IN* __restrict__ in, OUT* __restrict__ out,
                                                               const float* __restrict__ kern, int N, int nL) {
    __shared__ __align__(16) float xs[kAT][kAT];
    __shared__ float ks[2 * kAT];
    const int n0 = blockIdx.y * kAT, l0 = blockIdx.x * kAT;
    float tot[4][4];
    analyticPartial<IN>(in, kern, N, nL, n0, l0, 0, kAT, xs, ks, tot);
    analyticStore<IN, OUT>(in, out, N, nL, n0, l0, tot);
}

constexpr int kFftThreads = 1024;  // upper bound; a launch uses min(1024, N / 2) threads (one butterfly each per stage)

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
template <typename T> __device__ __forceinline__ float ldf(const T* p) { return static_cast<float>(__ldg(p)); }

constexpr int kFftOneLog = 11;  // ONE: N <= 2^11, one butterfly per thread and stage

// Envelopes of scanlines (2 b, 2 b + 1) of a [N][nL] image by FFT (N = 2^logN): see the file comment.
// ONE (N / 2 threads, N <= 2^kFftOneLog): each thread's twiddle of every stage is loaded into registers
// before the transforms, so no stage waits on a twiddle load.
template <typename IN, typename OUT, bool ONE>
__global__ void __launch_bounds__(kFftThreads) analyticFftKernel(const IN* __restrict__ in, OUT* __restrict__ out,
                                                                 const float2* __restrict__ tw, int N, int logN, int nL) {
    extern __shared__ float2 fsm[];
    float2* z = fsm;  // N values
    const int tid = threadIdx.x, nt = blockDim.x;
    const int l = 2 * static_cast<int>(blockIdx.x);
    const bool two = l + 1 < nL;
    const int half = N >> 1;
    float2 wr[ONE ? kFftOneLog : 1];
    if constexpr (ONE) {
#pragma unroll
        for (int s = 1; s <= kFftOneLog; s++)
            if (s <= logN) wr[s - 1] = __ldg(tw + ((1 << (s - 1)) - 1) + (tid & ((1 << (s - 1)) - 1)));
    }
    for (int n = tid; n < N; n += nt) {
        const size_t base = static_cast<size_t>(n) * nL + l;
        const float x = ldf(in + base), y = two ? ldf(in + base + 1) : 0.0f;
        z[__brev(static_cast<uint32_t>(n)) >> (32 - logN)] = make_float2(x, y);
    }
    __syncthreads();
    // forward transform, decimation in time: stage s joins blocks of 2^(s-1) with exp(-2 pi i j / 2^s)
    // (the stage's twiddles are contiguous in global memory: L1-resident, no shared-memory bank
    // conflicts for any stage)
    if constexpr (ONE) {
#pragma unroll
        for (int s = 1; s <= kFftOneLog; s++) {
            if (s > logN) break;
            const int h = 1 << (s - 1), b = tid;
            const int j = b & (h - 1);
            const int i0 = ((b >> (s - 1)) << s) + j, i1 = i0 + h;
            const float2 t = cmulf(wr[s - 1], z[i1]);
            const float2 a = z[i0];
            z[i0] = make_float2(__fadd_rn(a.x, t.x), __fadd_rn(a.y, t.y));
            z[i1] = make_float2(__fsub_rn(a.x, t.x), __fsub_rn(a.y, t.y));
            __syncthreads();
        }
    } else {
        for (int s = 1; s <= logN; s++) {
            const int h = 1 << (s - 1);
            const float2* ws = tw + (h - 1);
            for (int b = tid; b < half; b += nt) {
                const int j = b & (h - 1);
                const int i0 = ((b >> (s - 1)) << s) + j, i1 = i0 + h;
                const float2 t = cmulf(__ldg(ws + j), z[i1]);
                const float2 a = z[i0];
                z[i0] = make_float2(__fadd_rn(a.x, t.x), __fadd_rn(a.y, t.y));
                z[i1] = make_float2(__fsub_rn(a.x, t.x), __fsub_rn(a.y, t.y));
            }
            __syncthreads();
        }
    }
    // times -i sgn(k): positive frequencies (1 .. N/2 - 1) (re, im) -> (im, -re), negative ones
    // (N/2 + 1 .. N - 1) -> (-im, re), DC and Nyquist -> 0
    for (int k = tid; k < N; k += nt) {
        const float2 v = z[k];
        z[k] = (k == 0 || k == half) ? make_float2(0.0f, 0.0f) : (k < half ? make_float2(v.y, -v.x) : make_float2(-v.y, v.x));
    }
    __syncthreads();
    // inverse transform, decimation in frequency: stage s splits blocks of 2^s with exp(+2 pi i j / 2^s)
    if constexpr (ONE) {
#pragma unroll
        for (int s = kFftOneLog; s >= 1; s--) {
            if (s > logN) continue;
            const int h = 1 << (s - 1), b = tid;
            const int j = b & (h - 1);
            const int i0 = ((b >> (s - 1)) << s) + j, i1 = i0 + h;
            const float2 a = z[i0], c = z[i1];
            const float2 wj = wr[s - 1];
            z[i0] = make_float2(__fadd_rn(a.x, c.x), __fadd_rn(a.y, c.y));
            z[i1] = cmulf(make_float2(__fsub_rn(a.x, c.x), __fsub_rn(a.y, c.y)), make_float2(wj.x, -wj.y));
            __syncthreads();
        }
    } else {
        for (int s = logN; s >= 1; s--) {
            const int h = 1 << (s - 1);
            const float2* ws = tw + (h - 1);
            for (int b = tid; b < half; b += nt) {
                const int j = b & (h - 1);
                const int i0 = ((b >> (s - 1)) << s) + j, i1 = i0 + h;
                const float2 a = z[i0], c = z[i1];
                const float2 wj = __ldg(ws + j);
                z[i0] = make_float2(__fadd_rn(a.x, c.x), __fadd_rn(a.y, c.y));
                z[i1] = cmulf(make_float2(__fsub_rn(a.x, c.x), __fsub_rn(a.y, c.y)), make_float2(wj.x, -wj.y));
            }
            __syncthreads();
        }
    }
    const float invN = __fdiv_rn(1.0f, static_cast<float>(N));
    for (int n = tid; n < N; n += nt) {
        const float2 hv = z[__brev(static_cast<uint32_t>(n)) >> (32 - logN)];
        const size_t base = static_cast<size_t>(n) * nL + l;
        const float x = ldf(in + base), hx = __fmul_rn(hv.x, invN);
        out[base] = clampCast<OUT>(__fsqrt_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(hx, hx))));
        if (two) {
            const float y = ldf(in + base + 1), hy = __fmul_rn(hv.y, invN);
            out[base + 1] = clampCast<OUT>(__fsqrt_rn(__fadd_rn(__fmul_rn(y, y), __fmul_rn(hy, hy))));
        }
    }
}

}  // namespace
}  // namespace sb

using namespace sb;

extern "C" {

int sb_analytic_plan_create(uint32_t num_samples, sb_analytic_plan** out) {
    SB_REQUIRE(out, "sb_analytic_plan_create: null argument");
    *out = nullptr;
    SB_REQUIRE(num_samples >= 1 && num_samples <= (1u << 24), "sb_analytic_plan_create: %u samples out of range",
               num_samples);
    const uint32_t N = num_samples;
    const int J = N % 2 == 0 ? static_cast<int>(N / 2) - 1 : static_cast<int>((N - 1) / 2);
    std::vector<float> k(N, 0.0f);
    const double pi = 3.14159265358979323846;
    for (uint32_t n = 1; n < N && J > 0; n++) {
        // sum_{j=1..J} sin(j t) = sin(J t / 2) sin((J + 1) t / 2) / sin(t / 2), t = 2 pi n / N
        const double t = 2.0 * pi * static_cast<double>(n) / N;
        const double s = std::sin(J * t / 2.0) * std::sin((J + 1) * t / 2.0) / std::sin(t / 2.0);
        k[n] = static_cast<float>(2.0 / N * s);
    }
    auto p = new sb_analytic_plan();
    p->n = N;
    cudaError_t e = cudaMalloc(&p->dK, N * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(p->dK, k.data(), N * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && fftLength(N)) {
        std::vector<float2> tw(N - 1);
        for (uint32_t h = 1; h < N; h <<= 1)  // stage with blocks of 2h: exp(-2 pi i j / (2 h)), j < h
            for (uint32_t j = 0; j < h; j++) {
                const double a = pi * static_cast<double>(j) / h;
                tw[h - 1 + j] = make_float2(static_cast<float>(std::cos(a)), static_cast<float>(-std::sin(a)));
            }
        e = cudaMalloc(&p->dTw, (N - 1) * sizeof(float2));
        if (e == cudaSuccess) e = cudaMemcpy(p->dTw, tw.data(), (N - 1) * sizeof(float2), cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {
        cudaFree(p->dK);
        cudaFree(p->dTw);
        delete p;
        return cudaFail(e, "sb_analytic_plan_create");
    }
    *out = p;
    return SB_OK;
}

int sb_analytic_plan_destroy(sb_analytic_plan* p) {
    if (p) {
        cudaFree(p->dK);
        cudaFree(p->dTw);
        delete p;
    }
    return SB_OK;
}

int sb_analytic_env_run(const sb_analytic_plan* p, const void* in, int in_dtype, void* out, int out_dtype,
                        uint32_t num_scanlines, sb_stream stream) {
    SB_REQUIRE(p && in && out, "sb_analytic_env_run: null argument");
    SB_REQUIRE(in_dtype == SB_INT16 || in_dtype == SB_FLOAT32, "sb_analytic_env_run: input dtype %d unsupported", in_dtype);
    SB_REQUIRE(out_dtype == SB_INT16 || out_dtype == SB_FLOAT32, "sb_analytic_env_run: output dtype %d unsupported",
               out_dtype);
    if (num_scanlines == 0) return SB_OK;
    const int N = static_cast<int>(p->n), nL = static_cast<int>(num_scanlines);
    if (p->dTw) {  // power-of-two length: the FFT path
        int logN = 0;
        while ((1 << logN) < N) logN++;
        const size_t shm = static_cast<size_t>(N) * sizeof(float2);
        const unsigned grid = static_cast<unsigned>((nL + 1) / 2);
        const int fftThreads = std::min(kFftThreads, N / 2);
        const bool one = fftThreads == N / 2 && logN <= kFftOneLog;
        cudaStream_t stf = S(stream);
#define SB_AF(IT, OT)                                                                                                  \
    do {                                                                                                               \
        if (one) {                                                                                                     \
            SB_CUDA(cudaFuncSetAttribute(analyticFftKernel<IT, OT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                         static_cast<int>(shm)));                                                      \
            analyticFftKernel<IT, OT, true><<<grid, fftThreads, shm, stf>>>(static_cast<const IT*>(in),                \
                                                                             static_cast<OT*>(out), p->dTw, N, logN, nL); \
        } else {                                                                                                       \
            SB_CUDA(cudaFuncSetAttribute(analyticFftKernel<IT, OT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                         static_cast<int>(shm)));                                                      \
            analyticFftKernel<IT, OT, false><<<grid, fftThreads, shm, stf>>>(static_cast<const IT*>(in),               \
                                                                              static_cast<OT*>(out), p->dTw, N, logN, nL); \
        }                                                                                                              \
    } while (0)
        if (in_dtype == SB_INT16 && out_dtype == SB_FLOAT32) SB_AF(int16_t, float);
        else if (in_dtype == SB_INT16) SB_AF(int16_t, int16_t);
        else if (out_dtype == SB_FLOAT32) SB_AF(float, float);
        else SB_AF(float, int16_t);
#undef SB_AF
        SB_CHECK_LAUNCH("analyticFftKernel");
        return SB_OK;
    }
    dim3 grid((nL + kAT - 1) / kAT, (N + kAT - 1) / kAT);
    SB_REQUIRE(grid.y <= 65535u, "sb_analytic_env_run: %d samples exceed the grid", N);
    cudaStream_t st = S(stream);
    // split the input range over a cluster when the tiles alone leave the GPU mostly idle and each
    // CTA still gets at least two chunks
    const bool split = static_cast<long>(grid.x) * grid.y < 8L * smCount() && N >= 2 * kASplit * kAT;
    dim3 gridSplit(grid.x, grid.y, kASplit);
#define SB_AN(IT, OT)                                                                                                  \
    do {                                                                                                               \
        if (split)                                                                                                     \
            analyticEnvClusterKernel<IT, OT><<<gridSplit, kAThreads, 0, st>>>(static_cast<const IT*>(in),              \
                                                                               static_cast<OT*>(out), p->dK, N, nL);  \
        else                                                                                                           \
            analyticEnvKernel<IT, OT><<<grid, kAThreads, 0, st>>>(static_cast<const IT*>(in), static_cast<OT*>(out),   \
                                                                  p->dK, N, nL);                                       \
    } while (0)
    if (in_dtype == SB_INT16 && out_dtype == SB_FLOAT32) SB_AN(int16_t, float);
    else if (in_dtype == SB_INT16) SB_AN(int16_t, int16_t);
    else if (out_dtype == SB_FLOAT32) SB_AN(float, float);
    else SB_AN(float, int16_t);
#undef SB_AN
    SB_CHECK_LAUNCH("analyticEnvKernel");
    return SB_OK;
}

}  // extern "C"
