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
#include <cmath>
#include <cstdint>
#include <vector>

#include "common.cuh"

struct sb_analytic_plan {
    uint32_t n = 0;
    float* dK = nullptr;  // k[0..N)
};

namespace sb {
namespace {

constexpr int kAT = 32;   // samples and scanlines per CTA tile, and samples per staged chunk
constexpr int kAThreads = 64;

template <typename IN, typename OUT>
__global__ void __launch_bounds__(kAThreads) analyticEnvKernel(const IN* __restrict__ in, OUT* __restrict__ out,
                                                               const float* __restrict__ kern, int N, int nL) {
    __shared__ __align__(16) float xs[kAT][kAT];  // [m - m0][line - l0]
    __shared__ float ks[2 * kAT];                 // k[(n0 - m0 + d) mod N], d = -(kAT - 1) .. kAT - 1
    const int tid = threadIdx.x;
    const int ty = tid / 8, tx = tid % 8;  // sample group (4 samples), line group (4 lines)
    const int n0 = blockIdx.y * kAT, l0 = blockIdx.x * kAT;
    float tot[4][4], acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) tot[i][j] = 0.0f;
    for (int m0 = 0; m0 < N; m0 += kAT) {
        __syncthreads();  // the previous chunk's reads are done
        for (int e = tid; e < kAT * kAT; e += kAThreads) {
            const int mm = e / kAT, ll = e % kAT;
            const int m = m0 + mm, l = l0 + ll;
            xs[mm][ll] = (m < N && l < nL) ? toFloat(in[static_cast<size_t>(m) * nL + l]) : 0.0f;
        }
        for (int e = tid; e < 2 * kAT - 1; e += kAThreads) {
            int d = n0 - m0 + e - (kAT - 1);  // in (-N, N)
            d %= N;
            if (d < 0) d += N;
            ks[e] = __ldg(kern + d);
        }
        __syncthreads();
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
            out[o] = clampCast<OUT>(sqrtf(fmaf(x, x, tot[i][j] * tot[i][j])));
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
    if (e != cudaSuccess) {
        cudaFree(p->dK);
        delete p;
        return cudaFail(e, "sb_analytic_plan_create");
    }
    *out = p;
    return SB_OK;
}

int sb_analytic_plan_destroy(sb_analytic_plan* p) {
    if (p) {
        cudaFree(p->dK);
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
    dim3 grid((nL + kAT - 1) / kAT, (N + kAT - 1) / kAT);
    SB_REQUIRE(grid.y <= 65535u, "sb_analytic_env_run: %d samples exceed the grid", N);
    cudaStream_t st = S(stream);
#define SB_AN(IT, OT) \
    analyticEnvKernel<IT, OT><<<grid, kAThreads, 0, st>>>(static_cast<const IT*>(in), static_cast<OT*>(out), p->dK, N, nL)
    if (in_dtype == SB_INT16 && out_dtype == SB_FLOAT32) SB_AN(int16_t, float);
    else if (in_dtype == SB_INT16) SB_AN(int16_t, int16_t);
    else if (out_dtype == SB_FLOAT32) SB_AN(float, float);
    else SB_AN(float, int16_t);
#undef SB_AN
    SB_CHECK_LAUNCH("analyticEnvKernel");
    return SB_OK;
}

}  // extern "C"
