// Temporal filter: weighted mean of the last images of a stream (TemporalFilter::filter,
// Beamformer/TemporalFilter.cu:22-110, WorkType float):
//   out[i] = clampCast(sum_k w_k x_k[i] / sum_k w_k), k over the images oldest first,
// every product and sum a separately rounded float operation in the reference's order.
// HBM-streaming: one pass over the N inputs and the output; each thread moves 16 bytes of every input
// per step (8 int16 or 4 float samples) when the buffers allow it, over a grid of resident CTAs.
#include <algorithm>
#include <cstdint>

#include "common.cuh"

namespace sb {
namespace {

constexpr int kMaxTemporalImages = 50;  // TemporalFilterNode "numImages" range (TemporalFilterNode.cpp:39)

struct TemporalArgs {
    const void* img[kMaxTemporalImages];
    float w[kMaxTemporalImages];
    uint32_t n;
    uint64_t numel;
    void* out;
};

template <typename T, int VEC> struct VecOf;
template <> struct VecOf<int16_t, 8> { using type = uint4; };
template <> struct VecOf<float, 4> { using type = float4; };
template <> struct VecOf<int16_t, 1> { using type = int16_t; };
template <> struct VecOf<float, 1> { using type = float; };

// VEC outputs of one step as whole vector stores (dst is aligned to the vector: out is 16-byte aligned)
template <typename OUT, int VEC>
__device__ __forceinline__ void storeVec(OUT* dst, const float (&v)[VEC]) {
    if constexpr (VEC == 1) {
        dst[0] = clampCast<OUT>(v[0]);
    } else if constexpr (sizeof(OUT) == 4) {
#pragma unroll
        for (int j = 0; j < VEC; j += 4)
            reinterpret_cast<float4*>(dst)[j / 4] = make_float4(clampCast<float>(v[j]), clampCast<float>(v[j + 1]),
                                                                clampCast<float>(v[j + 2]), clampCast<float>(v[j + 3]));
    } else {
        uint32_t w[VEC / 2];
#pragma unroll
        for (int j = 0; j < VEC; j += 2)
            w[j / 2] = static_cast<uint16_t>(clampCast<int16_t>(v[j])) |
                       (static_cast<uint32_t>(static_cast<uint16_t>(clampCast<int16_t>(v[j + 1]))) << 16);
        if constexpr (VEC == 8) *reinterpret_cast<uint4*>(dst) = make_uint4(w[0], w[1], w[2], w[3]);
        else *reinterpret_cast<uint2*>(dst) = make_uint2(w[0], w[1]);
    }
}

template <typename IN, typename OUT, int VEC>
__global__ void __launch_bounds__(256) temporalFilterKernel(TemporalArgs a) {
    using V = typename VecOf<IN, VEC>::type;
    float wsum = 0.0f;
    for (uint32_t k = 0; k < a.n; k++) wsum = __fadd_rn(wsum, a.w[k]);
    const uint64_t nVec = a.numel / VEC;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < nVec; v += stride) {
        float acc[VEC];
#pragma unroll
        for (int j = 0; j < VEC; j++) acc[j] = 0.0f;
        for (uint32_t k = 0; k < a.n; k++) {
            const V raw = __ldcs(static_cast<const V*>(a.img[k]) + v);  // streamed once: evict first
            const IN* x = reinterpret_cast<const IN*>(&raw);
#pragma unroll
            for (int j = 0; j < VEC; j++) acc[j] = __fadd_rn(acc[j], __fmul_rn(a.w[k], toFloat(x[j])));
        }
#pragma unroll
        for (int j = 0; j < VEC; j++) acc[j] = __fdiv_rn(acc[j], wsum);
        storeVec<OUT, VEC>(static_cast<OUT*>(a.out) + v * VEC, acc);
    }
    // the elements past the last whole vector
    const uint64_t tail = nVec * VEC + static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (VEC > 1 && tail < a.numel) {
        float acc = 0.0f;
        for (uint32_t k = 0; k < a.n; k++) acc = __fadd_rn(acc, __fmul_rn(a.w[k], toFloat(static_cast<const IN*>(a.img[k])[tail])));
        static_cast<OUT*>(a.out)[tail] = clampCast<OUT>(__fdiv_rn(acc, wsum));
    }
}

template <typename IN, typename OUT>
int launchTemporal(const TemporalArgs& a, bool vec, cudaStream_t st) {
    constexpr int V = sizeof(IN) == 2 ? 8 : 4;
    const uint64_t units = vec ? a.numel / V : a.numel;
    const uint64_t maxGrid = static_cast<uint64_t>(smCount()) * 8;  // 8 resident CTAs of 256 per SM
    const unsigned grid = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(maxGrid, (units + 255) / 256)));
    if (vec) temporalFilterKernel<IN, OUT, V><<<grid, 256, 0, st>>>(a);
    else temporalFilterKernel<IN, OUT, 1><<<grid, 256, 0, st>>>(a);
    SB_CHECK_LAUNCH("temporalFilterKernel");
    return SB_OK;
}

}  // namespace
}  // namespace sb

using namespace sb;

extern "C" int sb_temporal_filter_run(const void* const* images, uint32_t num_images, const double* weights, int in_dtype,
                                      void* out, int out_dtype, uint64_t numel, sb_stream stream) {
    SB_REQUIRE(images, "sb_temporal_filter_run: null image array");
    SB_REQUIRE(num_images >= 1 && num_images <= static_cast<uint32_t>(kMaxTemporalImages),
               "sb_temporal_filter_run: num_images %u not in [1, %d]", num_images, kMaxTemporalImages);
    SB_REQUIRE(in_dtype == SB_INT16 || in_dtype == SB_FLOAT32, "sb_temporal_filter_run: input dtype %d unsupported", in_dtype);
    SB_REQUIRE(out_dtype == SB_INT16 || out_dtype == SB_FLOAT32, "sb_temporal_filter_run: output dtype %d unsupported",
               out_dtype);
    if (numel == 0) return SB_OK;  // empty images (their data pointers may be null)
    SB_REQUIRE(out, "sb_temporal_filter_run: null output");
    TemporalArgs a;
    bool aligned = (reinterpret_cast<uintptr_t>(out) % 16) == 0;
    for (uint32_t k = 0; k < num_images; k++) {
        SB_REQUIRE(images[k], "sb_temporal_filter_run: image %u is null", k);
        a.img[k] = images[k];
        a.w[k] = weights ? static_cast<float>(weights[k]) : 1.0f;
        aligned = aligned && (reinterpret_cast<uintptr_t>(images[k]) % 16) == 0;
    }
    a.n = num_images;
    a.numel = numel;
    a.out = out;
    cudaStream_t st = S(stream);
    if (in_dtype == SB_INT16 && out_dtype == SB_FLOAT32) return launchTemporal<int16_t, float>(a, aligned, st);
    if (in_dtype == SB_INT16) return launchTemporal<int16_t, int16_t>(a, aligned, st);
    if (out_dtype == SB_FLOAT32) return launchTemporal<float, float>(a, aligned, st);
    return launchTemporal<float, int16_t>(a, aligned, st);
}
