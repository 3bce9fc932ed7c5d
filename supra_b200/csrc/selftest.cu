// Self-tests (no reference counterpart). The bounded-wait failure path: The staged and persistent
// kernels wait on mbarriers with a poll limit; when a wait gives up they raise the device error flag
// that sb_check_device_errors reports as SB_ERR_TIMEOUT, and return normally, so the context stays
// usable. This kernel exercises exactly that path without any fault: one thread initialises an
// mbarrier for one arrival and, unless `arrive` is set, never arrives, then waits with the given poll
// limit; a wait that runs out sets the flag and the kernel returns.
#include <cstdint>

#include "common.cuh"
#include "tma.cuh"

namespace sb {
namespace {

__global__ void boundedWaitProbeKernel(uint32_t polls, int arrive, int* errFlag, int* completed) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x != 0) return;
    mbarInit(&bar, 1);
    mbarInitFence();
    if (arrive) {
        uint64_t state;
        asm volatile("mbarrier.arrive.shared::cta.b64 %0, [%1];" : "=l"(state) : "r"(smemAddr(&bar)) : "memory");
    }
    const bool done = mbarWaitBounded(&bar, 0, polls);
    if (!done) atomicExch(errFlag, 1);
    *completed = done ? 1 : 0;
}

// sqrtNewton against __fsqrt_rn on the float bit patterns [lo, hi) (equal bits, or both NaN): count and
// lowest mismatch.
__global__ void sqrtCheckKernel(uint32_t lo, uint64_t hi, unsigned long long* bad, uint32_t* first) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t b = lo + static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; b < hi; b += stride) {
        const float x = __uint_as_float(static_cast<uint32_t>(b));
        const float g = sqrtNewton(x), e = __fsqrt_rn(x);
        if (isnan(g) != isnan(e) || (!isnan(e) && __float_as_uint(g) != __float_as_uint(e))) {
            atomicAdd(bad, 1ull);
            atomicMin(first, static_cast<uint32_t>(b));
        }
    }
}

}  // namespace
}  // namespace sb

using namespace sb;

extern "C" int sb_selftest_bounded_wait(uint32_t polls, int arrive, int* completed_host, sb_stream stream) {
    SB_REQUIRE(polls >= 1 && polls <= (1u << 20), "sb_selftest_bounded_wait: polls %u not in [1, 2^20]", polls);
    int* err = deviceErrorFlag();
    if (!err) return fail(SB_ERR_NO_MEMORY, "sb_selftest_bounded_wait: no device error flag");
    int* dDone = nullptr;
    cudaStream_t st = S(stream);
    SB_CUDA(cudaMallocAsync(&dDone, sizeof(int), st));
    boundedWaitProbeKernel<<<1, 32, 0, st>>>(polls, arrive, err, dDone);
    cudaError_t e = cudaGetLastError();
    int h = -1;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, dDone, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFreeAsync(dDone, st);
    if (e != cudaSuccess) return cudaFail(e, "sb_selftest_bounded_wait");
    if (completed_host) *completed_host = h;
    return SB_OK;
}

extern "C" int sb_selftest_sqrt(uint32_t first_bits, uint64_t end_bits, uint64_t* mismatches, uint32_t* first_mismatch,
                                sb_stream stream) {
    SB_REQUIRE(end_bits <= (1ull << 32) && first_bits <= end_bits, "sb_selftest_sqrt: range [%u, %llu) not inside 2^32",
               first_bits, static_cast<unsigned long long>(end_bits));
    SB_REQUIRE(mismatches, "sb_selftest_sqrt: null mismatch count");
    cudaStream_t st = S(stream);
    unsigned long long* dBad = nullptr;
    SB_CUDA(cudaMallocAsync(&dBad, sizeof(unsigned long long) + sizeof(uint32_t), st));
    uint32_t* dFirst = reinterpret_cast<uint32_t*>(dBad + 1);
    cudaError_t e = cudaMemsetAsync(dBad, 0, sizeof(unsigned long long), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(dFirst, 0xFF, sizeof(uint32_t), st);
    if (e == cudaSuccess && end_bits > first_bits) {
        sqrtCheckKernel<<<smCount() * 8, 256, 0, st>>>(first_bits, end_bits, dBad, dFirst);
        e = cudaGetLastError();
    }
    unsigned long long hb = 0;
    uint32_t hf = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hb, dBad, sizeof(hb), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hf, dFirst, sizeof(hf), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFreeAsync(dBad, st);
    if (e != cudaSuccess) return cudaFail(e, "sb_selftest_sqrt");
    *mismatches = hb;
    if (first_mismatch) *first_mismatch = hf;
    return SB_OK;
}
