// Self-test of the bounded-wait failure path (no reference counterpart). The staged and persistent
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
