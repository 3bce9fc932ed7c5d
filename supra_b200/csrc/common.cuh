// Shared helpers of the supra_b200 CUDA library: status handling, dtype dispatch, clampCast.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cfloat>
#include <cstdio>
#include <string>

#include "supra_b200.h"

namespace sb {

// Thread-local last error message (returned by sb_last_error()).
void setError(const char* fmt, ...);
int fail(int code, const char* fmt, ...);
int cudaFail(cudaError_t e, const char* what);

#define SB_CUDA(call)                                                        \
    do {                                                                     \
        cudaError_t _e = (call);                                             \
        if (_e != cudaSuccess) return ::sb::cudaFail(_e, #call);             \
    } while (0)

#define SB_CHECK_LAUNCH(name)                                                \
    do {                                                                     \
        cudaError_t _e = cudaGetLastError();                                 \
        if (_e != cudaSuccess) return ::sb::cudaFail(_e, name);              \
    } while (0)

#define SB_REQUIRE(cond, ...)                                                \
    do {                                                                     \
        if (!(cond)) return ::sb::fail(SB_ERR_INVALID_ARG, __VA_ARGS__);     \
    } while (0)

inline cudaStream_t S(sb_stream s) { return reinterpret_cast<cudaStream_t>(s); }

inline size_t dtypeSize(int dt) {
    switch (dt) {
    case SB_INT16: return 2;
    case SB_FLOAT32: return 4;
    case SB_UINT8: return 1;
    case SB_COMPLEX64: return 8;
    case SB_UINT16: return 2;
    default: return 0;
    }
}

// clampCast (SupraLib/utilities/cudaUtility.h:111-147): clamp to the type's range, then truncate.
template <typename T> __device__ __forceinline__ T clampCast(float x);
template <> __device__ __forceinline__ float clampCast<float>(float x) { return fminf(fmaxf(x, -FLT_MAX), FLT_MAX); }
template <> __device__ __forceinline__ int16_t clampCast<int16_t>(float x) {
    return static_cast<int16_t>(fminf(fmaxf(x, -32767.0f), 32767.0f));
}
template <> __device__ __forceinline__ uint8_t clampCast<uint8_t>(float x) {
    return static_cast<uint8_t>(fminf(fmaxf(x, 0.0f), 255.0f));
}
template <> __device__ __forceinline__ uint16_t clampCast<uint16_t>(float x) {
    return static_cast<uint16_t>(fminf(fmaxf(x, 0.0f), 65535.0f));
}

template <typename T> __device__ __forceinline__ float toFloat(T v) { return static_cast<float>(v); }

// Square root by one Newton step from the hardware reciprocal square root (Markstein's refinement:
// s = x y, the residual r = x - s^2 exactly by a fused multiply-add, then s + r y / 2). On this GPU it
// equals __fsqrt_rn bit for bit for every x in [2^-102, FLT_MAX] (sb_selftest_sqrt compares all of
// them); callers use it only where their arguments provably lie in that range.
#ifdef __CUDACC__
__device__ __forceinline__ float sqrtNewton(float x) {
    const float y = rsqrtf(x);
    const float s = __fmul_rn(x, y);
    const float r = __fmaf_rn(-s, s, x);
    return __fmaf_rn(r, __fmul_rn(0.5f, y), s);
}
#endif

// Number of SMs of the current device (cached per device).
int smCount();

// Per-device int in global memory that kernels set when a bounded wait gives up (nullptr if it
// could not be allocated).
int* deviceErrorFlag();
// sb_das_run_static's wait-failure flag on the current device (in its static scratch), or null
// before that entry point's first call there.
int* staticWaitFlag();

}  // namespace sb
