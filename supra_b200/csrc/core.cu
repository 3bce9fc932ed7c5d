// Status handling, version, and the host-side design helpers exported through the C ABI.
#include <cstdarg>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "design.h"

namespace sb {

static thread_local std::string g_lastError;

void setError(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_lastError = buf;
}

int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_lastError = buf;
    return code;
}

int cudaFail(cudaError_t e, const char* what) {
    setError("%s: %s (%d)", what, cudaGetErrorString(e), static_cast<int>(e));
    return e == cudaErrorMemoryAllocation ? SB_ERR_NO_MEMORY : SB_ERR_CUDA;
}

int smCount() {
    static std::mutex m;
    static int cache[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    std::lock_guard<std::mutex> l(m);
    if (cache[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        cache[dev] = n;
    }
    return cache[dev];
}

int* deviceErrorFlag() {
    static std::mutex m;
    static int* flags[64] = {nullptr};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> l(m);
    if (!flags[dev]) {
        int* f = nullptr;
        if (cudaMalloc(&f, sizeof(int)) != cudaSuccess) return nullptr;
        if (cudaMemset(f, 0, sizeof(int)) != cudaSuccess) {
            cudaFree(f);
            return nullptr;
        }
        flags[dev] = f;
    }
    return flags[dev];
}

}  // namespace sb

extern "C" {

int sb_check_device_errors(int reset) {
    int* f = sb::deviceErrorFlag();
    if (!f) return sb::fail(SB_ERR_NO_MEMORY, "sb_check_device_errors: no device flag");
    SB_CUDA(cudaDeviceSynchronize());
    int h = 0;
    SB_CUDA(cudaMemcpy(&h, f, sizeof(int), cudaMemcpyDeviceToHost));
    if (reset && h) SB_CUDA(cudaMemset(f, 0, sizeof(int)));
    // the allocation-free DAS entry point keeps its own flag in its static scratch
    if (int* fs = sb::staticWaitFlag()) {
        int hs = 0;
        SB_CUDA(cudaMemcpy(&hs, fs, sizeof(int), cudaMemcpyDeviceToHost));
        if (reset && hs) SB_CUDA(cudaMemset(fs, 0, sizeof(int)));
        h |= hs;
    }
    if (h) return sb::fail(SB_ERR_TIMEOUT, "a device-side bounded wait gave up (staged channel data never arrived)");
    return SB_OK;
}

const char* sb_last_error(void) { return sb::g_lastError.c_str(); }

int sb_version(int* major, int* minor) {
    if (major) *major = 0;
    if (minor) *minor = 1;
    return SB_OK;
}

int sb_window_lut(int window_type, float window_parameter, uint32_t num_entries, float* out_host) {
    SB_REQUIRE(out_host != nullptr && num_entries >= 2, "sb_window_lut: bad output / size");
    SB_REQUIRE(window_type >= 0 && window_type <= 3, "sb_window_lut: window type %d", window_type);
    std::vector<float> lut = sb::windowLut(window_type, window_parameter, num_entries);
    for (uint32_t i = 0; i < num_entries; i++) out_host[i] = lut[i];
    return SB_OK;
}

int sb_fir_design(uint32_t length, int type, int window, double sampling_frequency, double frequency,
                  double bandwidth, float* out_host) {
    SB_REQUIRE(out_host != nullptr && length >= 1, "sb_fir_design: bad output / length");
    SB_REQUIRE(type >= 0 && type <= 3 && window >= 0 && window <= 3, "sb_fir_design: bad type/window");
    std::vector<float> f = sb::firDesign(length, type, window, sampling_frequency, frequency, bandwidth);
    for (uint32_t i = 0; i < length; i++) out_host[i] = f[i];
    return SB_OK;
}

}  // extern "C"
