// Host runtime pieces shared by all stages: last-error bookkeeping, device properties.
#include "common.cuh"

#include <atomic>
#include <cstring>
#include <mutex>
#include <string>

namespace cuev {

namespace {
thread_local std::string g_last_error;
std::atomic<long long> g_launches{0};
} // namespace

void note_launch(int count) { g_launches.fetch_add(count, std::memory_order_relaxed); }

void set_last_error(cudaError_t e, const char *file, int line) {
    char buf[512];
    snprintf(buf, sizeof(buf), "CUDA error %s at %s:%d", cudaGetErrorString(e), file, line);
    g_last_error = buf;
}

void set_last_message(const char *msg) { g_last_error = msg ? msg : ""; }

int num_sms() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (cached[dev] == 0) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
            v = 148;
        cached[dev] = v;
    }
    return cached[dev];
}

size_t max_dynamic_smem(const void *func) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        optin = 227 * 1024;
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, func) != cudaSuccess) return 0;
    return (size_t)optin > fa.sharedSizeBytes ? (size_t)optin - fa.sharedSizeBytes : 0;
}

} // namespace cuev

extern "C" const char *cuev_last_error(void) { return cuev::g_last_error.c_str(); }

extern "C" long long cuev_kernel_launches(void) { return cuev::g_launches.load(); }
