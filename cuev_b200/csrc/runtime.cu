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

namespace {
std::mutex g_attr_mu;
struct AttrSet {
    const void *func;
    unsigned long long devs; // bit d: set on device d
    size_t bytes;
};
AttrSet g_attr[128];
int g_attr_n = 0;
std::atomic<unsigned long long> g_wait_limit{0};
std::atomic<bool> g_wait_limit_touched{false};
} // namespace

int ensure_dyn_smem(const void *func, size_t bytes) {
    int dev = 0;
    CUEV_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_attr_mu);
    AttrSet *e = nullptr;
    for (int i = 0; i < g_attr_n; ++i)
        if (g_attr[i].func == func) e = &g_attr[i];
    if (e && dev >= 0 && dev < 64 && (e->devs >> dev & 1ull) && e->bytes >= bytes) return CUEV_OK;
    CUEV_TRY(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    if (!e && g_attr_n < 128) {
        e = &g_attr[g_attr_n++];
        *e = AttrSet{func, 0ull, bytes};
    }
    if (e) {
        if (e->bytes != bytes) e->devs = 0ull, e->bytes = bytes;
        if (dev >= 0 && dev < 64) e->devs |= 1ull << dev;
    }
    return CUEV_OK;
}

__global__ void set_wait_limit_kernel(int *status, unsigned lo, unsigned hi) {
    status[DEV_STATUS_LIMIT_LO] = (int)lo;
    status[DEV_STATUS_LIMIT_HI] = (int)hi;
}

int apply_wait_limit(int *status, cudaStream_t stream) {
    const unsigned long long v = g_wait_limit.load();
    if (v == 0 && !g_wait_limit_touched.load()) return CUEV_OK; // default: words stay zero
    set_wait_limit_kernel<<<1, 1, 0, stream>>>(status, (unsigned)(v & 0xFFFFFFFFull),
                                               (unsigned)(v >> 32));
    note_launch();
    CUEV_TRY(cudaGetLastError());
    return CUEV_OK;
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

extern "C" int cuev_debug_set_wait_limit_ns(unsigned long long ns) {
    cuev::g_wait_limit.store(ns);
    cuev::g_wait_limit_touched.store(true);
    return CUEV_OK;
}
