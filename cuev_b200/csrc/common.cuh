// Shared helpers for the cuEV-B200 eigensolver kernels (sm_100a only).
//
// Error model: every host entry returns a cuev_status (include/cuev_b200.h).  Device code never
// traps; kernels that can fail (bounded spin-waits, non-finite input) write a code into a small
// device status word that the host reads after the stage.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

#include "../../include/cuev_b200.h"

namespace cuev {

// Host-side error propagation: return the status to the C-ABI caller instead of exit(1)
// (the reference's CUDA_CHECK at include/common.h:9-16 terminates the process).
#define CUEV_TRY(expr)                                                                             \
    do {                                                                                           \
        cudaError_t _e = (expr);                                                                   \
        if (_e != cudaSuccess) {                                                                   \
            cuev::set_last_error(_e, __FILE__, __LINE__);                                          \
            return CUEV_ERR_CUDA;                                                                  \
        }                                                                                          \
    } while (0)

#define CUEV_CHECK_STATUS(expr)                                                                    \
    do {                                                                                           \
        int _s = (expr);                                                                           \
        if (_s != CUEV_OK) return _s;                                                              \
    } while (0)

void set_last_error(cudaError_t e, const char *file, int line);
void set_last_message(const char *msg);

inline int div_up(int a, int b) { return (a + b - 1) / b; }
inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

int num_sms();
// Count of kernels this library has launched (exported as cuev_kernel_launches).
void note_launch(int count = 1);
// Largest dynamic shared-memory size a kernel may request (opt-in limit minus its static part).
size_t max_dynamic_smem(const void *func);

// Device status word layout (one int per failure class; first writer wins).
enum DevStatusSlot : int {
    DEV_STATUS_CODE = 0,      // a cuev_status code, 0 = ok
    DEV_STATUS_WHERE = 1,     // kernel-specific detail (e.g. sweep index that timed out)
    DEV_STATUS_LIMIT_LO = 2,  // bounded-wait limit in ns (low, high word); 0 = the default 2 s.
    DEV_STATUS_LIMIT_HI = 3,  // Only cuev_debug_set_wait_limit_ns sets it (failure-path tests).
    DEV_STATUS_WORDS = 4
};

// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) applies to the current device only: set it
// once per (kernel, device).
int ensure_dyn_smem(const void *func, size_t bytes);
// Write the wait limit chosen by cuev_debug_set_wait_limit_ns into status words 2-3 (stream
// ordered; no-op while the limit is the default).
int apply_wait_limit(int *status, cudaStream_t stream);

#ifdef __CUDACC__

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

/// Limit of a bounded wait: 2 s unless a failure-path test lowered it (status words 2-3).
__device__ __forceinline__ uint64_t wait_limit_ns(const int *status) {
    const uint64_t v = ((uint64_t)(unsigned)status[DEV_STATUS_LIMIT_HI] << 32) |
                       (unsigned)status[DEV_STATUS_LIMIT_LO];
    return v ? v : 2000000000ull;
}

/// Record a device-side failure (first failure wins); never traps.
__device__ __forceinline__ void dev_fail(int *status, int code, int where) {
    if (atomicCAS(&status[DEV_STATUS_CODE], 0, code) == 0) status[DEV_STATUS_WHERE] = where;
}

__device__ __forceinline__ int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(int *p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned ld_acquire_u(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

template <typename T> __device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename T> __device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

/// Block-wide all-reduce sum (every thread gets the total). `red` holds >= 32 values.
template <typename T, int NTHREADS> __device__ __forceinline__ T block_sum(T v, T *red) {
    constexpr int NW = NTHREADS / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    if (NW == 1) return v;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    T r = lane < NW ? red[lane] : T(0);
    r = warp_sum(r);
    return r;
}

/// Software grid barrier for cooperative launches, with a bounded wait.
///
/// All CTAs of the launch must be co-resident (cudaLaunchCooperativeKernel guarantees it).
/// `bar[0]` = arrival counter, `bar[1]` = generation.  Every CTA reads the generation once at
/// kernel start (`gen`), before its first arrival.  Returns false (and records
/// CUEV_ERR_TIMEOUT) if the generation does not advance within `limit_ns`.
struct GridBarrier {
    unsigned *bar;
    unsigned gen;
    unsigned nblocks;

    __device__ void init(unsigned *b) {
        bar = b;
        nblocks = gridDim.x * gridDim.y * gridDim.z;
        __shared__ unsigned s_gen;
        if (threadIdx.x == 0) s_gen = ld_acquire_u(&b[1]);
        __syncthreads();
        gen = s_gen;
        __syncthreads();
    }

    /// Returns true on success.  Must be called by all threads of every CTA.
    __device__ bool sync(int *status, int where) {
        const uint64_t limit_ns = wait_limit_ns(status);
        __shared__ int s_ok;
        __syncthreads();
        if (threadIdx.x == 0) {
            int ok = 1;
            __threadfence();
            unsigned arrived = atomicAdd(&bar[0], 1u);
            if (arrived == nblocks - 1) {
                atomicExch(&bar[0], 0u);
                __threadfence();
                atomicAdd(&bar[1], 1u);
            } else {
                const uint64_t t0 = global_ns();
                while (ld_acquire_u(&bar[1]) == gen) {
                    if (global_ns() - t0 > limit_ns) {
                        dev_fail(status, CUEV_ERR_TIMEOUT, where);
                        ok = 0;
                        break;
                    }
                    __nanosleep(32);
                }
            }
            // A CTA that observed an earlier failure must not keep going either.
            if (ok && ld_acquire(&status[DEV_STATUS_CODE]) != 0) ok = 0;
            s_ok = ok;
        }
        __syncthreads();
        gen += 1;
        return s_ok != 0;
    }
};

#endif // __CUDACC__

} // namespace cuev
