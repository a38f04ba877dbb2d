// C-ABI wrappers around the FP64 GEMM kernels (the replacement for the reference's cuev::cublas
// wrappers, src/cuda/cublas.cu:15-56).  Split-K scratch for these standalone entries comes from
// a small per-device cache that grows on demand; the solver itself uses its workspace pool.
#include "common.cuh"
#include "gemm.cuh"
#include "tcgemm.cuh"

#include <mutex>

namespace cuev {
namespace {

struct ScratchCache {
    std::mutex mu;
    void *ptr[64] = {nullptr};
    size_t bytes[64] = {0};
};
ScratchCache g_scratch;

int scratch_get(size_t bytes, double **out, cudaStream_t stream) {
    *out = nullptr;
    if (bytes == 0) return CUEV_OK;
    int dev = 0;
    CUEV_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return CUEV_ERR_INVALID;
    std::lock_guard<std::mutex> lk(g_scratch.mu);
    if (g_scratch.bytes[dev] < bytes) {
        CUEV_TRY(cudaStreamSynchronize(stream));
        if (g_scratch.ptr[dev]) CUEV_TRY(cudaFree(g_scratch.ptr[dev]));
        g_scratch.ptr[dev] = nullptr;
        g_scratch.bytes[dev] = 0;
        if (cudaMalloc(&g_scratch.ptr[dev], bytes) != cudaSuccess) {
            cudaGetLastError();
            set_last_message("split-K scratch allocation failed");
            return CUEV_ERR_ALLOC;
        }
        g_scratch.bytes[dev] = bytes;
    }
    *out = (double *)g_scratch.ptr[dev];
    return CUEV_OK;
}

int run_gemm(GemmArgs a, int ta, int tb, cudaStream_t stream) {
    const int ktot = a.k + a.k2;
    a.splits = gemm_splitk_count(a.m, a.n, ktot, a.c_lower);
    if (a.splits > 1) {
        CUEV_CHECK_STATUS(scratch_get((size_t)a.splits * a.m * a.n * sizeof(double), &a.ws, stream));
    }
    return gemm_launch(a, ta, tb, stream);
}

} // namespace
} // namespace cuev

using namespace cuev;

extern "C" int cuev_dgemm(void *stream, int ta, int tb, int m, int n, int k, double alpha,
                          const double *A, int lda, const double *B, int ldb, double beta,
                          double *C, int ldc) {
    if (m < 0 || n < 0 || k < 0 || !C || (k > 0 && (!A || !B))) return CUEV_ERR_INVALID;
    if (ldc < m || lda < (ta ? k : m) || ldb < (tb ? n : k)) return CUEV_ERR_INVALID;
    GemmArgs a{};
    a.m = m, a.n = n, a.k = k;
    a.A = A, a.lda = lda, a.B = B, a.ldb = ldb, a.C = C, a.ldc = ldc;
    a.alpha = alpha, a.beta = beta;
    return run_gemm(a, ta, tb, (cudaStream_t)stream);
}

extern "C" int cuev_dsymm_lower(void *stream, int m, int n, double alpha, const double *A, int lda,
                                const double *B, int ldb, double beta, double *C, int ldc) {
    if (m < 0 || n < 0 || !C || (m > 0 && (!A || !B))) return CUEV_ERR_INVALID;
    if (lda < m || ldb < m || ldc < m) return CUEV_ERR_INVALID;
    GemmArgs a{};
    a.m = m, a.n = n, a.k = m;
    a.A = A, a.lda = lda, a.B = B, a.ldb = ldb, a.C = C, a.ldc = ldc;
    a.alpha = alpha, a.beta = beta, a.symm_a = 1;
    return run_gemm(a, 0, 0, (cudaStream_t)stream);
}

extern "C" int cuev_dsyr2k_lower(void *stream, int n, int k, double alpha, const double *A,
                                 int lda, const double *B, int ldb, double beta, double *C,
                                 int ldc) {
    if (n < 0 || k < 0 || !C || (k > 0 && (!A || !B))) return CUEV_ERR_INVALID;
    if (lda < n || ldb < n || ldc < n) return CUEV_ERR_INVALID;
    // alpha (A B^T + B A^T) = alpha [A | B] [B | A]^T : one GEMM over a two-segment K.
    GemmArgs a{};
    a.m = n, a.n = n, a.k = k, a.k2 = k;
    a.A = A, a.lda = lda, a.A2 = B, a.lda2 = ldb;
    a.B = B, a.ldb = ldb, a.B2 = A, a.ldb2 = lda;
    a.C = C, a.ldc = ldc, a.alpha = alpha, a.beta = beta, a.c_lower = 1;
    return run_gemm(a, 0, 1, (cudaStream_t)stream);
}

// FP64 GEMM emulated on the int8 tensor cores (tcgemm.cuh): `slices` 7-bit slices per operand
// (7 gives FP64-level products, 4 FP32-level ones).  Slices and the kernel's status word live in
// the same per-device scratch as the split-K partials above.  Blocks until the product is done,
// so that a bounded wait that gave up inside the kernel is returned as CUEV_ERR_TIMEOUT.
extern "C" int cuev_dgemm_i8(void *stream, int ta, int tb, int m, int n, int k, int slices,
                             double alpha, const double *A, int lda, const double *B, int ldb,
                             double beta, double *C, int ldc) {
    if (m < 0 || n < 0 || k < 0 || !C || (k > 0 && (!A || !B))) return CUEV_ERR_INVALID;
    if (ldc < m || lda < (ta ? k : m) || ldb < (tb ? n : k)) return CUEV_ERR_INVALID;
    if (slices < 1 || slices > 8) {
        set_last_message("cuev_dgemm_i8: slices must be in 1..8");
        return CUEV_ERR_INVALID;
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (m == 0 || n == 0) return CUEV_OK;
    if (k == 0 || alpha == 0.0) return cuev_dgemm(stream, ta, tb, m, n, k, alpha, A, lda, B, ldb,
                                                  beta, C, ldc);
    const size_t need = i8_gemm_scratch_bytes(m, n, k, slices) + 256;
    double *scr = nullptr;
    CUEV_CHECK_STATUS(scratch_get(need, &scr, st));
    int *status = (int *)((char *)scr + need - 256);
    CUEV_TRY(cudaMemsetAsync(status, 0, sizeof(int) * DEV_STATUS_WORDS, st));
    CUEV_CHECK_STATUS(apply_wait_limit(status, st));
    CUEV_CHECK_STATUS(i8_dgemm(ta, tb, 0, m, n, k, slices, alpha, A, lda, B, ldb, beta, C, ldc, 0,
                               scr, status, st));
    int host[DEV_STATUS_WORDS] = {0};
    CUEV_TRY(cudaMemcpyAsync(host, status, sizeof(host), cudaMemcpyDeviceToHost, st));
    CUEV_TRY(cudaStreamSynchronize(st));
    if (host[DEV_STATUS_CODE] != 0) {
        set_last_message("cuev_dgemm_i8: a bounded wait in the tensor-core kernel gave up");
        return host[DEV_STATUS_CODE];
    }
    return CUEV_OK;
}
