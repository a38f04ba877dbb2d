// cuev_dgemm_noalloc: the split-K FP64 GEMM behind cuev_dgemm, for callers that cannot allocate
// device memory.
//
// cuev_dgemm gets its split-K partial-sum buffer from cudaMalloc the first time a problem needs
// it.  Some callers cannot let a library do that: a serving process whose device memory is
// fully owned by its framework's caching allocator (a foreign cudaMalloc can fail or fragment
// that pool), or a latency-critical loop where a device allocation can block the host on a
// device-wide synchronisation.  This entry point computes the same product with the partial
// sums in a fixed array that lives in the library itself, so it never allocates.
//
// The array is NOALLOC_SCRATCH_DOUBLES doubles (16 MiB) of device memory; every GPU that loads
// the library holds it until the process exits.  A call needs 2 * m * n doubles of it at least
// (a two-way split of K), so m * n is limited to NOALLOC_MAX_MN = 1,048,576.
//
// When the 16 MiB are committed: with lazy module loading (CUDA_MODULE_LOADING=LAZY, the default
// since CUDA 12) the array is created when the library's module is first loaded on a device,
// which can be this entry's first call there.  A caller whose framework reserves most of the
// device memory up front should make one call (a warm-up) before the framework takes its pool.
#include "common.cuh"
#include "gemm.cuh"

#include <algorithm>
#include <mutex>

namespace cuev {
namespace {

constexpr size_t NOALLOC_SCRATCH_DOUBLES = size_t(2) << 20; // 16 MiB
constexpr size_t NOALLOC_MAX_MN = NOALLOC_SCRATCH_DOUBLES / 2;

// Split-K partial sums of cuev_dgemm_noalloc.  Host code must not use this name as a device
// address: the device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_SCRATCH_DOUBLES];

std::mutex g_noalloc_mu;
double *g_noalloc_ptr[64] = {nullptr};

// Device address of the scratch array on the current device, looked up once per device
// (the first cuev_dgemm_noalloc call on a device does this).
int noalloc_scratch(double **out) {
    *out = nullptr;
    int dev = 0;
    CUEV_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) {
        set_last_message("cuev_dgemm_noalloc: device index out of range");
        return CUEV_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            set_last_error(e != cudaSuccess ? e : cudaErrorInvalidSymbol, __FILE__, __LINE__);
            return CUEV_ERR_CUDA;
        }
        g_noalloc_ptr[dev] = static_cast<double *>(p);
    }
    *out = g_noalloc_ptr[dev];
    return CUEV_OK;
}

} // namespace
} // namespace cuev

using namespace cuev;

extern "C" int cuev_dgemm_noalloc(void *stream, int ta, int tb, int m, int n, int k, double alpha,
                                  const double *A, int lda, const double *B, int ldb, double beta,
                                  double *C, int ldc) {
    if (m < 0 || n < 0 || k < 0 || !C || (k > 0 && (!A || !B))) {
        set_last_message("cuev_dgemm_noalloc: negative size or null pointer");
        return CUEV_ERR_INVALID;
    }
    if (ldc < m || lda < (ta ? k : m) || ldb < (tb ? n : k)) {
        set_last_message("cuev_dgemm_noalloc: leading dimension smaller than the matrix");
        return CUEV_ERR_INVALID;
    }
    if ((size_t)m * (size_t)n > NOALLOC_MAX_MN) {
        char msg[200];
        snprintf(msg, sizeof(msg),
                 "cuev_dgemm_noalloc: m*n = %lld exceeds the static-scratch limit of %zu "
                 "(use cuev_dgemm)",
                 (long long)m * n, NOALLOC_MAX_MN);
        set_last_message(msg);
        return CUEV_ERR_INVALID;
    }
    double *scratch = nullptr;
    CUEV_CHECK_STATUS(noalloc_scratch(&scratch));
    GemmArgs a{};
    a.m = m, a.n = n, a.k = k;
    a.A = A, a.lda = lda, a.B = B, a.ldb = ldb, a.C = C, a.ldc = ldc;
    a.alpha = alpha, a.beta = beta;
    // K is split at least two ways (when K has two or more 16-deep tiles) and as far as the
    // scratch allows.  Each split writes every element of its m x n partial before the
    // reduction reads it, so nothing has to be cleared between calls.
    const size_t mn = (size_t)m * n;
    int splits = gemm_splitk_count(m, n, k, 0);
    splits = (int)std::min<size_t>((size_t)std::max(splits, 2),
                                   mn ? NOALLOC_SCRATCH_DOUBLES / mn : 1);
    if (k < 32) splits = 1;
    a.splits = splits;
    a.ws = splits > 1 ? scratch : nullptr;
    return gemm_launch(a, ta, tb, (cudaStream_t)stream);
}
