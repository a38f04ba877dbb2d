// Differentiation form: the adjoint (reverse-mode derivative) of the symmetric eigensolve.
//
// For A = V diag(lam) V^T and a loss with cotangents lambar (eigenvalues) and Vbar
// (eigenvectors), the cotangent of A is
//     Abar = V ( diag(lambar) + sym(F o (V^T Vbar)) ) V^T,   F_ij = 1 / (lam_j - lam_i),
// with sym(X) = (X + X^T)/2 and F_ij = 0 on the diagonal and wherever |lam_j - lam_i| < gap_tol
// (near-degenerate pairs, whose true derivative is unbounded, are masked).  Only lam and V are
// needed from the forward solve, so nothing is recomputed.  The reference has no such form.
//
// Work: three n x n x n FP64 DMMA GEMMs (6 n^3 flops).  The Hadamard product with F and the
// diag(lambar) term are applied in the epilogue of the first GEMM (G = V^T Vbar), G is then
// symmetrised in place with a shared-memory tile transpose, and Abar = (V G) V^T.
#include "common.cuh"
#include "gemm.cuh"

#include <mutex>

namespace cuev {
namespace {

constexpr int TT = 32;

// G <- (G + G^T) / 2, tiles (bi, bj) with bi <= bj; each CTA handles one tile pair.
__global__ void symmetrize_kernel(double *__restrict__ G, int n, long long ld) {
    __shared__ double a[TT][TT + 1], b[TT][TT + 1];
    const int bi = blockIdx.y, bj = blockIdx.x;
    if (bi > bj) return;
    const int tx = threadIdx.x, ty = threadIdx.y; // 32 x 8
    for (int r = ty; r < TT; r += 8) {
        const int i = bi * TT + tx, j = bj * TT + r; // a[r][tx] = G(i, j)
        a[r][tx] = (i < n && j < n) ? G[i + (long long)j * ld] : 0.0;
        const int i2 = bj * TT + tx, j2 = bi * TT + r; // b[r][tx] = G(i2, j2)
        b[r][tx] = (i2 < n && j2 < n) ? G[i2 + (long long)j2 * ld] : 0.0;
    }
    __syncthreads();
    for (int r = ty; r < TT; r += 8) {
        // G(bi*TT + tx, bj*TT + r) = (a[r][tx] + G(bj*TT + r, bi*TT + tx)) / 2, the latter is b[tx][r]
        const int i = bi * TT + tx, j = bj * TT + r;
        const double v = 0.5 * (a[r][tx] + b[tx][r]);
        if (i < n && j < n) G[i + (long long)j * ld] = v;
        const int i2 = bj * TT + tx, j2 = bi * TT + r;
        const double v2 = 0.5 * (b[r][tx] + a[tx][r]);
        if (i2 < n && j2 < n) G[i2 + (long long)j2 * ld] = v2;
    }
}

__global__ void diag_fill_kernel(double *__restrict__ G, int n, long long ld,
                                 const double *__restrict__ lambar) {
    const long long total = (long long)n * n;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % n), j = (int)(idx / n);
        G[i + (long long)j * ld] = (i == j && lambar) ? lambar[i] : 0.0;
    }
}

__global__ void widen_kernel(const float *__restrict__ s, double *__restrict__ d, long long cnt) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cnt;
         i += (long long)gridDim.x * blockDim.x)
        d[i] = (double)s[i];
}
__global__ void narrow_kernel(const double *__restrict__ s, float *__restrict__ d, long long cnt) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cnt;
         i += (long long)gridDim.x * blockDim.x)
        d[i] = (float)s[i];
}

// n x n scratch for V G, cached per device (grows on demand).
std::mutex g_adj_mu;
void *g_adj_buf[64] = {nullptr};
size_t g_adj_bytes[64] = {0};

int adj_scratch(size_t bytes, double **out, cudaStream_t st) {
    int dev = 0;
    CUEV_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return CUEV_ERR_INVALID;
    std::lock_guard<std::mutex> lk(g_adj_mu);
    if (g_adj_bytes[dev] < bytes) {
        CUEV_TRY(cudaStreamSynchronize(st));
        if (g_adj_buf[dev]) CUEV_TRY(cudaFree(g_adj_buf[dev]));
        g_adj_buf[dev] = nullptr;
        g_adj_bytes[dev] = 0;
        if (cudaMalloc(&g_adj_buf[dev], bytes) != cudaSuccess) {
            cudaGetLastError();
            set_last_message("eigh adjoint: scratch allocation failed");
            return CUEV_ERR_ALLOC;
        }
        g_adj_bytes[dev] = bytes;
    }
    *out = (double *)g_adj_buf[dev];
    return CUEV_OK;
}

int adjoint_d(const double *V, const double *lam, const double *Vbar, const double *lambar, int n,
              double gap_tol, double *Abar, cudaStream_t st) {
    if (n < 0 || (n > 0 && (!V || !lam || !Abar))) return CUEV_ERR_INVALID;
    if (n == 0) return CUEV_OK;
    double *Y = nullptr;
    CUEV_CHECK_STATUS(adj_scratch(sizeof(double) * (size_t)n * n, &Y, st));
    // G = diag(lambar) + F o (V^T Vbar), written into Abar
    if (Vbar) {
        GemmArgs g{};
        g.m = n, g.n = n, g.k = n;
        g.A = V, g.lda = n, g.B = Vbar, g.ldb = n, g.C = Abar, g.ldc = n;
        g.alpha = 1.0, g.beta = 0.0, g.splits = 1;
        g.epi = 1, g.epi_lam = lam, g.epi_lambar = lambar, g.epi_gap = gap_tol;
        CUEV_CHECK_STATUS(gemm_launch(g, 1, 0, st));
    } else {
        diag_fill_kernel<<<4 * num_sms(), 256, 0, st>>>(Abar, n, n, lambar); note_launch();
        CUEV_TRY(cudaGetLastError());
    }
    const int nb = div_up(n, TT);
    symmetrize_kernel<<<dim3(nb, nb), dim3(32, 8), 0, st>>>(Abar, n, n); note_launch();
    CUEV_TRY(cudaGetLastError());
    // Abar = (V G) V^T
    GemmArgs y{};
    y.m = n, y.n = n, y.k = n;
    y.A = V, y.lda = n, y.B = Abar, y.ldb = n, y.C = Y, y.ldc = n;
    y.alpha = 1.0, y.beta = 0.0, y.splits = 1;
    CUEV_CHECK_STATUS(gemm_launch(y, 0, 0, st));
    GemmArgs z{};
    z.m = n, z.n = n, z.k = n;
    z.A = Y, z.lda = n, z.B = V, z.ldb = n, z.C = Abar, z.ldc = n;
    z.alpha = 1.0, z.beta = 0.0, z.splits = 1;
    CUEV_CHECK_STATUS(gemm_launch(z, 0, 1, st));
    return CUEV_OK;
}

} // namespace
} // namespace cuev

using namespace cuev;

extern "C" int cuev_dsyev_adjoint(const double *V, const double *lam, const double *Vbar,
                                  const double *lambar, int n, double gap_tol, double *Abar,
                                  void *stream) {
    return adjoint_d(V, lam, Vbar, lambar, n, gap_tol, Abar, (cudaStream_t)stream);
}

extern "C" int cuev_ssyev_adjoint(const float *V, const float *lam, const float *Vbar,
                                  const float *lambar, int n, float gap_tol, float *Abar,
                                  void *stream) {
    if (n < 0 || (n > 0 && (!V || !lam || !Abar))) return CUEV_ERR_INVALID;
    if (n == 0) return CUEV_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const long long nn = (long long)n * n;
    double *buf = nullptr;
    if (cudaMallocAsync((void **)&buf, sizeof(double) * (3 * nn + 2 * n), st) != cudaSuccess) {
        cudaGetLastError();
        set_last_message("FP32 adjoint: widening buffer allocation failed");
        return CUEV_ERR_ALLOC;
    }
    double *V64 = buf, *Vb64 = buf + nn, *A64 = buf + 2 * nn, *l64 = buf + 3 * nn,
           *lb64 = l64 + n;
    const int blocks = 4 * num_sms();
    widen_kernel<<<blocks, 256, 0, st>>>(V, V64, nn); note_launch();
    if (Vbar) { widen_kernel<<<blocks, 256, 0, st>>>(Vbar, Vb64, nn); note_launch(); }
    widen_kernel<<<1, 256, 0, st>>>(lam, l64, n); note_launch();
    if (lambar) { widen_kernel<<<1, 256, 0, st>>>(lambar, lb64, n); note_launch(); }
    int s = adjoint_d(V64, l64, Vbar ? Vb64 : nullptr, lambar ? lb64 : nullptr, n, (double)gap_tol,
                      A64, st);
    if (s == CUEV_OK) { narrow_kernel<<<blocks, 256, 0, st>>>(A64, Abar, nn); note_launch(); }
    cudaFreeAsync(buf, st);
    return s;
}
