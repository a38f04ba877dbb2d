// Precision form, FP64 half: Ogita–Aishima iterative refinement of an approximate symmetric
// eigendecomposition (T. Ogita, K. Aishima, "Iterative refinement for symmetric eigenvalue
// decomposition", Japan J. Indust. Appl. Math. 35 (2018), Algorithm 1).  The reference has no
// such stage.
//
// For symmetric A (lower triangle read) and approximate eigenvectors X (n x n, columns), one step:
//   G = X^T X,  R = I - G,  S = X^T (A X),  lam_i = s_ii / g_ii            (= s_ii / (1 - r_ii))
//   delta = 2 (||S - diag(lam)|| + ||A|| ||R||)
//   E_ii = r_ii / 2,  E_ij = (s_ij + lam_j r_ij) / (lam_j - lam_i)  if |lam_j - lam_i| > delta,
//                     E_ij = r_ij / 2                                 otherwise      (i != j)
//   X <- X (I + E),  eigenvalues <- lam.
// For well separated eigenvalues the error of X falls quadratically.  The 2-norms of the method
// are replaced by Frobenius norms (upper bounds: delta only grows, which moves more pairs to the
// clustered branch and keeps the step safe), and ||A||_2 = max_i |lam_i|.
//
// Work per step: A X as a SYMM (2 n^3), X^T (A X) (2 n^3), the lower triangle of X^T X (n^3) and
// X (I + E) (2 n^3) on the FP64 DMMA GEMM, plus O(n^2) elementwise kernels and deterministic
// reductions (fixed grid, fixed summation order, so repeated calls agree bit for bit).
#include "common.cuh"
#include "gemm.cuh"
#include "refine.cuh"
#include "tcgemm.cuh"

#include <algorithm>
#include <cmath>
#include <mutex>

namespace cuev {
namespace {

constexpr int RF_THREADS = 256;

// scratch: AX (then I + E), S, G, X_new (n^2 each), partial sums, lam, scalars
std::mutex g_rf_mu;
std::mutex g_rf_call_mu; // one refinement at a time: the calls share the scratch below
void *g_rf_buf[64] = {nullptr};
size_t g_rf_bytes[64] = {0};

int rf_scratch(size_t bytes, void **out, cudaStream_t st) {
    int dev = 0;
    CUEV_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return CUEV_ERR_INVALID;
    std::lock_guard<std::mutex> lk(g_rf_mu);
    if (g_rf_bytes[dev] < bytes) {
        CUEV_TRY(cudaStreamSynchronize(st));
        if (g_rf_buf[dev]) CUEV_TRY(cudaFree(g_rf_buf[dev]));
        g_rf_buf[dev] = nullptr;
        g_rf_bytes[dev] = 0;
        if (cudaMalloc(&g_rf_buf[dev], bytes) != cudaSuccess) {
            cudaGetLastError();
            set_last_message("eigenpair refinement: scratch allocation failed");
            return CUEV_ERR_ALLOC;
        }
        g_rf_bytes[dev] = bytes;
    }
    *out = g_rf_buf[dev];
    return CUEV_OK;
}

__device__ __forceinline__ double block_sum(double v, double *red) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int q = 0; q < RF_THREADS / 32; ++q) s += red[q];
    __syncthreads();
    return s; // valid in thread 0
}

// lam_i = s_ii / g_ii
__global__ void rf_lambda_kernel(const double *__restrict__ S, const double *__restrict__ G,
                                 int n, double *__restrict__ lam) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const size_t d = (size_t)i * n + i;
        lam[i] = S[d] / G[d];
    }
}

// Per-block partial sums of ||S - diag(lam)||_F^2 and ||I - G||_F^2 (G lower triangle: each
// off-diagonal entry counted twice) and max |lam_i|: part[3 * block + {0, 1, 2}].
__global__ void __launch_bounds__(RF_THREADS)
    rf_norms_kernel(const double *__restrict__ S, const double *__restrict__ G,
                    const double *__restrict__ lam, int n, int s_lower,
                    double *__restrict__ part) {
    __shared__ double red[RF_THREADS / 32];
    double so = 0.0, ro = 0.0, am = 0.0;
    const size_t total = (size_t)n * n;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(idx % n), j = (int)(idx / n);
        const double s = S[idx];
        if (i == j) {
            const double ds = s - lam[i];
            const double dr = 1.0 - G[idx];
            so += ds * ds;
            ro += dr * dr;
            am = fmax(am, fabs(lam[i]));
        } else if (!s_lower) {
            so += s * s;
            if (i > j) ro += 2.0 * G[idx] * G[idx];
        } else if (i > j) { // lower triangles only: each off-diagonal entry stands for two
            so += 2.0 * s * s;
            ro += 2.0 * G[idx] * G[idx];
        }
    }
    so = block_sum(so, red);
    ro = block_sum(ro, red);
    am = warp_max(am);
    __shared__ double mx[RF_THREADS / 32];
    if ((threadIdx.x & 31) == 0) mx[threadIdx.x >> 5] = am;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int q = 0; q < RF_THREADS / 32; ++q) m = fmax(m, mx[q]);
        part[3 * blockIdx.x + 0] = so;
        part[3 * blockIdx.x + 1] = ro;
        part[3 * blockIdx.x + 2] = m;
    }
}

// scal[0] = ||S - diag||_F, scal[1] = ||R||_F, scal[2] = max|lam|, scal[3] = delta
__global__ void rf_finish_kernel(const double *__restrict__ part, int nblocks,
                                 double *__restrict__ scal) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double so = 0.0, ro = 0.0, am = 0.0;
    for (int q = 0; q < nblocks; ++q) {
        so += part[3 * q + 0];
        ro += part[3 * q + 1];
        am = fmax(am, part[3 * q + 2]);
    }
    scal[0] = sqrt(so);
    scal[1] = sqrt(ro);
    scal[2] = am;
    scal[3] = 2.0 * (scal[0] + am * scal[1]);
}

// B = I + E from S (full) and G (lower triangle).  The computed S = X^T (A X) is not exactly
// symmetric; its antisymmetric rounding part, divided by a small gap, would break
// E_ij + E_ji = r_ij (the identity that keeps X (I + E) orthonormal to second order), so the
// symmetric part (s_ij + s_ji) / 2 is used.
// With s_lower, S holds only its lower triangle (computed as a symmetric product) and that is
// s_ij; with e_only, B receives E itself (for X <- X + X E).
__global__ void rf_update_kernel(const double *__restrict__ S, const double *__restrict__ G,
                                 const double *__restrict__ lam, const double *__restrict__ scal,
                                 int n, int s_lower, int e_only, double *__restrict__ B) {
    const double delta = scal[3];
    const size_t total = (size_t)n * n;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(idx % n), j = (int)(idx / n);
        const size_t mir = (size_t)i * n + j; // element (j, i)
        const double g = i >= j ? G[idx] : G[mir];
        double e;
        if (i == j) {
            e = 0.5 * (1.0 - g); // r_ii / 2
        } else {
            const double r = -g; // r_ij = -g_ij off the diagonal
            const double gap = lam[j] - lam[i];
            const double sij = s_lower ? (i >= j ? S[idx] : S[mir]) : 0.5 * (S[idx] + S[mir]);
            e = fabs(gap) > delta ? (sij + lam[j] * r) / gap : 0.5 * r;
        }
        B[idx] = (i == j && !e_only ? 1.0 : 0.0) + e;
    }
}

int gemm_plain(int ta, int tb, int m, int n, int k, double alpha, const double *A, int lda,
               const double *B, int ldb, double beta, double *C, int ldc, int c_lower,
               cudaStream_t st) {
    GemmArgs g{};
    g.m = m, g.n = n, g.k = k;
    g.A = A, g.lda = lda, g.B = B, g.ldb = ldb, g.C = C, g.ldc = ldc;
    g.alpha = alpha, g.beta = beta, g.splits = 1, g.c_lower = c_lower;
    return gemm_launch(g, ta, tb, st);
}

} // namespace

size_t refine_scratch_bytes(int n, int products) {
    const size_t nn = (size_t)n * n;
    const int nblocks = 4 * num_sms();
    size_t b = align256(sizeof(double) * (4 * nn + 3 * (size_t)nblocks + n + 8)) + 256;
    if (products == CUEV_PRODUCTS_INT8) b += 2 * i8_operand_bytes(n, n, RF_SLICES_HI);
    return b;
}

int refine_core(const double *A, const I8Operand *A_sl, int n, double *eval, double *X,
                int max_iters, double tol, int products, cudaStream_t st,
                cuev_refine_info *info) {
    if (n < 0 || max_iters < 0) return CUEV_ERR_INVALID;
    if (products != CUEV_PRODUCTS_FP64 && products != CUEV_PRODUCTS_INT8) {
        set_last_message("eigenpair refinement: unknown product precision");
        return CUEV_ERR_INVALID;
    }
    if (info) *info = cuev_refine_info{};
    if (n == 0 || max_iters == 0) return CUEV_OK;
    if ((!A && !A_sl) || !eval || !X) return CUEV_ERR_INVALID;
    const size_t nn = (size_t)n * n;
    const int nblocks = 4 * num_sms();
    const bool emu = products == CUEV_PRODUCTS_INT8;
    std::lock_guard<std::mutex> call_lock(g_rf_call_mu); // held until the call has synchronised
    // A's own slices when the caller did not bring them
    const size_t a_sl_bytes = (emu && !A_sl) ? i8_operand_bytes(n, n, RF_SLICES_HI) : 0;
    void *buf = nullptr;
    CUEV_CHECK_STATUS(rf_scratch(refine_scratch_bytes(n, products) + a_sl_bytes, &buf, st));
    double *AX = (double *)buf, *S = AX + nn, *G = S + nn, *Xn = G + nn;
    double *part = Xn + nn, *lam = part + 3 * (size_t)nblocks, *scal = lam + n;
    char *tail = (char *)buf + align256(sizeof(double) * (4 * nn + 3 * (size_t)nblocks + n + 8));
    int *status = (int *)tail;
    tail += 256;
    I8Operand Xk, Yk, Aown;
    if (emu) {
        i8_operand_init(tail, n, n, RF_SLICES_HI, Xk);
        tail += i8_operand_bytes(n, n, RF_SLICES_HI);
        i8_operand_init(tail, n, n, RF_SLICES_HI, Yk);
        tail += i8_operand_bytes(n, n, RF_SLICES_HI);
        CUEV_TRY(cudaMemsetAsync(status, 0, sizeof(int) * DEV_STATUS_WORDS, st));
        CUEV_CHECK_STATUS(apply_wait_limit(status, st));
        if (!A_sl) {
            i8_operand_init(tail, n, n, RF_SLICES_HI, Aown);
            CUEV_CHECK_STATUS(i8_slice(A, n, I8_SRC_SYML, Aown, st));
            A_sl = &Aown;
        }
    }
    const int eb = std::min(nblocks, div_up(n, RF_THREADS));
    double host[4] = {0, 0, 0, 0};
    int hstat[DEV_STATUS_WORDS] = {0};
    // Each pass measures the current X (G, S, lam, norms) and, unless it has converged, replaces
    // X by X (I + E); the eigenvalues returned are the lam of the last pass (Algorithm 1 returns
    // the new X with the lam computed from the old one).
    int it = 0;
    for (; it < max_iters; ++it) {
        if (!emu) {
            // A X (A symmetric, lower triangle), S = X^T (A X), lower(G) = lower(X^T X)
            GemmArgs y{};
            y.m = n, y.n = n, y.k = n;
            y.A = A, y.lda = n, y.B = X, y.ldb = n, y.C = AX, y.ldc = n;
            y.alpha = 1.0, y.beta = 0.0, y.splits = 1, y.symm_a = 1;
            CUEV_CHECK_STATUS(gemm_launch(y, 0, 0, st));
            CUEV_CHECK_STATUS(gemm_plain(1, 0, n, n, n, 1.0, X, n, AX, n, 0.0, S, n, 0, st));
            CUEV_CHECK_STATUS(gemm_plain(1, 0, n, n, n, 1.0, X, n, X, n, 0.0, G, n, 1, st));
        } else {
            // X's slices serve as op(B) = X of A X and as op(A) = X^T of X^T (A X) and X^T X
            CUEV_CHECK_STATUS(i8_slice(X, n, I8_SRC_KMAJ, Xk, st));
            CUEV_CHECK_STATUS(i8_gemm(*A_sl, Xk, RF_SLICES_HI, 1.0, 0.0, AX, n, 0, status, st));
            CUEV_CHECK_STATUS(i8_slice(AX, n, I8_SRC_KMAJ, Yk, st));
            CUEV_CHECK_STATUS(i8_gemm(Xk, Yk, RF_SLICES_HI, 1.0, 0.0, S, n, 1, status, st));
            CUEV_CHECK_STATUS(i8_gemm(Xk, Xk, RF_SLICES_HI, 1.0, 0.0, G, n, 1, status, st));
        }
        rf_lambda_kernel<<<eb, RF_THREADS, 0, st>>>(S, G, n, lam); note_launch();
        rf_norms_kernel<<<nblocks, RF_THREADS, 0, st>>>(S, G, lam, n, emu ? 1 : 0, part);
        note_launch();
        rf_finish_kernel<<<1, 32, 0, st>>>(part, nblocks, scal); note_launch();
        CUEV_TRY(cudaGetLastError());
        CUEV_TRY(cudaMemcpyAsync(host, scal, sizeof(host), cudaMemcpyDeviceToHost, st));
        if (emu)
            CUEV_TRY(cudaMemcpyAsync(hstat, status, sizeof(hstat), cudaMemcpyDeviceToHost, st));
        CUEV_TRY(cudaStreamSynchronize(st));
        if (hstat[DEV_STATUS_CODE] != 0) {
            set_last_message("eigenpair refinement: a bounded wait in the tensor-core GEMM gave up");
            return hstat[DEV_STATUS_CODE];
        }
        if (!std::isfinite(host[0]) || !std::isfinite(host[1])) {
            set_last_message("eigenpair refinement: non-finite residual");
            return CUEV_ERR_NONFINITE;
        }
        if (tol > 0.0 && host[1] <= tol && host[0] <= tol * std::max(host[2], 1e-300)) break;
        if (!emu) {
            // B = I + E into the A X buffer (free once S is formed), then X <- X B
            rf_update_kernel<<<nblocks, RF_THREADS, 0, st>>>(S, G, lam, scal, n, 0, 0, AX);
            note_launch();
            CUEV_TRY(cudaGetLastError());
            CUEV_CHECK_STATUS(gemm_plain(0, 0, n, n, n, 1.0, X, n, AX, n, 0.0, Xn, n, 0, st));
            CUEV_TRY(cudaMemcpyAsync(X, Xn, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st));
        } else {
            // E into the A X buffer, then X <- X + X E: X's row slices are taken before X is
            // updated in place, so the epilogue's read of X (beta = 1) sees the old X
            rf_update_kernel<<<nblocks, RF_THREADS, 0, st>>>(S, G, lam, scal, n, 1, 1, AX);
            note_launch();
            CUEV_TRY(cudaGetLastError());
            I8Operand Xr, Ek;
            i8_operand_init(Yk.data, n, n, RF_SLICES_CORR, Xr);
            i8_operand_init(Xk.data, n, n, RF_SLICES_CORR, Ek);
            CUEV_CHECK_STATUS(i8_slice(X, n, I8_SRC_RMAJ, Xr, st));
            CUEV_CHECK_STATUS(i8_slice(AX, n, I8_SRC_KMAJ, Ek, st));
            CUEV_CHECK_STATUS(i8_gemm(Xr, Ek, RF_SLICES_CORR, 1.0, 1.0, X, n, 0, status, st));
        }
    }
    CUEV_TRY(cudaMemcpyAsync(eval, lam, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    if (emu) CUEV_TRY(cudaMemcpyAsync(hstat, status, sizeof(hstat), cudaMemcpyDeviceToHost, st));
    CUEV_TRY(cudaStreamSynchronize(st));
    if (hstat[DEV_STATUS_CODE] != 0) {
        set_last_message("eigenpair refinement: a bounded wait in the tensor-core GEMM gave up");
        return hstat[DEV_STATUS_CODE];
    }
    if (info) {
        info->iterations = it;
        info->offdiag_fro = host[0];
        info->orth_fro = host[1];
        info->anorm = host[2];
    }
    return CUEV_OK;
}

} // namespace cuev

extern "C" int cuev_dsyev_refine(const double *A, int n, double *eval, double *evec,
                                 int max_iters, double tol, void *stream,
                                 cuev_refine_info *info) {
    return cuev::refine_core(A, nullptr, n, eval, evec, max_iters, tol, CUEV_PRODUCTS_FP64,
                             (cudaStream_t)stream, info);
}

extern "C" int cuev_dsyev_refine_ex(const double *A, int n, double *eval, double *evec,
                                    int max_iters, double tol, int products, void *stream,
                                    cuev_refine_info *info) {
    return cuev::refine_core(A, nullptr, n, eval, evec, max_iters, tol, products,
                             (cudaStream_t)stream, info);
}
