// Batched eigensolver for many small symmetric matrices (n <= 64 here; 64 < n <= 512 in
// batched_mid.cu), one CTA per matrix: the "batched small-n eigh" path for framework wrappers that
// carry stacks of small problems.  The reference has no batched entry (its solve takes one
// matrix).
//
// Method: two-sided cyclic Jacobi with the round-robin (tournament) ordering, so each round
// rotates n/2 disjoint index pairs at once.  For a pair (p, q) the rotation is the symmetric
// 2 x 2 Schur decomposition (G. H. Golub, C. F. Van Loan, Matrix Computations, 4th ed.,
// Algorithm 8.5.1): tau = (a_qq - a_pp) / (2 a_pq), t = sign(tau) / (|tau| + sqrt(1 + tau^2)),
// c = 1 / sqrt(1 + t^2), s = t c, and with J = [c s; -s c] in the (p, q) plane
// A <- J^T A J zeroes a_pq (then stored as an exact zero) and V <- V J accumulates the
// eigenvectors.  A rotation is skipped when |a_pq| <= eps sqrt(|a_pp a_qq|) (or a_pq is below
// the smallest normal number); a sweep that skips every pair ends the
// iteration (at most 60 sweeps, else CUEV_ERR_CONVERGENCE).  Jacobi converges quadratically and
// gives eigenvalues with small relative error.  The eigenpairs are then ranked in parallel and
// written in ascending order.
//
// Layout: A is batch x (n x n column-major, stride n^2), lower triangle read, not modified;
// eval batch x n, evec batch x (n x n column-major).  A and V live in shared memory, padded to
// M x M with M in {8, 16, 32, 64} the smallest that holds n (2 M (M + 1) doubles, 66 KB at
// M = 64); the padding rows and columns are zero and every pair with an index >= n is skipped, so
// they never mix with the matrix.  M and the thread count (32, 64, 256, 256) are compile-time,
// so the index arithmetic of the update loops is shifts and masks.
#include "common.cuh"

#include <mutex>

namespace cuev {
namespace {

constexpr int BJ_MAXN = 64;
constexpr int BMID_MAXN = 512;
constexpr int BJ_MAX_SWEEPS = 60;

template <int M, int NT>
__global__ void __launch_bounds__(NT)
    batched_jacobi_kernel(const double *__restrict__ A, int n, double *__restrict__ eval,
                          double *__restrict__ evec, int *__restrict__ status) {
    extern __shared__ __align__(16) double bj_smem[];
    constexpr int LD = M + 1;
    constexpr int HALF = M / 2;
    double *sA = bj_smem;     // sA[i * LD + j] = A(i, j)
    double *sV = sA + M * LD; // sV[i * LD + j] = V(i, j)
    __shared__ double cs_c[HALF], cs_s[HALF];
    __shared__ int cs_p[HALF], cs_q[HALF];
    __shared__ int s_rot;
    const int tid = threadIdx.x;
    const long long bofs = (long long)blockIdx.x * n * n;
    const double *Ab = A + bofs;

    for (int idx = tid; idx < M * M; idx += NT) {
        const int i = idx % M, j = idx / M;
        double v = 0.0;
        if (i < n && j < n) v = i >= j ? Ab[i + (long long)j * n] : Ab[j + (long long)i * n];
        sA[i * LD + j] = v;
        sV[i * LD + j] = (i == j) ? 1.0 : 0.0;
    }
    __syncthreads();

    const double eps = 2.220446049250313e-16;
    const double tiny = 2.2250738585072014e-308;
    bool converged = (n <= 1);
    for (int sweep = 0; sweep < BJ_MAX_SWEEPS && !converged; ++sweep) {
        if (tid == 0) s_rot = 0;
        __syncthreads();
        for (int r = 0; r < M - 1; ++r) {
            // pairs of this round: slot 0 fixed, slots 1..M-1 rotate by r
            if (tid < HALF) {
                auto pos = [&](int slot) { return slot == 0 ? 0 : 1 + (slot - 1 + r) % (M - 1); };
                int p = pos(tid), q = pos(M - 1 - tid);
                if (p > q) { const int x = p; p = q; q = x; }
                double c = 1.0, sn = 0.0;
                if (q < n) {
                    const double apq = sA[p * LD + q];
                    const double app = sA[p * LD + p], aqq = sA[q * LD + q];
                    if (fabs(apq) > tiny && fabs(apq) > eps * sqrt(fabs(app) * fabs(aqq))) {
                        const double tau = (aqq - app) / (2.0 * apq);
                        const double t =
                            (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                        c = 1.0 / sqrt(1.0 + t * t);
                        sn = t * c;
                        atomicAdd(&s_rot, 1);
                    }
                }
                cs_p[tid] = p, cs_q[tid] = q;
                cs_c[tid] = c, cs_s[tid] = sn;
            }
            __syncthreads();
            // rows: A <- J^T A  (rows p, q of every column j)
            for (int idx = tid; idx < HALF * M; idx += NT) {
                const int k = idx / M, j = idx % M;
                const double sn = cs_s[k];
                if (sn == 0.0) continue;
                const double c = cs_c[k];
                const int p = cs_p[k], q = cs_q[k];
                const double ap = sA[p * LD + j], aq = sA[q * LD + j];
                sA[p * LD + j] = c * ap - sn * aq;
                sA[q * LD + j] = sn * ap + c * aq;
            }
            __syncthreads();
            // columns: A <- A J, V <- V J  (columns p, q of every row i)
            for (int idx = tid; idx < 2 * HALF * M; idx += NT) {
                const int which = idx / (HALF * M), rem = idx % (HALF * M);
                const int k = rem / M, i = rem % M;
                const double sn = cs_s[k];
                if (sn == 0.0) continue;
                const double c = cs_c[k];
                const int p = cs_p[k], q = cs_q[k];
                double *X = which ? sV : sA;
                const double xp = X[i * LD + p], xq = X[i * LD + q];
                X[i * LD + p] = c * xp - sn * xq;
                X[i * LD + q] = sn * xp + c * xq;
            }
            __syncthreads();
            // the rotated pair's off-diagonal entry is zero by construction: store it exactly
            if (tid < HALF && cs_s[tid] != 0.0) {
                sA[cs_p[tid] * LD + cs_q[tid]] = 0.0;
                sA[cs_q[tid] * LD + cs_p[tid]] = 0.0;
            }
            __syncthreads();
        }
        converged = (s_rot == 0);
        __syncthreads();
    }
    if (!converged && tid == 0) dev_fail(status, CUEV_ERR_CONVERGENCE, blockIdx.x);

    // rank the eigenvalues (ties broken by index) and write ascending eigenpairs
    double *ev = eval + (long long)blockIdx.x * n;
    double *V = evec + bofs;
    for (int i = tid; i < n; i += NT) {
        const double li = sA[i * LD + i];
        int rank = 0;
        for (int j = 0; j < n; ++j) {
            const double lj = sA[j * LD + j];
            rank += (lj < li) || (lj == li && j < i);
        }
        ev[rank] = li;
        for (int row = 0; row < n; ++row) V[row + (long long)rank * n] = sV[row * LD + i];
    }
}

template <int M, int NT>
int launch_jacobi(const double *A, int n, int batch, double *eval, double *evec, int *status,
                  cudaStream_t st) {
    auto kern = batched_jacobi_kernel<M, NT>;
    const size_t smem = sizeof(double) * 2 * (size_t)M * (M + 1);
    CUEV_CHECK_STATUS(ensure_dyn_smem((const void *)kern, smem));
    kern<<<batch, NT, smem, st>>>(A, n, eval, evec, status);
    note_launch();
    CUEV_TRY(cudaGetLastError());
    return CUEV_OK;
}

// small per-device status buffer (one word per failure class); calls are serialised so that one
// call's reset cannot hide another call's failure
std::mutex g_bj_mu;
std::mutex g_bj_call_mu;
int *g_bj_status[64] = {nullptr};

} // namespace

// 64 < n <= 512: Householder tridiagonalisation + implicit QL, one CTA per matrix (batched_mid.cu)
int batched_eigh_mid(const double *A, int n, int batch, double *eval, double *evec, int *status,
                     cudaStream_t st);

int batched_eigh_d(const double *A, int n, int batch, double *eval, double *evec,
                   cudaStream_t st) {
    if (n < 0 || batch < 0) return CUEV_ERR_INVALID;
    if (n == 0 || batch == 0) return CUEV_OK;
    if (!A || !eval || !evec) return CUEV_ERR_INVALID;
    if (n > BMID_MAXN) {
        set_last_message("batched eigensolver: n > 512 (use the full solver per matrix)");
        return CUEV_ERR_UNSUPPORTED;
    }
    int dev = 0;
    CUEV_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return CUEV_ERR_INVALID;
    std::lock_guard<std::mutex> call_lock(g_bj_call_mu); // held until the call has synchronised
    int *status = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_bj_mu);
        if (!g_bj_status[dev]) CUEV_TRY(cudaMalloc(&g_bj_status[dev], DEV_STATUS_WORDS * sizeof(int)));
        status = g_bj_status[dev];
    }
    CUEV_TRY(cudaMemsetAsync(status, 0, DEV_STATUS_WORDS * sizeof(int), st));
    if (n <= 8)
        CUEV_CHECK_STATUS((launch_jacobi<8, 32>(A, n, batch, eval, evec, status, st)));
    else if (n <= 16)
        CUEV_CHECK_STATUS((launch_jacobi<16, 64>(A, n, batch, eval, evec, status, st)));
    else if (n <= 32)
        CUEV_CHECK_STATUS((launch_jacobi<32, 256>(A, n, batch, eval, evec, status, st)));
    else if (n <= BJ_MAXN)
        CUEV_CHECK_STATUS((launch_jacobi<64, 256>(A, n, batch, eval, evec, status, st)));
    else
        CUEV_CHECK_STATUS(batched_eigh_mid(A, n, batch, eval, evec, status, st));
    int host[DEV_STATUS_WORDS] = {0};
    CUEV_TRY(cudaMemcpyAsync(host, status, sizeof(host), cudaMemcpyDeviceToHost, st));
    CUEV_TRY(cudaStreamSynchronize(st));
    if (host[DEV_STATUS_CODE] != 0) {
        char msg[128];
        if (host[DEV_STATUS_CODE] == CUEV_ERR_NONFINITE)
            snprintf(msg, sizeof(msg), "batched eigensolver: NaN or Inf in matrix %d",
                     host[DEV_STATUS_WHERE]);
        else
            snprintf(msg, sizeof(msg), "batched eigensolver: %s did not converge (matrix %d)",
                     n <= BJ_MAXN ? "Jacobi" : "QL", host[DEV_STATUS_WHERE]);
        set_last_message(msg);
        return host[DEV_STATUS_CODE];
    }
    return CUEV_OK;
}

} // namespace cuev

extern "C" int cuev_dsyevd_batched(const double *A, int n, int batch, double *eval, double *evec,
                                   void *stream) {
    return cuev::batched_eigh_d(A, n, batch, eval, evec, (cudaStream_t)stream);
}
