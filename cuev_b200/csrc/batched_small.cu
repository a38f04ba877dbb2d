// Batched eigensolver for many small symmetric matrices (n <= 64), one CTA per matrix: the
// "batched small-n eigh" path for framework wrappers that carry stacks of small problems.  The
// reference has no batched entry (its solve takes one matrix).
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
// eval batch x n, evec batch x (n x n column-major).  A and V live in shared memory
// (2 m (m + 1) doubles, m = n rounded up to even, 66 KB at n = 64).
#include "common.cuh"

#include <mutex>

namespace cuev {
namespace {

constexpr int BJ_THREADS = 256;
constexpr int BJ_MAXN = 64;
constexpr int BJ_MAX_SWEEPS = 60;

__global__ void __launch_bounds__(BJ_THREADS)
    batched_jacobi_kernel(const double *__restrict__ A, int n, double *__restrict__ eval,
                          double *__restrict__ evec, int *__restrict__ status) {
    extern __shared__ __align__(16) double bj_smem[];
    const int m = n + (n & 1); // even; index n is a dummy when n is odd
    const int LD = m + 1;
    double *sA = bj_smem;           // sA[i * LD + j] = A(i, j)
    double *sV = sA + m * LD;       // sV[i * LD + j] = V(i, j)
    __shared__ double cs_c[BJ_MAXN / 2], cs_s[BJ_MAXN / 2];
    __shared__ int cs_p[BJ_MAXN / 2], cs_q[BJ_MAXN / 2];
    __shared__ int s_rot;
    const int tid = threadIdx.x;
    const long long bofs = (long long)blockIdx.x * n * n;
    const double *Ab = A + bofs;

    for (int idx = tid; idx < m * m; idx += BJ_THREADS) {
        const int i = idx % m, j = idx / m;
        double v = 0.0;
        if (i < n && j < n) v = i >= j ? Ab[i + (long long)j * n] : Ab[j + (long long)i * n];
        sA[i * LD + j] = v;
        sV[i * LD + j] = (i == j) ? 1.0 : 0.0;
    }
    __syncthreads();

    const double eps = 2.220446049250313e-16;
    const double tiny = 2.2250738585072014e-308;
    const int half = m / 2;
    bool converged = (m <= 1);
    for (int sweep = 0; sweep < BJ_MAX_SWEEPS && !converged; ++sweep) {
        if (tid == 0) s_rot = 0;
        __syncthreads();
        for (int r = 0; r < m - 1; ++r) {
            // pairs of this round: slot 0 fixed, slots 1..m-1 rotate by r
            if (tid < half) {
                auto pos = [&](int slot) { return slot == 0 ? 0 : 1 + (slot - 1 + r) % (m - 1); };
                int p = pos(tid), q = pos(m - 1 - tid);
                if (p > q) { const int x = p; p = q; q = x; }
                double c = 1.0, s = 0.0;
                if (q < n) {
                    const double apq = sA[p * LD + q];
                    const double app = sA[p * LD + p], aqq = sA[q * LD + q];
                    if (fabs(apq) > tiny && fabs(apq) > eps * sqrt(fabs(app) * fabs(aqq))) {
                        const double tau = (aqq - app) / (2.0 * apq);
                        const double t =
                            (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                        c = 1.0 / sqrt(1.0 + t * t);
                        s = t * c;
                        atomicAdd(&s_rot, 1);
                    }
                }
                cs_p[tid] = p, cs_q[tid] = q;
                cs_c[tid] = c, cs_s[tid] = s;
            }
            __syncthreads();
            // rows: A <- J^T A  (rows p, q of every column j)
            for (int idx = tid; idx < half * m; idx += BJ_THREADS) {
                const int k = idx / m, j = idx % m;
                const double s = cs_s[k];
                if (s == 0.0) continue;
                const double c = cs_c[k];
                const int p = cs_p[k], q = cs_q[k];
                const double ap = sA[p * LD + j], aq = sA[q * LD + j];
                sA[p * LD + j] = c * ap - s * aq;
                sA[q * LD + j] = s * ap + c * aq;
            }
            __syncthreads();
            // columns: A <- A J, V <- V J  (columns p, q of every row i)
            for (int idx = tid; idx < 2 * half * m; idx += BJ_THREADS) {
                const int which = idx / (half * m), rem = idx % (half * m);
                const int k = rem / m, i = rem % m;
                const double s = cs_s[k];
                if (s == 0.0) continue;
                const double c = cs_c[k];
                const int p = cs_p[k], q = cs_q[k];
                double *X = which ? sV : sA;
                const double xp = X[i * LD + p], xq = X[i * LD + q];
                X[i * LD + p] = c * xp - s * xq;
                X[i * LD + q] = s * xp + c * xq;
            }
            __syncthreads();
            // the rotated pair's off-diagonal entry is zero by construction: store it exactly
            if (tid < half && cs_s[tid] != 0.0) {
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
    for (int i = tid; i < n; i += BJ_THREADS) {
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

// small per-device status buffer (one word per failure class); calls are serialised so that one
// call's reset cannot hide another call's failure
std::mutex g_bj_mu;
std::mutex g_bj_call_mu;
int *g_bj_status[64] = {nullptr};

} // namespace

int batched_eigh_d(const double *A, int n, int batch, double *eval, double *evec,
                   cudaStream_t st) {
    if (n < 0 || batch < 0) return CUEV_ERR_INVALID;
    if (n == 0 || batch == 0) return CUEV_OK;
    if (!A || !eval || !evec) return CUEV_ERR_INVALID;
    if (n > BJ_MAXN) {
        set_last_message("batched eigensolver: n > 64 (use the full solver per matrix)");
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
    const int m = n + (n & 1);
    const size_t smem = sizeof(double) * 2 * (size_t)m * (m + 1);
    CUEV_CHECK_STATUS(ensure_dyn_smem((const void *)batched_jacobi_kernel,
                                      sizeof(double) * 2 * BJ_MAXN * (BJ_MAXN + 1)));
    CUEV_TRY(cudaMemsetAsync(status, 0, DEV_STATUS_WORDS * sizeof(int), st));
    batched_jacobi_kernel<<<batch, BJ_THREADS, smem, st>>>(A, n, eval, evec, status);
    note_launch();
    CUEV_TRY(cudaGetLastError());
    int host[DEV_STATUS_WORDS] = {0};
    CUEV_TRY(cudaMemcpyAsync(host, status, sizeof(host), cudaMemcpyDeviceToHost, st));
    CUEV_TRY(cudaStreamSynchronize(st));
    if (host[DEV_STATUS_CODE] != 0) {
        char msg[128];
        snprintf(msg, sizeof(msg), "batched eigensolver: Jacobi did not converge (matrix %d)",
                 host[DEV_STATUS_WHERE]);
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
