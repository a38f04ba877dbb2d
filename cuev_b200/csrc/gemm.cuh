// FP64 tensor-core GEMM for sm_100a: C = alpha * op(A) * op(B) + beta * C, column-major.
//
// tcgen05 has no f64 kind, so FP64 contractions run on the DMMA path
// (`mma.sync.aligned.m16n8k8.row.col.f64`), fed by a multi-stage cp.async shared-memory
// pipeline synchronised on mbarriers.  One kernel template covers every contraction the solver needs:
//   - plain GEMM with op(A), op(B) in {N, T}                       (reference cublas::gemm)
//   - SYMM with A symmetric, lower triangle read                  (reference cublas::symm LOWER)
//   - SYR2K as one GEMM over a two-segment K: [A1 | A2] [B1 | B2]^T, lower triangle written
//                                                                  (reference cublas::syr2k LOWER)
//   - deterministic split-K (partials in a workspace, then a reduction kernel)
//   - batched problems whose sizes live in device memory (D&C merges of one tree level)
#pragma once
#include "common.cuh"

namespace cuev {

struct GemmArgs {
    int m, n, k;             // op(A): m x k, op(B): k x n   (first K segment)
    int k2;                  // second K segment length (0 = none)
    const double *A, *A2;    // op(A) = A (or A^T); A2 is the second K segment of op(A)
    const double *B, *B2;
    long long lda, lda2, ldb, ldb2;
    double *C;
    long long ldc;
    double alpha, beta;
    int c_lower;             // 1: only C(i, j) with i >= j is computed and written
    int symm_a;              // 1: A is symmetric m x m, only its lower triangle is read
    double *ws;              // split-K partial sums: splits x (m x n), ld m
    int splits;
    // Optional eigh-adjoint epilogue (m == n): C_ii = lambar_i and, for i != j,
    // C_ij = alpha acc_ij / (lam_j - lam_i), or 0 when |lam_j - lam_i| < epi_gap.
    // Not combined with split-K.
    const double *epi_lam, *epi_lambar;
    double epi_gap;
    int epi;
};

// Host launchers (gemm.cu).  All enqueue on `stream` and return a cuev_status.
int gemm_launch(const GemmArgs &a, int ta, int tb, cudaStream_t stream);
// Batched form: `dev_args` is an array of `count` GemmArgs in device memory (all with the same
// ta/tb, no split-K).  max_m/max_n bound every problem's m/n (they size the grid).
int gemm_batched_launch(const GemmArgs *dev_args, int count, int max_m, int max_n, int ta, int tb,
                        cudaStream_t stream);

// Records CUEV_ERR_TIMEOUT (detail -100) in `status` (stream ordered) if a stage wait of any GEMM
// has given up since the library was loaded (sticky; the waits only depend on the CTA's own
// copies, so this means a device fault).
int gemm_fold_fault(int *status, cudaStream_t stream);

// Split-K workspace needed by gemm_launch for a problem (0 when no split is used).
size_t gemm_splitk_workspace(int m, int n, int k_total, int ta, int tb, int c_lower);
// Split-K count for gemm_launch (at most max_splits, which callers derive from their scratch).
int gemm_splitk_count(int m, int n, int k_total, int c_lower, int max_splits = 32);

} // namespace cuev
