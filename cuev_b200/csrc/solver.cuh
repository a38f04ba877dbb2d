// Internal stage interfaces and the device workspace of one solve.
//
// Data layout in HBM (FP64, column-major, ld = n unless noted):
//   A      caller's n x n input, lower triangle read; used as the DBBR working matrix, then as
//          D&C scratch once the band has been packed
//   Y      n x n   DBBR Householder vectors (panel j: columns j..j+b-1, rows j+b..n-1;
//                  zero above) — Q_s = prod_j (I - Y_j T_j Y_j^T)
//   Z      n x k   DBBR two-sided companion of the current k-block
//   Wp     n x b   W = Y_j T_j of the current panel
//   Tp     b x b per panel (n/b + 1 of them)
//   Tblk   k x k per k-block: aggregated WY factor for the back-transform
//   B      2b x n  packed band + bulge space, B[(i - j) + j 2b] = A(i, j)  (L2-resident)
//   U      n x n   bulge-chasing reflectors, column s = all hops of sweep s (rows s+1..n-1)
//   d, e   tridiagonal
//   Q2, S  n x n   D&C merge scratch (compressed eigenvector blocks, secular differences)
#pragma once
#include "common.cuh"
#include "gemm.cuh"
#include "tcgemm.cuh"

namespace cuev {

struct Workspace {
    int n = 0, b = 0, k = 0;
    int dev = 0;
    cudaStream_t stream = nullptr;
    // high-priority stream and two events for the back-transform's overlap of BC-back's last,
    // partial wave with the SBR-back of the columns already finished
    cudaStream_t side = nullptr;
    cudaEvent_t ev_a = nullptr, ev_b = nullptr;
    // host-buffer entry: while host_evec is set, the back-transform copies the finished
    // eigenvector columns to it (the whole waves' columns on the side stream while the last
    // columns are still being computed; ev_c / ev_d order those copies)
    double *host_evec = nullptr;
    cudaEvent_t ev_c = nullptr, ev_d = nullptr;

    double *Y = nullptr, *Z = nullptr, *Wp = nullptr, *Tp = nullptr, *Tblk = nullptr;
    double *tau = nullptr, *Dwk = nullptr, *Gblk = nullptr;
    double *B = nullptr, *U = nullptr, *d = nullptr, *e = nullptr;
    int *prog = nullptr; // 2n words: bulge-chase progress per sweep (hops done, betas written)
    unsigned *bar = nullptr; // grid-barrier words for cooperative kernels
    int *status = nullptr;   // device status words (DEV_STATUS_WORDS ints)
    double *dc_flops = nullptr; // flops of the D&C merge GEMMs of the last tridi_dc (after deflation)
    double *qr_part = nullptr;
    size_t qr_part_elems = 0;
    double *splitk = nullptr;
    size_t splitk_bytes = 0;

    // D&C
    double *dc_Q2 = nullptr, *dc_S = nullptr, *dc_T = nullptr, *dc_vec = nullptr;
    int *dc_int = nullptr;
    size_t dc_vec_elems = 0, dc_int_elems = 0;
    GemmArgs *dc_gemm_args = nullptr;
    int dc_gemm_args_cap = 0;

    double *tmp_nn = nullptr; // n x n scratch (back-transform / D&C output staging)

    // Precision form (cuev_dsyevd_mixed) and the FP32 entry: while `mixed` is set, the
    // back-transform's large GEMMs run as FP32-level int8 tensor-core products (MIXED_SLICES
    // slices).  Buffers are allocated on first use: the slices of one GEMM's operands and, for the
    // refinement, A's FP64-level slices (taken before the band reduction overwrites A).
    int mixed = 0;
    void *mx_pool = nullptr;
    size_t mx_bytes = 0;
    bool mx_has_a = false;
    I8Operand a_sl;
    void *i8_scratch = nullptr;
    size_t i8_scratch_bytes = 0;
    // FP32 entry: while `fp32` is set (b = 32), BC-back runs in FP32 on float copies of U and of
    // the eigenvector columns (f32_pool: Uf and Mf, n x n floats each)
    int fp32 = 0;
    void *f32_pool = nullptr;
    float *Uf = nullptr, *Mf = nullptr;

    void *pool = nullptr;
    size_t pool_bytes = 0;
};

// Allocation / release of a workspace for (n, b, k).
int workspace_create(int n, int b, int k, cudaStream_t stream, Workspace **out);
// Allocate the precision form's buffers (GEMM slices; with_a_slices: also A's slices).
int workspace_enable_mixed(Workspace *ws, bool with_a_slices);
// Allocate the FP32 entry's float copies of U and of the eigenvectors.
int workspace_enable_fp32(Workspace *ws);
void workspace_destroy(Workspace *ws);
// Check the device status word (synchronises the stream); returns its cuev_status.
int workspace_check_status(Workspace *ws, const char *stage);

// GEMM on the workspace's stream, with split-K scratch from the workspace.
int ws_gemm(Workspace *ws, int ta, int tb, int m, int n, int k, double alpha, const double *A,
            long long lda, const double *B, long long ldb, double beta, double *C, long long ldc);
int ws_gemm2(Workspace *ws, int ta, int tb, int m, int n, int k, int k2, double alpha,
             const double *A, long long lda, const double *A2, long long lda2, const double *B,
             long long ldb, const double *B2, long long ldb2, double beta, double *C,
             long long ldc, int c_lower);
int ws_symm(Workspace *ws, int m, int n, double alpha, const double *A, long long lda,
            const double *B, long long ldb, double beta, double *C, long long ldc);

// Stage 1: DBBR (dbbr.cu)
int panel_qr(Workspace *ws, double *A, long long lda, double *Y, long long ldy, double *tau,
             double *T, double *W, long long ldw, int rows, int b);
int dbbr_reduce(Workspace *ws, double *A);
int dbbr_pack(Workspace *ws, const double *A, long long lda, double *B);

// Stage 2: bulge chasing (bulge.cu)
int bc_chase(Workspace *ws, double *B, double *d, double *e);

// Stage 3: tridiagonal divide and conquer (tridi.cu)
int tridi_dc(Workspace *ws, const double *d, const double *e, double *eval, double *evec);
// Eigenvalues only of the tridiagonal (bisection; tridi_eigvals.cu).
int tridi_eigvals(Workspace *ws, const double *d, const double *e, double *eval);

// Stage 4: back-transform (backtransform.cu)
int bc_back(Workspace *ws, double *M, long long ldm);
int sbr_back(Workspace *ws, double *M, long long ldm);
// M <- Q_s Q_b M (both stages), overlapped where BC-back's grid ends in a partial wave; records
// bc_end (when not null) once BC-back has finished every column.
int back_transform(Workspace *ws, double *M, long long ldm, cudaEvent_t bc_end);

} // namespace cuev
