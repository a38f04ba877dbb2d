// FP64 products on the int8 tensor cores (tcgen05.mma.kind::i8), by error-free slicing.
//
// Method: Ozaki scheme with integer slices (K. Ozaki, T. Ogita, S. Oishi, S. M. Rump, "Error-free
// transformations of matrix multiplication by using fast routines of matrix multiplication and its
// applications", Numer. Algorithms 59 (2012); its int8 tensor-core form: H. Ootomo, K. Ozaki,
// R. Yokota, "DGEMM on integer matrix multiplication unit", IJHPCA 38 (2024)).
//
// Every row r of op(A) (and column of op(B)) is scaled by a power of two 2^-e_r with
// max_k |op(A)(r, k)| < 2^e_r and cut into s signed 7-bit integer slices:
//     op(A)(r, k) = 2^e_r * sum_{p=1..s} 2^(-7p) a_p(r, k) + rest,  |a_p| <= 127,  |rest| < 2^(e_r - 7s).
// The product is then
//     op(A) op(B) ~= 2^(e_r + f_c) * sum_{d=2..s+1} 2^(-7d) L_d,   L_d = sum_{p+q=d} a_p b_q,
// where each L_d is an exact int32 sum of int8 products (tensor cores, int32 accumulation in
// TMEM; K is cut into groups small enough that no int32 sum can overflow) and the levels are
// added in FP64 from the most significant one down.  The dropped terms (p + q > s + 1) and the
// slice remainders bound the error by about (s + 2) 2^(-7s) 2^(e_r + f_c) K per entry: s = 7
// gives FP64-level products (2^-49 relative to the row and column maxima), s = 4 FP32-level ones.
#pragma once
#include "common.cuh"

namespace cuev {

// Slices of the precision form's stage GEMMs and of its refinement measurements.  The stage
// products are those of the back-transform, whose Householder operand rows hold a unit entry
// next to entries of order 1/sqrt(n): the row scaling is set by the unit entry, so 5 slices
// (35 bits of the row maximum) leave about FP32-level accuracy (2^-28) for the small entries,
// which is what one refinement step needs to reach a residual of 1e-13.
constexpr int MIXED_SLICES = 5;
constexpr int RF_SLICES_HI = 7;

// int8 slices of one GEMM operand op(X) (rows x k), K-major: byte (r, kk) of slice p (0-based) is
// data[p * slice_stride + r * k_ld + kk]; k_ld is k rounded up to 128 and the padding is zero.
struct I8Operand {
    int8_t *data = nullptr;
    int *exps = nullptr;                 // e_r per row
    unsigned long long *rmax = nullptr;  // row maxima (FP64 bit patterns), slicing scratch
    int rows = 0, k = 0, s = 0;
    long long k_ld = 0;
    size_t slice_stride = 0;
};

// How op(X)(r, kk) is read from the column-major source X (ld ldx):
enum I8SliceSrc {
    I8_SRC_KMAJ = 0, // X[kk + r ldx]  (op(A) = A^T, or op(B) = B)
    I8_SRC_RMAJ = 1, // X[r + kk ldx]  (op(A) = A,   or op(B) = B^T)
    I8_SRC_SYML = 2  // symmetric, lower triangle stored: r >= kk ? X[r + kk ldx] : X[kk + r ldx]
};

// Device bytes for one operand (slices, exponents, row-max scratch).
size_t i8_operand_bytes(int rows, int k, int s);
// Lay an operand out in `buf` (i8_operand_bytes(rows, k, s) bytes, 256-byte aligned).
void i8_operand_init(void *buf, int rows, int k, int s, I8Operand &op);
// Slice op(X) into `op` (shape and slice count fixed by i8_operand_init).
int i8_slice(const double *X, long long ldx, int src, I8Operand &op, cudaStream_t st);

// C (m x n, column-major, ld ldc) = alpha * op(A) op(B) + beta * C from sliced operands
// (A.rows = m, B.rows = n, A.k == B.k), keeping the levels d <= levels + 1.  c_lower: only
// C(i, j) with i >= j is written.  Failures of the kernel's bounded waits are recorded in
// status (CUEV_ERR_TIMEOUT).  beta == 0 does not read C.
int i8_gemm(const I8Operand &A, const I8Operand &B, int levels, double alpha, double beta,
            double *C, long long ldc, int c_lower, int *status, cudaStream_t st);

// One call: slice op(A), op(B) (ta/tb: 0 = N, 1 = T; symm_a: A symmetric, lower triangle) into
// `scratch` (i8_gemm_scratch_bytes bytes) and multiply.
size_t i8_gemm_scratch_bytes(int m, int n, int k, int s);
int i8_dgemm(int ta, int tb, int symm_a, int m, int n, int k, int s, double alpha,
             const double *A, long long lda, const double *B, long long ldb, double beta,
             double *C, long long ldc, int c_lower, void *scratch, int *status, cudaStream_t st);

} // namespace cuev
