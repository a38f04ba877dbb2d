// Ogita-Aishima eigenpair refinement (refine.cu), shared by cuev_dsyev_refine(_ex) and the
// precision-form solve.
#pragma once
#include "common.cuh"
#include "tcgemm.cuh"

namespace cuev {

// Slice counts of the int8 tensor-core products (error ~ 14 2^(-7s) sqrt(n) rowmax colmax):
// the measurements A X, X^T (A X) and X^T X need FP64-level accuracy; the correction X E
// (entries of E are O(error of X)) needs it only relative to E.

constexpr int RF_SLICES_CORR = 5;

// products: CUEV_PRODUCTS_FP64 (DMMA) or CUEV_PRODUCTS_INT8 (tcgen05 int8 emulation).  A_sl, if
// not null, is A already sliced (I8_SRC_SYML, RF_SLICES_HI slices): A itself is then not read
// and may have been overwritten.
int refine_core(const double *A, const I8Operand *A_sl, int n, double *eval, double *X,
                int max_iters, double tol, int products, cudaStream_t st,
                cuev_refine_info *info);

// Device bytes of the scratch refine_core keeps per device for (n, products), without A's slices.
size_t refine_scratch_bytes(int n, int products);

} // namespace cuev
