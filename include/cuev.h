/*
 * cuev.h — C++ drop-in header for libcuev_b200.so.
 *
 * Declares exactly the reference's public entry (include/cuev.h:31-33 and the SolveTimer of
 * include/cuda/handle.h:25-37), so code written against cuEV compiles and links unchanged:
 *
 *     cuev::symm_eig_solve<double>(A, n, eval, evec, stream, &timer);
 *
 * The float and double instantiations are exported with the reference's mangled names.  As in the
 * reference, the call blocks until the result is ready and terminates the process (exit(1)) on
 * error; use the C entries in cuev_b200.h to get a status code instead.
 */
#pragma once
#include <cuda_runtime.h>

#include "cuev_b200.h"

namespace cuev {

/// Per-stage timings for one symm_eig_solve (same layout as cuev_timer).
struct SolveTimer {
    float dbbr_ms = 0;       ///< full -> band (DBBR)
    float bc_ms = 0;         ///< band -> tridiagonal (bulge chasing)
    float dc_ms = 0;         ///< tridiagonal D&C
    float bt_ms = 0;         ///< back-transform (evec = Q_s Q_b Q_d)
    float total_ms = 0;      ///< whole-solve wall clock
    float bt_copyin_ms = 0;  ///< 0: the back-transform works in place on evec
    float bt_qb_ms = 0;      ///< BC-Back  M <- Q_b M
    float bt_qs_ms = 0;      ///< SBR-Back M <- Q_s M after BC-back ends (part of it overlaps BC-back)
    float bt_copyout_ms = 0; ///< 0: no copy-out
};

/**
 * Compute all eigenvalues and eigenvectors of a real symmetric matrix.
 *
 * @tparam T      float or double
 * @param[in,out] A      n x n symmetric matrix (column-major, lower triangle read), overwritten
 * @param[in]     n      matrix dimension
 * @param[out]    eval   eigenvalues in ascending order, length n
 * @param[out]    evec   eigenvectors as columns, n x n (column-major); may be nullptr here
 *                       (eigenvalues only, an extension over the reference)
 * @param[in]     stream CUDA stream
 * @param[out]    timer  optional per-stage timing breakdown
 */
template <typename T>
void symm_eig_solve(T *A, int n, T *eval, T *evec, cudaStream_t stream,
                    SolveTimer *timer = nullptr);

} // namespace cuev
