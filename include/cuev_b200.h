/*
 * cuev_b200.h — C ABI of the B200-native cuEV symmetric eigensolver (libcuev_b200.so).
 *
 * Drop-in target: cuEV's `cuev::symm_eig_solve<T>(T *A, int n, T *eval, T *evec,
 * cudaStream_t stream, SolveTimer *timer)` (reference include/cuev.h:31-33).  The C++ template
 * with that exact signature and mangled name is declared in include/cuev.h and forwards here.
 *
 * Conventions (same as the reference, README.md:10-12, CONVENTIONS.md:126):
 *   - all matrices column-major, leading dimension n unless an `ld` argument says otherwise;
 *   - only the LOWER triangle of A is read (reference src/cuda/dbbr.cu:175,222) and A is
 *     overwritten;
 *   - eval ascending, evec column j = eigenvector of eval[j] (sign unspecified);
 *   - every pointer argument is a device pointer unless the name ends in `_host`;
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).  Solves are
 *     host-blocking like the reference (src/cuda/solver.cu:59); stage entries are asynchronous.
 *
 * Errors: every entry returns a cuev_status.  The reference prints and calls exit(1)
 * (include/common.h:9-34); here the C++ shim in include/cuev.h keeps that behaviour while the C
 * entries return the code.  cuev_last_error() gives a human-readable message.
 */
#ifndef CUEV_B200_H
#define CUEV_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum cuev_status {
    CUEV_OK = 0,
    CUEV_ERR_INVALID = -1,     /* bad argument (n < 0, null pointer, unsupported b/k, ...) */
    CUEV_ERR_ALLOC = -2,       /* device workspace allocation failed */
    CUEV_ERR_CUDA = -3,        /* a CUDA runtime call failed */
    CUEV_ERR_TIMEOUT = -4,     /* a bounded device wait gave up (wavefront / grid barrier) */
    CUEV_ERR_NONFINITE = -5,   /* NaN or Inf met in the input */
    CUEV_ERR_CONVERGENCE = -6, /* an iteration (leaf QL, secular solver, refinement) failed */
    CUEV_ERR_UNSUPPORTED = -7  /* form not built for this dtype / size */
} cuev_status;

/* Per-stage timings; same fields, order and meaning as cuev::SolveTimer
 * (reference include/cuda/handle.h:25-37). */
typedef struct cuev_timer {
    float dbbr_ms;       /* full -> band (DBBR, incl. pack) */
    float bc_ms;         /* band -> tridiagonal (bulge chasing) */
    float dc_ms;         /* tridiagonal divide and conquer (on the GPU here) */
    float bt_ms;         /* back-transform evec = Q_s * Q_b * Q_d */
    float total_ms;      /* whole-solve wall clock */
    float bt_copyin_ms;  /* kept for layout compatibility (no copy-in is needed here: 0) */
    float bt_qb_ms;      /* BC-Back  M <- Q_b * M */
    float bt_qs_ms;      /* SBR-Back M <- Q_s * M, the part after BC-back ends (SBR-back of the
                            columns BC-back finished early overlaps its last wave) */
    float bt_copyout_ms; /* kept for layout compatibility (0) */
} cuev_timer;

/* Blocking parameters.  0 selects the default for the size.  b in {32, 64}; k a multiple of b. */
typedef struct cuev_config {
    int nbw; /* band width b (reference hard-codes 32, src/cuda/solver.cu:33) */
    int nk;  /* DBBR outer block k (reference hard-codes 512) */
} cuev_config;

/* ---------------------------------------------------------------------------------------------
 * Full solves
 * ------------------------------------------------------------------------------------------ */

/* Plain FP64 solve.  Replaces cuev::symm_eig_solve<double> (reference src/cuda/solver.cu:25-73,
 * instantiated at :79).  timer may be NULL.  evec may be NULL (no reference counterpart: the
 * reference always forms eigenvectors): then only the eigenvalues are computed, by bisection on
 * the tridiagonal after the band reduction and bulge chase, with no D&C and no back-transform. */
int cuev_dsyevd(double *A, int n, double *eval, double *evec, void *stream, cuev_timer *timer);

/* Same with explicit blocking (reference: handle_alloc(n, nbw, nk, stream),
 * src/cuda/handle.cu:16). cfg may be NULL. */
int cuev_dsyevd_cfg(double *A, int n, double *eval, double *evec, void *stream, cuev_timer *timer,
                    const cuev_config *cfg);

/* Host-buffer form of cuev_dsyevd (no reference counterpart: the reference takes device
 * pointers): A_host (n x n column-major, lower triangle read, not modified), eval_host (n) and
 * evec_host (n x n, or NULL for eigenvalues only) in host memory (pinned for full copy speed).
 * A is copied in, solved on `stream`, and the eigenvector columns are copied out as they become
 * final (the columns of BC-back's whole waves while the last columns' back-transform runs).
 * Device buffers ((2 n^2 + n) doubles) are kept per device between calls and released by
 * cuev_release_workspace.  Blocks until done. */
int cuev_dsyevd_host(const double *A_host, int n, double *eval_host, double *evec_host,
                     void *stream, cuev_timer *timer);

/* FP32 interface.  Replaces cuev::symm_eig_solve<float> (reference src/cuda/solver.cu:78).
 * The float input is widened and solved by the FP64 band reduction, bulge chase and D&C; BC-back
 * runs in FP32 (b = 32; on float copies of the reflectors and eigenvectors, n^2 floats each, kept
 * with the cached workspace) and the SBR-back products (the back-transform's GEMMs) on the int8
 * tensor cores at FP32-level accuracy (5 slices); the results are rounded back to FP32.
 * Accuracy is FP32-level (residual and orthogonality per sqrt(n) about 2e-6 at n = 3072, 4e-6 at
 * n = 16384). */
int cuev_ssyevd(float *A, int n, float *eval, float *evec, void *stream, cuev_timer *timer);

/* Batched eigensolver for many small matrices (no reference counterpart: the reference solves one
 * matrix per call).  A holds `batch` symmetric n x n matrices, n <= 512, each column-major and
 * stored one after another (stride n*n); only their lower triangles are read and A is not
 * modified.  eval receives batch x n ascending eigenvalues, evec batch x (n x n) eigenvector
 * columns.  One CTA per matrix: two-sided Jacobi in shared memory for n <= 64; Householder
 * tridiagonalisation, implicit QL and back-transform in a per-CTA device workspace (kept per
 * device, 3 n^2 doubles per resident CTA) for 64 < n <= 512.  n > 512 returns
 * CUEV_ERR_UNSUPPORTED.  Blocks until done; calls are serialised. */
int cuev_dsyevd_batched(const double *A, int n, int batch, double *eval, double *evec,
                        void *stream);

/* Differentiation form (no reference counterpart): cotangent of A for the eigensolve,
 *   Abar = V (diag(lambar) + sym(F o (V^T Vbar))) V^T,  F_ij = 1/(lam_j - lam_i),
 * sym(X) = (X + X^T)/2, F_ij = 0 on the diagonal and where |lam_j - lam_i| < gap_tol (masked
 * near-degenerate pairs).  V, Vbar, Abar are n x n column-major; lam, lambar length n; Vbar or
 * lambar may be NULL (zero cotangent).  Only lam and V from the forward solve are needed.
 * Enqueued on `stream`, asynchronous. */
int cuev_dsyev_adjoint(const double *V, const double *lam, const double *Vbar,
                       const double *lambar, int n, double gap_tol, double *Abar, void *stream);
/* (The adjoint keeps V G in one n x n scratch buffer per device: adjoint calls that can overlap on
 * the GPU, on different streams, must not share a device.) */
/* FP32 interface of the same (computed in FP64 internally). */
int cuev_ssyev_adjoint(const float *V, const float *lam, const float *Vbar, const float *lambar,
                       int n, float gap_tol, float *Abar, void *stream);

/* Precision form, refinement half (no reference counterpart): Ogita-Aishima iterative
 * refinement of an approximate eigendecomposition of the symmetric A (n x n, lower triangle
 * read, not modified).  evec (n x n, columns) is improved in place and eval receives the refined
 * eigenvalues.  Each step costs 7 n^3 FP64 flop; the step measures ||I - X^T X||_F and
 * ||X^T A X - diag(lam)||_F first and stops early once both are <= tol (relative to max|lam| for
 * the second; tol <= 0 runs all max_iters steps).  info may be NULL.  Blocks until done. */
typedef struct cuev_refine_info {
    int iterations;     /* refinement steps applied */
    double offdiag_fro; /* ||X^T A X - diag(lam)||_F of the last X measured */
    double orth_fro;    /* ||I - X^T X||_F of the last X measured */
    double anorm;       /* max |lam_i|, the ||A||_2 estimate */
} cuev_refine_info;
int cuev_dsyev_refine(const double *A, int n, double *eval, double *evec, int max_iters,
                      double tol, void *stream, cuev_refine_info *info);

/* Arithmetic of the refinement's n x n products. */
typedef enum cuev_products {
    CUEV_PRODUCTS_FP64 = 0, /* FP64 DMMA (7 n^3 flop per step) */
    CUEV_PRODUCTS_INT8 = 1  /* int8 tensor cores (tcgen05.mma.kind::i8) with 7-bit operand slices:
                               A X, X^T A X and X^T X from 7 slices per operand (FP64-level, error
                               ~ 2^-49 relative to the row and column maxima), the correction X E
                               from 5; X^T X and X^T A X are formed as lower triangles */
} cuev_products;
/* cuev_dsyev_refine with a choice of product arithmetic (no reference counterpart). */
int cuev_dsyev_refine_ex(const double *A, int n, double *eval, double *evec, int max_iters,
                         double tol, int products, void *stream, cuev_refine_info *info);

/* Precision form (no reference counterpart): a mixed-precision solve refined to FP64.  Same
 * arguments and result as cuev_dsyevd (A overwritten, eval ascending, evec columns), computed
 * in two parts:
 *   1. a first solve whose back-transform products Y^T M, T X and Y X (SBR-back, each of at
 *      least 2^30 multiply-adds) run on the int8 tensor cores at FP32-level accuracy (5 slices;
 *      the reflectors' unit entries set their rows' scale, so 5 slices leave ~2^-28 for the rest);
 *      the band reduction, bulge chase, D&C and BC-back stay FP64;
 *   2. Ogita-Aishima refinement of those eigenpairs against the original A with FP64-level
 *      int8 tensor-core products (CUEV_PRODUCTS_INT8), at most max_refine_iters steps, stopping
 *      once ||I - X^T X||_F <= tol and ||X^T A X - diag||_F <= tol max|lam| (tol <= 0: all steps).
 * The original A is kept as int8 slices before the first part overwrites it.  info and timer may
 * be NULL; timer holds the first part's stages.  Blocks until done. */
typedef struct cuev_mixed_info {
    int refine_iterations; /* refinement steps applied */
    double offdiag_fro;    /* ||X^T A X - diag(lam)||_F at the last measurement */
    double orth_fro;       /* ||I - X^T X||_F at the last measurement */
    double anorm;          /* max |lam_i| */
    float first_ms;        /* first solve, incl. slicing A */
    float refine_ms;       /* refinement */
} cuev_mixed_info;
int cuev_dsyevd_mixed(double *A, int n, double *eval, double *evec, void *stream,
                      cuev_timer *timer, int max_refine_iters, double tol,
                      cuev_mixed_info *info);

/* Release the cached device workspace (the solves keep one pool per (n, b, k) between calls, the
 * batched eigensolver one buffer per device for 64 < n <= 512, the FP32 and host-buffer entries
 * one buffer each per device, (2 n^2 + n) doubles). */
int cuev_release_workspace(void);

/* Message for the last failing call on this host thread ("" if none). */
const char *cuev_last_error(void);

/* Number of CUDA kernels this library has launched since it was loaded (profiling aid). */
long long cuev_kernel_launches(void);

/* Flops of the divide-and-conquer merge GEMMs of the last full solve (with eigenvectors) on this
 * host thread, counted on the device after deflation: sum over merges of
 * 2 (n1 k (ct1 + ct2) + n2 k (ct2 + ct3)) (profiling aid; the upper bound without deflation is
 * 4/3 n^3). */
double cuev_last_dc_flops(void);

/* Failure-path testing (no reference counterpart; the reference has no bounded waits).  Every
 * device-side wait of the library (bulge-chase hand-off, grid barriers, BC-back's warp pipeline,
 * the tensor-core GEMM's mbarriers) gives up after 2 s and the call returns CUEV_ERR_TIMEOUT.
 * This sets that limit for the calls that follow (0 restores 2 s), so a test can make the waits
 * run out on purpose and check that the error is reported and the next call succeeds.  Not
 * meant for production use: a short limit turns ordinary waiting into failures. */
int cuev_debug_set_wait_limit_ns(unsigned long long ns);

/* ---------------------------------------------------------------------------------------------
 * Stage-level API used by the stage tests.  Mirrors the reference's SolverHandle<T> and
 * cuev::kernels::* launchers (include/cuda/handle.h:61-100, include/cuda/kernels.cuh:47-155).
 * A handle owns the workspace for one (n, b, k); every stage call is enqueued on the handle's
 * stream and returns without synchronising.
 * ------------------------------------------------------------------------------------------ */
typedef struct cuev_handle_s *cuev_handle;

/* Replaces cuev::handle_alloc<double> (reference src/cuda/handle.cu:16-94). */
int cuev_handle_create(int n, int nbw, int nk, void *stream, cuev_handle *out);
/* Replaces cuev::handle_free<double> (reference src/cuda/handle.cu:96-101). */
int cuev_handle_destroy(cuev_handle h);

/* Device buffers owned by the handle (what the reference tests read from ws.B, ws.d, ...). */
typedef enum cuev_buffer {
    CUEV_BUF_B = 0, /* packed band, 2b x n, ld 2b (reference ws.B) */
    CUEV_BUF_D = 1, /* tridiagonal diagonal, n */
    CUEV_BUF_E = 2, /* tridiagonal sub-diagonal, n-1 */
    CUEV_BUF_Y = 3, /* DBBR reflectors, n x n, ld n (reference ws.Y) */
    CUEV_BUF_U = 4, /* bulge-chasing reflectors, column s = sweep s, ld n (reference ws.U) */
    CUEV_BUF_TAU = 5 /* DBBR Householder scalars, n (one per reflector column) */
} cuev_buffer;
int cuev_handle_buffer(cuev_handle h, int which, void **ptr, long long *ld);

/* Panel QR of a rows x b panel (b <= 64): R in the upper triangle of A, unit lower-trapezoidal
 * reflectors in Y (ld ldy), scalars in tau (b), block factor T (b x b, ld b, upper) with
 * H_0...H_{b-1} = I - Y T Y^T.  Replaces kernels::dbbr_panel_qr (reference src/cuda/dbbr.cu:124-143:
 * cuSOLVER geqrf + extract + larft). */
int cuev_dbbr_panel_qr(cuev_handle h, double *A, int lda, double *Y, int ldy, double *tau,
                       double *T, int rows, int b);

/* Full-to-band reduction of the lower triangle of A (ld n) in place; the band is also packed
 * into the handle's B.  Replaces kernels::dbbr_reduce (reference src/cuda/dbbr.cu:145-229). */
int cuev_dbbr_reduce(cuev_handle h, double *A);

/* Pack the lower band of A (ld n) into B (2b x n).  Replaces kernels::dbbr_pack
 * (reference src/cuda/dbbr.cu:116-122). */
int cuev_dbbr_pack(cuev_handle h, const double *A, double *B);

/* Band -> tridiagonal (d, e); reflectors kept in the handle's U.  Replaces kernels::bc_chase
 * (reference src/cuda/bulge.cu:231-247). */
int cuev_bc_chase(cuev_handle h, double *B, double *d, double *e);

/* Tridiagonal divide and conquer on the GPU: eval ascending, evec = eigenvectors of the
 * tridiagonal (n x n, ld n).  d and e are not modified.  Replaces kernels::tridi_dc (reference
 * src/cuda/tridi.cu:425-452, a host LAPACK D&C). */
int cuev_tridi_dc(cuev_handle h, const double *d, const double *e, double *eval, double *evec);

/* Eigenvalues only of the tridiagonal (d, e), ascending, by bisection on Sturm counts (one thread
 * per eigenvalue).  No reference counterpart: the stage the eigenvalues-only solve (evec == NULL)
 * runs in place of cuev_tridi_dc. */
int cuev_tridi_eigvals(cuev_handle h, const double *d, const double *e, double *eval);

/* M <- Q_b M (n x n, ld ldm).  Replaces kernels::bc_back (reference src/cuda/backtransform.cu:183-207). */
int cuev_bc_back(cuev_handle h, double *M, int ldm);

/* M <- Q_s M (n x n, ld ldm).  Replaces kernels::sbr_back (reference src/cuda/backtransform.cu:210-230). */
int cuev_sbr_back(cuev_handle h, double *M, int ldm);

/* evec <- Q_s Q_b evec.  Replaces kernels::back_transform (reference src/cuda/backtransform.cu:232-275).
 * Blocks until done and returns CUEV_ERR_TIMEOUT if one of BC-back's bounded waits gave up. */
int cuev_back_transform(cuev_handle h, double *evec, cuev_timer *timer);

/* FP64 tensor-core GEMM used by every stage: C = alpha op(A) op(B) + beta C (column-major).
 * ta/tb: 0 = N, 1 = T.  Replaces the reference's cuev::cublas::gemm wrapper
 * (src/cuda/cublas.cu:15-26). */
int cuev_dgemm(void *stream, int ta, int tb, int m, int n, int k, double alpha, const double *A,
               int lda, const double *B, int ldb, double beta, double *C, int ldc);
/* (cuev_dgemm, cuev_dsymm_lower and cuev_dsyr2k_lower keep split-K partial sums in one buffer per
 * device: calls that can overlap on the GPU, on different streams, must not share a device.) */

/* Same product as cuev_dgemm, for callers that cannot allocate device memory.  No counterpart in
 * the reference.  cuev_dgemm takes its split-K partial-sum buffer from cudaMalloc; a caller whose
 * device memory is owned by its framework's caching allocator, or that must not block on a
 * device allocation (latency-critical serving loops), can use this entry instead: it allocates
 * nothing and keeps the partial sums in a fixed 16 MiB array inside the library (held on every
 * GPU that loads the library until the process exits).
 *   - Limit: m * n <= 1048576; larger problems return CUEV_ERR_INVALID (use cuev_dgemm).
 *   - The first call on a device looks up the array's device address (cudaGetSymbolAddress);
 *     make that first call before any stream capture on that device.
 *   - All calls share the array: calls that overlap on the GPU (other streams, other host
 *     threads) race and give wrong results; serialise them.  Every partial sum is written by the
 *     call before it is read, so no clearing is needed between calls. */
int cuev_dgemm_noalloc(void *stream, int ta, int tb, int m, int n, int k, double alpha,
                       const double *A, int lda, const double *B, int ldb, double beta, double *C,
                       int ldc);

/* Same product as cuev_dgemm emulated on the int8 tensor cores (no reference counterpart):
 * every row of op(A) and column of op(B) is scaled by a power of two and cut into `slices`
 * (1..8) signed 7-bit integer slices; the slice products run as tcgen05.mma.kind::i8 with int32
 * accumulation in TMEM and are summed in FP64.  Error per entry ~ 14 2^(-7 slices) sqrt(k)
 * rowmax_i(op(A)) colmax_j(op(B)): 7 slices give FP64-level, 4 FP32-level products.  Slices
 * live in the same per-device scratch as cuev_dgemm's split-K partials.  Blocks until done. */
int cuev_dgemm_i8(void *stream, int ta, int tb, int m, int n, int k, int slices, double alpha,
                  const double *A, int lda, const double *B, int ldb, double beta, double *C,
                  int ldc);

/* C = alpha A B + beta C with A symmetric (m x m, lower triangle read).  Replaces
 * cuev::cublas::symm(LEFT, LOWER) (reference src/cuda/cublas.cu:28-37). */
int cuev_dsymm_lower(void *stream, int m, int n, double alpha, const double *A, int lda,
                     const double *B, int ldb, double beta, double *C, int ldc);

/* Lower triangle of C = alpha (A B^T + B A^T) + beta C, C n x n, A and B n x k.  Replaces
 * cuev::cublas::syr2k(LOWER, N) (reference src/cuda/cublas.cu:48-56). */
int cuev_dsyr2k_lower(void *stream, int n, int k, double alpha, const double *A, int lda,
                      const double *B, int ldb, double beta, double *C, int ldc);

#ifdef __cplusplus
}
#endif

#endif /* CUEV_B200_H */
