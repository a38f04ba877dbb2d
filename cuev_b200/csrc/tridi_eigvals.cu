// Eigenvalues only of the symmetric tridiagonal T (diagonal d, off-diagonal e): the stage that
// replaces divide and conquer when the caller asks for no eigenvectors (evec == NULL).  The
// reference always forms eigenvectors; this path has no counterpart there.
//
// Method: bisection on Sturm counts, one thread per eigenvalue (W. Barth, R. S. Martin,
// J. H. Wilkinson, "Calculation of the eigenvalues of a symmetric tridiagonal matrix by the
// method of bisection", Numer. Math. 9 (1967)), as multisection.  count(x) = number of
// eigenvalues below x = number of negative pivots q_i of T - x I = L D L^T:
//     q_0 = d_0 - x,   q_i = d_i - x - e_{i-1}^2 / q_{i-1},
// with |q_i| < pivmin replaced by -pivmin (the guard of LAPACK's bisection, which keeps the
// recurrence finite; the floor here is raised to 2^-100 on the scaled problem, see sturm_quot).
// Thread i keeps lo, hi with count(lo) <= i < count(hi) starting from the Gershgorin interval and
// cuts it into EV_K + 1 pieces per pass until its width is below 2 eps (max(|lo|, |hi|) + ||T||)
// (about 35 passes at EV_K = 2, at most 128).  The Sturm count is backward stable, so every
// eigenvalue is accurate to O(eps ||T||) absolutely, which is the accuracy of the eigenvalues of
// the full solve.
//
// Work: about 70 n^2 quotient-and-FMA steps, spread over n threads; d and e^2 are read by every
// thread in the same order, so a warp's loads are broadcasts served by L1.  With one warp per SM
// sub-partition (n threads in all) the FP64 and XU pipes of the occupied sub-partitions set the
// rate.
#include "solver.cuh"

#include <algorithm>

namespace cuev {
namespace {

constexpr int EV_THREADS = 128;
constexpr int EV_K = 2; // multisection points per thread and pass (measured best of 1, 2, 4, 8, 12)

// scaled copies: ds = d / s, e2 = (e / s)^2; scal[0] = s, scal[1] = pivmin, scal[2..3] = Gershgorin
__global__ void ev_prepare_kernel(const double *__restrict__ d, const double *__restrict__ e, int n,
                                  double *__restrict__ ds, double *__restrict__ e2,
                                  double *__restrict__ scal) {
    __shared__ double red[EV_THREADS];
    double mx = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        mx = fmax(mx, fabs(d[i]));
        if (i < n - 1) mx = fmax(mx, fabs(e[i]));
    }
    red[threadIdx.x] = mx;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
        __syncthreads();
    }
    const double sc = red[0] > 0.0 ? red[0] : 1.0;
    __syncthreads();
    double lo = 1e300, hi = -1e300, me2 = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double di = d[i] / sc;
        const double em = i > 0 ? fabs(e[i - 1]) / sc : 0.0;
        const double ep = i < n - 1 ? fabs(e[i]) / sc : 0.0;
        ds[i] = di;
        if (i < n - 1) {
            e2[i] = ep * ep;
            me2 = fmax(me2, ep * ep);
        }
        lo = fmin(lo, di - em - ep);
        hi = fmax(hi, di + em + ep);
    }
    // block reductions of lo (min), hi (max), me2 (max)
    red[threadIdx.x] = lo;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] = fmin(red[threadIdx.x], red[threadIdx.x + s]);
        __syncthreads();
    }
    const double glo = red[0];
    __syncthreads();
    red[threadIdx.x] = hi;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
        __syncthreads();
    }
    const double ghi = red[0];
    __syncthreads();
    red[threadIdx.x] = me2;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double tiny = 2.2250738585072014e-308; // smallest normal double
        // LAPACK's pivot floor, raised to 2^-100 (far below the 2 eps ||T|| stopping width on
        // the scaled problem) so that every pivot stays where sturm_quot is valid
        const double pivmin = fmax(tiny * fmax(1.0, red[0]), 0x1p-100);
        const double eps = 2.220446049250313e-16;
        const double w = fmax(fabs(glo), fabs(ghi));
        scal[0] = sc;
        scal[1] = pivmin;
        scal[2] = glo - 4.0 * eps * w - 4.0 * pivmin; // widened so the ends are strict bounds
        scal[3] = ghi + 4.0 * eps * w + 4.0 * pivmin;
    }
}

// f / q for the Sturm recurrence, without a branch: a float reciprocal seed r ~ 1/q (~22 correct
// bits), two Newton-Raphson steps r <- r + r (1 - q r) (each doubles the correct bits: ~44, then
// the full 53), the product y = f r and one residual correction y <- y + r (f - q y)
// (P. Markstein, "Computation of elementary functions on the IBM RISC System/6000 processor",
// IBM J. Res. Develop. 34 (1990) 111-119), which leaves y within one rounding of f / q.  Valid
// for 2^-100 <= |q| <= 2^101 (q, its float rounding and 1/q are normal floats): the pivot floor
// and the scaling (|d|, |e| <= 1, |x| <= 3) keep every pivot there.  A division with a slow path
// would end a basic block per quotient; straight-line code lets the scheduler interleave the
// independent recurrences of one thread.
__device__ __forceinline__ double sturm_quot(double f, double q) {
    float rf;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rf) : "f"((float)q));
    double r = (double)rf;
    r = fma(r, fma(-q, r, 1.0), r);
    r = fma(r, fma(-q, r, 1.0), r);
    const double y = f * r;
    return fma(r, fma(-q, y, f), y);
}

// Multisection: thread i splits its interval [lo, hi) at K interior points and evaluates the K
// Sturm counts in one pass over T (K independent recurrences per loaded d_r, e_r^2), then keeps
// the piece between the last point with count <= i and the first with count > i.  The invariant
// count(lo) <= i < count(hi) holds whatever the counts are, so the result never depends on the
// counts being monotone.
template <int K>
__global__ void __launch_bounds__(EV_THREADS)
    ev_bisect_kernel(const double *__restrict__ ds, const double *__restrict__ e2, int n,
                     const double *__restrict__ scal, double *__restrict__ eval) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double sc = scal[0], pivmin = scal[1];
    double lo = scal[2], hi = scal[3];
    const double eps = 2.220446049250313e-16;
    const double atol = 2.0 * eps * fmax(fabs(scal[2]), fabs(scal[3])) + 4.0 * pivmin;
    for (int it = 0; it < 128; ++it) {
        const double width = hi - lo;
        if (width <= 2.0 * eps * fmax(fabs(lo), fabs(hi)) + atol) break;
        const double h = width / (K + 1);
        double x[K], q[K];
        int cnt[K];
#pragma unroll
        for (int j = 0; j < K; ++j) {
            x[j] = fmin(lo + (j + 1) * h, hi);
            q[j] = ds[0] - x[j];
            if (fabs(q[j]) < pivmin) q[j] = -pivmin;
            cnt[j] = q[j] < 0.0;
        }
        for (int r = 1; r < n; ++r) {
            const double d = ds[r], f = e2[r - 1];
#pragma unroll
            for (int j = 0; j < K; ++j) {
                q[j] = (d - x[j]) - sturm_quot(f, q[j]);
                if (fabs(q[j]) < pivmin) q[j] = -pivmin;
                cnt[j] += q[j] < 0.0;
            }
        }
        int jf = K; // first point with count > i
#pragma unroll
        for (int j = K - 1; j >= 0; --j)
            if (cnt[j] > i) jf = j;
        double nlo = lo, nhi = hi;
#pragma unroll
        for (int j = 0; j < K; ++j) {
            if (j == jf) nhi = x[j];
            if (j == jf - 1) nlo = x[j];
        }
        if (nlo == lo && nhi == hi) break; // no representable point left between them
        lo = nlo, hi = nhi;
    }
    eval[i] = 0.5 * (lo + hi) * sc;
}

} // namespace

int tridi_eigvals(Workspace *ws, const double *d, const double *e, double *eval) {
    const int n = ws->n;
    if (n <= 0) return CUEV_OK;
    // scratch in the D&C vectors (unused on this path): ds[n], e2[n], scal[4]
    double *ds = ws->dc_vec, *e2 = ds + n, *scal = e2 + n;
    ev_prepare_kernel<<<1, EV_THREADS, 0, ws->stream>>>(d, e, n, ds, e2, scal); note_launch();
    CUEV_TRY(cudaGetLastError());
    ev_bisect_kernel<EV_K><<<div_up(n, EV_THREADS), EV_THREADS, 0, ws->stream>>>(ds, e2, n, scal,
                                                                             eval);
    note_launch();
    CUEV_TRY(cudaGetLastError());
    return CUEV_OK;
}

} // namespace cuev
