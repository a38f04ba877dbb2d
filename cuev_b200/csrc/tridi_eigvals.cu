// Eigenvalues only of the symmetric tridiagonal T (diagonal d, off-diagonal e): the stage that
// replaces divide and conquer when the caller asks for no eigenvectors (evec == NULL).  The
// reference always forms eigenvectors; this path has no counterpart there.
//
// Method: bisection on Sturm counts, one thread per eigenvalue (W. Barth, R. S. Martin,
// J. H. Wilkinson, "Calculation of the eigenvalues of a symmetric tridiagonal matrix by the
// method of bisection", Numer. Math. 9 (1967)).  count(x) = number of eigenvalues below x =
// number of negative pivots q_i of T - x I = L D L^T:
//     q_0 = d_0 - x,   q_i = d_i - x - e_{i-1}^2 / q_{i-1},
// with |q_i| < pivmin replaced by -pivmin (the guard used by LAPACK's bisection, which keeps the
// count monotone in x and the recurrence finite).  Thread i keeps lo, hi with
// count(lo) <= i < count(hi) starting from the Gershgorin interval and halves it until its width
// is below 2 eps (max(|lo|, |hi|) + ||T||) (about 55 steps, at most 128).  The Sturm
// count is backward stable, so every eigenvalue is accurate to O(eps ||T||) absolutely, which is
// the accuracy of the eigenvalues of the full solve.
//
// Work: about 60 n^2 divide-and-FMA steps, spread over n independent threads; d and e^2 are read
// by every thread in the same order, so a warp's loads are broadcasts served by L1/L2.
#include "solver.cuh"

#include <algorithm>

namespace cuev {
namespace {

constexpr int EV_THREADS = 128;

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
        const double pivmin = tiny * fmax(1.0, red[0]);
        const double eps = 2.220446049250313e-16;
        const double w = fmax(fabs(glo), fabs(ghi));
        scal[0] = sc;
        scal[1] = pivmin;
        scal[2] = glo - 4.0 * eps * w - 4.0 * pivmin; // widened so the ends are strict bounds
        scal[3] = ghi + 4.0 * eps * w + 4.0 * pivmin;
    }
}

__device__ __forceinline__ int sturm_count(const double *__restrict__ ds,
                                           const double *__restrict__ e2, int n, double x,
                                           double pivmin) {
    double q = ds[0] - x;
    if (fabs(q) < pivmin) q = -pivmin;
    int cnt = q < 0.0;
    for (int i = 1; i < n; ++i) {
        q = (ds[i] - x) - e2[i - 1] / q;
        if (fabs(q) < pivmin) q = -pivmin;
        cnt += q < 0.0;
    }
    return cnt;
}

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
        const double mid = 0.5 * (lo + hi);
        if (mid <= lo || mid >= hi) break; // no representable point left between them
        if (sturm_count(ds, e2, n, mid, pivmin) > i)
            hi = mid;
        else
            lo = mid;
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
    ev_bisect_kernel<<<div_up(n, EV_THREADS), EV_THREADS, 0, ws->stream>>>(ds, e2, n, scal, eval);
    note_launch();
    CUEV_TRY(cudaGetLastError());
    return CUEV_OK;
}

} // namespace cuev
