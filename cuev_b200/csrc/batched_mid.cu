// Batched eigensolver for stacks of medium symmetric matrices (64 < n <= 512), one CTA of 512
// threads per matrix (persistent over the stack).  The reference has no batched entry; the small
// sizes (n <= 64) run the shared-memory Jacobi of batched_small.cu.
//
// Per matrix, in a per-CTA global workspace (three n x n FP64 buffers, L2/HBM resident); thread r
// owns row r of the matrix (column-major storage, so a column access is coalesced):
//  1. Householder tridiagonalisation of the lower triangle (LAPACK's dsytd2 scheme): for column
//     j, x = A(j+1:n, j), beta = -sign(x0) ||x||, tau = (beta - x0) / beta, v = x / (x0 - beta)
//     with v0 = 1; p = tau A22 v, w = p - (tau/2)(p^T v) v, A22 -= v w^T + w v^T.  The rank-2
//     update of column j+1 is done first, its reflector formed, and the rest of the update is
//     fused with the next product A22' v' into one read-write pass over the trailing matrix.
//  2. Implicit QL with Wilkinson shifts on (d, e) (Bowdler, Martin, Reinsch, Wilkinson, "The QR
//     and QL algorithms for symmetric matrices", Numer. Math. 11 (1968); EISPACK tql2), on the
//     tridiagonal scaled by a power of two to unit maximum.  One thread generates the Givens
//     rotations of QL_K sweeps at a time into shared memory while the others apply the previous
//     QL_K sweeps to their row of Z: the sweeps of a batch are applied in one pass over the row as
//     a wavefront (sweep s runs two columns behind sweep s - 1, Van Zee, van de Geijn,
//     Quintana-Orti, "Restructuring the tridiagonal and bidiagonal QR algorithms for
//     performance", ACM TOMS 40 (2014)), in a register window with loads issued QL_D columns
//     ahead.
//  3. Z is transposed through shared-memory tiles, then the reflectors are applied in blocks of
//     BT_K from the last, each block as I - V T V^T (compact WY, T upper triangular: Schreiber,
//     Van Loan, SIAM J. Sci. Stat. Comput. 10 (1989)), with one thread per column of Z.
//  4. Eigenpairs are ranked (ties by index) and written in ascending order through a permuting
//     tiled transpose.
// QL sweeps are bounded (60 per eigenvalue, then CUEV_ERR_CONVERGENCE in the status word); NaN or
// Inf in the input gives CUEV_ERR_NONFINITE and NaN outputs for that matrix.
#include "common.cuh"

#include <algorithm>
#include <mutex>

namespace cuev {
namespace {

constexpr int BMID_MAXN = 512;
constexpr int BMID_MAX_ITERS = 60;
constexpr int PF = 8; // loads in flight per thread in the row passes

// NT threads own rows t, t + NT, ... (R rows each) of matrices with n <= NT R; QL applies K
// sweeps per pass over a row (prefetch distance QL_D, register window 2K + QL_D); the
// back-transform takes BTK reflectors per block.  Shared memory is sized so that several CTAs
// (and so several rotation generators) share an SM.  During QL the last warp only generates
// rotations (lane 0) and the rows are spread over the other NT - 32 threads: a generating lane
// in a warp that also applies rotations would serialise the warp's two paths.
template <int NT_, int R_, int K_, int BTK_> struct MidCfg {
    static constexpr int NT = NT_, R = R_, K = K_, BTK = BTK_;
    static constexpr int MAXN = NT * R;
    static constexpr int QL_D = 8;
    static constexpr int QL_W = 2 * K + QL_D;
    static constexpr int GEN = NT - 32;  // the thread that generates the rotations
    static constexpr int NAPP = NT - 32; // the threads that apply them
    static_assert(NT % 32 == 0 && NT >= BTK && BTK % 2 == 0, "shape");
};

template <class C> struct MidSmem {
    double d[C::MAXN], e[C::MAXN], tau[C::MAXN];
    double red[C::NT / 32];
    double tile[32][33];
    int rank[C::MAXN];
    double alpha, scale;
    int fail;
    union {
        struct {
            double v[2][C::MAXN]; // reflectors of the current and the next column
            double w[C::MAXN];
        } tri;
        struct {
            double2 rot[2][C::K][C::MAXN]; // (c, s) of pair (i, i+1), two batches
            int lo[2][C::K], hi[2][C::K], cnt[2];
        } ql;
        struct {
            double V[C::MAXN * C::BTK];       // V(row, k) at [(row - j0 - 1) * BTK + k]
            double G[2][C::BTK][C::BTK + 1];  // V^T V, two partial sums (even and odd rows)
            double T[C::BTK][C::BTK + 1];
        } bt;
    } u;
};

template <int NT> __device__ __forceinline__ double bmid_block_sum(double v, double *red) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads(); // red[] may still be read by the previous reduction
    if (lane == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < NT / 32; ++q) s += red[q];
    return s; // every thread, same order: identical result everywhere
}

template <int NT> __device__ __forceinline__ double bmid_block_max(double v, double *red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < NT / 32; ++q) s = fmax(s, red[q]);
    return s;
}

// dst (row-major view: dst[r n + c]) = src column-major (src[r + c n]), n x n, through 32 x 33
// shared-memory tiles.
template <int NT>
__device__ void bmid_transpose(const double *__restrict__ src, double *__restrict__ dst, int n,
                               double (*tile)[33]) {
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int c0 = 0; c0 < n; c0 += 32)
        for (int r0 = 0; r0 < n; r0 += 32) {
            for (int yy = ty; yy < 32; yy += NT / 32) { // read columns c0+yy, rows r0+tx
                const int r = r0 + tx, c = c0 + yy;
                tile[yy][tx] = (r < n && c < n) ? src[r + (size_t)c * n] : 0.0;
            }
            __syncthreads();
            for (int yy = ty; yy < 32; yy += NT / 32) { // write rows r0+yy, columns c0+tx
                const int r = r0 + yy, c = c0 + tx;
                if (r < n && c < n) dst[(size_t)r * n + c] = tile[tx][yy];
            }
            __syncthreads();
        }
}

// V (column-major) with column rank[c] = column c of Z, Z given row-major (Zr[r n + c]).
template <int NT>
__device__ void bmid_write_sorted(const double *__restrict__ Zr, double *__restrict__ V, int n,
                                  const int *rank, double (*tile)[33]) {
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int c0 = 0; c0 < n; c0 += 32)
        for (int r0 = 0; r0 < n; r0 += 32) {
            for (int yy = ty; yy < 32; yy += NT / 32) { // Zr rows r0+yy, columns c0+tx
                const int r = r0 + yy, c = c0 + tx;
                tile[yy][tx] = (r < n && c < n) ? Zr[(size_t)r * n + c] : 0.0;
            }
            __syncthreads();
            for (int yy = ty; yy < 32; yy += NT / 32) { // column c0+yy, rows r0+tx
                const int r = r0 + tx, c = c0 + yy;
                if (r < n && c < n) V[r + (size_t)rank[c] * n] = tile[tx][yy];
            }
            __syncthreads();
        }
}

// sum over c in [c0, n) of A(r, c) v[c], with A(r, c) = arow[c n]; PF loads in flight.
__device__ __forceinline__ double row_dot(const double *__restrict__ arow, int n, int c0,
                                          const double *v) {
    double acc[PF];
#pragma unroll
    for (int q = 0; q < PF; ++q) acc[q] = 0.0;
    int c = c0;
    for (; c + PF <= n; c += PF) {
        double a[PF];
#pragma unroll
        for (int q = 0; q < PF; ++q) a[q] = arow[(size_t)(c + q) * n];
#pragma unroll
        for (int q = 0; q < PF; ++q) acc[q] = fma(a[q], v[c + q], acc[q]);
    }
    for (; c < n; ++c) acc[0] = fma(arow[(size_t)c * n], v[c], acc[0]);
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < PF; ++q) s += acc[q];
    return s;
}

// For c in [c0, n): A(r, c) -= vr wo[c] + wr vo[c] (stored back), and returns the sum of the
// updated A(r, c) vn[c].  The loads of the next PF columns are issued before the stores of the
// current ones (the addresses are disjoint).
__device__ __forceinline__ double row_update_dot(double *arow, int n, int c0, double vr,
                                                 double wr, const double *vo, const double *wo,
                                                 const double *vn) {
    double acc0 = 0.0, acc1 = 0.0;
    int c = c0;
    const int full = c0 + ((n - c0) / PF) * PF;
    double a[PF];
    if (c < full) {
#pragma unroll
        for (int q = 0; q < PF; ++q) a[q] = arow[(size_t)(c + q) * n];
    }
    for (; c < full; c += PF) {
        double b[PF];
        const bool more = c + PF < full; // uniform
        if (more) {
#pragma unroll
            for (int q = 0; q < PF; ++q) b[q] = arow[(size_t)(c + PF + q) * n];
        }
#pragma unroll
        for (int q = 0; q < PF; ++q) {
            const double x = a[q] - (vr * wo[c + q] + wr * vo[c + q]);
            arow[(size_t)(c + q) * n] = x;
            if (q & 1)
                acc1 = fma(x, vn[c + q], acc1);
            else
                acc0 = fma(x, vn[c + q], acc0);
        }
        if (more) {
#pragma unroll
            for (int q = 0; q < PF; ++q) a[q] = b[q];
        }
    }
    for (; c < n; ++c) {
        const double x = arow[(size_t)c * n] - (vr * wo[c] + wr * vo[c]);
        arow[(size_t)c * n] = x;
        acc0 = fma(x, vn[c], acc0);
    }
    return acc0 + acc1;
}

// Householder reflector of column j from x (row t + k NT holds x[k] = A(t + k NT, j) where that
// row is >= j + 1).  Every thread returns beta and tau, and v[k] for its rows (v_{j+1} = 1, zero
// for rows <= j).  Called by all threads (block reductions).
template <class C>
__device__ __forceinline__ void bmid_reflector(const double (&x)[C::R], int j, int n,
                                               MidSmem<C> &sm, double &beta, double &tau,
                                               double (&v)[C::R]) {
    const int t = threadIdx.x;
    double ss = 0.0;
#pragma unroll
    for (int k = 0; k < C::R; ++k) {
        const int r = t + k * C::NT;
        if (r == j + 1) sm.alpha = x[k];
        if (r >= j + 2 && r < n) ss = fma(x[k], x[k], ss);
    }
    double sig = bmid_block_sum<C::NT>(ss, sm.red);
    const double alpha = sm.alpha; // written before the reduction's barriers
    double nrm = sqrt(alpha * alpha + sig);
    if (!(sig > 1e-280 && nrm < 1e280)) {
        // squares out of range (uniform branch: sig is the same everywhere): the norm again,
        // scaled by max |x|
        double xm = 0.0;
#pragma unroll
        for (int k = 0; k < C::R; ++k) {
            const int r = t + k * C::NT;
            if (r >= j + 1 && r < n) xm = fmax(xm, fabs(x[k]));
        }
        xm = bmid_block_max<C::NT>(xm, sm.red);
        if (xm > 0.0 && xm <= 1.79e308) {
            double s2 = 0.0;
#pragma unroll
            for (int k = 0; k < C::R; ++k) {
                const int r = t + k * C::NT;
                const double xs = x[k] / xm;
                if (r >= j + 2 && r < n) s2 = fma(xs, xs, s2);
            }
            sig = bmid_block_sum<C::NT>(s2, sm.red);
            const double as = alpha / xm;
            nrm = xm * sqrt(as * as + sig);
        } else {
            if (xm != 0.0 && t == 0) sm.fail = 2; // Inf from an overflow
            sig = 0.0;                           // (or a zero column)
            nrm = xm;
        }
    }
    tau = 0.0;
    beta = alpha;
    if (sig != 0.0) {
        beta = -copysign(nrm, alpha);
        tau = (beta - alpha) / beta;
    }
#pragma unroll
    for (int k = 0; k < C::R; ++k) {
        const int r = t + k * C::NT;
        v[k] = (r == j + 1) ? 1.0 : 0.0;
        if (sig != 0.0 && r >= j + 2 && r < n) v[k] = x[k] / (alpha - beta);
    }
}

// QL state of the generating thread between batches: the current l, the sweeps spent on it, and
// the first negligible e index >= l (mk) and >= l + 1 (mk1), -1 when not known.
struct QLState {
    int l, iter, mk, mk1;
};

// Generator (one thread): the next sweeps of implicit QL on (sm.d, sm.e), at most K, into batch
// `buf`.  Sweep s rotates the pairs (i, i+1) for i = hi[s] down to lo[s] with
// (c, s) = rot[buf][s][i].  The tridiagonal has unit scale, so c and s come from one reciprocal
// square root unless f^2 + g^2 is tiny (then hypot).  The deflation test of every e the sweep
// rewrites is made as it is written, so the next sweep starts without a scan.
template <class C> __device__ void ql_generate(MidSmem<C> &sm, int buf, int n, QLState &q) {
    const double eps = 2.220446049250313e-16, tiny = 2.2250738585072014e-308;
    double *d = sm.d, *E = sm.e;
    auto negl = [&](double e, double a, double b) {
        return fabs(e) <= eps * (fabs(a) + fabs(b)) || fabs(e) < tiny;
    };
    int cnt = 0;
    while (cnt < C::K && q.l < n) {
        const int l = q.l;
        if (q.mk < l) {
            int m = l;
            while (m < n - 1 && !negl(E[m], d[m], d[m + 1])) ++m;
            q.mk = m;
            q.mk1 = m > l ? m : -1;
        }
        const int m = q.mk;
        if (m == l) { // d[l] converged
            ++q.l;
            q.iter = 0;
            q.mk = q.mk1;
            q.mk1 = -1;
            continue;
        }
        if (q.iter >= BMID_MAX_ITERS) { // stop: the matrix is reported as failed
            sm.fail = 1;
            q.l = n;
            break;
        }
        ++q.iter;
        double g = (d[l + 1] - d[l]) / (2.0 * E[l]);
        double r = hypot(g, 1.0);
        g = d[m] - d[l] + E[l] / (g + copysign(r, g));
        double s = 1.0, c = 1.0, p = 0.0;
        int ilow = l, mnext = m;
        bool split = false;
        double2 *rot = sm.u.ql.rot[buf][cnt];
        double Ei = E[m - 1], di = d[m - 1], di1 = d[m], dprev = 0.0;
        for (int i = m - 1; i >= l; --i) {
            const double En = (i > l) ? E[i - 1] : 0.0, dn = (i > l) ? d[i - 1] : 0.0;
            const double f = s * Ei, b = c * Ei;
            const double r2 = f * f + g * g;
            double rr;
            if (r2 > 1e-280) {
                const double ri = rsqrt(r2);
                rr = r2 * ri;
                s = f * ri;
                c = g * ri;
            } else {
                rr = hypot(f, g);
                if (rr == 0.0) { // split: the rotations m-1 .. i+1 stand
                    E[i + 1] = 0.0;
                    d[i + 1] = di1 - p;
                    E[m] = 0.0;
                    split = true;
                    ilow = i + 1;
                    break;
                }
                s = f / rr;
                c = g / rr;
            }
            E[i + 1] = rr;
            g = di1 - p;
            r = (di - g) * s + 2.0 * c * b;
            p = s * r;
            const double dnew = g + p;
            d[i + 1] = dnew;
            g = c * r - b;
            rot[i] = make_double2(c, s);
            if (i <= m - 2 && negl(rr, dnew, dprev)) mnext = i + 1; // e[i+1] final now
            dprev = dnew;
            Ei = En;
            di1 = di;
            di = dn;
        }
        if (!split) {
            d[l] -= p;
            E[l] = g;
            E[m] = 0.0;
            q.mk1 = mnext;
            q.mk = negl(g, d[l], dprev) ? l : mnext;
        } else {
            q.mk = q.mk1 = -1;
        }
        sm.u.ql.lo[buf][cnt] = ilow;
        sm.u.ql.hi[buf][cnt] = m - 1;
        ++cnt;
    }
    sm.u.ql.cnt[buf] = cnt;
}

// Applies the sweeps of batch `buf` to one row of Z (z(e) = zrow[e n]) as a wavefront: at time
// tau sweep s rotates the pair P - tau + 2s (P, Q: the highest and lowest pair of the batch);
// column P + 1 - u lives in window slot u mod W, is loaded QL_D steps before sweep 0 reaches it
// and stored once sweep K - 1 has passed it.  lo/hi/P/Q are the same in every thread.
template <class C>
__device__ __forceinline__ void ql_apply_row(double *zrow, int n, const MidSmem<C> &sm, int buf) {
    constexpr int K = C::K, D = C::QL_D, W = C::QL_W;
    int lo[K], hi[K];
    int P = -1, Q = n;
    const int cnt = sm.u.ql.cnt[buf];
#pragma unroll
    for (int s = 0; s < K; ++s) {
        lo[s] = 1;
        hi[s] = 0;
        if (s < cnt) {
            lo[s] = sm.u.ql.lo[buf][s];
            hi[s] = sm.u.ql.hi[buf][s];
            if (lo[s] <= hi[s]) {
                P = max(P, hi[s]);
                Q = min(Q, lo[s]);
            }
        }
    }
    if (P < Q) return;
    const int steps = P - Q + 2 * K;
    const double2 *rot = sm.u.ql.rot[buf][0];
    double z[W];
#pragma unroll
    for (int u = 0; u <= D; ++u) {
        const int e = P + 1 - u;
        z[u] = (e >= Q) ? zrow[(size_t)e * n] : 0.0;
    }
    for (int t0 = 0; t0 < steps; t0 += W) {
#pragma unroll
        for (int rho = 0; rho < W; ++rho) {
            const int tau = t0 + rho;
            if (tau < steps) {
                {
                    const int e = P - tau - D;
                    if (e >= Q) z[(rho + 1 + D) % W] = zrow[(size_t)e * n];
                }
#pragma unroll
                for (int s = 0; s < K; ++s) {
                    const int i = P - tau + 2 * s;
                    if (i >= lo[s] && i <= hi[s]) {
                        const double2 cs = rot[s * C::MAXN + i];
                        double &zl = z[(rho + 1 - 2 * s + W * K) % W]; // column i
                        double &zh = z[(rho - 2 * s + W * K) % W];     // column i + 1
                        const double a = zl, cr = zh;
                        zh = cs.y * a + cs.x * cr;
                        zl = cs.x * a - cs.y * cr;
                    }
                }
                {
                    const int e = P - tau + 2 * K - 1;
                    if (e >= Q && e <= P + 1) zrow[(size_t)e * n] = z[(rho + 2 - 2 * K + W * K) % W];
                }
            }
        }
    }
}

// Z <- (I - V T V^T) Z for the reflectors j0 .. j0 + BTK - 1 (those > n - 3, or with tau = 0,
// contribute nothing), Z row-major (Zr[row n + col]); thread t owns columns t + k NT.  Called
// by all threads.
template <class C>
__device__ void bt_block(double *Zr, const double *Aw, int n, int j0, MidSmem<C> &sm) {
    constexpr int BTK = C::BTK;
    const int t = threadIdx.x;
    const int rows = n - j0 - 1; // rows j0+1 .. n-1
    double *V = sm.u.bt.V;
    // V(row, k): 1 at row j0+k+1, the stored reflector below it, zero above
    for (int idx = t; idx < rows * BTK; idx += C::NT) {
        const int k = idx % BTK, row = j0 + 1 + idx / BTK;
        const int j = j0 + k;
        double v = 0.0;
        if (j <= n - 3) {
            if (row == j + 1)
                v = 1.0;
            else if (row > j + 1)
                v = Aw[row + (size_t)j * n];
        }
        V[idx] = v;
    }
    __syncthreads();
    // G = V^T V (upper triangle): entry (a, b) over the even or the odd rows per thread (the
    // lanes of a warp read one row of V: broadcasts, no bank conflicts)
    for (int idx = t; idx < 2 * BTK * BTK; idx += C::NT) {
        const int pr = idx % (BTK * BTK), half = idx / (BTK * BTK);
        const int a = pr / BTK, b = pr % BTK;
        if (a <= b) {
            double s0 = 0.0, s1 = 0.0;
            int q = half;
            for (; q + 2 < rows; q += 4) {
                s0 = fma(V[q * BTK + a], V[q * BTK + b], s0);
                s1 = fma(V[(q + 2) * BTK + a], V[(q + 2) * BTK + b], s1);
            }
            if (q < rows) s0 = fma(V[q * BTK + a], V[q * BTK + b], s0);
            sm.u.bt.G[half][a][b] = s0 + s1;
        }
    }
    __syncthreads();
    // T upper triangular, row a by thread a (kept in shared memory as it is formed):
    // T(a, a) = tau_a, T(a, i) = -tau_i sum_{b = a .. i-1} T(a, b) G(b, i)
    if (t < BTK) {
        const int a = t;
        double *Trow = sm.u.bt.T[a];
        for (int i = 0; i < a; ++i) Trow[i] = 0.0;
        Trow[a] = (j0 + a <= n - 3) ? sm.tau[j0 + a] : 0.0;
        for (int i = a + 1; i < BTK; ++i) {
            const double ti = (j0 + i <= n - 3) ? sm.tau[j0 + i] : 0.0;
            double s = 0.0;
            for (int b = a; b < i; ++b)
                s = fma(Trow[b], sm.u.bt.G[0][b][i] + sm.u.bt.G[1][b][i], s);
            Trow[i] = -ti * s;
        }
    }
    __syncthreads();
#pragma unroll 1
    for (int kc = 0; kc < C::R; ++kc) {
        const int col = t + kc * C::NT;
        if (col >= n) break;
        double *zc = Zr + (size_t)(j0 + 1) * n + col; // column col, rows j0+1 ..
        double w[BTK];
#pragma unroll
        for (int k = 0; k < BTK; ++k) w[k] = 0.0;
        int q = 0;
        for (; q + 4 <= rows; q += 4) {
            double zv[4];
#pragma unroll
            for (int h = 0; h < 4; ++h) zv[h] = zc[(size_t)(q + h) * n];
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                const double2 *vr = reinterpret_cast<const double2 *>(V + (q + h) * BTK);
#pragma unroll
                for (int k2 = 0; k2 < BTK / 2; ++k2) {
                    const double2 vv = vr[k2];
                    w[2 * k2] = fma(vv.x, zv[h], w[2 * k2]);
                    w[2 * k2 + 1] = fma(vv.y, zv[h], w[2 * k2 + 1]);
                }
            }
        }
        for (; q < rows; ++q) {
            const double zq = zc[(size_t)q * n];
#pragma unroll
            for (int k = 0; k < BTK; ++k) w[k] = fma(V[q * BTK + k], zq, w[k]);
        }
        // w <- T w in place (T upper triangular: entry a needs w[b >= a] only)
#pragma unroll
        for (int a = 0; a < BTK; ++a) {
            double s = 0.0;
#pragma unroll
            for (int b = 0; b < BTK; ++b)
                if (b >= a) s = fma(sm.u.bt.T[a][b], w[b], s);
            w[a] = s;
        }
        q = 0;
        for (; q + 4 <= rows; q += 4) {
            double zv[4];
#pragma unroll
            for (int h = 0; h < 4; ++h) zv[h] = zc[(size_t)(q + h) * n];
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                const double2 *vr = reinterpret_cast<const double2 *>(V + (q + h) * BTK);
                double s0 = 0.0, s1 = 0.0;
#pragma unroll
                for (int k2 = 0; k2 < BTK / 2; ++k2) {
                    const double2 vv = vr[k2];
                    s0 = fma(vv.x, w[2 * k2], s0);
                    s1 = fma(vv.y, w[2 * k2 + 1], s1);
                }
                zc[(size_t)(q + h) * n] = zv[h] - (s0 + s1);
            }
        }
        for (; q < rows; ++q) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < BTK; ++k) s = fma(V[q * BTK + k], w[k], s);
            zc[(size_t)q * n] -= s;
        }
    }
    __syncthreads(); // V is rewritten by the next block
}

template <class C>
__global__ void __launch_bounds__(C::NT, (65536 / 128) / C::NT)
    batched_mid_kernel(const double *__restrict__ A, int n, int batch, double *__restrict__ eval,
                       double *__restrict__ evec, double *__restrict__ work,
                       int *__restrict__ status) {
    constexpr int NT = C::NT, R = C::R;
    extern __shared__ __align__(16) unsigned char bmid_smem_raw[];
    MidSmem<C> &sm = *reinterpret_cast<MidSmem<C> *>(bmid_smem_raw);
    const int t = threadIdx.x;
    const size_t nn = (size_t)n * n;
    double *Aw = work + (size_t)blockIdx.x * 3 * nn; // reflectors below the subdiagonal
    double *Zc = Aw + nn;                            // QL eigenvectors, column-major
    double *Zr = Zc + nn;                            // the same, row-major (back-transform)

    for (int mat = blockIdx.x; mat < batch; mat += gridDim.x) {
        const double *Ab = A + (size_t)mat * nn;
        // ---- symmetric copy of the lower triangle (every stored entry is read once as itself)
        int bad = 0;
        for (size_t idx = t; idx < nn; idx += NT) {
            const int i = (int)(idx % n), j = (int)(idx / n);
            const double a = i >= j ? Ab[idx] : Ab[j + (size_t)i * n];
            bad |= !isfinite(a);
            Aw[idx] = a;
        }
        if (t == 0) sm.fail = 0;
        if (__syncthreads_or(bad)) { // uniform: NaN or Inf in the input, outputs set to NaN
            const double qnan = __longlong_as_double(0x7ff8000000000000LL);
            for (size_t idx = t; idx < nn; idx += NT) evec[(size_t)mat * nn + idx] = qnan;
            for (int r = t; r < n; r += NT) eval[(size_t)mat * n + r] = qnan;
            if (t == 0) dev_fail(status, CUEV_ERR_NONFINITE, mat);
            continue;
        }

        // ---- 1. tridiagonalisation (n >= 3); thread t owns rows t + k NT
        {
            double *vc = sm.u.tri.v[0], *vn = sm.u.tri.v[1], *sw = sm.u.tri.w;
            double beta, tau, v[R], p[R], x[R];
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const int r = t + k * NT;
                x[k] = (r >= 1 && r < n) ? Aw[r] : 0.0; // column 0
            }
            bmid_reflector<C>(x, 0, n, sm, beta, tau, v);
            if (t == 0) sm.d[0] = Aw[0];
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const int r = t + k * NT;
                if (r >= 1 && r < n) {
                    vc[r] = v[k];
                    Aw[r] = (r == 1) ? beta : v[k];
                }
            }
            __syncthreads();
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const int r = t + k * NT;
                p[k] = (r >= 1 && r < n) ? tau * row_dot(Aw + r, n, 1, vc) : 0.0;
            }
            for (int j = 0; j + 2 < n; ++j) {
                double pvl = 0.0;
#pragma unroll
                for (int k = 0; k < R; ++k) {
                    const int r = t + k * NT;
                    if (r >= j + 1 && r < n) pvl = fma(p[k], v[k], pvl);
                }
                const double pv = bmid_block_sum<NT>(pvl, sm.red);
                double wr[R];
#pragma unroll
                for (int k = 0; k < R; ++k) {
                    const int r = t + k * NT;
                    wr[k] = p[k] - 0.5 * tau * pv * v[k];
                    if (r >= j + 1 && r < n) sw[r] = wr[k];
                }
                if (t == 0) {
                    sm.e[j] = beta;
                    sm.tau[j] = tau;
                }
                __syncthreads();
                if (j + 3 < n) {
                    // column j+1 of the rank-2 update, then its reflector
                    double a[R];
#pragma unroll
                    for (int k = 0; k < R; ++k) {
                        const int r = t + k * NT;
                        a[k] = 0.0;
                        if (r >= j + 1 && r < n) {
                            a[k] = Aw[r + (size_t)(j + 1) * n] -
                                   (v[k] * sw[j + 1] + wr[k] * vc[j + 1]);
                            if (r == j + 1) sm.d[j + 1] = a[k];
                        }
                    }
                    double beta2, tau2, v2[R];
                    bmid_reflector<C>(a, j + 1, n, sm, beta2, tau2, v2);
#pragma unroll
                    for (int k = 0; k < R; ++k) {
                        const int r = t + k * NT;
                        if (r >= j + 2 && r < n) {
                            vn[r] = v2[k];
                            Aw[r + (size_t)(j + 1) * n] = (r == j + 2) ? beta2 : v2[k];
                        }
                    }
                    __syncthreads();
                    // the rest of the update fused with p' = tau' A22' v'
#pragma unroll
                    for (int k = 0; k < R; ++k) {
                        const int r = t + k * NT;
                        p[k] = (r >= j + 2 && r < n)
                                   ? tau2 * row_update_dot(Aw + r, n, j + 2, v[k], wr[k], vc, sw, vn)
                                   : 0.0;
                        v[k] = v2[k];
                    }
                    double *tmp = vc;
                    vc = vn;
                    vn = tmp;
                    beta = beta2;
                    tau = tau2;
                } else {
                    // j = n - 3: the trailing 2 x 2 block
#pragma unroll
                    for (int k = 0; k < R; ++k) {
                        const int r = t + k * NT;
                        if (r >= n - 2 && r < n) {
                            const double a0 =
                                Aw[r + (size_t)(n - 2) * n] - (v[k] * sw[n - 2] + wr[k] * vc[n - 2]);
                            const double a1 =
                                Aw[r + (size_t)(n - 1) * n] - (v[k] * sw[n - 1] + wr[k] * vc[n - 1]);
                            if (r == n - 2) {
                                sm.d[n - 2] = a0;
                            } else {
                                sm.d[n - 1] = a1;
                                sm.e[n - 2] = a0;
                            }
                        }
                    }
                }
            }
            if (t == 0) {
                sm.e[n - 1] = 0.0;
                sm.tau[n - 2] = 0.0;
            }
        }
        // Z = I (column-major)
        for (size_t idx = t; idx < nn; idx += NT) Zc[idx] = (idx % n == idx / n) ? 1.0 : 0.0;
        __syncthreads();

        // ---- 2. implicit QL on the tridiagonal scaled to unit maximum
        {
            double mx = 0.0;
            int nonfin = 0;
            for (int r = t; r < n; r += NT) {
                mx = fmax(mx, fmax(fabs(sm.d[r]), fabs(sm.e[r])));
                nonfin |= !(isfinite(sm.d[r]) && isfinite(sm.e[r]));
            }
            if (!__syncthreads_or(nonfin) && sm.fail == 0) {
                mx = bmid_block_max<NT>(mx, sm.red);
                const double sc = mx > 0.0 ? ldexp(1.0, -ilogb(mx)) : 1.0; // exact power of two
                for (int r = t; r < n; r += NT) {
                    sm.d[r] *= sc;
                    sm.e[r] *= sc;
                }
                if (t == 0) sm.scale = sc;
                __syncthreads();
                QLState q{0, 0, -1, -1}; // used by the generating thread only
                if (t == C::GEN) ql_generate<C>(sm, 0, n, q);
                __syncthreads();
                for (int b = 0;; ++b) {
                    const int buf = b & 1;
                    if (sm.u.ql.cnt[buf] == 0) break; // uniform
                    if (t == C::GEN) ql_generate<C>(sm, buf ^ 1, n, q);
#pragma unroll 1
                    for (int r = t; t < C::NAPP && r < n; r += C::NAPP)
                        ql_apply_row<C>(Zc + r, n, sm, buf);
                    __syncthreads();
                }
                for (int r = t; r < n; r += NT) sm.d[r] /= sm.scale;
            } else if (t == 0) {
                sm.fail = 2;
            }
            __syncthreads();
        }
        if (t == 0 && sm.fail)
            dev_fail(status, sm.fail == 2 ? CUEV_ERR_NONFINITE : CUEV_ERR_CONVERGENCE, mat);

        // ---- 3. back-transform Z <- H_0 ... H_(n-3) Z on the row-major copy, last block first
        bmid_transpose<NT>(Zc, Zr, n, sm.tile);
        for (int j0 = ((n - 3) / C::BTK) * C::BTK; j0 >= 0; j0 -= C::BTK)
            bt_block<C>(Zr, Aw, n, j0, sm);

        // ---- 4. ascending order: rank, then a permuting transpose into evec
        for (int r = t; r < n; r += NT) {
            const double li = sm.d[r];
            int rank = 0;
            for (int q2 = 0; q2 < n; ++q2) {
                const double lq = sm.d[q2];
                rank += (lq < li) || (lq == li && q2 < r);
            }
            sm.rank[r] = rank;
            eval[(size_t)mat * n + rank] = li;
        }
        __syncthreads();
        bmid_write_sorted<NT>(Zr, evec + (size_t)mat * nn, n, sm.rank, sm.tile);
    }
}

// Shapes: n <= 128: 128 threads, one row each (four CTAs per SM); n <= 256: 128 threads, two rows
// each (four per SM); n <= 512: 256 threads, two rows each (two per SM).
using MidSmall = MidCfg<128, 1, 6, 16>;
using MidMedium = MidCfg<128, 2, 4, 16>;
using MidLarge = MidCfg<256, 2, 4, 16>;

// per-device workspace (calls are serialised by the batched entry in batched_small.cu)
std::mutex g_bm_mu;
void *g_bm_buf[64] = {nullptr};
size_t g_bm_bytes[64] = {0};

template <class C>
int launch_mid(const double *A, int n, int batch, double *eval, double *evec, int *status,
               cudaStream_t st, int dev) {
    auto kern = batched_mid_kernel<C>;
    const size_t smem = sizeof(MidSmem<C>);
    CUEV_CHECK_STATUS(ensure_dyn_smem((const void *)kern, smem));
    int per_sm = 0;
    CUEV_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, C::NT, smem));
    const int grid = std::min(batch, num_sms() * std::max(per_sm, 1));
    const size_t bytes = (size_t)grid * 3 * n * n * sizeof(double);
    // the lock is held until the launch is enqueued: a release frees the buffer only after it
    // (cudaFree waits for the device)
    std::lock_guard<std::mutex> lk(g_bm_mu);
    if (g_bm_bytes[dev] < bytes) {
        CUEV_TRY(cudaStreamSynchronize(st));
        if (g_bm_buf[dev]) CUEV_TRY(cudaFree(g_bm_buf[dev]));
        g_bm_buf[dev] = nullptr;
        g_bm_bytes[dev] = 0;
        if (cudaMalloc(&g_bm_buf[dev], bytes) != cudaSuccess) {
            cudaGetLastError();
            set_last_message("batched eigensolver: workspace allocation failed");
            return CUEV_ERR_ALLOC;
        }
        g_bm_bytes[dev] = bytes;
    }
    kern<<<grid, C::NT, smem, st>>>(A, n, batch, eval, evec, (double *)g_bm_buf[dev], status);
    note_launch();
    CUEV_TRY(cudaGetLastError());
    return CUEV_OK;
}

} // namespace

// Stacks of 64 < n <= 512 matrices, launched on st (called by batched_eigh_d, which validates
// the arguments, owns the status word and synchronises).
int batched_eigh_mid(const double *A, int n, int batch, double *eval, double *evec, int *status,
                     cudaStream_t st) {
    if (n < 3 || n > BMID_MAXN || batch <= 0) return CUEV_ERR_INVALID;
    int dev = 0;
    CUEV_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return CUEV_ERR_INVALID;
    if (n <= MidSmall::MAXN) return launch_mid<MidSmall>(A, n, batch, eval, evec, status, st, dev);
    if (n <= MidMedium::MAXN) return launch_mid<MidMedium>(A, n, batch, eval, evec, status, st, dev);
    return launch_mid<MidLarge>(A, n, batch, eval, evec, status, st, dev);
}

// Frees the mid-size workspaces of every device (cuev_release_workspace).
void batched_mid_release() {
    std::lock_guard<std::mutex> lk(g_bm_mu);
    int cur = 0;
    if (cudaGetDevice(&cur) != cudaSuccess) return;
    for (int d = 0; d < 64; ++d)
        if (g_bm_buf[d]) {
            if (cudaSetDevice(d) == cudaSuccess) cudaFree(g_bm_buf[d]);
            g_bm_buf[d] = nullptr;
            g_bm_bytes[d] = 0;
        }
    cudaSetDevice(cur);
    cudaGetLastError();
}

} // namespace cuev
