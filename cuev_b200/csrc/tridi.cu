// Stage 3: symmetric tridiagonal divide and conquer, entirely on the GPU.
//
// The reference runs this stage on the host with LAPACK pieces (src/cuda/tridi.cu:106-452:
// dsteqr leaves, dlaed2 deflation, dlaed4 secular roots, dlamrg) and ships Q2/S blocks over PCIe
// for every merge GEMM.  Here the same mathematics (Cuppen's tearing, Dongarra-Sorensen/Gu-
// Eisenstat deflation, secular equation, Loewner weights) is restated as batched GPU kernels.
// The split tree is the reference's (halve every part while the largest exceeds 64 rows,
// tridi.cu:268-283), so all sub-problems of one tree level are processed together:
//
//   leaves      dc_leaf_kernel         one warp per leaf: implicit QL with Wilkinson shift
//   per level   dc_deflate_kernel      z, merge of the two sorted halves, deflation scan
//               dc_rotate_kernel       Givens rotations + type-compressed copy (row-parallel)
//               dc_secular_kernel      one warp per root: two-pole rational model + bisection
//               dc_lowner_kernel       Loewner weights (accurate eigenvectors)
//               dc_svec_kernel         rank-one eigenvector matrix, type-ordered rows
//               batched DMMA GEMM      Q_new = Q2c * S for every merge, top and bottom blocks
//               dc_order_kernel        final ascending order (roots merged with deflated)
//               dc_permute_kernel      write the merged eigenvectors back
//
// All waits are bounded: the only loops are fixed-count iterations (QL <= 60 sweeps per
// eigenvalue, secular <= 100 steps with bisection fallback); failures set CUEV_ERR_CONVERGENCE.
#include "solver.cuh"

#include <algorithm>
#include <cfloat>
#include <cstring>
#include <vector>

namespace cuev {
namespace {

constexpr int LEAF_MAX = 64; // SMLSIZ of the reference (src/cuda/tridi.cu:63)
constexpr double EPS = DBL_EPSILON;

struct MergeDesc {
    int off, nm, n1, pad;
    long long base; // offset (elements) of this merge's n_m^2 regions in the level buffers
};

// per-merge device info words
enum { MI_K = 0, MI_CT1, MI_CT2, MI_CT3, MI_ND, MI_NROT, MI_WORDS = 8 };

struct DcArrays {
    // doubles, length n each
    double *E, *z, *dsort, *zsort, *dlam, *w, *lam, *what, *dval, *rc, *rs, *newd;
    // ints, length n each
    int *perm, *tsort, *ndcol, *ndtyp, *cpos, *dcol, *rp, *rq, *src;
    int *info; // MI_WORDS per merge
    double *scale; // [0] = max norm
};

// ------------------------------------------------------------------------------------------
// scaling
// ------------------------------------------------------------------------------------------
__global__ void dc_norm_kernel(const double *__restrict__ d, const double *__restrict__ e, int n,
                               double *scale, int *status) {
    __shared__ double red[32];
    double m = 0.0;
    bool bad = false;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double a = fabs(d[i]);
        m = fmax(m, a);
        bad |= !isfinite(d[i]);
        if (i < n - 1) {
            m = fmax(m, fabs(e[i]));
            bad |= !isfinite(e[i]);
        }
    }
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        v = warp_max(v);
        if (threadIdx.x == 0) scale[0] = v;
    }
    if (bad) dev_fail(status, CUEV_ERR_NONFINITE, -1);
}

__global__ void dc_scale_in_kernel(const double *__restrict__ d, const double *__restrict__ e,
                                   double *__restrict__ D, double *__restrict__ E, int n,
                                   const double *scale) {
    const double s = scale[0] > 0.0 ? 1.0 / scale[0] : 1.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        D[i] = d[i] * s;
        E[i] = (i < n - 1) ? e[i] * s : 0.0;
    }
}

__global__ void dc_scale_out_kernel(double *__restrict__ D, int n, const double *scale) {
    const double s = scale[0] > 0.0 ? scale[0] : 1.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        D[i] *= s;
}

// ------------------------------------------------------------------------------------------
// leaves: implicit QL with Wilkinson shift (Bowdler-Martin-Reinsch-Wilkinson), one warp each
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(32)
    dc_leaf_kernel(const int2 *__restrict__ leaves, double *__restrict__ D,
                   const double *__restrict__ E, double *__restrict__ Q, long long ldq, int n,
                   int *status) {
    __shared__ double sd[LEAF_MAX], se[LEAF_MAX];
    __shared__ double Z[LEAF_MAX][LEAF_MAX + 1];
    __shared__ double rcs[LEAF_MAX], rsn[LEAF_MAX];
    __shared__ int s_nrot, s_lo;
    const int lane = threadIdx.x;
    const int2 lf = leaves[blockIdx.x];
    const int off = lf.x, m = lf.y;

    // load with the rank-one tearing of the neighbouring cuts (d -= |e_cut|)
    for (int i = lane; i < m; i += 32) {
        double di = D[off + i];
        if (i == 0 && off > 0) di -= fabs(E[off - 1]);
        if (i == m - 1 && off + m < n) di -= fabs(E[off + m - 1]);
        sd[i] = di;
        se[i] = (i < m - 1) ? E[off + i] : 0.0;
    }
    for (int idx = lane; idx < m * m; idx += 32) {
        const int r = idx % m, c = idx / m;
        Z[r][c] = (r == c) ? 1.0 : 0.0;
    }
    __syncwarp();

    bool failed = false;
    for (int l = 0; l < m && !failed; ++l) {
        for (int iter = 0;; ++iter) {
            // all lanes agree on mm (same shared data)
            int mm = l;
            for (; mm < m - 1; ++mm) {
                const double dd = fabs(sd[mm]) + fabs(sd[mm + 1]);
                if (fabs(se[mm]) <= EPS * dd) break;
            }
            if (mm == l) break;
            if (iter >= 60) {
                failed = true;
                break;
            }
            if (lane == 0) {
                double g = (sd[l + 1] - sd[l]) / (2.0 * se[l]);
                double r = hypot(g, 1.0);
                g = sd[mm] - sd[l] + se[l] / (g + copysign(r, g));
                double s = 1.0, c = 1.0, p = 0.0;
                int i = mm - 1;
                int nrot = 0;
                bool underflow = false;
                for (; i >= l; --i) {
                    const double f = s * se[i];
                    const double bb = c * se[i];
                    r = hypot(f, g);
                    se[i + 1] = r;
                    if (r == 0.0) {
                        sd[i + 1] -= p;
                        se[mm] = 0.0;
                        underflow = true;
                        break;
                    }
                    s = f / r;
                    c = g / r;
                    g = sd[i + 1] - p;
                    r = (sd[i] - g) * s + 2.0 * c * bb;
                    p = s * r;
                    sd[i + 1] = g + p;
                    g = c * r - bb;
                    rcs[nrot] = c;
                    rsn[nrot] = s;
                    ++nrot;
                }
                if (!underflow) {
                    sd[l] -= p;
                    se[l] = g;
                    se[mm] = 0.0;
                }
                s_nrot = nrot;
                s_lo = mm - 1; // rotation t acts on columns (s_lo - t, s_lo - t + 1)
            }
            __syncwarp();
            const int nrot = s_nrot, ilo = s_lo;
            for (int rrow = lane; rrow < m; rrow += 32) {
                for (int t = 0; t < nrot; ++t) {
                    const int i = ilo - t;
                    const double c = rcs[t], s = rsn[t];
                    const double f = Z[rrow][i + 1];
                    Z[rrow][i + 1] = s * Z[rrow][i] + c * f;
                    Z[rrow][i] = c * Z[rrow][i] - s * f;
                }
            }
            __syncwarp();
        }
    }
    if (failed) {
        if (lane == 0) dev_fail(status, CUEV_ERR_CONVERGENCE, off);
        return;
    }
    // ascending order (selection sort on columns)
    for (int i = 0; i < m - 1; ++i) {
        int kmin = i;
        double p = sd[i];
        for (int j = i + 1; j < m; ++j)
            if (sd[j] < p) kmin = j, p = sd[j];
        __syncwarp();
        if (kmin != i) {
            for (int rrow = lane; rrow < m; rrow += 32) {
                const double t = Z[rrow][i];
                Z[rrow][i] = Z[rrow][kmin];
                Z[rrow][kmin] = t;
            }
            __syncwarp();
            if (lane == 0) {
                sd[kmin] = sd[i];
                sd[i] = p;
            }
        }
        __syncwarp();
    }
    for (int i = lane; i < m; i += 32) D[off + i] = sd[i];
    for (int idx = lane; idx < m * m; idx += 32) {
        const int r = idx % m, c = idx / m;
        Q[(off + r) + (long long)(off + c) * ldq] = Z[r][c];
    }
}

// ------------------------------------------------------------------------------------------
// deflation (one CTA per merge)
// ------------------------------------------------------------------------------------------
constexpr int DF_THREADS = 512;
constexpr int DF_CHUNK = 1536;

__device__ __forceinline__ int lower_bound_d(const double *a, int len, double x) {
    int lo = 0, hi = len;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}
__device__ __forceinline__ int upper_bound_d(const double *a, int len, double x) {
    int lo = 0, hi = len;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] <= x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(DF_THREADS)
    dc_deflate_kernel(const MergeDesc *__restrict__ descs, double *__restrict__ D,
                      const double *__restrict__ Q, long long ldq, DcArrays a) {
    __shared__ double s_d[DF_CHUNK], s_z[DF_CHUNK];
    __shared__ int s_t[DF_CHUNK], s_c[DF_CHUNK];
    __shared__ double red[32];
    const MergeDesc md = descs[blockIdx.x];
    const int off = md.off, nm = md.nm, n1 = md.n1;
    const int tid = threadIdx.x;
    const double rho_in = a.E[off + n1 - 1];
    const double rho = 2.0 * fabs(rho_in);
    const double zsign = rho_in < 0.0 ? -1.0 : 1.0;
    const double inv_sqrt2 = 0.70710678118654752440;
    const double *Qb = Q + off + (long long)off * ldq;
    const double *Db = D + off;

    // z and the sorted merge of the two halves (each half ascending)
    double zmax = 0.0;
    for (int i = tid; i < nm; i += DF_THREADS) {
        double zi;
        int pos;
        if (i < n1) {
            zi = Qb[(n1 - 1) + (long long)i * ldq];
            pos = i + lower_bound_d(Db + n1, nm - n1, Db[i]);
        } else {
            zi = zsign * Qb[n1 + (long long)i * ldq];
            pos = (i - n1) + upper_bound_d(Db, n1, Db[i]);
        }
        zi *= inv_sqrt2;
        a.z[off + i] = zi;
        a.perm[off + pos] = i;
        zmax = fmax(zmax, fabs(zi));
    }
    zmax = warp_max(zmax);
    if ((tid & 31) == 0) red[tid >> 5] = zmax;
    __syncthreads();
    if (tid < 32) {
        double v = tid < DF_THREADS / 32 ? red[tid] : 0.0;
        v = warp_max(v);
        if (tid == 0) red[0] = v;
    }
    __syncthreads();
    zmax = red[0];
    const double dmax = fmax(fmax(fabs(Db[0]), fabs(Db[n1 - 1])),
                             fmax(fabs(Db[n1]), fabs(Db[nm - 1])));
    const double tol = 8.0 * EPS * fmax(dmax, zmax);
    __syncthreads();
    // sorted copies (the scan then streams them in order)
    for (int idx = tid; idx < nm; idx += DF_THREADS) {
        const int i = a.perm[off + idx];
        a.dsort[off + idx] = Db[i];
        a.zsort[off + idx] = a.z[off + i];
        a.tsort[off + idx] = i < n1 ? 1 : 3;
    }
    __syncthreads();

    // sequential deflation scan (thread 0), input staged in shared memory chunk by chunk.
    // Candidate pj is carried in registers.
    int k = 0, nd = 0, nrot = 0;
    int pj = -1, pt = 0;
    double pz = 0.0, pdv = 0.0;
    for (int c0 = 0; c0 < nm; c0 += DF_CHUNK) {
        const int cl = min(DF_CHUNK, nm - c0);
        __syncthreads();
        for (int t = tid; t < cl; t += DF_THREADS) {
            s_d[t] = a.dsort[off + c0 + t];
            s_z[t] = a.zsort[off + c0 + t];
            s_t[t] = a.tsort[off + c0 + t];
            s_c[t] = a.perm[off + c0 + t];
        }
        __syncthreads();
        if (tid == 0) {
            for (int t = 0; t < cl; ++t) {
                const int j = s_c[t];
                double zj = s_z[t], dj = s_d[t];
                int tj = s_t[t];
                if (rho * fabs(zj) <= tol) { // small z: deflate j as is
                    a.dcol[off + nd] = j;
                    a.dval[off + nd] = dj;
                    ++nd;
                    continue;
                }
                if (pj < 0) {
                    pj = j, pz = zj, pdv = dj, pt = tj;
                    continue;
                }
                const double tau = hypot(zj, pz);
                const double cc = zj / tau, ss = -pz / tau;
                const double tt = dj - pdv;
                if (fabs(tt * cc * ss) <= tol) { // close poles: rotate, deflate pj
                    a.rp[off + nrot] = pj;
                    a.rq[off + nrot] = j;
                    a.rc[off + nrot] = cc;
                    a.rs[off + nrot] = ss;
                    ++nrot;
                    const double dp = pdv * cc * cc + dj * ss * ss;
                    dj = pdv * ss * ss + dj * cc * cc;
                    if (tj != pt) tj = 2;
                    a.dcol[off + nd] = pj;
                    a.dval[off + nd] = dp;
                    ++nd;
                    pj = j, pz = tau, pdv = dj, pt = tj;
                } else {
                    a.dlam[off + k] = pdv;
                    a.w[off + k] = pz;
                    a.ndcol[off + k] = pj;
                    a.ndtyp[off + k] = pt;
                    ++k;
                    pj = j, pz = zj, pdv = dj, pt = tj;
                }
            }
        }
    }
    if (tid == 0) {
        if (pj >= 0) {
            a.dlam[off + k] = pdv;
            a.w[off + k] = pz;
            a.ndcol[off + k] = pj;
            a.ndtyp[off + k] = pt;
            ++k;
        }
        // type-ordered compressed positions: [type 1 | type 2 | type 3]
        int ct[4] = {0, 0, 0, 0};
        for (int i = 0; i < k; ++i) ct[a.ndtyp[off + i]]++;
        int base[4] = {0, 0, ct[1], ct[1] + ct[2]};
        for (int i = 0; i < k; ++i) a.cpos[off + i] = base[a.ndtyp[off + i]]++;
        int *info = a.info + blockIdx.x * MI_WORDS;
        info[MI_K] = k;
        info[MI_CT1] = ct[1];
        info[MI_CT2] = ct[2];
        info[MI_CT3] = ct[3];
        info[MI_ND] = nd;
        info[MI_NROT] = nrot;
    }
}

// ------------------------------------------------------------------------------------------
// rotations + compression: Q2c[:, cpos(i)] = Q[:, ndcol(i)] (i < k), Q2c[:, k + d] = deflated
// grid (row chunks, merges); one thread per row of the merged block
// ------------------------------------------------------------------------------------------
__global__ void dc_rotate_kernel(const MergeDesc *__restrict__ descs, double *__restrict__ Q,
                                 long long ldq, double *__restrict__ Q2, DcArrays a) {
    const MergeDesc md = descs[blockIdx.y];
    const int off = md.off, nm = md.nm;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nm) return;
    const int *info = a.info + blockIdx.y * MI_WORDS;
    const int k = info[MI_K], nd = info[MI_ND], nrot = info[MI_NROT];
    double *Qr = Q + (off + r) + (long long)off * ldq; // Qr[c * ldq] = Q(off + r, off + c)
    for (int t = 0; t < nrot; ++t) {
        const int p = a.rp[off + t], q = a.rq[off + t];
        const double c = a.rc[off + t], s = a.rs[off + t];
        const double x = Qr[(long long)p * ldq], y = Qr[(long long)q * ldq];
        Qr[(long long)p * ldq] = c * x + s * y;
        Qr[(long long)q * ldq] = c * y - s * x;
    }
    double *Q2b = Q2 + md.base;
    for (int i = 0; i < k; ++i)
        Q2b[r + (long long)a.cpos[off + i] * nm] = Qr[(long long)a.ndcol[off + i] * ldq];
    for (int dd = 0; dd < nd; ++dd)
        Q2b[r + (long long)(k + dd) * nm] = Qr[(long long)a.dcol[off + dd] * ldq];
}

__device__ __forceinline__ int find_merge(const MergeDesc *descs, int count, int g) {
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (descs[mid].off <= g)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// ------------------------------------------------------------------------------------------
// secular equation: 1 + rho sum_i w_i^2 / (d_i - lambda) = 0, one warp per root
// ------------------------------------------------------------------------------------------
__global__ void dc_secular_kernel(const MergeDesc *__restrict__ descs, int count, int n,
                                  double *__restrict__ Dl, DcArrays a, int *status) {
    const int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (g >= n) return;
    const int mi = find_merge(descs, count, g);
    const MergeDesc md = descs[mi];
    const int j = g - md.off;
    const int k = a.info[mi * MI_WORDS + MI_K];
    if (j >= k) return;
    const int off = md.off;
    const double rho = 2.0 * fabs(a.E[off + md.n1 - 1]);
    const double *dl = a.dlam + off;
    const double *w = a.w + off;
    double *Delta = Dl + md.base + (long long)j * k;

    // origin: the pole nearer to the root
    int org = j;
    double hi_bound, lo_bound;
    if (j < k - 1) {
        const double gap = dl[j + 1] - dl[j];
        const double mid = 0.5 * gap;
        double f = 0.0;
        for (int i = lane; i < k; i += 32) f += w[i] * w[i] / ((dl[i] - dl[j]) - mid);
        f = 1.0 + rho * warp_sum(f);
        if (f >= 0.0) { // root in (d_j, mid]
            org = j;
            lo_bound = 0.0;
            hi_bound = mid;
        } else { // root in (mid, d_{j+1})
            org = j + 1;
            lo_bound = -mid;
            hi_bound = 0.0;
        }
    } else {
        double wn = 0.0;
        for (int i = lane; i < k; i += 32) wn += w[i] * w[i];
        wn = warp_sum(wn);
        org = j;
        lo_bound = 0.0;
        hi_bound = rho * wn;
    }
    const double dorg = dl[org];
    const int jl = j, jr = j + 1; // the two poles bracketing the root (jr == k: none)
    const double dlo = dl[jl] - dorg;
    const double dhi = (jr < k) ? dl[jr] - dorg : 0.0;

    double tau = (org == j) ? 0.5 * hi_bound : 0.5 * lo_bound;
    if (j == k - 1) tau = hi_bound; // g(hi_bound) >= 0 for the last root
    bool conv = false;
    for (int it = 0; it < 100; ++it) {
        // psi (poles <= j), phi (poles > j) and derivatives at tau
        double psi = 0.0, dpsi = 0.0, phi = 0.0, dphi = 0.0;
        for (int i = lane; i < k; i += 32) {
            const double del = (dl[i] - dorg) - tau;
            const double inv = 1.0 / del;
            const double t = w[i] * inv;
            const double tw = w[i] * t;
            if (i <= j) {
                psi += tw;
                dpsi += t * t;
            } else {
                phi += tw;
                dphi += t * t;
            }
        }
        psi = rho * warp_sum(psi);
        dpsi = rho * warp_sum(dpsi);
        phi = rho * warp_sum(phi);
        dphi = rho * warp_sum(dphi);
        const double gval = 1.0 + psi + phi;
        if (gval == 0.0) {
            conv = true;
            break;
        }
        if (gval < 0.0)
            lo_bound = fmax(lo_bound, tau);
        else
            hi_bound = fmin(hi_bound, tau);
        const double errb = 8.0 * EPS * (2.0 + fabs(psi) + fabs(phi));
        if (fabs(gval) <= errb || (hi_bound - lo_bound) <= 4.0 * EPS * fmax(fabs(lo_bound), fabs(hi_bound))) {
            conv = true;
            break;
        }
        // two-pole model: C + b/(Dl - eta) + e/(Dh - eta)
        const double Dlo = dlo - tau, Dhi = dhi - tau;
        const double bcoef = dpsi * Dlo * Dlo;
        double eta;
        if (jr < k) {
            const double ecoef = dphi * Dhi * Dhi;
            const double Cc = gval - bcoef / Dlo - ecoef / Dhi;
            const double A1 = Cc * (Dlo + Dhi) + bcoef + ecoef;
            const double A0 = Dlo * Dhi * gval;
            if (Cc == 0.0) {
                eta = A0 / A1;
            } else {
                const double disc = sqrt(fmax(0.0, A1 * A1 - 4.0 * Cc * A0));
                const double q = -0.5 * (-A1 + copysign(disc, -A1));
                const double r1 = q / Cc, r2 = (q != 0.0) ? A0 / q : 0.0;
                // the root inside (Dlo, Dhi)
                eta = (r1 > Dlo && r1 < Dhi) ? r1 : r2;
            }
        } else {
            const double Cc = gval - bcoef / Dlo;
            eta = (Cc > 0.0) ? Dlo + bcoef / Cc : 0.5 * (lo_bound + hi_bound) - tau;
        }
        double tnew = tau + eta;
        if (!(tnew > lo_bound && tnew < hi_bound) || !isfinite(tnew))
            tnew = 0.5 * (lo_bound + hi_bound);
        if (tnew == tau) {
            conv = true;
            break;
        }
        tau = tnew;
    }
    if (!conv && lane == 0) dev_fail(status, CUEV_ERR_CONVERGENCE, g);
    for (int i = lane; i < k; i += 32) Delta[i] = (dl[i] - dorg) - tau;
    if (lane == 0) a.lam[off + j] = dorg + tau;
}

// Loewner weights: what_i = sign(w_i) sqrt(-Delta_ii prod_{j != i} Delta_ij / (d_i - d_j))
__global__ void dc_lowner_kernel(const MergeDesc *__restrict__ descs, int count, int n,
                                 const double *__restrict__ Dl, DcArrays a) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const int mi = find_merge(descs, count, g);
    const MergeDesc md = descs[mi];
    const int i = g - md.off;
    const int k = a.info[mi * MI_WORDS + MI_K];
    if (i >= k) return;
    const int off = md.off;
    const double *dl = a.dlam + off;
    const double *Delta = Dl + md.base;
    const double di = dl[i];
    double p = Delta[i + (long long)i * k];
    for (int j = 0; j < k; ++j) {
        if (j == i) continue;
        p *= Delta[i + (long long)j * k] / (di - dl[j]);
    }
    a.what[off + i] = copysign(sqrt(fmax(-p, 0.0)), a.w[off + i]);
}

// S_c[cpos(i), j] = what_i / Delta_ij, normalised per column; one warp per column j
__global__ void dc_svec_kernel(const MergeDesc *__restrict__ descs, int count, int n,
                               const double *__restrict__ Dl, double *__restrict__ S, DcArrays a) {
    const int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (g >= n) return;
    const int mi = find_merge(descs, count, g);
    const MergeDesc md = descs[mi];
    const int j = g - md.off;
    const int k = a.info[mi * MI_WORDS + MI_K];
    if (j >= k) return;
    const int off = md.off;
    const double *Delta = Dl + md.base + (long long)j * k;
    double *Sc = S + md.base + (long long)j * k;
    double ss = 0.0;
    for (int i = lane; i < k; i += 32) {
        const double v = a.what[off + i] / Delta[i];
        ss += v * v;
    }
    ss = warp_sum(ss);
    const double inv = 1.0 / sqrt(ss);
    for (int i = lane; i < k; i += 32) Sc[a.cpos[off + i]] = a.what[off + i] / Delta[i] * inv;
}

// GEMM descriptors: top rows use columns [0, ct1+ct2), bottom rows [ct1, ct1+ct2+ct3)
// also counts the merge's GEMM flops, 2 (n1 k (ct1 + ct2) + n2 k (ct2 + ct3)), into *flops
__global__ void dc_gemm_prep_kernel(const MergeDesc *__restrict__ descs, int count,
                                    double *Q2, double *S, double *Out, GemmArgs *args, DcArrays a,
                                    double *flops) {
    const int mi = blockIdx.x * blockDim.x + threadIdx.x;
    if (mi >= count) return;
    const MergeDesc md = descs[mi];
    const int *info = a.info + mi * MI_WORDS;
    const int k = info[MI_K], ct1 = info[MI_CT1], ct2 = info[MI_CT2], ct3 = info[MI_CT3];
    const int nm = md.nm, n1 = md.n1, n2 = nm - n1;
    GemmArgs top{}, bot{};
    top.m = (k > 0) ? n1 : 0;
    top.n = k;
    top.k = ct1 + ct2;
    top.A = Q2 + md.base;
    top.lda = nm;
    top.B = S + md.base;
    top.ldb = k > 0 ? k : 1;
    top.C = Out + md.base;
    top.ldc = nm;
    top.alpha = 1.0;
    top.splits = 1;
    bot = top;
    bot.m = (k > 0) ? n2 : 0;
    bot.k = ct2 + ct3;
    bot.A = Q2 + md.base + n1 + (long long)ct1 * nm;
    bot.B = S + md.base + ct1;
    bot.C = Out + md.base + n1;
    args[2 * mi] = top;
    args[2 * mi + 1] = bot;
    atomicAdd(flops, 2.0 * ((double)top.m * top.n * top.k + (double)bot.m * bot.n * bot.k));
}

// final order: roots (ascending) merged with the deflated eigenvalues (ranked here)
__global__ void dc_order_kernel(const MergeDesc *__restrict__ descs, double *__restrict__ D,
                                DcArrays a) {
    const MergeDesc md = descs[blockIdx.x];
    const int off = md.off;
    const int *info = a.info + blockIdx.x * MI_WORDS;
    const int k = info[MI_K], nd = info[MI_ND];
    const double *lam = a.lam + off;
    const double *dv = a.dval + off;
    // deflated: rank among deflated (ties by index) + roots strictly smaller
    for (int t = threadIdx.x; t < nd; t += blockDim.x) {
        const double x = dv[t];
        int r = 0;
        for (int u = 0; u < nd; ++u) {
            const double y = dv[u];
            r += (y < x) || (y == x && u < t);
        }
        const int pos = r + lower_bound_d(lam, k, x);
        a.newd[off + pos] = x;
        a.src[off + pos] = k + t;
    }
    // roots: index + deflated values <= root
    for (int j = threadIdx.x; j < k; j += blockDim.x) {
        const double x = lam[j];
        int c = 0;
        for (int u = 0; u < nd; ++u) c += dv[u] <= x;
        const int pos = j + c;
        a.newd[off + pos] = x;
        a.src[off + pos] = j;
    }
    __syncthreads();
    for (int p = threadIdx.x; p < md.nm; p += blockDim.x) D[off + p] = a.newd[off + p];
}

// Q(off + r, off + p) = source column src(p): GEMM output (src < k) or deflated (src >= k)
__global__ void dc_permute_kernel(const MergeDesc *__restrict__ descs, double *__restrict__ Q,
                                  long long ldq, const double *__restrict__ Out,
                                  const double *__restrict__ Q2, DcArrays a) {
    const MergeDesc md = descs[blockIdx.z];
    const int nm = md.nm, off = md.off;
    const int p = blockIdx.y;
    if (p >= nm) return;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nm) return;
    const int s = a.src[off + p];
    const double v = (s < a.info[blockIdx.z * MI_WORDS + MI_K]) ? Out[md.base + r + (long long)s * nm]
                                                               : Q2[md.base + r + (long long)s * nm];
    Q[(off + r) + (long long)(off + p) * ldq] = v;
}

} // namespace

int tridi_dc(Workspace *ws, const double *d, const double *e, double *eval, double *evec) {
    const int n = ws->n;
    cudaStream_t st = ws->stream;
    if (n <= 0) return CUEV_OK;
    CUEV_TRY(cudaMemsetAsync(ws->dc_flops, 0, sizeof(double), st));
    const long long ldq = n;

    // device scratch carve-up
    DcArrays a{};
    {
        double *v = ws->dc_vec;
        double **dv[] = {&a.E, &a.z, &a.dsort, &a.zsort, &a.dlam, &a.w, &a.lam, &a.what,
                         &a.dval, &a.rc, &a.rs, &a.newd, &a.scale};
        for (double **p : dv) {
            *p = v;
            v += n;
        }
        int *iv = ws->dc_int;
        int **ip[] = {&a.perm, &a.tsort, &a.ndcol, &a.ndtyp, &a.cpos, &a.dcol, &a.rp, &a.rq, &a.src};
        for (int **p : ip) {
            *p = iv;
            iv += n;
        }
        a.info = iv; // MI_WORDS per merge (<= n/32 merges per level)
    }

    // split tree (host): every part is halved while the largest exceeds LEAF_MAX
    std::vector<std::vector<int2>> levels;
    levels.push_back({make_int2(0, n)});
    while (levels.back().back().y > LEAF_MAX) {
        std::vector<int2> nxt;
        for (auto p : levels.back()) {
            nxt.push_back(make_int2(p.x, p.y / 2));
            nxt.push_back(make_int2(p.x + p.y / 2, p.y - p.y / 2));
        }
        levels.push_back(nxt);
    }
    const std::vector<int2> &leaves = levels.back();

    // merge descriptors for all levels, uploaded once (leaf list first)
    std::vector<MergeDesc> all;
    std::vector<int> lvl_start, lvl_count, lvl_maxm, lvl_maxnm;
    for (int L = (int)levels.size() - 2; L >= 0; --L) {
        lvl_start.push_back((int)all.size());
        long long base = 0;
        int maxm = 0, maxnm = 0;
        for (auto p : levels[L]) {
            MergeDesc md{p.x, p.y, p.y / 2, 0, base};
            base += (long long)p.y * p.y;
            maxm = std::max(maxm, std::max(md.n1, md.nm - md.n1));
            maxnm = std::max(maxnm, md.nm);
            all.push_back(md);
        }
        lvl_count.push_back((int)levels[L].size());
        lvl_maxm.push_back(maxm);
        lvl_maxnm.push_back(maxnm);
    }
    const size_t leaf_bytes = leaves.size() * sizeof(int2);
    const size_t desc_bytes = all.size() * sizeof(MergeDesc);
    if (leaf_bytes + desc_bytes > ws->dc_gemm_args_cap * sizeof(GemmArgs) / 2 ||
        2 * (size_t)(levels.size() > 1 ? levels[levels.size() - 2].size() : 1) >
            (size_t)ws->dc_gemm_args_cap / 2) {
        set_last_message("tridi_dc: descriptor space too small");
        return CUEV_ERR_INVALID;
    }
    // descriptor memory: second half of the GEMM-args area
    char *dbase = (char *)(ws->dc_gemm_args + ws->dc_gemm_args_cap / 2);
    int2 *d_leaves = (int2 *)dbase;
    MergeDesc *d_descs = (MergeDesc *)(dbase + align256(leaf_bytes));
    std::vector<char> hbuf(align256(leaf_bytes) + desc_bytes);
    memcpy(hbuf.data(), leaves.data(), leaf_bytes);
    if (desc_bytes) memcpy(hbuf.data() + align256(leaf_bytes), all.data(), desc_bytes);
    CUEV_TRY(cudaMemcpyAsync(dbase, hbuf.data(), hbuf.size(), cudaMemcpyHostToDevice, st));

    // scale, clear Q, leaves
    dc_norm_kernel<<<1, 1024, 0, st>>>(d, e, n, a.scale, ws->status); note_launch();
    dc_scale_in_kernel<<<std::max(1, std::min(1024, div_up(n, 256))), 256, 0, st>>>(d, e, eval,
                                                                                   a.E, n, a.scale); note_launch();
    CUEV_TRY(cudaMemsetAsync(evec, 0, sizeof(double) * (size_t)n * n, st));
    dc_leaf_kernel<<<(int)leaves.size(), 32, 0, st>>>(d_leaves, eval, a.E, evec, ldq, n,
                                                      ws->status); note_launch();
    CUEV_TRY(cudaGetLastError());

    double *Q2 = ws->dc_Q2, *Dl = ws->dc_S, *S = ws->dc_T;
    for (size_t li = 0; li < lvl_start.size(); ++li) {
        const int cnt = lvl_count[li];
        const MergeDesc *dd = d_descs + lvl_start[li];
        const int maxnm = lvl_maxnm[li];
        dc_deflate_kernel<<<cnt, DF_THREADS, 0, st>>>(dd, eval, evec, ldq, a); note_launch();
        dc_rotate_kernel<<<dim3(div_up(maxnm, 128), cnt), 128, 0, st>>>(dd, evec, ldq, Q2, a); note_launch();
        dc_secular_kernel<<<div_up(n * 32, 256), 256, 0, st>>>(dd, cnt, n, Dl, a, ws->status); note_launch();
        dc_lowner_kernel<<<div_up(n, 256), 256, 0, st>>>(dd, cnt, n, Dl, a); note_launch();
        dc_svec_kernel<<<div_up(n * 32, 256), 256, 0, st>>>(dd, cnt, n, Dl, S, a); note_launch();
        // Delta is dead now: the GEMM output goes to its region
        dc_gemm_prep_kernel<<<div_up(cnt, 128), 128, 0, st>>>(dd, cnt, Q2, S, Dl, ws->dc_gemm_args,
                                                              a, ws->dc_flops); note_launch();
        CUEV_TRY(cudaGetLastError());
        CUEV_CHECK_STATUS(gemm_batched_launch(ws->dc_gemm_args, 2 * cnt, lvl_maxm[li], maxnm, 0, 0,
                                              st));
        dc_order_kernel<<<cnt, 512, 0, st>>>(dd, eval, a); note_launch();
        dc_permute_kernel<<<dim3(div_up(maxnm, 128), maxnm, cnt), 128, 0, st>>>(dd, evec, ldq, Dl,
                                                                               Q2, a); note_launch();
        CUEV_TRY(cudaGetLastError());
    }
    dc_scale_out_kernel<<<std::max(1, std::min(1024, div_up(n, 256))), 256, 0, st>>>(eval, n,
                                                                                    a.scale); note_launch();
    CUEV_TRY(cudaGetLastError());
    return CUEV_OK;
}

} // namespace cuev
