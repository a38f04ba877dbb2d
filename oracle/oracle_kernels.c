/*
 * oracle_kernels.c — TEST INFRASTRUCTURE ONLY (the oracle).  Plain-C restatement of the
 * reference's sequential bulge chasing and BC-Back, used by tests/, smoke() and bench.py's CPU
 * baseline to check the CUDA library.  Never linked into or called by the product.
 *
 * Follows the reference (paths relative to the cuEV project):
 *   householder      src/cuda/bulge.cu:64-90   unit w, H = I - 2 w w^T, beta = -sign(x0)||x||
 *   bc_apply_step    src/cuda/bulge.cu:100-147 p = 2 A w over [cq, hi], kappa = w^T p,
 *                                              y = p - kappa w, A -= w y^T + y w^T in the band
 *   bc_chase_kernel  src/cuda/bulge.cu:167-216 hop geometry, U[:, s] storage
 *   bc_extract       src/cuda/bulge.cu:219-224 d = B[0, :], e = B[1, :]
 *   bc_back          src/cuda/backtransform.cu:58-62 (Q_b M = reflectors applied in reverse)
 * Executed sequentially (one sweep after the other), i.e. the semantics the GPU wavefront must
 * reproduce.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

static double band_sym(const double *B, int i, int j, int ldb) {
    if (i < j) {
        int t = i;
        i = j;
        j = t;
    }
    return B[(i - j) + (long)j * ldb];
}

/* Packed band B (2b x n, ld 2b) -> tridiagonal d (n), e (n-1); reflectors in U (ld ldu). */
void oracle_bc_chase(double *B, int n, int b, double *U, long ldu, double *d, double *e) {
    const int ldb = 2 * b;
    double *x = (double *)malloc(sizeof(double) * (size_t)(b + 1));
    double *p = (double *)malloc(sizeof(double) * (size_t)(3 * b + 2));
    double *sw = (double *)malloc(sizeof(double) * (size_t)(3 * b + 2));
    double *y = (double *)malloc(sizeof(double) * (size_t)(3 * b + 2));
    for (int s = 0; s < n - 2; ++s) {
        for (int c = s;; c = (c == s) ? s + 1 : c + b) {
            int r0, r1, cq;
            if (c == s) {
                r0 = s + 1;
                r1 = (s + b < n - 1) ? s + b : n - 1;
                cq = s;
            } else {
                if (c + b >= n) break;
                r0 = c + b;
                r1 = (c + 2 * b - 1 < n - 1) ? c + 2 * b - 1 : n - 1;
                cq = c;
            }
            const int L = r1 - r0 + 1;
            const int lo = cq;
            const int hi = (r1 + b < n - 1) ? r1 + b : n - 1;
            const int W = hi - lo + 1;
            /* reflector */
            double ss = 0.0;
            for (int t = 0; t < L; ++t) {
                x[t] = band_sym(B, r0 + t, cq, ldb);
                ss += x[t] * x[t];
            }
            if (ss == 0.0) {
                for (int t = 0; t < L; ++t) x[t] = 0.0;
            } else {
                const double a0 = x[0];
                const double beta = -((a0 >= 0.0) ? 1.0 : -1.0) * sqrt(ss);
                const double v0 = a0 - beta;
                const double inv = 1.0 / sqrt(v0 * v0 + (ss - a0 * a0));
                x[0] = v0;
                for (int t = 0; t < L; ++t) x[t] *= inv;
            }
            /* p = 2 A w, sw = w on the window rows */
            for (int idx = 0; idx < W; ++idx) {
                const int i = lo + idx;
                double acc = 0.0;
                for (int t = 0; t < L; ++t) acc += band_sym(B, i, r0 + t, ldb) * x[t];
                p[idx] = 2.0 * acc;
                sw[idx] = (i >= r0 && i <= r1) ? x[i - r0] : 0.0;
            }
            double kappa = 0.0;
            for (int t = 0; t < L; ++t) kappa += x[t] * p[(r0 + t) - lo];
            for (int idx = 0; idx < W; ++idx) y[idx] = p[idx] - kappa * sw[idx];
            /* rank-2 update inside the stored band */
            for (int j = lo; j <= hi; ++j) {
                const double wj = sw[j - lo], yj = y[j - lo];
                for (int dd = 0; dd < ldb; ++dd) {
                    const int i = j + dd;
                    if (i > hi) break;
                    const double upd = sw[i - lo] * yj + y[i - lo] * wj;
                    if (upd != 0.0) B[dd + (long)j * ldb] -= upd;
                }
            }
            for (int t = 0; t < L; ++t) U[(r0 + t) + (long)s * ldu] = x[t];
        }
    }
    for (int i = 0; i < n; ++i) {
        d[i] = B[(long)i * ldb];
        if (i < n - 1) e[i] = B[1 + (long)i * ldb];
    }
    free(x);
    free(p);
    free(sw);
    free(y);
}

/* M (n x ncols, ld ldm) <- Q_b M: reflectors (s, h) applied from the last generated to the
 * first.  Hop h of sweep s covers rows [s+1+hb, min(s+(h+1)b, n-1)] of U[:, s]. */
void oracle_bc_back(const double *U, long ldu, double *M, long ldm, int n, int ncols, int b) {
#pragma omp parallel for schedule(static)
    for (int col = 0; col < ncols; ++col) {
        double *m = M + (long)col * ldm;
        for (int s = n - 3; s >= 0; --s) {
            for (int r0 = s + 1; r0 <= n - 1; r0 += b) {
                const int r1 = (r0 + b - 1 < n - 1) ? r0 + b - 1 : n - 1;
                const double *w = U + (long)s * ldu;
                double dot = 0.0;
                for (int i = r0; i <= r1; ++i) dot += w[i] * m[i];
                dot *= 2.0;
                for (int i = r0; i <= r1; ++i) m[i] -= dot * w[i];
            }
        }
    }
}
