/* Forwards the eight LAPACK symbols the reference's host D&C calls (src/cuda/tridi.cu:40-53) to
 * the copies exported, with a scipy_ prefix, by scipy's bundled OpenBLAS.  Test infrastructure:
 * only used to build the reference itself into oracle/_ref for comparison runs. */
#include <stddef.h>

#define FWD_STEQR(T, P)                                                                            \
    void P##steqr_(const char *c, const int *n, T *d, T *e, T *z, const int *ldz, T *w, int *info); \
    void scipy_##P##steqr_(const char *, const int *, T *, T *, T *, const int *, T *, int *, size_t); \
    void P##steqr_(const char *c, const int *n, T *d, T *e, T *z, const int *ldz, T *w, int *info) { \
        scipy_##P##steqr_(c, n, d, e, z, ldz, w, info, (size_t)1);                                  \
    }
FWD_STEQR(double, d)
FWD_STEQR(float, s)

#define FWD_LAED2(T, P)                                                                            \
    void scipy_##P##laed2_(int *, const int *, const int *, T *, T *, const int *, int *, T *, T *, \
                           T *, T *, T *, int *, int *, int *, int *, int *);                      \
    void P##laed2_(int *k, const int *n, const int *n1, T *d, T *q, const int *ldq, int *indxq,    \
                   T *rho, T *z, T *dl, T *w, T *q2, int *ix, int *ixc, int *ixp, int *ct,         \
                   int *info) {                                                                    \
        scipy_##P##laed2_(k, n, n1, d, q, ldq, indxq, rho, z, dl, w, q2, ix, ixc, ixp, ct, info);  \
    }
FWD_LAED2(double, d)
FWD_LAED2(float, s)

#define FWD_LAED4(T, P)                                                                            \
    void scipy_##P##laed4_(const int *, const int *, const T *, const T *, T *, const T *, T *,    \
                           int *);                                                                 \
    void P##laed4_(const int *n, const int *i, const T *d, const T *z, T *delta, const T *rho,     \
                   T *dlam, int *info) {                                                           \
        scipy_##P##laed4_(n, i, d, z, delta, rho, dlam, info);                                      \
    }
FWD_LAED4(double, d)
FWD_LAED4(float, s)

#define FWD_LAMRG(T, P)                                                                            \
    void scipy_##P##lamrg_(const int *, const int *, const T *, const int *, const int *, int *);  \
    void P##lamrg_(const int *n1, const int *n2, const T *a, const int *s1, const int *s2,        \
                   int *index) {                                                                   \
        scipy_##P##lamrg_(n1, n2, a, s1, s2, index);                                               \
    }
FWD_LAMRG(double, d)
FWD_LAMRG(float, s)
