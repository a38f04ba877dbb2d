// Batched eigensolver for stacks of medium symmetric matrices (64 < n <= 512), one CTA of 512
// threads per matrix (persistent over the stack).  The reference has no batched entry; the small
// sizes (n <= 64) run the shared-memory Jacobi of batched_small.cu.
//
// Per matrix, in a per-CTA global workspace (three n x n FP64 buffers, L2/HBM resident):
//  1. Householder tridiagonalisation of the lower triangle (unblocked, LAPACK's dsytd2 scheme):
//     for column j, x = A(j+1:n, j), beta = -sign(x0) ||x||, tau = (beta - x0) / beta,
//     v = x / (x0 - beta) with v0 = 1; p = tau A22 v, w = p - (tau/2)(p^T v) v,
//     A22 -= v w^T + w v^T; thread t owns row j+1+t, so every column access is coalesced.
//  2. Implicit QL with Wilkinson shifts on (d, e) (Bowdler, Martin, Reinsch, Wilkinson,
//     "The QR and QL algorithms for symmetric matrices", Numer. Math. 11 (1968); EISPACK tql2):
//     thread 0 generates each sweep's Givens rotations from (d, e) in shared memory, then every
//     thread applies the sweep to its own row of Z (column-major, so rotating columns i, i+1 is a
//     coalesced access across threads), carrying the running column through the sweep.
//  3. Z is transposed through shared-memory tiles, then the reflectors are applied in reverse
//     order, Z <- H_j Z, with one thread per column (coalesced in the transposed layout).
//  4. Eigenpairs are ranked (ties by index) and written in ascending order through a permuting
//     tiled transpose.
// QL sweeps are bounded (60 per eigenvalue, then CUEV_ERR_CONVERGENCE in the status word).
#include "common.cuh"

#include <algorithm>
#include <mutex>

namespace cuev {
namespace {

constexpr int BMID_NT = 512;
constexpr int BMID_MAXN = 512;
constexpr int BMID_MAX_ITERS = 60;

__device__ __forceinline__ double bmid_block_sum(double v, double *red) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads(); // red[] may still be read by the previous reduction
    if (lane == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < BMID_NT / 32; ++q) s += red[q];
    return s; // every thread, same order: identical result everywhere
}

__device__ __forceinline__ double bmid_block_max(double v, double *red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < BMID_NT / 32; ++q) s = fmax(s, red[q]);
    return s;
}

// dst (row-major view: dst[r n + c]) = src column-major (src[r + c n]), n x n, through 32 x 33
// shared-memory tiles.
__device__ void bmid_transpose(const double *__restrict__ src, double *__restrict__ dst, int n,
                               double (*tile)[33]) {
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5; // 32 x 16 threads
    for (int c0 = 0; c0 < n; c0 += 32)
        for (int r0 = 0; r0 < n; r0 += 32) {
            for (int yy = ty; yy < 32; yy += BMID_NT / 32) { // read columns c0+yy, rows r0+tx
                const int r = r0 + tx, c = c0 + yy;
                tile[yy][tx] = (r < n && c < n) ? src[r + (size_t)c * n] : 0.0;
            }
            __syncthreads();
            for (int yy = ty; yy < 32; yy += BMID_NT / 32) { // write rows r0+yy, columns c0+tx
                const int r = r0 + yy, c = c0 + tx;
                if (r < n && c < n) dst[(size_t)r * n + c] = tile[tx][yy];
            }
            __syncthreads();
        }
}

__global__ void __launch_bounds__(BMID_NT, 1)
    batched_mid_kernel(const double *__restrict__ A, int n, int batch, double *__restrict__ eval,
                       double *__restrict__ evec, double *__restrict__ work,
                       int *__restrict__ status) {
    __shared__ double sd[BMID_MAXN], sE[BMID_MAXN], stau[BMID_MAXN];
    __shared__ double sv[BMID_MAXN], sw[BMID_MAXN], scs[BMID_MAXN], ssn[BMID_MAXN];
    __shared__ double red[BMID_NT / 32];
    __shared__ double tile[32][33];
    __shared__ int s_m, s_ilow, s_fail;
    __shared__ int srank[BMID_MAXN];
    const int t = threadIdx.x;
    const size_t nn = (size_t)n * n;
    double *Aw = work + (size_t)blockIdx.x * 3 * nn; // reflectors below the subdiagonal
    double *Zc = Aw + nn;                            // QL eigenvectors, column-major
    double *Zr = Zc + nn;                            // the same, row-major (back-transform)

    for (int mat = blockIdx.x; mat < batch; mat += gridDim.x) {
        const double *Ab = A + (size_t)mat * nn;
        // ---- symmetric copy of the lower triangle (every stored entry is read once as itself)
        int bad = 0;
        for (size_t idx = t; idx < nn; idx += BMID_NT) {
            const int i = (int)(idx % n), j = (int)(idx / n);
            const double a = i >= j ? Ab[idx] : Ab[j + (size_t)i * n];
            bad |= !isfinite(a);
            Aw[idx] = a;
        }
        if (t == 0) s_fail = 0;
        if (__syncthreads_or(bad)) { // uniform: NaN or Inf in the input, outputs set to NaN
            const double qnan = __longlong_as_double(0x7ff8000000000000LL);
            for (size_t idx = t; idx < nn; idx += BMID_NT) evec[(size_t)mat * nn + idx] = qnan;
            if (t < n) eval[(size_t)mat * n + t] = qnan;
            if (t == 0) dev_fail(status, CUEV_ERR_NONFINITE, mat);
            continue;
        }

        // ---- 1. tridiagonalisation
        for (int j = 0; j + 2 < n; ++j) {
            const int L = n - j - 1;
            double *col = Aw + (size_t)j * n + j + 1; // x = col[0 .. L)
            const double x = t < L ? col[t] : 0.0;
            if (t == 0) sv[0] = x;
            double sig = bmid_block_sum((t >= 1 && t < L) ? x * x : 0.0, red);
            const double alpha = sv[0]; // written before the reduction's barriers
            double nrm = sqrt(alpha * alpha + sig);
            if (!(sig > 1e-280 && nrm < 1e280)) {
                // squares out of range (uniform branch: sig is the same everywhere): redo the
                // norm scaled by max |x|
                const double xm = bmid_block_max(t < L ? fabs(x) : 0.0, red);
                if (xm > 0.0 && xm <= 1.79e308) {
                    const double xs = x / xm, as = alpha / xm;
                    sig = bmid_block_sum((t >= 1 && t < L) ? xs * xs : 0.0, red);
                    nrm = xm * sqrt(as * as + sig);
                } else {
                    sig = xm > 0.0 ? xm : 0.0; // zero column, or non-finite (left to QL's limit)
                    nrm = xm;
                }
            }
            double tau = 0.0, beta = alpha, vt = (t == 0) ? 1.0 : 0.0;
            if (sig != 0.0) {
                beta = -copysign(nrm, alpha);
                tau = (beta - alpha) / beta;
                vt = (t == 0) ? 1.0 : x / (alpha - beta);
            }
            __syncthreads(); // everyone has read sv[0]
            if (t < L) {
                sv[t] = vt;
                col[t] = (t == 0) ? beta : vt; // e_j on the subdiagonal, v below it
            }
            __syncthreads();
            // p = tau A22 v (thread t: row j+1+t)
            const double *A22 = Aw + (size_t)(j + 1) * n + j + 1;
            double pt = 0.0;
            if (t < L) {
                double p0 = 0.0, p1 = 0.0;
                int k = 0;
                for (; k + 1 < L; k += 2) {
                    p0 = fma(A22[t + (size_t)k * n], sv[k], p0);
                    p1 = fma(A22[t + (size_t)(k + 1) * n], sv[k + 1], p1);
                }
                if (k < L) p0 = fma(A22[t + (size_t)k * n], sv[k], p0);
                pt = tau * (p0 + p1);
            }
            const double pv = bmid_block_sum(t < L ? pt * vt : 0.0, red);
            const double wt = pt - 0.5 * tau * pv * vt;
            if (t < L) sw[t] = wt;
            __syncthreads();
            if (t < L && tau != 0.0) {
                double *Ar = Aw + (size_t)(j + 1) * n + j + 1 + t;
                for (int k = 0; k < L; ++k)
                    Ar[(size_t)k * n] -= vt * sw[k] + wt * sv[k];
            }
            if (t == 0) {
                sd[j] = Aw[(size_t)j * n + j];
                sE[j] = beta;
                stau[j] = tau;
            }
            __syncthreads();
        }
        if (t == 0) {
            if (n >= 2) {
                sd[n - 2] = Aw[(size_t)(n - 2) * n + n - 2];
                sE[n - 2] = Aw[(size_t)(n - 2) * n + n - 1];
                stau[n - 2] = 0.0;
            }
            sd[n - 1] = Aw[(size_t)(n - 1) * n + n - 1];
            sE[n - 1] = 0.0;
        }
        for (size_t idx = t; idx < nn; idx += BMID_NT)
            Zc[idx] = (idx % n == idx / n) ? 1.0 : 0.0;
        __syncthreads();

        // ---- 2. implicit QL, rotations applied to the rows of Zc
        const double eps = 2.220446049250313e-16;
        if (t == 0)
            for (int i = 0; i < n; ++i)
                if (!isfinite(sd[i]) || !isfinite(sE[i])) s_fail = 2; // overflow in the reduction
        __syncthreads();
        for (int l = (s_fail ? n : 0); l < n; ++l) {
            for (int iter = 0;; ++iter) {
                if (t == 0) {
                    int m = l;
                    while (m < n - 1) {
                        const double dd = fabs(sd[m]) + fabs(sd[m + 1]);
                        if (fabs(sE[m]) <= eps * dd || fabs(sE[m]) < 2.2250738585072014e-308)
                            break;
                        ++m;
                    }
                    if (m == l) {
                        s_m = -1;
                    } else if (iter >= BMID_MAX_ITERS) {
                        s_m = -1;
                        s_fail = 1; // stop: the matrix is reported as failed
                    } else {
                        double g = (sd[l + 1] - sd[l]) / (2.0 * sE[l]);
                        double r = hypot(g, 1.0);
                        g = sd[m] - sd[l] + sE[l] / (g + copysign(r, g));
                        double s = 1.0, c = 1.0, p = 0.0;
                        int i = m - 1, ilow = l;
                        bool underflow = false;
                        for (; i >= l; --i) {
                            const double f = s * sE[i], b = c * sE[i];
                            r = hypot(f, g);
                            sE[i + 1] = r;
                            if (r == 0.0) { // split: the rotations m-1 .. i+1 stand
                                sd[i + 1] -= p;
                                sE[m] = 0.0;
                                underflow = true;
                                ilow = i + 1;
                                break;
                            }
                            s = f / r;
                            c = g / r;
                            g = sd[i + 1] - p;
                            r = (sd[i] - g) * s + 2.0 * c * b;
                            p = s * r;
                            sd[i + 1] = g + p;
                            g = c * r - b;
                            scs[i] = c;
                            ssn[i] = s;
                        }
                        if (!underflow) {
                            sd[l] -= p;
                            sE[l] = g;
                            sE[m] = 0.0;
                        }
                        s_m = m;
                        s_ilow = ilow;
                    }
                }
                __syncthreads();
                const int m = s_m, ilow = s_ilow, fail = s_fail;
                __syncthreads(); // thread 0 rewrites s_m for the next sweep
                if (fail) l = n;  // uniform: leave both loops
                if (m < 0) break; // uniform
                if (t < n) {
                    // the sweep's rotations, highest pair first, on row t: columns m, m-1, ...;
                    // loads run 8 columns ahead of the stores (disjoint addresses)
                    double *zr = Zc + t;
                    double carry = zr[(size_t)m * n];
                    int i = m - 1;
                    for (; i - 7 >= ilow; i -= 8) {
                        double a[8];
#pragma unroll
                        for (int q = 0; q < 8; ++q) a[q] = zr[(size_t)(i - q) * n];
#pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            const double c = scs[i - q], s = ssn[i - q];
                            zr[(size_t)(i - q + 1) * n] = s * a[q] + c * carry;
                            carry = c * a[q] - s * carry;
                        }
                    }
                    for (; i >= ilow; --i) {
                        const double a = zr[(size_t)i * n];
                        const double c = scs[i], s = ssn[i];
                        zr[(size_t)(i + 1) * n] = s * a + c * carry;
                        carry = c * a - s * carry;
                    }
                    zr[(size_t)ilow * n] = carry;
                }
                __syncthreads();
            }
        }
        if (t == 0 && s_fail)
            dev_fail(status, s_fail == 2 ? CUEV_ERR_NONFINITE : CUEV_ERR_CONVERGENCE, mat);

        // ---- 3. back-transform Z <- H_0 ... H_(n-3) Z on the row-major copy
        bmid_transpose(Zc, Zr, n, tile);
        for (int j = n - 3; j >= 0; --j) {
            const int L = n - j - 1;
            const double tau = stau[j];
            if (tau == 0.0) continue; // uniform
            const double *vcol = Aw + (size_t)j * n + j + 1; // v0 = 1 (row j+1 holds e_j)
            if (t < L) sv[t] = (t == 0) ? 1.0 : vcol[t];
            __syncthreads();
            if (t < n) {
                double *zc = Zr + (size_t)(j + 1) * n + t; // column t, rows j+1 ..
                double z0 = 0.0, z1 = 0.0;
                int k = 0;
                for (; k + 1 < L; k += 2) {
                    z0 = fma(sv[k], zc[(size_t)k * n], z0);
                    z1 = fma(sv[k + 1], zc[(size_t)(k + 1) * n], z1);
                }
                if (k < L) z0 = fma(sv[k], zc[(size_t)k * n], z0);
                const double z = tau * (z0 + z1);
                for (k = 0; k < L; ++k) zc[(size_t)k * n] -= sv[k] * z;
            }
            __syncthreads();
        }

        // ---- 4. ascending order: rank, then a permuting transpose into evec
        if (t < n) {
            const double li = sd[t];
            int rank = 0;
            for (int q = 0; q < n; ++q) {
                const double lq = sd[q];
                rank += (lq < li) || (lq == li && q < t);
            }
            srank[t] = rank;
            eval[(size_t)mat * n + rank] = li;
        }
        __syncthreads();
        double *V = evec + (size_t)mat * nn;
        {
            const int tx = t & 31, ty = t >> 5;
            for (int c0 = 0; c0 < n; c0 += 32)
                for (int r0 = 0; r0 < n; r0 += 32) {
                    for (int yy = ty; yy < 32; yy += BMID_NT / 32) { // Zr rows r0+yy, cols c0+tx
                        const int r = r0 + yy, c = c0 + tx;
                        tile[yy][tx] = (r < n && c < n) ? Zr[(size_t)r * n + c] : 0.0;
                    }
                    __syncthreads();
                    for (int yy = ty; yy < 32; yy += BMID_NT / 32) { // column c0+yy, rows r0+tx
                        const int r = r0 + tx, c = c0 + yy;
                        if (r < n && c < n) V[r + (size_t)srank[c] * n] = tile[tx][yy];
                    }
                    __syncthreads();
                }
        }
    }
}

// per-device workspace (calls are serialised by the batched entry in batched_small.cu)
std::mutex g_bm_mu;
void *g_bm_buf[64] = {nullptr};
size_t g_bm_bytes[64] = {0};

} // namespace

// Stacks of 64 < n <= 512 matrices, launched on st (called by batched_eigh_d, which validates
// the arguments, owns the status word and synchronises).
int batched_eigh_mid(const double *A, int n, int batch, double *eval, double *evec, int *status,
                     cudaStream_t st) {
    if (n <= 0 || n > BMID_MAXN || batch <= 0) return CUEV_ERR_INVALID;
    int dev = 0;
    CUEV_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return CUEV_ERR_INVALID;
    const int grid = std::min(batch, num_sms());
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
    batched_mid_kernel<<<grid, BMID_NT, 0, st>>>(A, n, batch, eval, evec, (double *)g_bm_buf[dev],
                                                 status);
    note_launch();
    CUEV_TRY(cudaGetLastError());
    return CUEV_OK;
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
