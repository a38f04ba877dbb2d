// Stage 2: bulge chasing, packed band (width b) -> symmetric tridiagonal (d, e).
//
// Hop geometry and reflector convention follow the reference (src/cuda/bulge.cu:64-216,
// Wang et al. Algorithm 2): sweep s first reduces column s with a reflector on rows
// [s+1, s+b], then chases the bulge: hop c = s+1, s+1+b, ... reduces column c on rows
// [c+b, c+2b-1].  Each reflector is the unit vector w (H = I - 2 w w^T) with
// beta = -sign(x0) ||x||, and all reflectors of sweep s are stored contiguously in U[:, s].
//
// B200 design:
//  * one persistent CTA per in-flight sweep (grid-strided), launched cooperatively so that
//    every CTA is co-resident (the reference relies on an occupancy cap, bulge.cu:238-243);
//  * the packed band (2b x n doubles, 8-34 MB) lives in the 126 MB L2; all band reads use
//    ld.global.cg so no SM sees a stale L1 line of data another SM has just rewritten;
//  * hand-off between sweeps is acquire/release on prog[] with a BOUNDED wait (the reference
//    spins forever, bulge.cu:194-196); on timeout the kernel records CUEV_ERR_TIMEOUT and exits;
//  * the wavefront condition is derived from the packed-column footprint of a hop ([cq, r1]):
//    sweep s may run its hop once sweep s-1 has completed every hop that starts at or before
//    r1, i.e. prog[s-1] >= r1 - b + 1.  That is a two-hop lag instead of the reference's
//    four (prog >= c + 3b), which halves the pipeline fill.
//  * per hop the b x 3b strip of the symmetric window that the reflector touches is gathered
//    into shared memory once; each updated element (rank-2 H A H) goes straight back to the band
//    from the thread that computes it, with no barrier between update and write-back.
#include "solver.cuh"

#include <algorithm>
#include <climits>

namespace cuev {
namespace {

constexpr int BC_THREADS = 256;

template <int BW> struct ChaseSmem {
    double S[BW][3 * BW + 1]; // strip: S[k][ii] = A(lo + ii, r0 + k)
    double w[BW];             // reflector
    double p[3 * BW];         // p = 2 A w over the window rows
    double red[2];            // beta, kappa
};

template <int BW>
__global__ void __launch_bounds__(BC_THREADS)
    bc_chase_kernel(double *__restrict__ Bp, double *__restrict__ U, long long ldu, int n, int b,
                    int *prog, int *status) {
    constexpr int NT = BC_THREADS;
    constexpr int NLEFT = (BW * BW + NT - 1) / NT;    // left-block elements per thread
    constexpr int NLOW = (2 * BW * BW + NT - 1) / NT; // lower-part elements per thread
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ChaseSmem<BW> &sm = *reinterpret_cast<ChaseSmem<BW> *>(smem_raw);
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int ldb = 2 * b;
    const int nsweeps = n - 2;
    __shared__ int s_abort;

    for (int s = blockIdx.x; s < nsweeps; s += gridDim.x) {
        for (int hop = 0;; ++hop) {
            int cq, r0, r1;
            if (hop == 0) {
                cq = s, r0 = s + 1, r1 = min(s + b, n - 1);
            } else {
                const int c = s + 1 + (hop - 1) * b;
                if (c + b >= n) break;
                cq = c, r0 = c + b, r1 = min(c + 2 * b - 1, n - 1);
            }
            const int L = r1 - r0 + 1;
            const int lo = cq, hi = min(n - 1, r1 + b);
            const int W = hi - lo + 1;
            const int off = r0 - lo; // strip row of reflector row r0

            // ---- wait for sweep s-1 to finish every hop that starts at or before r1
            if (tid == 0) {
                int ok = 1;
                if (s > 0) {
                    const int need = r1 - b + 1;
                    const uint64_t t0 = global_ns();
                    const uint64_t limit = wait_limit_ns(status);
                    // the clock is read every 256 polls, or every poll under a short limit
                    const int every = limit < 1000000ull ? 0 : 255;
                    int spins = 0;
                    while (ld_acquire(&prog[s - 1]) < need) {
                        if ((++spins & every) == 0) {
                            if (global_ns() - t0 > limit ||
                                ld_acquire(&status[DEV_STATUS_CODE]) != 0) {
                                dev_fail(status, CUEV_ERR_TIMEOUT, s);
                                ok = 0;
                                break;
                            }
                        }
                    }
                }
                s_abort = !ok;
            }
            __syncthreads(); // thread 0's acquire + the barrier order the loads below
            if (s_abort) return;

            // ---- gather the strip S[k][ii] = A(lo+ii, r0+k), all loads in flight at once.
            // left block (rows above r0): packed column i, contiguous along k
            double vl[NLEFT], vw[NLOW];
#pragma unroll
            for (int q = 0; q < NLEFT; ++q) {
                const int idx = tid + q * NT;
                const int k = idx % BW, ii = idx / BW;
                const bool ok = (ii < off) && (k < L);
                const int i = lo + ii, j = r0 + k;
                vl[q] = ok ? __ldcg(&Bp[(j - i) + (long long)i * ldb]) : 0.0;
            }
            // rows r0..hi: packed column j (lower triangle only; the upper half of the
            // diagonal block follows by symmetry)
#pragma unroll
            for (int q = 0; q < NLOW; ++q) {
                const int idx = tid + q * NT;
                const int ii = off + idx % (2 * BW), k = idx / (2 * BW);
                const int i = lo + ii, j = r0 + k;
                const bool ok = (ii < W) && (k < L) && (i >= j);
                vw[q] = ok ? __ldcg(&Bp[(i - j) + (long long)j * ldb]) : 0.0;
            }
#pragma unroll
            for (int q = 0; q < NLEFT; ++q) {
                const int idx = tid + q * NT;
                const int k = idx % BW, ii = idx / BW;
                if (ii < off && k < L) sm.S[k][ii] = vl[q];
            }
#pragma unroll
            for (int q = 0; q < NLOW; ++q) {
                const int idx = tid + q * NT;
                const int ii = off + idx % (2 * BW), k = idx / (2 * BW);
                const int i = lo + ii, j = r0 + k;
                if (ii < W && k < L && i >= j) sm.S[k][ii] = vw[q];
            }
            __syncthreads();
            // upper part of the diagonal block by symmetry; Householder of x = S[0:L][0]
            for (int idx = tid; idx < BW * BW; idx += NT) {
                const int a = idx % BW, k = idx / BW; // row r0+a, column r0+k
                if (a < k && k < L) sm.S[k][off + a] = sm.S[a][off + k];
            }
            if (warp == 0) {
                double ss = 0.0;
                for (int k = lane; k < L; k += 32) {
                    const double v = sm.S[k][0];
                    ss += v * v;
                }
                ss = warp_sum(ss);
                const double x0 = sm.S[0][0];
                if (ss == 0.0) {
                    for (int k = lane; k < L; k += 32) sm.w[k] = 0.0;
                    if (lane == 0) sm.red[0] = 0.0;
                } else {
                    const double sgn = (x0 >= 0.0) ? 1.0 : -1.0;
                    const double beta = -sgn * sqrt(ss);
                    const double v0 = x0 - beta;
                    const double inv = 1.0 / sqrt(v0 * v0 + (ss - x0 * x0));
                    for (int k = lane; k < L; k += 32) sm.w[k] = (k == 0 ? v0 : sm.S[k][0]) * inv;
                    if (lane == 0) sm.red[0] = beta;
                }
            }
            __syncthreads();

            // ---- p = 2 A w over the window rows
            for (int ii = tid; ii < W; ii += NT) {
                // four chains: this dot product is on the hop's critical path
                double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
                int k = 0;
                for (; k + 3 < L; k += 4) {
                    a0 = fma(sm.S[k][ii], sm.w[k], a0);
                    a1 = fma(sm.S[k + 1][ii], sm.w[k + 1], a1);
                    a2 = fma(sm.S[k + 2][ii], sm.w[k + 2], a2);
                    a3 = fma(sm.S[k + 3][ii], sm.w[k + 3], a3);
                }
                for (; k < L; ++k) a0 = fma(sm.S[k][ii], sm.w[k], a0);
                sm.p[ii] = 2.0 * ((a0 + a1) + (a2 + a3));
            }
            __syncthreads();
            // kappa = w^T p over the reflector rows (every warp computes it)
            double kl = 0.0;
            for (int k = lane; k < L; k += 32) kl += sm.w[k] * sm.p[off + k];
            const double kappa = warp_sum(kl);
            const double beta = sm.red[0];

            for (int k = tid; k < L; k += NT) U[(r0 + k) + (long long)s * ldu] = sm.w[k];

            // ---- rank-2 update A -= w_row y_col^T + y_row w_col^T with y = p - kappa w, each
            // element stored to the band straight from the thread that updates it (the strip is
            // gathered afresh by the next hop, so shared memory keeps the old values); the
            // reduced column is set exactly: A(r0, cq) = beta, A(r0+1:r1, cq) = 0.
            // left block (rows above r0, packed column i, contiguous along k)
#pragma unroll
            for (int q = 0; q < NLEFT; ++q) {
                const int idx = tid + q * NT;
                const int k = idx % BW, ii = idx / BW;
                if (ii >= off || k >= L) continue;
                double v;
                if (ii == 0) {
                    v = (k == 0) ? beta : 0.0;
                } else { // kr = ii - off < 0: w_row = 0
                    v = sm.S[k][ii] - sm.p[ii] * sm.w[k];
                }
                const int i = lo + ii, j = r0 + k;
                __stcg(&Bp[(j - i) + (long long)i * ldb], v);
            }
            // rows r0..hi, lower triangle (packed column j, contiguous along i)
#pragma unroll
            for (int q = 0; q < NLOW; ++q) {
                const int idx = tid + q * NT;
                const int ii = off + idx % (2 * BW), k = idx / (2 * BW);
                const int i = lo + ii, j = r0 + k;
                if (ii >= W || k >= L || i < j) continue;
                const int kr = ii - off;
                const double wr = kr < L ? sm.w[kr] : 0.0;
                const double wk = sm.w[k];
                const double yr = sm.p[ii] - kappa * wr;
                const double yc = sm.p[off + k] - kappa * wk;
                __stcg(&Bp[(i - j) + (long long)j * ldb], sm.S[k][ii] - (wr * yc + yr * wk));
            }

            // ---- publish: the barrier orders every thread's stores before thread 0's release
            // (release is cumulative over what thread 0 has observed through the barrier)
            __syncthreads();
            if (tid == 0) st_release(&prog[s], cq);
        }
        if (tid == 0) {
            __threadfence();
            st_release(&prog[s], INT_MAX);
        }
        __syncthreads();
    }
}

__global__ void bc_extract_kernel(const double *__restrict__ Bp, double *__restrict__ d,
                                  double *__restrict__ e, int n, int b) {
    const int ldb = 2 * b;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        d[i] = Bp[(long long)i * ldb];
        if (i < n - 1) e[i] = Bp[1 + (long long)i * ldb];
    }
}

template <int BW> int launch_chase(Workspace *ws, double *B) {
    const int n = ws->n, b = ws->b;
    const int nsweeps = n - 2;
    const size_t smem = sizeof(ChaseSmem<BW>);
    auto kern = bc_chase_kernel<BW>;
    CUEV_CHECK_STATUS(ensure_dyn_smem((const void *)kern, smem));
    int per_sm = 0;
    CUEV_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BC_THREADS, smem));
    const int cap = std::max(1, per_sm) * num_sms();
    int grid = std::max(1, std::min(nsweeps, cap));
    double *U = ws->U;
    long long ldu = n;
    int nn = n, bb = b;
    void *args[] = {&B, &U, &ldu, &nn, &bb, &ws->prog, &ws->status};
    note_launch();
    CUEV_TRY(cudaLaunchCooperativeKernel((void *)kern, dim3(grid), dim3(BC_THREADS), args, smem,
                                         ws->stream));
    return CUEV_OK;
}

} // namespace

int bc_chase(Workspace *ws, double *B, double *d, double *e) {
    const int n = ws->n, b = ws->b;
    CUEV_TRY(cudaMemsetAsync(ws->U, 0, sizeof(double) * (size_t)n * n, ws->stream));
    if (n > 2) {
        // prog = -1: no hop completed yet
        CUEV_TRY(cudaMemsetAsync(ws->prog, 0xFF, sizeof(int) * (size_t)n, ws->stream));
        if (b == 32)
            CUEV_CHECK_STATUS(launch_chase<32>(ws, B));
        else if (b == 64)
            CUEV_CHECK_STATUS(launch_chase<64>(ws, B));
        else
            return CUEV_ERR_INVALID;
    }
    if (n > 0) {
        bc_extract_kernel<<<std::max(1, std::min(1024, div_up(n, 256))), 256, 0, ws->stream>>>(
            B, d, e, n, b); note_launch();
        CUEV_TRY(cudaGetLastError());
    }
    return CUEV_OK;
}

} // namespace cuev
