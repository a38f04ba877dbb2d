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
//    into shared memory once, updated there (rank-2 H A H) and written back once.
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
    double y[3 * BW];         // y = p - kappa w
    double red[32];
};

template <int BW>
__global__ void __launch_bounds__(BC_THREADS)
    bc_chase_kernel(double *__restrict__ Bp, double *__restrict__ U, long long ldu, int n, int b,
                    int *prog, int *status) {
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
                    int spins = 0;
                    while (ld_acquire(&prog[s - 1]) < need) {
                        if ((++spins & 255) == 0) {
                            if (global_ns() - t0 > 2000000000ull ||
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
            __syncthreads();
            if (s_abort) return;
            __threadfence();

            // ---- gather the strip S[k][ii] = A(lo+ii, r0+k): rows above r0 (left block)
            // are stored in packed columns i (contiguous along k), the rest in packed column j.
            for (int idx = tid; idx < off * L; idx += BC_THREADS) {
                const int k = idx % L, ii = idx / L;
                const int i = lo + ii, j = r0 + k;
                sm.S[k][ii] = __ldcg(&Bp[(j - i) + (long long)i * ldb]);
            }
            for (int idx = tid; idx < (W - off) * L; idx += BC_THREADS) {
                const int ii = off + idx % (W - off), k = idx / (W - off);
                const int i = lo + ii, j = r0 + k;
                if (i >= j) sm.S[k][ii] = __ldcg(&Bp[(i - j) + (long long)j * ldb]);
            }
            __syncthreads();
            // upper part of the diagonal block by symmetry
            for (int idx = tid; idx < L * L; idx += BC_THREADS) {
                const int a = idx % L, k = idx / L; // row r0+a, column r0+k, a < k
                if (a < k) sm.S[k][off + a] = sm.S[a][off + k];
            }

            // ---- Householder of x = A(r0:r1, cq) = S[0:L][0]
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
            for (int ii = tid; ii < W; ii += BC_THREADS) {
                double acc = 0.0;
#pragma unroll 8
                for (int k = 0; k < L; ++k) acc += sm.S[k][ii] * sm.w[k];
                sm.p[ii] = 2.0 * acc;
            }
            __syncthreads();
            // kappa = w^T p (over the reflector rows)
            if (warp == 0) {
                double kl = 0.0;
                for (int k = lane; k < L; k += 32) kl += sm.w[k] * sm.p[off + k];
                kl = warp_sum(kl);
                if (lane == 0) sm.red[1] = kl;
            }
            __syncthreads();
            const double kappa = sm.red[1];
            for (int ii = tid; ii < W; ii += BC_THREADS) {
                const int k = ii - off;
                const double wr = (k >= 0 && k < L) ? sm.w[k] : 0.0;
                sm.y[ii] = sm.p[ii] - kappa * wr;
            }
            __syncthreads();

            // ---- rank-2 update of the strip: S -= w_row y_col^T + y_row w_col^T
            for (int idx = tid; idx < W * L; idx += BC_THREADS) {
                const int ii = idx % W, k = idx / W;
                const int kr = ii - off;
                const double wr = (kr >= 0 && kr < L) ? sm.w[kr] : 0.0;
                sm.S[k][ii] -= wr * sm.y[off + k] + sm.y[ii] * sm.w[k];
            }
            __syncthreads();
            // the reduced column is exact: A(r0, cq) = beta, A(r0+1:r1, cq) = 0
            if (tid < L) sm.S[tid][0] = (tid == 0) ? sm.red[0] : 0.0;
            __syncthreads();

            // ---- scatter back (lower triangle of the strip, and the left block)
            for (int idx = tid; idx < off * L; idx += BC_THREADS) {
                const int k = idx % L, ii = idx / L;
                const int i = lo + ii, j = r0 + k;
                __stcg(&Bp[(j - i) + (long long)i * ldb], sm.S[k][ii]);
            }
            for (int idx = tid; idx < (W - off) * L; idx += BC_THREADS) {
                const int ii = off + idx % (W - off), k = idx / (W - off);
                const int i = lo + ii, j = r0 + k;
                if (i >= j) __stcg(&Bp[(i - j) + (long long)j * ldb], sm.S[k][ii]);
            }
            // reflector -> U[r0:r1, s]
            for (int k = tid; k < L; k += BC_THREADS) U[(r0 + k) + (long long)s * ldu] = sm.w[k];

            // ---- publish (release)
            __syncthreads();
            if (tid == 0) {
                __threadfence();
                st_release(&prog[s], cq);
            }
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
    static bool attr = false;
    if (!attr) {
        CUEV_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr = true;
    }
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
