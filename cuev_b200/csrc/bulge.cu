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
//  * the wavefront condition is derived from the footprints of the hops: hop h of sweep s
//    (window rows [cq, r1 + b], reflector rows [r0, r1]) overlaps hop h+1 of sweep s-1 on a
//    block and hop h+2 of sweep s-1 on one element only, A(r1 + b, r1) (the first entry of
//    that hop's reduced column, which it sets to its beta and hop h later rewrites).  So hop h
//    waits until sweep s-1 has completed hop h+1 (prog[s-1] >= r1 - b, the start of that hop)
//    and has written the beta of hop h+2 (prog_ref[s-1] >= r1 - b + 1); hop h+2 writes that
//    element right after its reflector is formed and publishes it, and leaves it alone in its
//    update.  The reference waits for four hops (prog >= c + 3b).
//  * per hop the b x 3b strip of the symmetric window that the reflector touches is gathered
//    into shared memory once; each updated element (rank-2 H A H) goes straight back to the band
//    from the thread that computes it, with no barrier between update and write-back.
#include "solver.cuh"

#include <algorithm>
#include <climits>

namespace cuev {
namespace {

// Threads per hop.  b = 64's window (2b x 3b) is four times b = 32's, so it runs twice the threads
// (n = 16384, b = 64: 355 -> 286 ms; n = 8192: 174 -> 140 ms).  At b = 32 the hop is bound by its
// L2 round trips and fences, not its arithmetic: 384 and 512 threads measured the same as 256.
template <int BW> constexpr int chase_threads() { return BW == 64 ? 512 : 256; }

template <int BW> struct ChaseSmem {
    double S[BW][3 * BW + 1]; // strip: S[k][ii] = A(lo + ii, r0 + k)
    double w[BW];             // reflector
    double p[3 * BW];         // p = 2 A w over the window rows
    double beta;
    double kap[chase_threads<BW>() / 32]; // per-warp partial sums of kappa = w^T p
};

template <int BW>
__global__ void __launch_bounds__(chase_threads<BW>())
    bc_chase_kernel(double *__restrict__ Bp, double *__restrict__ U, long long ldu, int n, int b,
                    int *prog, int *status) {
    int *prog_ref = prog + n; // per sweep: cq of the last hop whose beta is in the band
    constexpr int NT = chase_threads<BW>();
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
            int cq, r0, r1u; // r1u: last reflector row before clipping to the matrix
            if (hop == 0) {
                cq = s, r0 = s + 1, r1u = s + b;
            } else {
                const int c = s + 1 + (hop - 1) * b;
                if (c + b >= n) break;
                cq = c, r0 = c + b, r1u = c + 2 * b - 1;
            }
            const int r1 = min(r1u, n - 1);
            const int L = r1 - r0 + 1;
            const int lo = cq, hi = min(n - 1, r1 + b);
            const int W = hi - lo + 1;
            const int off = r0 - lo; // strip row of reflector row r0

            // ---- wait for sweep s-1: every hop that starts at or before r1u - b completed, and
            // the beta of the hop that starts in (r1u - b, r1u] written.  The thresholds come from
            // the unclipped r1u: at the end of the matrix sweep s-1 has no hop that far on, so
            // the wait runs to its end-of-sweep release (with the clipped r1 the thresholds fall
            // below the counters' initial -1 when n <= b, and nothing would be waited for).
            if (tid == 0) {
                int ok = 1;
                if (s > 0) {
                    const int need = r1u - b + 1;
                    const uint64_t t0 = global_ns();
                    const uint64_t limit = wait_limit_ns(status);
                    // the clock is read every 256 polls, or every poll under a short limit
                    const int every = limit < 1000000ull ? 0 : 255;
                    int spins = 0;
                    while (ld_acquire(&prog[s - 1]) < need - 1 ||
                           ld_acquire(&prog_ref[s - 1]) < need) {
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
            // Householder of x = A(r0 : r1, cq).  b = 32: straight from the gathered registers
            // (lane k of warp 0 holds x[k] in vl[0], the left-block element ii = 0, zero for
            // k >= L), before the barrier; b = 64: from the strip after it.
            if constexpr (BW == 32) {
                if (warp == 0) {
                    const double xk = vl[0];
                    const double ss = warp_sum(xk * xk);
                    const double x0 = __shfl_sync(0xffffffffu, xk, 0);
                    double wk = 0.0;
                    if (ss != 0.0) {
                        const double beta = (x0 >= 0.0) ? -sqrt(ss) : sqrt(ss);
                        const double v0 = x0 - beta;
                        wk = (lane == 0 ? v0 : xk) * rsqrt(v0 * v0 + (ss - x0 * x0));
                        if (lane == 0) sm.beta = beta;
                    } else if (lane == 0) {
                        sm.beta = 0.0;
                    }
                    sm.w[lane] = wk;
                }
                __syncthreads();
            } else {
                __syncthreads();
                if (warp == 0) {
                    double ss = 0.0;
                    for (int k = lane; k < L; k += 32) ss = fma(sm.S[k][0], sm.S[k][0], ss);
                    ss = warp_sum(ss);
                    const double x0 = sm.S[0][0];
                    if (ss == 0.0) {
                        for (int k = lane; k < BW; k += 32) sm.w[k] = 0.0;
                        if (lane == 0) sm.beta = 0.0;
                    } else {
                        const double beta = (x0 >= 0.0) ? -sqrt(ss) : sqrt(ss);
                        const double v0 = x0 - beta;
                        const double inv = rsqrt(v0 * v0 + (ss - x0 * x0));
                        for (int k = lane; k < BW; k += 32)
                            sm.w[k] = k < L ? (k == 0 ? v0 : sm.S[k][0]) * inv : 0.0;
                        if (lane == 0) sm.beta = beta;
                    }
                }
                __syncthreads();
            }

            // ---- p = 2 A w over the window rows (TPR threads per row, the upper half of the
            // diagonal block read from its mirror), and per-warp partial sums of
            // kappa = w^T p over the reflector rows (rows off .. off + L - 1)
            {
                // threads per row: as many (4, 2 or 1) as leave the last warp without a row
                constexpr int TPR = (NT > 4 * 3 * BW + 31) ? 4 : (NT > 2 * 3 * BW + 31) ? 2 : 1;
                constexpr int KP = BW / TPR;                 // k range per thread
                constexpr int PW = (3 * BW * TPR + 31) / 32; // warps that hold rows
                static_assert(PW < NT / 32, "the last warp holds no row");
                const int h = tid % TPR, ii = tid / TPR; // every lane of a row warp shuffles
                const bool act = ii < W;
                double kp = 0.0;
                if (tid == NT - 1) {
                    // this hop's beta, A(r0, cq), for the next sweep (see the wait above); the
                    // release orders the store before the flag
                    __stcg(&Bp[(r0 - cq) + (long long)cq * ldb], sm.beta);
                    st_release(&prog_ref[s], cq);
                }
                if (warp < PW) {
                    const int a = ii - off; // row within the diagonal block when 0 <= a < L
                    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
                    const int k0 = h * KP, k1 = act ? min(L, k0 + KP) : k0;
                    int k = k0;
                    if (a >= 0 && a < L) {
                        // (an unconditional split of this loop at k = a made the compiler
                        // schedule the update phase below 1300 cycles slower per hop)
                        for (; k < k1; ++k) {
                            const double v = k > a ? sm.S[a][off + k] : sm.S[k][ii];
                            a0 = fma(v, sm.w[k], a0);
                        }
                    } else {
                        for (; k + 3 < k1; k += 4) {
                            a0 = fma(sm.S[k][ii], sm.w[k], a0);
                            a1 = fma(sm.S[k + 1][ii], sm.w[k + 1], a1);
                            a2 = fma(sm.S[k + 2][ii], sm.w[k + 2], a2);
                            a3 = fma(sm.S[k + 3][ii], sm.w[k + 3], a3);
                        }
                        for (; k < k1; ++k) a0 = fma(sm.S[k][ii], sm.w[k], a0);
                    }
                    double pr = (a0 + a1) + (a2 + a3);
#pragma unroll
                    for (int o = 1; o < TPR; o <<= 1) pr += __shfl_xor_sync(0xffffffffu, pr, o);
                    pr *= 2.0;
                    if (act && h == 0) {
                        sm.p[ii] = pr;
                        if (a >= 0 && a < L) kp = fma(sm.w[a], pr, kp);
                    }
                }
                if (warp < PW) kp = warp_sum(kp);
                if (lane == 0) sm.kap[warp] = kp;
            }
            __syncthreads();
            double kappa = 0.0;
#pragma unroll
            for (int q = 0; q < NT / 32; ++q) kappa += sm.kap[q];
            const double beta = sm.beta;

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
                if (ii == 0 && k == 0) continue; // beta: written before the p phase
                double v;
                if (ii == 0) {
                    v = 0.0;
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

            // ---- publish: the barrier orders every thread's stores before the release (which is
            // cumulative over what the releasing thread has observed through the barrier).  The
            // last thread releases, so that thread 0 goes on to the next hop's wait while the
            // release's fence drains; the same thread publishes the end of the sweep below, so
            // prog[s] only grows.
            __syncthreads();
            if (tid == NT - 1) st_release(&prog[s], cq);
        }
        if (tid == NT - 1) {
            __threadfence();
            st_release(&prog_ref[s], INT_MAX);
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
    CUEV_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, chase_threads<BW>(), smem));
    // at most two CTAs per SM: a hop's latency grows with the CTAs that share its SM, and two per
    // SM still keep more sweeps in flight than the wavefront needs (n = 16384: 3 per SM 179.7 ms,
    // 2 per SM 175.6, 1 per SM 176.1)
    const int cap = std::min(2, std::max(1, per_sm)) * num_sms();
    int grid = std::max(1, std::min(nsweeps, cap));
    double *U = ws->U;
    long long ldu = n;
    int nn = n, bb = b;
    void *args[] = {&B, &U, &ldu, &nn, &bb, &ws->prog, &ws->status};
    note_launch();
    CUEV_TRY(cudaLaunchCooperativeKernel((void *)kern, dim3(grid), dim3(chase_threads<BW>()), args, smem,
                                         ws->stream));
    return CUEV_OK;
}

} // namespace

int bc_chase(Workspace *ws, double *B, double *d, double *e) {
    const int n = ws->n, b = ws->b;
    CUEV_TRY(cudaMemsetAsync(ws->U, 0, sizeof(double) * (size_t)n * n, ws->stream));
    if (n > 2) {
        // prog, prog_ref = -1: no hop completed, no beta written yet
        CUEV_TRY(cudaMemsetAsync(ws->prog, 0xFF, 2 * sizeof(int) * (size_t)n, ws->stream));
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
