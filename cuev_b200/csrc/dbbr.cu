// Stage 1: double-blocked band reduction (DBBR), full symmetric -> band of width b.
//
// Algorithm (Wang et al. 2025, Algorithm 1, as run by the reference src/cuda/dbbr.cu:145-229):
// the matrix is processed in k-column blocks; inside a block, b-column panels are factorised
// (panel QR -> Y, T), the two-sided companion Z = P - 1/2 Y (W^T P) with P = A W, W = Y T is
// built against the not-yet-updated trailing matrix (corrected for the block's earlier panels),
// the next panel is updated eagerly ("green" update) and the trailing matrix once per block with
// one SYR2K.
//
// What is B200-specific here:
//  * the panel QR (reference: cuSOLVER geqrf + extract + syrk + larft, dbbr.cu:124-143) is ONE
//    cooperative kernel: the rows x b panel is split across up to one CTA per SM and stays in
//    shared memory for the whole factorisation; each column costs one bounded grid barrier.  The
//    same kernel emits the unit-lower Y, tau, the block factor T and W = Y T;
//  * every contraction runs on the FP64 DMMA GEMM (gemm.cu): SYMM reading the lower triangle,
//    the deferral correction and the green update as two-segment-K GEMMs, the SYR2K as a
//    lower-triangle two-segment GEMM.
#include "solver.cuh"

#include <algorithm>
#include <mutex>
#include <cooperative_groups.h>

namespace cuev {
namespace {

constexpr int QR_THREADS = 256;
constexpr int QR_TARGET_ROWS = 128; // rows per CTA the launcher aims for
constexpr int QRC_THREADS = 512;    // cluster variant: up to ~800 rows per CTA

// Shared-memory layout of panel_qr_kernel<BW>:
//   sP  [chunk][BW + 1]  this CTA's rows of the panel
//   sGT [BW][BW]         G = V^T V below the diagonal (sGT[c][q] = G[q][c], q < c), T above
//   sp, srow, stau [BW]  reduced dot products, broadcast row c, tau
//   sred [QR_THREADS]    row-group partial sums
template <int BW> size_t panel_qr_smem(int chunk) {
    return sizeof(double) * ((size_t)chunk * (BW + 1) + BW * BW + 3 * BW + QR_THREADS);
}

template <int BW>
__global__ void __launch_bounds__(QR_THREADS)
    panel_qr_kernel(double *__restrict__ A, long long lda, double *__restrict__ Y, long long ldy,
                    double *__restrict__ tau, double *__restrict__ T, double *__restrict__ W,
                    long long ldw, int rows, int b, int chunk, double *__restrict__ part,
                    unsigned *bar, int *status) {
    constexpr int NRG = QR_THREADS / BW; // row groups
    constexpr int LD = BW + 1;
    extern __shared__ __align__(16) double sm[];
    double *sP = sm;
    double *sGT = sP + (size_t)chunk * LD;
    double *sp = sGT + BW * BW;
    double *srow = sp + BW;
    double *stau = srow + BW;
    double *sred = stau + BW;

    const int tid = threadIdx.x;
    const int P = gridDim.x, cta = blockIdx.x;
    const int r0 = cta * chunk;
    const int cnt = max(0, min(rows, r0 + chunk) - r0);
    const int j = tid % BW, rg = tid / BW;

    GridBarrier gb;
    gb.init(bar);

    // load this CTA's rows (column-major global -> row-major shared)
    for (int idx = tid; idx < cnt * b; idx += QR_THREADS) {
        const int r = idx % cnt, c = idx / cnt;
        sP[r * LD + c] = A[(r0 + r) + (long long)c * lda];
    }
    for (int idx = tid; idx < cnt * (BW - b); idx += QR_THREADS) { // unused columns (b < BW)
        const int r = idx % cnt, c = b + idx / cnt;
        sP[r * LD + c] = 0.0;
    }
    for (int idx = tid; idx < BW * BW; idx += QR_THREADS) sGT[idx] = 0.0;
    __syncthreads();

    const int ncols = min(rows, b);
    double *rowc = part + 2 * (size_t)P * BW; // 2 x BW broadcast slots after the partials

    for (int c = 0; c < ncols; ++c) {
        const int buf = c & 1;
        // (1) partial dots over this CTA's rows strictly below row c:  p_j = sum x_r a_j[r]
        double acc = 0.0;
        const int rstart = max(0, c + 1 - r0);
        for (int r = rstart + rg; r < cnt; r += NRG) acc += sP[r * LD + c] * sP[r * LD + j];
        sred[tid] = acc;
        __syncthreads();
        if (rg == 0) {
            double s = 0.0;
#pragma unroll
            for (int q = 0; q < NRG; ++q) s += sred[q * BW + j];
            part[((size_t)buf * P + cta) * BW + j] = s;
            if (c >= r0 && c < r0 + cnt) rowc[buf * BW + j] = sP[(c - r0) * LD + j];
        }
        if (!gb.sync(status, c)) return;

        // (2) deterministic reduction of the P partials: NRG threads per column j
        {
            double s = 0.0;
            for (int q = rg; q < P; q += NRG) s += __ldcg(&part[((size_t)buf * P + q) * BW + j]);
            sred[tid] = s;
            __syncthreads();
            if (rg == 0) {
                double tot = 0.0;
#pragma unroll
                for (int q = 0; q < NRG; ++q) tot += sred[q * BW + j];
                sp[j] = tot;
                srow[j] = __ldcg(&rowc[buf * BW + j]);
            }
            __syncthreads();
        }

        // (3) Householder reflector for x = A[c:, c]  (H = I - tau v v^T, v[c] = 1)
        const double alpha = srow[c];
        const double s2 = sp[c];
        double beta = alpha, tauc = 0.0, scal = 0.0;
        if (s2 > 0.0) {
            beta = -copysign(hypot(alpha, sqrt(s2)), alpha);
            tauc = (beta - alpha) / beta;
            scal = 1.0 / (alpha - beta);
        }
        if (!isfinite(s2) || !isfinite(alpha)) {
            if (tid == 0) dev_fail(status, CUEV_ERR_NONFINITE, c);
        }
        // (4) apply H to the trailing columns of own rows (j > c); v_r = scal * x_r for r > c
        if (tauc != 0.0) {
            const int jcol = j;
            if (jcol > c && jcol < b) {
                const double wj = srow[jcol] + scal * sp[jcol]; // v^T a_j
                const double f = tauc * wj;
                for (int r = max(0, c - r0) + rg; r < cnt; r += NRG) {
                    const int grow = r0 + r;
                    const double v = (grow == c) ? 1.0 : scal * sP[r * LD + c];
                    sP[r * LD + jcol] -= f * v;
                }
            }
        }
        // G[q][c] = v_q^T v_c for q < c
        if (tid < c) sGT[c * BW + tid] = srow[tid] + scal * sp[tid];
        if (tid == 0) stau[c] = tauc;
        __syncthreads();
        // (5) store v_c (scaled) and beta in column c of own rows
        for (int r = max(0, c - r0) + tid; r < cnt; r += QR_THREADS) {
            const int grow = r0 + r;
            if (grow == c)
                sP[r * LD + c] = beta;
            else if (grow > c)
                sP[r * LD + c] *= scal;
        }
        __syncthreads();
    }
    for (int c = ncols + tid; c < BW; c += QR_THREADS) stau[c] = 0.0;
    __syncthreads();

    // T: T[c][c] = tau_c,  T[q][c] = -tau_c sum_{p=q}^{c-1} T[q][p] G[p][c]   (q < c)
    // (T stored in the upper triangle of sGT, G below it)
    for (int c = 0; c < b; ++c) {
        if (tid < c) {
            double s = 0.0;
            for (int p = tid; p < c; ++p) {
                const double tqp = (p == tid) ? stau[tid] : sGT[tid * BW + p];
                s += tqp * sGT[c * BW + p];
            }
            sred[tid] = -stau[c] * s;
        }
        __syncthreads();
        if (tid < c) sGT[tid * BW + c] = sred[tid];
        __syncthreads();
    }

    // outputs: A (R above, v below), Y (unit lower trapezoid), W = Y T; CTA 0 writes T, tau
    for (int idx = tid; idx < cnt * b; idx += QR_THREADS) {
        const int r = idx % cnt, c = idx / cnt;
        const int grow = r0 + r;
        const double a = sP[r * LD + c];
        A[grow + (long long)c * lda] = a;
        Y[grow + (long long)c * ldy] = grow > c ? a : (grow == c ? 1.0 : 0.0);
    }
    if (W) {
        for (int idx = tid; idx < cnt * b; idx += QR_THREADS) {
            const int r = idx % cnt, c = idx / cnt;
            const int grow = r0 + r;
            double s = 0.0;
            const int pmax = min(c, grow); // Y[r][p] is zero for p > grow
            for (int p = 0; p <= pmax; ++p) {
                const double y = grow > p ? sP[r * LD + p] : 1.0; // p == grow -> unit diagonal
                const double tpc = (p == c) ? stau[c] : sGT[p * BW + c];
                s += y * tpc;
            }
            W[grow + (long long)c * ldw] = s;
        }
    }
    if (cta == 0) {
        for (int idx = tid; idx < b * b; idx += QR_THREADS) {
            const int q = idx % b, c = idx / b;
            T[q + (long long)c * b] = q < c ? sGT[q * BW + c] : (q == c ? stau[c] : 0.0);
        }
        for (int c = tid; c < b; c += QR_THREADS) tau[c] = stau[c];
    }
}

// Cluster variant of the panel QR for panels that fit in the shared memory of one thread-block
// cluster (up to 16 CTAs of one GPC): the same column loop, but each column's partial dot
// products are exchanged through distributed shared memory behind one hardware cluster barrier,
// instead of global partials behind a grid barrier through L2.  Two partial buffers alternate by
// column parity: a CTA overwrites the buffer of column c-1 only after the cluster barrier of
// column c, which every CTA reaches after its reads of column c-1.
template <int BW> size_t panel_qr_cluster_smem(int chunk) {
    return sizeof(double) *
           ((size_t)chunk * (BW + 1) + BW * BW + 3 * BW + QRC_THREADS + 4 * BW + 4);
}

template <int BW>
__global__ void __launch_bounds__(QRC_THREADS)
    panel_qr_cluster_kernel(double *__restrict__ A, long long lda, double *__restrict__ Y,
                            long long ldy, double *__restrict__ tau, double *__restrict__ T,
                            double *__restrict__ W, long long ldw, int rows, int b, int chunk,
                            int *status) {
    namespace cg = cooperative_groups;
    constexpr int NRG = QRC_THREADS / BW; // row groups
    constexpr int LD = BW + 1;
    extern __shared__ __align__(16) double sm[];
    double *sP = sm;
    double *sGT = sP + (size_t)chunk * LD;
    double *sp = sGT + BW * BW;
    double *srow = sp + BW;
    double *stau = srow + BW;
    double *sred = stau + BW;
    double *spart = sred + QRC_THREADS; // [2][BW] this CTA's partial dot products
    double *sroww = spart + 2 * BW;    // [2][BW] row c of the panel (owner CTA only)
    double *shh = sroww + 2 * BW;      // beta, tau, scale of the current reflector

    cg::cluster_group cl = cg::this_cluster();
    const int tid = threadIdx.x;
    const int P = (int)cl.num_blocks(), cta = (int)cl.block_rank();
    const int r0 = cta * chunk;
    const int cnt = max(0, min(rows, r0 + chunk) - r0);
    const int j = tid % BW, rg = tid / BW;

    for (int idx = tid; idx < cnt * b; idx += QRC_THREADS) {
        const int r = idx % cnt, c = idx / cnt;
        sP[r * LD + c] = A[(r0 + r) + (long long)c * lda];
    }
    for (int idx = tid; idx < cnt * (BW - b); idx += QRC_THREADS) {
        const int r = idx % cnt, c = b + idx / cnt;
        sP[r * LD + c] = 0.0;
    }
    for (int idx = tid; idx < BW * BW; idx += QRC_THREADS) sGT[idx] = 0.0;
    __syncthreads();

    const int ncols = min(rows, b);
    for (int c = 0; c < ncols; ++c) {
        const int buf = c & 1;
        // (1) partial dots over this CTA's rows strictly below row c
        // four independent chains: a CTA holds up to ~800 rows, 50 per thread and column
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
        int r = max(0, c + 1 - r0) + rg;
        for (; r + 3 * NRG < cnt; r += 4 * NRG) {
            a0 = fma(sP[r * LD + c], sP[r * LD + j], a0);
            a1 = fma(sP[(r + NRG) * LD + c], sP[(r + NRG) * LD + j], a1);
            a2 = fma(sP[(r + 2 * NRG) * LD + c], sP[(r + 2 * NRG) * LD + j], a2);
            a3 = fma(sP[(r + 3 * NRG) * LD + c], sP[(r + 3 * NRG) * LD + j], a3);
        }
        for (; r < cnt; r += NRG) a0 = fma(sP[r * LD + c], sP[r * LD + j], a0);
        sred[tid] = (a0 + a1) + (a2 + a3);
        __syncthreads();
        if (rg == 0) {
            double s = 0.0;
#pragma unroll
            for (int q = 0; q < NRG; ++q) s += sred[q * BW + j];
            spart[buf * BW + j] = s;
            if (c >= r0 && c < r0 + cnt) sroww[buf * BW + j] = sP[(c - r0) * LD + j];
        }
        cl.sync();

        // (2) every CTA reduces all partials in the same fixed order (identical results); lane c
        //     of the first row group also forms the reflector's scalars
        {
            double s = 0.0;
            for (int q = rg; q < P; q += NRG) s += cl.map_shared_rank(spart, q)[buf * BW + j];
            sred[tid] = s;
            __syncthreads();
            if (rg == 0) {
                double tot = 0.0;
#pragma unroll
                for (int q = 0; q < NRG; ++q) tot += sred[q * BW + j];
                const double rowc = cl.map_shared_rank(sroww, c / chunk)[buf * BW + j];
                sp[j] = tot;
                srow[j] = rowc;
                if (j == c) {
                    // (3) Householder reflector for x = A[c:, c]  (H = I - tau v v^T, v[c] = 1)
                    const double alpha = rowc, s2 = tot;
                    double beta = alpha, tauc = 0.0, scal = 0.0;
                    if (s2 > 0.0) {
                        beta = -copysign(hypot(alpha, sqrt(s2)), alpha);
                        tauc = (beta - alpha) / beta;
                        scal = 1.0 / (alpha - beta);
                    }
                    if (!isfinite(s2) || !isfinite(alpha)) dev_fail(status, CUEV_ERR_NONFINITE, c);
                    shh[0] = beta, shh[1] = tauc, shh[2] = scal;
                }
            }
            __syncthreads();
        }
        const double beta = shh[0], tauc = shh[1], scal = shh[2];

        // (4) store v_c (scaled) and beta in column c of own rows
        for (int r = max(0, c - r0) + tid; r < cnt; r += QRC_THREADS) {
            const int grow = r0 + r;
            if (grow == c)
                sP[r * LD + c] = beta;
            else if (grow > c)
                sP[r * LD + c] *= scal;
        }
        if (tid < c) sGT[c * BW + tid] = srow[tid] + scal * sp[tid];
        if (tid == 0) stau[c] = tauc;
        __syncthreads();
        // (5) apply H to the trailing columns j > c of own rows, a_j -= tau (v^T a_j) v: the
        //     (b - 1 - c) columns x own rows spread over all threads, column fastest
        const int nact = b - 1 - c;
        if (tauc != 0.0 && nact > 0) {
            const int groups = QRC_THREADS / nact;
            if (tid < groups * nact) {
                const int jj = c + 1 + tid % nact, g0 = tid / nact;
                const double f = tauc * (srow[jj] + scal * sp[jj]); // tau v^T a_j
#pragma unroll 4
                for (int r = max(0, c + 1 - r0) + g0; r < cnt; r += groups)
                    sP[r * LD + jj] -= f * sP[r * LD + c];
                if (g0 == 0 && c >= r0 && c < r0 + cnt) sP[(c - r0) * LD + jj] -= f; // v[c] = 1
            }
        }
        __syncthreads();
    }
    for (int c = ncols + tid; c < BW; c += QRC_THREADS) stau[c] = 0.0;
    __syncthreads();

    // T: T[c][c] = tau_c,  T[q][c] = -tau_c sum_{p=q}^{c-1} T[q][p] G[p][c]   (q < c)
    for (int c = 0; c < b; ++c) {
        if (tid < c) {
            double s = 0.0;
            for (int p = tid; p < c; ++p) {
                const double tqp = (p == tid) ? stau[tid] : sGT[tid * BW + p];
                s += tqp * sGT[c * BW + p];
            }
            sred[tid] = -stau[c] * s;
        }
        __syncthreads();
        if (tid < c) sGT[tid * BW + c] = sred[tid];
        __syncthreads();
    }

    for (int idx = tid; idx < cnt * b; idx += QRC_THREADS) {
        const int r = idx % cnt, c = idx / cnt;
        const int grow = r0 + r;
        const double a = sP[r * LD + c];
        A[grow + (long long)c * lda] = a;
        Y[grow + (long long)c * ldy] = grow > c ? a : (grow == c ? 1.0 : 0.0);
    }
    if (W) {
        for (int idx = tid; idx < cnt * b; idx += QRC_THREADS) {
            const int r = idx % cnt, c = idx / cnt;
            const int grow = r0 + r;
            double s = 0.0;
            const int pmax = min(c, grow);
            for (int p = 0; p <= pmax; ++p) {
                const double y = grow > p ? sP[r * LD + p] : 1.0;
                const double tpc = (p == c) ? stau[c] : sGT[p * BW + c];
                s += y * tpc;
            }
            W[grow + (long long)c * ldw] = s;
        }
    }
    if (cta == 0) {
        for (int idx = tid; idx < b * b; idx += QRC_THREADS) {
            const int q = idx % b, c = idx / b;
            T[q + (long long)c * b] = q < c ? sGT[q * BW + c] : (q == c ? stau[c] : 0.0);
        }
        for (int c = tid; c < b; c += QRC_THREADS) tau[c] = stau[c];
    }
    cl.sync(); // no CTA leaves while another may still read its shared memory
}

// Pack the lower band: B[r + j 2b] = A(j + r, j) for r <= b, 0 for b < r < 2b.
__global__ void pack_kernel(const double *__restrict__ A, long long lda, double *__restrict__ B,
                            int n, int b) {
    const int ldb = 2 * b;
    const long long total = (long long)ldb * n;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(idx % ldb);
        const int jc = (int)(idx / ldb);
        const int i = jc + r;
        B[idx] = (r <= b && i < n) ? A[i + (long long)jc * lda] : 0.0;
    }
}

// Largest cluster the cluster kernel can run with (16 needs the non-portable opt-in; 0 = none),
// probed once per instantiation and device with the occupancy API at the full shared-memory size
// (the function attributes it sets apply to the current device only).
template <int BW> int panel_qr_cluster_max() {
    static int cache[64];
    static bool init = false;
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    if (!init) {
        for (int &c : cache) c = -1;
        init = true;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return 0;
    }
    int &cached = cache[dev];
    if (cached >= 0) return cached;
    cached = 0;
    auto kern = panel_qr_cluster_kernel<BW>;
    const size_t smem = max_dynamic_smem((const void *)kern);
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess ||
        cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
            cudaSuccess) {
        cudaGetLastError();
        return cached;
    }
    for (int cl : {16, 8}) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(cl);
        cfg.blockDim = dim3(QRC_THREADS);
        cfg.dynamicSmemBytes = smem;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = cl, at[0].val.clusterDim.y = 1, at[0].val.clusterDim.z = 1;
        cfg.attrs = at, cfg.numAttrs = 1;
        int nclusters = 0;
        if (cudaOccupancyMaxActiveClusters(&nclusters, (void *)kern, &cfg) == cudaSuccess &&
            nclusters >= 1) {
            cached = cl;
            break;
        }
        cudaGetLastError();
    }
    return cached;
}

// Launch the cluster kernel if the panel fits one cluster; returns CUEV_ERR_UNSUPPORTED if not.
template <int BW> int launch_panel_qr_cluster(Workspace *ws, double *A, long long lda, double *Y,
                                              long long ldy, double *tau, double *T, double *W,
                                              long long ldw, int rows, int b) {
    const int clmax = panel_qr_cluster_max<BW>();
    if (clmax == 0) return CUEV_ERR_UNSUPPORTED;
    auto kern = panel_qr_cluster_kernel<BW>;
    const size_t max_smem = max_dynamic_smem((const void *)kern);
    int cl = std::max(1, std::min(clmax, div_up(rows, QR_TARGET_ROWS)));
    int chunk = div_up(rows, cl);
    while (panel_qr_cluster_smem<BW>(chunk) > max_smem && cl < clmax) {
        ++cl;
        chunk = div_up(rows, cl);
    }
    if (panel_qr_cluster_smem<BW>(chunk) > max_smem) return CUEV_ERR_UNSUPPORTED;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cl);
    cfg.blockDim = dim3(QRC_THREADS);
    cfg.dynamicSmemBytes = panel_qr_cluster_smem<BW>(chunk);
    cfg.stream = ws->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cl, at[0].val.clusterDim.y = 1, at[0].val.clusterDim.z = 1;
    cfg.attrs = at, cfg.numAttrs = 1;
    note_launch();
    CUEV_TRY(cudaLaunchKernelEx(&cfg, kern, A, lda, Y, ldy, tau, T, W, ldw, rows, b, chunk,
                                ws->status));
    return CUEV_OK;
}

template <int BW> int launch_panel_qr(Workspace *ws, double *A, long long lda, double *Y,
                                      long long ldy, double *tau, double *T, double *W,
                                      long long ldw, int rows, int b) {
    const int sms = num_sms();
    int P = std::max(1, std::min(sms, div_up(rows, QR_TARGET_ROWS)));
    int chunk = div_up(rows, P);
    auto kern = panel_qr_kernel<BW>;
    // shared memory bound: grow P (up to one CTA per SM) if the chunk does not fit
    static size_t max_smem = 0;
    if (max_smem == 0) max_smem = max_dynamic_smem((const void *)kern);
    while (panel_qr_smem<BW>(chunk) > max_smem && P < sms) {
        ++P;
        chunk = div_up(rows, P);
    }
    if (panel_qr_smem<BW>(chunk) > max_smem) {
        set_last_message("panel QR: panel too tall for the shared-memory resident kernel");
        return CUEV_ERR_UNSUPPORTED;
    }
    if ((size_t)(2 * P + 2) * BW > ws->qr_part_elems) {
        set_last_message("panel QR: partial-sum buffer too small");
        return CUEV_ERR_INVALID;
    }
    const size_t smem = panel_qr_smem<BW>(chunk);
    CUEV_CHECK_STATUS(ensure_dyn_smem((const void *)kern, max_smem));
    CUEV_TRY(cudaMemsetAsync(ws->bar, 0, 2 * sizeof(unsigned), ws->stream));
    void *args[] = {&A, &lda, &Y, &ldy, &tau, &T, &W, &ldw, &rows, &b, &chunk,
                    &ws->qr_part, &ws->bar, &ws->status};
    note_launch();
    CUEV_TRY(cudaLaunchCooperativeKernel((void *)kern, dim3(P), dim3(QR_THREADS), args, smem,
                                         ws->stream));
    return CUEV_OK;
}

} // namespace

int panel_qr(Workspace *ws, double *A, long long lda, double *Y, long long ldy, double *tau,
             double *T, double *W, long long ldw, int rows, int b) {
    if (rows <= 0 || b <= 0) return CUEV_OK;
    if (b <= 32) {
        const int st = launch_panel_qr_cluster<32>(ws, A, lda, Y, ldy, tau, T, W, ldw, rows, b);
        if (st != CUEV_ERR_UNSUPPORTED) return st;
        return launch_panel_qr<32>(ws, A, lda, Y, ldy, tau, T, W, ldw, rows, b);
    }
    if (b <= 64) {
        const int st = launch_panel_qr_cluster<64>(ws, A, lda, Y, ldy, tau, T, W, ldw, rows, b);
        if (st != CUEV_ERR_UNSUPPORTED) return st;
        return launch_panel_qr<64>(ws, A, lda, Y, ldy, tau, T, W, ldw, rows, b);
    }
    set_last_message("panel QR supports b <= 64");
    return CUEV_ERR_INVALID;
}

int dbbr_pack(Workspace *ws, const double *A, long long lda, double *B) {
    const long long total = 2LL * ws->b * ws->n;
    const int blocks = (int)std::min<long long>(8LL * num_sms(), (total + 255) / 256);
    pack_kernel<<<std::max(1, blocks), 256, 0, ws->stream>>>(A, lda, B, ws->n, ws->b); note_launch();
    CUEV_TRY(cudaGetLastError());
    return CUEV_OK;
}

namespace {
int build_block_t(Workspace *ws, int i, int w) {
    const int n = ws->n, b = ws->b, k = ws->k;
    const long long ld = n;
    const int rows = n - (i + b);
    double *Tb = ws->Tblk + (size_t)(i / k) * k * k;
    const double *Yb = ws->Y + (long long)i * ld + (i + b);
    CUEV_TRY(cudaMemsetAsync(Tb, 0, sizeof(double) * (size_t)k * k, ws->stream));
    // G = Y_blk^T Y_blk  (w x w, ld k)
    CUEV_CHECK_STATUS(ws_gemm(ws, 1, 0, w, w, rows, 1.0, Yb, ld, Yb, ld, 0.0, ws->Gblk, k));
    for (int q = 0; q * b < w; ++q) {
        const int qb = q * b;
        const double *Tq = ws->Tp + (size_t)((i + qb) / b) * b * b;
        CUEV_TRY(cudaMemcpy2DAsync(Tb + qb + (size_t)qb * k, k * sizeof(double), Tq,
                                   b * sizeof(double), b * sizeof(double), b,
                                   cudaMemcpyDeviceToDevice, ws->stream));
        if (q == 0) continue;
        double *X = ws->Dwk; // qb x b
        CUEV_CHECK_STATUS(ws_gemm(ws, 0, 0, qb, b, b, 1.0, ws->Gblk + (size_t)qb * k, k, Tq, b,
                                  0.0, X, qb));
        CUEV_CHECK_STATUS(ws_gemm(ws, 0, 0, qb, b, qb, -1.0, Tb, k, X, qb, 0.0,
                                  Tb + (size_t)qb * k, k));
    }
    return CUEV_OK;
}
} // namespace

int dbbr_reduce(Workspace *ws, double *A) {
    const int n = ws->n, b = ws->b, k = ws->k;
    const long long ld = n;
    double *Y = ws->Y, *Z = ws->Z, *Wp = ws->Wp;
    CUEV_TRY(cudaMemsetAsync(Y, 0, sizeof(double) * (size_t)n * n, ws->stream));

    for (int i = 0; i < n; i += k) {
        const int kc = std::min(k, n - i);
        int w = 0; // reflector columns accumulated in this block
        for (int j = i; j < i + kc && j + b < n; j += b) {
            const int rows = n - (j + b);
            double *Apan = A + (long long)j * ld + (j + b); // A[j+b:, j:j+b]
            double *Ypan = Y + (long long)j * ld + (j + b);
            double *Atr = A + (long long)(j + b) * ld + (j + b);
            double *Zcur = Z + (long long)(j - i) * ld + (j + b); // P / Z of this panel
            double *Tpan = ws->Tp + (size_t)(j / b) * b * b;
            double *Wpan = Wp + (j + b);
            const double *Yblk = Y + (long long)i * ld + (j + b); // Y[j+b:, i:i+w]
            const double *Zblk = Z + (j + b);                     // Z[j+b:, 0:w]

            // panel QR -> R (in A), Y, tau, T, W = Y T
            CUEV_CHECK_STATUS(
                panel_qr(ws, Apan, ld, Ypan, ld, ws->tau + j, Tpan, Wpan, ld, rows, b));
            // P0 = A_trail W (A_trail symmetric, lower triangle, not yet updated for this block)
            CUEV_CHECK_STATUS(ws_symm(ws, rows, b, 1.0, Atr, ld, Wpan, ld, 0.0, Zcur, ld));
            // The panel's Z, in the order of the reference (dbbr.cu:175-198):
            //   P = P0 - Y_blk D1 - Z_blk D2,  D1 = Z_blk^T W,  D2 = Y_blk^T W,
            //   C = W^T P,  Z = P - 1/2 Y_pan C.
            // Here with two dependent products fewer.  W^T P expands to
            // G - D2^T D1 - D1^T D2 (G = W^T P0), so C needs no pass over P; Z_cur sits right
            // after Z_blk in Z and Y_pan right after Y_blk in Y, so one product gives
            // E = [Z_blk | P0]^T W = [D1; G^T] and one two-segment product gives
            //   Z = P0 - [Y_blk | Y_pan] [D1; C^T / 2] - Z_blk D2.
            // C is symmetric in exact arithmetic; its transpose differs by rounding only.
            const int le = w + b;
            double *E = ws->Dwk;                        // (w + b) x b, ld w + b
            double *D2 = ws->Dwk + (size_t)k * b;       // w x b, ld w
            const double *ZP = Z + (j + b);             // Z[j+b:, 0:w+b] = [Z_blk | Z_cur]
            CUEV_CHECK_STATUS(ws_gemm(ws, 1, 0, le, b, rows, 1.0, ZP, ld, Wpan, ld, 0.0, E, le));
            if (w > 0) {
                CUEV_CHECK_STATUS(ws_gemm(ws, 1, 0, w, b, rows, 1.0, Yblk, ld, Wpan, ld, 0.0, D2, w));
                // E[w:w+b] = (G^T - D1^T D2 - D2^T D1) / 2 = C^T / 2
                CUEV_CHECK_STATUS(ws_gemm2(ws, 1, 0, b, b, w, w, -0.5, E, le, D2, w, D2, w, E, le,
                                           0.5, E + w, le, 0));
                const double *YP = Y + (long long)i * ld + (j + b); // [Y_blk | Y_pan]
                CUEV_CHECK_STATUS(ws_gemm2(ws, 0, 0, rows, b, le, w, -1.0, YP, ld, Zblk, ld, E, le,
                                           D2, w, 1.0, Zcur, ld, 0));
            } else {
                // first panel of the block: E = G^T, Z = P0 - 1/2 Y_pan G^T
                CUEV_CHECK_STATUS(ws_gemm(ws, 0, 0, rows, b, b, -0.5, Ypan, ld, E, le, 1.0, Zcur, ld));
            }
            w += b;
            // green update of the next panel's columns: A[j+b:, j+b:j+b+nb] -= Z Yg^T + Y Zg^T,
            // nb = b except at the end of the matrix, where the last columns number fewer than b
            // (n not a multiple of b): the update must stop at column n - 1
            if (j + b < i + kc) {
                const int nb = std::min(b, rows);
                const double *Yg = Y + (long long)i * ld + (j + b); // Y[j+b:j+b+nb, i:i+w]
                const double *Zg = Z + (j + b);                     // Z[j+b:j+b+nb, 0:w]
                CUEV_CHECK_STATUS(ws_gemm2(ws, 0, 1, rows, nb, w, w, -1.0, Zblk, ld, Yblk, ld, Yg,
                                           ld, Zg, ld, 1.0, Atr, ld, 0));
            }
        }
        // aggregated WY factor of the block for the back-transform:
        //   prod_q (I - Y_q T_q Y_q^T) = I - Y_blk T_blk Y_blk^T,
        //   T_blk[0:q, q] = -T_blk[0:q, 0:q] (Y_blk[:, 0:q]^T Y_q) T_q   (compact-WY merge)
        if (w > 0) CUEV_CHECK_STATUS(build_block_t(ws, i, w));
        // trailing update once per block: A[i+kc:, i+kc:] -= Y Z^T + Z Y^T (lower triangle)
        const int tn = n - (i + kc);
        if (tn > 0 && w > 0) {
            const double *Yt = Y + (long long)i * ld + (i + kc);
            const double *Zt = Z + (i + kc);
            double *At = A + (long long)(i + kc) * ld + (i + kc);
            CUEV_CHECK_STATUS(
                ws_gemm2(ws, 0, 1, tn, tn, w, w, -1.0, Yt, ld, Zt, ld, Zt, ld, Yt, ld, 1.0, At, ld, 1));
        }
    }
    return dbbr_pack(ws, A, ld, ws->B);
}

} // namespace cuev
