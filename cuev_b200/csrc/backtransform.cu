// Stage 4: back-transform of the tridiagonal eigenvectors, evec = Q_s Q_b Q_d.
//
// BC-Back (M <- Q_b M).  Q_b = H_(0,0) H_(0,1) ... H_(n-3,last) is the product of the
// bulge-chasing reflectors in the order they were generated, so M <- Q_b M applies them in
// reverse (reference src/cuda/backtransform.cu:58-62).  Reflector (s, h) of sweep s, hop h acts
// on rows [s+1+hb, s+(h+1)b] and is stored in U[:, s].
//
// Ordering used here (own derivation): cut the sweeps into tiles of TS consecutive sweeps and
// process tiles from the last to the first.  Inside a tile, apply the "hop blocks"
// h = 0, 1, 2, ... in increasing order, each block being the tile's TS reflectors of hop h in
// decreasing sweep order.  Two reflectors (s, h), (s', h') with s > s' overlap only if h' = h
// (|s - s'| < b) or h' = h + 1 (s - s' < 2b); in both cases the true reverse order and this
// order both apply (s, h) first, so the result is identical.  The payoff: block h+1 shares only
// TS-1 rows with block h, so a thread can own one column of M and march down it with a register
// window of TS+b-1 rows, applying TS reflectors per step with compile-time register indices and
// reading w from shared memory as warp-wide broadcasts.  Columns are independent, so there is
// no inter-thread communication at all.  (The reference slides a 256-row window per warp with
// cross-lane shuffles and only supports b = 32, backtransform.cu:16,35.)
//
// SBR-Back (M <- Q_s M).  Q_s = prod_j (I - Y_j T_j Y_j^T).  The reference applies each b-wide
// panel with two K = b GEMMs (backtransform.cu:210-230).  Here the panels of one DBBR k-block are
// merged into one compact-WY factor (I - Y_blk T_blk Y_blk^T, T_blk built in dbbr.cu), so the
// back-transform is three large DMMA GEMMs per k-block with K = rows or k.
#include "solver.cuh"

#include <algorithm>

namespace cuev {
namespace {

template <int BW, int TS> struct BcBackCfg {
    static constexpr int R = TS + BW - 1; // register rows per column
};

// One thread = one column of M.  NWARP warps per CTA.
template <int BW, int TS, int NWARP>
__global__ void __launch_bounds__(32 * NWARP)
    bc_back_kernel(const double *__restrict__ U, long long ldu, double *__restrict__ M,
                   long long ldm, int n, int ncols) {
    constexpr int R = BcBackCfg<BW, TS>::R;
    __shared__ __align__(16) double sW[TS][BW]; // reflectors of the current hop block
    const int col = blockIdx.x * (32 * NWARP) + threadIdx.x;
    const bool active = col < ncols;
    double *__restrict__ Mc = M + (long long)(active ? col : 0) * ldm;
    const int nsweeps = n - 2;
    if (nsweeps <= 0) return;

    double m[R];
    const int ntile = (nsweeps + TS - 1) / TS;
    for (int tile = ntile - 1; tile >= 0; --tile) {
        const int s0 = tile * TS;
        const int top = s0 + 1; // first row touched by the tile
        const int hmax = (n - 1 - top) / BW; // last hop block with rows inside the matrix
        // initial window: rows [top, top + R)
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const int row = top + i;
            m[i] = (active && row < n) ? Mc[row] : 0.0;
        }
        for (int h = 0; h <= hmax; ++h) {
            const int base = top + h * BW; // row of m[0]
            __syncthreads();
            // stage w of reflectors (s0 + t, h), rows [base + t, base + t + BW)
            for (int idx = threadIdx.x; idx < TS * BW; idx += 32 * NWARP) {
                const int t = idx / BW, i = idx % BW;
                const int s = s0 + t, row = base + t + i;
                sW[t][i] = (s < nsweeps && row < n) ? U[row + (long long)s * ldu] : 0.0;
            }
            __syncthreads();
            // apply in decreasing sweep order: m[t : t+BW] -= 2 (w^T m) w
#pragma unroll
            for (int t = TS - 1; t >= 0; --t) {
                double d0 = 0.0, d1 = 0.0, d2 = 0.0, d3 = 0.0;
#pragma unroll
                for (int i = 0; i < BW; i += 4) {
                    const double2 wa = *reinterpret_cast<const double2 *>(&sW[t][i]);
                    const double2 wb = *reinterpret_cast<const double2 *>(&sW[t][i + 2]);
                    d0 = fma(wa.x, m[t + i], d0);
                    d1 = fma(wa.y, m[t + i + 1], d1);
                    d2 = fma(wb.x, m[t + i + 2], d2);
                    d3 = fma(wb.y, m[t + i + 3], d3);
                }
                const double f = -2.0 * ((d0 + d1) + (d2 + d3));
#pragma unroll
                for (int i = 0; i < BW; i += 2) {
                    const double2 w = *reinterpret_cast<const double2 *>(&sW[t][i]);
                    m[t + i] = fma(f, w.x, m[t + i]);
                    m[t + i + 1] = fma(f, w.y, m[t + i + 1]);
                }
            }
            // rows [base, base + BW) are final for this tile; shift the window down by BW
#pragma unroll
            for (int i = 0; i < BW; ++i) {
                const int row = base + i;
                if (active && row < n) Mc[row] = m[i];
            }
            if (h < hmax) {
#pragma unroll
                for (int i = 0; i < R - BW; ++i) m[i] = m[i + BW];
#pragma unroll
                for (int i = R - BW; i < R; ++i) {
                    const int row = base + BW + i;
                    m[i] = (active && row < n) ? Mc[row] : 0.0;
                }
            } else {
                // flush the rest of the window
#pragma unroll
                for (int i = BW; i < R; ++i) {
                    const int row = base + i;
                    if (active && row < n) Mc[row] = m[i];
                }
            }
        }
    }
}

template <int BW, int TS> int launch_bc_back(Workspace *ws, double *M, long long ldm, int ncols) {
    constexpr int NWARP = 2;
    const int grid = div_up(ncols, 32 * NWARP);
    bc_back_kernel<BW, TS, NWARP><<<grid, 32 * NWARP, 0, ws->stream>>>(ws->U, ws->n, M, ldm,
                                                                       ws->n, ncols); note_launch();
    CUEV_TRY(cudaGetLastError());
    return CUEV_OK;
}

} // namespace

int bc_back(Workspace *ws, double *M, long long ldm) {
    if (ws->n <= 2) return CUEV_OK;
    if (ws->b == 32) return launch_bc_back<32, 32>(ws, M, ldm, ws->n);
    if (ws->b == 64) return launch_bc_back<64, 32>(ws, M, ldm, ws->n);
    return CUEV_ERR_INVALID;
}

int sbr_back(Workspace *ws, double *M, long long ldm) {
    const int n = ws->n, b = ws->b, k = ws->k;
    const long long ld = n;
    // scratch: X = Y_blk^T M and X2 = T_blk X, both (w x n) with w <= min(k, n), in the D&C
    // buffers (free once the tridiagonal eigenvectors are formed)
    double *X = ws->dc_S;
    double *X2 = ws->dc_Q2;
    // blocks in reverse order
    int last_i = 0;
    for (int i = 0; i < n; i += k) last_i = i;
    for (int i = last_i; i >= 0; i -= k) {
        const int kc = std::min(k, n - i);
        int w = 0;
        for (int j = i; j < i + kc && j + b < n; j += b) w += b;
        if (w == 0) continue;
        const int rows = n - (i + b);
        const double *Yb = ws->Y + (long long)i * ld + (i + b);
        const double *Tb = ws->Tblk + (size_t)(i / k) * k * k;
        double *Mb = M + (i + b);
        CUEV_CHECK_STATUS(ws_gemm(ws, 1, 0, w, n, rows, 1.0, Yb, ld, Mb, ldm, 0.0, X, w));
        CUEV_CHECK_STATUS(ws_gemm(ws, 0, 0, w, n, w, 1.0, Tb, k, X, w, 0.0, X2, w));
        CUEV_CHECK_STATUS(ws_gemm(ws, 0, 0, rows, n, w, -1.0, Yb, ld, X2, w, 1.0, Mb, ldm));
    }
    return CUEV_OK;
}

} // namespace cuev
