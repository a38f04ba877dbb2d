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

__device__ __forceinline__ void cp_async8(double *smem, const double *gmem, bool pred) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem),
                 "r"(pred ? 8 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
// 16-byte shared load of two reflector entries (broadcast: every lane reads the same address).
// Plain loads let the compiler re-read w for the update instead of keeping it live (volatile
// asm loads made it hoist them and spill).
__device__ __forceinline__ double2 lds2(const double *p) {
    return *reinterpret_cast<const double2 *>(p);
}

// One thread = one column of M; NWARP warps per CTA.  Shared memory (doubles):
//   sW  [2][TS][BW]       static: reflectors of the current and the next hop block (cp.async)
//   sIn [NT][BW+2]        dynamic: incoming rows of M for the next step (cp.async, coalesced)
//   sOut[NT][BW+2]        dynamic: finished rows of M, stored cooperatively (coalesced)
// The register window m[] is only ever indexed with compile-time constants and only exchanges
// data with shared memory, which keeps it at 95 doubles without spills.
template <int BW, int TS> constexpr size_t bc_back_smem(int nt) {
    return sizeof(double) * (2 * (size_t)nt * (BW + 2));
}

template <int BW, int TS, int NWARP>
__global__ void __launch_bounds__(32 * NWARP)
    bc_back_kernel(const double *__restrict__ U, long long ldu, double *__restrict__ M,
                   long long ldm, int n, int ncols) {
    constexpr int NT = 32 * NWARP;
    constexpr int R = TS + BW - 1; // register rows per column
    constexpr int KEEP = TS - 1;   // rows carried from one hop block to the next
    constexpr int MLD = BW + 2;    // 16-byte multiple, conflict-free 16-byte accesses
    // reflectors in a static array: with an extern (dynamic) base the compiler spills the window
    __shared__ __align__(16) double sW[2 * TS * BW];
    extern __shared__ __align__(16) double bsm[];
    double *sIn = bsm;
    double *sOut = bsm + NT * MLD;
    const int tid = threadIdx.x;
    const int col0 = blockIdx.x * NT;
    const int nsweeps = n - 2;
    if (nsweeps <= 0) return;

    // reflectors (s0 + t, h): rows [base + t, base + t + BW) of U[:, s0 + t]
    auto stage_w = [&](int buf, int s0, int base) {
        double *dst = sW + buf * TS * BW;
#pragma unroll 4
        for (int idx = tid; idx < TS * BW; idx += NT) {
            const int t = idx / BW, i = idx % BW;
            const int s = s0 + t, row = base + t + i;
            const bool ok = (s < nsweeps) && (row < n);
            cp_async8(dst + idx, ok ? U + row + (long long)s * ldu : U, ok);
        }
    };
    // rows [row0, row0 + BW) of the CTA's columns -> sIn, coalesced along rows
    auto stage_in = [&](int row0) {
#pragma unroll 4
        for (int idx = tid; idx < NT * BW; idx += NT) {
            const int i = idx % BW, c = idx / BW;
            const int row = row0 + i, cc = col0 + c;
            const bool ok = (cc < ncols) && (row < n);
            cp_async8(sIn + c * MLD + i, ok ? M + row + (long long)cc * ldm : M, ok);
        }
    };
    // sOut -> rows [row0, row0 + cnt) of the CTA's columns
    auto store_out = [&](int row0, int cnt) {
        for (int idx = tid; idx < NT * BW; idx += NT) {
            const int i = idx % BW, c = idx / BW;
            const int row = row0 + i, cc = col0 + c;
            if (i < cnt && cc < ncols && row < n) M[row + (long long)cc * ldm] = sOut[c * MLD + i];
        }
    };

    double m[R];
    const int ntile = (nsweeps + TS - 1) / TS;
    const int mycol = min(col0 + tid, ncols - 1); // clamped: out-of-range lanes compute garbage
    const bool active = col0 + tid < ncols;      // ... and never store it
    const double *Mc = M + (long long)mycol * ldm;
    for (int tile = ntile - 1; tile >= 0; --tile) {
        const int s0 = tile * TS;
        const int top = s0 + 1;              // first row touched by the tile
        const int hmax = (n - 1 - top) / BW; // last hop block with rows inside the matrix
        __syncthreads();
        stage_w(0, s0, top);
        stage_in(top + KEEP);
        cp_async_commit();
        // carried rows of the first step: [top, top + KEEP), rows past n read as 0
#pragma unroll
        for (int i = 0; i < KEEP; ++i) {
            const int row = top + i;
            const double v = Mc[min(row, n - 1)];
            m[i] = row < n ? v : 0.0;
        }
        for (int h = 0; h <= hmax; ++h) {
            const int base = top + h * BW; // row of m[0]
            cp_async_wait<0>();
            __syncthreads(); // sW[h & 1] and sIn complete; previous sOut stored
#pragma unroll
            for (int i = 0; i < BW; ++i) m[KEEP + i] = sIn[tid * MLD + i];
            __syncthreads(); // everyone has read sIn
            if (h < hmax) {
                stage_w((h + 1) & 1, s0, base + BW);
                stage_in(base + BW + KEEP);
            }
            cp_async_commit();
            const double *W = sW + (h & 1) * TS * BW;
            // apply in decreasing sweep order: m[t : t+BW] -= 2 (w^T m) w
#pragma unroll
            for (int t = TS - 1; t >= 0; --t) {
                const double *w = W + t * BW;
                double acc[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
                for (int i = 0; i < BW; i += 2) {
                    // compiler-only fence every 32 entries: keeps at most 32 w values in flight
                    if (i % 32 == 0) asm volatile("" ::: "memory");
                    const double2 ww = lds2(w + i);
                    acc[(i >> 1) & 3] = fma(ww.x, m[t + i], acc[(i >> 1) & 3]);
                    acc[4 + ((i >> 1) & 3)] = fma(ww.y, m[t + i + 1], acc[4 + ((i >> 1) & 3)]);
                }
                const double f =
                    -2.0 * (((acc[0] + acc[1]) + (acc[2] + acc[3])) +
                            ((acc[4] + acc[5]) + (acc[6] + acc[7])));
#pragma unroll
                for (int i = 0; i < BW; i += 2) {
                    if (i % 32 == 0) asm volatile("" ::: "memory");
                    const double2 ww = lds2(w + i);
                    m[t + i] = fma(f, ww.x, m[t + i]);
                    m[t + i + 1] = fma(f, ww.y, m[t + i + 1]);
                }
            }
            // rows [base, base + BW) are final for this tile; carry the rest down
#pragma unroll
            for (int i = 0; i < BW; ++i) sOut[tid * MLD + i] = m[i];
#pragma unroll
            for (int i = 0; i < KEEP; ++i) m[i] = m[i + BW];
            __syncthreads();
            store_out(base, BW);
        }
        // flush the carried rows [top + (hmax+1) BW, ... + KEEP)
        const int fbase = top + (hmax + 1) * BW;
        if (active) {
            double *Mw = M + (long long)mycol * ldm;
#pragma unroll
            for (int i = 0; i < KEEP; ++i)
                if (fbase + i < n) Mw[fbase + i] = m[i];
        }
    }
}

template <int BW, int TS> int launch_bc_back(Workspace *ws, double *M, long long ldm, int ncols) {
    constexpr int NWARP = 2;
    constexpr int NT = 32 * NWARP;
    const size_t smem = bc_back_smem<BW, TS>(NT);
    auto kern = bc_back_kernel<BW, TS, NWARP>;
    static bool attr = false;
    if (!attr) {
        CUEV_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr = true;
    }
    const int grid = div_up(ncols, NT);
    kern<<<grid, NT, smem, ws->stream>>>(ws->U, ws->n, M, ldm, ws->n, ncols); note_launch();
    CUEV_TRY(cudaGetLastError());
    return CUEV_OK;
}

} // namespace

int bc_back(Workspace *ws, double *M, long long ldm) {
    if (ws->n <= 2) return CUEV_OK;
    // register window R = TS + b - 1 rows: 79 rows keeps b = 32 spill-free (252 registers);
    // b = 64 needs the 64 reflector entries live as well and runs a shorter tile
    if (ws->b == 32) return launch_bc_back<32, 48>(ws, M, ldm, ws->n);
    if (ws->b == 64) return launch_bc_back<64, 16>(ws, M, ldm, ws->n);
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
