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
// window of TS+b rows, applying TS reflectors per step with compile-time register indices and
// reading w from shared memory as warp-wide broadcasts; the warps of a CTA run consecutive tiles
// as a pipeline (below).  b = 32 runs it with one lane per column, b = 64 with two (the window
// split between them).  (The reference slides a 256-row window per warp with cross-lane shuffles
// and only supports b = 32, backtransform.cu:16,35.)
//
// SBR-Back (M <- Q_s M).  Q_s = prod_j (I - Y_j T_j Y_j^T).  The reference applies each b-wide
// panel with two K = b GEMMs (backtransform.cu:210-230).  Here the panels of one DBBR k-block are
// merged into one compact-WY factor (I - Y_blk T_blk Y_blk^T, T_blk built in dbbr.cu), so the
// back-transform is three large DMMA GEMMs per k-block with K = rows or k.
#include "solver.cuh"

#include <algorithm>

namespace cuev {
namespace {

// One-element asynchronous copy (4 or 8 bytes); pred false: zero fill, nothing read.
template <typename T>
__device__ __forceinline__ void cp_async_el(T *smem, const T *gmem, bool pred) {
    constexpr int B = sizeof(T);
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(sa), "l"(gmem), "n"(B),
                 "r"(pred ? B : 0)
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
// 16-byte shared load into r[0 .. VN) (VN = 2 doubles or 4 floats)
__device__ __forceinline__ void lds16(const double *p, double *r) {
    const double2 v = *reinterpret_cast<const double2 *>(p);
    r[0] = v.x, r[1] = v.y;
}
__device__ __forceinline__ void lds16(const float *p, float *r) {
    const float4 v = *reinterpret_cast<const float4 *>(p);
    r[0] = v.x, r[1] = v.y, r[2] = v.z, r[3] = v.w;
}

// ---------------------------------------------------------------------------------------------
// Pipelined BC-Back, b = PB = 32.
//
// One thread per column gives only n threads of parallelism (n/32 warps: about 3.5 warps per SM
// at n = 16384), far too few to hide FP64 and shared-memory latency.  Here a
// CTA owns 32 columns and runs P warps over P consecutive sweep tiles at once, as a pipeline:
// warp p applies tile t while warp p+1 applies tile t-1 one hop block behind it.  Tile t emits
// its finished rows in hop order, chunk h = rows [top_t + 32h, top_t + 32h + 32); with a window
// of TS + 32 rows (KEEP = TS), the rows tile t-1 takes in at hop h are exactly chunk h of tile t,
// and the rows [top_{t-1}, top_t) it starts with have never been touched by a later tile, so they
// come straight from M.  Rows move between the warps of one round through shared-memory rings of
// two chunks (row-major [32 rows][32 columns]: lane c reads and writes column c, conflict-free);
// the last warp of a round hands its rows to the first warp of the next round through a global
// buffer X in the same row-major layout (256-byte coalesced rows), and only the warp that applies
// tile 0 writes M.  Each row of M is thus read once and written once; X is written and read once
// per round of P tiles.  Every wait is on a shared-memory counter, bounded by time, and all the
// warps that wait on one another belong to one CTA (so they are co-resident).
//
// Per hop a warp applies TS reflectors of length PB to its 32 columns: the reflector is loaded
// once from shared memory (16 broadcast 16-byte loads) into registers and used for both the dot
// product and the update, 64 FMAs per lane per reflector.
// Why the chunking is exact for any b: tile t-1's window at hop h is rows
// [top_t - TS + h b, top_t + h b + b), whose incoming rows [top_t + h b, + b) are tile t's chunk h,
// final for tile t once its hop h is done; and a reflector (s', h') of tile t - 1 commutes with
// every (s, h'') of tile t with h'' >= h' + 1 (their rows are disjoint), so running tile t - 1 one
// hop block behind tile t applies the reflectors in an order equivalent to the reverse order.
template <typename T, int TS, int P, int PB> struct PipeSmem {
    T w[P][2][TS][PB];        // reflectors of each warp's current and next hop block
    T ring[P - 1][2][PB][32]; // warp p -> warp p+1, two chunks of PB rows x 32 columns
    T xin[2][PB][32];         // warp 0: incoming rows (from X or, first tile, from M)
    int prod[P], cons[P];          // ring p: chunks written / chunks fully read (monotonic)
    int gprog;                     // chunks the last warp has written to X (monotonic)
    int abort_flag;                // set by a warp that gave up waiting
};

__device__ __forceinline__ int lds_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.cta.shared::cta.b32 %0, [%1];"
                 : "=r"(v)
                 : "r"((unsigned)__cvta_generic_to_shared(p))
                 : "memory");
    return v;
}
__device__ __forceinline__ void sts_release(int *p, int v) {
    asm volatile("st.release.cta.shared::cta.b32 [%0], %1;" ::"r"(
                     (unsigned)__cvta_generic_to_shared(p)),
                 "r"(v)
                 : "memory");
}
__device__ __forceinline__ void cp_async16_cg(void *smem, const void *gmem, bool pred) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem),
                 "r"(pred ? 16 : 0)
                 : "memory");
}

// Wait (all lanes) until *flag >= target.  Gives up after 2 s or when another warp gave up;
// returns false then (the caller returns after draining its copies).
__device__ __forceinline__ bool pipe_wait(const int *flag, int target, int *abort_flag,
                                          int *status, int where) {
    if (lds_acquire(flag) >= target) return true;
    const uint64_t t0 = global_ns();
    for (;;) {
        __nanosleep(32);
        if (lds_acquire(flag) >= target) return true;
        if (*(volatile int *)abort_flag) return false;
        if (global_ns() - t0 > wait_limit_ns(status)) {
            dev_fail(status, CUEV_ERR_TIMEOUT, where);
            *(volatile int *)abort_flag = 1;
            return false;
        }
    }
}

template <typename T, int TS, int P, int PB>
__global__ void __launch_bounds__(32 * P, 1)
    bc_back_pipe_kernel(const T *__restrict__ U, long long ldu, T *__restrict__ M,
                        long long ldm, T *__restrict__ X, int n, int ncols,
                        int *__restrict__ status) {
    static_assert(PB == 32, "band width 32 (b = 64 runs bc_back_pipe64_kernel)");
    constexpr int R = TS + PB;          // register window rows
    constexpr int VN = 16 / sizeof(T);  // elements per 16-byte copy or shared load
    extern __shared__ __align__(16) unsigned char pipe_smem_raw[];
    PipeSmem<T, TS, P, PB> &S = *reinterpret_cast<PipeSmem<T, TS, P, PB> *>(pipe_smem_raw);
    const int lane = threadIdx.x & 31, p = threadIdx.x >> 5;
    const int col0 = blockIdx.x * 32;
    const int mycol = min(col0 + lane, ncols - 1); // clamped: lanes past ncols never store to M
    const bool active = col0 + lane < ncols;
    const T *Mc = M + (long long)mycol * ldm;
    T *Xg = X + (size_t)blockIdx.x * n * 32; // row r of this CTA's columns: Xg[32 r + lane]
    const int nsweeps = n - 2;
    const int ntiles = (nsweeps + TS - 1) / TS;
    if (threadIdx.x < P) S.prod[threadIdx.x] = 0, S.cons[threadIdx.x] = 0;
    if (threadIdx.x == 0) S.gprog = 0, S.abort_flag = 0;
    __syncthreads(); // the only CTA-wide barrier: warps leave at different times

    // reflectors (s0 + j, hop of `rbase`): rows [rbase + j, rbase + j + PB) of U[:, s0 + j]
    auto stage_w = [&](int buf, int s0, int rbase) {
#pragma unroll
        for (int j = 0; j < TS; ++j) {
#pragma unroll
            for (int t = 0; t < PB / 32; ++t) {
                const int s = s0 + j, row = rbase + j + lane + 32 * t;
                const bool ok = (s < nsweeps) && (row < n);
                cp_async_el(&S.w[p][buf][j][lane + 32 * t], ok ? U + row + (long long)s * ldu : U,
                            ok);
            }
        }
    };
    // warp 0's incoming chunk: PB rows from X (coalesced 16-byte copies) ...
    auto stage_x = [&](int buf, int row0) {
#pragma unroll
        for (int q = 0; q < PB / VN; ++q) {
            const int e = (q * 32 + lane) * VN; // VN elements: row e / 32, columns e % 32 ..
            const int r = row0 + (e >> 5);
            const bool ok = r < n;
            cp_async16_cg(&S.xin[buf][e >> 5][e & 31], ok ? Xg + (size_t)r * 32 + (e & 31) : Xg,
                          ok);
        }
    };
    // ... or, for the first tile, from M (one column per lane; full chunks unpredicated)
    auto stage_m = [&](int buf, int row0) {
        if (row0 + PB <= n) {
#pragma unroll
            for (int i = 0; i < PB; ++i) cp_async_el(&S.xin[buf][i][lane], Mc + row0 + i, true);
        } else {
#pragma unroll
            for (int i = 0; i < PB; ++i) {
                const int r = row0 + i;
                const bool ok = r < n;
                cp_async_el(&S.xin[buf][i][lane], ok ? Mc + r : Mc, ok);
            }
        }
    };

    T m[R];
    int oseq = 0;  // chunks this warp has put into ring p (or X, for the last warp)
    int iseq = 0;  // chunks this warp has taken from ring p-1
    int xbase = 0; // warp 0: X sequence number of the current input tile's chunk 0
    bool ok = true;
    for (int t = ntiles - 1 - p; t >= 0 && ok; t -= P) {
        const int s0 = t * TS;
        const int top = s0 + 1;
        const int hmax = (n - 1 - top) / PB;
        const bool has_in = t + 1 <= ntiles - 1; // rows [top + TS, n) come from tile t + 1
        const int top_in = top + TS;
        const int hmax_in = has_in ? (n - 1 - top_in) / PB : -1;
        const bool first = !has_in; // only warp 0 of the first round
        const bool to_m = t == 0;
        const bool to_x = !to_m && p == P - 1;

        __syncwarp();
        stage_w(0, s0, top);
        if (p == 0) {
            if (first) {
                stage_m(0, top_in);
            } else if (hmax_in >= 0) {
                if (!pipe_wait(&S.gprog, xbase + 1, &S.abort_flag, status, -1)) { ok = false; break; }
                stage_x(0, top_in);
            }
        }
        cp_async_commit();
#pragma unroll
        for (int i = 0; i < TS; ++i) {
            const int row = top + i;
            const T v = Mc[min(row, n - 1)];
            m[i] = row < n ? v : T(0);
        }
        for (int h = 0; h <= hmax; ++h) {
            const int base = top + h * PB; // row of m[0]
            cp_async_wait<0>();
            __syncwarp();
            if (h < hmax) {
                stage_w((h + 1) & 1, s0, base + PB);
                if (p == 0) {
                    if (first) {
                        stage_m((h + 1) & 1, top_in + (h + 1) * PB);
                    } else if (h + 1 <= hmax_in) {
                        if (!pipe_wait(&S.gprog, xbase + h + 2, &S.abort_flag, status, -2)) {
                            ok = false;
                            break;
                        }
                        stage_x((h + 1) & 1, top_in + (h + 1) * PB);
                    }
                }
            }
            cp_async_commit();

            // incoming rows m[TS .. TS+32) = rows [base + TS, base + TS + 32) = chunk h of tile t+1
            if (p == 0) {
                if (first || h <= hmax_in) {
#pragma unroll
                    for (int i = 0; i < PB; ++i) m[TS + i] = S.xin[h & 1][i][lane];
                } else {
#pragma unroll
                    for (int i = 0; i < PB; ++i) m[TS + i] = T(0);
                }
            } else if (h <= hmax_in) {
                if (!pipe_wait(&S.prod[p - 1], iseq + 1, &S.abort_flag, status, -3)) {
                    ok = false;
                    break;
                }
                const int slot = iseq & 1;
#pragma unroll
                for (int i = 0; i < PB; ++i) m[TS + i] = S.ring[p - 1][slot][i][lane];
                __syncwarp();
                ++iseq;
                if (lane == 0) sts_release(&S.cons[p - 1], iseq);
            } else {
#pragma unroll
                for (int i = 0; i < PB; ++i) m[TS + i] = T(0);
            }

            // apply the tile's reflectors of this hop, last sweep first
            const T *W = &S.w[p][h & 1][0][0];
#pragma unroll
            for (int j = TS - 1; j >= 0; --j) {
                T wr[PB];
#pragma unroll
                for (int i = 0; i < PB; i += VN) lds16(W + j * PB + i, &wr[i]);
                T acc[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) acc[i] = wr[i] * m[j + i];
#pragma unroll
                for (int i = 8; i < PB; ++i) acc[i & 7] = fma(wr[i], m[j + i], acc[i & 7]);
                const T f = T(-2) * (((acc[0] + acc[1]) + (acc[2] + acc[3])) +
                                     ((acc[4] + acc[5]) + (acc[6] + acc[7])));
#pragma unroll
                for (int i = 0; i < PB; ++i) m[j + i] = fma(f, wr[i], m[j + i]);
            }

            // rows [base, base + PB) are final for this tile
            if (to_m) {
                if (active) {
                    T *Mw = M + (long long)mycol * ldm + base;
                    if (base + PB <= n) {
#pragma unroll
                        for (int i = 0; i < PB; ++i) Mw[i] = m[i];
                    } else {
#pragma unroll
                        for (int i = 0; i < PB; ++i)
                            if (base + i < n) Mw[i] = m[i];
                    }
                }
            } else if (to_x) {
                T *Xr = Xg + (size_t)base * 32 + lane;
                if (base + PB <= n) {
#pragma unroll
                    for (int i = 0; i < PB; ++i) __stcg(Xr + 32 * i, m[i]);
                } else {
#pragma unroll
                    for (int i = 0; i < PB; ++i)
                        if (base + i < n) __stcg(Xr + 32 * i, m[i]);
                }
                ++oseq;
                // The first warp of the next round reads these rows almost a whole tile later,
                // so the device-scope fence (the costliest step of a hop) is paid once per 8 hops
                // and at the end of the tile.
                if ((h & 7) == 7 || h == hmax) {
                    __threadfence();
                    __syncwarp();
                    if (lane == 0) sts_release(&S.gprog, oseq);
                }
            } else {
                if (!pipe_wait(&S.cons[p], oseq - 1, &S.abort_flag, status, -4)) {
                    ok = false;
                    break;
                }
                const int slot = oseq & 1;
#pragma unroll
                for (int i = 0; i < PB; ++i) S.ring[p][slot][i][lane] = m[i];
                __syncwarp();
                ++oseq;
                if (lane == 0) sts_release(&S.prod[p], oseq);
            }
#pragma unroll
            for (int i = 0; i < TS; ++i) m[i] = m[i + PB];
        }
        if (p == 0 && has_in) xbase += hmax_in + 1;
    }
    cp_async_wait<0>(); // leave no copy in flight, also on the early exits
}

// ---------------------------------------------------------------------------------------------
// Pipelined BC-Back for b = 64, two lanes per column.
//
// A 64-entry reflector and a TS + 64-row window do not fit one lane's registers together.  Here
// lanes c and c + 16 of a warp share column c: the upper lane (half 0) holds window rows
// [0, TS + 32), the lower lane (half 1) rows [32, TS + 64), so rows [32, 32 + TS) are held twice.
// Reflector j covers window rows [j, j + 64): its dot product is the upper lane's sum over its rows
// [j, j + 32) plus the lower lane's over its rows [j, j + 32) (window rows [32 + j, 64 + j)),
// joined by one shuffle (a + b in one lane and b + a in the other: the same value); then each
// lane updates all of its TS + 32 rows, so both copies of the shared rows see every update alike.
// Row k of a lane meets reflector entry k - j + 32 half: entry i of reflector j sits at position
// j + i of a zero-padded slot of TS + 64 entries, so both lanes run the same code with a per-lane
// offset, and entries outside [0, 64) read as zeros (an exact no-op in the update).
// After hop h the window's rows [0, 64) are final: each lane emits its rows [0, 32).  The next
// window's rows [0, TS) are the lower lane's rows [32, 32 + TS) (shuffled to the upper lane); the
// rest, and the lower lane's whole window, come from chunk h + 1 of tile t + 1.  The pipeline,
// rings and hand-off are those of the kernel above, with 64-row chunks of 16 columns.
template <int TS, int P> struct Pipe64Smem {
    static constexpr int WS = TS + 64; // zero-padded reflector slot
    double w[P][2][TS][WS];
    double ring[P - 1][2][64][16];
    double xin[2][64][16];
    int prod[P], cons[P];
    int gprog;
    int abort_flag;
};

// pipe_wait with the decision taken by the whole warp (the warp's lanes exchange values by
// shuffles, so none may leave the pipeline while the others go on)
__device__ __forceinline__ bool pipe_wait_warp(const int *flag, int target, int *abort_flag,
                                               int *status, int where) {
    if (__all_sync(0xffffffffu, lds_acquire(flag) >= target)) return true;
    const uint64_t t0 = global_ns();
    for (;;) {
        __nanosleep(32);
        if (__all_sync(0xffffffffu, lds_acquire(flag) >= target)) return true;
        const bool late = global_ns() - t0 > wait_limit_ns(status);
        if (__any_sync(0xffffffffu, late || *(volatile int *)abort_flag != 0)) {
            if ((threadIdx.x & 31) == 0) {
                if (late) dev_fail(status, CUEV_ERR_TIMEOUT, where);
                *(volatile int *)abort_flag = 1;
            }
            return false;
        }
    }
}

template <int TS, int P>
__global__ void __launch_bounds__(32 * P, 1)
    bc_back_pipe64_kernel(const double *__restrict__ U, long long ldu, double *__restrict__ M,
                          long long ldm, double *__restrict__ X, int n, int ncols,
                          int *__restrict__ status) {
    static_assert(TS % 2 == 0 && TS <= 32, "even tiles of at most 32 sweeps");
    using Smem = Pipe64Smem<TS, P>;
    constexpr int WS = Smem::WS;
    constexpr int R = TS + 32; // window rows per lane
    constexpr unsigned FULL = 0xffffffffu;
    extern __shared__ __align__(16) unsigned char pipe_smem_raw[];
    Smem &S = *reinterpret_cast<Smem *>(pipe_smem_raw);
    const int lane = threadIdx.x & 31, p = threadIdx.x >> 5;
    const int c = lane & 15, half = lane >> 4;
    const int col0 = blockIdx.x * 16;
    const int mycol = min(col0 + c, ncols - 1); // clamped: lanes past ncols never store to M
    const bool active = col0 + c < ncols;
    const double *Mc = M + (long long)mycol * ldm;
    double *Xg = X + (size_t)blockIdx.x * n * 16; // row r of this CTA's columns: Xg[16 r + c]
    const int nsweeps = n - 2;
    const int ntiles = (nsweeps + TS - 1) / TS;
    // staging writes only entries [j, j + 64) of slot j: the padding is zeroed once
    for (int i = threadIdx.x; i < P * 2 * TS * WS; i += blockDim.x) (&S.w[0][0][0][0])[i] = 0.0;
    if (threadIdx.x < P) S.prod[threadIdx.x] = 0, S.cons[threadIdx.x] = 0;
    if (threadIdx.x == 0) S.gprog = 0, S.abort_flag = 0;
    __syncthreads(); // the only CTA-wide barrier: warps leave at different times

    // reflectors (s0 + j, hop of `rbase`): rows [rbase + j, rbase + j + 64) of U[:, s0 + j]
    auto stage_w = [&](int buf, int s0, int rbase) {
#pragma unroll
        for (int j = 0; j < TS; ++j) {
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                const int i = lane + 32 * t;
                const int s = s0 + j, row = rbase + j + i;
                const bool okr = (s < nsweeps) && (row < n);
                cp_async_el(&S.w[p][buf][j][j + i], okr ? U + row + (long long)s * ldu : U, okr);
            }
        }
    };
    // warp 0's incoming chunk: 64 rows from X (16-byte copies) ...
    auto stage_x = [&](int buf, int row0) {
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int e = (q * 32 + lane) * 2; // row e / 16, columns e % 16 and e % 16 + 1
            const int r = row0 + (e >> 4);
            const bool okr = r < n;
            cp_async16_cg(&S.xin[buf][e >> 4][e & 15], okr ? Xg + (size_t)r * 16 + (e & 15) : Xg,
                          okr);
        }
    };
    // ... or, for the first tile, from M (each lane 32 rows of its column)
    auto stage_m = [&](int buf, int row0) {
        const int rb = row0 + 32 * half;
        if (row0 + 64 <= n) {
#pragma unroll
            for (int i = 0; i < 32; ++i)
                cp_async_el(&S.xin[buf][32 * half + i][c], Mc + rb + i, true);
        } else {
#pragma unroll
            for (int i = 0; i < 32; ++i) {
                const bool okr = rb + i < n;
                cp_async_el(&S.xin[buf][32 * half + i][c], okr ? Mc + rb + i : Mc, okr);
            }
        }
    };
    // incoming window rows [TS, TS + 64) = chunk rows [0, 64): the upper lane's rows [TS, TS + 32)
    // are chunk rows [0, 32), the lower lane's rows [0, TS + 32) chunk rows [32 - TS, 64)
    double m[R];
    auto take = [&](const double (*ch)[16]) {
#pragma unroll
        for (int k = 0; k < TS; ++k) {
            const double v = ch[32 - TS + k][c];
            m[k] = half ? v : m[k];
        }
#pragma unroll
        for (int k = TS; k < R; ++k) m[k] = ch[k - TS + 32 * half][c];
    };
    auto take_zero = [&]() {
#pragma unroll
        for (int k = 0; k < TS; ++k) m[k] = half ? 0.0 : m[k];
#pragma unroll
        for (int k = TS; k < R; ++k) m[k] = 0.0;
    };

    int oseq = 0;  // chunks this warp has put into ring p (or X, for the last warp)
    int iseq = 0;  // chunks this warp has taken from ring p-1
    int xbase = 0; // warp 0: X sequence number of the current input tile's chunk 0
    bool ok = true;
    for (int t = ntiles - 1 - p; t >= 0 && ok; t -= P) {
        const int s0 = t * TS;
        const int top = s0 + 1;
        const int hmax = (n - 1 - top) / 64;
        const bool has_in = t + 1 <= ntiles - 1; // rows [top + TS, n) come from tile t + 1
        const int top_in = top + TS;
        const int hmax_in = has_in ? (n - 1 - top_in) / 64 : -1;
        const bool first = !has_in; // only warp 0 of the first round
        const bool to_m = t == 0;
        const bool to_x = !to_m && p == P - 1;

        __syncwarp();
        stage_w(0, s0, top);
        if (p == 0) {
            if (first) {
                stage_m(0, top_in);
            } else if (hmax_in >= 0) {
                if (!pipe_wait_warp(&S.gprog, xbase + 1, &S.abort_flag, status, -1)) {
                    ok = false;
                    break;
                }
                stage_x(0, top_in);
            }
        }
        cp_async_commit();
        // the upper lane's rows [0, TS): rows no later tile touches (the lower lane's are
        // replaced by incoming rows)
#pragma unroll
        for (int i = 0; i < TS; ++i) {
            const int row = top + i;
            const double v = Mc[min(row, n - 1)];
            m[i] = row < n ? v : 0.0;
        }
        for (int h = 0; h <= hmax; ++h) {
            const int base = top + h * 64; // window row 0
            cp_async_wait<0>();
            __syncwarp();
            if (h < hmax) {
                stage_w((h + 1) & 1, s0, base + 64);
                if (p == 0) {
                    if (first) {
                        stage_m((h + 1) & 1, top_in + (h + 1) * 64);
                    } else if (h + 1 <= hmax_in) {
                        if (!pipe_wait_warp(&S.gprog, xbase + h + 2, &S.abort_flag, status, -2)) {
                            ok = false;
                            break;
                        }
                        stage_x((h + 1) & 1, top_in + (h + 1) * 64);
                    }
                }
            }
            cp_async_commit();

            if (p == 0) {
                if (first || h <= hmax_in)
                    take(S.xin[h & 1]);
                else
                    take_zero();
            } else if (h <= hmax_in) {
                if (!pipe_wait_warp(&S.prod[p - 1], iseq + 1, &S.abort_flag, status, -3)) {
                    ok = false;
                    break;
                }
                take(S.ring[p - 1][iseq & 1]);
                __syncwarp();
                ++iseq;
                if (lane == 0) sts_release(&S.cons[p - 1], iseq);
            } else {
                take_zero();
            }

            // apply the tile's reflectors of this hop, last sweep first
            const double *W = &S.w[p][h & 1][0][0] + 32 * half;
#pragma unroll
            for (int j = TS - 1; j >= 0; --j) {
                double wr[R];
#pragma unroll
                for (int k = 0; k < R; k += 2) {
                    const double2 v = lds2(W + j * WS + k);
                    wr[k] = v.x, wr[k + 1] = v.y;
                }
                double acc[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) acc[i] = wr[j + i] * m[j + i];
#pragma unroll
                for (int i = 8; i < 32; ++i) acc[i & 7] = fma(wr[j + i], m[j + i], acc[i & 7]);
                const double part = ((acc[0] + acc[1]) + (acc[2] + acc[3])) +
                                    ((acc[4] + acc[5]) + (acc[6] + acc[7]));
                const double f = -2.0 * (part + __shfl_xor_sync(FULL, part, 16));
#pragma unroll
                for (int k = 0; k < R; ++k) m[k] = fma(f, wr[k], m[k]);
            }

            // window rows [0, 64) are final for this tile: each lane's rows [0, 32)
            const int orow = base + 32 * half;
            if (to_m) {
                if (active) {
                    double *Mw = M + (long long)mycol * ldm + orow;
                    if (base + 64 <= n) {
#pragma unroll
                        for (int i = 0; i < 32; ++i) Mw[i] = m[i];
                    } else {
#pragma unroll
                        for (int i = 0; i < 32; ++i)
                            if (orow + i < n) Mw[i] = m[i];
                    }
                }
            } else if (to_x) {
                double *Xr = Xg + (size_t)orow * 16 + c;
                if (base + 64 <= n) {
#pragma unroll
                    for (int i = 0; i < 32; ++i) __stcg(Xr + 16 * i, m[i]);
                } else {
#pragma unroll
                    for (int i = 0; i < 32; ++i)
                        if (orow + i < n) __stcg(Xr + 16 * i, m[i]);
                }
                ++oseq;
                if ((h & 7) == 7 || h == hmax) {
                    __threadfence();
                    __syncwarp();
                    if (lane == 0) sts_release(&S.gprog, oseq);
                }
            } else {
                if (!pipe_wait_warp(&S.cons[p], oseq - 1, &S.abort_flag, status, -4)) {
                    ok = false;
                    break;
                }
                const int slot = oseq & 1;
#pragma unroll
                for (int i = 0; i < 32; ++i) S.ring[p][slot][32 * half + i][c] = m[i];
                __syncwarp();
                ++oseq;
                if (lane == 0) sts_release(&S.prod[p], oseq);
            }
            // next window rows [0, TS) = this window's rows [64, 64 + TS), the lower lane's
            // rows [32, 32 + TS)
#pragma unroll
            for (int k = 0; k < TS; ++k) m[k] = __shfl_xor_sync(FULL, m[32 + k], 16);
        }
        if (p == 0 && has_in) xbase += hmax_in + 1;
    }
    cp_async_wait<0>(); // leave no copy in flight, also on the early exits
}

// Columns [c0, c0 + ncols) of M (c0 a multiple of 32): CTA g owns columns c0 + 32 g .. + 31 and
// its hand-off rows in dc_S at the offset of its 32-column group, so launches over disjoint
// column ranges are independent and together do what one launch over all columns does.
// dst (rows x cols, ld ldd) = src (ld lds), FP64 <-> FP32.
template <typename S, typename D>
__global__ void convert_cols_kernel(const S *__restrict__ src, long long lds, D *__restrict__ dst,
                                    long long ldd, int rows, int cols) {
    const long long total = (long long)rows * cols;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long c = idx / rows, r = idx - c * rows;
        dst[r + c * ldd] = (D)src[r + c * lds];
    }
}

template <typename T, int TS, int P, int PB>
int launch_bc_back_pipe(Workspace *ws, cudaStream_t st, const T *U, T *M, long long ldm, int c0,
                        int ncols) {
    const int n = ws->n;
    if (ncols <= 0) return CUEV_OK;
    const size_t smem = sizeof(PipeSmem<T, TS, P, PB>);
    auto kern = bc_back_pipe_kernel<T, TS, P, PB>;
    CUEV_CHECK_STATUS(ensure_dyn_smem((const void *)kern, smem));
    const int grid = div_up(ncols, 32);
    // hand-off rows in dc_S (n x n doubles: room for either element type)
    T *Xc = reinterpret_cast<T *>(ws->dc_S) + (size_t)(c0 / 32) * n * 32;
    kern<<<grid, 32 * P, smem, st>>>(U, ws->n, M + (long long)c0 * ldm, ldm, Xc, n, ncols,
                                     ws->status);
    note_launch();
    CUEV_TRY(cudaGetLastError());
    return CUEV_OK;
}

template <int TS, int P>
int launch_bc_back_pipe64(Workspace *ws, cudaStream_t st, double *M, long long ldm, int c0,
                          int ncols) {
    const int n = ws->n;
    if (ncols <= 0) return CUEV_OK;
    const size_t smem = sizeof(Pipe64Smem<TS, P>);
    auto kern = bc_back_pipe64_kernel<TS, P>;
    CUEV_CHECK_STATUS(ensure_dyn_smem((const void *)kern, smem));
    const int grid = div_up(ncols, 16);
    // hand-off rows in dc_S: CTA g of this launch owns rows [0, n) x 16 at (c0 + 16 g) n
    double *Xc = ws->dc_S + (size_t)c0 * n;
    kern<<<grid, 32 * P, smem, st>>>(ws->U, ws->n, M + (long long)c0 * ldm, ldm, Xc, n, ncols,
                                     ws->status);
    note_launch();
    CUEV_TRY(cudaGetLastError());
    return CUEV_OK;
}

// Columns owned by one BC-back CTA.
int bc_back_group_cols(const Workspace *ws) { return ws->b == 64 ? 16 : 32; }

// One SBR-back product.  In the precision form (ws->mixed) products of at least 2^30
// multiply-adds run on the int8 tensor cores at FP32-level accuracy (MIXED_SLICES slices);
// smaller ones cost more in slicing than they save.
int bt_gemm(Workspace *ws, int ta, int tb, int m, int n, int k, double alpha, const double *A,
            long long lda, const double *B, long long ldb, double beta, double *C, long long ldc) {
    if (ws->mixed && alpha != 0.0 && (double)m * n * k >= 1073741824.0 &&
        i8_gemm_scratch_bytes(m, n, k, MIXED_SLICES) <= ws->i8_scratch_bytes)
        return i8_dgemm(ta, tb, 0, m, n, k, MIXED_SLICES, alpha, A, lda, B, ldb, beta, C, ldc, 0,
                        ws->i8_scratch, ws->status, ws->stream);
    return ws_gemm(ws, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

// BC-back over columns [c0, c0 + ncols): b = 32 runs 8 warps on 14-sweep tiles (46-row register
// window; at n = 16384 tiles of 12, 13, 14, 15 and 16 sweeps took 587, 585, 574, 599 and 619 ms,
// 8 sweeps or 10 warps spill); b = 64 runs 8 warps on 8-sweep tiles, two lanes per column (a
// 40-row window each; 205 KB of shared memory with the zero-padded reflectors and 64 x 16 rings).
int launch_bc_back_cols(Workspace *ws, cudaStream_t st, double *M, long long ldm, int c0,
                        int ncols) {
    if (ncols <= 0) return CUEV_OK;
    if (ws->b == 32 && ws->fp32) {
        // FP32 entry: the column range in FP32 (Mf, ld n) against U's float copy (made by
        // bc_back_prepare), 16 warps per CTA (the float window leaves the registers for them)
        const int n = ws->n;
        const int blocks = std::min(4 * num_sms(), div_up((long long)n * ncols, 256));
        convert_cols_kernel<<<blocks, 256, 0, st>>>(M + (long long)c0 * ldm, ldm,
                                                    ws->Mf + (long long)c0 * n, n, n, ncols);
        note_launch();
        CUEV_TRY(cudaGetLastError());
        CUEV_CHECK_STATUS(
            (launch_bc_back_pipe<float, 16, 16, 32>(ws, st, ws->Uf, ws->Mf, n, c0, ncols)));
        convert_cols_kernel<<<blocks, 256, 0, st>>>(ws->Mf + (long long)c0 * n, n,
                                                    M + (long long)c0 * ldm, ldm, n, ncols);
        note_launch();
        CUEV_TRY(cudaGetLastError());
        return CUEV_OK;
    }
    if (ws->b == 32) return launch_bc_back_pipe<double, 14, 8, 32>(ws, st, ws->U, M, ldm, c0, ncols);
    if (ws->b == 64) return launch_bc_back_pipe64<8, 8>(ws, st, M, ldm, c0, ncols);
    return CUEV_ERR_INVALID;
}

// The FP32 entry's BC-back reads a float copy of the reflectors.
int bc_back_prepare(Workspace *ws, cudaStream_t st) {
    if (!(ws->fp32 && ws->b == 32) || ws->n <= 2) return CUEV_OK;
    const int n = ws->n;
    const int blocks = std::min(4 * num_sms(), div_up((long long)n * n, 256));
    convert_cols_kernel<<<blocks, 256, 0, st>>>(ws->U, n, ws->Uf, n, n, n);
    note_launch();
    CUEV_TRY(cudaGetLastError());
    return CUEV_OK;
}

// M <- Q_s M on ncols columns of M, with X (w x ncols) and X2 (w x ncols) as scratch.
int sbr_back_cols(Workspace *ws, double *M, long long ldm, int ncols, double *X, double *X2) {
    const int n = ws->n, b = ws->b, k = ws->k;
    const long long ld = n;
    if (ncols <= 0) return CUEV_OK;
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
        CUEV_CHECK_STATUS(bt_gemm(ws, 1, 0, w, ncols, rows, 1.0, Yb, ld, Mb, ldm, 0.0, X, w));
        CUEV_CHECK_STATUS(bt_gemm(ws, 0, 0, w, ncols, w, 1.0, Tb, k, X, w, 0.0, X2, w));
        CUEV_CHECK_STATUS(bt_gemm(ws, 0, 0, rows, ncols, w, -1.0, Yb, ld, X2, w, 1.0, Mb, ldm));
    }
    return CUEV_OK;
}

} // namespace

int bc_back(Workspace *ws, double *M, long long ldm) {
    if (ws->n <= 2) return CUEV_OK;
    CUEV_CHECK_STATUS(bc_back_prepare(ws, ws->stream));
    return launch_bc_back_cols(ws, ws->stream, M, ldm, 0, ws->n);
}

int sbr_back(Workspace *ws, double *M, long long ldm) {
    // scratch: X = Y_blk^T M and X2 = T_blk X, both (w x n) with w <= min(k, n), in the D&C
    // buffers (free once the tridiagonal eigenvectors are formed)
    return sbr_back_cols(ws, M, ldm, ws->n, ws->dc_S, ws->dc_Q2);
}

// Both stages multiply M from the left, so M's columns are independent.  BC-back runs one CTA per
// 32 columns and one CTA per SM; when its grid ends in a partial wave (n = 16384: 512 CTAs, 3.46
// waves on 148 SMs) the columns of the whole waves go first, then the last wave runs on the
// high-priority side stream while the SBR-back of the finished columns fills the idle SMs, and
// the SBR-back of the last columns follows.  The early SBR-back uses dc_T and dc_Q2 as scratch:
// the late BC-back's hand-off rows live in dc_S.
int back_transform(Workspace *ws, double *M, long long ldm, cudaEvent_t bc_end) {
    const int n = ws->n;
    if (n > 2) CUEV_CHECK_STATUS(bc_back_prepare(ws, ws->stream));
    const int gw = bc_back_group_cols(ws);
    const int groups = div_up(std::max(n, 1), gw);
    const int full = groups / num_sms() * num_sms(); // groups in whole waves
    // host-buffer entry: contiguous columns only (ld = n)
    double *hV = (ws->host_evec && ldm == n) ? ws->host_evec : nullptr;
    const size_t col_bytes = sizeof(double) * (size_t)n;
    if (n <= 2 || full == 0 || full == groups || !ws->side) {
        if (n > 2) CUEV_CHECK_STATUS(launch_bc_back_cols(ws, ws->stream, M, ldm, 0, n));
        if (bc_end) CUEV_TRY(cudaEventRecord(bc_end, ws->stream));
        CUEV_CHECK_STATUS(sbr_back(ws, M, ldm));
        if (hV) CUEV_TRY(cudaMemcpyAsync(hV, M, col_bytes * n, cudaMemcpyDeviceToHost, ws->stream));
        return CUEV_OK;
    }
    const int c1 = full * gw;
    CUEV_CHECK_STATUS(launch_bc_back_cols(ws, ws->stream, M, ldm, 0, c1));
    CUEV_TRY(cudaEventRecord(ws->ev_a, ws->stream));
    CUEV_TRY(cudaStreamWaitEvent(ws->side, ws->ev_a, 0));
    int st = launch_bc_back_cols(ws, ws->side, M, ldm, c1, n - c1);
    if (st == CUEV_OK && bc_end && cudaEventRecord(bc_end, ws->side) != cudaSuccess)
        st = CUEV_ERR_CUDA;
    if (st == CUEV_OK && cudaEventRecord(ws->ev_b, ws->side) != cudaSuccess) st = CUEV_ERR_CUDA;
    if (st == CUEV_OK) st = sbr_back_cols(ws, M, ldm, c1, ws->dc_T, ws->dc_Q2);
    if (st == CUEV_OK && hV) {
        // columns [0, c1) are final: copy them out on the side stream (after its BC-back) while
        // the main stream computes the last columns
        if (cudaEventRecord(ws->ev_c, ws->stream) != cudaSuccess ||
            cudaStreamWaitEvent(ws->side, ws->ev_c, 0) != cudaSuccess ||
            cudaMemcpyAsync(hV, M, col_bytes * c1, cudaMemcpyDeviceToHost, ws->side) !=
                cudaSuccess ||
            cudaEventRecord(ws->ev_d, ws->side) != cudaSuccess)
            st = CUEV_ERR_CUDA;
    }
    if (st == CUEV_OK && cudaStreamWaitEvent(ws->stream, ws->ev_b, 0) != cudaSuccess)
        st = CUEV_ERR_CUDA;
    if (st == CUEV_OK) st = sbr_back_cols(ws, M + (long long)c1 * ldm, ldm, n - c1, ws->dc_T, ws->dc_Q2);
    if (st == CUEV_OK && hV) {
        if (cudaMemcpyAsync(hV + (size_t)c1 * n, M + (long long)c1 * ldm, col_bytes * (n - c1),
                            cudaMemcpyDeviceToHost, ws->stream) != cudaSuccess ||
            cudaStreamWaitEvent(ws->stream, ws->ev_d, 0) != cudaSuccess)
            st = CUEV_ERR_CUDA;
    }
    if (st != CUEV_OK) {
        // nothing of this call may outlive it on the side stream: join the side stream back into
        // the caller's stream (an event, not a host synchronisation, which would be illegal while
        // the caller's stream is being captured)
        if (cudaEventRecord(ws->ev_b, ws->side) == cudaSuccess)
            cudaStreamWaitEvent(ws->stream, ws->ev_b, 0);
        return st;
    }
    return CUEV_OK;
}

} // namespace cuev
