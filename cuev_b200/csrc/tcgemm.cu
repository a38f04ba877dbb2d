// int8 tensor-core GEMM for sm_100a (tcgen05.mma.kind::i8, TMA, TMEM) and the FP64 slicing
// around it (the method is described in tcgemm.cuh).
//
// Kernel shape: a persistent CTA per SM (up to the tile count), 10 warps:
//   warp 0     TMA producer: 128 x 128-byte tile of an A slice and BN x 128-byte tile of a B
//              slice per stage (SWIZZLE_128B, K-major), into a STAGES-deep shared-memory ring;
//   warp 1     allocates TMEM (two BN-column int32 accumulators) and, on one lane, issues the
//              tcgen05.mma (M = 128, N = BN, K = 32 bytes; four per stage) and the commits that
//              free a stage and that hand a finished accumulator to the epilogue;
//   warps 2-9  epilogue: tcgen05.ld of the accumulator (warp w reads TMEM lanes 32 (w % 4) ..),
//              release of the buffer, then C += 2^(e_r + f_c - 7d) alpha L_d in FP64 (the first
//              level of a tile writes alpha 2^(...) L_2 + beta C).
// One "group" is a run of (slice pair, 128-wide K chunk) items accumulated into one TMEM buffer;
// its length is capped at 1040 chunks, so |sum| <= 1040 * 128 * 127^2 < 2^31.  The two buffers let
// the MMA of group g + 1 run while the epilogue drains group g.  Every mbarrier wait is bounded
// (2 s): a wait that gives up records CUEV_ERR_TIMEOUT, every role stops, copies and MMAs in
// flight are waited for (bounded), TMEM is freed and the kernel returns.
#include "tcgemm.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

namespace cuev {
namespace {

constexpr int TC_BM = 128;       // tile rows (TMEM lanes)
constexpr int TC_BK = 128;       // K bytes per stage = one 128-byte swizzle row
constexpr int TC_THREADS = 320;  // 10 warps
constexpr int TC_GROUP_MAX = 1040;
constexpr int TC_GM = 16;        // tile rasterisation: 16 row tiles per column sweep

template <int BN> struct TcCfg {
    static constexpr int STAGES = BN == 256 ? 4 : 6;
    static constexpr int A_BYTES = TC_BM * TC_BK;
    static constexpr int B_BYTES = BN * TC_BK;
    static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
    static constexpr int SMEM = STAGES * STAGE_BYTES + 1024; // + alignment slack
    static constexpr int TMEM_COLS = 2 * BN;
};

// ---- PTX wrappers ------------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(bar), "r"(parity)
                 : "memory");
    return ok != 0;
}

// Bounded wait for the phase of parity `parity` of `bar`.  Gives up after 2 s (the status words'
// limit, lowered only by failure-path tests) or when another role has given up, recording
// CUEV_ERR_TIMEOUT.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int *abort_flag,
                                          int *status, int where) {
    uint64_t t0 = 0;
    for (uint32_t i = 0;; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 31u) == 31u) {
            if (*abort_flag) return false;
            const uint64_t t = global_ns();
            if (t0 == 0) {
                t0 = t;
            } else if (t - t0 > wait_limit_ns(status)) {
                *abort_flag = 1;
                dev_fail(status, CUEV_ERR_TIMEOUT, where);
                return false;
            }
        }
    }
}

// Bounded wait that ignores the abort flag (draining copies and MMAs already issued).
__device__ __forceinline__ void mbar_drain(uint32_t bar, uint32_t parity) {
    const uint64_t t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > 2000000000ull) return;
}

// Lane 0 waits (bounded); the outcome is the warp's.
__device__ __forceinline__ bool warp_wait(uint32_t bar, uint32_t parity, volatile int *abort_flag,
                                          int *status, int where) {
    int ok = 1;
    if ((threadIdx.x & 31) == 0) ok = mbar_wait(bar, parity, abort_flag, status, where) ? 1 : 0;
    ok = __shfl_sync(0xffffffffu, ok, 0);
    __syncwarp();
    return ok != 0;
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, uint32_t bar,
                                            int c0, int c1, int c2) {
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(dst),
                 "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(c0), "r"(c1), "r"(c2)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// K-major operand tile with 128-byte swizzle: rows of 128 bytes, 8-row atoms 1024 bytes apart
// (stride byte offset 1024, leading byte offset unused for swizzled K-major: 16), descriptor
// version 1 (bits 46-47), layout SWIZZLE_128B = 2 (bits 61-63).
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)(16u >> 4) << 16;
    d |= (uint64_t)(1024u >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// Instruction descriptor, kind::i8: D s32 (bits 4-5 = 2), A and B signed int8 (bits 7-9, 10-12
// = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28.
template <int BN> __device__ __forceinline__ uint32_t idesc_i8() {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
           ((uint32_t)(TC_BM >> 4) << 24);
}

__device__ __forceinline__ void umma_i8(uint32_t dtmem, uint64_t adesc, uint64_t bdesc,
                                        uint32_t idesc, uint32_t accumulate) {
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
                 "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
                 : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32"
                 " {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15,"
                 " %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31},"
                 " [%32];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                   "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                   "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]),
                   "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
                   "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
                   "=r"(v[30]), "=r"(v[31])
                 : "r"(taddr)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld_wait() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// 2^e as a double for e in [-1022, 1023] (clamped; the slicing keeps exponents well inside).
__device__ __forceinline__ double pow2i(int e) {
    e = max(-1022, min(1023, e));
    return __longlong_as_double((long long)(e + 1023) << 52);
}

// ---- work schedule -----------------------------------------------------------------------------

struct TcArgs {
    double *C;
    long long ldc;
    const int *ea, *eb; // row exponents of op(A) (m) and of op(B)^T (n)
    int *status;
    int m, n, k_chunks;
    int sa, sb, levels;
    int mt, nt;         // tile counts
    int c_lower;
    int ntiles;         // tiles actually computed
    double alpha, beta;
};

// Tile index -> (tm, tn): groups of TC_GM row tiles, column-major inside a group, so that a wave
// of CTAs shares a compact block of A rows and B columns in L2.  With c_lower the tiles wholly
// above the diagonal are skipped by the caller's count (see tile_of).
__device__ __forceinline__ void tile_of(const TcArgs &a, int BN, int t, int &tm, int &tn) {
    if (!a.c_lower) {
        const int per_group = TC_GM * a.nt;
        const int g = t / per_group, w = t % per_group;
        const int rows_in_g = min(TC_GM, a.mt - g * TC_GM);
        tn = w / rows_in_g;
        tm = g * TC_GM + w % rows_in_g;
        return;
    }
    // lower triangle: column tile tn holds the row tiles tm >= tm0(tn) = floor(tn BN / BM)
    int acc = 0;
    for (tn = 0; tn < a.nt; ++tn) {
        const int tm0 = (tn * BN) / TC_BM;
        const int cnt = max(0, a.mt - tm0);
        if (t < acc + cnt) {
            tm = tm0 + (t - acc);
            return;
        }
        acc += cnt;
    }
    tm = tn = 0;
}

template <int BN>
__global__ void __launch_bounds__(TC_THREADS, 1)
    i8_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                   const TcArgs a) {
    using Cfg = TcCfg<BN>;
    constexpr int S = Cfg::STAGES;
    extern __shared__ uint8_t tc_smem_raw[];
    __shared__ __align__(8) uint64_t bar_full[S], bar_empty[S], bar_tfull[2], bar_tempty[2],
        bar_done;
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t base = (smem_u32(tc_smem_raw) + 1023u) & ~1023u;

    if (threadIdx.x == 0) {
        for (int i = 0; i < S; ++i) {
            mbar_init(smem_u32(&bar_full[i]), 1);
            mbar_init(smem_u32(&bar_empty[i]), 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(smem_u32(&bar_tfull[i]), 1);
            mbar_init(smem_u32(&bar_tempty[i]), 8);
        }
        mbar_init(smem_u32(&bar_done), 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"((uint32_t)Cfg::TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    volatile int *abort_v = &abort_flag;

    if (warp == 0) {
        // ---------------- TMA producer (lane 0 issues; the warp stays converged) -------------
        if (lane == 0) {
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmA))
                         : "memory");
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmB))
                         : "memory");
        }
        uint32_t it = 0;
        bool ok = true;
        for (int t = blockIdx.x; ok && t < a.ntiles; t += gridDim.x) {
            int tm, tn;
            tile_of(a, BN, t, tm, tn);
            for (int d = 2; ok && d <= a.levels + 1; ++d) {
                const int p_lo = max(1, d - a.sb), p_hi = min(d - 1, a.sa);
                const int items = (p_hi - p_lo + 1) * a.k_chunks;
                for (int x = 0; x < items; ++x, ++it) {
                    const uint32_t st = it % S;
                    ok = warp_wait(smem_u32(&bar_empty[st]), ((it / S) & 1u) ^ 1u, abort_v,
                                   a.status, 1);
                    if (!ok) break;
                    if (lane == 0) {
                        const int p = p_lo + x / a.k_chunks, kc = x % a.k_chunks;
                        const uint32_t sa = base + st * Cfg::STAGE_BYTES;
                        const uint32_t fb = smem_u32(&bar_full[st]);
                        mbar_expect_tx(fb, Cfg::STAGE_BYTES);
                        tma_load_3d(sa, &tmA, fb, kc * TC_BK, tm * TC_BM, p - 1);
                        tma_load_3d(sa + Cfg::A_BYTES, &tmB, fb, kc * TC_BK, tn * BN, d - p - 1);
                    }
                    __syncwarp();
                }
            }
        }
        // copies still in flight land before the CTA can leave (the last S issues, one per stage)
        if (lane == 0)
            for (uint32_t j = (it > (uint32_t)S ? it - S : 0u); j < it; ++j)
                mbar_drain(smem_u32(&bar_full[j % S]), (j / S) & 1u);
        __syncwarp();
    } else if (warp == 1) {
        // ---------------- MMA issuer (lane 0 issues; the warp stays converged) ---------------
        const uint32_t idesc = idesc_i8<BN>();
        uint32_t it = 0, gc = 0;
        bool ok = true;
        for (int t = blockIdx.x; ok && t < a.ntiles; t += gridDim.x) {
            for (int d = 2; ok && d <= a.levels + 1; ++d) {
                const int p_lo = max(1, d - a.sb), p_hi = min(d - 1, a.sa);
                const int items = (p_hi - p_lo + 1) * a.k_chunks;
                for (int g0 = 0; ok && g0 < items; g0 += TC_GROUP_MAX, ++gc) {
                    const int g1 = min(items, g0 + TC_GROUP_MAX);
                    const uint32_t buf = gc & 1u;
                    ok = warp_wait(smem_u32(&bar_tempty[buf]), ((gc >> 1) & 1u) ^ 1u, abort_v,
                                   a.status, 2);
                    if (!ok) break;
                    tc_fence_after();
                    const uint32_t dt = tmem + buf * BN;
                    for (int x = g0; x < g1; ++x, ++it) {
                        const uint32_t st = it % S;
                        ok = warp_wait(smem_u32(&bar_full[st]), (it / S) & 1u, abort_v, a.status,
                                       3);
                        if (!ok) break;
                        tc_fence_after();
                        if (lane == 0) {
                            const uint32_t sa = base + st * Cfg::STAGE_BYTES;
                            const uint32_t sb = sa + Cfg::A_BYTES;
#pragma unroll
                            for (int j = 0; j < TC_BK / 32; ++j)
                                umma_i8(dt, umma_desc_sw128(sa + 32 * j),
                                        umma_desc_sw128(sb + 32 * j), idesc,
                                        (x > g0 || j > 0) ? 1u : 0u);
                            umma_commit(smem_u32(&bar_empty[st]));
                        }
                        __syncwarp();
                    }
                    if (!ok) break;
                    if (lane == 0) umma_commit(smem_u32(&bar_tfull[buf]));
                    __syncwarp();
                }
            }
        }
        // every MMA issued so far has finished once this commit's barrier flips
        if (lane == 0) {
            umma_commit(smem_u32(&bar_done));
            mbar_drain(smem_u32(&bar_done), 0);
        }
        __syncwarp();
    } else {
        // ---------------- epilogue (warps 2..9) ----------------
        const int ew = warp - 2;
        const int quad = warp & 3;       // TMEM lanes 32 quad .. 32 quad + 31
        const int half = ew >> 2;        // column half of the tile
        constexpr int NCH = BN / 64;     // 32-column chunks per warp
        uint32_t gc = 0;
        bool ok = true;
        for (int t = blockIdx.x; ok && t < a.ntiles; t += gridDim.x) {
            int tm, tn;
            tile_of(a, BN, t, tm, tn);
            const int row = tm * TC_BM + quad * 32 + lane;
            const bool row_ok = row < a.m;
            const int col0 = tn * BN + half * (BN / 2);
            const int er = row_ok ? a.ea[row] : 0;
            double *crow = a.C + (row_ok ? row : 0);
            bool first = true;
            for (int d = 2; ok && d <= a.levels + 1; ++d) {
                const int p_lo = max(1, d - a.sb), p_hi = min(d - 1, a.sa);
                const int items = (p_hi - p_lo + 1) * a.k_chunks;
                for (int g0 = 0; g0 < items; g0 += TC_GROUP_MAX, ++gc) {
                    const uint32_t buf = gc & 1u;
                    const bool mine = mbar_wait(smem_u32(&bar_tfull[buf]), (gc >> 1) & 1u,
                                                abort_v, a.status, 4);
                    ok = __all_sync(0xffffffffu, mine);
                    if (!ok) break;
                    tc_fence_after();
                    const uint32_t ta = tmem + ((uint32_t)(quad * 32) << 16) + buf * BN +
                                        half * (BN / 2);
                    const double rs = a.alpha * pow2i(er - 7 * d);
#pragma unroll 1
                    for (int c = 0; c < NCH; ++c) {
                        uint32_t v[32];
                        tmem_ld32(ta + 32 * c, v);
                        tmem_ld_wait();
                        if (c == NCH - 1) {
                            // the accumulator is free for the next group once its last chunk is
                            // in registers
                            tc_fence_before();
                            __syncwarp();
                            if (lane == 0) mbar_arrive(smem_u32(&bar_tempty[buf]));
                        }
                        const int cb = col0 + 32 * c;
                        const int fe = (cb + lane < a.n) ? a.eb[cb + lane] : 0;
                        // all 32 reads of C first (independent, in flight together), then the
                        // updates: interleaving them would serialise every read behind the
                        // previous store (they may alias as far as the compiler knows)
                        const bool need_old = !first || a.beta != 0.0;
#pragma unroll
                        for (int h = 0; h < 32; h += 16) {
                            double old[16];
#pragma unroll
                            for (int r = 0; r < 16; ++r) {
                                const int col = cb + h + r;
                                const bool ok_el =
                                    row_ok && col < a.n && !(a.c_lower && row < col);
                                old[r] = (need_old && ok_el) ? crow[(long long)col * a.ldc] : 0.0;
                            }
#pragma unroll
                            for (int r = 0; r < 16; ++r) {
                                const int col = cb + h + r;
                                const int fc = __shfl_sync(0xffffffffu, fe, h + r);
                                if (!row_ok || col >= a.n || (a.c_lower && row < col)) continue;
                                const double val = (double)(int)v[h + r] * rs * pow2i(fc);
                                crow[(long long)col * a.ldc] =
                                    first ? (a.beta != 0.0 ? val + a.beta * old[r] : val)
                                          : old[r] + val;
                            }
                        }
                    }
                    first = false;
                }
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"((uint32_t)Cfg::TMEM_COLS)
                     : "memory");
    }
}

// ---- slicing -----------------------------------------------------------------------------------

constexpr int SL_R = 32, SL_K = 128, SL_THREADS = 256;

// Stage the 32 x 128 tile (r0.., k0..) of op(X) in shared memory, zero outside rows x k.
__device__ __forceinline__ void load_slice_tile(const double *__restrict__ X, long long ldx,
                                                int src, int rows, int k, int r0, int k0,
                                                double (*t)[SL_K + 1]) {
    // read along whichever index is contiguous in X; a symmetric tile wholly above the diagonal
    // is a K-major read of the stored lower triangle
    const bool kfast = src == I8_SRC_KMAJ || (src == I8_SRC_SYML && r0 + SL_R - 1 < k0);
    for (int idx = threadIdx.x; idx < SL_R * SL_K; idx += SL_THREADS) {
        int r, kk;
        if (kfast) {
            kk = idx % SL_K;
            r = idx / SL_K;
        } else {
            r = idx % SL_R;
            kk = idx / SL_R;
        }
        const int gr = r0 + r, gk = k0 + kk;
        double v = 0.0;
        if (gr < rows && gk < k) {
            if (src == I8_SRC_KMAJ)
                v = X[gk + (long long)gr * ldx];
            else if (src == I8_SRC_RMAJ)
                v = X[gr + (long long)gk * ldx];
            else
                v = gr >= gk ? X[gr + (long long)gk * ldx] : X[gk + (long long)gr * ldx];
        }
        t[r][kk] = v;
    }
}

__global__ void __launch_bounds__(SL_THREADS)
    i8_rowmax_kernel(const double *__restrict__ X, long long ldx, int src, int rows, int k,
                     unsigned long long *__restrict__ rmax) {
    __shared__ double t[SL_R][SL_K + 1];
    const int k0 = blockIdx.x * SL_K, r0 = blockIdx.y * SL_R;
    load_slice_tile(X, ldx, src, rows, k, r0, k0, t);
    __syncthreads();
    const int r = threadIdx.x >> 3, seg = threadIdx.x & 7;
    double m = 0.0;
#pragma unroll
    for (int i = 0; i < 16; ++i) m = fmax(m, fabs(t[r][seg * 16 + i]));
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, 1));
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, 2));
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, 4));
    // non-negative doubles order like their bit patterns
    if (seg == 0 && r0 + r < rows && m > 0.0)
        atomicMax(&rmax[r0 + r], (unsigned long long)__double_as_longlong(m));
}

// e_r with max_r < 2^e_r (frexp exponent); 0 for an all-zero row.
__global__ void i8_exp_kernel(const unsigned long long *__restrict__ rmax, int rows,
                              int *__restrict__ exps) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
        const double m = __longlong_as_double((long long)rmax[r]);
        int e = 0;
        if (m > 0.0) frexp(m, &e);
        exps[r] = e;
    }
}

__global__ void __launch_bounds__(SL_THREADS)
    i8_slice_kernel(const double *__restrict__ X, long long ldx, int src, int rows, int k, int s,
                    const int *__restrict__ exps, int8_t *__restrict__ out, long long k_ld,
                    size_t slice_stride) {
    __shared__ double t[SL_R][SL_K + 1];
    const int k0 = blockIdx.x * SL_K, r0 = blockIdx.y * SL_R;
    load_slice_tile(X, ldx, src, rows, k, r0, k0, t);
    __syncthreads();
    const int r = threadIdx.x >> 3, seg = threadIdx.x & 7;
    const int gr = r0 + r;
    if (gr >= rows) return;
    // x 2^-e is exact (a power-of-two scaling); every later step (x *= 128, x -= trunc(x)) is
    // exact as well, so the slices are an error-free split of the leading 7 s bits
    const double sc = pow2i(-exps[gr]);
    double x[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = t[r][seg * 16 + i] * sc;
    int8_t *o = out + (long long)gr * k_ld + k0 + seg * 16;
    for (int p = 0; p < s; ++p) {
        uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            x[i] *= 128.0;
            const double a = trunc(x[i]); // |x| < 128, so |a| <= 127
            x[i] -= a;
            w[i >> 2] |= ((uint32_t)(int)a & 0xFFu) << (8 * (i & 3));
        }
        *reinterpret_cast<uint4 *>(o + p * slice_stride) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// ---- host side ---------------------------------------------------------------------------------

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::mutex g_encode_mu;

int get_encode(PFN_cuTensorMapEncodeTiled_v12000 *out) {
    std::lock_guard<std::mutex> lk(g_encode_mu);
    if (!g_encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        const cudaError_t e =
            cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) {
            cudaGetLastError();
            set_last_message("int8 tensor-core GEMM: cuTensorMapEncodeTiled not available");
            return CUEV_ERR_CUDA;
        }
        g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    *out = g_encode;
    return CUEV_OK;
}

// 3-D map over an operand's slices: (k_ld bytes, rows, s), box (128, box_rows, 1), 128-byte swizzle.
int make_map(const I8Operand &op, int box_rows, CUtensorMap *map) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = nullptr;
    CUEV_CHECK_STATUS(get_encode(&enc));
    const cuuint64_t dims[3] = {(cuuint64_t)op.k_ld, (cuuint64_t)op.rows, (cuuint64_t)op.s};
    const cuuint64_t strides[2] = {(cuuint64_t)op.k_ld, (cuuint64_t)op.slice_stride};
    const cuuint32_t box[3] = {(cuuint32_t)TC_BK, (cuuint32_t)box_rows, 1u};
    const cuuint32_t estr[3] = {1u, 1u, 1u};
    const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, (void *)op.data, dims, strides,
                           box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_last_message("int8 tensor-core GEMM: tensor map encoding failed");
        return CUEV_ERR_CUDA;
    }
    return CUEV_OK;
}

template <int BN> int launch_i8(const CUtensorMap &ma, const CUtensorMap &mb, const TcArgs &a,
                                int grid, cudaStream_t st) {
    auto kern = i8_gemm_kernel<BN>;
    CUEV_CHECK_STATUS(ensure_dyn_smem((const void *)kern, TcCfg<BN>::SMEM));
    kern<<<grid, TC_THREADS, TcCfg<BN>::SMEM, st>>>(ma, mb, a);
    note_launch();
    CUEV_TRY(cudaGetLastError());
    return CUEV_OK;
}

long long round_up(long long x, long long m) { return (x + m - 1) / m * m; }

} // namespace

size_t i8_operand_bytes(int rows, int k, int s) {
    const long long k_ld = round_up(std::max(k, 1), TC_BK);
    const size_t slice = align256((size_t)k_ld * std::max(rows, 1));
    return slice * (size_t)s + align256(sizeof(int) * (size_t)std::max(rows, 1)) +
           align256(sizeof(unsigned long long) * (size_t)std::max(rows, 1));
}

void i8_operand_init(void *buf, int rows, int k, int s, I8Operand &op) {
    op.rows = rows;
    op.k = k;
    op.s = s;
    op.k_ld = round_up(std::max(k, 1), TC_BK);
    op.slice_stride = align256((size_t)op.k_ld * std::max(rows, 1));
    char *p = (char *)buf;
    op.data = (int8_t *)p;
    p += op.slice_stride * (size_t)s;
    op.exps = (int *)p;
    p += align256(sizeof(int) * (size_t)std::max(rows, 1));
    op.rmax = (unsigned long long *)p;
}

int i8_slice(const double *X, long long ldx, int src, I8Operand &op, cudaStream_t st) {
    if (op.rows <= 0 || op.k <= 0) return CUEV_OK;
    if (op.s < 1 || op.s > 8) return CUEV_ERR_INVALID;
    CUEV_TRY(cudaMemsetAsync(op.rmax, 0, sizeof(unsigned long long) * op.rows, st));
    const dim3 grid(div_up((int)op.k_ld, SL_K), div_up(op.rows, SL_R));
    i8_rowmax_kernel<<<grid, SL_THREADS, 0, st>>>(X, ldx, src, op.rows, op.k, op.rmax);
    note_launch();
    i8_exp_kernel<<<std::min(1024, div_up(op.rows, 256)), 256, 0, st>>>(op.rmax, op.rows, op.exps);
    note_launch();
    i8_slice_kernel<<<grid, SL_THREADS, 0, st>>>(X, ldx, src, op.rows, op.k, op.s, op.exps,
                                                 op.data, op.k_ld, op.slice_stride);
    note_launch();
    CUEV_TRY(cudaGetLastError());
    return CUEV_OK;
}

int i8_gemm(const I8Operand &A, const I8Operand &B, int levels, double alpha, double beta,
            double *C, long long ldc, int c_lower, int *status, cudaStream_t st) {
    const int m = A.rows, n = B.rows;
    if (m <= 0 || n <= 0) return CUEV_OK;
    if (A.k != B.k || A.k_ld != B.k_ld || levels < 1 || levels > A.s + B.s - 1 || !status ||
        ldc < m) {
        set_last_message("int8 tensor-core GEMM: inconsistent operands");
        return CUEV_ERR_INVALID;
    }
    if (A.k <= 0 || alpha == 0.0) {
        set_last_message("int8 tensor-core GEMM: empty K or alpha == 0 not handled here");
        return CUEV_ERR_INVALID;
    }
    // The slices must be 16-byte aligned for TMA and the strides multiples of 16 (k_ld is a
    // multiple of 128, slice_stride of 256).
    if (((uintptr_t)A.data & 15) || ((uintptr_t)B.data & 15)) return CUEV_ERR_INVALID;
    const int BN = n > 128 ? 256 : 128;
    TcArgs a{};
    a.C = C, a.ldc = ldc, a.ea = A.exps, a.eb = B.exps, a.status = status;
    a.m = m, a.n = n, a.k_chunks = (int)(A.k_ld / TC_BK);
    a.sa = A.s, a.sb = B.s, a.levels = levels;
    a.mt = div_up(m, TC_BM), a.nt = div_up(n, BN);
    a.c_lower = c_lower;
    a.alpha = alpha, a.beta = beta;
    long long nt = (long long)a.mt * a.nt;
    if (c_lower) {
        nt = 0;
        for (int tn = 0; tn < a.nt; ++tn) nt += std::max(0, a.mt - (tn * BN) / TC_BM);
    }
    a.ntiles = (int)nt;
    if (a.ntiles <= 0) return CUEV_OK;
    CUtensorMap ma, mb;
    CUEV_CHECK_STATUS(make_map(A, TC_BM, &ma));
    CUEV_CHECK_STATUS(make_map(B, BN, &mb));
    const int grid = std::min(a.ntiles, num_sms());
    return BN == 256 ? launch_i8<256>(ma, mb, a, grid, st) : launch_i8<128>(ma, mb, a, grid, st);
}

size_t i8_gemm_scratch_bytes(int m, int n, int k, int s) {
    return i8_operand_bytes(m, k, s) + i8_operand_bytes(n, k, s);
}

int i8_dgemm(int ta, int tb, int symm_a, int m, int n, int k, int s, double alpha,
             const double *A, long long lda, const double *B, long long ldb, double beta,
             double *C, long long ldc, int c_lower, void *scratch, int *status, cudaStream_t st) {
    if (m <= 0 || n <= 0) return CUEV_OK;
    if (s < 1 || s > 8 || !scratch) return CUEV_ERR_INVALID;
    I8Operand oa, ob;
    i8_operand_init(scratch, m, k, s, oa);
    i8_operand_init((char *)scratch + i8_operand_bytes(m, k, s), n, k, s, ob);
    const int srcA = symm_a ? I8_SRC_SYML : (ta ? I8_SRC_KMAJ : I8_SRC_RMAJ);
    const int srcB = tb ? I8_SRC_RMAJ : I8_SRC_KMAJ;
    CUEV_CHECK_STATUS(i8_slice(A, lda, srcA, oa, st));
    CUEV_CHECK_STATUS(i8_slice(B, ldb, srcB, ob, st));
    return i8_gemm(oa, ob, s, alpha, beta, C, ldc, c_lower, status, st);
}

} // namespace cuev
