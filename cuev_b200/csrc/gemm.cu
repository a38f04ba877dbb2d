// FP64 DMMA GEMM kernels (see gemm.cuh for the contract).
#include "gemm.cuh"

#include <algorithm>
#include <type_traits>

namespace cuev {
namespace {

constexpr int PAD = 4; // row padding (doubles): keeps fragment reads bank-conflict free

// KS_: k-depth of one DMMA (8 or 16); the k16 shape needs twice the fragment registers.
// BK_: k-depth of one shared-memory stage (a multiple of KS_).
template <int BM_, int BN_, int WARPS_M_, int WARPS_N_, int STAGES_, int KS_ = 16, int BK_ = 16>
struct TileCfg {
    static constexpr int BM = BM_, BN = BN_, WARPS_M = WARPS_M_, WARPS_N = WARPS_N_;
    static constexpr int STAGES = STAGES_, KS = KS_, BK = BK_;
    static_assert(BK % KS == 0 && BK % 16 == 0, "stage depth");
    static_assert(KS == 8 || KS == 16, "DMMA k-depth");
    static constexpr int NT = 32 * WARPS_M * WARPS_N;
    static constexpr int WM = BM / WARPS_M, WN = BN / WARPS_N;
    static constexpr int MT = WM / 16, NTL = WN / 8;
    static_assert(WM % 16 == 0 && WN % 8 == 0, "warp tile must be a multiple of the DMMA shape");
    // every thread copies a whole number (>= 1) of 16-byte pairs of each operand tile per stage
    static_assert((BM / 2) * BK % NT == 0 && (BM / 2) * BK / NT >= 1, "A tile / threads");
    static_assert((BN / 2) * BK % NT == 0 && (BN / 2) * BK / NT >= 1, "B tile / threads");
};

using CfgBig = TileCfg<128, 128, 4, 4, 3, 16, 32>; // 16 warps (two per SMSP left the DMMA pipe idle), BK 32, k16 DMMA
// batched (D&C merge) problems read with 8-byte copies; on the mbarrier pipeline 32-deep stages
// and k16 beat 16-deep ones (D&C stage 213 -> 194 ms at n = 16384; they were slower with a CTA
// barrier per stage)
using CfgBigBatched = TileCfg<128, 128, 4, 4, 3, 16, 32>;
using CfgSkinny = TileCfg<128, 64, 4, 2, 4>;
using CfgSmall = TileCfg<64, 64, 2, 2, 4>;
using CfgN32 = TileCfg<128, 32, 8, 1, 4>; // N <= 32 (band width 32 panels): 16 x 32 warp tiles

__device__ __forceinline__ void cp_async8(double *smem, const double *gmem, bool pred) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int sz = pred ? 8 : 0; // src-size 0 => zero fill, nothing is read
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(sz)
                 : "memory");
}
// 16-byte copy; src_bytes in {0, 8, 16}, the rest of the 16 bytes is zero-filled
__device__ __forceinline__ void cp_async16(double *smem, const double *gmem, int src_bytes) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem),
                 "r"(src_bytes)
                 : "memory");
}

// Set (sticky) when a stage wait of a GEMM gave up (2 s); workspace_check_status folds it into
// the solver's status word.  The waits depend only on the CTA's own copies and warps.
__device__ int g_gemm_wait_fault = 0;

__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long *mb, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mb)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(unsigned long long *mb) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(mb)) : "memory");
}
// arrive on mb once every cp.async this thread has issued so far has completed
__device__ __forceinline__ void cp_async_arrive(unsigned long long *mb) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(mb))
                 : "memory");
}
// wait for the phase of parity `par` of mb to complete; false after 2 s
__device__ __forceinline__ bool mbar_wait(unsigned long long *mb, unsigned par) {
    const unsigned a = smem_u32(mb);
    unsigned done;
    asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; "
                 "selp.u32 %0, 1, 0, p; }"
                 : "=r"(done)
                 : "r"(a), "r"(par)
                 : "memory");
    if (done) return true;
    const uint64_t t0 = global_ns();
    for (int it = 1;; ++it) {
        asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; "
                     "selp.u32 %0, 1, 0, p; }"
                     : "=r"(done)
                     : "r"(a), "r"(par)
                     : "memory");
        if (done) return true;
        if ((it & 255) == 0 && global_ns() - t0 > 2000000000ull) return false;
    }
}

// D = A(16x8, row) * B(8x8, col) + D  (FP64 DMMA; g = lane/4, t = lane%4).  Fragments: a0 = A[g][t], a1 = A[g+8][t],
//   a2 = A[g][t+4], a3 = A[g+8][t+4];  b0 = B[t][g], b1 = B[t+4][g];  D as for m16n8k4.
__device__ __forceinline__ void dmma16x8x8(double (&d)[4], double a0, double a1, double a2,
                                           double a3, double b0, double b1) {
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
                 "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                 : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
                 : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}

// D = A(16x16, row) * B(16x8, col) + D (FP64 DMMA, sm_90+ shape).  Fragments extend the k8 layout:
//   a[2i] = A[g][t + 4i], a[2i+1] = A[g+8][t + 4i];  b[i] = B[t + 4i][g]  (i = 0..3).
__device__ __forceinline__ void dmma16x8x16(double (&d)[4], const double (&a)[8],
                                            const double (&b)[4]) {
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
                 "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
                 : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
                 : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]),
                   "d"(a[7]), "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

template <class C, bool TA, bool TB, bool SYMM> struct SmemLayout {
    static constexpr int BK = C::BK;
    // "outer-contiguous" tiles are stored [k][outer] (the global matrix is contiguous along the
    // outer index), the others [outer][k].
    static constexpr bool A_OUTER = SYMM || !TA;
    static constexpr bool B_OUTER = TB;
    // SYMM stages hold either layout (tiles above the diagonal are read transposed)
    static constexpr int A_ELEMS =
        SYMM ? (BK * (C::BM + PAD) > C::BM * (BK + PAD) ? BK * (C::BM + PAD) : C::BM * (BK + PAD))
             : (A_OUTER ? BK * (C::BM + PAD) : C::BM * (BK + PAD));
    static constexpr int B_ELEMS = B_OUTER ? BK * (C::BN + PAD) : C::BN * (BK + PAD);
    static constexpr int STAGE_ELEMS = A_ELEMS + B_ELEMS;
    static constexpr size_t BYTES = (size_t)C::STAGES * STAGE_ELEMS * sizeof(double);
};

// VEC = 2: global tiles are read as 16-byte pairs along their contiguous dimension (needs
// 16-byte aligned bases, even leading dimensions and an even first K segment); VEC = 1 reads
// single elements and accepts any alignment.
template <class C, bool TA, bool TB, bool SYMM, bool BATCHED, int VEC>
__global__ void __launch_bounds__(C::NT)
    dgemm_kernel(const GemmArgs args_val, const GemmArgs *__restrict__ args_arr) {
    using L = SmemLayout<C, TA, TB, SYMM>;
    constexpr int BK = C::BK;
    extern __shared__ __align__(16) double smem[];

    const GemmArgs a = BATCHED ? args_arr[blockIdx.z] : args_val;
    const int m = a.m, n = a.n, k1 = a.k;
    const int Ktot = a.k + a.k2;
    const int bm = blockIdx.x * C::BM, bn = blockIdx.y * C::BN;
    if (bm >= m || bn >= n) return;
    if (a.c_lower && bm + C::BM - 1 < bn) return; // tile strictly above the diagonal
    const int split = BATCHED ? 0 : blockIdx.z;
    const int splits = BATCHED ? 1 : a.splits;

    int kbeg = 0, kend = Ktot;
    if (splits > 1) {
        const int kchunk = ((Ktot + splits - 1) / splits + BK - 1) / BK * BK;
        kbeg = min(Ktot, split * kchunk);
        kend = min(Ktot, kbeg + kchunk);
    }
    const int ntiles = (kend - kbeg + BK - 1) / BK;

    const double *__restrict__ A = a.A;
    const double *__restrict__ A2 = a.A2;
    const double *__restrict__ B = a.B;
    const double *__restrict__ B2 = a.B2;
    const long long lda = a.lda, lda2 = a.lda2, ldb = a.ldb, ldb2 = a.ldb2;

    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wm0 = (warp % C::WARPS_M) * C::WM;
    const int wn0 = (warp / C::WARPS_M) * C::WN;

    // A tile of a SYMM stage: on/below the diagonal it is read as stored (m-contiguous, outer
    // layout); above the diagonal its mirror A(kg, i) is read (k-contiguous, [m][k] layout).
    auto symm_upper = [&](int k0) { return SYMM && (bm + C::BM - 1 < k0); };
    auto load_stage = [&](int slot, int k0) {
        double *sA = smem + slot * L::STAGE_ELEMS;
        double *sB = sA + L::A_ELEMS;
        // ---- A tile: op(A)[bm .. bm+BM) x [k0 .. k0+BK)
        if (SYMM) {
            const bool upper = symm_upper(k0);
            const bool lower = bm >= k0 + BK - 1;
            if (VEC == 2 && (upper || lower)) {
                if (lower) {
#pragma unroll
                    for (int it = 0; it < (C::BM / 2) * BK / C::NT; ++it) {
                        const int e = tid + it * C::NT;
                        const int r = 2 * (e % (C::BM / 2)), kk = e / (C::BM / 2);
                        const int i = bm + r, kg = k0 + kk;
                        const int nb = (i < m && kg < kend) ? (i + 1 < m ? 16 : 8) : 0;
                        cp_async16(sA + kk * (C::BM + PAD) + r, nb ? A + i + (long long)kg * lda : A, nb);
                    }
                } else {
#pragma unroll
                    for (int it = 0; it < C::BM * (BK / 2) / C::NT; ++it) {
                        const int e = tid + it * C::NT;
                        const int kk = 2 * (e % (BK / 2)), r = e / (BK / 2);
                        const int i = bm + r, kg = k0 + kk;
                        const int nb = (i < m && kg < kend) ? (kg + 1 < kend ? 16 : 8) : 0;
                        cp_async16(sA + r * (BK + PAD) + kk, nb ? A + kg + (long long)i * lda : A, nb);
                    }
                }
            } else {
#pragma unroll
                for (int it = 0; it < (C::BM * BK) / C::NT; ++it) {
                    const int e = tid + it * C::NT;
                    int r, kk;
                    if (!upper) {
                        r = e % C::BM;
                        kk = e / C::BM;
                    } else {
                        kk = e % BK;
                        r = e / BK;
                    }
                    const int i = bm + r, kg = k0 + kk;
                    const bool pred = (i < m) && (kg < kend);
                    const double *src = A;
                    if (pred) src = (i >= kg) ? A + i + (long long)kg * lda : A + kg + (long long)i * lda;
                    double *dst = upper ? sA + r * (BK + PAD) + kk : sA + kk * (C::BM + PAD) + r;
                    cp_async8(dst, src, pred);
                }
            }
        } else if (VEC == 2) {
            if (L::A_OUTER) { // A contiguous along m
#pragma unroll
                for (int it = 0; it < (C::BM / 2) * BK / C::NT; ++it) {
                    const int e = tid + it * C::NT;
                    const int r = 2 * (e % (C::BM / 2)), kk = e / (C::BM / 2);
                    const int i = bm + r, kg = k0 + kk;
                    const int nb = (i < m && kg < kend) ? (i + 1 < m ? 16 : 8) : 0;
                    const double *src = A;
                    if (nb) src = (kg < k1) ? A + i + (long long)kg * lda : A2 + i + (long long)(kg - k1) * lda2;
                    cp_async16(sA + kk * (C::BM + PAD) + r, src, nb);
                }
            } else { // A^T: contiguous along k
#pragma unroll
                for (int it = 0; it < C::BM * (BK / 2) / C::NT; ++it) {
                    const int e = tid + it * C::NT;
                    const int kk = 2 * (e % (BK / 2)), r = e / (BK / 2);
                    const int i = bm + r, kg = k0 + kk;
                    const int nb = (i < m && kg < kend) ? (kg + 1 < kend ? 16 : 8) : 0;
                    const double *src = A;
                    if (nb) src = (kg < k1) ? A + kg + (long long)i * lda : A2 + (kg - k1) + (long long)i * lda2;
                    cp_async16(sA + r * (BK + PAD) + kk, src, nb);
                }
            }
        } else {
#pragma unroll
            for (int it = 0; it < (C::BM * BK) / C::NT; ++it) {
                const int e = tid + it * C::NT;
                int r, kk;
                if (L::A_OUTER) {
                    r = e % C::BM;
                    kk = e / C::BM;
                } else {
                    kk = e % BK;
                    r = e / BK;
                }
                const int i = bm + r, kg = k0 + kk;
                const bool pred = (i < m) && (kg < kend);
                const double *src = A;
                if (pred) {
                    if (kg < k1) {
                        src = TA ? A + kg + (long long)i * lda : A + i + (long long)kg * lda;
                    } else {
                        const int q = kg - k1;
                        src = TA ? A2 + q + (long long)i * lda2 : A2 + i + (long long)q * lda2;
                    }
                }
                double *dst = L::A_OUTER ? sA + kk * (C::BM + PAD) + r : sA + r * (BK + PAD) + kk;
                cp_async8(dst, src, pred);
            }
        }
        // ---- B tile: op(B)[k0 .. k0+BK) x [bn .. bn+BN)
        if (VEC == 2) {
            if (L::B_OUTER) { // B^T: contiguous along n
#pragma unroll
                for (int it = 0; it < (C::BN / 2) * BK / C::NT; ++it) {
                    const int e = tid + it * C::NT;
                    const int c = 2 * (e % (C::BN / 2)), kk = e / (C::BN / 2);
                    const int j = bn + c, kg = k0 + kk;
                    const int nb = (j < n && kg < kend) ? (j + 1 < n ? 16 : 8) : 0;
                    const double *src = B;
                    if (nb) src = (kg < k1) ? B + j + (long long)kg * ldb : B2 + j + (long long)(kg - k1) * ldb2;
                    cp_async16(sB + kk * (C::BN + PAD) + c, src, nb);
                }
            } else { // B: contiguous along k
#pragma unroll
                for (int it = 0; it < C::BN * (BK / 2) / C::NT; ++it) {
                    const int e = tid + it * C::NT;
                    const int kk = 2 * (e % (BK / 2)), c = e / (BK / 2);
                    const int j = bn + c, kg = k0 + kk;
                    const int nb = (j < n && kg < kend) ? (kg + 1 < kend ? 16 : 8) : 0;
                    const double *src = B;
                    if (nb) src = (kg < k1) ? B + kg + (long long)j * ldb : B2 + (kg - k1) + (long long)j * ldb2;
                    cp_async16(sB + c * (BK + PAD) + kk, src, nb);
                }
            }
        } else {
#pragma unroll
            for (int it = 0; it < (C::BN * BK) / C::NT; ++it) {
                const int e = tid + it * C::NT;
                int c, kk;
                if (L::B_OUTER) {
                    c = e % C::BN;
                    kk = e / C::BN;
                } else {
                    kk = e % BK;
                    c = e / BK;
                }
                const int j = bn + c, kg = k0 + kk;
                const bool pred = (j < n) && (kg < kend);
                const double *src = B;
                if (pred) {
                    if (kg < k1) {
                        src = TB ? B + j + (long long)kg * ldb : B + kg + (long long)j * ldb;
                    } else {
                        const int q = kg - k1;
                        src = TB ? B2 + j + (long long)q * ldb2 : B2 + q + (long long)j * ldb2;
                    }
                }
                double *dst = L::B_OUTER ? sB + kk * (C::BN + PAD) + c : sB + c * (BK + PAD) + kk;
                cp_async8(dst, src, pred);
            }
        }
    };

    double acc[C::MT][C::NTL][4];
#pragma unroll
    for (int i = 0; i < C::MT; ++i)
#pragma unroll
        for (int j = 0; j < C::NTL; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.0;

    // one BK-deep stage of DMMA work; AOUT selects the A tile layout of this stage
    auto mma_stage = [&](const double *sA, const double *sB, auto aout) {
        constexpr bool AOUT = decltype(aout)::value;
        constexpr int KS = C::KS, NH = KS / 4; // fragment entries per row: k offsets 0, 4, ...
#pragma unroll
        for (int ks = 0; ks < BK / KS; ++ks) {
            const int kk = ks * KS + t;
            double af[C::MT][2 * NH], bf[C::NTL][NH];
#pragma unroll
            for (int mi = 0; mi < C::MT; ++mi) {
                const int r = wm0 + mi * 16 + g;
#pragma unroll
                for (int hh = 0; hh < NH; ++hh) {
                    const int k2 = kk + 4 * hh;
                    if (AOUT) {
                        af[mi][2 * hh] = sA[k2 * (C::BM + PAD) + r];
                        af[mi][2 * hh + 1] = sA[k2 * (C::BM + PAD) + r + 8];
                    } else {
                        af[mi][2 * hh] = sA[r * (BK + PAD) + k2];
                        af[mi][2 * hh + 1] = sA[(r + 8) * (BK + PAD) + k2];
                    }
                }
            }
#pragma unroll
            for (int ni = 0; ni < C::NTL; ++ni) {
                const int c = wn0 + ni * 8 + g;
#pragma unroll
                for (int hh = 0; hh < NH; ++hh) {
                    const int k2 = kk + 4 * hh;
                    bf[ni][hh] = L::B_OUTER ? sB[k2 * (C::BN + PAD) + c] : sB[c * (BK + PAD) + k2];
                }
            }
#pragma unroll
            for (int mi = 0; mi < C::MT; ++mi)
#pragma unroll
                for (int ni = 0; ni < C::NTL; ++ni) {
                    if constexpr (KS == 16)
                        dmma16x8x16(acc[mi][ni], af[mi], bf[ni]);
                    else
                        dmma16x8x8(acc[mi][ni], af[mi][0], af[mi][1], af[mi][2], af[mi][3],
                                   bf[ni][0], bf[ni][1]);
                }
        }
    };

    // Stage pipeline on mbarriers instead of a CTA barrier per stage: full[s] completes when the
    // cp.async copies of every thread into slot s have landed (cp.async.mbarrier.arrive), empty[s]
    // when every warp has read slot s.  A slot is refilled after the next stage has been computed,
    // so a warp waits for a slower one only when it is a whole stage ahead.  (With one barrier per
    // stage the DMMA pipe idled about a fifth of the time: 29.4 -> 33.1 TF/s at 8192^3.)
    __shared__ __align__(8) unsigned long long mb_full[C::STAGES], mb_empty[C::STAGES];
    if (tid == 0) {
#pragma unroll
        for (int s = 0; s < C::STAGES; ++s) {
            mbar_init(&mb_full[s], C::NT);
            mbar_init(&mb_empty[s], C::NT / 32);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < C::STAGES - 1; ++s) {
        if (s < ntiles) load_stage(s, kbeg + s * BK);
        cp_async_arrive(&mb_full[s]);
    }
    bool ok = true;
    for (int kt = 0; kt < ntiles; ++kt) {
        const int slot = kt % C::STAGES;
        if (!mbar_wait(&mb_full[slot], (unsigned)((kt / C::STAGES) & 1))) {
            ok = false;
            break;
        }
        const double *sA = smem + slot * L::STAGE_ELEMS;
        const double *sB = sA + L::A_ELEMS;
        if (SYMM && symm_upper(kbeg + kt * BK))
            mma_stage(sA, sB, std::integral_constant<bool, false>{});
        else
            mma_stage(sA, sB, std::integral_constant<bool, L::A_OUTER>{});
        __syncwarp();
        if (lane == 0) mbar_arrive(&mb_empty[slot]);
        // refill the slot of stage kt - 1 (stage kt + STAGES - 1) once every warp has read it
        const int pf = kt + C::STAGES - 1, ps = pf % C::STAGES;
        if (pf < ntiles) {
            if (pf >= C::STAGES &&
                !mbar_wait(&mb_empty[ps], (unsigned)(((pf - C::STAGES) / C::STAGES) & 1))) {
                ok = false;
                break;
            }
            load_stage(ps, kbeg + pf * BK);
        }
        cp_async_arrive(&mb_full[ps]);
    }
    asm volatile("cp.async.wait_all;" ::: "memory"); // no copy in flight, also after a timeout
    if (!ok) {
        atomicExch(&g_gemm_wait_fault, 1);
        return;
    }

    // epilogue
    const double alpha = a.alpha, beta = a.beta;
    double *__restrict__ Cp = a.C;
    const long long ldc = a.ldc;
    double *__restrict__ W = (splits > 1) ? a.ws + (size_t)split * m * n : nullptr;
#pragma unroll
    for (int mi = 0; mi < C::MT; ++mi)
#pragma unroll
        for (int ni = 0; ni < C::NTL; ++ni)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int row = bm + wm0 + mi * 16 + g + ((q & 2) ? 8 : 0);
                const int col = bn + wn0 + ni * 8 + 2 * t + (q & 1);
                if (row >= m || col >= n) continue;
                if (a.c_lower && row < col) continue;
                double v = alpha * acc[mi][ni][q];
                if (a.epi) {
                    if (row == col) {
                        v = a.epi_lambar ? a.epi_lambar[row] : 0.0;
                    } else {
                        const double gap = a.epi_lam[col] - a.epi_lam[row];
                        v = (fabs(gap) < a.epi_gap) ? 0.0 : v / gap;
                    }
                }
                if (W) {
                    W[row + (size_t)col * m] = v;
                } else {
                    double *cp = Cp + row + (long long)col * ldc;
                    *cp = (beta != 0.0) ? v + beta * (*cp) : v;
                }
            }
}

// C = sum_z W_z + beta C over the (masked) m x n output.
__global__ void splitk_reduce_kernel(int m, int n, int splits, const double *__restrict__ W,
                                     double beta, double *__restrict__ C, long long ldc,
                                     int c_lower) {
    const size_t total = (size_t)m * n;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        const int row = (int)(idx % m), col = (int)(idx / m);
        if (c_lower && row < col) continue;
        double s = 0.0;
        for (int z = 0; z < splits; ++z) s += W[z * total + idx];
        double *cp = C + row + (long long)col * ldc;
        *cp = (beta != 0.0) ? s + beta * (*cp) : s;
    }
}

template <class C, bool TA, bool TB, bool SYMM, bool BATCHED, int VEC>
int launch_cfg(const GemmArgs &a, const GemmArgs *dev_args, dim3 grid, cudaStream_t stream) {
    using L = SmemLayout<C, TA, TB, SYMM>;
    auto kern = dgemm_kernel<C, TA, TB, SYMM, BATCHED, VEC>;
    CUEV_CHECK_STATUS(ensure_dyn_smem((const void *)kern, L::BYTES));
    kern<<<grid, C::NT, L::BYTES, stream>>>(a, dev_args); note_launch();
    CUEV_TRY(cudaGetLastError());
    return CUEV_OK;
}

template <class C, bool SYMM, bool BATCHED>
int dispatch_t(const GemmArgs &a, const GemmArgs *dev_args, int ta, int tb, dim3 grid,
               cudaStream_t stream, bool vec2 = false) {
    if (SYMM) {
        if (vec2) return launch_cfg<C, false, false, true, BATCHED, 2>(a, dev_args, grid, stream);
        return launch_cfg<C, false, false, true, BATCHED, 1>(a, dev_args, grid, stream);
    }
    if (BATCHED) return launch_cfg<C, false, false, false, BATCHED, 1>(a, dev_args, grid, stream);
    if (vec2) {
        if (!ta && !tb) return launch_cfg<C, false, false, false, false, 2>(a, dev_args, grid, stream);
        if (!ta && tb) return launch_cfg<C, false, true, false, false, 2>(a, dev_args, grid, stream);
        if (ta && !tb) return launch_cfg<C, true, false, false, false, 2>(a, dev_args, grid, stream);
        return launch_cfg<C, true, true, false, false, 2>(a, dev_args, grid, stream);
    }
    if (!ta && !tb) return launch_cfg<C, false, false, false, false, 1>(a, dev_args, grid, stream);
    if (!ta && tb) return launch_cfg<C, false, true, false, false, 1>(a, dev_args, grid, stream);
    if (ta && !tb) return launch_cfg<C, true, false, false, false, 1>(a, dev_args, grid, stream);
    return launch_cfg<C, true, true, false, false, 1>(a, dev_args, grid, stream);
}

bool aligned16(const void *p) { return ((uintptr_t)p & 15) == 0; }

// 16-byte loads are legal when every base is 16-byte aligned, every leading dimension is even
// (so each column starts 16-byte aligned) and the first K segment has even length.
bool vec2_ok(const GemmArgs &a) {
    if (a.symm_a) return aligned16(a.A) && aligned16(a.B) && !(a.lda & 1) && !(a.ldb & 1);
    if (!aligned16(a.A) || !aligned16(a.B) || (a.lda & 1) || (a.ldb & 1)) return false;
    if (a.k2 > 0 && (!aligned16(a.A2) || !aligned16(a.B2) || (a.lda2 & 1) || (a.ldb2 & 1) || (a.k & 1)))
        return false;
    return true;
}

enum class Tile { Big, Skinny, Small, N32 };

Tile pick_tile(int m, int n) {
    if (n <= 32 && m > 64) return Tile::N32;
    if (m <= 64 && n <= 64) return Tile::Small;
    if (n <= 64 || m <= 64) return Tile::Skinny;
    return Tile::Big;
}

void tile_dims(Tile t, int &bm, int &bn) {
    switch (t) {
    case Tile::Big: bm = CfgBig::BM, bn = CfgBig::BN; break;
    case Tile::Skinny: bm = CfgSkinny::BM, bn = CfgSkinny::BN; break;
    case Tile::N32: bm = CfgN32::BM, bn = CfgN32::BN; break;
    default: bm = CfgSmall::BM, bn = CfgSmall::BN; break;
    }
}

__global__ void gemm_fold_fault_kernel(int *status) {
    if (g_gemm_wait_fault) dev_fail(status, CUEV_ERR_TIMEOUT, -100);
}

} // namespace

int gemm_fold_fault(int *status, cudaStream_t stream) {
    gemm_fold_fault_kernel<<<1, 1, 0, stream>>>(status);
    note_launch();
    CUEV_TRY(cudaGetLastError());
    return CUEV_OK;
}

// Split count from a wave model: with s splits the busiest SM runs ceil(tiles s / SMs) CTAs, each
// over 1/s of the K range, so the time goes as ceil(tiles s / SMs) / s.  Among the counts that
// give every SM a CTA (or the largest allowed, when none does), take the smallest one that no
// larger count beats by 2 % (a split costs a reduction over its m x n partials).  On the band
// reduction's SYMM (m x 32, K = m) this picks the measured best count to within a few percent for
// m = 2048 .. 16384, where "at least two CTAs per SM" picked counts up to 1.4x slower.
int gemm_splitk_count(int m, int n, int k_total, int c_lower, int max_splits) {
    if (m <= 0 || n <= 0 || k_total <= 0) return 1;
    const Tile tl = pick_tile(m, n);
    int bm, bn;
    tile_dims(tl, bm, bn);
    long long tiles = (long long)div_up(m, bm) * div_up(n, bn);
    if (c_lower) tiles = (tiles + div_up(n, bn)) / 2;
    const long long sms = num_sms();
    if (tiles >= 4 * sms) return 1; // four or more waves: the partial last one costs little
    // up to 32 splits where 16 cannot fill the SMs, else up to 16 (the range measured)
    const int scap = tiles * 16 < sms ? 32 : 16;
    const int smax = std::max(1, std::min({scap, k_total / 256, max_splits}));
    auto cost = [&](int s) { return (double)((tiles * s + sms - 1) / sms) / s; };
    int best = 0;
    double best_t = 0.0;
    for (int s = 1; s <= smax; ++s) {
        if (tiles * s < sms && s < smax) continue; // some SMs would idle
        const double t = cost(s);
        if (best == 0 || t < 0.98 * best_t) best = s, best_t = t;
    }
    return std::max(1, best);
}

size_t gemm_splitk_workspace(int m, int n, int k_total, int ta, int tb, int c_lower) {
    (void)ta;
    (void)tb;
    const int s = gemm_splitk_count(m, n, k_total, c_lower);
    return s > 1 ? (size_t)s * m * n * sizeof(double) : 0;
}

int gemm_launch(const GemmArgs &a_in, int ta, int tb, cudaStream_t stream) {
    GemmArgs a = a_in;
    if (a.m <= 0 || a.n <= 0) return CUEV_OK;
    const int ktot = a.k + a.k2;
    if (ktot <= 0 || a.alpha == 0.0) {
        // C = beta C on the (masked) output; reuse the reduction kernel with zero splits.
        const long long mn = (long long)a.m * a.n;
        splitk_reduce_kernel<<<(int)std::min<long long>(4096, (mn + 255) / 256), 256, 0, stream>>>(
            a.m, a.n, 0, nullptr, a.beta, a.C, a.ldc, a.c_lower); note_launch();
        CUEV_TRY(cudaGetLastError());
        return CUEV_OK;
    }
    if ((a.splits > 1 && a.ws == nullptr) || a.epi) a.splits = 1;
    if (a.splits < 1) a.splits = 1;
    const Tile tl = pick_tile(a.m, a.n);
    int bm, bn;
    tile_dims(tl, bm, bn);
    dim3 grid(div_up(a.m, bm), div_up(a.n, bn), a.splits);
    const bool v2 = vec2_ok(a);
    int st;
    switch (tl) {
    case Tile::Big:
        st = a.symm_a ? dispatch_t<CfgBig, true, false>(a, nullptr, 0, 0, grid, stream, v2)
                      : dispatch_t<CfgBig, false, false>(a, nullptr, ta, tb, grid, stream, v2);
        break;
    case Tile::Skinny:
        st = a.symm_a ? dispatch_t<CfgSkinny, true, false>(a, nullptr, 0, 0, grid, stream, v2)
                      : dispatch_t<CfgSkinny, false, false>(a, nullptr, ta, tb, grid, stream, v2);
        break;
    case Tile::N32:
        st = a.symm_a ? dispatch_t<CfgN32, true, false>(a, nullptr, 0, 0, grid, stream, v2)
                      : dispatch_t<CfgN32, false, false>(a, nullptr, ta, tb, grid, stream, v2);
        break;
    default:
        st = a.symm_a ? dispatch_t<CfgSmall, true, false>(a, nullptr, 0, 0, grid, stream, v2)
                      : dispatch_t<CfgSmall, false, false>(a, nullptr, ta, tb, grid, stream, v2);
        break;
    }
    if (st != CUEV_OK) return st;
    if (a.splits > 1) {
        const long long total = (long long)a.m * a.n;
        const int blocks = (int)std::min<long long>(4 * num_sms(), (total + 255) / 256);
        splitk_reduce_kernel<<<blocks, 256, 0, stream>>>(a.m, a.n, a.splits, a.ws, a.beta, a.C,
                                                         a.ldc, a.c_lower); note_launch();
        CUEV_TRY(cudaGetLastError());
    }
    return CUEV_OK;
}

int gemm_batched_launch(const GemmArgs *dev_args, int count, int max_m, int max_n, int ta,
                        int tb, cudaStream_t stream) {
    if (count <= 0 || max_m <= 0 || max_n <= 0) return CUEV_OK;
    Tile tl = pick_tile(max_m, max_n);
    if (tl == Tile::N32) tl = Tile::Skinny; // batched problems use the three base tiles
    int bm, bn;
    tile_dims(tl, bm, bn);
    GemmArgs dummy{};
    for (int z0 = 0; z0 < count; z0 += 65535) {
        const int cnt = std::min(65535, count - z0);
        dim3 grid(div_up(max_m, bm), div_up(max_n, bn), cnt);
        int st;
        switch (tl) {
        case Tile::Big:
            st = dispatch_t<CfgBigBatched, false, true>(dummy, dev_args + z0, ta, tb, grid, stream);
            break;
        case Tile::Skinny:
            st = dispatch_t<CfgSkinny, false, true>(dummy, dev_args + z0, ta, tb, grid, stream);
            break;
        default:
            st = dispatch_t<CfgSmall, false, true>(dummy, dev_args + z0, ta, tb, grid, stream);
            break;
        }
        if (st != CUEV_OK) return st;
    }
    return CUEV_OK;
}

} // namespace cuev
