// C ABI (include/cuev_b200.h) and the C++ drop-in shim (include/cuev.h).
//
// Full solves keep one cached workspace per device and (n, b, k) so repeated calls do not
// allocate; a call that finds the cached workspace busy (another host thread) allocates its own,
// which keeps the reference's reentrancy (its handle is per call, src/cuda/solver.cu:33,72).
#include "refine.cuh"
#include "solver.cuh"

#include "../../include/cuev.h"

#include <chrono>
#include <cstdlib>
#include <mutex>

struct cuev_handle_s {
    cuev::Workspace *ws;
};

namespace cuev {
namespace {

thread_local double g_last_dc_flops = 0.0;

struct CachedWs {
    Workspace *ws = nullptr;
    bool busy = false;
};
std::mutex g_cache_mu;
CachedWs g_cache[64];

int default_b(int n) {
    (void)n;
    return 32;
}
int default_k(int n, int b) {
    (void)b;
    return n >= 8192 ? 512 : 256;
}

int acquire_ws(int n, int b, int k, cudaStream_t stream, Workspace **out, bool *cached) {
    int dev = 0;
    CUEV_TRY(cudaGetDevice(&dev));
    *cached = false;
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        CachedWs &c = g_cache[dev & 63];
        if (!c.busy) {
            // a cached workspace that is not busy has no work in flight (solves block until
            // done); workspace_destroy waits for its own side stream
            if (c.ws && (c.ws->n != n || c.ws->b != b || c.ws->k != k)) {
                workspace_destroy(c.ws);
                c.ws = nullptr;
            }
            if (!c.ws) CUEV_CHECK_STATUS(workspace_create(n, b, k, stream, &c.ws));
            c.busy = true;
            c.ws->stream = stream;
            *out = c.ws;
            *cached = true;
            return CUEV_OK;
        }
    }
    return workspace_create(n, b, k, stream, out);
}

void release_ws(Workspace *ws, bool cached) {
    if (cached) {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        for (auto &c : g_cache)
            if (c.ws == ws) c.busy = false;
    } else {
        workspace_destroy(ws);
    }
}

// Non-finite scan of the lower triangle.
__global__ void nonfinite_scan_kernel(const double *__restrict__ A, int n, long long lda,
                                      int *status) {
    const long long total = (long long)n * n;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % n), j = (int)(idx / n);
        if (i >= j && !isfinite(A[i + (long long)j * lda])) {
            dev_fail(status, CUEV_ERR_NONFINITE, j);
            return;
        }
    }
}

__global__ void small_solve_kernel(const double *A, double *eval, double *evec) {
    eval[0] = A[0];
    if (evec) evec[0] = 1.0;
}

struct EventSet {
    cudaEvent_t e[6] = {};
    bool on = false;
    int create() {
        for (auto &x : e) CUEV_TRY(cudaEventCreate(&x));
        on = true;
        return CUEV_OK;
    }
    ~EventSet() {
        if (on)
            for (auto &x : e) cudaEventDestroy(x);
    }
};

// Clears the workspace's precision-form flag on every exit path.
struct MixedFlag {
    Workspace *ws;
    ~MixedFlag() {
        if (ws) ws->mixed = 0, ws->fp32 = 0;
    }
};

// mixed == nullptr: the plain FP64 solve.  Otherwise the solve runs with ws->mixed set (the
// back-transform on FP32-level tensor-core products) and, when `refine` is set (the precision
// form), A's FP64-level slices are taken first and the eigenpairs are refined afterwards.
struct MixedReq {
    bool refine;
    int max_iters;
    double tol;
    cuev_mixed_info *info;
    bool fp32_bc_back = false; // FP32 entry: BC-back in FP32
};

// evec_host (optional, with evec): the eigenvectors are also copied there, the finished columns
// while the back-transform's last columns are computed.
int solve_d(double *A, int n, double *eval, double *evec, cudaStream_t stream, cuev_timer *timer,
            const cuev_config *cfg, const MixedReq *mixed = nullptr, double *evec_host = nullptr) {
    if (n < 0) return CUEV_ERR_INVALID;
    if (n == 0) return CUEV_OK;
    if (!A || !eval) return CUEV_ERR_INVALID; // evec == NULL: eigenvalues only
    if (mixed && !evec) return CUEV_ERR_INVALID;
    auto wall0 = std::chrono::high_resolution_clock::now();
    if (n == 1) {
        small_solve_kernel<<<1, 1, 0, stream>>>(A, eval, evec); note_launch();
        CUEV_TRY(cudaGetLastError());
        if (evec && evec_host)
            CUEV_TRY(cudaMemcpyAsync(evec_host, evec, sizeof(double), cudaMemcpyDeviceToHost, stream));
        CUEV_TRY(cudaStreamSynchronize(stream));
        if (timer) *timer = cuev_timer{};
        return CUEV_OK;
    }
    int b = (cfg && cfg->nbw) ? cfg->nbw : default_b(n);
    int k = (cfg && cfg->nk) ? cfg->nk : default_k(n, b);
    Workspace *ws = nullptr;
    bool cached = false;
    CUEV_CHECK_STATUS(acquire_ws(n, b, k, stream, &ws, &cached));
    struct Guard {
        Workspace *ws;
        bool cached;
        ~Guard() { release_ws(ws, cached); }
    } guard{ws, cached};

    EventSet ev;
    if (timer) CUEV_CHECK_STATUS(ev.create());
    auto rec = [&](int i) -> int {
        if (timer) CUEV_TRY(cudaEventRecord(ev.e[i], stream));
        return CUEV_OK;
    };
    CUEV_CHECK_STATUS(apply_wait_limit(ws->status, stream));
    nonfinite_scan_kernel<<<4 * num_sms(), 256, 0, stream>>>(A, n, n, ws->status); note_launch();
    CUEV_TRY(cudaGetLastError());
    CUEV_CHECK_STATUS(workspace_check_status(ws, "input scan"));

    struct HostFlag {
        Workspace *ws;
        ~HostFlag() { ws->host_evec = nullptr; }
    } hflag{ws};
    ws->host_evec = evec ? evec_host : nullptr;
    MixedFlag mflag{nullptr};
    if (mixed) {
        CUEV_CHECK_STATUS(workspace_enable_mixed(ws, mixed->refine));
        // the refinement measures against the original A: keep it as FP64-level slices
        if (mixed->refine) CUEV_CHECK_STATUS(i8_slice(A, n, I8_SRC_SYML, ws->a_sl, stream));
        ws->mixed = 1;
        if (mixed->fp32_bc_back && ws->b == 32) {
            CUEV_CHECK_STATUS(workspace_enable_fp32(ws));
            ws->fp32 = 1;
        }
        mflag.ws = ws;
    }
    CUEV_CHECK_STATUS(rec(0));
    CUEV_CHECK_STATUS(dbbr_reduce(ws, A));
    CUEV_CHECK_STATUS(rec(1));
    CUEV_CHECK_STATUS(bc_chase(ws, ws->B, ws->d, ws->e));
    CUEV_CHECK_STATUS(rec(2));
    if (evec) {
        CUEV_CHECK_STATUS(tridi_dc(ws, ws->d, ws->e, eval, evec));
        CUEV_CHECK_STATUS(rec(3));
        // e[4]: BC-back done on every column (its last wave may overlap SBR-back)
        CUEV_CHECK_STATUS(back_transform(ws, evec, n, timer ? ev.e[4] : nullptr));
    } else { // eigenvalues only: bisection replaces D&C, no back-transform
        CUEV_CHECK_STATUS(tridi_eigvals(ws, ws->d, ws->e, eval));
        CUEV_CHECK_STATUS(rec(3));
        CUEV_CHECK_STATUS(rec(4));
    }
    CUEV_CHECK_STATUS(rec(5));
    CUEV_CHECK_STATUS(workspace_check_status(ws, "solve"));
    if (evec) // the stream is synchronised: an 8-byte read for the profiling counter
        CUEV_TRY(cudaMemcpy(&g_last_dc_flops, ws->dc_flops, sizeof(double), cudaMemcpyDeviceToHost));
    auto wall1 = std::chrono::high_resolution_clock::now();
    if (mixed && mixed->refine) {
        ws->mixed = 0;
        cuev_refine_info ri{};
        CUEV_CHECK_STATUS(refine_core(nullptr, &ws->a_sl, n, eval, evec, mixed->max_iters,
                                      mixed->tol, CUEV_PRODUCTS_INT8, stream, &ri));
        auto wall2 = std::chrono::high_resolution_clock::now();
        if (mixed->info) {
            cuev_mixed_info &mi = *mixed->info;
            mi.refine_iterations = ri.iterations;
            mi.offdiag_fro = ri.offdiag_fro;
            mi.orth_fro = ri.orth_fro;
            mi.anorm = ri.anorm;
            mi.first_ms = std::chrono::duration<float, std::milli>(wall1 - wall0).count();
            mi.refine_ms = std::chrono::duration<float, std::milli>(wall2 - wall1).count();
        }
    }
    if (timer) {
        float t[5];
        for (int i = 0; i < 5; ++i) CUEV_TRY(cudaEventElapsedTime(&t[i], ev.e[i], ev.e[i + 1]));
        *timer = cuev_timer{};
        timer->dbbr_ms = t[0];
        timer->bc_ms = t[1];
        timer->dc_ms = t[2];
        timer->bt_qb_ms = t[3];
        timer->bt_qs_ms = t[4];
        timer->bt_ms = t[3] + t[4];
        if (!evec) timer->bt_qb_ms = timer->bt_qs_ms = timer->bt_ms = 0.0f; // not run
        timer->total_ms = std::chrono::duration<float, std::milli>(wall1 - wall0).count();
    }
    return CUEV_OK;
}

// FP32 entry: per-device widening buffer kept between calls (grown on demand; a stream-ordered
// allocation and release of ~4 GB per call at n = 16384 cost several hundred ms); a call that finds
// it in use on another thread takes a stream-ordered allocation instead.
struct WidenBuf {
    double *p = nullptr;
    size_t bytes = 0;
    bool busy = false;
};
std::mutex g_wb_mu;
WidenBuf g_wb[64]; // FP32 entry
WidenBuf g_hb[64]; // host-buffer entry

// A cached per-device buffer of at least `need` bytes from `arr` (grown on demand), or, when it
// is in use on another thread, a stream-ordered allocation (*cached = false).
int devbuf_acquire(WidenBuf *arr, size_t need, cudaStream_t st, double **out, bool *cached,
                   int *dev_out, const char *what) {
    int dev = 0;
    CUEV_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return CUEV_ERR_INVALID;
    *dev_out = dev;
    *out = nullptr;
    *cached = false;
    {
        std::lock_guard<std::mutex> lk(g_wb_mu);
        WidenBuf &wb = arr[dev];
        if (!wb.busy) {
            if (wb.bytes < need) {
                if (wb.p) cudaFree(wb.p);
                wb.p = nullptr;
                wb.bytes = 0;
                if (cudaMalloc((void **)&wb.p, need) == cudaSuccess) {
                    wb.bytes = need;
                } else {
                    cudaGetLastError();
                    wb.p = nullptr;
                }
            }
            if (wb.p) {
                wb.busy = true;
                *out = wb.p;
                *cached = true;
            }
        }
    }
    if (!*out && cudaMallocAsync((void **)out, need, st) != cudaSuccess) {
        cudaGetLastError();
        *out = nullptr;
        char msg[128];
        snprintf(msg, sizeof(msg), "%s: device buffer allocation failed", what);
        set_last_message(msg);
        return CUEV_ERR_ALLOC;
    }
    return CUEV_OK;
}

// Give back a buffer from devbuf_acquire; the stream must be synchronised for a cached one.
void devbuf_release(WidenBuf *arr, int dev, double *p, bool cached, cudaStream_t st) {
    if (!p) return;
    if (!cached) {
        cudaFreeAsync(p, st);
        return;
    }
    std::lock_guard<std::mutex> lk(g_wb_mu);
    arr[dev].busy = false;
}

__global__ void widen_kernel(const float *__restrict__ s, double *__restrict__ d, long long cnt) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cnt;
         i += (long long)gridDim.x * blockDim.x)
        d[i] = (double)s[i];
}
__global__ void narrow_kernel(const double *__restrict__ s, float *__restrict__ d, long long cnt) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cnt;
         i += (long long)gridDim.x * blockDim.x)
        d[i] = (float)s[i];
}

} // namespace
} // namespace cuev

using namespace cuev;

extern "C" int cuev_dsyevd_cfg(double *A, int n, double *eval, double *evec, void *stream,
                               cuev_timer *timer, const cuev_config *cfg) {
    return solve_d(A, n, eval, evec, (cudaStream_t)stream, timer, cfg);
}

extern "C" int cuev_dsyevd(double *A, int n, double *eval, double *evec, void *stream,
                           cuev_timer *timer) {
    return solve_d(A, n, eval, evec, (cudaStream_t)stream, timer, nullptr);
}

extern "C" int cuev_dsyevd_mixed(double *A, int n, double *eval, double *evec, void *stream,
                                 cuev_timer *timer, int max_refine_iters, double tol,
                                 cuev_mixed_info *info) {
    if (max_refine_iters < 0) return CUEV_ERR_INVALID;
    if (info) *info = cuev_mixed_info{};
    if (n == 1) return solve_d(A, n, eval, evec, (cudaStream_t)stream, timer, nullptr);
    MixedReq req{true, max_refine_iters, tol, info};
    return solve_d(A, n, eval, evec, (cudaStream_t)stream, timer, nullptr, &req);
}

extern "C" int cuev_ssyevd(float *A, int n, float *eval, float *evec, void *stream,
                           cuev_timer *timer) {
    if (n < 0) return CUEV_ERR_INVALID;
    if (n == 0) return CUEV_OK;
    if (!A || !eval) return CUEV_ERR_INVALID; // evec == NULL: eigenvalues only
    cudaStream_t st = (cudaStream_t)stream;
    const long long nn = (long long)n * n;
    const size_t need = sizeof(double) * (2 * nn + n);
    int dev = 0;
    double *buf = nullptr;
    bool cached = false;
    CUEV_CHECK_STATUS(devbuf_acquire(g_wb, need, st, &buf, &cached, &dev, "FP32 entry"));
    double *A64 = buf, *V64 = buf + nn, *w64 = buf + 2 * nn;
    const int blocks = 4 * num_sms();
    widen_kernel<<<blocks, 256, 0, st>>>(A, A64, nn); note_launch();
    // FP32 results need FP32 accuracy only: BC-back runs in FP32 (b = 32) and the back-transform's
    // large products on the int8 tensor cores at FP32 level (the precision form's first solve,
    // without refinement)
    MixedReq first_only{false, 0, 0.0, nullptr, true};
    int s = solve_d(A64, n, w64, evec ? V64 : nullptr, st, timer, nullptr,
                    evec ? &first_only : nullptr);
    if (s == CUEV_OK) {
        if (evec) { narrow_kernel<<<blocks, 256, 0, st>>>(V64, evec, nn); note_launch(); }
        narrow_kernel<<<1, 256, 0, st>>>(w64, eval, n); note_launch();
        narrow_kernel<<<blocks, 256, 0, st>>>(A64, A, nn); note_launch(); // A is clobbered like the reference's
    }
    if (!cached) devbuf_release(g_wb, dev, buf, false, st);
    if (cudaStreamSynchronize(st) != cudaSuccess && s == CUEV_OK) s = CUEV_ERR_CUDA;
    if (cached) devbuf_release(g_wb, dev, buf, true, st);
    return s;
}

extern "C" int cuev_dsyevd_host(const double *A_host, int n, double *eval_host,
                                double *evec_host, void *stream, cuev_timer *timer) {
    if (n < 0) return CUEV_ERR_INVALID;
    if (n == 0) return CUEV_OK;
    if (!A_host || !eval_host) return CUEV_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    const long long nn = (long long)n * n;
    const size_t need = sizeof(double) * ((evec_host ? 2 * nn : nn) + n);
    int dev = 0;
    double *buf = nullptr;
    bool cached = false;
    CUEV_CHECK_STATUS(devbuf_acquire(g_hb, need, st, &buf, &cached, &dev, "host-buffer entry"));
    double *dA = buf, *dw = buf + nn, *dV = evec_host ? buf + nn + n : nullptr;
    int s = CUEV_OK;
    if (cudaMemcpyAsync(dA, A_host, sizeof(double) * nn, cudaMemcpyHostToDevice, st) != cudaSuccess)
        s = CUEV_ERR_CUDA;
    // the eigenvectors reach evec_host inside the solve (copied out column block by column block)
    if (s == CUEV_OK) s = solve_d(dA, n, dw, dV, st, timer, nullptr, nullptr, evec_host);
    if (s == CUEV_OK &&
        cudaMemcpyAsync(eval_host, dw, sizeof(double) * n, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        s = CUEV_ERR_CUDA;
    if (!cached) devbuf_release(g_hb, dev, buf, false, st);
    if (cudaStreamSynchronize(st) != cudaSuccess && s == CUEV_OK) s = CUEV_ERR_CUDA;
    if (cached) devbuf_release(g_hb, dev, buf, true, st);
    return s;
}

extern "C" double cuev_last_dc_flops(void) { return cuev::g_last_dc_flops; }

namespace cuev {
void batched_mid_release();
}

extern "C" int cuev_release_workspace(void) {
    cuev::batched_mid_release();
    {
        std::lock_guard<std::mutex> lk(cuev::g_wb_mu);
        int cur = 0;
        if (cudaGetDevice(&cur) == cudaSuccess) {
            for (cuev::WidenBuf *arr : {cuev::g_wb, cuev::g_hb})
                for (int d = 0; d < 64; ++d)
                    if (arr[d].p && !arr[d].busy) {
                        if (cudaSetDevice(d) == cudaSuccess) cudaFree(arr[d].p);
                        arr[d].p = nullptr;
                        arr[d].bytes = 0;
                    }
            cudaSetDevice(cur);
        }
        cudaGetLastError();
    }
    std::lock_guard<std::mutex> lk(g_cache_mu);
    for (auto &c : g_cache) {
        if (c.ws && !c.busy) {
            workspace_destroy(c.ws);
            c.ws = nullptr;
        }
    }
    return CUEV_OK;
}

// ---------------------------------------------------------------------------------------------
// Stage-level API
// ---------------------------------------------------------------------------------------------
extern "C" int cuev_handle_create(int n, int nbw, int nk, void *stream, cuev_handle *out) {
    if (!out) return CUEV_ERR_INVALID;
    *out = nullptr;
    Workspace *ws = nullptr;
    CUEV_CHECK_STATUS(workspace_create(n, nbw, nk, (cudaStream_t)stream, &ws));
    *out = new cuev_handle_s{ws};
    return CUEV_OK;
}

extern "C" int cuev_handle_destroy(cuev_handle h) {
    if (!h) return CUEV_ERR_INVALID;
    if (h->ws) {
        cudaStreamSynchronize(h->ws->stream);
        workspace_destroy(h->ws);
    }
    delete h;
    return CUEV_OK;
}

extern "C" int cuev_handle_buffer(cuev_handle h, int which, void **ptr, long long *ld) {
    if (!h || !h->ws || !ptr || !ld) return CUEV_ERR_INVALID;
    Workspace *ws = h->ws;
    switch (which) {
    case CUEV_BUF_B: *ptr = ws->B, *ld = 2LL * ws->b; break;
    case CUEV_BUF_D: *ptr = ws->d, *ld = ws->n; break;
    case CUEV_BUF_E: *ptr = ws->e, *ld = ws->n; break;
    case CUEV_BUF_Y: *ptr = ws->Y, *ld = ws->n; break;
    case CUEV_BUF_U: *ptr = ws->U, *ld = ws->n; break;
    case CUEV_BUF_TAU: *ptr = ws->tau, *ld = ws->n; break;
    default: return CUEV_ERR_INVALID;
    }
    return CUEV_OK;
}

#define HCHECK(h)                                                                                  \
    do {                                                                                           \
        if (!(h) || !(h)->ws) return CUEV_ERR_INVALID;                                             \
        CUEV_CHECK_STATUS(apply_wait_limit((h)->ws->status, (h)->ws->stream));                     \
    } while (0)

extern "C" int cuev_dbbr_panel_qr(cuev_handle h, double *A, int lda, double *Y, int ldy,
                                  double *tau, double *T, int rows, int b) {
    HCHECK(h);
    if (rows < 0 || b <= 0 || b > 64 || lda < rows || ldy < rows || !A || !Y || !tau || !T)
        return CUEV_ERR_INVALID;
    CUEV_CHECK_STATUS(panel_qr(h->ws, A, lda, Y, ldy, tau, T, nullptr, 0, rows, b));
    return workspace_check_status(h->ws, "dbbr_panel_qr");
}

extern "C" int cuev_dbbr_reduce(cuev_handle h, double *A) {
    HCHECK(h);
    if (!A) return CUEV_ERR_INVALID;
    CUEV_CHECK_STATUS(dbbr_reduce(h->ws, A));
    return workspace_check_status(h->ws, "dbbr_reduce");
}

extern "C" int cuev_dbbr_pack(cuev_handle h, const double *A, double *B) {
    HCHECK(h);
    if (!A || !B) return CUEV_ERR_INVALID;
    return dbbr_pack(h->ws, A, h->ws->n, B);
}

extern "C" int cuev_bc_chase(cuev_handle h, double *B, double *d, double *e) {
    HCHECK(h);
    if (!B || !d || !e) return CUEV_ERR_INVALID;
    CUEV_CHECK_STATUS(bc_chase(h->ws, B, d, e));
    return workspace_check_status(h->ws, "bc_chase");
}

extern "C" int cuev_tridi_dc(cuev_handle h, const double *d, const double *e, double *eval,
                             double *evec) {
    HCHECK(h);
    if (!d || !e || !eval || !evec) return CUEV_ERR_INVALID;
    CUEV_CHECK_STATUS(tridi_dc(h->ws, d, e, eval, evec));
    return workspace_check_status(h->ws, "tridi_dc");
}

extern "C" int cuev_tridi_eigvals(cuev_handle h, const double *d, const double *e, double *eval) {
    HCHECK(h);
    if (!d || !e || !eval) return CUEV_ERR_INVALID;
    CUEV_CHECK_STATUS(tridi_eigvals(h->ws, d, e, eval));
    return workspace_check_status(h->ws, "tridi_eigvals");
}

extern "C" int cuev_bc_back(cuev_handle h, double *M, int ldm) {
    HCHECK(h);
    if (!M || ldm < h->ws->n) return CUEV_ERR_INVALID;
    return bc_back(h->ws, M, ldm);
}

extern "C" int cuev_sbr_back(cuev_handle h, double *M, int ldm) {
    HCHECK(h);
    if (!M || ldm < h->ws->n) return CUEV_ERR_INVALID;
    return sbr_back(h->ws, M, ldm);
}

extern "C" int cuev_back_transform(cuev_handle h, double *evec, cuev_timer *timer) {
    HCHECK(h);
    if (!evec) return CUEV_ERR_INVALID;
    Workspace *ws = h->ws;
    EventSet ev;
    if (timer) CUEV_CHECK_STATUS(ev.create());
    if (timer) CUEV_TRY(cudaEventRecord(ev.e[0], ws->stream));
    CUEV_CHECK_STATUS(back_transform(ws, evec, ws->n, timer ? ev.e[1] : nullptr));
    if (timer) {
        CUEV_TRY(cudaEventRecord(ev.e[2], ws->stream));
        CUEV_TRY(cudaEventSynchronize(ev.e[2]));
        *timer = cuev_timer{};
        CUEV_TRY(cudaEventElapsedTime(&timer->bt_qb_ms, ev.e[0], ev.e[1]));
        CUEV_TRY(cudaEventElapsedTime(&timer->bt_qs_ms, ev.e[1], ev.e[2]));
        timer->bt_ms = timer->bt_qb_ms + timer->bt_qs_ms;
    }
    return workspace_check_status(ws, "back_transform");
}

// ---------------------------------------------------------------------------------------------
// C++ drop-in: cuev::symm_eig_solve<T> with the reference's signature and mangled names.
// ---------------------------------------------------------------------------------------------
static_assert(sizeof(cuev::SolveTimer) == sizeof(cuev_timer), "SolveTimer layout");

namespace cuev {
template <>
void symm_eig_solve<double>(double *A, int n, double *eval, double *evec, cudaStream_t stream,
                            SolveTimer *timer) {
    const int st = cuev_dsyevd(A, n, eval, evec, stream, reinterpret_cast<cuev_timer *>(timer));
    if (st != CUEV_OK) {
        fprintf(stderr, "cuev::symm_eig_solve<double> failed: %d (%s)\n", st, cuev_last_error());
        exit(1);
    }
}
template <>
void symm_eig_solve<float>(float *A, int n, float *eval, float *evec, cudaStream_t stream,
                           SolveTimer *timer) {
    const int st = cuev_ssyevd(A, n, eval, evec, stream, reinterpret_cast<cuev_timer *>(timer));
    if (st != CUEV_OK) {
        fprintf(stderr, "cuev::symm_eig_solve<float> failed: %d (%s)\n", st, cuev_last_error());
        exit(1);
    }
}
} // namespace cuev
