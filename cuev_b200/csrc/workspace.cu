// Device workspace of one (n, b, k) solve: a single pool allocation carved into the buffers
// listed in solver.cuh.  The reference allocates and frees its pool on every call
// (src/cuda/handle.cu:16-101); here the solve entry points cache one workspace per device and
// (n, b, k) so the steady state does no cudaMalloc.
#include "solver.cuh"

#include <algorithm>

namespace cuev {

namespace {
// split-K partials: room for two splits of a k x n product (the SBR-back's Y^T M and T X, 512
// tiles of 128 x 128 at k = 512: 3.5 waves, which split in two run as 7 half-length waves instead
// of 4 full ones; SBR-back 368 -> 351 ms at n = 16384), and at least three waves' worth of
// 128 x 128 tiles
size_t splitk_cap_bytes(size_t n, int k) {
    return std::max((size_t)3 * num_sms() * 128 * 128, 2 * (size_t)k * n) * sizeof(double);
}
} // namespace

int workspace_create(int n, int b, int k, cudaStream_t stream, Workspace **out) {
    *out = nullptr;
    if (n < 0 || (b != 32 && b != 64) || k < b || k % b != 0) {
        set_last_message("workspace: need b in {32, 64} and k a positive multiple of b");
        return CUEV_ERR_INVALID;
    }
    Workspace *ws = new Workspace();
    ws->n = n, ws->b = b, ws->k = k, ws->stream = stream;
    CUEV_TRY(cudaGetDevice(&ws->dev));
    const size_t N = (size_t)std::max(n, 1);
    const size_t nn = N * N;
    const size_t s = sizeof(double);
    const int sms = num_sms();

    struct Item {
        void **p;
        size_t bytes;
    };
    ws->qr_part_elems = (size_t)(2 * sms + 2) * 64;
    ws->splitk_bytes = splitk_cap_bytes(N, k);
    ws->dc_vec_elems = 24 * N + 64;
    ws->dc_int_elems = 24 * N + 64;
    ws->dc_gemm_args_cap = 2 * (int)(N / 8 + 8);
    Item items[] = {
        {(void **)&ws->Y, nn * s},
        {(void **)&ws->U, nn * s},
        {(void **)&ws->dc_Q2, nn * s},
        // dc_S also carries BC-Back's round-to-round rows: ceil(n/32) groups of n x 32
        {(void **)&ws->dc_S, N * ((N + 31) / 32 * 32) * s},
        {(void **)&ws->dc_T, nn * s},
        {(void **)&ws->Z, N * k * s},
        {(void **)&ws->Wp, N * b * s},
        {(void **)&ws->Tp, (N / b + 2) * b * b * s},
        {(void **)&ws->Tblk, (N / k + 2) * (size_t)k * k * s},
        {(void **)&ws->tau, (N + 64) * s},
        {(void **)&ws->Dwk, 2 * (size_t)k * b * s},
        {(void **)&ws->Gblk, (size_t)k * k * s},
        {(void **)&ws->B, 2 * (size_t)b * N * s},
        {(void **)&ws->d, N * s},
        {(void **)&ws->e, N * s},
        {(void **)&ws->prog, 2 * N * sizeof(int)}, // chase: hops done, betas written
        {(void **)&ws->bar, 64},
        {(void **)&ws->status, DEV_STATUS_WORDS * sizeof(int)},
        {(void **)&ws->dc_flops, sizeof(double)},
        {(void **)&ws->qr_part, ws->qr_part_elems * s},
        {(void **)&ws->splitk, ws->splitk_bytes},
        {(void **)&ws->dc_vec, ws->dc_vec_elems * s},
        {(void **)&ws->dc_int, ws->dc_int_elems * sizeof(int)},
        {(void **)&ws->dc_gemm_args, (size_t)ws->dc_gemm_args_cap * sizeof(GemmArgs)},
    };
    size_t total = 0;
    for (auto &it : items) total += align256(it.bytes);
    if (cudaMalloc(&ws->pool, total) != cudaSuccess) {
        cudaGetLastError();
        delete ws;
        char msg[160];
        snprintf(msg, sizeof(msg), "workspace allocation of %.2f GB failed", total / 1e9);
        set_last_message(msg);
        return CUEV_ERR_ALLOC;
    }
    ws->pool_bytes = total;
    size_t off = 0;
    for (auto &it : items) {
        *it.p = (char *)ws->pool + off;
        off += align256(it.bytes);
    }
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess ||
        cudaStreamCreateWithPriority(&ws->side, cudaStreamNonBlocking, greatest) != cudaSuccess ||
        cudaEventCreateWithFlags(&ws->ev_a, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ws->ev_b, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ws->ev_c, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ws->ev_d, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        workspace_destroy(ws);
        set_last_message("workspace: stream or event creation failed");
        return CUEV_ERR_CUDA;
    }
    CUEV_TRY(cudaMemsetAsync(ws->status, 0, DEV_STATUS_WORDS * sizeof(int), stream));
    CUEV_TRY(cudaMemsetAsync(ws->bar, 0, 64, stream));
    *out = ws;
    return CUEV_OK;
}

// The operands of the largest mixed GEMM (the SBR-back's Y^T M: k x n by n x n, FP32-level
// slices) and, for the refinement, A's FP64-level slices.
int workspace_enable_mixed(Workspace *ws, bool with_a_slices) {
    if (ws->mx_pool && (ws->mx_has_a || !with_a_slices)) return CUEV_OK;
    if (ws->mx_pool) { // grow: A's slices were not allocated yet
        CUEV_TRY(cudaStreamSynchronize(ws->stream));
        cudaFree(ws->mx_pool);
        ws->mx_pool = nullptr;
    }
    const int n = std::max(ws->n, 1);
    const size_t a_bytes = with_a_slices ? i8_operand_bytes(n, n, RF_SLICES_HI) : 0;
    const size_t g_bytes = i8_gemm_scratch_bytes(std::max(ws->k, n), n, n, MIXED_SLICES);
    const size_t total = align256(a_bytes) + align256(g_bytes);
    if (cudaMalloc(&ws->mx_pool, total) != cudaSuccess) {
        cudaGetLastError();
        ws->mx_pool = nullptr;
        char msg[160];
        snprintf(msg, sizeof(msg), "precision form: allocation of %.2f GB failed", total / 1e9);
        set_last_message(msg);
        return CUEV_ERR_ALLOC;
    }
    ws->mx_bytes = total;
    ws->mx_has_a = with_a_slices;
    char *p = (char *)ws->mx_pool;
    ws->i8_scratch = p;
    ws->i8_scratch_bytes = g_bytes;
    p += align256(g_bytes);
    if (with_a_slices) i8_operand_init(p, n, n, RF_SLICES_HI, ws->a_sl);
    return CUEV_OK;
}

int workspace_enable_fp32(Workspace *ws) {
    if (ws->f32_pool) return CUEV_OK;
    const size_t nn = (size_t)std::max(ws->n, 1) * std::max(ws->n, 1);
    const size_t total = 2 * align256(nn * sizeof(float));
    if (cudaMalloc(&ws->f32_pool, total) != cudaSuccess) {
        cudaGetLastError();
        ws->f32_pool = nullptr;
        char msg[160];
        snprintf(msg, sizeof(msg), "FP32 entry: allocation of %.2f GB failed", total / 1e9);
        set_last_message(msg);
        return CUEV_ERR_ALLOC;
    }
    ws->Uf = (float *)ws->f32_pool;
    ws->Mf = (float *)((char *)ws->f32_pool + align256(nn * sizeof(float)));
    return CUEV_OK;
}

void workspace_destroy(Workspace *ws) {
    if (!ws) return;
    if (ws->mx_pool) cudaFree(ws->mx_pool);
    if (ws->f32_pool) cudaFree(ws->f32_pool);
    if (ws->side) cudaStreamSynchronize(ws->side), cudaStreamDestroy(ws->side);
    if (ws->ev_a) cudaEventDestroy(ws->ev_a);
    if (ws->ev_b) cudaEventDestroy(ws->ev_b);
    if (ws->ev_c) cudaEventDestroy(ws->ev_c);
    if (ws->ev_d) cudaEventDestroy(ws->ev_d);
    if (ws->pool) cudaFree(ws->pool);
    delete ws;
}

int workspace_check_status(Workspace *ws, const char *stage) {
    int h[DEV_STATUS_WORDS] = {0};
    CUEV_CHECK_STATUS(gemm_fold_fault(ws->status, ws->stream));
    CUEV_TRY(cudaMemcpyAsync(h, ws->status, sizeof(h), cudaMemcpyDeviceToHost, ws->stream));
    CUEV_TRY(cudaStreamSynchronize(ws->stream));
    if (h[DEV_STATUS_CODE] != 0) {
        char msg[200];
        snprintf(msg, sizeof(msg), "%s: device status %d (detail %d)", stage, h[DEV_STATUS_CODE],
                 h[DEV_STATUS_WHERE]);
        set_last_message(msg);
        // clear for the next call
        CUEV_TRY(cudaMemsetAsync(ws->status, 0, DEV_STATUS_WORDS * sizeof(int), ws->stream));
        CUEV_TRY(cudaMemsetAsync(ws->bar, 0, 64, ws->stream));
        return h[DEV_STATUS_CODE];
    }
    return CUEV_OK;
}

// splits whose m x n partials fit the workspace's split-K scratch
static int splitk_fit(const Workspace *ws, int m, int n) {
    const size_t one = (size_t)m * n * sizeof(double);
    return one ? (int)std::min<size_t>(32, ws->splitk_bytes / one) : 32;
}

int ws_gemm2(Workspace *ws, int ta, int tb, int m, int n, int k, int k2, double alpha,
             const double *A, long long lda, const double *A2, long long lda2, const double *B,
             long long ldb, const double *B2, long long ldb2, double beta, double *C,
             long long ldc, int c_lower) {
    GemmArgs a{};
    a.m = m, a.n = n, a.k = k, a.k2 = k2;
    a.A = A, a.lda = lda, a.A2 = A2, a.lda2 = lda2;
    a.B = B, a.ldb = ldb, a.B2 = B2, a.ldb2 = ldb2;
    a.C = C, a.ldc = ldc, a.alpha = alpha, a.beta = beta, a.c_lower = c_lower;
    int splits = gemm_splitk_count(m, n, k + k2, c_lower, splitk_fit(ws, m, n));
    while (splits > 1 && (size_t)splits * m * n * sizeof(double) > ws->splitk_bytes) --splits;
    a.splits = splits;
    a.ws = splits > 1 ? ws->splitk : nullptr;
    return gemm_launch(a, ta, tb, ws->stream);
}

int ws_gemm(Workspace *ws, int ta, int tb, int m, int n, int k, double alpha, const double *A,
            long long lda, const double *B, long long ldb, double beta, double *C, long long ldc) {
    return ws_gemm2(ws, ta, tb, m, n, k, 0, alpha, A, lda, nullptr, 0, B, ldb, nullptr, 0, beta, C,
                    ldc, 0);
}

int ws_symm(Workspace *ws, int m, int n, double alpha, const double *A, long long lda,
            const double *B, long long ldb, double beta, double *C, long long ldc) {
    GemmArgs a{};
    a.m = m, a.n = n, a.k = m;
    a.A = A, a.lda = lda, a.B = B, a.ldb = ldb, a.C = C, a.ldc = ldc;
    a.alpha = alpha, a.beta = beta, a.symm_a = 1;
    int splits = gemm_splitk_count(m, n, m, 0, splitk_fit(ws, m, n));
    while (splits > 1 && (size_t)splits * m * n * sizeof(double) > ws->splitk_bytes) --splits;
    a.splits = splits;
    a.ws = splits > 1 ? ws->splitk : nullptr;
    return gemm_launch(a, 0, 0, ws->stream);
}

} // namespace cuev
