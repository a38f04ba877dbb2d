// Runs the reference solver (built from its own sources) on a matrix file.  Test infrastructure:
// golden outputs (tests/golden/make_ref_golden.py) and the reference arm of bench.py.
//   ref_driver <n> <in.bin> <eval_out.bin|-> [evec_out.bin|-] [reps] [warmup]
// in.bin: n*n doubles, column-major.  Each of warmup + reps solves copies A from pinned host
// memory, calls cuev::symm_eig_solve<double> (the reference's public entry, stock code path) and
// copies eval and evec back; the outputs of the last solve are written.  One JSON line per timed
// solve: the reference's SolveTimer, the solve's device time (CUDA events around the call) and
// the end-to-end time including both copies.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include <cuda_runtime.h>

#include "cuev.h"

static int fail(const char *what) {
    fprintf(stderr, "ref_driver: %s\n", what);
    return 2;
}

int main(int argc, char **argv) {
    if (argc < 4) {
        fprintf(stderr, "usage: %s n in.bin eval.bin|- [evec.bin|-] [reps] [warmup]\n", argv[0]);
        return 2;
    }
    const int n = atoi(argv[1]);
    const char *evec_path = argc > 4 ? argv[4] : "-";
    const int reps = argc > 5 ? atoi(argv[5]) : 1;
    const int warmup = argc > 6 ? atoi(argv[6]) : 0;
    if (n <= 0 || reps < 1 || warmup < 0) return fail("bad arguments");
    const size_t nn = (size_t)n * n;
    double *hA = nullptr, *hw = nullptr, *hV = nullptr;
    if (cudaMallocHost((void **)&hA, nn * sizeof(double)) != cudaSuccess ||
        cudaMallocHost((void **)&hw, n * sizeof(double)) != cudaSuccess ||
        cudaMallocHost((void **)&hV, nn * sizeof(double)) != cudaSuccess)
        return fail("pinned host allocation failed");
    FILE *f = fopen(argv[2], "rb");
    if (!f || fread(hA, sizeof(double), nn, f) != nn) return fail("cannot read the input");
    fclose(f);
    double *dA, *dw, *dV;
    if (cudaMalloc(&dA, nn * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&dw, n * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&dV, nn * sizeof(double)) != cudaSuccess)
        return fail("device allocation failed");
    cudaStream_t st;
    cudaStreamCreate(&st);
    cudaEvent_t e0, e1, e2, e3;
    cudaEventCreate(&e0), cudaEventCreate(&e1), cudaEventCreate(&e2), cudaEventCreate(&e3);
    for (int r = 0; r < warmup + reps; ++r) {
        cuev::SolveTimer t;
        memset(&t, 0, sizeof(t));
        cudaEventRecord(e0, st);
        cudaMemcpyAsync(dA, hA, nn * sizeof(double), cudaMemcpyHostToDevice, st);
        cudaEventRecord(e1, st);
        cuev::symm_eig_solve<double>(dA, n, dw, dV, st, &t);
        cudaEventRecord(e2, st);
        cudaMemcpyAsync(hw, dw, n * sizeof(double), cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(hV, dV, nn * sizeof(double), cudaMemcpyDeviceToHost, st);
        cudaEventRecord(e3, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) return fail("CUDA error");
        if (r < warmup) continue;
        float solve_ms = 0.f, e2e_ms = 0.f;
        cudaEventElapsedTime(&solve_ms, e1, e2);
        cudaEventElapsedTime(&e2e_ms, e0, e3);
        printf("{\"n\": %d, \"dbbr_ms\": %.3f, \"bc_ms\": %.3f, \"dc_ms\": %.3f, \"bt_ms\": %.3f, "
               "\"total_ms\": %.3f, \"solve_ms\": %.3f, \"e2e_ms\": %.3f}\n",
               n, t.dbbr_ms, t.bc_ms, t.dc_ms, t.bt_ms, t.total_ms, solve_ms, e2e_ms);
        fflush(stdout);
    }
    if (strcmp(argv[3], "-") != 0) {
        f = fopen(argv[3], "wb");
        if (!f) return fail("cannot write eval");
        fwrite(hw, sizeof(double), n, f);
        fclose(f);
    }
    if (strcmp(evec_path, "-") != 0) {
        f = fopen(evec_path, "wb");
        if (!f) return fail("cannot write evec");
        fwrite(hV, sizeof(double), nn, f);
        fclose(f);
    }
    return 0;
}
