// Runs the reference solver (built from its own sources) on a matrix file.  Test infrastructure.
//   ref_driver <n> <in.bin> <eval_out.bin> [evec_out.bin]
// in.bin: n*n doubles, column-major.  Prints one JSON line with the reference's SolveTimer.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include <cuda_runtime.h>

#include "cuev.h"

int main(int argc, char **argv) {
    if (argc < 4) {
        fprintf(stderr, "usage: %s n in.bin eval.bin [evec.bin]\n", argv[0]);
        return 2;
    }
    const int n = atoi(argv[1]);
    const size_t nn = (size_t)n * n;
    std::vector<double> A(nn), w(n), V(nn);
    FILE *f = fopen(argv[2], "rb");
    if (!f || fread(A.data(), sizeof(double), nn, f) != nn) {
        fprintf(stderr, "cannot read %s\n", argv[2]);
        return 2;
    }
    fclose(f);
    double *dA, *dw, *dV;
    cudaMalloc(&dA, nn * sizeof(double));
    cudaMalloc(&dw, n * sizeof(double));
    cudaMalloc(&dV, nn * sizeof(double));
    cudaStream_t st;
    cudaStreamCreate(&st);
    cudaMemcpy(dA, A.data(), nn * sizeof(double), cudaMemcpyHostToDevice);
    cuev::SolveTimer t;
    cuev::symm_eig_solve<double>(dA, n, dw, dV, st, &t);
    cudaMemcpy(w.data(), dw, n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaMemcpy(V.data(), dV, nn * sizeof(double), cudaMemcpyDeviceToHost);
    f = fopen(argv[3], "wb");
    fwrite(w.data(), sizeof(double), n, f);
    fclose(f);
    if (argc > 4) {
        f = fopen(argv[4], "wb");
        fwrite(V.data(), sizeof(double), nn, f);
        fclose(f);
    }
    printf("{\"n\": %d, \"dbbr_ms\": %.3f, \"bc_ms\": %.3f, \"dc_ms\": %.3f, \"bt_ms\": %.3f, "
           "\"total_ms\": %.3f}\n",
           n, t.dbbr_ms, t.bc_ms, t.dc_ms, t.bt_ms, t.total_ms);
    return 0;
}
