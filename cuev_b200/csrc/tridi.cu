// Stage 3: tridiagonal divide and conquer on the GPU (placeholder until the kernels land).
#include "solver.cuh"

namespace cuev {
int tridi_dc(Workspace *ws, const double *d, const double *e, double *eval, double *evec) {
    (void)ws, (void)d, (void)e, (void)eval, (void)evec;
    set_last_message("tridi_dc: not built yet");
    return CUEV_ERR_UNSUPPORTED;
}
} // namespace cuev
