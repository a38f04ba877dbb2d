"""cuev_dgemm_noalloc — the GEMM entry for callers that cannot allocate device memory (e.g. a
process whose framework's caching allocator owns the GPU memory, or a latency-critical loop that
must not block on a device allocation).  It must give the same result as cuev_dgemm, which
allocates its split-K scratch with cudaMalloc, on consecutive calls that reuse the shared static
scratch, and both must agree with torch fp64.  Collected last so that a failure here does not
hide the other tests."""
import pytest

from conftest import colmajor, logical

pytestmark = pytest.mark.gpu

# (ta, tb, m, n, k): tall-skinny reductions that split K (the D = Y^T W shape of the band
# reduction), a general product and an odd-sized one
# the D = Y^T W shape of the band reduction), a general product, an odd-sized one, k = 32 (two
# 16-deep K tiles split two ways: the second split's partial must be written even when its K
# range is short) and m * n exactly at the 1,048,576 limit with a two-way split
CASES = [(1, 0, 512, 64, 16384), (0, 0, 128, 64, 50000), (0, 1, 300, 200, 4000),
         (1, 1, 97, 33, 3001), (0, 0, 64, 64, 32), (0, 0, 1024, 1024, 512)]


def _inputs(cuda, ta, tb, m, n, k, seed):
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    A = torch.randn((k, m) if ta else (m, k), generator=g, dtype=torch.float64).to(cuda)
    B = torch.randn((n, k) if tb else (k, n), generator=g, dtype=torch.float64).to(cuda)
    C0 = torch.randn(m, n, generator=g, dtype=torch.float64).to(cuda)
    return A, B, C0


@pytest.mark.parametrize("ta,tb,m,n,k", CASES)
def test_noalloc_matches_dgemm_twice(cuda, ta, tb, m, n, k):
    import torch
    import cuev_b200 as cv
    alpha, beta = 0.75, -1.5
    for call in range(2):  # the second call reuses scratch left over by the first
        A, B, C0 = _inputs(cuda, ta, tb, m, n, k, seed=1000 * call + m + n + k)
        ref = colmajor(C0)
        out = colmajor(C0)
        cv.dgemm(ta, tb, m, n, k, alpha, colmajor(A), A.shape[0], colmajor(B), B.shape[0], beta,
                 ref, m)
        cv.dgemm_noalloc(ta, tb, m, n, k, alpha, colmajor(A), A.shape[0], colmajor(B),
                         B.shape[0], beta, out, m)
        torch.cuda.synchronize()
        opA = A.t() if ta else A
        opB = B.t() if tb else B
        scale = (opA.abs() @ opB.abs()).max().item() * abs(alpha) + abs(beta) * C0.abs().max().item()
        err = (logical(out) - logical(ref)).abs().max().item()
        assert err <= 1e-14 * k ** 0.5 * scale, (call, err)
        # and against torch fp64 directly (an independent product, not the same kernel family)
        want = alpha * (opA @ opB) + beta * C0
        err_t = (logical(out) - want).abs().max().item()
        assert err_t <= 1e-14 * k ** 0.5 * scale, (call, err_t)


def test_noalloc_allocates_nothing(cuda):
    """After a warm-up call (which may load the library's module on this device and so commit
    the static array), further calls leave the device's free memory unchanged."""
    import torch
    import cuev_b200 as cv
    m, n, k = 700, 500, 9000
    A, B, C0 = _inputs(cuda, 0, 0, m, n, k, seed=5)
    Acm, Bcm, Ccm = colmajor(A), colmajor(B), colmajor(C0)
    cv.dgemm_noalloc(0, 0, m, n, k, 1.0, Acm, m, Bcm, k, 0.0, Ccm, m)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(5):
        cv.dgemm_noalloc(0, 0, m, n, k, 1.0, Acm, m, Bcm, k, 0.5, Ccm, m)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_invalid_arguments_have_messages(cuda):
    import torch
    import cuev_b200 as cv
    A = torch.zeros(64, dtype=torch.float64, device=cuda)
    with pytest.raises(cv.CuevError) as ei:
        cv.dgemm_noalloc(0, 0, 8, 8, 8, 1.0, A, 4, A, 8, 0.0, A, 8)  # lda < m
    assert ei.value.status == -1 and "leading dimension" in str(ei.value)


def test_noalloc_rejects_oversize(cuda):
    import torch
    import cuev_b200 as cv
    m = n = 1025  # m * n > 1048576
    A = torch.zeros(m * 64, dtype=torch.float64, device=cuda)
    B = torch.zeros(64 * n, dtype=torch.float64, device=cuda)
    C = torch.zeros(m * n, dtype=torch.float64, device=cuda)
    with pytest.raises(cv.CuevError) as ei:
        cv.dgemm_noalloc(0, 0, m, n, 64, 1.0, A, m, B, 64, 0.0, C, m)
    assert ei.value.status == -1
    assert "static-scratch limit" in str(ei.value)
