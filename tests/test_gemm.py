"""FP64 DMMA GEMM / SYMM / SYR2K parity against torch fp64 (the reference's cuBLAS calls,
src/cuda/cublas.cu:15-56, are what these kernels replace)."""
import pytest

from conftest import colmajor, logical

pytestmark = pytest.mark.gpu

CASES = [(1, 1, 1), (17, 9, 5), (64, 64, 64), (130, 70, 33), (257, 129, 300), (1000, 64, 2000),
         (64, 1000, 777), (513, 515, 517), (96, 32, 4096)]


@pytest.mark.parametrize("ta", [0, 1])
@pytest.mark.parametrize("tb", [0, 1])
@pytest.mark.parametrize("m,n,k", CASES)
def test_dgemm(cuda, ta, tb, m, n, k):
    import torch
    import cuev_b200 as cv
    g = torch.Generator(device="cpu").manual_seed(m * 7 + n * 13 + k)
    A = torch.randn((k, m) if ta else (m, k), generator=g, dtype=torch.float64).to(cuda)
    B = torch.randn((n, k) if tb else (k, n), generator=g, dtype=torch.float64).to(cuda)
    Cl = torch.randn(m, n, generator=g, dtype=torch.float64).to(cuda)
    Acm, Bcm, Ccm = colmajor(A), colmajor(B), colmajor(Cl)
    alpha, beta = 1.25, -0.5
    cv.dgemm(ta, tb, m, n, k, alpha, Acm, A.shape[0], Bcm, B.shape[0], beta, Ccm, m)
    torch.cuda.synchronize()
    opA = A.t() if ta else A
    opB = B.t() if tb else B
    ref = alpha * (opA @ opB) + beta * Cl
    err = (logical(Ccm) - ref).abs().max().item()
    scale = (opA.abs() @ opB.abs()).max().item() * abs(alpha) + 1.0
    assert err <= 1e-14 * max(1, k) ** 0.5 * scale + 1e-13, err


@pytest.mark.parametrize("m,n", [(5, 3), (64, 64), (200, 32), (1031, 64), (4096, 64)])
def test_dsymm_lower(cuda, m, n):
    import torch
    import cuev_b200 as cv
    g = torch.Generator(device="cpu").manual_seed(m + n)
    A = torch.randn(m, m, generator=g, dtype=torch.float64).to(cuda)  # only lower is read
    S = torch.tril(A) + torch.tril(A, -1).t()
    B = torch.randn(m, n, generator=g, dtype=torch.float64).to(cuda)
    Ccm = colmajor(torch.zeros(m, n, dtype=torch.float64, device=cuda))
    cv.dsymm_lower(m, n, 1.0, colmajor(A), m, colmajor(B), m, 0.0, Ccm, m)
    torch.cuda.synchronize()
    ref = S @ B
    assert (logical(Ccm) - ref).abs().max().item() < 1e-12 * m ** 0.5


@pytest.mark.parametrize("n,k", [(7, 3), (128, 64), (333, 96), (1500, 512)])
def test_dsyr2k_lower(cuda, n, k):
    import torch
    import cuev_b200 as cv
    g = torch.Generator(device="cpu").manual_seed(n * 3 + k)
    Y = torch.randn(n, k, generator=g, dtype=torch.float64).to(cuda)
    Z = torch.randn(n, k, generator=g, dtype=torch.float64).to(cuda)
    C0 = torch.randn(n, n, generator=g, dtype=torch.float64).to(cuda)
    Ccm = colmajor(C0)
    cv.dsyr2k_lower(n, k, -1.0, colmajor(Y), n, colmajor(Z), n, 1.0, Ccm, n)
    torch.cuda.synchronize()
    out = logical(Ccm)
    ref = C0 - Y @ Z.t() - Z @ Y.t()
    lo = torch.tril(torch.ones(n, n, dtype=torch.bool, device=cuda))
    assert (out - ref)[lo].abs().max().item() < 1e-12 * k ** 0.5
    assert torch.equal(out[~lo], C0[~lo])  # strict upper triangle untouched
