"""FP64 products emulated on the int8 tensor cores (``cuev_dgemm_i8``: tcgen05.mma.kind::i8 behind
TMA, accumulators in TMEM) against torch fp64.

With s slices per operand the error of entry (i, j) is bounded by about
(s + 2) 2^(-7s) K rowmax_i(op(A)) colmax_j(op(B)) (the dropped slice products and remainders);
measured it stays near 14 2^(-7s) sqrt(K) rowmax colmax.  The tests allow 32 2^(-7s) sqrt(K)
rowmax colmax plus FP64 rounding of the beta term."""
import math

import pytest

from conftest import colmajor, logical

pytestmark = pytest.mark.gpu


def _bound(opA, opB, s, alpha, beta, C0):
    k = opA.shape[1]
    rm = opA.abs().amax(dim=1, keepdim=True)
    cm = opB.abs().amax(dim=0, keepdim=True)
    return (32.0 * 2.0 ** (-7 * s) * math.sqrt(max(k, 1)) * abs(alpha) * rm * cm
            + 1e-15 * (abs(alpha) * (opA.abs() @ opB.abs()) + abs(beta) * C0.abs()) + 1e-300)


CASES = [(128, 128, 128), (1, 1, 1), (17, 9, 5), (130, 70, 33), (257, 300, 129),
         (1000, 64, 2000), (64, 1000, 777), (513, 515, 517)]


@pytest.mark.parametrize("s", [7, 4])
@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 0), (0, 1), (1, 1)])
@pytest.mark.parametrize("m,n,k", CASES)
def test_dgemm_i8_vs_torch(cuda, s, ta, tb, m, n, k):
    import torch
    import cuev_b200 as cv
    g = torch.Generator(device="cpu").manual_seed(m * 7 + n * 13 + k + s)
    A = torch.randn((k, m) if ta else (m, k), generator=g, dtype=torch.float64).to(cuda)
    B = torch.randn((n, k) if tb else (k, n), generator=g, dtype=torch.float64).to(cuda)
    C0 = torch.randn(m, n, generator=g, dtype=torch.float64).to(cuda)
    Ccm = colmajor(C0)
    alpha, beta = 1.25, -0.5
    cv.dgemm_i8(ta, tb, m, n, k, s, alpha, colmajor(A), A.shape[0], colmajor(B), B.shape[0],
                beta, Ccm, m)
    torch.cuda.synchronize()
    opA = A.t() if ta else A
    opB = B.t() if tb else B
    ref = alpha * (opA @ opB) + beta * C0
    err = (logical(Ccm) - ref).abs()
    bound = _bound(opA, opB, s, alpha, beta, C0)
    assert bool((err <= bound).all()), (err / bound).max().item()


def test_dgemm_i8_scaled_rows_and_zero_rows(cuda):
    """Rows and columns spanning 2^-60 .. 2^60 and all-zero rows: the per-row power-of-two scaling
    keeps each entry's error relative to its own row and column."""
    import torch
    import cuev_b200 as cv
    m, n, k = 300, 260, 640
    g = torch.Generator(device="cpu").manual_seed(11)
    A = torch.randn(m, k, generator=g, dtype=torch.float64)
    B = torch.randn(k, n, generator=g, dtype=torch.float64)
    A *= torch.pow(2.0, torch.randint(-60, 61, (m, 1), generator=g).double())
    B *= torch.pow(2.0, torch.randint(-60, 61, (1, n), generator=g).double())
    A[5] = 0.0
    B[:, 7] = 0.0
    A, B = A.to(cuda), B.to(cuda)
    Ccm = colmajor(torch.zeros(m, n, dtype=torch.float64, device=cuda))
    cv.dgemm_i8(0, 0, m, n, k, 7, 1.0, colmajor(A), m, colmajor(B), k, 0.0, Ccm, m)
    torch.cuda.synchronize()
    ref = A @ B
    err = (logical(Ccm) - ref).abs()
    assert bool((err <= _bound(A, B, 7, 1.0, 0.0, ref * 0)).all())
    assert float(logical(Ccm)[5].abs().max()) == 0.0
    assert float(logical(Ccm)[:, 7].abs().max()) == 0.0


def test_dgemm_i8_long_k_group_split(cuda):
    """K = 20000 with entries at the top of their slice range: the deepest level holds 7 slice
    pairs x 157 K chunks, more than the 1040 chunks one int32 accumulation may take, so the kernel
    must cut it into two groups (else the int32 sums would overflow)."""
    import torch
    import cuev_b200 as cv
    m, n, k = 128, 256, 20000
    A = torch.full((m, k), 0.999999, dtype=torch.float64, device=cuda)
    B = torch.full((k, n), -0.999999, dtype=torch.float64, device=cuda)
    A[:, ::3] = 0.987654321
    Ccm = colmajor(torch.zeros(m, n, dtype=torch.float64, device=cuda))
    cv.dgemm_i8(0, 0, m, n, k, 7, 1.0, colmajor(A), m, colmajor(B), k, 0.0, Ccm, m)
    torch.cuda.synchronize()
    ref = A @ B
    rel = ((logical(Ccm) - ref).abs() / ref.abs()).max().item()
    assert rel < 1e-13, rel


def test_dgemm_i8_repeat_is_deterministic(cuda):
    import torch
    import cuev_b200 as cv
    m, n, k = 700, 900, 1100
    g = torch.Generator(device="cpu").manual_seed(5)
    A = torch.randn(m, k, generator=g, dtype=torch.float64).to(cuda)
    B = torch.randn(k, n, generator=g, dtype=torch.float64).to(cuda)
    outs = []
    for _ in range(2):
        Ccm = colmajor(torch.zeros(m, n, dtype=torch.float64, device=cuda))
        cv.dgemm_i8(0, 0, m, n, k, 7, 1.0, colmajor(A), m, colmajor(B), k, 0.0, Ccm, m)
        outs.append(Ccm)
    torch.cuda.synchronize()
    assert torch.equal(outs[0], outs[1])
