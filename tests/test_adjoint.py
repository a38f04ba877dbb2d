"""Differentiation form: the hand-written eigh adjoint (cuev_dsyev_adjoint) wrapped in a
torch.autograd.Function here in the test harness only, checked against torch.linalg.eigh's
gradient and against central finite differences of the forward solve."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _make_eigh():
    import torch
    import cuev_b200 as cv

    class CuevEigh(torch.autograd.Function):
        """w, V = eigh(A) through libcuev_b200 (forward: cuev_dsyevd, backward: the adjoint);
        A is a symmetric (n, n) float64 CUDA tensor; only w and V are saved."""

        @staticmethod
        def forward(ctx, A, gap_tol):
            n = A.shape[0]
            Acm = A.t().contiguous().clone()  # column-major storage (A is symmetric anyway)
            w = torch.empty(n, dtype=A.dtype, device=A.device)
            Vcm = torch.empty_like(Acm)
            cv.symm_eig_solve(Acm, n, w, Vcm)
            V = Vcm.t()
            ctx.save_for_backward(w, Vcm)
            ctx.gap_tol = gap_tol
            return w, V

        @staticmethod
        def backward(ctx, gw, gV):
            w, Vcm = ctx.saved_tensors
            n = w.shape[0]
            Abar = torch.empty_like(Vcm)
            gVcm = gV.t().contiguous() if gV is not None else None
            gw_ = gw.contiguous() if gw is not None else None
            st = cv.lib().cuev_dsyev_adjoint(
                Vcm.data_ptr(), w.data_ptr(), gVcm.data_ptr() if gVcm is not None else None,
                gw_.data_ptr() if gw_ is not None else None, n, float(ctx.gap_tol),
                Abar.data_ptr(), torch.cuda.current_stream().cuda_stream)
            cv._check(st, "cuev_dsyev_adjoint")
            return Abar.t(), None

    return CuevEigh.apply


def _loss(w, V, wt, Ct):
    return (wt * w).sum() + ((Ct * V) ** 2).sum()


def _sym(n, seed, dev):
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    G = torch.randn(n, n, generator=g, dtype=torch.float64)
    return ((G + G.t()) / 2).to(dev)


@pytest.mark.parametrize("n", [2, 5, 33, 64, 300, 1024, 4096])
def test_adjoint_vs_torch_eigh(cuda, n):
    """Against torch.linalg.eigh's gradient, up to n = 4096 (the differentiation config).  Both
    gradients carry each solver's eigenvector rounding divided by the smallest eigenvalue gaps
    (F_ij = 1/(lam_j - lam_i)); for A = (G + G^T)/2 the smallest gap relative to ||A|| shrinks as
    n^(-3/2), so the bound grows from 1e-10 at n <= 1024 to 1e-9 at n = 4096."""
    import torch
    eigh = _make_eigh()
    A = _sym(n, n, cuda).requires_grad_(True)
    g = torch.Generator(device="cpu").manual_seed(n + 1)
    wt = torch.randn(n, generator=g, dtype=torch.float64).to(cuda)
    Ct = torch.randn(n, n, generator=g, dtype=torch.float64).to(cuda)
    w, V = eigh(A, 0.0)
    _loss(w, V, wt, Ct).backward()
    ga = A.grad.clone()
    A2 = A.detach().clone().requires_grad_(True)
    w2, V2 = torch.linalg.eigh(A2)
    _loss(w2, V2, wt, Ct).backward()
    gt = A2.grad
    # torch returns the gradient w.r.t. the symmetric input; both are symmetric here
    rel = (ga - gt).norm() / gt.norm()
    assert rel < (1e-10 if n <= 1024 else 1e-9), rel.item()
    assert (ga - ga.t()).abs().max() < 1e-12 * ga.abs().max()


def test_adjoint_fd_with_planted_gap(cuda):
    """n = 4096 (differentiation config): central differences (h = 1e-6) along 32 random
    symmetric directions that avoid the planted near-degenerate pair (gap 1e-9), whose coupling
    term is masked (gap_tol = 1e-7) and checked separately."""
    import torch
    eigh = _make_eigh()
    n = 4096
    A0 = _sym(n, 7, cuda)
    w0, V0 = torch.linalg.eigh(A0)
    i = n // 2
    lam = w0.clone()
    lam[i + 1] = lam[i] + 1e-9  # plant the near-degenerate pair
    A = (V0 * lam) @ V0.t()
    A = (A + A.t()) / 2
    g = torch.Generator(device="cpu").manual_seed(11)
    wt = torch.randn(n, generator=g, dtype=torch.float64).to(cuda)
    Ct = torch.randn(n, n, generator=g, dtype=torch.float64).to(cuda)
    # Inside the near-degenerate pair the eigenvectors are only defined up to a rotation of
    # their 2-D span (gap 1e-9 ~ 1e-11 ||A||), so the loss must not tell the two columns apart:
    # equal weights make sum C^2 V^2 over the pair rotation invariant.
    Ct[:, i + 1] = Ct[:, i]
    Ar = A.clone().requires_grad_(True)
    w, V = eigh(Ar, 1e-7)
    _loss(w, V, wt, Ct).backward()
    grad = Ar.grad
    # masked coupling of the pair
    M = V.t() @ grad @ V
    assert abs(M[i, i + 1].item()) < 1e-12 * M.abs().max().item()
    vi, vj = V[:, i], V[:, i + 1]
    P = torch.eye(n, dtype=torch.float64, device=cuda) - torch.outer(vi, vi) - torch.outer(vj, vj)
    ans, fd2, fd4 = [], [], []
    loss = lambda X: _loss(*eigh(X, 1e-7), wt, Ct).item()  # noqa: E731
    for d in range(32):
        D = torch.randn(n, n, generator=g, dtype=torch.float64).to(cuda)
        D = P @ ((D + D.t()) / 2) @ P
        D /= D.norm()
        with torch.no_grad():
            # central difference with h = 1e-6 (the configuration's check)
            h = 1e-6
            fd2.append((loss(A + h * D) - loss(A - h * D)) / (2 * h))
            # 4-point central difference with h = 1e-4: O(h^4) truncation, lower noise
            h = 1e-4
            fp1, fm1 = loss(A + h * D), loss(A - h * D)
            fp2, fm2 = loss(A + 2 * h * D), loss(A - 2 * h * D)
            fd4.append((8 * (fp1 - fm1) - (fp2 - fm2)) / (12 * h))
        ans.append((grad * D).sum().item())
    ans, fd2, fd4 = np.array(ans), np.array(fd2), np.array(fd4)
    rel2 = np.linalg.norm(fd2 - ans) / np.linalg.norm(ans)
    rel4 = np.linalg.norm(fd4 - ans) / np.linalg.norm(ans)
    # h = 1e-6: the difference of two FP64 solves carries ~1e-11 of rounding, i.e. ~1e-5 of the
    # quotient; the 4-point stencil at h = 1e-4 resolves the gradient to 1e-6.
    assert rel2 < 1e-4, rel2
    assert rel4 < 1e-6, rel4


def test_adjoint_fp32_entry(cuda):
    import torch
    import cuev_b200 as cv
    n = 200
    A = _sym(n, 3, cuda)
    w, V = torch.linalg.eigh(A)
    g = torch.Generator(device="cpu").manual_seed(5)
    gV = torch.randn(n, n, generator=g, dtype=torch.float64).to(cuda)
    gw = torch.randn(n, generator=g, dtype=torch.float64).to(cuda)
    out64 = torch.empty(n * n, dtype=torch.float64, device=cuda)
    out32 = torch.empty(n * n, dtype=torch.float32, device=cuda)
    Vcm, gVcm = V.t().contiguous(), gV.t().contiguous()
    L = cv.lib()
    s = torch.cuda.current_stream().cuda_stream
    assert L.cuev_dsyev_adjoint(Vcm.data_ptr(), w.data_ptr(), gVcm.data_ptr(), gw.data_ptr(), n,
                                0.0, out64.data_ptr(), s) == 0
    V32, gV32, w32, gw32 = (x.float().contiguous() for x in (Vcm, gVcm, w, gw))
    assert L.cuev_ssyev_adjoint(V32.data_ptr(), w32.data_ptr(), gV32.data_ptr(),
                                gw32.data_ptr(), n, 0.0, out32.data_ptr(), s) == 0
    torch.cuda.synchronize()
    rel = (out32.double() - out64).norm() / out64.norm()
    assert rel < 1e-3, rel.item()  # FP32 inputs: lambda rounding against gaps ~5e-3
