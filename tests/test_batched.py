"""Batched small-n eigensolver (cuev_dsyevd_batched, one CTA per matrix: Jacobi for n <= 64,
Householder + implicit QL for 64 < n <= 512) against LAPACK per matrix."""
import numpy as np
import pytest

from oracle import cuev_oracle as O


def _check(A, w, V, tol=1e-13):
    wr, _ = O.eigh_batched(A)
    L = np.tril(A)
    S = L + np.swapaxes(L, 1, 2) - np.einsum("bii->bi", L)[:, :, None] * np.eye(A.shape[1])
    n = A.shape[1]
    anorm = np.maximum(np.abs(wr).max(axis=1), 1e-300)
    assert (np.abs(w - wr).max(axis=1) <= tol * anorm).all()
    R = S @ V - V * w[:, None, :]
    assert (np.linalg.norm(R, axis=(1, 2)) <= tol * n * anorm).all()
    O_ = np.swapaxes(V, 1, 2) @ V - np.eye(n)
    assert (np.linalg.norm(O_, axis=(1, 2)) <= tol * n).all()
    assert (np.diff(w, axis=1) >= 0).all()


def test_oracle_batched_symmetrises_lower():
    rng = np.random.default_rng(0)
    A = rng.standard_normal((3, 5, 5))          # not symmetric: only the lower triangle counts
    w, V = O.eigh_batched(A)
    S = np.tril(A[1]) + np.tril(A[1], -1).T
    assert np.abs(w[1] - np.linalg.eigvalsh(S)).max() < 1e-14


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 9, 16, 17, 31, 32, 33, 64])
def test_batched_random(cuda, n):
    import torch
    import cuev_b200 as cv
    rng = np.random.default_rng(100 + n)
    A = rng.standard_normal((97, n, n))          # lower triangles define the matrices
    w, V = cv.eigh_batched(torch.from_numpy(A).to(cuda))
    _check(A, w.cpu().numpy(), V.cpu().numpy())


@pytest.mark.gpu
def test_batched_degenerate_and_scaled(cuda):
    import torch
    import cuev_b200 as cv
    n = 24
    rng = np.random.default_rng(7)
    mats = [np.eye(n), np.zeros((n, n)), 1e200 * np.eye(n)]
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    lam = np.repeat([1.0, -2.0, 3.0], 8)
    mats.append((Q * lam) @ Q.T)                  # triple eigenvalues
    G = rng.standard_normal((n, n))
    mats.append(1e-150 * (G + G.T))               # tiny entries
    mats.append(1e150 * (G + G.T))                # huge entries
    A = np.stack(mats)
    w, V = cv.eigh_batched(torch.from_numpy(A).to(cuda))
    _check(A, w.cpu().numpy(), V.cpu().numpy(), tol=1e-13)


@pytest.mark.gpu
@pytest.mark.parametrize("n,batch", [(65, 300), (100, 40), (128, 33), (257, 12), (512, 6)])
def test_batched_mid_random(cuda, n, batch):
    # batch 300 > the SM count: CTAs loop over several matrices (workspace reuse)
    import torch
    import cuev_b200 as cv
    rng = np.random.default_rng(200 + n)
    A = rng.standard_normal((batch, n, n))
    A[1::3] *= 1e-3
    w, V = cv.eigh_batched(torch.from_numpy(A).to(cuda))
    _check(A, w.cpu().numpy(), V.cpu().numpy())


@pytest.mark.gpu
def test_batched_mid_degenerate_and_scaled(cuda):
    import torch
    import cuev_b200 as cv
    n = 96
    rng = np.random.default_rng(8)
    mats = [np.eye(n), np.zeros((n, n)), 1e200 * np.eye(n), np.diag(np.arange(n, 0, -1.0))]
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    lam = np.repeat([1.0, -2.0, 3.0], 32)
    mats.append((Q * lam) @ Q.T)                  # eigenvalues of multiplicity 32
    G = rng.standard_normal((n, n))
    mats.append(1e-150 * (G + G.T))               # tiny entries (squares below the normal range)
    mats.append(1e160 * (G + G.T))                # huge entries (squares overflow unscaled)
    T = np.diag(np.full(n - 1, 1.0), -1) + np.diag(np.full(n - 1, 1.0), 1)
    mats.append(T)                                # already tridiagonal, zero diagonal
    A = np.stack(mats)
    w, V = cv.eigh_batched(torch.from_numpy(A).to(cuda))
    _check(A, w.cpu().numpy(), V.cpu().numpy(), tol=1e-13)


@pytest.mark.gpu
def test_batched_mid_nonfinite(cuda):
    import torch
    import cuev_b200 as cv
    A = np.stack([np.eye(80), np.eye(80)])
    A[1, 40, 3] = np.nan
    with pytest.raises(cv.CuevError, match="NaN or Inf in matrix 1"):
        cv.eigh_batched(torch.from_numpy(A).to(cuda))
    w, V = cv.eigh_batched(torch.from_numpy(A[:1]).to(cuda))   # usable afterwards
    assert np.allclose(w.cpu().numpy(), 1.0)


@pytest.mark.gpu
def test_batched_errors(cuda):
    import torch
    import cuev_b200 as cv
    with pytest.raises(cv.CuevError):
        cv.eigh_batched(torch.zeros(2, 513, 513, dtype=torch.float64, device=cuda))
    w, V = cv.eigh_batched(torch.zeros(0, 8, 8, dtype=torch.float64, device=cuda))
    assert w.shape == (0, 8)
