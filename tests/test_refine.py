"""Precision form, refinement half: cuev_dsyev_refine (Ogita-Aishima) against LAPACK dsyevd and
the oracle's restatement of the same iteration."""
import numpy as np
import pytest

from oracle import cuev_oracle as O


def _sym(n, seed):
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((n, n))
    return (G + G.T) / 2


def test_oracle_refinement_converges_from_fp32():
    """The restatement itself: FP32-rounded LAPACK eigenvectors -> FP64 accuracy in 2 steps."""
    A = _sym(300, 11)
    w, V = np.linalg.eigh(A)
    lam, X = O.refine_ogita_aishima(A, V.astype(np.float32).astype(np.float64), 2)
    m = O.metrics(A, lam, X, w)
    assert m["resid_n_norm2"] < 1e-14 and m["orth_fro"] < 1e-12
    assert m["max_dlambda_rel"] < 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("n", [257, 1024])
def test_refine_from_fp32_start(cuda, n):
    import torch
    import cuev_b200 as cv
    A = _sym(n, 100 + n)
    w_ref, V = np.linalg.eigh(A)
    X0 = V.astype(np.float32).astype(np.float64)          # FP32-accurate start (~6e-8)
    dA = torch.from_numpy(A.T.copy()).cuda()               # column-major storage (A symmetric)
    dX = torch.from_numpy(X0.T.copy()).cuda()              # column j of X -> row j of the tensor
    dw = torch.empty(n, dtype=torch.float64, device="cuda")
    info = cv.refine(dA, n, dw, dX, max_iters=2)
    assert info.iterations == 2
    X = dX.cpu().numpy().T
    lam = dw.cpu().numpy()
    m = O.metrics(A, lam, X, w_ref)
    assert m["resid_n_norm2"] <= 1e-13, m
    assert m["orth_fro"] / np.sqrt(n) <= 1e-13, m
    assert m["max_dlambda_rel"] <= 1e-12, m
    # same iteration on the CPU
    lam_o, X_o = O.refine_ogita_aishima(A, X0, 2)
    assert np.abs(lam - lam_o).max() <= 1e-12 * np.abs(w_ref).max()
    assert np.abs(X - X_o).max() <= 1e-10
    # the input matrix is not modified
    assert np.array_equal(dA.cpu().numpy().T, A)


@pytest.mark.gpu
def test_refine_early_stop_and_clusters(cuda):
    """A spectrum with a tight cluster (its pairs take the orthogonalising branch in the first
    step, when delta is large, and rotate once delta has fallen below their gaps) and a
    tolerance-driven stop: the first measurement already meets a loose tolerance."""
    import torch
    import cuev_b200 as cv
    n = 512
    rng = np.random.default_rng(5)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    lam0 = np.sort(rng.uniform(-1, 1, n))
    lam0[100:108] = 0.3 + 1e-9 * np.arange(8)              # cluster, spread 7e-9
    A = (Q * lam0) @ Q.T
    A = (A + A.T) / 2
    w_ref, V = np.linalg.eigh(A)
    X0 = V.astype(np.float32).astype(np.float64)
    dA = torch.from_numpy(A.T.copy()).cuda()
    dX = torch.from_numpy(X0.T.copy()).cuda()
    dw = torch.empty(n, dtype=torch.float64, device="cuda")
    info = cv.refine(dA, n, dw, dX, max_iters=3)
    X = dX.cpu().numpy().T
    m = O.metrics(A, dw.cpu().numpy(), X, w_ref)
    assert m["orth_fro"] / np.sqrt(n) <= 1e-13, m
    assert m["max_dlambda_rel"] <= 1e-12, m
    assert m["resid_n_norm2"] <= 1e-13, m
    # loose tolerance: stops at the first measurement (no step applied)
    dX2 = torch.from_numpy(V.T.copy()).cuda()
    info2 = cv.refine(dA, n, dw, dX2, max_iters=3, tol=1e-6)
    assert info2.iterations == 0 and info2.orth_fro < 1e-6


@pytest.mark.gpu
def test_refine_invalid_arguments(cuda):
    import torch
    import cuev_b200 as cv
    A = torch.eye(4, dtype=torch.float64, device="cuda")
    w = torch.empty(4, dtype=torch.float64, device="cuda")
    X = torch.eye(4, dtype=torch.float64, device="cuda")
    with pytest.raises(cv.CuevError):
        cv.refine(A, -1, w, X)
    info = cv.refine(A, 4, w, X, max_iters=0)
    assert info.iterations == 0
