"""Precision form: cuev_dsyevd_mixed (FP32-level int8 tensor-core first solve + Ogita-Aishima
refinement with FP64-level int8 tensor-core products) and cuev_dsyev_refine_ex against LAPACK
dsyevd and the reference solver's own outputs.

Bounds (the FP64 form's): eigenvalues within 1e-12 ||A||_2, residual ||AV - V diag(w)||_F /
(n ||A||_2) <= 1e-13.  Orthogonality is stated: the int8 products measure X^T X to about
2^-49 rowmax colmax sqrt(n) per entry, so ||V^T V - I||_F / sqrt(n) is held to 1e-12 (the FP64
form's test uses 1e-13)."""
from pathlib import Path

import numpy as np
import pytest

from oracle import cuev_oracle as O

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


def _sym(n, seed):
    G = np.random.default_rng(seed).standard_normal((n, n))
    return (G + G.T) / 2


def _solve_mixed(A, iters=2, tol=0.0):
    import torch
    import cuev_b200 as cv
    n = A.shape[0]
    dA = torch.from_numpy(A.ravel(order="F").copy()).cuda()
    w = torch.zeros(n, dtype=torch.float64, device="cuda")
    V = torch.zeros(n * n, dtype=torch.float64, device="cuda")
    info = cv.symm_eig_solve_mixed(dA, n, w, V, max_refine_iters=iters, tol=tol)
    torch.cuda.synchronize()
    return w.cpu().numpy(), V.cpu().numpy().reshape((n, n)).T, info


@pytest.mark.parametrize("n", [257, 1024])
def test_refine_int8_products_from_fp32_start(cuda, n):
    import torch
    import cuev_b200 as cv
    A = _sym(n, 100 + n)
    w_ref, V = np.linalg.eigh(A)
    X0 = V.astype(np.float32).astype(np.float64)
    dA = torch.from_numpy(A.T.copy()).cuda()
    dX = torch.from_numpy(X0.T.copy()).cuda()
    dw = torch.empty(n, dtype=torch.float64, device="cuda")
    info = cv.refine(dA, n, dw, dX, max_iters=2, products=cv.PRODUCTS_INT8)
    assert info.iterations == 2
    m = O.metrics(A, dw.cpu().numpy(), dX.cpu().numpy().T, w_ref)
    assert m["resid_n_norm2"] <= 1e-13, m
    assert m["max_dlambda_rel"] <= 1e-12, m
    assert m["orth_fro"] / np.sqrt(n) <= 1e-12, m
    # same iteration on the CPU (the oracle's FP64 restatement)
    lam_o, X_o = O.refine_ogita_aishima(A, X0, 2)
    assert np.abs(dw.cpu().numpy() - lam_o).max() <= 1e-12 * np.abs(w_ref).max()
    assert np.abs(dX.cpu().numpy().T - X_o).max() <= 1e-9
    assert np.array_equal(dA.cpu().numpy().T, A)   # A is not modified


@pytest.mark.parametrize("n", [2, 20, 100, 1024, 4096])
def test_mixed_solve_vs_lapack(cuda, n):
    A = _sym(n, 7 * n)
    w_ref = np.linalg.eigvalsh(A)
    w, V, info = _solve_mixed(A, iters=2)
    m = O.metrics(A, w, V, w_ref)
    assert info.refine_iterations == 2
    assert m["max_dlambda_rel"] <= 1e-12, m
    assert m["resid_n_norm2"] <= 1e-13, m
    assert m["orth_fro"] / np.sqrt(n) <= 1e-12, m
    assert info.first_ms > 0 and info.refine_ms > 0


def test_mixed_first_part_is_low_precision_and_refinement_recovers(cuda):
    """n = 4096: the large back-transform GEMMs run on FP32-level int8 products, so before any
    refinement step the orthogonality is far from FP64's; one or two steps restore it."""
    n = 4096
    A = _sym(n, 4242)
    w_ref = np.linalg.eigvalsh(A)
    w0, V0, _ = _solve_mixed(A, iters=0)
    m0 = O.metrics(A, w0, V0, w_ref)
    assert m0["orth_fro"] > 1e-10, m0          # FP64 form: ~1e-13 at this size
    w2, V2, info = _solve_mixed(A, iters=2)
    m2 = O.metrics(A, w2, V2, w_ref)
    assert m2["orth_fro"] < m0["orth_fro"] * 1e-3, (m0, m2)
    assert m2["resid_n_norm2"] <= 1e-13 and m2["max_dlambda_rel"] <= 1e-12, m2


def test_mixed_tolerance_stop(cuda):
    A = _sym(600, 3)
    _, _, info = _solve_mixed(A, iters=5, tol=1e-10)
    assert 0 <= info.refine_iterations < 5
    assert info.orth_fro <= 1e-10


def test_mixed_matches_reference_outputs(cuda):
    """Eigenvalues and eigenvectors against the reference solver's own outputs at n = 1024
    (tests/golden, made by running the reference built from its sources)."""
    g = np.load(GOLD / "ref_eig_n1024.npz")
    n = 1024
    G = np.random.default_rng(n).standard_normal((n, n))
    A = (G + G.T) / 2
    w, V, _ = _solve_mixed(A, iters=2)
    wr = g["eval"]
    assert np.abs(w - wr).max() / np.abs(wr).max() < 1e-12
    if "evec" in g:
        align = np.abs(np.sum(V * g["evec"], axis=0))
    else:
        align = np.abs(np.sum(V[:, g["evec_cols"]] * g["evec_sample"], axis=0))
    assert np.abs(1.0 - align).max() < 1e-9


def test_mixed_invalid_arguments(cuda):
    import torch
    import cuev_b200 as cv
    A = torch.eye(4, dtype=torch.float64, device="cuda")
    w = torch.empty(4, dtype=torch.float64, device="cuda")
    V = torch.empty(16, dtype=torch.float64, device="cuda")
    with pytest.raises(cv.CuevError):
        cv.symm_eig_solve_mixed(A, 4, w, V, max_refine_iters=-1)
    with pytest.raises(cv.CuevError):
        cv.symm_eig_solve_mixed(A, -3, w, V)
