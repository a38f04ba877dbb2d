"""Golden outputs of the reference solver itself (ynkrue/cuEV built from its sources and run on a
B200 by tests/golden/make_ref_golden.py): the oracle (CPU) and the CUDA library (GPU) must agree
with them on the same seeded inputs."""
from pathlib import Path

import numpy as np
import pytest

from oracle import cuev_oracle as O

GOLD = Path(__file__).resolve().parent / "golden"
SIZES = [256, 512, 1024]


def _load(n):
    f = GOLD / f"ref_eig_n{n}.npz"
    assert f.exists(), f"missing golden fixture {f.name}"
    return np.load(f)


def _input(n):
    G = np.random.default_rng(n).standard_normal((n, n))
    return (G + G.T) / 2


def _check_vectors(g, V):
    if "evec" in g:
        Vr = g["evec"]
        align = np.abs(np.sum(V * Vr, axis=0))
    else:
        cols = g["evec_cols"]
        align = np.abs(np.sum(V[:, cols] * g["evec_sample"], axis=0))
    assert np.abs(1.0 - align).max() < 1e-10, np.abs(1.0 - align).max()


@pytest.mark.parametrize("n", SIZES)
def test_oracle_matches_reference_outputs(n):
    """Pins the oracle to the reference's own outputs (CPU)."""
    g = _load(n)
    A = _input(n)
    w, V = O.symm_eig_solve(np.asfortranarray(A), 32, 512)
    wr = g["eval"]
    assert np.abs(w - wr).max() / np.abs(wr).max() < 1e-13
    _check_vectors(g, V)


@pytest.mark.gpu
@pytest.mark.parametrize("n", SIZES)
def test_library_matches_reference_outputs(cuda, n):
    import torch
    import cuev_b200 as cv
    g = _load(n)
    A = _input(n)
    dA = torch.from_numpy(A.ravel(order="F").copy()).to(cuda)
    w = torch.zeros(n, dtype=torch.float64, device=cuda)
    V = torch.zeros(n * n, dtype=torch.float64, device=cuda)
    cv.symm_eig_solve(dA, n, w, V)  # default blocking
    torch.cuda.synchronize()
    wr = g["eval"]
    wh = w.cpu().numpy()
    assert np.abs(wh - wr).max() / np.abs(wr).max() < 1e-13
    _check_vectors(g, V.cpu().numpy().reshape((n, n)).T)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [8192, 16384])
def test_library_matches_reference_eigenvalues_large(cuda, n):
    """Parity at the bench sizes: the reference's own eigenvalues of the same seeded matrix
    (tests/golden/ref_eval_n{n}.npz, b = 32 as the reference hard-codes) within 1e-12 relative."""
    import torch
    import cuev_b200 as cv
    f = GOLD / f"ref_eval_n{n}.npz"
    assert f.exists(), f"missing golden fixture {f.name}"
    wr = np.load(f)["eval"]
    A = _input(n)
    dA = torch.from_numpy(A.ravel(order="F").copy()).to(cuda)
    del A
    w = torch.zeros(n, dtype=torch.float64, device=cuda)
    V = torch.zeros(n * n, dtype=torch.float64, device=cuda)
    cv.symm_eig_solve(dA, n, w, V)
    torch.cuda.synchronize()
    wh = w.cpu().numpy()
    assert np.abs(wh - wr).max() / np.abs(wr).max() < 1e-12
