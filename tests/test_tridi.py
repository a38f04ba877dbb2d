"""GPU tridiagonal divide and conquer against the oracle (the reference's host D&C over LAPACK,
src/cuda/tridi.cu) and the reference's tridi tests (test/cuda/test_tridi.cu)."""
import numpy as np
import pytest

from oracle import cuev_oracle as O

pytestmark = pytest.mark.gpu


def _run_dc(cuda, d, e, b=32):
    import torch
    import cuev_b200 as cv
    n = len(d)
    ee = np.zeros(max(n, 1))
    ee[: n - 1] = e[: n - 1]
    with cv.SolverHandle(max(n, 1), b, 256) as h:
        dd = torch.from_numpy(np.ascontiguousarray(d, dtype=np.float64)).to(cuda)
        de = torch.from_numpy(ee).to(cuda)
        w = torch.zeros(n, dtype=torch.float64, device=cuda)
        V = torch.zeros(n * n, dtype=torch.float64, device=cuda)
        h.tridi_dc(dd, de, w, V)
        torch.cuda.synchronize()
    return w.cpu().numpy(), V.cpu().numpy().reshape((n, n)).T.copy()


def _check(d, e, w, V, tol_res, tol_orth):
    n = len(d)
    T = O.tridiag_dense(d, e[: n - 1])
    tn = max(np.linalg.norm(T), 1e-300)
    assert np.all(np.diff(w) >= 0), "eigenvalues not ascending"
    assert np.linalg.norm(T @ V - V * w) / tn < tol_res
    assert np.linalg.norm(V.T @ V - np.eye(n)) / np.sqrt(n) < tol_orth
    ref = np.linalg.eigvalsh(T)
    scale = max(np.abs(ref).max(), 1e-300)
    assert np.abs(w - ref).max() / scale < 1e-12


@pytest.mark.parametrize("n,tol", [(48, 1e-10), (100, 1e-10), (500, 1e-9)])
def test_reference_cases(cuda, n, tol):
    """test/cuda/test_tridi.cu:76-84 inputs (fill_random seeds 11 and 23) and tolerances."""
    d = O.glibc_fill(n, 11)
    e = O.glibc_fill(n - 1, 23)
    w, V = _run_dc(cuda, d, e)
    _check(d, e, w, V, tol, tol)
    wo, Vo = O.tridi_dc(d, e)
    assert np.abs(w - wo).max() < 1e-13 * np.abs(wo).max()


@pytest.mark.parametrize("n", [1, 2, 3, 63, 64, 65, 129, 1000, 2049, 4096])
def test_random(cuda, n):
    rng = np.random.default_rng(100 + n)
    d = rng.standard_normal(n)
    e = rng.standard_normal(max(n - 1, 0))
    w, V = _run_dc(cuda, d, e)
    _check(d, e, w, V, 1e-13, 1e-13)


@pytest.mark.parametrize("kind", ["diag", "zero", "wilkinson", "clusters", "tiny_e", "graded",
                                  "ones", "glued"])
def test_deflation_heavy(cuda, kind):
    n = 700
    rng = np.random.default_rng(7)
    if kind == "diag":
        d, e = rng.standard_normal(n), np.zeros(n - 1)
    elif kind == "zero":
        d, e = np.zeros(n), np.zeros(n - 1)
    elif kind == "wilkinson":
        m = (n - 1) // 2
        d = np.abs(np.arange(-m, n - m, dtype=np.float64))
        e = np.ones(n - 1)
    elif kind == "clusters":
        d = np.repeat(rng.standard_normal(n // 50), 50)[:n] + 1e-12 * rng.standard_normal(n)
        e = 1e-9 * rng.standard_normal(n - 1)
    elif kind == "tiny_e":
        d = rng.standard_normal(n)
        e = rng.standard_normal(n - 1)
        e[::7] = 1e-300
    elif kind == "graded":
        d = 10.0 ** (-np.arange(n) / 50.0)
        e = 0.1 * 10.0 ** (-np.arange(n - 1) / 50.0)
    elif kind == "ones":
        d, e = np.full(n, 2.0), np.ones(n - 1)
    else:  # glued Wilkinson blocks W21+ with glue 1e-10
        blk = np.abs(np.arange(-10, 11, dtype=np.float64))
        reps = n // 21 + 1
        d = np.tile(blk, reps)[:n]
        e = np.tile(np.r_[np.ones(20), 1e-10], reps)[: n - 1]
    w, V = _run_dc(cuda, d, e)
    T = O.tridiag_dense(d, e)
    tn = max(np.linalg.norm(T), 1e-300)
    assert np.all(np.diff(w) >= 0)
    assert np.linalg.norm(T @ V - V * w) / tn < 1e-13 or np.linalg.norm(T) == 0
    assert np.linalg.norm(V.T @ V - np.eye(n)) / np.sqrt(n) < 1e-13
    ref = np.linalg.eigvalsh(T)
    assert np.abs(w - ref).max() <= 1e-12 * max(np.abs(ref).max(), 1e-300) + 1e-300
