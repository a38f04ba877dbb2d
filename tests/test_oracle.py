"""Pin the oracle (CPU restatement of the reference) before trusting it.

Each case is one of the reference's own tests (test/cuda/test_*.cu) run on the oracle with the
same inputs (the C library's rand() stream behind fill_random, test/cuda/test.h:74-78) and the
same tolerances, plus a full-solve comparison with LAPACK dsyevd.  CPU only."""
import numpy as np
import pytest
import scipy.linalg as sla

from oracle import cuev_oracle as O


def _rel_spec(A_sym, S_sym):
    ev_ref = np.linalg.eigvalsh(A_sym)
    ev = np.linalg.eigvalsh(S_sym)
    return np.abs(ev - ev_ref).max() / (ev_ref[-1] - ev_ref[0])


@pytest.mark.parametrize("rows,b,tol", [(256, 32, 1e-10), (512, 64, 1e-10)])
def test_panel_qr_reference_cases(rows, b, tol):
    """test/cuda/test_dbbr.cu:196-251 (dbbr_panel_qr.fp64_square / fp64_wide)."""
    A0 = O.glibc_fill(rows * b, 12345).reshape((rows, b), order="F")
    qr, Y, tau, T = O.dbbr_panel_qr(A0)
    R = np.triu(qr)[:, :b]
    recon = R - Y @ (T @ (Y.T @ R))
    assert np.linalg.norm(recon - A0) / np.linalg.norm(A0) < tol
    Q = np.eye(rows) - Y @ T @ Y.T
    assert np.linalg.norm(Q.T @ Q - np.eye(rows)) / np.sqrt(rows) < tol


@pytest.mark.parametrize("n,b,k", [(256, 64, 256), (512, 32, 128)])
def test_dbbr_reduce_reference_cases(n, b, k):
    """test/cuda/test_dbbr.cu:255-298 (dbbr_reduce.fp64_oneblock / fp64_multiblock)."""
    A0 = O.glibc_fill(n * n, 7).reshape((n, n), order="F")
    A, Y, W, _ = O.dbbr_reduce(A0, b, k)
    band = np.tril(np.triu(A, -b))  # lower band incl. diagonal
    S = band + np.tril(band, -1).T
    assert _rel_spec(O.sym_from_lower(A0), S) < 1e-9


@pytest.mark.parametrize("n,b,k", [(256, 64, 256), (512, 64, 256)])
def test_bc_chase_reference_cases(n, b, k):
    """test/cuda/test_bulge.cu:365-409 (bc_chase.fp64_oneblock / fp64_multiblock)."""
    A0 = O.glibc_fill(n * n, 7).reshape((n, n), order="F")
    A, Y, W, _ = O.dbbr_reduce(A0, b, k)
    d, e, U, _ = O.bc_chase(O.bc_pack(A, b), b)
    assert _rel_spec(O.sym_from_lower(A0), O.tridiag_dense(d, e)) < 1e-9


@pytest.mark.parametrize("n,tol", [(48, 1e-10), (100, 1e-10), (500, 1e-9)])
def test_tridi_dc_reference_cases(n, tol):
    """test/cuda/test_tridi.cu:22-84 (tridi_dc.fp64_leaf / onemerge / multilevel)."""
    d = O.glibc_fill(n, 11)
    e = O.glibc_fill(n - 1, 23)
    w, V = O.tridi_dc(d, e)
    T = O.tridiag_dense(d, e)
    assert np.linalg.norm(T @ V - V * w) / np.linalg.norm(T) < tol
    assert np.linalg.norm(V.T @ V - np.eye(n)) / np.sqrt(n) < tol
    assert np.all(np.diff(w) >= 0)
    np.testing.assert_allclose(w, np.linalg.eigvalsh(T), atol=1e-12 * np.abs(w).max())


@pytest.mark.parametrize("n", [256, 384, 777])
def test_backtransform_reference_cases(n):
    """test/cuda/test_backtransform.cu:176-233: Q_s^T A Q_s = Band, Q_b^T Band Q_b = Tri."""
    b, k = 32, 128
    A0 = O.glibc_fill(n * n, 7).reshape((n, n), order="F")
    A = O.sym_from_lower(A0)
    Ab, Y, W, _ = O.dbbr_reduce(A0, b, k)
    B = O.bc_pack(Ab, b)
    Band = O.band_dense(B, b)
    d, e, U, _ = O.bc_chase(B, b)
    Tri = O.tridiag_dense(d, e)
    Qs = O.sbr_back(Y, W, np.eye(n), b)
    Qb = O.bc_back(U, np.eye(n), b)
    rs = np.linalg.norm(Qs.T @ A @ Qs - Band) / np.linalg.norm(Band)
    rb = np.linalg.norm(Qb.T @ Band @ Qb - Tri) / np.linalg.norm(Tri)
    assert rs < 1e-9 and rb < 1e-9


@pytest.mark.parametrize("n,b,k", [(3, 32, 256), (65, 32, 256), (300, 32, 256), (777, 32, 128),
                                   (1024, 32, 256), (513, 64, 512)])
def test_full_solve_vs_dsyevd(n, b, k):
    rng = np.random.default_rng(n)
    G = rng.standard_normal((n, n))
    A = (G + G.T) / 2
    w, V = O.symm_eig_solve(np.asfortranarray(A), b, k)
    w_ref = sla.eigh(A, eigvals_only=True, driver="evd")
    m = O.metrics(A, w, V, w_ref)
    assert m["max_dlambda_rel"] < 1e-12
    assert m["resid_n_norm2"] < 1e-13
    assert m["orth_fro"] < 1e-11 * np.sqrt(n)


def test_dlaed4_known_answer():
    """Secular-equation roots of diag(d) + rho z z^T from LAPACK dlaed4 (the routine the
    reference calls per root, src/cuda/tridi.cu:137-143) against a dense eigensolver."""
    rng = np.random.default_rng(5)
    k = 40
    d = np.sort(rng.standard_normal(k))
    z = rng.standard_normal(k)
    z /= np.linalg.norm(z)
    rho = 0.7
    lam = np.empty(k)
    delta = np.zeros(k * k)
    for j in range(k):
        lam[j], info = O.lap_laed4(k, j + 1, d, z, delta, j * k, rho)
        assert info == 0
    ref = np.linalg.eigvalsh(np.diag(d) + rho * np.outer(z, z))
    np.testing.assert_allclose(lam, ref, rtol=0, atol=1e-14)
    # interlacing: d_j < lambda_j < d_{j+1}
    assert np.all(lam[:-1] > d[:-1]) and np.all(lam[:-1] < d[1:])
