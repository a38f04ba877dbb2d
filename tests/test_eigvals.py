"""Eigenvalues-only path: the bisection stage (cuev_tridi_eigvals) against LAPACK's tridiagonal
eigenvalues, and the eigenvalues-only solve (evec = NULL) against the full solve and dsyevd."""
import numpy as np
import pytest
import scipy.linalg as sla

from oracle import cuev_oracle as O


def _tridiagonals():
    rng = np.random.default_rng(17)
    out = []
    for n in (1, 2, 3, 100, 1000, 5000):
        out.append((f"random{n}", rng.standard_normal(n), rng.standard_normal(max(n - 1, 0))))
    n = 400
    out.append(("graded", 10.0 ** -np.linspace(0, 12, n), 10.0 ** -np.linspace(0, 12, n - 1) * 0.5))
    out.append(("diagonal", np.repeat([1.0, -2.0, 3.5, 0.0], 100), np.zeros(399)))
    # glued Wilkinson W21+ blocks: pairs of nearly equal eigenvalues
    w = np.abs(np.arange(-10, 11, dtype=float))
    d = np.concatenate([w] * 20)
    e = np.concatenate([np.concatenate([np.ones(20), [1e-14]]) for _ in range(20)])[:-1]
    out.append(("glued_wilkinson", d, e))
    out.append(("scaled_1e150", 1e150 * rng.standard_normal(300), 1e150 * rng.standard_normal(299)))
    return out


def test_sturm_quotient_method():
    """The straight-line quotient of the bisection kernel (tridi_eigvals.cu: sturm_quot) restated
    with exact rounding: a float reciprocal seed off by up to one float ulp (rcp.approx.f32's
    bound), two Newton steps and Markstein's residual correction land within one rounding of f / q
    over the pivot range 2^-100 <= |q| <= 2^101 that the kernel's pivot floor guarantees."""
    from fractions import Fraction as F

    def fma(a, b, c):
        return float(F(a) * F(b) + F(c))

    rng = np.random.default_rng(11)
    q_all = rng.uniform(1.0, 2.0, 3000) * 2.0 ** rng.integers(-100, 101, 3000)
    q_all *= np.where(rng.random(3000) < 0.5, -1.0, 1.0)
    f_all = rng.random(3000)
    f_all[:50] = 0.0
    f_all[50:100] = 1e-310  # subnormal e^2
    for q, f in zip(q_all.tolist(), f_all.tolist()):
        q32 = np.float32(q)
        r32 = np.float32(1.0) / q32
        exact = F(f) / F(q)
        for seed in (r32, np.nextafter(r32, np.float32(np.inf)), np.nextafter(r32, np.float32(-np.inf))):
            r = float(seed)
            r = fma(r, fma(-q, r, 1.0), r)
            r = fma(r, fma(-q, r, 1.0), r)
            y = float(F(f) * F(r))
            y = fma(r, fma(-q, y, f), y)
            ulp = float(np.spacing(abs(float(exact)))) if exact != 0 else 0.0
            assert abs(F(y) - exact) <= F(ulp), (q, f, y, float(exact))


def test_oracle_matches_dense():
    rng = np.random.default_rng(3)
    d, e = rng.standard_normal(50), rng.standard_normal(49)
    T = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
    assert np.abs(O.tridi_eigvals(d, e) - np.linalg.eigvalsh(T)).max() < 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("case", _tridiagonals(), ids=lambda c: c[0])
def test_tridi_eigvals_stage(cuda, case):
    import torch
    import cuev_b200 as cv
    name, d, e = case
    n = d.size
    ref = O.tridi_eigvals(d, e)
    with cv.SolverHandle(n, 32, 256) as h:
        dd = torch.from_numpy(d.copy()).to(cuda)
        de = torch.from_numpy(np.concatenate([e, [0.0]])).to(cuda)
        w = torch.empty(n, dtype=torch.float64, device=cuda)
        h.tridi_eigvals(dd, de, w)
        torch.cuda.synchronize()
    got = w.cpu().numpy()
    tnorm = max(np.abs(d).max(), np.abs(e).max() if e.size else 0.0, 1e-300)
    assert np.all(np.diff(got) >= 0), name
    assert np.abs(got - ref).max() <= 1e-13 * tnorm, (name, np.abs(got - ref).max() / tnorm)


@pytest.mark.gpu
@pytest.mark.parametrize("n,nbw", [(1, 32), (2, 32), (3, 32), (20, 32), (257, 32), (2048, 32),
                                   (40, 64), (300, 64), (1024, 64)])
def test_eigvals_only_solve(cuda, n, nbw):
    import torch
    import cuev_b200 as cv
    rng = np.random.default_rng(n)
    G = rng.standard_normal((n, n))
    A = (G + G.T) / 2
    ref = sla.eigh(A, eigvals_only=True, driver="evd")
    dA = torch.from_numpy(A.ravel(order="F").copy()).to(cuda)
    w = torch.zeros(n, dtype=torch.float64, device=cuda)
    t = cv.Timer()
    cv.symm_eig_solve(dA, n, w, None, timer=t, nbw=nbw, nk=256)
    torch.cuda.synchronize()
    got = w.cpu().numpy()
    anorm = np.abs(ref).max()
    assert np.abs(got - ref).max() <= 1e-12 * anorm
    if n > 1:
        assert t.bt_ms == 0.0
        # same eigenvalues as the full solve (which runs D&C)
        dA2 = torch.from_numpy(A.ravel(order="F").copy()).to(cuda)
        w2 = torch.zeros(n, dtype=torch.float64, device=cuda)
        V2 = torch.zeros(n * n, dtype=torch.float64, device=cuda)
        cv.symm_eig_solve(dA2, n, w2, V2, nbw=nbw, nk=256)
        assert np.abs(got - w2.cpu().numpy()).max() <= 1e-12 * anorm


@pytest.mark.gpu
def test_eigvals_only_clustered_and_fp32(cuda):
    import torch
    import cuev_b200 as cv
    n = 2048
    rng = np.random.default_rng(9)
    centres = 10.0 ** rng.uniform(-6, 0, 32)
    cl = np.concatenate([c * (1 + 1e-10 * rng.uniform(-1, 1, n // 64)) for c in centres])
    lam = rng.permutation(np.concatenate([cl, 10.0 ** rng.uniform(-6, 0, n - cl.size)]))
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    A = (Q * lam) @ Q.T
    A = (A + A.T) / 2
    w = cv.eigvalsh(torch.from_numpy(A).to(cuda))
    assert np.abs(w.cpu().numpy() - np.sort(lam)).max() <= 1e-12
    A32 = torch.from_numpy(A.astype(np.float32).ravel(order="F").copy()).to(cuda)
    w32 = torch.zeros(n, dtype=torch.float32, device=cuda)
    cv.symm_eig_solve(A32, n, w32, None)
    ref32 = np.linalg.eigvalsh(A.astype(np.float32).astype(np.float64))
    assert np.abs(w32.cpu().numpy() - ref32).max() <= 1e-6
