"""Failure paths without a GPU fault: every device-side wait of the library is bounded.  A test
hook (cuev_debug_set_wait_limit_ns) shortens the bound so that the bulge chase's hand-off waits,
BC-back's warp-pipeline waits and the panel QR's grid barrier give up on purpose; the call must
return CUEV_ERR_TIMEOUT, leave no kernel running, and the next call with the normal bound must
succeed with correct results.  Nothing here can hang: a wait that gives up returns."""
import numpy as np
import pytest

from oracle import cuev_oracle as O

pytestmark = pytest.mark.gpu
TIMEOUT = -4


def _sym(n, seed):
    G = np.random.default_rng(seed).standard_normal((n, n))
    return (G + G.T) / 2


def _solve(A):
    import torch
    import cuev_b200 as cv
    n = A.shape[0]
    dA = torch.from_numpy(A.ravel(order="F").copy()).cuda()
    w = torch.zeros(n, dtype=torch.float64, device="cuda")
    V = torch.zeros(n * n, dtype=torch.float64, device="cuda")
    cv.symm_eig_solve(dA, n, w, V)
    torch.cuda.synchronize()
    return w.cpu().numpy(), V.cpu().numpy().reshape((n, n)).T


def test_solve_waits_time_out_then_next_solve_succeeds(cuda):
    import cuev_b200 as cv
    A = _sym(2048, 31)
    try:
        cv.debug_set_wait_limit_ns(1)
        with pytest.raises(cv.CuevError) as err:
            _solve(A)
        assert err.value.status == TIMEOUT, err.value
    finally:
        cv.debug_set_wait_limit_ns(0)
    w, V = _solve(A)
    m = O.metrics(A, w, V, np.linalg.eigvalsh(A))
    assert m["max_dlambda_rel"] < 1e-12 and m["resid_n_norm2"] < 1e-13, m


@pytest.mark.parametrize("nbw", [32, 64])
def test_bc_back_pipeline_waits_time_out_then_recover(cuda, nbw):
    """Stage entries: the first stages run with the normal bound; the back-transform (BC-back's
    warp pipeline waits on shared-memory counters of its neighbour warps; at b = 64 each wait is
    decided by a vote of the warp's lanes) then runs with a 1 ns bound and must report the
    timeout; rerun with the normal bound it must be exact again."""
    import torch
    import cuev_b200 as cv
    n = 1024
    A = _sym(n, 77)
    w_ref = np.linalg.eigvalsh(A)
    with cv.SolverHandle(n, nbw=nbw, nk=256) as h:
        dA = torch.from_numpy(A.ravel(order="F").copy()).cuda()
        h.dbbr_reduce(dA)
        B, _ = h.buffer(cv.BUF_B, 2 * nbw, n)
        d = torch.zeros(n, dtype=torch.float64, device="cuda")
        e = torch.zeros(n, dtype=torch.float64, device="cuda")
        h.bc_chase(B, d, e)
        w = torch.zeros(n, dtype=torch.float64, device="cuda")
        Q = torch.zeros(n * n, dtype=torch.float64, device="cuda")
        h.tridi_dc(d, e, w, Q)
        torch.cuda.synchronize()
        Q0 = Q.clone()
        try:
            cv.debug_set_wait_limit_ns(1)
            with pytest.raises(cv.CuevError) as err:
                h.back_transform(Q)
            assert err.value.status == TIMEOUT, err.value
        finally:
            cv.debug_set_wait_limit_ns(0)
        Q.copy_(Q0)
        h.back_transform(Q)
        torch.cuda.synchronize()
        V = Q.cpu().numpy().reshape((n, n)).T
        m = O.metrics(A, w.cpu().numpy(), V, w_ref)
        assert m["resid_n_norm2"] < 1e-13 and m["orth_fro"] < 1e-11, m
