"""Stage-level parity of the CUDA kernels against the oracle, mirroring the reference's stage
tests (test/cuda/test_dbbr.cu, test_bulge.cu, test_backtransform.cu) on the same inputs."""
import numpy as np
import pytest

from oracle import cuev_oracle as O

pytestmark = pytest.mark.gpu


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _cm(X):
    """numpy logical matrix -> device tensor holding its column-major storage."""
    import torch
    return torch.from_numpy(np.asfortranarray(X).ravel(order="F").copy()).cuda()


def _np_cm(t, rows, cols, ld=None):
    ld = rows if ld is None else ld
    a = t.detach().cpu().numpy().ravel()[: ld * cols]
    return a.reshape((cols, ld)).T[:rows, :].copy()


@pytest.mark.parametrize("rows,b", [(256, 32), (512, 64), (1000, 64), (5000, 32), (9, 32),
                                    (40, 64), (20000, 64)])
def test_panel_qr_vs_oracle(cuda, rows, b):
    import torch
    import cuev_b200 as cv
    A0 = O.glibc_fill(rows * b, 12345).reshape((rows, b), order="F")
    qr, Y, tau, T = O.dbbr_panel_qr(A0)
    with cv.SolverHandle(max(rows, 2 * b), b, b) as h:
        dA = _cm(A0)
        dY = torch.zeros(rows * b, dtype=torch.float64, device=cuda)
        dtau = torch.zeros(b, dtype=torch.float64, device=cuda)
        dT = torch.zeros(b * b, dtype=torch.float64, device=cuda)
        h.dbbr_panel_qr(dA, rows, dY, rows, dtau, dT, rows, b)
        torch.cuda.synchronize()
    Rg = np.triu(_np_cm(dA, rows, b))
    Yg, Tg = _np_cm(dY, rows, b), _np_cm(dT, b, b)
    tg = dtau.cpu().numpy()
    scale = np.linalg.norm(A0)
    assert np.abs(Rg - np.triu(qr)[:, :b]).max() < 1e-12 * scale
    assert np.abs(Yg - Y).max() < 1e-11
    assert np.abs(tg - tau).max() < 1e-13
    assert np.abs(Tg - T).max() < 1e-11
    # the reference's invariants (test_dbbr.cu:223-245)
    recon = Rg - Yg @ (Tg @ (Yg.T @ Rg))
    assert np.linalg.norm(recon - A0) / scale < 1e-10


@pytest.mark.parametrize("n,b,k", [(256, 64, 256), (512, 32, 128), (777, 32, 128),
                                   (1024, 32, 256), (1100, 64, 512)])
def test_dbbr_reduce_vs_oracle(cuda, n, b, k):
    import torch
    import cuev_b200 as cv
    A0 = O.glibc_fill(n * n, 7).reshape((n, n), order="F")
    Ao, Yo, Wo, _ = O.dbbr_reduce(A0, b, k)
    with cv.SolverHandle(n, b, k) as h:
        dA = _cm(A0)
        h.dbbr_reduce(dA)
        torch.cuda.synchronize()
        Bt, ldb = h.buffer(cv.BUF_B, 2 * b, n)
        Bg = _np_cm(Bt.reshape(-1), 2 * b, n, ldb)
    Bo = O.bc_pack(Ao, b)
    scale = np.abs(Bo).max()
    assert np.abs(Bg - Bo).max() < 1e-10 * scale
    S = O.band_dense(Bg, b)
    ev_ref = np.linalg.eigvalsh(O.sym_from_lower(A0))
    ev = np.linalg.eigvalsh(S)
    assert np.abs(ev - ev_ref).max() / (ev_ref[-1] - ev_ref[0]) < 1e-9


@pytest.mark.parametrize("n,b", [(256, 64), (512, 64), (513, 32), (1024, 32), (2000, 64),
                                 (20, 32), (32, 32), (40, 64), (64, 64)])
def test_bc_chase_vs_oracle(cuda, n, b):
    """n <= b included: every sweep is then a single hop clipped at the matrix end, and each
    must wait for the previous sweep to finish."""
    import torch
    import cuev_b200 as cv
    rng = np.random.default_rng(n + b)
    G = rng.standard_normal((n, n))
    A = (G + G.T) / 2
    Bo = O.bc_pack(np.tril(np.triu(A, -b)), b)  # a band matrix packed
    do, eo, Uo, _ = O.bc_chase(Bo, b)
    with cv.SolverHandle(n, b, max(b, 256 // b * b)) as h:
        dB = _cm(Bo)
        dd = torch.zeros(n, dtype=torch.float64, device=cuda)
        de = torch.zeros(n, dtype=torch.float64, device=cuda)
        h.bc_chase(dB, dd, de)
        torch.cuda.synchronize()
        Ut, ldu = h.buffer(cv.BUF_U, n, n)
        Ug = _np_cm(Ut.reshape(-1), n, n, ldu)
    dg, eg = dd.cpu().numpy(), de.cpu().numpy()[: n - 1]
    scale = np.abs(np.linalg.eigvalsh(O.band_dense(Bo, b))).max()
    assert np.abs(dg - do).max() < 1e-10 * scale
    assert np.abs(eg - eo).max() < 1e-10 * scale
    assert np.abs(Ug - Uo).max() < 1e-8
    ev_ref = np.linalg.eigvalsh(O.band_dense(Bo, b))
    ev = np.linalg.eigvalsh(O.tridiag_dense(dg, eg))
    assert np.abs(ev - ev_ref).max() / scale < 1e-12


@pytest.mark.parametrize("n,b,k", [(256, 32, 128), (384, 32, 128), (777, 32, 128),
                                   (1024, 32, 128), (1000, 64, 512), (130, 64, 128),
                                   (777, 64, 128)])
def test_backtransform_vs_oracle(cuda, n, b, k):
    """Q_b and Q_s materialised by applying the GPU back-transform to I (the reference's
    test_backtransform.cu:162-215), checked against the oracle applied to the same reflectors
    and against the similarity invariants."""
    import torch
    import cuev_b200 as cv
    A0 = O.glibc_fill(n * n, 7).reshape((n, n), order="F")
    A = O.sym_from_lower(A0)
    with cv.SolverHandle(n, b, k) as h:
        dA = _cm(A0)
        h.dbbr_reduce(dA)
        Bt, ldb = h.buffer(cv.BUF_B, 2 * b, n)
        Bg = _np_cm(Bt.reshape(-1), 2 * b, n, ldb)
        Band = O.band_dense(Bg, b)
        dd = torch.zeros(n, dtype=torch.float64, device=cuda)
        de = torch.zeros(n, dtype=torch.float64, device=cuda)
        h.bc_chase(Bt.reshape(-1), dd, de)
        torch.cuda.synchronize()
        Ut, ldu = h.buffer(cv.BUF_U, n, n)
        Ug = _np_cm(Ut.reshape(-1), n, n, ldu)
        Yt, ldy = h.buffer(cv.BUF_Y, n, n)
        Yg = _np_cm(Yt.reshape(-1), n, n, ldy)
        Tri = O.tridiag_dense(dd.cpu().numpy(), de.cpu().numpy()[: n - 1])
        Mq = _cm(np.eye(n))
        h.bc_back(Mq, n)
        torch.cuda.synchronize()
        Qb = _np_cm(Mq, n, n)
        Ms = _cm(np.eye(n))
        h.sbr_back(Ms, n)
        torch.cuda.synchronize()
        Qs = _np_cm(Ms, n, n)
    Qb_o = O.bc_back(Ug, np.eye(n), b)
    assert np.abs(Qb - Qb_o).max() < 1e-12
    # SBR-back beside the oracle's (reference backtransform.cu:210-230 restated): the oracle's
    # band reduction of the same input, its reflectors applied panel by panel to I
    _, Yo, Wo, _ = O.dbbr_reduce(A0, b, k)
    Qs_o = O.sbr_back(Yo, Wo, np.eye(n), b)
    assert np.abs(Qs - Qs_o).max() < 1e-10, np.abs(Qs - Qs_o).max()
    rb = np.linalg.norm(Qb.T @ Band @ Qb - Tri) / np.linalg.norm(Tri)
    assert rb < 1e-9
    rs = np.linalg.norm(Qs.T @ A @ Qs - Band) / np.linalg.norm(Band)
    assert rs < 1e-9
    assert np.linalg.norm(Qs.T @ Qs - np.eye(n)) / np.sqrt(n) < 1e-12
