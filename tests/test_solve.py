"""Full solve through the C ABI (the drop-in for cuev::symm_eig_solve<T>) against host LAPACK
dsyevd and against the oracle (the reference pipeline restated on the CPU)."""
import ctypes as C

import numpy as np
import pytest
import scipy.linalg as sla

from oracle import cuev_oracle as O

pytestmark = pytest.mark.gpu


def _solve(cuda, A, nbw=0, nk=0, timer=None):
    import torch
    import cuev_b200 as cv
    n = A.shape[0]
    dA = torch.from_numpy(np.asfortranarray(A).ravel(order="F").copy()).to(cuda)
    w = torch.zeros(n, dtype=torch.float64, device=cuda)
    V = torch.zeros(n * n, dtype=torch.float64, device=cuda)
    cv.symm_eig_solve(dA, n, w, V, timer=timer, nbw=nbw, nk=nk)
    torch.cuda.synchronize()
    return w.cpu().numpy(), V.cpu().numpy().reshape((n, n)).T.copy()


def _sym(n, seed):
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((n, n))
    return (G + G.T) / 2


@pytest.mark.parametrize("n,nbw,nk", [(2, 32, 256), (3, 32, 256), (33, 32, 256), (65, 32, 256),
                                      (100, 32, 256), (257, 32, 128), (777, 32, 128),
                                      (1024, 32, 256), (1024, 64, 512), (1500, 64, 256),
                                      (2, 64, 128), (3, 64, 128), (40, 64, 128), (65, 64, 128),
                                      (100, 64, 128), (130, 64, 128), (20, 32, 128),
                                      (31, 32, 128), (32, 32, 128), (63, 64, 128), (64, 64, 128),
                                      (64, 32, 128), (96, 32, 128), (128, 64, 128),
                                      (300, 32, 32), (300, 64, 64), (2048, 0, 0)])
def test_solve_vs_dsyevd(cuda, n, nbw, nk):
    A = _sym(n, n + nbw)
    w, V = _solve(cuda, A, nbw, nk)
    w_ref = sla.eigh(A, eigvals_only=True, driver="evd")
    m = O.metrics(A, w, V, w_ref)
    assert m["max_dlambda_rel"] < 1e-12, m
    assert m["resid_n_norm2"] < 1e-13, m
    assert m["orth_fro"] / np.sqrt(n) < 1e-13, m


def test_config1_n1024_vs_oracle(cuda):
    """Config C1: n = 1024, b = 32, k = 256, A = (G + G^T)/2 from a seeded N(0,1) G; compared
    with the oracle (reference pipeline) on the same input: eigenvalues and eigenvectors (up to
    sign, all eigenvalues of this matrix are simple)."""
    n = 1024
    A = _sym(n, 1)
    w, V = _solve(cuda, A, 32, 256)
    wo, Vo = O.symm_eig_solve(np.asfortranarray(A), 32, 256)
    assert np.abs(w - wo).max() / np.abs(wo).max() < 1e-13
    align = np.abs(np.sum(V * Vo, axis=0))
    assert np.abs(1 - align).max() < 1e-10


def test_clustered_spectrum(cuda):
    """Scaled-down config C2: half the spectrum in tight clusters (spread 1e-10), half
    log-uniform on [1e-6, 1]; exercises D&C deflation."""
    n = 2048
    rng = np.random.default_rng(2)
    ncl = 32
    centers = 10.0 ** rng.uniform(-6, 0, ncl)
    cl = np.concatenate([c * (1 + 1e-10 * rng.uniform(-1, 1, n // 2 // ncl)) for c in centers])
    rest = 10.0 ** rng.uniform(-6, 0, n - cl.size)
    lam = rng.permutation(np.concatenate([cl, rest]))
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    A = (Q * lam) @ Q.T
    A = (A + A.T) / 2
    w, V = _solve(cuda, A, 64, 512)
    w_ref = sla.eigh(A, eigvals_only=True, driver="evd")
    m = O.metrics(A, w, V, w_ref)
    assert m["max_dlambda_rel"] < 1e-12, m
    assert m["resid_n_norm2"] < 1e-13, m
    assert m["orth_fro"] / np.sqrt(n) < 1e-13, m


@pytest.mark.parametrize("nbw", [64, 32])
def test_config2_full_size(cuda, nbw):
    """Config C2 at full size: n = 8192, A = Q diag(lam) Q^T with Q from the QR of a seeded
    Gaussian, half of lam in 64 clusters of 64 (members centre * (1 + 1e-10 U(-1, 1)), centres
    log-uniform on [1e-6, 1]) and half log-uniform on [1e-6, 1]; k = 512.  The exact spectrum is
    known, so the eigenvalues are checked against it (the matrix is formed on the GPU in FP64)."""
    import torch
    import cuev_b200 as cv
    n = 8192
    rng = np.random.default_rng(8192)
    centres = 10.0 ** rng.uniform(-6, 0, 64)
    cl = np.concatenate([c * (1 + 1e-10 * rng.uniform(-1, 1, 64)) for c in centres])
    rest = 10.0 ** rng.uniform(-6, 0, n - cl.size)
    lam = rng.permutation(np.concatenate([cl, rest]))
    G = torch.from_numpy(rng.standard_normal((n, n))).to(cuda)
    Q, _ = torch.linalg.qr(G)
    del G
    lt = torch.from_numpy(lam).to(cuda)
    A = (Q * lt[None, :]) @ Q.t()
    A = (A + A.t()) * 0.5                        # symmetric: row- and column-major storage agree
    del Q
    A0 = A.clone()
    w = torch.zeros(n, dtype=torch.float64, device=cuda)
    V = torch.zeros(n, n, dtype=torch.float64, device=cuda)
    cv.symm_eig_solve(A, n, w, V, nbw=nbw, nk=512)
    torch.cuda.synchronize()
    anorm = float(np.abs(lam).max())
    dl = float((w.cpu() - torch.from_numpy(np.sort(lam))).abs().max()) / anorm
    Vl = V.t()                                   # column-major storage -> logical matrix
    resid = float(torch.linalg.norm(A0 @ Vl - Vl * w[None, :])) / (n * anorm)
    O_ = Vl.t() @ Vl
    O_.diagonal().sub_(1.0)
    orth = float(torch.linalg.norm(O_)) / np.sqrt(n)
    assert dl < 1e-12, dl
    assert resid < 1e-13, resid
    assert orth < 1e-13, orth


@pytest.mark.parametrize("n,nbw", [(4740, 32), (4768, 32), (2372, 64), (2384, 64)])
def test_backtransform_overlap_last_group(cuda, n, nbw):
    """The back-transform's BC-back grid at n = 4740 / 4768 (b = 32) is 148 groups of 32 columns
    (one whole wave on 148 SMs) plus one group 4 / 32 columns wide, and at n = 2372 / 2384
    (b = 64, 16 columns per CTA) 148 groups of 16 plus one of 4 / 16: the whole wave runs first,
    then the one-CTA last wave beside the SBR-back of the first columns, then the SBR-back of the
    last columns.  Every column must come out right: residual and orthogonality over all of V, and
    the eigenvalues against the eigenvalues-only path (bisection, no back-transform)."""
    import torch
    import cuev_b200 as cv
    g = torch.Generator(device=cuda).manual_seed(n)
    G = torch.randn(n, n, dtype=torch.float64, device=cuda, generator=g)
    A = (G + G.t()) * 0.5                        # symmetric: row- and column-major storage agree
    del G
    A0 = A.clone()
    w_bis = torch.zeros(n, dtype=torch.float64, device=cuda)
    cv.symm_eig_solve(A0.clone(), n, w_bis, None, nbw=nbw, nk=256)
    w = torch.zeros(n, dtype=torch.float64, device=cuda)
    V = torch.zeros(n, n, dtype=torch.float64, device=cuda)
    cv.symm_eig_solve(A, n, w, V, nbw=nbw, nk=256)
    torch.cuda.synchronize()
    anorm = float(w_bis.abs().max())
    dl = float((w - w_bis).abs().max()) / anorm
    Vl = V.t()                                   # column-major storage -> logical matrix
    R = A0 @ Vl - Vl * w[None, :]
    resid = float(torch.linalg.norm(R)) / (n * anorm)
    worst_col = float(torch.linalg.norm(R, dim=0).max()) / anorm
    O_ = Vl.t() @ Vl
    O_.diagonal().sub_(1.0)
    orth = float(torch.linalg.norm(O_)) / np.sqrt(n)
    assert dl < 1e-12, dl
    assert resid < 1e-13, resid
    assert worst_col < 1e-11, worst_col
    assert orth < 1e-13, orth


@pytest.mark.parametrize("n,nbw,nk", [(4740, 32, 256), (777, 32, 128), (100, 32, 256),
                                      (1500, 64, 256), (131, 64, 128)])
def test_no_access_past_the_matrix(cuda, n, nbw, nk):
    """n not a multiple of b: the band reduction's last panel update covers fewer than b columns
    and must stop at column n - 1.  A (and V, w) sit at the front of larger device buffers filled
    with a sentinel; after the full solve and the eigenvalues-only solve every sentinel is intact
    (writes past the matrix would change them) and the results are right."""
    import torch
    import cuev_b200 as cv
    A = _sym(n, n + 5)
    pad = 64 * n + 4096
    sent = 12345.0

    def padded(numel, init=None):
        buf = torch.full((numel + pad,), sent, dtype=torch.float64, device=cuda)
        if init is not None:
            buf[:numel] = init
        return buf

    a_col = torch.from_numpy(np.asfortranarray(A).ravel(order="F").copy()).to(cuda)
    for evec in (True, False):
        bA = padded(n * n, a_col)
        bw = padded(n)
        bV = padded(n * n) if evec else None
        cv.symm_eig_solve(bA[: n * n], n, bw[:n], bV[: n * n] if evec else None, nbw=nbw, nk=nk)
        torch.cuda.synchronize()
        for buf, numel in ((bA, n * n), (bw, n)) + (((bV, n * n),) if evec else ()):
            tail = buf[numel:]
            assert bool((tail == sent).all()), int((tail != sent).sum())
        w = bw[:n].cpu().numpy()
        w_ref = np.linalg.eigvalsh(A)
        assert np.abs(w - w_ref).max() / np.abs(w_ref).max() < 1e-12
        if evec:
            V = bV[: n * n].cpu().numpy().reshape((n, n)).T
            resid = np.linalg.norm(A @ V - V * w) / (n * np.abs(w_ref).max())
            assert resid < 1e-13, resid


@pytest.mark.parametrize("entry", ["fp32", "mixed"])
def test_no_access_past_the_buffers_other_entries(cuda, entry):
    """The FP32 entry and the precision form at n = 1001 (not a multiple of 32): the caller's
    A, w and V sit at the front of sentinel-filled buffers, which must come back intact."""
    import torch
    import cuev_b200 as cv
    n = 1001
    A = _sym(n, 17)
    dt = torch.float32 if entry == "fp32" else torch.float64
    pad = 64 * n + 4096
    sent = 12345.0
    a_col = torch.from_numpy(np.asfortranarray(A).ravel(order="F").copy()).to(cuda, dt)
    bufs = [torch.full((numel + pad,), sent, dtype=dt, device=cuda) for numel in (n * n, n, n * n)]
    bA, bw, bV = bufs
    bA[: n * n] = a_col
    if entry == "fp32":
        cv.symm_eig_solve(bA[: n * n], n, bw[:n], bV[: n * n])
    else:
        cv.symm_eig_solve_mixed(bA[: n * n], n, bw[:n], bV[: n * n])
    torch.cuda.synchronize()
    for buf, numel in zip(bufs, (n * n, n, n * n)):
        assert bool((buf[numel:] == sent).all()), int((buf[numel:] != sent).sum())
    w = bw[:n].double().cpu().numpy()
    w_ref = np.linalg.eigvalsh(A)
    tol = 1e-5 if entry == "fp32" else 1e-12
    assert np.abs(w - w_ref).max() / np.abs(w_ref).max() < tol


def test_timer_and_reuse(cuda):
    import cuev_b200 as cv
    A = _sym(600, 3)
    t = cv.Timer()
    w1, V1 = _solve(cuda, A, 32, 256, timer=t)
    w2, V2 = _solve(cuda, A, 32, 256)  # cached workspace, identical result
    assert np.array_equal(w1, w2) and np.array_equal(V1, V2)
    d = t.as_dict()
    assert d["dbbr_ms"] > 0 and d["bc_ms"] > 0 and d["dc_ms"] > 0 and d["bt_ms"] > 0
    assert d["total_ms"] >= d["dbbr_ms"]


@pytest.mark.parametrize("n", [2, 20, 33, 65, 300, 3072])
def test_fp32_entry(cuda, n):
    """symm_eig_solve<float>: BC-back runs in FP32 and, at n = 3072, the back-transform's products
    (>= 2^30 multiply-adds) on the FP32-level int8 tensor-core path; the reference's own FP32
    tests allow 1e-3 (test/cuda/test_dbbr.cu:152-164), these bounds are tighter (measured 1.7e-6
    residual and 2.1e-6 orthogonality at n = 3072)."""
    import torch
    import cuev_b200 as cv
    A = _sym(n, 4).astype(np.float32)
    dA = torch.from_numpy(np.asfortranarray(A).ravel(order="F").copy()).to(cuda)
    w = torch.zeros(n, dtype=torch.float32, device=cuda)
    V = torch.zeros(n * n, dtype=torch.float32, device=cuda)
    cv.symm_eig_solve(dA, n, w, V)
    torch.cuda.synchronize()
    Vn = V.cpu().numpy().reshape((n, n)).T.astype(np.float64)
    wn = w.cpu().numpy().astype(np.float64)
    A64 = A.astype(np.float64)
    assert np.linalg.norm(A64 @ Vn - Vn * wn) / np.linalg.norm(A64) < 1e-5
    assert np.abs(wn - np.linalg.eigvalsh(A64)).max() < 1e-5 * np.abs(wn).max()
    assert np.linalg.norm(Vn.T @ Vn - np.eye(n)) / np.sqrt(n) < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 300, 5000])
def test_host_entry(cuda, n):
    """cuev_dsyevd_host copies A in, solves and copies the eigenvectors out as they become final
    (at n = 5000 the columns of BC-back's whole waves leave while the last columns are computed);
    the results are the device entry's, bit for bit."""
    import torch
    import cuev_b200 as cv
    A = _sym(n, 11)
    w_h, V_h = cv.eigh_host(A)
    dA = torch.from_numpy(np.asfortranarray(A).ravel(order="F").copy()).to(cuda)
    w = torch.zeros(n, dtype=torch.float64, device=cuda)
    V = torch.zeros(n * n, dtype=torch.float64, device=cuda)
    cv.symm_eig_solve(dA, n, w, V)
    torch.cuda.synchronize()
    assert np.array_equal(w_h.numpy(), w.cpu().numpy())
    assert np.array_equal(V_h.t().contiguous().numpy().ravel(), V.cpu().numpy())
    w2, V2 = cv.eigh_host(A, evec=False)                      # eigenvalues only (bisection)
    assert V2 is None
    assert np.abs(w2.numpy() - w_h.numpy()).max() <= 1e-12 * max(1.0, np.abs(w_h.numpy()).max())


def test_error_codes(cuda):
    import torch
    import cuev_b200 as cv
    L = cv.lib()
    assert L.cuev_dsyevd(None, -1, None, None, None, None) == -1
    assert L.cuev_dsyevd(None, 0, None, None, None, None) == 0
    n = 64
    A = torch.from_numpy(np.asfortranarray(_sym(n, 5)).ravel(order="F").copy()).to(cuda)
    A[3 * n + 10] = float("nan")
    w = torch.zeros(n, dtype=torch.float64, device=cuda)
    V = torch.zeros(n * n, dtype=torch.float64, device=cuda)
    st = L.cuev_dsyevd(A.data_ptr(), n, w.data_ptr(), V.data_ptr(), None, None)
    assert st == -5  # CUEV_ERR_NONFINITE
    assert b"device status" in L.cuev_last_error()
    # the library stays usable afterwards
    A2 = _sym(n, 6)
    w2, V2 = _solve(cuda, A2)
    assert np.abs(w2 - np.linalg.eigvalsh(A2)).max() < 1e-12 * np.abs(w2).max()


def test_concurrent_solves_on_two_threads(cuda):
    """Two host threads, each with its own stream, solve different matrices at the same time (one
    finds the cached workspace busy and takes its own), three rounds; every result must match
    LAPACK."""
    import threading
    import torch
    import cuev_b200 as cv
    jobs = [(777, 32, 128), (1000, 64, 256)]
    mats = {n: _sym(n, 40 + n) for n, _, _ in jobs}
    refs = {n: sla.eigh(mats[n], eigvals_only=True, driver="evd") for n in mats}
    errors = []

    def worker(n, nbw, nk):
        try:
            s = torch.cuda.Stream()
            with torch.cuda.stream(s):
                for _ in range(3):
                    A = mats[n]
                    dA = torch.from_numpy(np.asfortranarray(A).ravel(order="F").copy()).to(cuda)
                    w = torch.zeros(n, dtype=torch.float64, device=cuda)
                    V = torch.zeros(n * n, dtype=torch.float64, device=cuda)
                    cv.symm_eig_solve(dA, n, w, V, stream=s, nbw=nbw, nk=nk)
                    s.synchronize()
                    wn = w.cpu().numpy()
                    Vn = V.cpu().numpy().reshape((n, n)).T
                    m = O.metrics(A, wn, Vn, refs[n])
                    if not (m["max_dlambda_rel"] < 1e-12 and m["resid_n_norm2"] < 1e-13):
                        errors.append((n, m))
        except Exception as exc:  # reported below, on the main thread
            errors.append((n, repr(exc)))

    threads = [threading.Thread(target=worker, args=job) for job in jobs]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
