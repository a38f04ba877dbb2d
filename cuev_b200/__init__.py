"""cuev_b200 — B200-native symmetric eigensolver (drop-in for cuEV's ``symm_eig_solve``).

The product is ``libcuev_b200.so`` (hand-written sm_100a CUDA behind the C ABI in
``include/cuev_b200.h``).  This module is the Python host side: it loads that library with
ctypes and mirrors the reference's C++ interface on torch device tensors:

* ``symm_eig_solve(A, n, eval, evec, stream=None, timer=None)``  — reference
  ``cuev::symm_eig_solve<T>`` (include/cuev.h:31-33): A is overwritten, eval ascending, evec
  columns are eigenvectors, column-major (a torch tensor ``X`` holding a column-major matrix is
  passed as ``X`` whose memory is column-major, i.e. ``X.T`` of a row-major view).
* ``SolverHandle`` + stage functions — reference ``SolverHandle<T>`` / ``cuev::kernels::*``
  (include/cuda/handle.h:61-100, include/cuda/kernels.cuh:47-155).

There is no CPU fallback: if the library is missing the import of any entry fails loudly.
torch is used only for device memory and streams.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libcuev_b200.so"

CUEV_OK = 0
STATUS_NAMES = {
    0: "CUEV_OK", -1: "CUEV_ERR_INVALID", -2: "CUEV_ERR_ALLOC", -3: "CUEV_ERR_CUDA",
    -4: "CUEV_ERR_TIMEOUT", -5: "CUEV_ERR_NONFINITE", -6: "CUEV_ERR_CONVERGENCE",
    -7: "CUEV_ERR_UNSUPPORTED",
}

BUF_B, BUF_D, BUF_E, BUF_Y, BUF_U, BUF_TAU = range(6)


class CuevError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str = ""):
        self.status = status
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)} {msg}".strip())


class Timer(C.Structure):
    """Same field order as the reference's cuev::SolveTimer (include/cuda/handle.h:25-37)."""

    _fields_ = [(n, C.c_float) for n in (
        "dbbr_ms", "bc_ms", "dc_ms", "bt_ms", "total_ms",
        "bt_copyin_ms", "bt_qb_ms", "bt_qs_ms", "bt_copyout_ms")]

    def as_dict(self):
        return {n: float(getattr(self, n)) for n, _ in self._fields_}


class Config(C.Structure):
    _fields_ = [("nbw", C.c_int), ("nk", C.c_int)]


class MixedInfo(C.Structure):
    """cuev_mixed_info: refinement steps, last measured norms and the two parts' times."""

    _fields_ = [("refine_iterations", C.c_int), ("offdiag_fro", C.c_double),
                ("orth_fro", C.c_double), ("anorm", C.c_double), ("first_ms", C.c_float),
                ("refine_ms", C.c_float)]

    def as_dict(self):
        return {n: (float(getattr(self, n)) if n != "refine_iterations"
                    else int(getattr(self, n))) for n, _ in self._fields_}


PRODUCTS_FP64, PRODUCTS_INT8 = 0, 1


class RefineInfo(C.Structure):
    """cuev_refine_info: steps applied and the norms measured on the last X."""

    _fields_ = [("iterations", C.c_int), ("offdiag_fro", C.c_double), ("orth_fro", C.c_double),
                ("anorm", C.c_double)]


_VP, _I, _D, _DP, _FP = C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_void_p
_SIGS = {
    "cuev_dsyevd": [_DP, _I, _DP, _DP, _VP, C.POINTER(Timer)],
    "cuev_dsyevd_cfg": [_DP, _I, _DP, _DP, _VP, C.POINTER(Timer), C.POINTER(Config)],
    "cuev_ssyevd": [_FP, _I, _FP, _FP, _VP, C.POINTER(Timer)],
    "cuev_dsyevd_host": [_VP, _I, _VP, _VP, _VP, C.POINTER(Timer)],
    "cuev_release_workspace": [],
    "cuev_handle_create": [_I, _I, _I, _VP, C.POINTER(C.c_void_p)],
    "cuev_handle_destroy": [_VP],
    "cuev_handle_buffer": [_VP, _I, C.POINTER(C.c_void_p), C.POINTER(C.c_longlong)],
    "cuev_dbbr_panel_qr": [_VP, _DP, _I, _DP, _I, _DP, _DP, _I, _I],
    "cuev_dbbr_reduce": [_VP, _DP],
    "cuev_dbbr_pack": [_VP, _DP, _DP],
    "cuev_bc_chase": [_VP, _DP, _DP, _DP],
    "cuev_tridi_dc": [_VP, _DP, _DP, _DP, _DP],
    "cuev_tridi_eigvals": [_VP, _DP, _DP, _DP],
    "cuev_bc_back": [_VP, _DP, _I],
    "cuev_sbr_back": [_VP, _DP, _I],
    "cuev_back_transform": [_VP, _DP, C.POINTER(Timer)],
    "cuev_dgemm": [_VP, _I, _I, _I, _I, _I, _D, _DP, _I, _DP, _I, _D, _DP, _I],
    "cuev_dgemm_noalloc": [_VP, _I, _I, _I, _I, _I, _D, _DP, _I, _DP, _I, _D, _DP, _I],
    "cuev_dgemm_i8": [_VP, _I, _I, _I, _I, _I, _I, _D, _DP, _I, _DP, _I, _D, _DP, _I],
    "cuev_dsymm_lower": [_VP, _I, _I, _D, _DP, _I, _DP, _I, _D, _DP, _I],
    "cuev_dsyr2k_lower": [_VP, _I, _I, _D, _DP, _I, _DP, _I, _D, _DP, _I],
    "cuev_dsyev_refine": [_DP, _I, _DP, _DP, _I, _D, _VP, C.POINTER(RefineInfo)],
    "cuev_dsyev_refine_ex": [_DP, _I, _DP, _DP, _I, _D, _I, _VP, C.POINTER(RefineInfo)],
    "cuev_dsyevd_mixed": [_DP, _I, _DP, _DP, _VP, C.POINTER(Timer), _I, _D,
                          C.POINTER(MixedInfo)],
    "cuev_dsyevd_batched": [_DP, _I, _I, _DP, _DP, _VP],
    "cuev_debug_set_wait_limit_ns": [C.c_ulonglong],
    "cuev_dsyev_adjoint": [_DP, _DP, _DP, _DP, _I, _D, _DP, _VP],
    "cuev_ssyev_adjoint": [_FP, _FP, _FP, _FP, _I, C.c_float, _FP, _VP],
}

_lib = None


def lib() -> C.CDLL:
    """Load libcuev_b200.so (built by ``python -m cuev_b200.build``).  Raises if absent."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m cuev_b200.build` "
                "(there is no CPU fallback)")
        L = C.CDLL(str(LIB_PATH))
        for name, args in _SIGS.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.argtypes = args
            fn.restype = C.c_int
        L.cuev_last_error.restype = C.c_char_p
        L.cuev_last_error.argtypes = []
        if hasattr(L, "cuev_last_dc_flops"):
            L.cuev_last_dc_flops.restype = C.c_double
            L.cuev_last_dc_flops.argtypes = []
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return [n for n in list(_SIGS) + ["cuev_last_error", "cuev_last_dc_flops"]
            if hasattr(lib(), n)]


def _check(status: int, where: str):
    if status != CUEV_OK:
        raise CuevError(status, where, lib().cuev_last_error().decode(errors="replace"))


def _ptr(t) -> int | None:
    if t is None:
        return None
    return t.data_ptr()


def _stream(stream):
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    if hasattr(stream, "cuda_stream"):
        return stream.cuda_stream
    return int(stream)


def _need_f64(*ts):
    import torch
    for t in ts:
        if t is not None:
            if not t.is_cuda:
                raise ValueError("cuev_b200 takes device tensors (pass .cuda())")
            if t.dtype != torch.float64:
                raise ValueError(f"expected float64, got {t.dtype}")
            if not t.is_contiguous():
                raise ValueError("tensors must be contiguous (column-major data in memory)")


# ------------------------------------------------------------------------------------------
# Full solves (reference include/cuev.h:31-33)
# ------------------------------------------------------------------------------------------
def symm_eig_solve(A, n: int, eval, evec, stream=None, timer: Timer | None = None,
                   nbw: int = 0, nk: int = 0) -> None:
    """In-place FP64/FP32 solve on device tensors; same argument meaning as the reference.

    ``A`` holds the n x n column-major matrix (lower triangle read, overwritten), ``eval`` gets
    the ascending eigenvalues and ``evec`` the eigenvectors as columns (column-major).
    """
    import torch
    t = C.byref(timer) if timer is not None else None
    if A.dtype == torch.float32:
        st = lib().cuev_ssyevd(_ptr(A), n, _ptr(eval), _ptr(evec), _stream(stream), t)
        _check(st, "cuev_ssyevd")
        return
    _need_f64(A, eval, evec)
    cfg = Config(nbw, nk)
    st = lib().cuev_dsyevd_cfg(_ptr(A), n, _ptr(eval), _ptr(evec), _stream(stream), t,
                               C.byref(cfg))
    _check(st, "cuev_dsyevd")


def eigh(A_rowmajor_sym, nbw: int = 0, nk: int = 0):
    """Convenience: eigen-decomposition of a symmetric torch matrix (returns w, V with
    A = V diag(w) V^T, V's columns the eigenvectors).  Uses the lower triangle."""
    import torch
    n = A_rowmajor_sym.shape[0]
    Acm = A_rowmajor_sym.t().contiguous().clone()  # column-major storage of A
    w = torch.empty(n, dtype=Acm.dtype, device=Acm.device)
    Vcm = torch.empty_like(Acm)
    symm_eig_solve(Acm, n, w, Vcm, nbw=nbw, nk=nk)
    return w, Vcm.t()


def refine(A, n: int, eval, evec, max_iters: int = 2, tol: float = 0.0,
           stream=None, products: int = PRODUCTS_FP64) -> RefineInfo:
    """Ogita-Aishima refinement in place: ``evec`` (column-major n x n eigenvector columns) is
    improved against the symmetric ``A`` (column-major, lower triangle read, not modified) and
    ``eval`` receives the refined eigenvalues.  ``products``: PRODUCTS_FP64 (DMMA) or
    PRODUCTS_INT8 (int8 tensor cores).  Returns the step count and measured norms."""
    _need_f64(A, eval, evec)
    info = RefineInfo()
    if products == PRODUCTS_FP64:
        st = lib().cuev_dsyev_refine(_ptr(A), n, _ptr(eval), _ptr(evec), max_iters, tol,
                                     _stream(stream), C.byref(info))
    else:
        st = lib().cuev_dsyev_refine_ex(_ptr(A), n, _ptr(eval), _ptr(evec), max_iters, tol,
                                        int(products), _stream(stream), C.byref(info))
    _check(st, "cuev_dsyev_refine")
    return info


def symm_eig_solve_mixed(A, n: int, eval, evec, max_refine_iters: int = 2, tol: float = 0.0,
                         stream=None, timer: Timer | None = None) -> MixedInfo:
    """Precision form (``cuev_dsyevd_mixed``): same arguments and result as ``symm_eig_solve``
    (FP64 tensors, A overwritten); FP32-level tensor-core first solve, then refinement with
    FP64-level int8 tensor-core products.  Returns the refinement record."""
    _need_f64(A, eval, evec)
    info = MixedInfo()
    t = C.byref(timer) if timer is not None else None
    st = lib().cuev_dsyevd_mixed(_ptr(A), n, _ptr(eval), _ptr(evec), _stream(stream), t,
                                 int(max_refine_iters), float(tol), C.byref(info))
    _check(st, "cuev_dsyevd_mixed")
    return info


def eigvalsh(A_rowmajor_sym, nbw: int = 0, nk: int = 0):
    """Eigenvalues only (ascending) of a symmetric torch matrix: band reduction, bulge chase and
    bisection, no eigenvectors.  Uses the lower triangle."""
    import torch
    n = A_rowmajor_sym.shape[0]
    Acm = A_rowmajor_sym.t().contiguous().clone()
    w = torch.empty(n, dtype=Acm.dtype, device=Acm.device)
    symm_eig_solve(Acm, n, w, None, nbw=nbw, nk=nk)
    return w


def eigh_batched(A_batch):
    """Eigen-decompositions of a stack of small symmetric matrices (batch, n, n), n <= 512, in one
    launch.  Returns (w, V) with A[b] = V[b] diag(w[b]) V[b]^T; reads the lower triangles."""
    import torch
    if A_batch.dim() != 3 or A_batch.shape[1] != A_batch.shape[2]:
        raise ValueError("expected a (batch, n, n) tensor")
    bsz, n = A_batch.shape[0], A_batch.shape[1]
    Acm = A_batch.transpose(1, 2).contiguous()     # column-major storage of each matrix
    _need_f64(Acm)
    w = torch.empty(bsz, n, dtype=torch.float64, device=Acm.device)
    Vcm = torch.empty_like(Acm)
    _check(lib().cuev_dsyevd_batched(_ptr(Acm), n, bsz, _ptr(w), _ptr(Vcm),
                                     _stream(None)), "cuev_dsyevd_batched")
    return w, Vcm.transpose(1, 2)


def eigh_host(A, evec: bool = True, stream=None, timer: Timer | None = None):
    """Host-buffer solve (cuev_dsyevd_host): A is a (n, n) float64 array on the host, symmetric
    (its lower triangle is read; a C-ordered array is the transpose, the same for a symmetric
    matrix).  Returns (w, V) as host torch tensors (pinned), V column-major with eigenvectors as
    columns (V[:, i] for w[i]); V is None when evec is False."""
    import numpy as np
    import torch
    A_np = np.ascontiguousarray(np.asarray(A, dtype=np.float64))
    n = A_np.shape[0]
    if A_np.shape != (n, n):
        raise ValueError("expected a square matrix")
    hA = torch.from_numpy(A_np.T.copy()).pin_memory()          # column-major storage
    w = torch.empty(n, dtype=torch.float64).pin_memory()
    V = torch.empty(n * n, dtype=torch.float64).pin_memory() if evec else None
    st = lib().cuev_dsyevd_host(hA.data_ptr(), n, w.data_ptr(), V.data_ptr() if evec else None,
                                _stream(stream), C.byref(timer) if timer else None)
    _check(st, "cuev_dsyevd_host")
    return w, (V.view(n, n).t() if evec else None)


def debug_set_wait_limit_ns(ns: int) -> None:
    """Failure-path tests only: every bounded device wait gives up after `ns` nanoseconds
    (0 restores the default 2 s)."""
    _check(lib().cuev_debug_set_wait_limit_ns(int(ns)), "cuev_debug_set_wait_limit_ns")


def release_workspace():
    _check(lib().cuev_release_workspace(), "cuev_release_workspace")


# ------------------------------------------------------------------------------------------
# Stage-level API (reference SolverHandle<T> + cuev::kernels::*)
# ------------------------------------------------------------------------------------------
class SolverHandle:
    """Mirror of the reference ``SolverHandle<double>`` (handle_alloc / handle_free).

    ``buffer()`` returns torch views of the handle's device buffers.  The workspace is released
    only once the handle is closed AND every such view is gone, so a view that outlives the
    ``with`` block (a traceback that prints it, say) never reads freed device memory."""

    def __init__(self, n: int, nbw: int = 32, nk: int = 512, stream=None):
        self.n, self.nbw, self.nk = n, nbw, nk
        self._stream = _stream(stream)
        self._views = 0
        self._closed = False
        h = C.c_void_p()
        _check(lib().cuev_handle_create(n, nbw, nk, self._stream, C.byref(h)),
               "cuev_handle_create")
        self.h = h

    def _destroy(self):
        if getattr(self, "h", None):
            h, self.h = self.h, None
            _check(lib().cuev_handle_destroy(h), "cuev_handle_destroy")

    def _view_gone(self):
        self._views -= 1
        if self._closed and self._views == 0:
            self._destroy()

    def close(self):
        self._closed = True
        if getattr(self, "_views", 0) == 0:
            self._destroy()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self._closed = True
            self._destroy()
        except Exception:
            pass

    def buffer(self, which: int, rows: int, cols: int):
        """A torch view (column-major storage as a (cols, ld) row-major tensor) of a handle
        buffer; returns (tensor, ld)."""
        import torch
        import weakref
        p = C.c_void_p()
        ld = C.c_longlong()
        _check(lib().cuev_handle_buffer(self.h, which, C.byref(p), C.byref(ld)),
               "cuev_handle_buffer")
        t, holder = _wrap_device(p.value, cols * ld.value, torch.float64, with_holder=True)
        # the tensor's storage keeps `holder` alive; when the last tensor sharing it is gone the
        # holder is collected and the handle may free its workspace
        self._views += 1
        fin = weakref.finalize(holder, self._view_gone)
        fin.atexit = False  # at interpreter exit the process releases the device memory anyway
        return t.view(cols, ld.value), ld.value

    # stage launchers -----------------------------------------------------------------------
    def dbbr_panel_qr(self, A, lda, Y, ldy, tau, T, rows, b):
        _check(lib().cuev_dbbr_panel_qr(self.h, _ptr(A), lda, _ptr(Y), ldy, _ptr(tau),
                                         _ptr(T), rows, b), "dbbr_panel_qr")

    def dbbr_reduce(self, A):
        _check(lib().cuev_dbbr_reduce(self.h, _ptr(A)), "dbbr_reduce")

    def dbbr_pack(self, A, B):
        _check(lib().cuev_dbbr_pack(self.h, _ptr(A), _ptr(B)), "dbbr_pack")

    def bc_chase(self, B, d, e):
        _check(lib().cuev_bc_chase(self.h, _ptr(B), _ptr(d), _ptr(e)), "bc_chase")

    def tridi_dc(self, d, e, eval, evec):
        _check(lib().cuev_tridi_dc(self.h, _ptr(d), _ptr(e), _ptr(eval), _ptr(evec)),
               "tridi_dc")

    def tridi_eigvals(self, d, e, eval):
        _check(lib().cuev_tridi_eigvals(self.h, _ptr(d), _ptr(e), _ptr(eval)), "tridi_eigvals")

    def bc_back(self, M, ldm):
        _check(lib().cuev_bc_back(self.h, _ptr(M), ldm), "bc_back")

    def sbr_back(self, M, ldm):
        _check(lib().cuev_sbr_back(self.h, _ptr(M), ldm), "sbr_back")

    def back_transform(self, evec, timer: Timer | None = None):
        t = C.byref(timer) if timer is not None else None
        _check(lib().cuev_back_transform(self.h, _ptr(evec), t), "back_transform")


def _wrap_device(ptr: int, numel: int, dtype, with_holder: bool = False):
    """Non-owning torch view of device memory owned by the library (torch keeps a reference to
    the interface object for as long as the tensor's storage lives)."""
    import torch

    class _Holder:
        pass

    h = _Holder()
    h.__cuda_array_interface__ = {
        "shape": (numel,), "typestr": "<f8" if dtype == torch.float64 else "<f4",
        "data": (ptr, False), "version": 2, "strides": None,
    }
    t = torch.as_tensor(h, device="cuda")
    return (t, h) if with_holder else t


# ------------------------------------------------------------------------------------------
# GEMM entries (reference cuev::cublas wrappers)
# ------------------------------------------------------------------------------------------
def dgemm(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc, stream=None):
    _check(lib().cuev_dgemm(_stream(stream), int(ta), int(tb), m, n, k, alpha, _ptr(A), lda,
                            _ptr(B), ldb, beta, _ptr(Cm), ldc), "cuev_dgemm")


def dgemm_noalloc(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc, stream=None):
    """``cuev_dgemm`` without any device allocation (split-K partials in the library's fixed
    16 MiB array; m * n <= 1048576; concurrent calls race)."""
    _check(lib().cuev_dgemm_noalloc(_stream(stream), int(ta), int(tb), m, n, k, alpha, _ptr(A),
                                    lda, _ptr(B), ldb, beta, _ptr(Cm), ldc), "cuev_dgemm_noalloc")


def dgemm_i8(ta, tb, m, n, k, slices, alpha, A, lda, B, ldb, beta, Cm, ldc, stream=None):
    """``cuev_dgemm_i8``: the same product emulated on the int8 tensor cores from ``slices``
    7-bit slices per operand (7: FP64-level, 4: FP32-level accuracy)."""
    _check(lib().cuev_dgemm_i8(_stream(stream), int(ta), int(tb), m, n, k, int(slices), alpha,
                               _ptr(A), lda, _ptr(B), ldb, beta, _ptr(Cm), ldc), "cuev_dgemm_i8")


def dsymm_lower(m, n, alpha, A, lda, B, ldb, beta, Cm, ldc, stream=None):
    _check(lib().cuev_dsymm_lower(_stream(stream), m, n, alpha, _ptr(A), lda, _ptr(B), ldb,
                                  beta, _ptr(Cm), ldc), "cuev_dsymm_lower")


def dsyr2k_lower(n, k, alpha, A, lda, B, ldb, beta, Cm, ldc, stream=None):
    _check(lib().cuev_dsyr2k_lower(_stream(stream), n, k, alpha, _ptr(A), lda, _ptr(B), ldb,
                                   beta, _ptr(Cm), ldc), "cuev_dsyr2k_lower")
