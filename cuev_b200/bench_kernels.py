"""Per-kernel timings of libcuev_b200 through its C ABI (CUDA events on the launching stream).

    python -m cuev_b200.bench_kernels gemm M N K [--ta] [--tb]   DMMA GEMM vs torch (cuBLAS)
    python -m cuev_b200.bench_kernels i8gemm M N K [--slices S]  FP64 GEMM emulated on int8 tcgen05
    python -m cuev_b200.bench_kernels symm M N                   C = A B, A symmetric (lower)
    python -m cuev_b200.bench_kernels syr2k N K                  lower(C) = A B^T + B A^T
    python -m cuev_b200.bench_kernels stages N                   every solver stage on its own
    python -m cuev_b200.bench_kernels refine N [--iters K]       Ogita-Aishima refinement
    python -m cuev_b200.bench_kernels eigvals N                  eigenvalues-only solve
    python -m cuev_b200.bench_kernels mixed N [--iters K]        precision form vs FP64 solve
    python -m cuev_b200.bench_kernels overlap N                  D&C and BC-back alone / together
    python -m cuev_b200.bench_kernels adjoint N                  eigh forward + adjoint
    python -m cuev_b200.bench_kernels batched N BATCH            batched small-n eigh vs torch

`stages` runs the pipeline through the stage entry points (cuev_dbbr_reduce, cuev_bc_chase,
cuev_tridi_dc, cuev_bc_back, cuev_sbr_back) with an event pair around each, so a profiler can
select one stage's kernels with few launches before them.  Inputs are seeded random matrices
(A = (G + G^T)/2, G iid N(0,1)).
"""
from __future__ import annotations

import argparse
import json
import statistics

import torch

import cuev_b200 as cv


def _time(fn, reps: int, warmup: int) -> float:
    """Median milliseconds of fn() over reps launches, after warmup launches."""
    st = torch.cuda.current_stream()
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    out = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fn()
        e1.record(st)
        torch.cuda.synchronize()
        out.append(e0.elapsed_time(e1))
    return statistics.median(out)


def _rand(rows, cols, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    return torch.randn(rows, cols, dtype=torch.float64, device="cuda", generator=g)


def run_gemm(a):
    m, n, k = a.M, a.N, a.K
    # column-major operands: a (rows x cols) column-major matrix is a (cols, rows) torch tensor
    A = _rand(m if a.ta else k, k if a.ta else m, 1)   # op(A) = m x k
    B = _rand(k if a.tb else n, n if a.tb else k, 2)   # op(B) = k x n
    Cm = torch.zeros(n, m, dtype=torch.float64, device="cuda")
    lda = k if a.ta else m
    ldb = n if a.tb else k
    ms = _time(lambda: cv.dgemm(a.ta, a.tb, m, n, k, 1.0, A, lda, B, ldb, 0.0, Cm, m),
               a.reps, a.warmup)
    # cuBLAS on the same product, for scale
    At = A.t() if not a.ta else A       # logical op(A) as a row-major (m, k) view
    Bt = B.t() if not a.tb else B
    ref_ms = _time(lambda: torch.matmul(At, Bt), a.reps, a.warmup)
    fl = 2.0 * m * n * k
    return {"kernel": "dgemm", "m": m, "n": n, "k": k, "ta": a.ta, "tb": a.tb,
            "ms": round(ms, 4), "tflops": round(fl / ms / 1e9, 3),
            "cublas_ms": round(ref_ms, 4), "cublas_tflops": round(fl / ref_ms / 1e9, 3)}


def run_i8gemm(a):
    """cuev_dgemm_i8 (slicing + tcgen05 int8 products, one call); int8 TOPS count
    s (s + 1) / 2 slice products of 2 m n k operations each."""
    m, n, k, s = a.M, a.N, a.K, a.slices
    A = _rand(k, m, 1)
    B = _rand(n, k, 2)
    Cm = torch.zeros(n, m, dtype=torch.float64, device="cuda")
    ms = _time(lambda: cv.dgemm_i8(0, 0, m, n, k, s, 1.0, A, m, B, k, 0.0, Cm, m),
               a.reps, a.warmup)
    ref_ms = _time(lambda: torch.matmul(A.t(), B.t()), a.reps, a.warmup)
    fl = 2.0 * m * n * k
    ops = fl * s * (s + 1) / 2
    return {"kernel": "dgemm_i8", "m": m, "n": n, "k": k, "slices": s, "ms": round(ms, 4),
            "fp64_equiv_tflops": round(fl / ms / 1e9, 3), "int8_tops": round(ops / ms / 1e9, 1),
            "cublas_dgemm_ms": round(ref_ms, 4), "cublas_tflops": round(fl / ref_ms / 1e9, 3)}


def run_symm(a):
    m, n = a.M, a.N
    A = _rand(m, m, 1)
    B = _rand(n, m, 2)
    Cm = torch.zeros(n, m, dtype=torch.float64, device="cuda")
    ms = _time(lambda: cv.dsymm_lower(m, n, 1.0, A, m, B, m, 0.0, Cm, m), a.reps, a.warmup)
    fl = 2.0 * m * m * n
    return {"kernel": "dsymm_lower", "m": m, "n": n, "ms": round(ms, 4),
            "tflops": round(fl / ms / 1e9, 3)}


def run_syr2k(a):
    n, k = a.M, a.N
    A = _rand(k, n, 1)
    B = _rand(k, n, 2)
    Cm = torch.zeros(n, n, dtype=torch.float64, device="cuda")
    ms = _time(lambda: cv.dsyr2k_lower(n, k, 1.0, A, n, B, n, 0.0, Cm, n), a.reps, a.warmup)
    fl = 2.0 * n * n * k  # lower triangle of two products
    return {"kernel": "dsyr2k_lower", "n": n, "k": k, "ms": round(ms, 4),
            "tflops": round(fl / ms / 1e9, 3)}


def run_stages(a):
    n = a.M
    A0 = _rand(n, n, 7)
    A0 = ((A0 + A0.t()) * 0.5).contiguous()
    A = torch.empty_like(A0)
    h = cv.SolverHandle(n, a.nbw, a.nk)
    try:
        b = a.nbw
        Bt, ldb = h.buffer(cv.BUF_B, 2 * b, n)
        d = torch.empty(n, dtype=torch.float64, device="cuda")
        e = torch.empty(n, dtype=torch.float64, device="cuda")
        w = torch.empty(n, dtype=torch.float64, device="cuda")
        V = torch.empty(n, n, dtype=torch.float64, device="cuda")
        names = ["dbbr_reduce", "bc_chase", "tridi_dc", "bc_back", "sbr_back"]
        times = {k: [] for k in names}
        st = torch.cuda.current_stream()
        for rep in range(a.warmup + a.reps):
            A.copy_(A0)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(len(names) + 1)]
            ev[0].record(st)
            h.dbbr_reduce(A)
            ev[1].record(st)
            h.bc_chase(Bt, d, e)
            ev[2].record(st)
            h.tridi_dc(d, e, w, V)
            ev[3].record(st)
            h.bc_back(V, n)
            ev[4].record(st)
            h.sbr_back(V, n)
            ev[5].record(st)
            torch.cuda.synchronize()
            if rep >= a.warmup:
                for i, k in enumerate(names):
                    times[k].append(ev[i].elapsed_time(ev[i + 1]))
        out = {k: round(statistics.median(v), 3) for k, v in times.items()} if a.reps else {}
        flops = {"bc_back": 2.0 * n ** 3, "sbr_back": 2.0 * n ** 3}
        rates = {k + "_tflops": round(flops[k] / out[k] / 1e9, 3) for k in flops if k in out}
        return {"kernel": "stages", "n": n, "nbw": a.nbw, "nk": a.nk, "ms": out, **rates}
    finally:
        h.close()


def run_overlap(a):
    """How much of BC-back (FP64 FMA, one CTA per SM) can hide under the divide and conquer
    (DMMA merge GEMMs and latency-bound kernels) when both run at once: the only gain open to a
    reordered back-transform that applies Q_b while D&C runs.  Two handles on two streams, each
    after its own band reduction and chase of the same matrix; times by CUDA events."""
    n = a.M
    A0 = _rand(n, n, 7)
    A0 = ((A0 + A0.t()) * 0.5).contiguous()
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    h1 = cv.SolverHandle(n, a.nbw, a.nk, stream=s1)
    h2 = cv.SolverHandle(n, a.nbw, a.nk, stream=s2)
    try:
        b = a.nbw
        vec = lambda: torch.empty(n, dtype=torch.float64, device="cuda")  # noqa: E731
        d1, e1, w1, d2, e2 = vec(), vec(), vec(), vec(), vec()
        Q1 = torch.empty(n, n, dtype=torch.float64, device="cuda")
        M2 = _rand(n, n, 11)
        for h, st, d, e in ((h1, s1, d1, e1), (h2, s2, d2, e2)):
            A = A0.clone()
            with torch.cuda.stream(st):
                h.dbbr_reduce(A)
                Bt, _ = h.buffer(cv.BUF_B, 2 * b, n)
                h.bc_chase(Bt, d, e)
            torch.cuda.synchronize()
            del A, Bt
        res = {"dc": [], "bc_back": [], "together": []}
        for rep in range(a.warmup + a.reps):
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
            # alone
            ev[0].record(s1)
            h1.tridi_dc(d1, e1, w1, Q1)
            ev[1].record(s1)
            torch.cuda.synchronize()
            ev[2].record(s2)
            h2.bc_back(M2, n)
            ev[3].record(s2)
            torch.cuda.synchronize()
            # together: both streams start at one event
            ev[4].record(s1)
            s2.wait_event(ev[4])
            h2.bc_back(M2, n)
            e_b = torch.cuda.Event(enable_timing=True)
            e_b.record(s2)
            h1.tridi_dc(d1, e1, w1, Q1)
            s1.wait_event(e_b)
            ev[5].record(s1)
            torch.cuda.synchronize()
            if rep >= a.warmup:
                res["dc"].append(ev[0].elapsed_time(ev[1]))
                res["bc_back"].append(ev[2].elapsed_time(ev[3]))
                res["together"].append(ev[4].elapsed_time(ev[5]))
        out = {k: round(statistics.median(v), 2) for k, v in res.items()}
        out["hidden_ms"] = round(out["dc"] + out["bc_back"] - out["together"], 2)
        return {"kernel": "overlap_dc_bc_back", "n": n, "nbw": a.nbw, "nk": a.nk, **out}
    finally:
        h1.close()
        h2.close()


def run_refine(a):
    """FP64 solve, eigenvectors rounded to FP32, then K refinement steps against A."""
    n = a.M
    A0 = _rand(n, n, 7)
    A0 = ((A0 + A0.t()) * 0.5).contiguous()
    A = A0.clone()
    w = torch.empty(n, dtype=torch.float64, device="cuda")
    V = torch.empty_like(A0)
    cv.symm_eig_solve(A, n, w, V)
    V32 = V.float().double()                       # FP32-accurate start
    out = {"kernel": "refine", "n": n, "iters": a.iters}

    def metrics(X, lam):
        Xl = X.t()                                 # column-major storage -> logical matrix
        R = A0 @ Xl - Xl * lam[None, :]
        resid = float(torch.linalg.norm(R) / (n * lam.abs().max()))
        O = Xl.t() @ Xl
        O.diagonal().sub_(1.0)
        return resid, float(torch.linalg.norm(O))

    out["start_resid"], out["start_orth"] = metrics(V32, w)
    times = []
    for rep in range(a.warmup + a.reps):
        X = V32.clone()
        lam = torch.empty_like(w)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        st = torch.cuda.current_stream()
        e0.record(st)
        info = cv.refine(A0, n, lam, X, max_iters=a.iters)
        e1.record(st)
        torch.cuda.synchronize()
        if rep >= a.warmup:
            times.append(e0.elapsed_time(e1))
    out["ms"] = round(statistics.median(times), 3)
    out["tflops_7n3_per_step"] = round(7.0 * n ** 3 * a.iters / out["ms"] / 1e9, 3)
    out["resid"], out["orth"] = metrics(X, lam)
    out["info"] = {"iterations": info.iterations, "offdiag_fro": info.offdiag_fro,
                   "orth_fro": info.orth_fro}
    return out


def _metrics_gpu(A, w, Vcm):
    """Residual ||A V - V diag(w)||_F / (n ||A||_2), orthogonality ||V^T V - I||_F (FP64 on the
    GPU; ||A||_2 = max |w|)."""
    n = A.shape[0]
    V = Vcm.view(n, n).t()
    R = A @ V - V * w[None, :]
    an = w.abs().max()
    I = torch.eye(n, dtype=torch.float64, device="cuda")
    return {"resid_n_norm2": float(torch.linalg.norm(R) / (n * an)),
            "orth_fro": float(torch.linalg.norm(V.t() @ V - I))}


def run_mixed(a):
    """The same seeded matrix through cuev_dsyevd (FP64) and cuev_dsyevd_mixed (FP32-level int8
    tensor-core first solve + --iters refinement steps); solve times by CUDA events."""
    n = a.M
    G = _rand(n, n, 7)
    A = (G + G.t()) / 2
    del G
    st = torch.cuda.current_stream()
    out = {"n": n, "refine_iters": a.iters}
    for form in ("fp64", "mixed"):
        ts = []
        for r in range(a.warmup + a.reps):
            Acm = A.clone()  # symmetric: its storage is its column-major storage
            w = torch.empty(n, dtype=torch.float64, device="cuda")
            V = torch.empty(n * n, dtype=torch.float64, device="cuda")
            tm = cv.Timer()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(st)
            if form == "fp64":
                cv.symm_eig_solve(Acm, n, w, V, timer=tm)
                info = None
            else:
                info = cv.symm_eig_solve_mixed(Acm, n, w, V, max_refine_iters=a.iters, timer=tm)
            e1.record(st)
            torch.cuda.synchronize()
            if r >= a.warmup:
                ts.append(e0.elapsed_time(e1))
            del Acm
        rec = {"ms": round(statistics.median(ts), 2), "stages": tm.as_dict()}
        if info is not None:
            rec["refine"] = info.as_dict()
        rec.update(_metrics_gpu(A, w, V))
        out[form] = rec
        del V
        torch.cuda.empty_cache()
    out["speedup_mixed_vs_fp64"] = round(out["fp64"]["ms"] / out["mixed"]["ms"], 3)
    return out


def run_eigvals(a):
    """Eigenvalues-only solve (evec = NULL) through the C ABI, with the per-stage timer."""
    n = a.M
    A0 = _rand(n, n, 7)
    A0 = ((A0 + A0.t()) * 0.5).contiguous()
    A = torch.empty_like(A0)
    w = torch.empty(n, dtype=torch.float64, device="cuda")
    t = cv.Timer()
    times, stages = [], []
    for rep in range(a.warmup + a.reps):
        A.copy_(A0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        st = torch.cuda.current_stream()
        e0.record(st)
        cv.symm_eig_solve(A, n, w, None, timer=t, nbw=a.nbw, nk=a.nk)
        e1.record(st)
        torch.cuda.synchronize()
        if rep >= a.warmup:
            times.append(e0.elapsed_time(e1))
            stages.append(t.as_dict())
    med = statistics.median(times)
    last = stages[-1]
    return {"kernel": "eigvals_only_solve", "n": n, "nbw": a.nbw, "nk": a.nk,
            "ms": round(med, 3), "dbbr_ms": round(last["dbbr_ms"], 3),
            "bc_ms": round(last["bc_ms"], 3), "bisection_ms": round(last["dc_ms"], 3)}


def run_adjoint(a):
    """Forward solve plus the adjoint (cuev_dsyev_adjoint) for seeded cotangents: the
    differentiation form's forward + backward time."""
    import ctypes as C
    n = a.M
    A0 = _rand(n, n, 7)
    A0 = ((A0 + A0.t()) * 0.5).contiguous()
    A = torch.empty_like(A0)
    w = torch.empty(n, dtype=torch.float64, device="cuda")
    V = torch.empty_like(A0)
    gw = _rand(1, n, 8).reshape(n)
    gV = _rand(n, n, 9)
    Abar = torch.empty_like(A0)
    L = cv.lib()
    st = torch.cuda.current_stream()
    fwd, bwd = [], []
    for rep in range(a.warmup + a.reps):
        A.copy_(A0)
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record(st)
        cv.symm_eig_solve(A, n, w, V, nbw=a.nbw, nk=a.nk)
        e[1].record(st)
        r = L.cuev_dsyev_adjoint(V.data_ptr(), w.data_ptr(), gV.data_ptr(), gw.data_ptr(), n,
                                 C.c_double(1e-12), Abar.data_ptr(), st.cuda_stream)
        cv._check(r, "cuev_dsyev_adjoint")
        e[2].record(st)
        torch.cuda.synchronize()
        if rep >= a.warmup:
            fwd.append(e[0].elapsed_time(e[1]))
            bwd.append(e[1].elapsed_time(e[2]))
    f, b = statistics.median(fwd), statistics.median(bwd)
    return {"kernel": "eigh_fwd_bwd", "n": n, "fwd_ms": round(f, 3), "bwd_ms": round(b, 3),
            "fwd_bwd_ms": round(f + b, 3),
            "bwd_tflops_6n3": round(6.0 * n ** 3 / b / 1e9, 3)}


def run_batched(a):
    n, bsz = a.M, a.N
    G = torch.randn(bsz, n, n, dtype=torch.float64, device="cuda",
                    generator=torch.Generator(device="cuda").manual_seed(3))
    A = (G + G.transpose(1, 2)) * 0.5
    ms = _time(lambda: cv.eigh_batched(A), a.reps, a.warmup)
    ref_ms = _time(lambda: torch.linalg.eigh(A), a.reps, a.warmup)
    return {"kernel": "eigh_batched", "n": n, "batch": bsz, "ms": round(ms, 3),
            "torch_linalg_eigh_ms": round(ref_ms, 3)}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("what", choices=["gemm", "i8gemm", "symm", "syr2k", "stages", "refine",
                                     "eigvals", "adjoint", "batched", "mixed", "overlap"])
    ap.add_argument("M", type=int)
    ap.add_argument("N", type=int, nargs="?", default=0)
    ap.add_argument("K", type=int, nargs="?", default=0)
    ap.add_argument("--ta", type=int, default=0)
    ap.add_argument("--tb", type=int, default=0)
    ap.add_argument("--nbw", type=int, default=32)
    ap.add_argument("--nk", type=int, default=0)
    ap.add_argument("--iters", type=int, default=2)
    ap.add_argument("--slices", type=int, default=7)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=2)
    a = ap.parse_args(argv)
    if a.what in ("stages", "eigvals", "adjoint", "overlap") and a.nk == 0:
        a.nk = 512 if a.M >= 8192 else 256
    fn = {"gemm": run_gemm, "i8gemm": run_i8gemm, "symm": run_symm, "syr2k": run_syr2k, "stages": run_stages,
          "refine": run_refine, "eigvals": run_eigvals, "adjoint": run_adjoint,
          "batched": run_batched, "mixed": run_mixed, "overlap": run_overlap}[a.what]
    print(json.dumps(fn(a)), flush=True)


if __name__ == "__main__":
    main()
