#!/usr/bin/env python
"""Benchmark: dense symmetric eigensolve (all eigenvalues + eigenvectors) on B200.

One "step" is one full solve of an n x n FP64 matrix A = (G + G^T)/2, G iid N(0, 1) from a seed,
through cuev_b200 (DBBR -> pack -> bulge chase -> GPU D&C -> back-transform).  The headline
workload is n = 16384, the size the reference's headline throughput is quoted on; the matrix
(2.1 GB) is far larger than the 126 MB L2, so no flush is needed between steps.

Reported (one JSON line on rank 0):
  value      whole-job TFLOP/s = world x steps x 6.67 n^3 / (max over ranks of device time)
             (work model: DBBR 4/3 n^3 + D&C <= 4/3 n^3 + back-transform 4 n^3)
  e2e        the same metric through the C ABI with HOST buffers (cuev_dsyevd_host): every step
             copies A from pinned host memory, solves, and copies eval + evec back (the finished
             eigenvector columns leave while the last columns' back-transform runs)
  roofline   the bulge-chasing back-transform kernel (2 n^3 FLOP over its column-range launches,
             timed from the first start to the last end) against the FP64 peak measured in the
             same run (cuBLAS DGEMM 8192^3)
  cpu_baseline  the oracle (CPU restatement of the reference pipeline) on a bounded sample
  stage_roofline  per-stage throughput against the same FP64 peak (DBBR, chase L2 model, D&C
             merge flops counted on the device, back-transform) and the whole solve's fraction
  mixed_refine  the precision form (cuev_dsyevd_mixed) on the same matrix: time, speed-up over
             the FP64 form, refinement steps and accuracy (outside the headline's timed region)
  fwd_bwd    forward solve + adjoint (cuev_dsyev_adjoint) at n and at 4096
  fp32_entry  the FP32 entry (cuev_ssyevd, BC-back in FP32) on the same matrix rounded to FP32:
             time, speed-up over the FP64 form, stage times and accuracy
The reference arm (--impl reference) runs the reference built from its own sources
(oracle/_ref/ref_driver) on the same matrix, steps and warm-up where that build and a GPU exist,
else the oracle port on a bounded CPU sample.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuev|reference] [--n N]
Multi-GPU (replicas only: every rank solves its own matrix; no collective on the data path):
  python -m torch.distributed.run --nproc-per-node N --master-addr 127.0.0.1 bench.py --gpus N
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import tempfile
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FLOP_MODEL = 20.0 / 3.0  # (4/3 + 4/3 + 4) n^3 per solve


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def metric_name(n):
    return f"eigh n={n} FP64 (all eigenpairs), TFLOP/s at 6.67 n^3 per solve"


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Max of a per-rank timing over all ranks (replicas: the job ends with the slowest)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_tflops(world: int, steps: int, n: int, total_ms: float) -> float:
    """Aggregate throughput of `world` replicas each doing `steps` solves of size n."""
    return world * steps * FLOP_MODEL * n ** 3 / (total_ms * 1e-3) / 1e12


# ------------------------------------------------------------------------------------------
# clocks sampled during the timed region
# ------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu_index = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, name = tempfile.mkstemp(prefix=f"cuev_clocks_gpu{self.gpu_index}_", suffix=".csv")
            self.path = Path(name)
            self.fh = os.fdopen(fd, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.gpu_index), "-lms", "200"], stdout=self.fh,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------------------------------
# CPU baseline: the oracle (CPU restatement of the reference pipeline)
# ------------------------------------------------------------------------------------------
def cpu_oracle_sample(n_cpu: int, repeats: int = 1):
    import numpy as np
    from oracle import cuev_oracle as O  # checker / CPU arm only
    O.build()
    rng = np.random.default_rng(4321)
    G = rng.standard_normal((n_cpu, n_cpu))
    A = np.asfortranarray((G + G.T) / 2)
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        O.symm_eig_solve(A, 32, 256)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    return FLOP_MODEL * n_cpu ** 3 / t / 1e12, t


def lapack_dsyevd_sample(n_cpu: int):
    import numpy as np
    import scipy.linalg as sla
    rng = np.random.default_rng(4321)
    G = rng.standard_normal((n_cpu, n_cpu))
    A = (G + G.T) / 2
    t0 = time.perf_counter()
    sla.eigh(A, driver="evd")
    t = time.perf_counter() - t0
    return FLOP_MODEL * n_cpu ** 3 / t / 1e12, t


def _bench_matrix(n: int, dev, seed: int):
    """The bench's input, A = (G + G^T)/2 with G from torch's generator on the device (both arms
    use the same seed, hence the same matrix)."""
    import torch
    g = torch.Generator(device=dev).manual_seed(seed)
    A0 = torch.randn(n, n, dtype=torch.float64, device=dev, generator=g)
    return ((A0 + A0.t()) * 0.5).contiguous()


def run_reference_driver(args, driver: Path):
    """The reference's own build (oracle/_ref/ref_driver: the reference's sources compiled
    unmodified; GPU stages plus its host LAPACK divide and conquer) on the bench's matrix: each
    step copies A from pinned host memory, calls cuev::symm_eig_solve<double> and copies eval and
    evec back."""
    import torch
    n = args.n
    dev = torch.device("cuda", 0)
    A0 = _bench_matrix(n, dev, 1234)
    shm = Path("/dev/shm")
    with tempfile.TemporaryDirectory(dir=str(shm) if shm.is_dir() else None) as td:
        fin = Path(td) / "A.bin"
        A0.cpu().numpy().tofile(fin)  # symmetric: row-major bytes are its column-major storage
        del A0
        torch.cuda.empty_cache()
        res = subprocess.run([str(driver), str(n), str(fin), "-", "-", str(args.steps),
                              str(args.warmup)], capture_output=True, text=True,
                             timeout=60 + 120 * (args.steps + args.warmup))
    if res.returncode != 0:
        raise RuntimeError(f"reference driver failed: {res.stderr[-400:]}")
    recs = [json.loads(x) for x in res.stdout.splitlines() if x.startswith("{")]
    solve = statistics.median(r["solve_ms"] for r in recs)
    e2e = statistics.median(r["e2e_ms"] for r in recs)
    stages = {k: round(statistics.median(r[k] for r in recs), 3)
              for k in ("dbbr_ms", "bc_ms", "dc_ms", "bt_ms")}
    return solve, e2e, stages, len(recs)


def run_reference(args, rank, world):
    """The reference arm.  Where the reference built here from its own sources exists
    (oracle/_ref/ref_driver) and a GPU is present, that build runs the bench's own workload
    (same n, same matrix, same steps and warm-up).  Otherwise the reference pipeline restated on
    the host cores (the oracle port) runs a bounded sample."""
    if rank != 0:
        return 0
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    driver = ROOT / "oracle" / "_ref" / "ref_driver"
    have_gpu = False
    try:
        import torch
        have_gpu = torch.cuda.is_available()
    except Exception:
        pass
    base = {"impl": "reference", "metric": metric_name(args.n), "unit": "TFLOP/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic"}
    if driver.exists() and have_gpu:
        n = args.n
        solve_ms, e2e_ms, stages, cnt = run_reference_driver(args, driver)
        value = FLOP_MODEL * n ** 3 / (solve_ms * 1e-3) / 1e12
        line = dict(base)
        line.update({
            "value": round(value, 6), "ms_per_step": round(solve_ms, 3),
            "config": {"workload": f"eigh n={n}: A=(G+G^T)/2, G iid N(0,1), FP64, all "
                                   "eigenvalues and eigenvectors (the same matrix as the cuev "
                                   "arm)", "n": n, "nbw": 32, "nk": 512},
            "stage_ms": stages,
            "cpu_baseline": {"value": round(value, 6), "unit": "TFLOP/s", "cores": cores,
                             "kind": "reference",
                             "sample": f"the reference built from its own sources "
                                       f"(oracle/_ref/ref_driver) at n={n}, {cnt} timed solves "
                                       "after the warm-up: its GPU stages plus its host LAPACK "
                                       f"divide and conquer (OpenMP, up to {cores} host threads)"},
            "e2e": {"value": round(FLOP_MODEL * n ** 3 / (e2e_ms * 1e-3) / 1e12, 6),
                    "unit": "TFLOP/s", "h2d_bytes_per_step": 8 * n * n,
                    "d2h_bytes_per_step": 8 * n * n + 8 * n, "ms_per_step": round(e2e_ms, 3)},
        })
        print(json.dumps(line), flush=True)
        return 0
    n_cpu = args.cpu_n
    for _ in range(args.warmup):
        cpu_oracle_sample(n_cpu)
    vals, secs = [], []
    for _ in range(args.steps):
        v, t = cpu_oracle_sample(n_cpu)
        vals.append(v)
        secs.append(t)
    value = statistics.median(vals)
    line = dict(base)
    line.update({
        "value": round(value, 6), "ms_per_step": round(1000 * statistics.median(secs), 3),
        "config": {"workload": f"eigh A=(G+G^T)/2, G iid N(0,1); bounded CPU sample n={n_cpu}",
                   "n": args.n, "sample_n": n_cpu},
        "cpu_baseline": {"value": round(value, 6), "unit": "TFLOP/s", "cores": cores,
                         "kind": "port",
                         "sample": f"one full oracle solve at n={n_cpu} per step (median of "
                                   f"{args.steps}); BLAS calls use all {cores} host threads, "
                                   "bulge chase and LAPACK D&C pieces run sequentially"},
        "e2e": {"value": round(value, 6), "unit": "TFLOP/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    })
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------------------------
# the GPU arm
# ------------------------------------------------------------------------------------------
def run_cuev(args, rank, world, local_rank):
    import ctypes as C

    import torch
    import cuev_b200 as cv

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
    n = args.n
    lib = cv.lib()
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream

    # input: A = (G + G^T)/2 (symmetric, so column-major storage == row-major storage)
    A0 = _bench_matrix(n, dev, 1234 + rank)
    A = torch.empty_like(A0)
    w = torch.empty(n, dtype=torch.float64, device=dev)
    V = torch.empty_like(A0)
    cfg = cv.Config(args.nbw, args.nk)
    timer = cv.Timer()

    def solve():
        st = lib.cuev_dsyevd_cfg(A.data_ptr(), n, w.data_ptr(), V.data_ptr(), sp, C.byref(timer),
                                 C.byref(cfg))
        if st != 0:
            raise RuntimeError(f"cuev_dsyevd failed: {st} {lib.cuev_last_error().decode()}")

    for _ in range(max(3, args.warmup)):
        A.copy_(A0)
        solve()
    torch.cuda.synchronize()

    # FP64 peak reference measured in this run: cuBLAS DGEMM 8192^3
    a = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    torch.matmul(a, a)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 1e30
    for _ in range(3):
        e0.record()
        torch.matmul(a, a)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    fp64_peak = 2 * 8192 ** 3 / (best * 1e-3) / 1e12
    del a
    torch.cuda.empty_cache()

    # ---- timed region
    gpu_index = local_rank
    cvd = os.environ.get("CUDA_VISIBLE_DEVICES")
    if cvd:
        ids = [x for x in cvd.split(",") if x.strip()]
        if local_rank < len(ids) and ids[local_rank].strip().isdigit():
            gpu_index = int(ids[local_rank])
    clocks = ClockSampler(gpu_index)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    launches0 = lib.cuev_kernel_launches()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    stage = {"dbbr_ms": [], "bc_ms": [], "dc_ms": [], "bt_qb_ms": [], "bt_qs_ms": []}
    dc_flops = 0.0
    for i in range(args.steps):
        A.copy_(A0)  # restore the (overwritten) input outside the timed pair
        ev[i][0].record(stream)
        solve()
        ev[i][1].record(stream)
        for k2 in stage:
            stage[k2].append(getattr(timer, k2))
        dc_flops = lib.cuev_last_dc_flops()
    torch.cuda.synchronize()
    launches = lib.cuev_kernel_launches() - launches0
    clk = clocks.stop()
    total_ms = max_over_ranks(sum(e0_.elapsed_time(e1_) for e0_, e1_ in ev), dist, dev)
    ms_per = total_ms / args.steps
    value = whole_job_tflops(world, args.steps, n, total_ms)

    # accuracy of the last solve (device, cuBLAS): ||AV - VL||_F / (n ||A||_2), ||V^T V - I||_F
    with torch.no_grad():
        Vl = V.t()  # column-major storage -> logical matrix
        R = A0 @ Vl - Vl * w[None, :]
        anorm = w.abs().max()
        resid = float(torch.linalg.norm(R) / (n * anorm))
        resid_ref = float(torch.linalg.norm(R) / torch.linalg.norm(A0))
        del R
        O_ = Vl.t() @ Vl
        O_.diagonal().sub_(1.0)
        orth = float(torch.linalg.norm(O_))
        del O_
        torch.cuda.empty_cache()

    # ---- end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        hA = torch.empty(n * n, dtype=torch.float64, pin_memory=True)
        hA.copy_(A0.reshape(-1).cpu())
        hw = torch.empty(n, dtype=torch.float64, pin_memory=True)
        hV = torch.empty(n * n, dtype=torch.float64, pin_memory=True)
        steps_e2e = max(1, min(args.steps, 2))

        def solve_host():
            # cuev_dsyevd_host: copy in, solve, eigenvectors copied out as they become final
            st = lib.cuev_dsyevd_host(hA.data_ptr(), n, hw.data_ptr(), hV.data_ptr(), sp, None)
            if st != 0:
                raise RuntimeError(f"cuev_dsyevd_host failed: {st} "
                                   f"{lib.cuev_last_error().decode()}")

        solve_host()  # warm-up: the entry's device buffers are kept between calls
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        tot = 0.0
        for _ in range(steps_e2e):
            x0, x1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            x0.record(stream)
            solve_host()
            x1.record(stream)
            torch.cuda.synchronize()
            tot += x0.elapsed_time(x1)
        tot = max_over_ranks(tot, dist, dev)
        e2e = {"value": round(whole_job_tflops(world, steps_e2e, n, tot), 4),
               "unit": "TFLOP/s", "h2d_bytes_per_step": 8 * n * n,
               "d2h_bytes_per_step": 8 * n * n + 8 * n,
               "ms_per_step": round(tot / steps_e2e, 3)}

    # ---- precision form on the same matrix (outside the headline's timed region)
    mixed = None
    if not args.no_mixed:
        minfo = cv.MixedInfo()
        mtimer = cv.Timer()

        def solve_mixed():
            st = lib.cuev_dsyevd_mixed(A.data_ptr(), n, w.data_ptr(), V.data_ptr(), sp,
                                       C.byref(mtimer), args.mixed_iters, 0.0, C.byref(minfo))
            if st != 0:
                raise RuntimeError(f"cuev_dsyevd_mixed failed: {st} "
                                   f"{lib.cuev_last_error().decode()}")

        w64 = w.clone()  # FP64-form eigenvalues of the same matrix
        A.copy_(A0)
        solve_mixed()  # warm-up (allocates the precision form's buffers once)
        mts, parts = [], []
        for _ in range(max(1, min(args.steps, 3))):
            A.copy_(A0)
            m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            m0.record(stream)
            solve_mixed()
            m1.record(stream)
            torch.cuda.synchronize()
            mts.append(m0.elapsed_time(m1))
            parts.append((minfo.first_ms, minfo.refine_ms))
        mms = max_over_ranks(statistics.median(mts), dist, dev)
        with torch.no_grad():
            Vl = V.t()
            R = A0 @ Vl - Vl * w[None, :]
            m_resid = float(torch.linalg.norm(R) / (n * w.abs().max()))
            del R
            O_ = Vl.t() @ Vl
            O_.diagonal().sub_(1.0)
            m_orth = float(torch.linalg.norm(O_))
            del O_
            m_dl = float((w - w64).abs().max() / w64.abs().max())
            torch.cuda.empty_cache()
        mixed = {"form": "first solve with the SBR-back GEMMs on FP32-level int8 tensor-core "
                         f"products, then {args.mixed_iters} Ogita-Aishima step(s) with "
                         "FP64-level int8 tensor-core products (cuev_dsyevd_mixed)",
                 "ms_per_step": round(mms, 3),
                 "value": round(whole_job_tflops(world, 1, n, mms), 4),
                 "speedup_vs_fp64": round(ms_per / mms, 3),
                 "first_ms": round(statistics.median(p_[0] for p_ in parts), 2),
                 "refine_ms": round(statistics.median(p_[1] for p_ in parts), 2),
                 "refine_iterations": int(minfo.refine_iterations),
                 "first_stage_ms": {k2: round(getattr(mtimer, k2), 2)
                                    for k2 in ("dbbr_ms", "bc_ms", "dc_ms", "bt_qb_ms",
                                               "bt_qs_ms")},
                 "accuracy": {"resid_n_norm2": m_resid, "orth_fro": m_orth,
                              "max_dlambda_vs_fp64_rel": m_dl}}

    # ---- FP32 entry (cuev_ssyevd) on the same matrix rounded to FP32
    fp32 = None
    if not args.no_fp32:
        A32 = A0.to(torch.float32)
        Aw = torch.empty_like(A32)
        w32 = torch.empty(n, dtype=torch.float32, device=dev)
        V32 = torch.empty_like(A32)
        ftimer = cv.Timer()
        fts, fparts = [], []
        for r_ in range(1 + max(1, min(args.steps, 3))):  # the first run is a warm-up
            Aw.copy_(A32)
            f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            f0.record(stream)
            st = lib.cuev_ssyevd(Aw.data_ptr(), n, w32.data_ptr(), V32.data_ptr(), sp,
                                 C.byref(ftimer))
            f1.record(stream)
            torch.cuda.synchronize()
            if st != 0:
                raise RuntimeError(f"cuev_ssyevd failed: {st} {lib.cuev_last_error().decode()}")
            if r_ >= 1:
                fts.append(f0.elapsed_time(f1))
                fparts.append({k2: getattr(ftimer, k2) for k2 in ("dbbr_ms", "bc_ms", "dc_ms",
                                                                   "bt_ms")})
        fms = max_over_ranks(statistics.median(fts), dist, dev)
        with torch.no_grad():
            A64 = A32.to(torch.float64)
            Vl = V32.t().to(torch.float64)
            wl = w32.to(torch.float64)
            R = A64 @ Vl - Vl * wl[None, :]
            f_resid = float(torch.linalg.norm(R) / torch.linalg.norm(A64))
            del R
            O_ = Vl.t() @ Vl
            O_.diagonal().sub_(1.0)
            f_orth = float(torch.linalg.norm(O_) / n ** 0.5)
            del O_, Vl, A64
            torch.cuda.empty_cache()
        fp32 = {"form": "cuev_ssyevd: FP64 band reduction, chase and D&C; BC-back in FP32; "
                        "SBR-back on FP32-level int8 tensor-core products",
                "ms_per_step": round(fms, 3),
                "speedup_vs_fp64": round(ms_per / fms, 3),
                "stage_ms": {k2: round(statistics.median(p_[k2] for p_ in fparts), 2)
                             for k2 in ("dbbr_ms", "bc_ms", "dc_ms", "bt_ms")},
                "accuracy": {"resid_fro_rel": f_resid, "orth_fro_per_sqrt_n": f_orth}}
        del A32, Aw, V32, w32

    # ---- differentiation form: forward solve + adjoint (backward), at n and at 4096
    fwd_bwd = None
    if not args.no_adjoint:
        def fb(nn_, A0_):
            A_ = torch.empty_like(A0_)
            w_ = torch.empty(nn_, dtype=torch.float64, device=dev)
            V_ = torch.empty_like(A0_)
            gw = torch.randn(nn_, dtype=torch.float64, device=dev,
                             generator=torch.Generator(device=dev).manual_seed(8))
            gV = torch.randn(nn_, nn_, dtype=torch.float64, device=dev,
                             generator=torch.Generator(device=dev).manual_seed(9))
            Ab = torch.empty_like(A0_)
            fwds, bwds = [], []
            for r_ in range(3):
                A_.copy_(A0_)
                e_ = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
                e_[0].record(stream)
                st = lib.cuev_dsyevd(A_.data_ptr(), nn_, w_.data_ptr(), V_.data_ptr(), sp, None)
                e_[1].record(stream)
                st2 = lib.cuev_dsyev_adjoint(V_.data_ptr(), w_.data_ptr(), gV.data_ptr(),
                                             gw.data_ptr(), nn_, C.c_double(1e-12),
                                             Ab.data_ptr(), sp)
                e_[2].record(stream)
                torch.cuda.synchronize()
                if st or st2:
                    raise RuntimeError(f"fwd/bwd failed: {st} {st2}")
                if r_ >= 1:
                    fwds.append(e_[0].elapsed_time(e_[1]))
                    bwds.append(e_[1].elapsed_time(e_[2]))
            f_, b_ = statistics.median(fwds), statistics.median(bwds)
            del A_, V_, gV, Ab
            torch.cuda.empty_cache()
            return {"fwd_ms": round(f_, 3), "bwd_ms": round(b_, 3),
                    "fwd_bwd_ms": round(f_ + b_, 3),
                    "bwd_tflops": round(6.0 * nn_ ** 3 / (b_ * 1e-3) / 1e12, 3)}
        fwd_bwd = {str(n): fb(n, A0)}
        if n != 4096:
            fwd_bwd["4096"] = fb(4096, _bench_matrix(4096, dev, 4096))

    med = {k2: statistics.median(v) for k2, v in stage.items()}
    bcb_ms = med["bt_qb_ms"]
    bcb_flops = 2.0 * n ** 3
    achieved = bcb_flops / (bcb_ms * 1e-3) / 1e12
    traffic = None
    tfile = ROOT / "profiles" / "bc_back_traffic.json"
    if tfile.exists():
        try:
            tj = json.loads(tfile.read_text())
            # DRAM bytes per launch grow as n^3: the round-to-round hand-off buffer (n x n) is
            # written and read once per round of 8 sweep tiles (n / 112 rounds); M itself is
            # read and written once (n^2).  Scaled from one ncu capture at a smaller n.
            traffic = int(tj["dram_bytes"] * (n / tj["n"]) ** 3)
        except Exception:
            traffic = None
    # per-stage figures (algorithmic work / stage time; FP64 peak measured in this run)
    bq = med["bt_qb_ms"] + med["bt_qs_ms"]
    stage_rf = {
        "dbbr": {"tflops": round((4.0 / 3.0) * n ** 3 / (med["dbbr_ms"] * 1e-3) / 1e12, 3)},
        "bulge_chase": {"l2_gbs_model": round(48.0 * n * n * 32 / (med["bc_ms"] * 1e-3) / 1e9, 1),
                        "note": "48 n^2 b bytes (the 2b x 3b window read and written per hop), "
                                "b = 32; latency bound (per sweep two hops and a reflector on the critical path)"},
        "divide_and_conquer": {"tflops": round(dc_flops / (med["dc_ms"] * 1e-3) / 1e12, 3),
                               "merge_gflop": round(dc_flops / 1e9, 1),
                               "note": "merge GEMM flops counted on the device after deflation "
                                       "(cuev_last_dc_flops; 4/3 n^3 without deflation) over the "
                                       "whole D&C stage time"},
        "back_transform": {"tflops": round(4.0 * n ** 3 / (bq * 1e-3) / 1e12, 3),
                           "note": "BC-back 2 n^3 + SBR-back 2 n^3 over BC-back's wall time "
                                   "plus the SBR-back time after it"},
    }
    for v_ in stage_rf.values():
        if "tflops" in v_:
            v_["frac"] = round(v_["tflops"] / fp64_peak, 4)
    stage_rf["whole_solve_frac"] = round(value / world / fp64_peak, 4)
    roofline = {"kernel": "bc_back_pipe_kernel (M <- Q_b M)", "bound": "fp64_fma",
                "achieved": round(achieved, 3), "peak": round(fp64_peak, 3), "unit": "TFLOP/s",
                "frac": round(achieved / fp64_peak, 4), "traffic": traffic,
                "peak_source": "FP64: cuBLAS DGEMM 8192^3 measured in this run (no FP64 figure "
                               "in MEASURED_PEAKS.json); the kernel runs on the FP64 FMA pipe, "
                               "which on this part has the DMMA rate and is shared with it",
                "algorithmic_bytes_per_launch": int(8 * (2 * n * n + n * n // 2)),
                "algorithmic_flop_per_launch": bcb_flops}

    if rank == 0:
        cpu = None
        if not args.no_cpu:
            v_cpu, t_cpu = cpu_oracle_sample(args.cpu_n)
            v_lap, t_lap = lapack_dsyevd_sample(args.cpu_n)
            cpu = {"value": round(v_cpu, 6), "unit": "TFLOP/s", "cores": os.cpu_count(),
                   "kind": "port",
                   "sample": f"one oracle solve (reference pipeline on the CPU) at n={args.cpu_n}"
                             f": {t_cpu:.2f} s; BLAS calls threaded over the host cores, bulge "
                             "chase and LAPACK D&C pieces sequential",
                   "lapack_dsyevd": {"value": round(v_lap, 6), "unit": "TFLOP/s",
                                     "seconds": round(t_lap, 3), "n": args.cpu_n}}
        line = {
            "metric": metric_name(n), "value": round(value, 4), "unit": "TFLOP/s",
            "n_gpus": world, "steps": args.steps, "warmup": max(3, args.warmup),
            "ms_per_step": round(ms_per, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"eigh n={n}: A=(G+G^T)/2, G iid N(0,1), FP64 form, "
                                   "all eigenvalues and eigenvectors",
                       "n": n, "nbw": args.nbw or "default", "nk": args.nk or "default",
                       "parallelism": f"replicas x{world}",
                       "l2": "inputs (2.1 GB per matrix) exceed the 126 MB L2; no flush"},
            "stage_ms": {k2: round(v, 3) for k2, v in med.items()},
            "tflops_ref_convention": round(world * args.steps * (4.0 / 3.0) * n ** 3
                                           / (total_ms * 1e-3) / 1e12, 4),
            "accuracy": {"resid_n_norm2": resid, "resid_fro_rel": resid_ref, "orth_fro": orth},
            "gpu_launches": int(launches),
            "roofline": roofline,
            "stage_roofline": stage_rf,
            "mixed_refine": mixed,
            "fwd_bwd": fwd_bwd,
            "fp32_entry": fp32,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["cuev", "reference"], default="cuev")
    ap.add_argument("--n", type=int, default=16384)
    ap.add_argument("--nbw", type=int, default=0)
    ap.add_argument("--nk", type=int, default=0)
    ap.add_argument("--cpu-n", type=int, default=2048)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-fp32", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--mixed-iters", type=int, default=1)
    args = ap.parse_args(argv)
    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local_rank = _env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_cuev(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
