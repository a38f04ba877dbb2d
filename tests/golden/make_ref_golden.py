"""Generate golden outputs by running the reference solver itself (built from its sources by
oracle/ref/Makefile into oracle/_ref/) on seeded inputs.  Runs on a GPU machine; writes
  tests/golden/ref_eig_n{n}.npz   eval (and evec for n=256) of A = (G + G^T)/2, G from
                                  numpy default_rng(n).standard_normal((n, n))
  tests/golden/ref_eval_n{n}.npz  eval only, same input, at the large sizes (--eval-sizes)
  <out>/ref_timings.jsonl         the reference's SolveTimer per size
Usage: python tests/golden/make_ref_golden.py [--out DIR] [--golden-sizes ...]
                                              [--eval-sizes 8192,16384] [--timing-sizes ...]
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
DRIVER = ROOT / "oracle" / "_ref" / "ref_driver"


def sym_input(n: int) -> np.ndarray:
    G = np.random.default_rng(n).standard_normal((n, n))
    return (G + G.T) / 2


def run_ref(A: np.ndarray, want_vec: bool, timeout: int):
    n = A.shape[0]
    with tempfile.TemporaryDirectory() as td:
        fin, fw, fv = (os.path.join(td, x) for x in ("A.bin", "w.bin", "V.bin"))
        np.asfortranarray(A).ravel(order="F").tofile(fin)
        cmd = [str(DRIVER), str(n), fin, fw, fv if want_vec else "-"]
        res = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
        if res.returncode != 0:
            raise RuntimeError(f"reference failed (n={n}): {res.stderr[-500:]}")
        timer = json.loads(res.stdout.strip().splitlines()[-1])
        w = np.fromfile(fw, dtype=np.float64)
        V = np.fromfile(fv, dtype=np.float64).reshape((n, n)).T if want_vec else None
        return w, V, timer


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(ROOT / "tests" / "golden"))
    ap.add_argument("--golden-sizes", default="256,512,1024")
    ap.add_argument("--eval-sizes", default="8192,16384")
    ap.add_argument("--timing-sizes", default="")
    ap.add_argument("--timeout", type=int, default=600)
    args = ap.parse_args()
    out = Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    for n in [int(x) for x in args.golden_sizes.split(",") if x]:
        A = sym_input(n)
        w, V, timer = run_ref(A, True, args.timeout)
        payload = {"n": n, "eval": w, "seed": n}
        if n <= 256:
            payload["evec"] = V
        else:  # 16 columns of the eigenvector matrix, spread over the spectrum
            cols = np.linspace(0, n - 1, 16).astype(int)
            payload["evec_cols"] = cols
            payload["evec_sample"] = V[:, cols]
        np.savez_compressed(out / f"ref_eig_n{n}.npz", **payload)
        print(json.dumps({"golden": n, **timer}), flush=True)
    for n in [int(x) for x in args.eval_sizes.split(",") if x]:
        A = sym_input(n)
        w, _, timer = run_ref(A, False, args.timeout)
        np.savez_compressed(out / f"ref_eval_n{n}.npz", n=n, eval=w, seed=n)
        print(json.dumps({"golden_eval": n, **timer}), flush=True)
    with open(out / "ref_timings.jsonl", "a") as fh:
        for n in [int(x) for x in args.timing_sizes.split(",") if x]:
            A = sym_input(n)
            try:
                w, _, timer = run_ref(A, False, args.timeout)
                timer["impl"] = "reference (oracle/_ref, GPU + host LAPACK D&C)"
            except Exception as exc:  # noqa: BLE001
                timer = {"n": n, "error": str(exc)[:300]}
            fh.write(json.dumps(timer) + "\n")
            print(json.dumps(timer), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
