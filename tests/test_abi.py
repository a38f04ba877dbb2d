"""The C ABI library loads and exports everything include/*.h declares (CPU only, no compute)."""
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HDR = ROOT / "include" / "cuev_b200.h"
LIB = ROOT / "cuev_b200" / "libcuev_b200.so"

# mangled names of the reference's explicit instantiations (src/cuda/solver.cu:78-79)
MANGLED = ["_ZN4cuev14symm_eig_solveIdEEvPT_iS2_S2_P11CUstream_stPNS_10SolveTimerE",
           "_ZN4cuev14symm_eig_solveIfEEvPT_iS2_S2_P11CUstream_stPNS_10SolveTimerE"]


def declared_c_functions():
    text = HDR.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cuev_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    if not LIB.exists():
        from cuev_b200 import build
        build.build()
    import cuev_b200
    return cuev_b200.lib()


def test_every_declared_symbol_is_exported(lib):
    names = declared_c_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_cpp_dropin_symbols_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB)], capture_output=True,
                         text=True, check=True).stdout
    for m in MANGLED:
        assert m in out, m


def test_cpp_dropin_links(tmp_path):
    """A program written against the reference's API compiles against include/cuev.h and links
    against libcuev_b200.so unchanged (it is not run: no GPU here)."""
    src = tmp_path / "user.cpp"
    src.write_text(
        '#include "cuev.h"\n'
        "int main() {\n"
        "  double *A = nullptr, *w = nullptr, *V = nullptr; cuev::SolveTimer t;\n"
        "  if (A) cuev::symm_eig_solve<double>(A, 0, w, V, (cudaStream_t)0, &t);\n"
        "  float *a = nullptr; if (a) cuev::symm_eig_solve<float>(a, 0, a, a, 0);\n"
        "  return 0;\n}\n")
    exe = tmp_path / "user"
    r = subprocess.run(["g++", "-std=c++17", "-I", str(ROOT / "include"),
                        "-I", "/usr/local/cuda/include", str(src), "-o", str(exe),
                        "-L", str(LIB.parent), "-lcuev_b200",
                        f"-Wl,-rpath,{LIB.parent}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_last_error_without_gpu(lib):
    # argument validation happens before any CUDA call
    assert lib.cuev_dsyevd(None, -1, None, None, None, None) == -1
    assert lib.cuev_handle_create(16, 48, 96, None, None) == -1
    assert isinstance(lib.cuev_last_error(), bytes)
