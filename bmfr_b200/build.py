"""Build recipe of the in-tree native library bmfr_b200/libbmfr_b200.so.

CUDA sources are compiled by nvcc for sm_100a only
(-gencode arch=compute_100a,code=sm_100a); host C++ sources by the system
g++ with OpenMP.  Objects go to bmfr_b200/_build/ and are rebuilt when a
source or header is newer.  Run ``python bmfr_b200/build.py``.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
INCLUDE = ROOT / "include"
LIB = PKG / "libbmfr_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build bmfr_b200")


def _gxx() -> str:
    # The system compiler carries the OpenMP runtime spec.
    return "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"


NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC",
                     "-Xptxas", "-warn-spills", f"-I{INCLUDE}", f"-I{CSRC}"]
GXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", f"-I{INCLUDE}", f"-I{CSRC}"]


def _headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h")))


def _stale(obj: Path, src: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(p.stat().st_mtime > t for p in [src, *deps])


def _compile(src: Path, verbose: bool) -> Path:
    obj = BUILD / (src.name + ".o")
    if not _stale(obj, src, _headers()):
        return obj
    if src.suffix == ".cu":
        cmd = [_nvcc(), "-ccbin", _gxx(), *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
    else:
        cmd = [_gxx(), *GXX_FLAGS, "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compiling {src.name} failed:\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False) -> Path:
    """Compiles and links libbmfr_b200.so; returns its path."""
    BUILD.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), sources))
    if not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [_nvcc(), "-ccbin", _gxx(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs),
               "-Xcompiler", "-fopenmp", "-lgomp", "-cudart", "static"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"linking {LIB.name} failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def build_oracle(verbose: bool = False) -> Path:
    """Builds the CPU oracle (test infrastructure) with its Makefile."""
    oracle = ROOT / "oracle"
    r = subprocess.run(["make", "-C", str(oracle)], capture_output=True, text=True)
    if verbose:
        print(r.stdout, r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"building the oracle failed:\n{r.stdout}\n{r.stderr}")
    return oracle / "libbmfr_oracle.so"


REFERENCE_CL = Path("/root/reference/opencl/bmfr.cl")


def build_reference(verbose: bool = False) -> Path | None:
    """Compiles the reference's own kernels for the CPU (test
    infrastructure: oracle/ref_cl -> oracle/_ref/libbmfr_ref.so) when the
    reference source is present; otherwise keeps a library built earlier."""
    oracle = ROOT / "oracle"
    if not REFERENCE_CL.exists():
        lib = oracle / "_ref" / "libbmfr_ref.so"
        return lib if lib.exists() else None
    r = subprocess.run(["make", "-C", str(oracle), "ref", f"REF_SRC={REFERENCE_CL}", f"PYTHON={sys.executable}"],
                       capture_output=True, text=True)
    if verbose:
        print(r.stdout, r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"building the reference kernels failed:\n{r.stdout}\n{r.stderr}")
    return oracle / "_ref" / "libbmfr_ref.so"


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
    print(build_oracle(verbose="-v" in sys.argv))
    print(build_reference(verbose="-v" in sys.argv))
