"""Build recipe of the in-tree native libraries: bmfr_b200/libbmfr_b200.so
(the denoising pipeline) and bmfr_scene/libbmfr_scene.so (the procedural
input source, kept apart so that code that only needs inputs maps no
pipeline code).

CUDA sources are compiled by nvcc for sm_100a only
(-gencode arch=compute_100a,code=sm_100a); host C++ sources by the system
g++ with OpenMP.  Objects go to each package's _build/ and are rebuilt when
a source or header is newer.  Run ``python bmfr_b200/build.py``.
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
SCENE_PKG = ROOT / "bmfr_scene"
SCENE_LIB = SCENE_PKG / "libbmfr_scene.so"

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
                     "-Xptxas", "-warn-spills", f"-I{INCLUDE}"]
GXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", f"-I{INCLUDE}"]


def _headers(csrc: Path) -> list[Path]:
    return sorted(list(csrc.glob("*.cuh")) + list(csrc.glob("*.h")) + list(INCLUDE.glob("*.h")))


def _stale(obj: Path, src: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(p.stat().st_mtime > t for p in [src, *deps])


def _compile(src: Path, build: Path, verbose: bool) -> Path:
    csrc = src.parent
    obj = build / (src.name + ".o")
    if not _stale(obj, src, _headers(csrc)):
        return obj
    if src.suffix == ".cu":
        cmd = [_nvcc(), "-ccbin", _gxx(), *NVCC_FLAGS, f"-I{csrc}", "-c", str(src), "-o", str(obj)]
    else:
        cmd = [_gxx(), *GXX_FLAGS, f"-I{csrc}", "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compiling {src.name} failed:\n{r.stdout}\n{r.stderr}")
    return obj


def _build_lib(csrc: Path, build: Path, lib: Path, verbose: bool) -> Path:
    build.mkdir(exist_ok=True)
    sources = sorted(csrc.glob("*.cu")) + sorted(csrc.glob("*.cpp"))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, build, verbose), sources))
    if not lib.exists() or any(o.stat().st_mtime > lib.stat().st_mtime for o in objs):
        cmd = [_nvcc(), "-ccbin", _gxx(), *ARCH, "-shared", "-o", str(lib), *map(str, objs),
               "-Xcompiler", "-fopenmp", "-lgomp", "-cudart", "static"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"linking {lib.name} failed:\n{r.stdout}\n{r.stderr}")
    return lib


def build(verbose: bool = False) -> Path:
    """Compiles and links libbmfr_b200.so and libbmfr_scene.so; returns the
    pipeline library's path."""
    _build_lib(SCENE_PKG / "csrc", SCENE_PKG / "_build", SCENE_LIB, verbose)
    return _build_lib(CSRC, BUILD, LIB, verbose)


def build_oracle(verbose: bool = False) -> Path:
    """Builds the CPU oracle (test infrastructure) with its Makefile."""
    oracle = ROOT / "oracle"
    r = subprocess.run(["make", "-C", str(oracle)], capture_output=True, text=True)
    if verbose:
        print(r.stdout, r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"building the oracle failed:\n{r.stdout}\n{r.stderr}")
    return oracle / "libbmfr_oracle.so"


def build_reference(reference_cl: str | os.PathLike | None = None, verbose: bool = False) -> Path | None:
    """Compiles the reference's own kernels for the CPU (test
    infrastructure: oracle/ref_cl -> oracle/_ref/libbmfr_ref.so) from the
    reference's opencl/bmfr.cl, given as `reference_cl` or by the
    environment variable BMFR_REFERENCE_CL; without that source, keeps a
    library built earlier."""
    oracle = ROOT / "oracle"
    src = reference_cl or os.environ.get("BMFR_REFERENCE_CL")
    if not src or not Path(src).exists():
        lib = oracle / "_ref" / "libbmfr_ref.so"
        return lib if lib.exists() else None
    r = subprocess.run(["make", "-C", str(oracle), "ref", f"REF_SRC={src}", f"PYTHON={sys.executable}"],
                       capture_output=True, text=True)
    if verbose:
        print(r.stdout, r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"building the reference kernels failed:\n{r.stdout}\n{r.stderr}")
    return oracle / "_ref" / "libbmfr_ref.so"


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
    print(build_oracle(verbose="-v" in sys.argv))
    print(build_reference(verbose="-v" in sys.argv))   # with BMFR_REFERENCE_CL set
