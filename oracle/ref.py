"""TEST INFRASTRUCTURE ONLY — the reference's own OpenCL kernels
(opencl/bmfr.cl) compiled for the CPU by g++ (oracle/ref_cl: prepare.py,
cl_compat.h, ref_runner.cpp) into oracle/_ref/libbmfr_ref.so.

`RefKernels` has the interface of `oracle.Oracle` (the same configuration,
buffers and method signatures), so `OraclePipeline(RefKernels(...))` runs the
reference host program's frame loop over the reference's kernels.  The tests
use it to pin the oracle restatement and to write the golden fixtures.

The library is built from the reference's source where it lies (`make -C
oracle ref REF_SRC=<opencl/bmfr.cl>`, or BMFR_REFERENCE_CL set in the
environment when this module loads it); without that source, only a library
built earlier can be used.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

from .oracle import Oracle, Cfg, _p, FITTER_REFERENCE

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
LIB = REF_DIR / "libbmfr_ref.so"
def _source() -> Path | None:
    """The reference's opencl/bmfr.cl named by BMFR_REFERENCE_CL, if it exists."""
    src = os.environ.get("BMFR_REFERENCE_CL")
    return Path(src) if src and Path(src).exists() else None


def available() -> bool:
    """True if the library exists or can be built from the reference source."""
    return LIB.exists() or _source() is not None


def build() -> Path:
    """Builds oracle/_ref/libbmfr_ref.so from the reference's kernel source."""
    src = _source()
    if src is None:
        raise FileNotFoundError("reference kernel source not found: set BMFR_REFERENCE_CL to its opencl/bmfr.cl")
    subprocess.run(["make", "-C", str(HERE), "ref", f"REF_SRC={src}"], check=True, capture_output=True)
    return LIB


_lib = None


def _load() -> C.CDLL:
    global _lib
    if _lib is None:
        if _source() is not None:
            build()          # make: a no-op when the library is current
        if not LIB.exists():
            raise FileNotFoundError(f"{LIB} is not built and the reference source is absent")
        lib = C.CDLL(str(LIB))
        vp = C.c_void_p
        cfg = C.POINTER(Cfg)
        lib.ref_accumulate_noisy_data.argtypes = [cfg] + [vp] * 13 + [C.c_int]
        lib.ref_fitter.argtypes = [cfg, vp, vp, vp, C.c_int]
        lib.ref_weighted_sum.argtypes = [cfg, vp, vp, vp, vp, vp, C.c_int]
        lib.ref_accumulate_filtered_data.argtypes = [cfg] + [vp] * 8 + [C.c_int]
        lib.ref_taa.argtypes = [cfg, vp, vp, vp, vp, C.c_int]
        for n in ("ref_accumulate_noisy_data", "ref_fitter", "ref_weighted_sum", "ref_accumulate_filtered_data",
                  "ref_taa"):
            getattr(lib, n).restype = C.c_int
        _lib = lib
    return _lib


class RefKernels(Oracle):
    """The reference's five kernels, run on the CPU, on host arrays."""

    def __init__(self, *args, **kwargs):
        super().__init__(*args, **kwargs)
        self.lib = _load()

    def accumulate_noisy_data(self, prev_pix, accept, cur_n, prev_n, cur_p, prev_p, cur_noisy, prev_noisy,
                              prev_spp, cur_spp, tmp, matrix, offset, frame):
        import numpy as np
        m = np.ascontiguousarray(matrix, dtype=np.float32)
        o = np.ascontiguousarray(offset, dtype=np.float32)
        rc = self.lib.ref_accumulate_noisy_data(C.byref(self.cfg), _p(prev_pix), _p(accept), _p(cur_n), _p(prev_n),
                                                _p(cur_p), _p(prev_p), _p(cur_noisy), _p(prev_noisy), _p(prev_spp),
                                                _p(cur_spp), _p(tmp), _p(m), _p(o), int(frame))
        assert rc == 0

    def fitter(self, weights, mins_maxs, tmp, frame, mode=FITTER_REFERENCE):
        if mode != FITTER_REFERENCE:
            raise ValueError("the reference has one fitter arithmetic")
        rc = self.lib.ref_fitter(C.byref(self.cfg), _p(weights), _p(mins_maxs), _p(tmp), int(frame))
        if rc != 0:
            raise RuntimeError("reference fitter: work-items of a group did not meet at the same barriers")

    def fitter_fp64(self, *a, **k):
        raise NotImplementedError("the reference has no FP64 fitter")

    def fitter_matrix(self, *a, **k):
        raise NotImplementedError("the reference has no least-squares matrix export")

    def weighted_sum(self, weights, mins_maxs, out, cur_n, cur_p, frame):
        assert self.lib.ref_weighted_sum(C.byref(self.cfg), _p(weights), _p(mins_maxs), _p(out), _p(cur_n),
                                         _p(cur_p), int(frame)) == 0

    def accumulate_filtered_data(self, filtered, prev_pix, accept, albedo, tone_mapped, cur_spp, acc_prev,
                                 acc_cur, frame):
        assert self.lib.ref_accumulate_filtered_data(C.byref(self.cfg), _p(filtered), _p(prev_pix), _p(accept),
                                                     _p(albedo), _p(tone_mapped), _p(cur_spp), _p(acc_prev),
                                                     _p(acc_cur), int(frame)) == 0

    def taa(self, prev_pix, new_frame, result, prev_result, frame):
        assert self.lib.ref_taa(C.byref(self.cfg), _p(prev_pix), _p(new_frame), _p(result), _p(prev_result),
                                int(frame)) == 0
