"""TEST INFRASTRUCTURE ONLY — numpy front end of the CPU oracle
(oracle/bmfr_oracle.cpp, a restatement of opencl/bmfr.cl).

Only tests, the smoke check and the CPU-baseline leg of bench.py use this
module, as the checker; the product never imports it.

Pinned to the reference itself: the reference's own kernels, compiled for
the CPU by oracle/ref_cl (oracle/ref.py), give bit-identical outputs on the
same inputs (tests/test_reference_pin.py, fixtures in tests/golden/).
"""
from __future__ import annotations

import ctypes as C
import time
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libbmfr_oracle.so"

FITTER_REFERENCE = 0
FITTER_FP32 = 1
FITTER_FP64 = 2


class Cfg(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("noise_amount", C.c_double),
                ("blend_alpha", C.c_float), ("second_blend_alpha", C.c_float), ("taa_blend_alpha", C.c_float),
                ("position_limit_squared", C.c_float), ("normal_limit_squared", C.c_float),
                ("use_half", C.c_int), ("threads", C.c_int)]


def _load() -> C.CDLL:
    if not LIB.exists():
        subprocess.run(["make", "-C", str(HERE)], check=True, capture_output=True)
    lib = C.CDLL(str(LIB))
    vp = C.c_void_p
    lib.orc_random.restype = C.c_float
    lib.orc_random.argtypes = [C.c_uint32]
    lib.orc_mirror.restype = C.c_int
    lib.orc_mirror.argtypes = [C.c_int, C.c_int]
    lib.orc_round_half.restype = C.c_float
    lib.orc_round_half.argtypes = [C.c_float]
    lib.orc_add_random.restype = C.c_float
    lib.orc_add_random.argtypes = [C.c_float, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double]
    lib.orc_sizes.argtypes = [C.POINTER(Cfg), C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lib.orc_accumulate_noisy_data.argtypes = [C.POINTER(Cfg)] + [vp] * 13 + [C.c_int]
    lib.orc_fitter.argtypes = [C.POINTER(Cfg), vp, vp, vp, C.c_int, C.c_int]
    lib.orc_fitter_fp64.argtypes = [C.POINTER(Cfg), vp, vp, vp, C.c_int]
    lib.orc_fitter_matrix.argtypes = [C.POINTER(Cfg), vp, C.c_int, vp]
    lib.orc_weighted_sum.argtypes = [C.POINTER(Cfg), vp, vp, vp, vp, vp, C.c_int]
    lib.orc_accumulate_filtered_data.argtypes = [C.POINTER(Cfg)] + [vp] * 8 + [C.c_int]
    lib.orc_taa.argtypes = [C.POINTER(Cfg), vp, vp, vp, vp, C.c_int]
    for n in ("orc_accumulate_noisy_data", "orc_fitter", "orc_fitter_fp64", "orc_fitter_matrix", "orc_weighted_sum",
              "orc_accumulate_filtered_data", "orc_taa", "orc_sizes"):
        getattr(lib, n).restype = None
    return lib


lib = _load()


def _p(a):
    return C.c_void_p(None) if a is None else C.c_void_p(a.ctypes.data)


class Oracle:
    """The reference's five kernels on host arrays (H, W, 3 float32 images)."""

    def __init__(self, width, height, position_limit_squared=0.01, normal_limit_squared=0.1, use_half=True,
                 noise_amount=1e-2, blend_alpha=0.2, second_blend_alpha=0.1, taa_blend_alpha=0.2, threads=0):
        self.cfg = Cfg(width, height, noise_amount, blend_alpha, second_blend_alpha, taa_blend_alpha,
                       position_limit_squared, normal_limit_squared, 1 if use_half else 0, threads)
        mw, mh, b = C.c_int(), C.c_int(), C.c_int()
        lib.orc_sizes(C.byref(self.cfg), C.byref(mw), C.byref(mh), C.byref(b))
        self.width, self.height = width, height
        self.margin_width, self.margin_height, self.blocks = mw.value, mh.value, b.value
        self.tmp_dtype = np.float16 if use_half else np.float32

    def new_tmp(self):
        return np.zeros(self.blocks * 13 * 1024, dtype=self.tmp_dtype)

    def accumulate_noisy_data(self, prev_pix, accept, cur_n, prev_n, cur_p, prev_p, cur_noisy, prev_noisy,
                              prev_spp, cur_spp, tmp, matrix, offset, frame):
        m = np.ascontiguousarray(matrix, dtype=np.float32)
        o = np.ascontiguousarray(offset, dtype=np.float32)
        lib.orc_accumulate_noisy_data(C.byref(self.cfg), _p(prev_pix), _p(accept), _p(cur_n), _p(prev_n),
                                      _p(cur_p), _p(prev_p), _p(cur_noisy), _p(prev_noisy), _p(prev_spp),
                                      _p(cur_spp), _p(tmp), _p(m), _p(o), int(frame))

    def fitter(self, weights, mins_maxs, tmp, frame, mode=FITTER_REFERENCE):
        lib.orc_fitter(C.byref(self.cfg), _p(weights), _p(mins_maxs), _p(tmp), int(frame), int(mode))

    def fitter_fp64(self, weights64, mins_maxs, tmp, frame):
        lib.orc_fitter_fp64(C.byref(self.cfg), _p(weights64), _p(mins_maxs), _p(tmp), int(frame))

    def fitter_matrix(self, tmp, frame):
        """Each block's least-squares system after scaling and noise, float64 (blocks, 13, 1024)."""
        out = np.empty((self.blocks, 13, 1024), dtype=np.float64)
        lib.orc_fitter_matrix(C.byref(self.cfg), _p(tmp), int(frame), _p(out))
        return out

    def weighted_sum(self, weights, mins_maxs, out, cur_n, cur_p, frame):
        lib.orc_weighted_sum(C.byref(self.cfg), _p(weights), _p(mins_maxs), _p(out), _p(cur_n), _p(cur_p),
                             int(frame))

    def accumulate_filtered_data(self, filtered, prev_pix, accept, albedo, tone_mapped, cur_spp, acc_prev,
                                 acc_cur, frame):
        lib.orc_accumulate_filtered_data(C.byref(self.cfg), _p(filtered), _p(prev_pix), _p(accept), _p(albedo),
                                         _p(tone_mapped), _p(cur_spp), _p(acc_prev), _p(acc_cur), int(frame))

    def taa(self, prev_pix, new_frame, result, prev_result, frame):
        lib.orc_taa(C.byref(self.cfg), _p(prev_pix), _p(new_frame), _p(result), _p(prev_result), int(frame))


class OraclePipeline:
    """The reference host program's frame loop (opencl/bmfr.cpp:417-485) over
    the oracle kernels, with the six double buffers swapped every frame."""

    STAGES = ("accumulate_noisy_data", "fitter", "weighted_sum", "accumulate_filtered_data", "taa")

    def __init__(self, oracle: Oracle, fitter_mode=FITTER_REFERENCE):
        self.o = oracle
        self.mode = fitter_mode
        H, W = oracle.height, oracle.width
        z3 = lambda: np.zeros((H, W, 3), dtype=np.float32)
        self.normals, self.positions, self.noisy = [z3(), z3()], [z3(), z3()], [z3(), z3()]
        self.acc, self.result = [z3(), z3()], [z3(), z3()]
        self.spp = [np.zeros((H, W), np.uint8), np.zeros((H, W), np.uint8)]
        self.tmp = oracle.new_tmp()
        self.filtered, self.tone_mapped = z3(), z3()
        self.prev_pix = np.zeros((H, W, 2), dtype=np.float32)
        self.accept = np.zeros((H, W), dtype=np.uint8)
        self.weights = np.zeros(oracle.blocks * 30, dtype=np.float32)
        self.mins_maxs = np.zeros(oracle.blocks * 12, dtype=np.float32)
        self.frame = 0

    def step(self, albedo, normals, positions, noisy, matrix, offset):
        f = self.frame
        c, p = f & 1, (f & 1) ^ 1
        self.normals[c][...] = normals
        self.positions[c][...] = positions
        self.noisy[c][...] = noisy
        o = self.o
        t = [time.perf_counter()]
        o.accumulate_noisy_data(self.prev_pix, self.accept, self.normals[c], self.normals[p], self.positions[c],
                                self.positions[p], self.noisy[c], self.noisy[p], self.spp[p], self.spp[c],
                                self.tmp, matrix, offset, f)
        t.append(time.perf_counter())
        self.tmp_after_accumulate = self.tmp.copy()
        t.append(time.perf_counter())
        o.fitter(self.weights, self.mins_maxs, self.tmp, f, self.mode)
        t.append(time.perf_counter())
        o.weighted_sum(self.weights, self.mins_maxs, self.filtered, self.normals[c], self.positions[c], f)
        t.append(time.perf_counter())
        alb = np.ascontiguousarray(albedo, dtype=np.float32)
        o.accumulate_filtered_data(self.filtered, self.prev_pix, self.accept, alb, self.tone_mapped, self.spp[c],
                                   self.acc[p], self.acc[c], f)
        t.append(time.perf_counter())
        o.taa(self.prev_pix, self.tone_mapped, self.result[c], self.result[p], f)
        t.append(time.perf_counter())
        # Seconds per stage of this frame (the reference's per-kernel
        # profile, opencl/bmfr.cpp:488-517); the copy of tmp_data is left out.
        self.stage_seconds = dict(zip(self.STAGES, (t[1] - t[0], t[3] - t[2], t[4] - t[3], t[5] - t[4],
                                                    t[6] - t[5])))
        self.frame = f + 1
        return self.result[c]
