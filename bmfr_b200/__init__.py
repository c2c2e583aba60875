"""bmfr_b200 — B200 (sm_100a) implementation of the BMFR per-frame denoising
pipeline (Blockwise Multi-Order Feature Regression, opencl/bmfr.cl).

The five stages keep the reference kernels' names and argument lists
(accumulate_noisy_data, fitter, weighted_sum, accumulate_filtered_data, taa);
``Plan`` also runs the reference host program's frame loop
(opencl/bmfr.cpp:417-485) on plan-owned history buffers.  All compute is in
the native library libbmfr_b200.so; torch is used only to hold device memory
and to name CUDA streams.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from bmfr_scene import Scene  # the input source (its own library, libbmfr_scene.so)

from . import _native
from ._native import (BatchTuning, ServerConfig, ServerStats, BmfrError, FrameInputs, FrameIO, Params, PlanBuffers,
                      Sizes, check, lib, PIPELINE_FUSED, PIPELINE_STAGED, QR_CHOLESKY2, QR_HOUSEHOLDER, QR_REFERENCE)

__all__ = [
    "Plan", "Batch", "Server", "Router", "Scene", "BmfrError", "default_params", "block_offsets",
    "accumulate_noisy_data", "fitter", "fitter_fp64", "weighted_sum", "accumulate_filtered_data", "taa",
    "write_pfm", "read_pfm", "psnr",
    "PIPELINE_FUSED", "PIPELINE_STAGED", "QR_REFERENCE", "QR_CHOLESKY2", "QR_HOUSEHOLDER", "library_path",
]

library_path = _native.library_path


def default_params(**overrides) -> Params:
    """The reference's compile-time options (opencl/bmfr.cpp:56-118) as a Params."""
    p = Params()
    check(lib.bmfr_params_default(C.byref(p)), "bmfr_params_default")
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise AttributeError(f"unknown BMFR parameter {k!r}")
        setattr(p, k, v)
    return p


def block_offsets() -> np.ndarray:
    """BLOCK_OFFSETS (opencl/bmfr.cl:267-285) as a (16, 2) int array."""
    out = (C.c_int * 32)()
    check(lib.bmfr_block_offsets(out), "bmfr_block_offsets")
    return np.array(out, dtype=np.int32).reshape(16, 2)


def _stream_ptr(stream) -> C.c_void_p:
    if stream is None:
        import torch
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(stream.cuda_stream)


def _ptr(t, name: str, nbytes: int | None = None, optional: bool = False) -> C.c_void_p:
    """Device pointer of a contiguous CUDA tensor (or None)."""
    if t is None:
        if optional:
            return C.c_void_p(None)
        raise ValueError(f"{name} must not be None")
    if isinstance(t, int):
        return C.c_void_p(t)
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if nbytes is not None and t.numel() * t.element_size() < nbytes:
        raise ValueError(f"{name} holds {t.numel() * t.element_size()} bytes, needs {nbytes}")
    return C.c_void_p(t.data_ptr())


def _mem_ptr(t, name: str, nbytes: int | None = None) -> C.c_void_p:
    """Address of host (numpy array, CPU tensor) or device (CUDA tensor) memory."""
    if isinstance(t, np.ndarray):
        if not t.flags.c_contiguous:
            raise ValueError(f"{name} must be contiguous")
        if nbytes is not None and t.nbytes < nbytes:
            raise ValueError(f"{name} holds {t.nbytes} bytes, needs {nbytes}")
        return C.c_void_p(t.ctypes.data)
    if hasattr(t, "is_cuda") and not t.is_cuda:
        if not t.is_contiguous():
            raise ValueError(f"{name} must be contiguous")
        if nbytes is not None and t.numel() * t.element_size() < nbytes:
            raise ValueError(f"{name} holds {t.numel() * t.element_size()} bytes, needs {nbytes}")
        return C.c_void_p(t.data_ptr())
    return _ptr(t, name, nbytes)


def _f32(values, n: int, name: str):
    a = np.ascontiguousarray(np.asarray(values, dtype=np.float32).reshape(-1))
    if a.size != n:
        raise ValueError(f"{name} needs {n} floats")
    return a, a.ctypes.data_as(C.POINTER(C.c_float))


class Plan:
    """Sizes of one image stream plus the frame pipeline's history buffers.

    ``Plan(1280, 720)`` uses the reference's defaults; keyword arguments
    override fields of Params (e.g. ``pipeline=PIPELINE_STAGED``).
    """

    def __init__(self, width: int, height: int, params: Params | None = None, **overrides):
        self.params = params if params is not None else default_params(**overrides)
        h = C.c_void_p()
        check(lib.bmfr_plan_create(C.byref(self.params), int(width), int(height), C.byref(h)),
              "bmfr_plan_create")
        self._h = h
        s = Sizes()
        check(lib.bmfr_plan_sizes(h, C.byref(s)), "bmfr_plan_sizes")
        self.sizes = s
        self.width, self.height = s.image_width, s.image_height

    @property
    def handle(self) -> C.c_void_p:
        if self._h is None:
            raise BmfrError(_native.BMFR_E_STATE, "plan destroyed")
        return self._h

    def close(self) -> None:
        if getattr(self, "_h", None) is not None:
            lib.bmfr_plan_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- frame pipeline (opencl/bmfr.cpp:417-485) --------------------------
    @property
    def frame_number(self) -> int:
        return lib.bmfr_plan_frame_number(self.handle)

    def frame_inputs(self) -> FrameInputs:
        fi = FrameInputs()
        check(lib.bmfr_plan_frame_inputs(self.handle, C.byref(fi)), "bmfr_plan_frame_inputs")
        return fi

    def upload_frame(self, albedo, normals, positions, noisy, stream=None) -> None:
        """Copies one frame's four host buffers (float32, H*W*3) into the plan."""
        arrs = []
        n = self.width * self.height * 3
        for name, a in (("albedo", albedo), ("normals", normals), ("positions", positions), ("noisy", noisy)):
            if hasattr(a, "data_ptr"):
                if a.is_cuda or a.numel() != n or a.dtype.itemsize != 4 or not a.is_contiguous():
                    raise ValueError(f"{name}: contiguous float32 host tensor of {n} values expected")
                arrs.append(C.c_void_p(a.data_ptr()))
            else:
                a = np.ascontiguousarray(a, dtype=np.float32)
                if a.size != n:
                    raise ValueError(f"{name}: {n} values expected")
                arrs.append(C.c_void_p(a.ctypes.data))
        check(lib.bmfr_plan_upload_frame(self.handle, *arrs, _stream_ptr(stream)), "bmfr_plan_upload_frame")

    def denoise_frame(self, prev_frame_camera_matrix, pixel_offset, stream=None) -> None:
        """Runs the five stages for the next frame and swaps the histories."""
        m, mp = _f32(prev_frame_camera_matrix, 16, "prev_frame_camera_matrix")
        o, op = _f32(pixel_offset, 2, "pixel_offset")
        check(lib.bmfr_denoise_frame(self.handle, mp, op, _stream_ptr(stream)), "bmfr_denoise_frame")

    def denoise_frame_io(self, albedo, normals, positions, noisy, previous_normals, previous_positions,
                         prev_frame_camera_matrix, pixel_offset, result=None, stream=None) -> None:
        """denoise_frame on caller-owned device tensors (float32, H*W*3)."""
        n = self.width * self.height * 12
        first = self.frame_number == 0
        io = FrameIO(_ptr(albedo, "albedo", n), _ptr(normals, "normals", n), _ptr(positions, "positions", n),
                     _ptr(noisy, "noisy", n), _ptr(previous_normals, "previous_normals", n, optional=first),
                     _ptr(previous_positions, "previous_positions", n, optional=first),
                     _ptr(result, "result", n, optional=True))
        m, mp = _f32(prev_frame_camera_matrix, 16, "prev_frame_camera_matrix")
        o, op = _f32(pixel_offset, 2, "pixel_offset")
        check(lib.bmfr_denoise_frame_io(self.handle, C.byref(io), mp, op, _stream_ptr(stream)),
              "bmfr_denoise_frame_io")

    def denoise_frames(self, frames, prev_frame_camera_matrices, pixel_offsets, stream=None) -> None:
        """Consecutive frames in one call (bmfr_denoise_frames): `frames` is a
        sequence of dicts with the keys of denoise_frame_io's buffers
        (albedo, normals, positions, noisy, previous_normals,
        previous_positions, optional result), one camera matrix and pixel
        offset per frame.  Outputs equal those of one denoise_frame_io call per
        frame; the staged pipeline overlaps each frame's accumulation with the
        previous frame's later stages."""
        count = len(frames)
        n = self.width * self.height * 12
        first = self.frame_number
        ios = (FrameIO * max(count, 1))()
        for k, fr in enumerate(frames):
            at0 = first + k == 0
            ios[k] = FrameIO(_ptr(fr["albedo"], "albedo", n), _ptr(fr["normals"], "normals", n),
                             _ptr(fr["positions"], "positions", n), _ptr(fr["noisy"], "noisy", n),
                             _ptr(fr.get("previous_normals"), "previous_normals", n, optional=at0),
                             _ptr(fr.get("previous_positions"), "previous_positions", n, optional=at0),
                             _ptr(fr.get("result"), "result", n, optional=True))
        mats = np.ascontiguousarray(np.asarray(prev_frame_camera_matrices, dtype=np.float32).reshape(-1))
        offs = np.ascontiguousarray(np.asarray(pixel_offsets, dtype=np.float32).reshape(-1))
        if mats.size != 16 * count or offs.size != 2 * count:
            raise ValueError(f"{count} camera matrices (16 floats) and pixel offsets (2 floats) expected")
        fp = C.POINTER(C.c_float)
        check(lib.bmfr_denoise_frames(self.handle, count, ios, mats.ctypes.data_as(fp), offs.ctypes.data_as(fp),
                                      _stream_ptr(stream)), "bmfr_denoise_frames")

    def result_ptr(self) -> int:
        p = C.c_void_p()
        check(lib.bmfr_plan_result(self.handle, C.byref(p)), "bmfr_plan_result")
        return p.value

    def download_result(self, out=None, stream=None) -> np.ndarray:
        """Copies the last TAA output to host memory (blocking unless `out`
        is a pinned tensor and a stream is given)."""
        if out is None:
            out = np.empty((self.height, self.width, 3), dtype=np.float32)
            check(lib.bmfr_plan_download_result(self.handle, C.c_void_p(out.ctypes.data), _stream_ptr(stream)),
                  "bmfr_plan_download_result")
            import torch
            torch.cuda.current_stream().synchronize() if stream is None else stream.synchronize()
            return out
        check(lib.bmfr_plan_download_result(self.handle, C.c_void_p(out.data_ptr()), _stream_ptr(stream)),
              "bmfr_plan_download_result")
        return out

    def enable_profiling(self, enable: bool = True) -> None:
        check(lib.bmfr_plan_enable_profiling(self.handle, int(enable)), "bmfr_plan_enable_profiling")

    def check_device(self, stream=None) -> None:
        """Waits for `stream`; raises BmfrError (BMFR_E_TIMEOUT) if a kernel
        of this plan gave up a bounded wait, and clears that status."""
        check(lib.bmfr_plan_check_device(self.handle, _stream_ptr(stream)), "bmfr_plan_check_device")

    def probe_bounded_wait(self, limit_us: int, stream=None) -> None:
        """Enqueues a wait that runs out after `limit_us` (the failure path
        of the bounded waits, without a fault); check_device then raises."""
        check(lib.bmfr_plan_probe_bounded_wait(self.handle, int(limit_us), _stream_ptr(stream)),
              "bmfr_plan_probe_bounded_wait")

    STAGES = ("accumulate_noisy_data", "fitter", "weighted_sum+accumulate_filtered_data", None, "taa")
    FUSED_STAGES = ("noise_table", "block_kernel", "weighted_sum+accumulate_filtered_data", None, "taa")

    def stage_times(self) -> dict:
        """Milliseconds per kernel of the last profiled frame (the staged
        pipeline's four kernels, or the fused pipeline's three)."""
        ms = (C.c_float * 5)()
        check(lib.bmfr_plan_stage_times(self.handle, ms), "bmfr_plan_stage_times")
        names = self.FUSED_STAGES if self.params.pipeline == PIPELINE_FUSED else self.STAGES
        return {n: float(v) for n, v in zip(names, ms) if n is not None}

    def keep_intermediates(self, enable: bool = True) -> None:
        """Also write the filtered frame of every frame (for inspection;
        outputs are unchanged)."""
        check(lib.bmfr_plan_keep_intermediates(self.handle, int(enable)), "bmfr_plan_keep_intermediates")

    def buffers(self) -> PlanBuffers:
        b = PlanBuffers()
        check(lib.bmfr_plan_buffers_get(self.handle, C.byref(b)), "bmfr_plan_buffers_get")
        return b

    def reset(self) -> None:
        check(lib.bmfr_plan_reset(self.handle), "bmfr_plan_reset")


# -- the five stages (drop-in for opencl/bmfr.cl's kernels) ------------------

def accumulate_noisy_data(plan: Plan, out_prev_frame_pixel, accept_bools, current_normals, previous_normals,
                          current_positions, previous_positions, current_noisy, previous_noisy, previous_spp,
                          current_spp, tmp_data, prev_frame_camera_matrix, pixel_offset, frame_number: int,
                          stream=None) -> None:
    """opencl/bmfr.cl:290-485; current_noisy is updated in place."""
    px = plan.width * plan.height
    hist = frame_number > 0
    m, mp = _f32(prev_frame_camera_matrix, 16, "prev_frame_camera_matrix")
    o, op = _f32(pixel_offset, 2, "pixel_offset")
    check(lib.bmfr_accumulate_noisy_data(
        plan.handle, _ptr(out_prev_frame_pixel, "out_prev_frame_pixel", px * 8),
        _ptr(accept_bools, "accept_bools", px), _ptr(current_normals, "current_normals", px * 12),
        _ptr(previous_normals, "previous_normals", px * 12, optional=not hist),
        _ptr(current_positions, "current_positions", px * 12),
        _ptr(previous_positions, "previous_positions", px * 12, optional=not hist),
        _ptr(current_noisy, "current_noisy", px * 12),
        _ptr(previous_noisy, "previous_noisy", px * 12, optional=not hist),
        _ptr(previous_spp, "previous_spp", px, optional=not hist), _ptr(current_spp, "current_spp", px),
        _ptr(tmp_data, "tmp_data", plan.sizes.tmp_data_bytes), mp, op, int(frame_number),
        _stream_ptr(stream)), "accumulate_noisy_data")


def fitter(plan: Plan, weights, mins_maxs, tmp_data, frame_number: int, stream=None) -> None:
    """opencl/bmfr.cl:490-700."""
    check(lib.bmfr_fitter(plan.handle, _ptr(weights, "weights", plan.sizes.weights_bytes),
                          _ptr(mins_maxs, "mins_maxs", plan.sizes.mins_maxs_bytes),
                          _ptr(tmp_data, "tmp_data", plan.sizes.tmp_data_bytes), int(frame_number),
                          _stream_ptr(stream)), "fitter")


def fitter_fp64(plan: Plan, weights64, mins_maxs, tmp_data, frame_number: int, stream=None) -> None:
    """The fitter in double precision (weights64: float64, blocks*10*3)."""
    check(lib.bmfr_fitter_fp64(plan.handle, _ptr(weights64, "weights64", plan.sizes.weights_bytes * 2),
                               _ptr(mins_maxs, "mins_maxs", plan.sizes.mins_maxs_bytes),
                               _ptr(tmp_data, "tmp_data", plan.sizes.tmp_data_bytes), int(frame_number),
                               _stream_ptr(stream)), "fitter_fp64")


def weighted_sum(plan: Plan, weights, mins_maxs, output, current_normals, current_positions, current_noisy,
                 frame_number: int, stream=None) -> None:
    """opencl/bmfr.cl:703-758 (current_noisy is unused, as in the reference)."""
    px = plan.width * plan.height
    check(lib.bmfr_weighted_sum(plan.handle, _ptr(weights, "weights", plan.sizes.weights_bytes),
                                _ptr(mins_maxs, "mins_maxs", plan.sizes.mins_maxs_bytes),
                                _ptr(output, "output", px * 12), _ptr(current_normals, "current_normals", px * 12),
                                _ptr(current_positions, "current_positions", px * 12),
                                _ptr(current_noisy, "current_noisy", optional=True), int(frame_number),
                                _stream_ptr(stream)), "weighted_sum")


def accumulate_filtered_data(plan: Plan, filtered_frame, in_prev_frame_pixel, accept_bools, albedo,
                             tone_mapped_frame, current_spp, accumulated_prev_frame, accumulated_frame,
                             frame_number: int, stream=None) -> None:
    """opencl/bmfr.cl:761-857."""
    px = plan.width * plan.height
    hist = frame_number > 0
    check(lib.bmfr_accumulate_filtered_data(
        plan.handle, _ptr(filtered_frame, "filtered_frame", px * 12),
        _ptr(in_prev_frame_pixel, "in_prev_frame_pixel", px * 8, optional=not hist),
        _ptr(accept_bools, "accept_bools", px, optional=not hist), _ptr(albedo, "albedo", px * 12),
        _ptr(tone_mapped_frame, "tone_mapped_frame", px * 12),
        _ptr(current_spp, "current_spp", px, optional=not hist),
        _ptr(accumulated_prev_frame, "accumulated_prev_frame", px * 12, optional=not hist),
        _ptr(accumulated_frame, "accumulated_frame", px * 12), int(frame_number), _stream_ptr(stream)),
        "accumulate_filtered_data")


def taa(plan: Plan, in_prev_frame_pixel, new_frame, result_frame, prev_frame, frame_number: int,
        stream=None) -> None:
    """opencl/bmfr.cl:860-974."""
    px = plan.width * plan.height
    check(lib.bmfr_taa(plan.handle, _ptr(in_prev_frame_pixel, "in_prev_frame_pixel", px * 8),
                       _ptr(new_frame, "new_frame", px * 12), _ptr(result_frame, "result_frame", px * 12),
                       _ptr(prev_frame, "prev_frame", px * 12, optional=frame_number == 0), int(frame_number),
                       _stream_ptr(stream)), "taa")


# -- many streams (include/bmfr_batch.h) -------------------------------------

class Batch:
    """Many streams of uneven size denoised together, one step per frame of any
    subset of them (see include/bmfr_batch.h for the fused and staged steps)."""

    def __init__(self, params: Params | None = None, memory_budget_bytes: int = 0, **overrides):
        self.params = params if params is not None else default_params(**overrides)
        h = C.c_void_p()
        check(lib.bmfr_batch_create(C.byref(self.params), int(memory_budget_bytes), C.byref(h)), "bmfr_batch_create")
        self._h = h
        self.sizes = {}

    @property
    def handle(self):
        if self._h is None:
            raise BmfrError(_native.BMFR_E_STATE, "batch destroyed")
        return self._h

    def close(self):
        if getattr(self, "_h", None) is not None:
            lib.bmfr_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def stream_bytes(params: Params, width: int, height: int, own_inputs: bool = False) -> int:
        n = C.c_size_t()
        check(lib.bmfr_batch_stream_bytes(C.byref(params), width, height, int(own_inputs), C.byref(n)),
              "bmfr_batch_stream_bytes")
        return n.value

    def add_stream(self, width: int, height: int, own_inputs: bool = False) -> int:
        slot = C.c_int()
        check(lib.bmfr_batch_add_stream(self.handle, int(width), int(height), int(own_inputs), C.byref(slot)),
              "bmfr_batch_add_stream")
        self.sizes[slot.value] = (int(width), int(height))
        return slot.value

    def remove_stream(self, slot: int) -> None:
        check(lib.bmfr_batch_remove_stream(self.handle, int(slot)), "bmfr_batch_remove_stream")
        self.sizes.pop(slot, None)

    def reset_stream(self, slot: int) -> None:
        check(lib.bmfr_batch_reset_stream(self.handle, int(slot)), "bmfr_batch_reset_stream")

    def frame(self, slot: int) -> int:
        v = lib.bmfr_batch_stream_frame(self.handle, int(slot))
        if v < 0:
            check(v, "bmfr_batch_stream_frame")
        return v

    def reserve(self, nbytes: int) -> None:
        """Grows the stream memory pool to at least nbytes (blocking)."""
        check(lib.bmfr_batch_reserve(self.handle, int(nbytes)), "bmfr_batch_reserve")

    @property
    def bytes_in_use(self) -> int:
        return lib.bmfr_batch_bytes_in_use(self.handle)

    def stream_inputs(self, slot: int) -> FrameInputs:
        fi = FrameInputs()
        check(lib.bmfr_batch_stream_inputs(self.handle, int(slot), C.byref(fi)), "bmfr_batch_stream_inputs")
        return fi

    @staticmethod
    def frame_io(albedo, normals, positions, noisy, previous_normals=None, previous_positions=None,
                 result=None) -> FrameIO:
        """A FrameIO of device tensors (or raw device addresses)."""
        return FrameIO(_ptr(albedo, "albedo"), _ptr(normals, "normals"), _ptr(positions, "positions"),
                       _ptr(noisy, "noisy"), _ptr(previous_normals, "previous_normals", optional=True),
                       _ptr(previous_positions, "previous_positions", optional=True),
                       _ptr(result, "result", optional=True))

    def _args(self, slots, io, matrices, offsets):
        n = len(slots)
        sl = (C.c_int * n)(*slots)
        iop = None
        if io is not None:
            arr = (FrameIO * n)()
            for k, v in enumerate(io):
                arr[k] = v if v is not None else FrameIO()
            iop = arr
        m, mp = _f32(matrices, 16 * n, "matrices")
        o, op = _f32(offsets, 2 * n, "offsets")
        return n, sl, iop, (m, o), mp, op

    def step(self, slots, matrices, offsets, io=None, stream=None) -> None:
        """Denoises the next frame of each stream in `slots`: one graph launch
        (fused step) or each stream's plan kernels on the batch's worker
        streams, joined into `stream` (staged step)."""
        n, sl, iop, keep, mp, op = self._args(slots, io, matrices, offsets)
        check(lib.bmfr_batch_step(self.handle, n, sl, iop, mp, op, _stream_ptr(stream)), "bmfr_batch_step")

    def snapshot_bytes(self, slot: int) -> int:
        n = C.c_size_t()
        check(lib.bmfr_batch_snapshot_bytes(self.handle, int(slot), C.byref(n)), "bmfr_batch_snapshot_bytes")
        return n.value

    def snapshot(self, slot: int, out=None, stream=None):
        """The stream's history snapshot into `out` (a host numpy uint8 array
        or a device tensor of snapshot_bytes(slot) bytes; new host array if None)."""
        n = self.snapshot_bytes(slot)
        if out is None:
            out = np.empty(n, dtype=np.uint8)
        check(lib.bmfr_batch_snapshot(self.handle, int(slot), _mem_ptr(out, "out", n), _stream_ptr(stream)),
              "bmfr_batch_snapshot")
        return out

    def restore(self, snapshot, stream=None) -> int:
        """Adds a stream from a snapshot; returns its slot."""
        sl = C.c_int()
        check(lib.bmfr_batch_restore(self.handle, _mem_ptr(snapshot, "snapshot"), _stream_ptr(stream), C.byref(sl)),
              "bmfr_batch_restore")
        return sl.value

    def result_ptr(self, slot: int) -> int:
        p = C.c_void_p()
        check(lib.bmfr_batch_stream_result(self.handle, int(slot), C.byref(p)), "bmfr_batch_stream_result")
        return p.value

    @property
    def tuning(self) -> BatchTuning:
        t = BatchTuning()
        check(lib.bmfr_batch_get_tuning(self.handle, C.byref(t)), "bmfr_batch_get_tuning")
        return t

    def set_tuning(self, block_ctas_per_sm=0, taa_tile_w=30, taa_tile_h=32, staging_depth=0, pixel_pass=0) -> None:
        t = BatchTuning(block_ctas_per_sm, taa_tile_w, taa_tile_h, staging_depth, pixel_pass)
        check(lib.bmfr_batch_set_tuning(self.handle, C.byref(t)), "bmfr_batch_set_tuning")

    def autotune(self, slots, matrices, offsets, io=None, steps=3, stream=None):
        """Times candidate tunings of the fused step on real steps of these
        streams (advancing their histories) and keeps the fastest; the
        staged step has nothing to tune and is only timed.  Returns
        (tuning, mean ms per step)."""
        n, sl, iop, keep, mp, op = self._args(slots, io, matrices, offsets)
        t = BatchTuning()
        ms = C.c_float()
        check(lib.bmfr_batch_autotune(self.handle, n, sl, iop, mp, op, int(steps), _stream_ptr(stream),
                                      C.byref(t), C.byref(ms)), "bmfr_batch_autotune")
        return t, ms.value


class Server:
    """Continuous batching of frame requests from many render streams
    (include/bmfr_batch.h, bmfr_server_*)."""

    def __init__(self, params: Params | None = None, memory_budget_bytes: int = 0, max_streams_per_step: int = 0,
                 own_inputs: bool = False, max_steps_in_flight: int = 0, reserve_bytes: int = 0, **overrides):
        self.params = params if params is not None else default_params(pipeline=PIPELINE_FUSED, **overrides)
        cfg = ServerConfig(int(memory_budget_bytes), int(max_streams_per_step), int(own_inputs),
                           int(max_steps_in_flight), int(reserve_bytes))
        h = C.c_void_p()
        check(lib.bmfr_server_create(C.byref(self.params), C.byref(cfg), C.byref(h)), "bmfr_server_create")
        self._h = h

    @property
    def handle(self):
        if self._h is None:
            raise BmfrError(_native.BMFR_E_STATE, "server destroyed")
        return self._h

    def close(self):
        if getattr(self, "_h", None) is not None:
            lib.bmfr_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def open_stream(self, width: int, height: int) -> int:
        sid = C.c_int()
        check(lib.bmfr_server_open_stream(self.handle, int(width), int(height), C.byref(sid)),
              "bmfr_server_open_stream")
        return sid.value

    def close_stream(self, sid: int) -> None:
        check(lib.bmfr_server_close_stream(self.handle, int(sid)), "bmfr_server_close_stream")

    def submit(self, sid: int, matrix, offset, io: FrameIO | None = None) -> int:
        m, mp = _f32(matrix, 16, "matrix")
        o, op = _f32(offset, 2, "offset")
        rid = C.c_uint64()
        check(lib.bmfr_server_submit(self.handle, int(sid), C.byref(io) if io is not None else None, mp, op,
                                     C.byref(rid)), "bmfr_server_submit")
        return rid.value

    def snapshot_bytes(self, sid: int) -> int:
        """Size of an open stream's history snapshot."""
        n = C.c_size_t()
        check(lib.bmfr_batch_snapshot_bytes(lib.bmfr_server_batch(self.handle), int(sid), C.byref(n)),
              "bmfr_batch_snapshot_bytes")
        return n.value

    def snapshot_stream(self, sid: int, out, stream=None):
        """bmfr_server_snapshot_stream into `out` (host numpy uint8 array or
        device tensor, at least batch snapshot_bytes long)."""
        check(lib.bmfr_server_snapshot_stream(self.handle, int(sid), _mem_ptr(out, "out"), _stream_ptr(stream)),
              "bmfr_server_snapshot_stream")
        return out

    def restore_stream(self, snapshot, stream=None) -> int:
        sid = C.c_int()
        check(lib.bmfr_server_restore_stream(self.handle, _mem_ptr(snapshot, "snapshot"), _stream_ptr(stream),
                                             C.byref(sid)), "bmfr_server_restore_stream")
        return sid.value

    def poll(self, rid: int):
        done, lat = C.c_int(), C.c_double()
        check(lib.bmfr_server_poll(self.handle, C.c_uint64(rid), C.byref(done), C.byref(lat)), "bmfr_server_poll")
        return bool(done.value), lat.value

    def drain(self, timeout_ms: float = 60000.0) -> None:
        check(lib.bmfr_server_drain(self.handle, float(timeout_ms)), "bmfr_server_drain")

    def stats(self) -> dict:
        st = ServerStats()
        check(lib.bmfr_server_stats_get(self.handle, C.byref(st)), "bmfr_server_stats_get")
        return {name: getattr(st, name) for name, _ in ServerStats._fields_}

    def reset_stats(self) -> None:
        check(lib.bmfr_server_stats_reset(self.handle), "bmfr_server_stats_reset")

    def set_tuning(self, t: BatchTuning) -> None:
        check(lib.bmfr_server_set_tuning(self.handle, C.byref(t)), "bmfr_server_set_tuning")


from .router import Router  # noqa: E402  (per-GPU servers behind one placement)


# -- image output (include/bmfr_image.h) -----------------------------------

def _host_f32(img, name):
    a = np.ascontiguousarray(img, dtype=np.float32)
    return a, a.ctypes.data_as(C.POINTER(C.c_float))


def write_pfm(path, image) -> None:
    """Writes an (H, W, 3) float image (top row first) as a PFM file."""
    a, p = _host_f32(image, "image")
    if a.ndim != 3 or a.shape[2] != 3:
        raise ValueError("image must be (H, W, 3)")
    check(lib.bmfr_write_pfm(str(path).encode(), a.shape[1], a.shape[0], p), "bmfr_write_pfm")


def read_pfm(path) -> np.ndarray:
    """Reads a colour PFM file as an (H, W, 3) float32 array, top row first."""
    w, h = C.c_int(), C.c_int()
    check(lib.bmfr_read_pfm(str(path).encode(), C.byref(w), C.byref(h), None, 0), "bmfr_read_pfm")
    out = np.empty((h.value, w.value, 3), dtype=np.float32)
    check(lib.bmfr_read_pfm(str(path).encode(), C.byref(w), C.byref(h), out.ctypes.data_as(C.POINTER(C.c_float)),
                            out.size), "bmfr_read_pfm")
    return out


def psnr(a, b, peak: float = 1.0) -> float:
    """PSNR in dB between two float images of the same size."""
    x, px = _host_f32(a, "a")
    y, py = _host_f32(b, "b")
    if x.size != y.size:
        raise ValueError("images differ in size")
    return float(lib.bmfr_psnr(px, py, x.size, float(peak)))

