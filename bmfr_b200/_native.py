"""ctypes binding of libbmfr_b200.so (include/bmfr_b200.h, bmfr_batch.h, bmfr_image.h).

The library is the product: importing this module loads it and raises if it
is missing — there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_LIB_PATH = Path(__file__).resolve().parent / "libbmfr_b200.so"

BMFR_OK = 0
BMFR_E_INVALID = -1
BMFR_E_CUDA = -2
BMFR_E_UNSUPPORTED = -3
BMFR_E_NOMEM = -4
BMFR_E_BUDGET = -5
BMFR_E_NOT_FOUND = -6
BMFR_E_AGAIN = -7
BMFR_E_TIMEOUT = -8
BMFR_E_STATE = -9
BMFR_E_TOO_LARGE = -10

PIPELINE_STAGED = 0
PIPELINE_FUSED = 1

QR_REFERENCE = 0      # the reference's Householder sequence and binary16 rounding
QR_CHOLESKY2 = 1      # precision form: CholeskyQR2 in FP32
QR_HOUSEHOLDER = 2    # precision form: the Householder sequence in FP32


class Params(C.Structure):
    _fields_ = [
        ("noise_amount", C.c_double),
        ("blend_alpha", C.c_float),
        ("second_blend_alpha", C.c_float),
        ("taa_blend_alpha", C.c_float),
        ("position_limit_squared", C.c_float),
        ("normal_limit_squared", C.c_float),
        ("use_half_precision_in_tmp_data", C.c_int),
        ("compressed_r", C.c_int),
        ("cache_tmp_data", C.c_int),
        ("fp32_qr", C.c_int),
        ("half_history", C.c_int),
        ("pipeline", C.c_int),
    ]


class Sizes(C.Structure):
    _fields_ = [
        ("image_width", C.c_int), ("image_height", C.c_int),
        ("workset_width", C.c_int), ("workset_height", C.c_int),
        ("margin_width", C.c_int), ("margin_height", C.c_int),
        ("blocks_x", C.c_int), ("blocks_y", C.c_int), ("blocks", C.c_int),
        ("tmp_data_bytes", C.c_size_t), ("weights_bytes", C.c_size_t),
        ("mins_maxs_bytes", C.c_size_t), ("pixel3_bytes", C.c_size_t),
    ]


class FrameInputs(C.Structure):
    _fields_ = [("albedo", C.c_void_p), ("normals", C.c_void_p),
                ("positions", C.c_void_p), ("noisy", C.c_void_p)]


class PlanBuffers(C.Structure):
    _fields_ = [("tmp_data", C.c_void_p), ("weights", C.c_void_p), ("mins_maxs", C.c_void_p),
                ("filtered", C.c_void_p), ("prev_frame_pixel", C.c_void_p),
                ("tone_mapped", C.c_void_p), ("accept", C.c_void_p), ("spp", C.c_void_p),
                ("accumulated_noisy", C.c_void_p), ("accumulated_filtered", C.c_void_p),
                ("result", C.c_void_p)]


class FrameIO(C.Structure):
    _fields_ = [("albedo", C.c_void_p), ("normals", C.c_void_p), ("positions", C.c_void_p),
                ("noisy", C.c_void_p), ("previous_normals", C.c_void_p),
                ("previous_positions", C.c_void_p), ("result", C.c_void_p)]


class BatchTuning(C.Structure):
    _fields_ = [("block_ctas_per_sm", C.c_int), ("taa_tile_w", C.c_int), ("taa_tile_h", C.c_int),
                ("staging_depth", C.c_int), ("pixel_pass", C.c_int)]


class ServerConfig(C.Structure):
    _fields_ = [("memory_budget_bytes", C.c_size_t), ("max_streams_per_step", C.c_int), ("own_inputs", C.c_int),
                ("max_steps_in_flight", C.c_int), ("reserve_bytes", C.c_size_t)]


class ServerStats(C.Structure):
    _fields_ = [("requests_submitted", C.c_uint64), ("requests_completed", C.c_uint64),
                ("steps", C.c_uint64), ("frames", C.c_uint64),
                ("streams_admitted", C.c_uint64), ("streams_rejected", C.c_uint64),
                ("p50_latency_ms", C.c_double), ("p99_latency_ms", C.c_double),
                ("max_latency_ms", C.c_double), ("mean_latency_ms", C.c_double),
                ("mean_frames_per_step", C.c_double), ("busy_seconds", C.c_double),
                ("elapsed_seconds", C.c_double)]


def _load() -> C.CDLL:
    if not _LIB_PATH.exists():
        raise ImportError(
            f"{_LIB_PATH} is missing: build it with `python bmfr_b200/build.py` "
            "(the CUDA library is required; there is no CPU fallback)")
    lib = C.CDLL(str(_LIB_PATH))
    vp, i, f, fp, u8p = C.c_void_p, C.c_int, C.c_float, C.POINTER(C.c_float), C.c_void_p
    sig = {
        "bmfr_params_default": (i, [C.POINTER(Params)]),
        "bmfr_plan_create": (i, [C.POINTER(Params), i, i, C.POINTER(vp)]),
        "bmfr_plan_destroy": (i, [vp]),
        "bmfr_plan_sizes": (i, [vp, C.POINTER(Sizes)]),
        "bmfr_plan_params": (i, [vp, C.POINTER(Params)]),
        "bmfr_block_offsets": (i, [C.POINTER(C.c_int)]),
        "bmfr_accumulate_noisy_data": (i, [vp, vp, u8p, vp, vp, vp, vp, vp, vp, u8p, u8p, vp, fp, fp, i, vp]),
        "bmfr_fitter": (i, [vp, vp, vp, vp, i, vp]),
        "bmfr_fitter_fp64": (i, [vp, vp, vp, vp, i, vp]),
        "bmfr_fitter_noalloc": (i, [C.POINTER(Params), i, i, vp, vp, vp, i, vp]),
        "bmfr_fitter_noalloc_check": (i, [vp]),
        "bmfr_fitter_noalloc_probe_bounded_wait": (i, [C.c_uint, vp]),
        "bmfr_weighted_sum": (i, [vp, vp, vp, vp, vp, vp, vp, i, vp]),
        "bmfr_accumulate_filtered_data": (i, [vp, vp, vp, u8p, vp, vp, u8p, vp, vp, i, vp]),
        "bmfr_taa": (i, [vp, vp, vp, vp, vp, i, vp]),
        "bmfr_plan_frame_inputs": (i, [vp, C.POINTER(FrameInputs)]),
        "bmfr_plan_upload_frame": (i, [vp, vp, vp, vp, vp, vp]),
        "bmfr_denoise_frame": (i, [vp, fp, fp, vp]),
        "bmfr_denoise_frame_io": (i, [vp, C.POINTER(FrameIO), fp, fp, vp]),
        "bmfr_denoise_frames": (i, [vp, i, C.POINTER(FrameIO), fp, fp, vp]),
        "bmfr_plan_result": (i, [vp, C.POINTER(vp)]),
        "bmfr_plan_download_result": (i, [vp, vp, vp]),
        "bmfr_plan_frame_number": (i, [vp]),
        "bmfr_plan_reset": (i, [vp]),
        "bmfr_plan_buffers_get": (i, [vp, C.POINTER(PlanBuffers)]),
        "bmfr_plan_keep_intermediates": (i, [vp, i]),
        "bmfr_plan_enable_profiling": (i, [vp, i]),
        "bmfr_plan_check_device": (i, [vp, vp]),
        "bmfr_plan_probe_bounded_wait": (i, [vp, C.c_uint, vp]),
        "bmfr_plan_stage_times": (i, [vp, fp]),
        "bmfr_batch_create": (i, [C.POINTER(Params), C.c_size_t, C.POINTER(vp)]),
        "bmfr_batch_destroy": (i, [vp]),
        "bmfr_batch_stream_bytes": (i, [C.POINTER(Params), i, i, i, C.POINTER(C.c_size_t)]),
        "bmfr_batch_add_stream": (i, [vp, i, i, i, C.POINTER(i)]),
        "bmfr_batch_remove_stream": (i, [vp, i]),
        "bmfr_batch_reset_stream": (i, [vp, i]),
        "bmfr_batch_stream_frame": (i, [vp, i]),
        "bmfr_batch_bytes_in_use": (C.c_size_t, [vp]),
        "bmfr_batch_reserve": (i, [vp, C.c_size_t]),
        "bmfr_batch_stream_inputs": (i, [vp, i, C.POINTER(FrameInputs)]),
        "bmfr_batch_step": (i, [vp, i, C.POINTER(i), C.POINTER(FrameIO), fp, fp, vp]),
        "bmfr_batch_stream_result": (i, [vp, i, C.POINTER(vp)]),
        "bmfr_batch_snapshot_bytes": (i, [vp, i, C.POINTER(C.c_size_t)]),
        "bmfr_batch_snapshot": (i, [vp, i, vp, vp]),
        "bmfr_batch_restore": (i, [vp, vp, vp, C.POINTER(i)]),
        "bmfr_server_snapshot_stream": (i, [vp, i, vp, vp]),
        "bmfr_server_restore_stream": (i, [vp, vp, vp, C.POINTER(i)]),
        "bmfr_batch_get_tuning": (i, [vp, C.POINTER(BatchTuning)]),
        "bmfr_batch_set_tuning": (i, [vp, C.POINTER(BatchTuning)]),
        "bmfr_batch_autotune": (i, [vp, i, C.POINTER(i), C.POINTER(FrameIO), fp, fp, i, vp,
                                    C.POINTER(BatchTuning), C.POINTER(C.c_float)]),
        "bmfr_server_create": (i, [C.POINTER(Params), C.POINTER(ServerConfig), C.POINTER(vp)]),
        "bmfr_server_destroy": (i, [vp]),
        "bmfr_server_open_stream": (i, [vp, i, i, C.POINTER(i)]),
        "bmfr_server_close_stream": (i, [vp, i]),
        "bmfr_server_stream_inputs": (i, [vp, i, C.POINTER(FrameInputs)]),
        "bmfr_server_submit": (i, [vp, i, C.POINTER(FrameIO), fp, fp, C.POINTER(C.c_uint64)]),
        "bmfr_server_poll": (i, [vp, C.c_uint64, C.POINTER(i), C.POINTER(C.c_double)]),
        "bmfr_server_drain": (i, [vp, C.c_double]),
        "bmfr_server_stats_get": (i, [vp, C.POINTER(ServerStats)]),
        "bmfr_server_stats_reset": (i, [vp]),
        "bmfr_server_batch": (vp, [vp]),
        "bmfr_server_set_tuning": (i, [vp, C.POINTER(BatchTuning)]),
        "bmfr_last_error": (C.c_char_p, []),
        "bmfr_status_string": (C.c_char_p, [i]),
        "bmfr_write_pfm": (i, [C.c_char_p, i, i, fp]),
        "bmfr_read_pfm": (i, [C.c_char_p, C.POINTER(i), C.POINTER(i), fp, C.c_size_t]),
        "bmfr_psnr": (C.c_double, [fp, fp, C.c_size_t, f]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


class BmfrError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = lib.bmfr_last_error().decode()
        super().__init__(f"{where}: {lib.bmfr_status_string(status).decode()} ({status}): {msg}")
        self.status = status


def check(status: int, where: str) -> None:
    if status != BMFR_OK:
        raise BmfrError(status, where)


def library_path() -> str:
    return os.fspath(_LIB_PATH)
