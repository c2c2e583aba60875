"""bmfr_scene — seeded procedural G-buffer source for the BMFR pipeline
(include/bmfr_scene.h, library bmfr_scene/libbmfr_scene.so).

The reference reads 60 EXR frames of features and its camera matrices from
a dataset header (opencl/bmfr.cpp:44-53, 145-172); neither exists here, so
this library renders an equivalent input stream on the host cores or on the
GPU.  It is a separate library from the denoising pipeline
(bmfr_b200/libbmfr_b200.so), so code that only needs inputs, such as a CPU
baseline, maps no pipeline code.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

__all__ = ["Scene", "SceneDesc", "SceneError", "library_path"]

_LIB_PATH = Path(__file__).resolve().parent / "libbmfr_scene.so"


class SceneDesc(C.Structure):
    _fields_ = [
        ("seed", C.c_uint64), ("width", C.c_int), ("height", C.c_int),
        ("sphere_count", C.c_int), ("orbit_degrees_per_frame", C.c_float),
        ("orbit_start_degrees", C.c_float), ("orbit_radius", C.c_float),
        ("camera_height", C.c_float), ("vertical_fov_degrees", C.c_float),
        ("noise_mu", C.c_float), ("noise_sigma", C.c_float),
        ("firefly_fraction", C.c_float), ("firefly_scale", C.c_float),
        ("plane_half_extent", C.c_float), ("position_limit_squared", C.c_float),
        ("normal_limit_squared", C.c_float),
    ]


def _load() -> C.CDLL:
    if not _LIB_PATH.exists():
        raise ImportError(f"{_LIB_PATH} is missing: build it with `python bmfr_b200/build.py`")
    lib = C.CDLL(str(_LIB_PATH))
    i, fp, vp = C.c_int, C.POINTER(C.c_float), C.c_void_p
    d = C.POINTER(SceneDesc)
    sig = {
        "bmfr_scene_default": (i, [d, C.c_uint64, i, i, i]),
        "bmfr_scene_camera": (i, [d, i, fp]),
        "bmfr_scene_pixel_offset": (i, [d, i, fp]),
        "bmfr_scene_render": (i, [d, i, fp, fp, fp, fp, fp, i]),
        "bmfr_scene_render_device": (i, [d, i, vp, vp, vp, vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


class SceneError(RuntimeError):
    def __init__(self, status: int, where: str):
        super().__init__(f"{where} failed with status {status}")
        self.status = status


def _check(status: int, where: str) -> None:
    if status != 0:
        raise SceneError(status, where)


def library_path() -> str:
    return os.fspath(_LIB_PATH)


def _dev(t, name: str, nbytes: int, optional: bool = False) -> C.c_void_p:
    if t is None:
        if optional:
            return C.c_void_p(None)
        raise ValueError(f"{name} must not be None")
    if isinstance(t, int):
        return C.c_void_p(t)
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError(f"{name} must be a contiguous CUDA tensor")
    if t.numel() * t.element_size() < nbytes:
        raise ValueError(f"{name} holds {t.numel() * t.element_size()} bytes, needs {nbytes}")
    return C.c_void_p(t.data_ptr())


def _stream(stream) -> C.c_void_p:
    if stream is None:
        import torch
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(stream.cuda_stream)


class Scene:
    """Seeded procedural stand-in for the reference's EXR dataset and
    camera_matrices.h (opencl/bmfr.cpp:44-53, 145-172)."""

    def __init__(self, seed: int, width: int, height: int, sphere_count: int = 12, **overrides):
        d = SceneDesc()
        _check(lib.bmfr_scene_default(C.byref(d), int(seed), int(width), int(height), int(sphere_count)),
               "bmfr_scene_default")
        for k, v in overrides.items():
            if not hasattr(d, k):
                raise AttributeError(f"unknown scene field {k!r}")
            setattr(d, k, v)
        self.desc = d
        self.width, self.height = width, height

    @property
    def position_limit_squared(self) -> float:
        return self.desc.position_limit_squared

    @property
    def normal_limit_squared(self) -> float:
        return self.desc.normal_limit_squared

    def camera(self, frame: int) -> np.ndarray:
        m = np.empty(16, dtype=np.float32)
        _check(lib.bmfr_scene_camera(C.byref(self.desc), int(frame), m.ctypes.data_as(C.POINTER(C.c_float))),
               "bmfr_scene_camera")
        return m

    def prev_camera(self, frame: int) -> np.ndarray:
        """camera_matrices[max(frame - 1, 0)], the matrix frame `frame` uses
        (opencl/bmfr.cpp:440-442)."""
        return self.camera(max(frame - 1, 0))

    def pixel_offset(self, frame: int) -> np.ndarray:
        o = np.empty(2, dtype=np.float32)
        _check(lib.bmfr_scene_pixel_offset(C.byref(self.desc), int(frame), o.ctypes.data_as(C.POINTER(C.c_float))),
               "bmfr_scene_pixel_offset")
        return o

    def render(self, frame: int, clean: bool = False, threads: int = 0) -> dict:
        H, W = self.height, self.width
        out = {k: np.empty((H, W, 3), dtype=np.float32) for k in ("albedo", "normals", "positions", "noisy")}
        cl = np.empty((H, W, 3), dtype=np.float32) if clean else None
        fp = C.POINTER(C.c_float)
        _check(lib.bmfr_scene_render(C.byref(self.desc), int(frame), out["albedo"].ctypes.data_as(fp),
                                     out["normals"].ctypes.data_as(fp), out["positions"].ctypes.data_as(fp),
                                     out["noisy"].ctypes.data_as(fp),
                                     cl.ctypes.data_as(fp) if cl is not None else None, int(threads)),
               "bmfr_scene_render")
        if cl is not None:
            out["clean"] = cl
        return out

    def render_device(self, frame: int, albedo, normals, positions, noisy, clean=None, stream=None) -> None:
        """Renders frame `frame` on the GPU into device tensors (H*W*3 float32)."""
        n = self.width * self.height * 12
        _check(lib.bmfr_scene_render_device(C.byref(self.desc), int(frame), _dev(albedo, "albedo", n),
                                            _dev(normals, "normals", n), _dev(positions, "positions", n),
                                            _dev(noisy, "noisy", n), _dev(clean, "clean", n, optional=True),
                                            _stream(stream)), "bmfr_scene_render_device")
