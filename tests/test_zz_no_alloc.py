"""bmfr_fitter_noalloc, the fitter entry point that allocates nothing.

Some callers cannot call cudaMalloc — a renderer whose engine owns all device
memory under a fixed budget, or per-frame code that cannot afford the device
synchronisation an allocation may cause — so this entry point keeps the
fitter's scratch (the frame's noise table and a status word) in a static
device array of the library instead of a plan's buffers.  This test calls it
through the C ABI and checks its weights and min/max values against the
plan-based bmfr_fitter on two calls in a row: each call must rewrite the
shared array, so the second call (another frame, another block content) must
not see anything left over from the first.
"""
import ctypes as C

import numpy as np
import pytest

import bmfr_b200 as B
from bmfr_b200 import _native
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def _tmp_for(sc, o, frame):
    """tmp_data of `frame` as the oracle's accumulate_noisy_data writes it."""
    W, H = o.width, o.height
    d, dp = sc.render(frame), sc.render(max(frame - 1, 0))
    tmp = o.new_tmp()
    o.accumulate_noisy_data(np.zeros((H, W, 2), np.float32), np.zeros((H, W), np.uint8), d["normals"],
                            dp["normals"], d["positions"], dp["positions"], d["noisy"].copy(), dp["noisy"],
                            np.ones((H, W), np.uint8), np.zeros((H, W), np.uint8), tmp, sc.prev_camera(frame),
                            sc.pixel_offset(frame), frame)
    return tmp


def test_fitter_noalloc_matches_fitter_on_two_calls(cuda):
    import torch
    W, H = 160, 96
    sc = B.Scene(31, W, H, 12)
    o = Oracle(W, H, sc.position_limit_squared, sc.normal_limit_squared)
    params = B.default_params(position_limit_squared=sc.position_limit_squared,
                              normal_limit_squared=sc.normal_limit_squared)
    plan = B.Plan(W, H, params=params)
    nb = plan.sizes.blocks
    stream = torch.cuda.current_stream()
    for frame in (5, 6):
        tmp = torch.from_numpy(_tmp_for(sc, o, frame)).to(cuda)
        w_ref = torch.zeros(nb * 30, dtype=torch.float32, device=cuda)
        mm_ref = torch.zeros(nb * 12, dtype=torch.float32, device=cuda)
        B.fitter(plan, w_ref, mm_ref, tmp, frame)
        w_na = torch.full((nb * 30,), float("nan"), dtype=torch.float32, device=cuda)
        mm_na = torch.full((nb * 12,), float("nan"), dtype=torch.float32, device=cuda)
        st = _native.lib.bmfr_fitter_noalloc(C.byref(params), W, H, C.c_void_p(w_na.data_ptr()),
                                            C.c_void_p(mm_na.data_ptr()), C.c_void_p(tmp.data_ptr()), frame,
                                            C.c_void_p(stream.cuda_stream))
        assert st == 0, _native.lib.bmfr_last_error().decode()
        torch.cuda.synchronize()
        a, b = w_na.cpu().numpy(), w_ref.cpu().numpy()
        assert np.isfinite(a).all()
        # Same tolerance as the parity tests: |a - b| <= 1e-3 * max(|b|, 1e-2);
        # the two entry points run the same kernel, so the values are equal.
        assert (np.abs(a - b) <= 1e-3 * np.maximum(np.abs(b), 1e-2)).all(), f"weights, frame {frame}"
        np.testing.assert_array_equal(mm_na.cpu().numpy(), mm_ref.cpu().numpy())
    plan.close()


def test_fitter_noalloc_rejects_bad_sizes(cuda):
    params = B.default_params()
    for w, h in ((16, 64), (20000, 64), (33, 64)):
        st = _native.lib.bmfr_fitter_noalloc(C.byref(params), w, h, C.c_void_p(1 << 20), C.c_void_p(1 << 20),
                                            C.c_void_p(1 << 20), 0, C.c_void_p(0))
        assert st != 0
        assert _native.lib.bmfr_last_error().decode()
