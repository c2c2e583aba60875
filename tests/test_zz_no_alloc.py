"""bmfr_fitter_noalloc, the fitter entry point that allocates nothing.

Some callers cannot call cudaMalloc — a renderer whose engine owns all device
memory under a fixed budget, or per-frame code that cannot afford the device
synchronisation an allocation may cause — so this entry point keeps the
fitter's scratch (the frame's noise table and a status word) in a static
device array of the library instead of a plan's buffers.  These tests call
it through the C ABI on two calls in a row and check its weights and min/max
values bit for bit against the oracle and against the plan-based
bmfr_fitter: each call must rewrite the shared array, so the second call
(another frame, other block contents) must see nothing left over from the
first.  A bounded wait that runs out inside it must reach the caller through
bmfr_fitter_noalloc_check.
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


def _noalloc(params, W, H, w, mm, tmp, frame, stream):
    st = _native.lib.bmfr_fitter_noalloc(C.byref(params), W, H, C.c_void_p(w.data_ptr()), C.c_void_p(mm.data_ptr()),
                                        C.c_void_p(tmp.data_ptr()), frame, C.c_void_p(stream.cuda_stream))
    assert st == 0, _native.lib.bmfr_last_error().decode()


def _check(stream):
    return _native.lib.bmfr_fitter_noalloc_check(C.c_void_p(stream.cuda_stream))


# 160x96: 24 blocks; 1280x720: 984 blocks, more than the persistent grid,
# so CTAs walk several blocks through both tile buffers; float32 tmp_data
# takes the one-dimensional bulk copy.
@pytest.mark.parametrize("W,H,use_half", [(160, 96, 1), (1280, 720, 1), (160, 96, 0)])
def test_fitter_noalloc_matches_oracle_on_two_calls(cuda, W, H, use_half):
    import torch
    sc = B.Scene(31, W, H, 12)
    o = Oracle(W, H, sc.position_limit_squared, sc.normal_limit_squared, use_half=bool(use_half))
    params = B.default_params(position_limit_squared=sc.position_limit_squared,
                              normal_limit_squared=sc.normal_limit_squared, use_half_precision_in_tmp_data=use_half)
    plan = B.Plan(W, H, params=params)
    nb = plan.sizes.blocks
    stream = torch.cuda.current_stream()
    for frame in (5, 6):
        tmp_host = _tmp_for(sc, o, frame)
        tmp = torch.from_numpy(tmp_host.copy()).to(cuda)
        w_or = np.zeros(nb * 30, np.float32)
        mm_or = np.zeros(nb * 12, np.float32)
        o.fitter(w_or, mm_or, tmp_host.copy(), frame)
        w_ref = torch.zeros(nb * 30, dtype=torch.float32, device=cuda)
        mm_ref = torch.zeros(nb * 12, dtype=torch.float32, device=cuda)
        B.fitter(plan, w_ref, mm_ref, tmp, frame)
        w_na = torch.full((nb * 30,), float("nan"), dtype=torch.float32, device=cuda)
        mm_na = torch.full((nb * 12,), float("nan"), dtype=torch.float32, device=cuda)
        _noalloc(params, W, H, w_na, mm_na, tmp, frame, stream)
        assert _check(stream) == 0, _native.lib.bmfr_last_error().decode()
        a, b = w_na.cpu().numpy(), w_ref.cpu().numpy()
        # Bit for bit: the oracle restates the reference's arithmetic, and the
        # two entry points run the same fit.
        np.testing.assert_array_equal(a, w_or, err_msg=f"weights vs oracle, frame {frame}")
        np.testing.assert_array_equal(mm_na.cpu().numpy(), mm_or, err_msg=f"mins_maxs vs oracle, frame {frame}")
        np.testing.assert_array_equal(a, b, err_msg=f"weights vs bmfr_fitter, frame {frame}")
        np.testing.assert_array_equal(mm_na.cpu().numpy(), mm_ref.cpu().numpy())
    plan.close()


def test_fitter_noalloc_reports_a_bounded_wait_that_ran_out(cuda):
    """The failure path without a fault: a diagnostic wait on the static
    array's status word runs out after 20 ms; the check reports
    BMFR_E_TIMEOUT once, clears the word, and the entry point then fits
    exactly as before."""
    import torch
    stream = torch.cuda.current_stream()
    assert _check(stream) == 0
    assert _native.lib.bmfr_fitter_noalloc_probe_bounded_wait(20000, C.c_void_p(stream.cuda_stream)) == 0
    assert _check(stream) == _native.BMFR_E_TIMEOUT
    assert "bounded wait" in _native.lib.bmfr_last_error().decode()
    assert _check(stream) == 0                     # cleared
    for bad in (0, 2_000_000):
        assert _native.lib.bmfr_fitter_noalloc_probe_bounded_wait(bad, C.c_void_p(stream.cuda_stream)) != 0

    W, H = 96, 64
    sc = B.Scene(32, W, H, 8)
    o = Oracle(W, H, sc.position_limit_squared, sc.normal_limit_squared)
    params = B.default_params(position_limit_squared=sc.position_limit_squared,
                              normal_limit_squared=sc.normal_limit_squared)
    tmp_host = _tmp_for(sc, o, 3)
    nb = o.blocks
    w_or, mm_or = np.zeros(nb * 30, np.float32), np.zeros(nb * 12, np.float32)
    o.fitter(w_or, mm_or, tmp_host.copy(), 3)
    tmp = torch.from_numpy(tmp_host.copy()).to(cuda)
    w = torch.empty(nb * 30, dtype=torch.float32, device=cuda)
    mm = torch.empty(nb * 12, dtype=torch.float32, device=cuda)
    _noalloc(params, W, H, w, mm, tmp, 3, stream)
    assert _check(stream) == 0
    np.testing.assert_array_equal(w.cpu().numpy(), w_or)
    np.testing.assert_array_equal(mm.cpu().numpy(), mm_or)


def test_fitter_noalloc_rejects_bad_sizes(cuda):
    params = B.default_params()
    for w, h in ((16, 64), (20000, 64), (33, 64)):
        st = _native.lib.bmfr_fitter_noalloc(C.byref(params), w, h, C.c_void_p(1 << 20), C.c_void_p(1 << 20),
                                            C.c_void_p(1 << 20), 0, C.c_void_p(0))
        assert st != 0
        assert _native.lib.bmfr_last_error().decode()
