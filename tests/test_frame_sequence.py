"""bmfr_denoise_frames: consecutive frames in one call, each frame's
accumulation overlapped with the previous frame's fitter, weighted sum and
TAA (staged pipeline).  The outputs must equal, bit for bit, those of one
bmfr_denoise_frame_io call per frame (the path the other parity tests pin to
the oracle), and the first case is also checked against the oracle's frame
loop directly (opencl/bmfr.cpp:417-485)."""
import ctypes as C

import numpy as np
import pytest

import bmfr_b200 as B
from bmfr_b200 import _native
from oracle.oracle import Oracle, OraclePipeline

from test_parity_pipeline import device_array
from test_parity_stages import assert_close

pytestmark = pytest.mark.gpu


def _device_frames(sc, n, cuda):
    import torch
    out = []
    for f in range(n):
        d = sc.render(f)
        out.append({k: torch.from_numpy(np.ascontiguousarray(d[k], dtype=np.float32)).reshape(-1).to(cuda)
                    for k in ("albedo", "normals", "positions", "noisy")})
    torch.cuda.synchronize()
    return out


def _io(frames, f, result):
    p = frames[max(f - 1, 0)]
    return dict(frames[f], previous_normals=p["normals"], previous_positions=p["positions"], result=result)


def _frame_by_frame(plan, sc, frames, cuda):
    import torch
    n = plan.width * plan.height * 3
    out = []
    for f in range(len(frames)):
        r = torch.empty(n, dtype=torch.float32, device=cuda)
        io = _io(frames, f, r)
        plan.denoise_frame_io(io["albedo"], io["normals"], io["positions"], io["noisy"], io["previous_normals"],
                              io["previous_positions"], sc.prev_camera(f), sc.pixel_offset(f), result=r)
        out.append(r)
    torch.cuda.synchronize()
    return [r.cpu().numpy() for r in out]


def _buffers(plan, staged):
    """The last frame's intermediates that a sequence writes into its
    alternating buffer set (bmfr_plan_buffers_get must return that set)."""
    H, W = plan.height, plan.width
    b = plan.buffers()
    out = {"weights": device_array(b.weights, (plan.sizes.blocks * 30,), np.float32),
           "accept": device_array(b.accept, (H, W), np.uint8),
           "prev_frame_pixel": device_array(b.prev_frame_pixel, (H, W, 2), np.float32)}
    if staged:
        out["tmp_data"] = device_array(b.tmp_data, (plan.sizes.tmp_data_bytes,), np.uint8)
    return out


# 128x96 over 17 frames: every BLOCK_OFFSETS entry (opencl/bmfr.cl:267-285)
# through the overlapped path; 1280x720: 984 blocks per frame; binary16
# histories with CholeskyQR2 (the precision form); the fused pipeline runs
# its frames one after another.  `calls` splits the frames over several calls
# (a call of one frame does not overlap; later calls continue the histories).
@pytest.mark.parametrize("W,H,calls,kw", [
    (128, 96, [2, 15], {}),
    (1280, 720, [4], {}),
    (256, 192, [1, 3, 2], {"half_history": 1, "fp32_qr": 1}),
    (200, 120, [5], {"pipeline": B.PIPELINE_FUSED}),
])
def test_sequence_equals_frame_by_frame(cuda, W, H, calls, kw):
    import torch
    n_frames = sum(calls)
    sc = B.Scene(41, W, H, 12)
    mk = lambda: B.Plan(W, H, position_limit_squared=sc.position_limit_squared,
                        normal_limit_squared=sc.normal_limit_squared, **kw)
    seq, one = mk(), mk()
    pool = _device_frames(sc, n_frames, cuda)
    want = _frame_by_frame(one, sc, pool, cuda)
    n = W * H * 3
    results = [torch.empty(n, dtype=torch.float32, device=cuda) for _ in range(n_frames)]
    f0 = 0
    for count in calls:
        # Inputs land in fresh buffers by copies queued on the same stream
        # just before the call, with no synchronisation: the overlapped
        # accumulations must start after them.
        frames = []
        for f in range(n_frames):
            frames.append({k: torch.full((n,), float("nan"), device=cuda) for k in pool[f]}
                          if f0 <= f < f0 + count else pool[f])
        for f in range(f0, f0 + count):
            for k in pool[f]:
                frames[f][k].copy_(pool[f][k])
        ios = [_io(frames, f, results[f]) for f in range(f0, f0 + count)]
        seq.denoise_frames(ios, [sc.prev_camera(f) for f in range(f0, f0 + count)],
                           [sc.pixel_offset(f) for f in range(f0, f0 + count)])
        f0 += count
    torch.cuda.synchronize()
    assert seq.frame_number == n_frames
    for f in range(n_frames):
        np.testing.assert_array_equal(results[f].cpu().numpy(), want[f], err_msg=f"frame {f}")
    got_last = device_array(seq.result_ptr(), (n,), np.float32)
    np.testing.assert_array_equal(got_last, want[-1])
    staged = kw.get("pipeline", B.PIPELINE_STAGED) == B.PIPELINE_STAGED
    a, b = _buffers(seq, staged), _buffers(one, staged)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    if W == 128:
        ref = OraclePipeline(Oracle(W, H, sc.position_limit_squared, sc.normal_limit_squared))
        for f in range(n_frames):
            d = sc.render(f)
            r = ref.step(d["albedo"], d["normals"], d["positions"], d["noisy"], sc.prev_camera(f),
                         sc.pixel_offset(f))
            assert_close(results[f].cpu().numpy().reshape(H, W, 3), r, f"oracle frame {f}", rtol=1e-4)
    seq.close()
    one.close()


def test_sequence_between_single_frames(cuda):
    """Single-frame calls and sequences interleave on one plan: frames 0, 1-3,
    4, 5-8 equal one call per frame, bit for bit.  The last sequence runs
    with stage profiling on, which keeps its frames in stream order, and
    leaves the last frame's stage times readable."""
    import torch
    W, H = 160, 96
    sc = B.Scene(43, W, H, 12)
    mk = lambda: B.Plan(W, H, position_limit_squared=sc.position_limit_squared,
                        normal_limit_squared=sc.normal_limit_squared)
    mixed, one = mk(), mk()
    pool = _device_frames(sc, 9, cuda)
    want = _frame_by_frame(one, sc, pool, cuda)
    n = W * H * 3
    results = [torch.empty(n, dtype=torch.float32, device=cuda) for _ in range(9)]
    for lo, hi in [(0, 1), (1, 4), (4, 5), (5, 9)]:
        if hi - lo == 1:
            io = _io(pool, lo, results[lo])
            mixed.denoise_frame_io(io["albedo"], io["normals"], io["positions"], io["noisy"],
                                   io["previous_normals"], io["previous_positions"], sc.prev_camera(lo),
                                   sc.pixel_offset(lo), result=results[lo])
        else:
            mixed.enable_profiling(lo == 5)
            mixed.denoise_frames([_io(pool, f, results[f]) for f in range(lo, hi)],
                                 [sc.prev_camera(f) for f in range(lo, hi)], [sc.pixel_offset(f) for f in range(lo, hi)])
    torch.cuda.synchronize()
    for f in range(9):
        np.testing.assert_array_equal(results[f].cpu().numpy(), want[f], err_msg=f"frame {f}")
    times = mixed.stage_times()
    assert len(times) == 4 and all(v > 0 for v in times.values()), times
    mixed.close()
    one.close()


def test_sequence_rejects_bad_arguments(cuda):
    """Every frame is checked before any is queued: a NULL input in the
    second entry, or a missing previous G-buffer after frame 0, fails with
    BMFR_E_INVALID and leaves the frame counter where it was."""
    import torch
    W, H = 64, 64
    sc = B.Scene(44, W, H, 8)
    plan = B.Plan(W, H, position_limit_squared=sc.position_limit_squared,
                  normal_limit_squared=sc.normal_limit_squared)
    pool = _device_frames(sc, 2, cuda)
    p = lambda t: C.c_void_p(t.data_ptr())
    nil = C.c_void_p(None)
    ios = (_native.FrameIO * 2)()
    ios[0] = _native.FrameIO(p(pool[0]["albedo"]), p(pool[0]["normals"]), p(pool[0]["positions"]),
                             p(pool[0]["noisy"]), nil, nil, nil)
    ios[1] = _native.FrameIO(nil, p(pool[1]["normals"]), p(pool[1]["positions"]), p(pool[1]["noisy"]),
                             p(pool[0]["normals"]), p(pool[0]["positions"]), nil)
    mats = np.zeros(32, np.float32)
    offs = np.zeros(4, np.float32)
    fp = C.POINTER(C.c_float)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    call = lambda k: _native.lib.bmfr_denoise_frames(plan.handle, k, ios, mats.ctypes.data_as(fp),
                                                     offs.ctypes.data_as(fp), stream)
    assert call(2) == _native.BMFR_E_INVALID
    assert "io[1]" in _native.lib.bmfr_last_error().decode()
    assert call(-1) == _native.BMFR_E_INVALID
    assert call(0) == 0
    assert plan.frame_number == 0
    # Frame 1 (second entry) without its previous G-buffer.
    ios[1] = _native.FrameIO(p(pool[1]["albedo"]), p(pool[1]["normals"]), p(pool[1]["positions"]),
                             p(pool[1]["noisy"]), nil, nil, nil)
    assert call(2) == _native.BMFR_E_INVALID
    assert plan.frame_number == 0
    torch.cuda.synchronize()
    plan.close()
