"""Batch and server steps holding streams of the batched and served
workloads' largest sizes (3840x2160 and 1920x1080) beside small ones: every
stream's output must equal, bit for bit, what its own plan gives alone."""
import numpy as np
import pytest

import bmfr_b200 as B
from test_batch import Stream, _device_result

pytestmark = pytest.mark.gpu

SIZES = [(3840, 2160), (1920, 1080), (96, 64), (200, 120)]


@pytest.mark.parametrize("pipeline", [B.PIPELINE_STAGED, B.PIPELINE_FUSED])
@pytest.mark.parametrize("qr", [B.QR_REFERENCE, B.QR_CHOLESKY2])
def test_batch_step_with_4k_and_1080p_streams(cuda, qr, pipeline):
    import torch
    kw = dict(fp32_qr=qr, half_history=1) if qr != B.QR_REFERENCE else {}
    params = B.default_params(pipeline=pipeline, **kw)
    streams = [Stream(60 + k, w, h, params, cuda) for k, (w, h) in enumerate(SIZES)]
    batch = B.Batch(params)
    slots = [batch.add_stream(s.w, s.h) for s in streams]
    for f in range(2):
        io = [s.io(f) for s in streams]
        mats = np.concatenate([s.sc.prev_camera(f) for s in streams])
        offs = np.concatenate([s.sc.pixel_offset(f) for s in streams])
        batch.step(slots, mats, offs, io=io)
        for k, s in enumerate(streams):
            want = s.plan_step(f).cpu().numpy().reshape(s.h, s.w, 3)
            got = _device_result(batch.result_ptr(slots[k]), s.w, s.h)
            np.testing.assert_array_equal(got, want, err_msg=f"{s.w}x{s.h} frame {f}")
    torch.cuda.synchronize()
    batch.close()
    for s in streams:
        s.plan.close()


@pytest.mark.parametrize("pipeline", [B.PIPELINE_STAGED, B.PIPELINE_FUSED])
def test_server_with_4k_and_1080p_streams(cuda, pipeline):
    import torch
    params = B.default_params(pipeline=pipeline, fp32_qr=B.QR_CHOLESKY2, half_history=1)
    streams = [Stream(70 + k, w, h, params, cuda) for k, (w, h) in enumerate(SIZES)]
    server = B.Server(params)
    ids = [server.open_stream(s.w, s.h) for s in streams]
    frames = 2
    for s in streams:
        s.frame(frames - 1)
    outs = {}
    for f in range(frames):
        for k, s in enumerate(streams):
            out = torch.empty(s.w * s.h * 3, dtype=torch.float32, device=cuda)
            outs[(k, f)] = out
            io = s.io(f)
            io.result = out.data_ptr()
            server.submit(ids[k], s.sc.prev_camera(f), s.sc.pixel_offset(f), io=io)
    server.drain(120000)
    torch.cuda.synchronize()
    st = server.stats()
    assert st["requests_completed"] == st["requests_submitted"] == frames * len(streams)
    for k, s in enumerate(streams):
        for f in range(frames):
            want = s.plan_step(f).cpu().numpy()
            np.testing.assert_array_equal(outs[(k, f)].cpu().numpy(), want, err_msg=f"{s.w}x{s.h} frame {f}")
    server.close()
    for s in streams:
        s.plan.close()
