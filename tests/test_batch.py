"""The many-stream engine (include/bmfr_batch.h): every stream's output in a
batch step must equal what a plan with the same parameters (the same
pipeline, fused or staged) produces for that stream alone — bit for bit,
since both run the same per-pixel and per-block bodies — whatever other
streams share the step."""
import numpy as np
import pytest

import bmfr_b200 as B

pytestmark = pytest.mark.gpu

SIZES = [(96, 64), (160, 96), (128, 128), (200, 120)]


class Stream:
    """One render stream: its scene, device frames and a reference plan."""

    def __init__(self, k, w, h, params, dev):
        import torch
        self.w, self.h = w, h
        self.sc = B.Scene(100 + k, w, h, 8 + 4 * k, orbit_degrees_per_frame=0.3 + 0.2 * k)
        self.frames = []
        self.dev = dev
        self.plan = B.Plan(w, h, params=params)
        self.torch = torch

    def frame(self, f):
        while len(self.frames) <= f:
            d = self.sc.render(len(self.frames))
            self.frames.append({k: self.torch.from_numpy(v).to(self.dev) for k, v in d.items()})
        return self.frames[f]

    def io(self, f):
        d, p = self.frame(f), self.frame(max(f - 1, 0))
        return B.Batch.frame_io(d["albedo"], d["normals"], d["positions"], d["noisy"], p["normals"], p["positions"])

    def plan_step(self, f):
        d, p = self.frame(f), self.frame(max(f - 1, 0))
        out = self.torch.empty(self.w * self.h * 3, dtype=self.torch.float32, device=self.dev)
        self.plan.denoise_frame_io(d["albedo"], d["normals"], d["positions"], d["noisy"], p["normals"],
                                   p["positions"], self.sc.prev_camera(f), self.sc.pixel_offset(f), result=out)
        return out


def _cudart():
    from test_parity_pipeline import _cudart as cudart
    return cudart()


def _device_result(ptr, w, h):
    import torch
    from test_parity_pipeline import device_array
    return device_array(ptr, (h, w, 3), np.float32)


@pytest.mark.parametrize("pipeline", [B.PIPELINE_FUSED, B.PIPELINE_STAGED])
@pytest.mark.parametrize("qr", [B.QR_REFERENCE, B.QR_CHOLESKY2, B.QR_HOUSEHOLDER])
def test_batch_equals_streams_alone(cuda, qr, pipeline):
    import torch
    kw = dict(fp32_qr=qr, half_history=1) if qr != B.QR_REFERENCE else {}
    params = B.default_params(pipeline=pipeline, **kw)
    streams = [Stream(k, w, h, params, cuda) for k, (w, h) in enumerate(SIZES)]
    batch = B.Batch(params)
    slots = [batch.add_stream(s.w, s.h) for s in streams]
    # Step schedule: all, a subset (stream 1 and 3 idle), all, all.
    schedule = [[0, 1, 2, 3], [0, 2], [0, 1, 2, 3], [3, 1, 0, 2]]
    frame = [0] * len(streams)
    for active in schedule:
        io = [streams[i].io(frame[i]) for i in active]
        mats = np.concatenate([streams[i].sc.prev_camera(frame[i]) for i in active])
        offs = np.concatenate([streams[i].sc.pixel_offset(frame[i]) for i in active])
        batch.step([slots[i] for i in active], mats, offs, io=io)
        for i in active:
            want = streams[i].plan_step(frame[i]).cpu().numpy().reshape(streams[i].h, streams[i].w, 3)
            got = _device_result(batch.result_ptr(slots[i]), streams[i].w, streams[i].h)
            np.testing.assert_array_equal(got, want, err_msg=f"stream {i} frame {frame[i]}")
            frame[i] += 1
            assert batch.frame(slots[i]) == frame[i]
    torch.cuda.synchronize()
    batch.close()


def test_staged_step_with_more_streams_than_workers(cuda):
    """Twelve streams (more than the staged step's worker CUDA streams, so a
    worker runs several streams' kernels in turn), all of them, then a
    subset in another order, then all again: every result equals its plan's
    bit for bit, and the whole step is complete when the caller's stream is."""
    import torch
    params = B.default_params(pipeline=B.PIPELINE_STAGED, fp32_qr=B.QR_CHOLESKY2, half_history=1)
    sizes = [SIZES[k % len(SIZES)] for k in range(12)]
    streams = [Stream(20 + k, w, h, params, cuda) for k, (w, h) in enumerate(sizes)]
    batch = B.Batch(params)
    slots = [batch.add_stream(s.w, s.h) for s in streams]
    caller = torch.cuda.Stream(device=cuda)
    schedule = [list(range(12)), [11, 3, 7, 0, 5], list(range(12))]
    frame = [0] * len(streams)
    for active in schedule:
        io = [streams[i].io(frame[i]) for i in active]
        mats = np.concatenate([streams[i].sc.prev_camera(frame[i]) for i in active])
        offs = np.concatenate([streams[i].sc.pixel_offset(frame[i]) for i in active])
        batch.step([slots[i] for i in active], mats, offs, io=io, stream=caller)
        caller.synchronize()
        # Read without a device-wide synchronisation: the worker streams are
        # non-blocking, so only the step's join into `caller` orders them
        # before this copy.
        got = {}
        for i in active:
            out = np.empty((streams[i].h, streams[i].w, 3), np.float32)
            assert _cudart().cudaMemcpy(out.ctypes.data, batch.result_ptr(slots[i]), out.nbytes, 2) == 0
            got[i] = out
        for i in active:
            want = streams[i].plan_step(frame[i]).cpu().numpy().reshape(streams[i].h, streams[i].w, 3)
            np.testing.assert_array_equal(got[i], want, err_msg=f"stream {i} frame {frame[i]}")
            frame[i] += 1
    torch.cuda.synchronize()
    batch.close()


@pytest.mark.parametrize("qr", [B.QR_REFERENCE, B.QR_CHOLESKY2])
def test_fused_step_with_the_pixel_pass(cuda, qr):
    """The fused step with its per-pixel stages as a pass over image tiles
    (the block kernel ends at the fit): every stream still equals its
    plan's output bit for bit, over steps of all streams and of a subset."""
    import torch
    kw = dict(fp32_qr=qr, half_history=1) if qr != B.QR_REFERENCE else {}
    params = B.default_params(pipeline=B.PIPELINE_FUSED, **kw)
    streams = [Stream(50 + k, w, h, params, cuda) for k, (w, h) in enumerate(SIZES)]
    batch = B.Batch(params)
    batch.set_tuning(pixel_pass=1)
    assert batch.tuning.pixel_pass == 1
    slots = [batch.add_stream(s.w, s.h) for s in streams]
    frame = [0] * len(streams)
    for active in ([0, 1, 2, 3], [2, 0], [0, 1, 2, 3]):
        io = [streams[i].io(frame[i]) for i in active]
        mats = np.concatenate([streams[i].sc.prev_camera(frame[i]) for i in active])
        offs = np.concatenate([streams[i].sc.pixel_offset(frame[i]) for i in active])
        batch.step([slots[i] for i in active], mats, offs, io=io)
        for i in active:
            s = streams[i]
            want = s.plan_step(frame[i]).cpu().numpy().reshape(s.h, s.w, 3)
            np.testing.assert_array_equal(_device_result(batch.result_ptr(slots[i]), s.w, s.h), want,
                                          err_msg=f"stream {i} frame {frame[i]}")
            frame[i] += 1
    torch.cuda.synchronize()
    batch.close()


@pytest.mark.parametrize("qr", [B.QR_REFERENCE, B.QR_CHOLESKY2])
def test_fused_step_queue_longer_than_the_grid(cuda, qr):
    """Two 640x360 streams: 572 blocks in the fused step's queue, more than
    its persistent CTAs, so CTAs take several blocks each; every result
    equals its plan's bit for bit."""
    import torch
    kw = dict(fp32_qr=qr, half_history=1) if qr != B.QR_REFERENCE else {}
    params = B.default_params(pipeline=B.PIPELINE_FUSED, **kw)
    streams = [Stream(40 + k, 640, 360, params, cuda) for k in range(2)]
    batch = B.Batch(params)
    slots = [batch.add_stream(s.w, s.h) for s in streams]
    for f in range(3):
        io = [s.io(f) for s in streams]
        mats = np.concatenate([s.sc.prev_camera(f) for s in streams])
        offs = np.concatenate([s.sc.pixel_offset(f) for s in streams])
        batch.step(slots, mats, offs, io=io)
        for k, s in enumerate(streams):
            want = s.plan_step(f).cpu().numpy().reshape(s.h, s.w, 3)
            np.testing.assert_array_equal(_device_result(batch.result_ptr(slots[k]), s.w, s.h), want,
                                          err_msg=f"stream {k} frame {f}")
    torch.cuda.synchronize()
    batch.close()


@pytest.mark.parametrize("pipeline", [B.PIPELINE_FUSED, B.PIPELINE_STAGED])
def test_batch_autotune_and_budget(cuda, pipeline):
    import torch
    params = B.default_params(pipeline=pipeline, fp32_qr=1, half_history=1)
    streams = [Stream(k, w, h, params, cuda) for k, (w, h) in enumerate(SIZES[:3])]
    batch = B.Batch(params)
    slots = [batch.add_stream(s.w, s.h) for s in streams]
    io = [s.io(0) for s in streams]
    mats = np.concatenate([s.sc.prev_camera(0) for s in streams])
    offs = np.concatenate([s.sc.pixel_offset(0) for s in streams])
    t, ms = batch.autotune(slots, mats, offs, io=io, steps=1)
    assert ms > 0 and (t.taa_tile_w, t.taa_tile_h) in [(30, 8), (30, 16), (30, 32), (30, 64)]
    if pipeline == B.PIPELINE_FUSED:
        assert 0 <= t.staging_depth <= 2 and t.block_ctas_per_sm >= 1
    else:   # the staged step launches the plan's kernels: nothing to tune
        assert t.staging_depth == 0
    # After tuning, a reset stream starts over and still matches its plan.
    for s_, sl in zip(streams, slots):
        batch.reset_stream(sl)
    batch.step(slots, mats, offs, io=io)
    for s_, sl in zip(streams, slots):
        want = s_.plan_step(0).cpu().numpy().reshape(s_.h, s_.w, 3)
        np.testing.assert_array_equal(_device_result(batch.result_ptr(sl), s_.w, s_.h), want)
    batch.close()

    need = B.Batch.stream_bytes(params, 200, 120)
    small = B.Batch(params, memory_budget_bytes=need + need // 2)
    small.add_stream(200, 120)
    with pytest.raises(B.BmfrError) as e:
        small.add_stream(200, 120)
    assert e.value.status == B._native.BMFR_E_BUDGET
    assert small.bytes_in_use == need
    small.close()
    torch.cuda.synchronize()


@pytest.mark.parametrize("to_device", [False, True])
def test_snapshot_and_restore(cuda, to_device):
    """A stream snapshotted between frames and restored into another batch
    continues exactly as the original: the next frames are bit-identical."""
    import torch
    params = B.default_params(pipeline=B.PIPELINE_STAGED, fp32_qr=1, half_history=1)
    st = Stream(3, 160, 96, params, cuda)
    a = B.Batch(params)
    sa = a.add_stream(st.w, st.h)

    def step(batch, slot, f):
        batch.step([slot], st.sc.prev_camera(f), st.sc.pixel_offset(f), io=[st.io(f)])
        return _device_result(batch.result_ptr(slot), st.w, st.h)

    for f in range(4):
        step(a, sa, f)
    n = a.snapshot_bytes(sa)
    snap = a.snapshot(sa, out=torch.empty(n, dtype=torch.uint8, device=cuda) if to_device else None)
    want = [step(a, sa, f) for f in range(4, 7)]
    b = B.Batch(params)
    b.add_stream(64, 64)            # another stream first, so the slot differs
    sb = b.restore(snap)
    assert b.frame(sb) == 4
    for k, f in enumerate(range(4, 7)):
        np.testing.assert_array_equal(step(b, sb, f), want[k], err_msg=f"frame {f}")
    other = B.Batch(B.default_params(pipeline=B.PIPELINE_STAGED))   # float histories: another format
    with pytest.raises(B.BmfrError):
        other.restore(snap)
    for x in (a, b, other):
        x.close()
    torch.cuda.synchronize()
