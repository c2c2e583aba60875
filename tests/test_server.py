"""The request server (continuous batching over the many-stream engine).

Frames of several streams are submitted while earlier steps run; every
result must equal what the stream's own plan produces alone (same
parameters and pipeline), streams are admitted against the memory budget,
and the statistics account for every request.
"""
import threading
import time

import numpy as np
import pytest

import bmfr_b200 as B
from test_batch import SIZES, Stream

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("pipeline", [B.PIPELINE_FUSED, B.PIPELINE_STAGED])
def test_results_alone_and_in_the_mix(cuda, pipeline):
    import torch
    params = B.default_params(pipeline=pipeline, fp32_qr=1, half_history=1)
    streams = [Stream(k, w, h, params, cuda) for k, (w, h) in enumerate(SIZES)]
    server = B.Server(params)
    ids = [server.open_stream(s.w, s.h) for s in streams]
    frames = 5
    for s in streams:   # render every frame up front; submissions must not wait on the host renderer
        s.frame(frames - 1)
    outs = {}

    def client(k):
        s = streams[k]
        rng = np.random.default_rng(k)
        for f in range(frames):
            out = torch.empty(s.w * s.h * 3, dtype=torch.float32, device=cuda)
            outs[(k, f)] = out
            io = s.io(f)
            io.result = out.data_ptr()
            server.submit(ids[k], s.sc.prev_camera(f), s.sc.pixel_offset(f), io=io)
            time.sleep(float(rng.uniform(0.0, 0.004)))   # arrivals interleave with steps

    threads = [threading.Thread(target=client, args=(k,)) for k in range(len(streams))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    server.drain(60000)
    torch.cuda.synchronize()
    st = server.stats()
    assert st["requests_completed"] == st["requests_submitted"] == frames * len(streams)
    assert st["p99_latency_ms"] >= st["p50_latency_ms"] > 0
    # Alone: each stream through its own plan.
    for k, s in enumerate(streams):
        for f in range(frames):
            want = s.plan_step(f).cpu().numpy()
            np.testing.assert_array_equal(outs[(k, f)].cpu().numpy(), want, err_msg=f"stream {k} frame {f}")
    server.close()


def test_admission_against_the_budget(cuda):
    params = B.default_params(pipeline=B.PIPELINE_FUSED, fp32_qr=1, half_history=1)
    need = B.Batch.stream_bytes(params, 320, 180)
    server = B.Server(params, memory_budget_bytes=2 * need + need // 2)
    a = server.open_stream(320, 180)
    b = server.open_stream(320, 180)
    with pytest.raises(B.BmfrError) as e:
        server.open_stream(320, 180)
    assert e.value.status == B._native.BMFR_E_BUDGET
    server.close_stream(a)                  # memory frees up ...
    c = server.open_stream(320, 180)        # ... and the next stream is admitted (in the freed slot)
    assert c != b
    st = server.stats()
    assert st["streams_admitted"] == 3 and st["streams_rejected"] == 1
    server.close_stream(c)
    with pytest.raises(B.BmfrError):
        server.submit(c, np.eye(4), [0.5, 0.5])   # closed stream
    with pytest.raises(B.BmfrError):
        server.submit(999, np.eye(4), [0.5, 0.5])   # never opened
    server.close()


def test_stream_moves_between_servers(cuda):
    """A stream snapshotted in one server and restored in another carries on
    with identical frames (serving migration between two frames)."""
    import torch
    params = B.default_params(pipeline=B.PIPELINE_STAGED, fp32_qr=1, half_history=1)
    st = Stream(2, 128, 128, params, cuda)
    one, two = B.Server(params), B.Server(params)
    sid = one.open_stream(st.w, st.h)

    def submit(server, s, f):
        out = torch.empty(st.w * st.h * 3, dtype=torch.float32, device=cuda)
        io = st.io(f)
        io.result = out.data_ptr()
        server.submit(s, st.sc.prev_camera(f), st.sc.pixel_offset(f), io=io)
        return out

    for f in range(3):
        submit(one, sid, f)
    snap = np.empty(B.Batch.stream_bytes(params, st.w, st.h), dtype=np.uint8)   # at least the snapshot's size
    one.snapshot_stream(sid, snap)
    want = [submit(one, sid, f) for f in range(3, 6)]
    one.drain()
    moved = two.restore_stream(snap)
    got = [submit(two, moved, f) for f in range(3, 6)]
    two.drain()
    torch.cuda.synchronize()
    for k in range(3):
        np.testing.assert_array_equal(got[k].cpu().numpy(), want[k].cpu().numpy(), err_msg=f"frame {3 + k}")
    one.close()
    two.close()


def test_router_over_two_servers_places_and_migrates(cuda):
    """The host-side router over two servers (two GPUs' worth, here on one
    device): streams go where the budget has room, requests follow their
    stream, and a stream moved between servers mid-sequence gives the frames
    its own plan gives."""
    import torch
    params = B.default_params(pipeline=B.PIPELINE_STAGED, fp32_qr=1, half_history=1)
    one_stream = B.Batch.stream_bytes(params, 200, 120)
    router = B.Router([B.Server(params), B.Server(params)], budget_bytes=2 * one_stream,
                      stream_bytes=lambda w, h: B.Batch.stream_bytes(params, w, h))
    streams = [Stream(80 + k, 200, 120, params, cuda) for k in range(3)]
    ids = [router.open_stream(s.w, s.h) for s in streams]
    assert sorted(router.gpu_of(i) for i in ids) == [0, 0, 1]
    outs = {}

    def submit(k, f):
        s = streams[k]
        out = torch.empty(s.w * s.h * 3, dtype=torch.float32, device=cuda)
        io = s.io(f)
        io.result = out.data_ptr()
        router.submit(ids[k], s.sc.prev_camera(f), s.sc.pixel_offset(f), io=io)
        outs[(k, f)] = out

    for f in range(2):
        for k in range(3):
            submit(k, f)
    moved = next(i for i, g in enumerate(router.gpu_of(x) for x in ids) if g == 0)
    assert router.migrate(ids[moved]) == 1               # the other server had room for one more
    for f in range(2, 4):
        for k in range(3):
            submit(k, f)
    router.drain()
    torch.cuda.synchronize()
    for k, s in enumerate(streams):
        for f in range(4):
            np.testing.assert_array_equal(outs[(k, f)].cpu().numpy(), s.plan_step(f).cpu().numpy(),
                                          err_msg=f"stream {k} frame {f}")
    router.close()
    for srv in router.servers:
        srv.close()
