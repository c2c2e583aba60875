"""End-to-end parity of the plan-managed frame pipeline (staged and fused
forms) with the oracle's frame loop, through host-buffer uploads."""
from pathlib import Path

import numpy as np
import pytest

import bmfr_b200 as B
from oracle.oracle import Oracle, OraclePipeline

from test_parity_stages import assert_close

pytestmark = pytest.mark.gpu


def _cudart():
    import ctypes
    import glob
    import os
    import torch
    cands = glob.glob(os.path.join(os.path.dirname(torch.__file__), "..", "nvidia", "cuda_runtime", "lib",
                                   "libcudart.so*")) + ["/usr/local/cuda/lib64/libcudart.so"]
    for c in cands:
        try:
            lib = ctypes.CDLL(c)
            lib.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
            return lib
        except OSError:
            continue
    raise RuntimeError("no CUDA runtime to read device buffers")


def device_array(ptr, shape, dtype):
    """Copies `shape` elements at device address `ptr` to a numpy array."""
    import torch
    torch.cuda.synchronize()
    out = np.empty(shape, dtype=dtype)
    assert _cudart().cudaMemcpy(out.ctypes.data, ptr, out.nbytes, 2) == 0
    return out


@pytest.mark.parametrize("pipeline", [B.PIPELINE_STAGED, B.PIPELINE_FUSED])
# 128x96 over 17 frames: every entry of the device's BLOCK_OFFSETS table
# (frame % 16, opencl/bmfr.cl:267-285) and the wrap back to entry 0.
# 1280x720: 984 blocks, more than the persistent fitter's CTAs, so each CTA
# fits several blocks through both tile buffers and both barrier phases.
# 1920x1080 and 3840x2160: the precision and many-stream workloads' sizes.
# 32x32 and 47x63: the smallest accepted images, whose mirrored margin
# reaches the last index mirror() serves (bmfr.cl:209-216), over all 16
# block offsets.
@pytest.mark.parametrize("W,H,frames", [(128, 96, 17), (256, 256, 8), (197, 131, 5), (1280, 720, 3),
                                        (1920, 1080, 2), (3840, 2160, 1), (32, 32, 17), (47, 63, 17)])
def test_pipeline_matches_oracle(cuda, pipeline, W, H, frames):
    _pipeline_parity(pipeline, W, H, frames, use_half=1)


# float32 tmp_data (USE_HALF_PRECISION_IN_TMP_DATA=0, opencl/bmfr.cpp:88):
# the fitter's one-dimensional bulk copy and float tile, over all 16 block
# offsets.
@pytest.mark.parametrize("pipeline", [B.PIPELINE_STAGED, B.PIPELINE_FUSED])
def test_pipeline_with_float_tmp_data_matches_oracle(cuda, pipeline):
    _pipeline_parity(pipeline, 64, 48, 17, use_half=0)


# Edge values (NaN, +-inf, beyond binary16; NaN and out-of-range positions)
# written into every fourth frame, carried by the histories in between: the
# case the oracle is pinned on against the compiled reference
# (tests/test_reference_pin.py, the same scene and draws).
@pytest.mark.parametrize("pipeline", [B.PIPELINE_STAGED, B.PIPELINE_FUSED])
def test_pipeline_with_edge_frames_matches_oracle(cuda, pipeline):
    _pipeline_parity(pipeline, 64, 48, 17, use_half=1, scene_seed=41, edge_seed=41)


def _pipeline_parity(pipeline, W, H, frames, use_half, scene_seed=21, edge_seed=None):
    import torch
    sc = B.Scene(scene_seed, W, H, 12)
    if edge_seed is not None:
        import sys
        golden = str(Path(__file__).resolve().parent / "golden")
        if golden not in sys.path:
            sys.path.insert(0, golden)
        import cases
        rng = np.random.default_rng(edge_seed)
    plan = B.Plan(W, H, pipeline=pipeline, position_limit_squared=sc.position_limit_squared,
                  normal_limit_squared=sc.normal_limit_squared, use_half_precision_in_tmp_data=use_half)
    plan.keep_intermediates(True)   # the tone-mapped frame is checked below
    ref = OraclePipeline(Oracle(W, H, sc.position_limit_squared, sc.normal_limit_squared, use_half=bool(use_half)))
    for f in range(frames):
        d = sc.render(f)
        if edge_seed is not None and f % 4 == 1:
            d = cases.edge_frame(d, rng, W, H)
        plan.upload_frame(d["albedo"], d["normals"], d["positions"], d["noisy"])
        plan.denoise_frame(sc.prev_camera(f), sc.pixel_offset(f))
        got = plan.download_result()
        want = ref.step(d["albedo"], d["normals"], d["positions"], d["noisy"], sc.prev_camera(f),
                        sc.pixel_offset(f))
        assert_close(got, want, f"result frame {f}", rtol=1e-4)
        # Intermediates of the frame: integer outputs and the fit bit-exact.
        bufs = plan.buffers()
        c = f & 1
        np.testing.assert_array_equal(device_array(bufs.accept, (H, W), np.uint8), ref.accept)
        np.testing.assert_array_equal(device_array(bufs.spp, (H, W), np.uint8), ref.spp[c])
        np.testing.assert_array_equal(device_array(bufs.prev_frame_pixel, (H, W, 2), np.float32), ref.prev_pix)
        np.testing.assert_array_equal(device_array(bufs.mins_maxs, ref.mins_maxs.shape, np.float32),
                                      ref.mins_maxs)
        gw = device_array(bufs.weights, ref.weights.shape, np.float32)
        np.testing.assert_array_equal(gw, ref.weights, err_msg=f"weights frame {f}")
        np.testing.assert_array_equal(device_array(bufs.accumulated_noisy, (H, W, 3), np.float32), ref.noisy[c])
        assert_close(device_array(bufs.tone_mapped, (H, W, 3), np.float32), ref.tone_mapped, "tone mapped",
                     rtol=1e-5)
    torch.cuda.synchronize()
    assert plan.frame_number == frames
    plan.close()


@pytest.mark.parametrize("half_history", [0, 1])
def test_kept_intermediates_change_no_output(cuda, half_history):
    """The plan runs weighted sum and filtered accumulation as one kernel;
    writing its filtered frame out for inspection must not change any output
    bit, and that frame must equal the drop-in weighted_sum's."""
    import torch
    W, H = 200, 120
    sc = B.Scene(24, W, H, 12)
    kw = dict(half_history=half_history, fp32_qr=1 if half_history else 0,
              position_limit_squared=sc.position_limit_squared, normal_limit_squared=sc.normal_limit_squared)
    plain, kept = B.Plan(W, H, **kw), B.Plan(W, H, **kw)
    kept.keep_intermediates(True)
    assert plain.buffers().filtered is None and kept.buffers().filtered is not None
    for f in range(4):
        d = sc.render(f)
        for pl in (plain, kept):
            pl.upload_frame(d["albedo"], d["normals"], d["positions"], d["noisy"])
            pl.denoise_frame(sc.prev_camera(f), sc.pixel_offset(f))
        np.testing.assert_array_equal(plain.download_result(), kept.download_result(), err_msg=f"frame {f}")
        hist = np.float16 if half_history else np.float32
        a, b = plain.buffers(), kept.buffers()
        np.testing.assert_array_equal(device_array(a.accumulated_filtered, (H, W, 3), hist),
                                      device_array(b.accumulated_filtered, (H, W, 3), hist))
        # The kept frame is the drop-in weighted_sum's output (float
        # histories only: the drop-in entry points take float buffers).
        if not half_history and f > 0:
            n = W * H * 3
            t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).reshape(-1).to(cuda)
            ptr = lambda p, shape, dt: torch.from_numpy(device_array(p, shape, dt)).reshape(-1).to(cuda)
            filt = torch.empty(n, dtype=torch.float32, device=cuda)
            B.weighted_sum(kept, ptr(b.weights, (kept.sizes.blocks * 30,), np.float32),
                           ptr(b.mins_maxs, (kept.sizes.blocks * 12,), np.float32), filt, t(d["normals"]),
                           t(d["positions"]), None, f)
            np.testing.assert_array_equal(filt.cpu().numpy().reshape(H, W, 3),
                                          device_array(b.filtered, (H, W, 3), np.float32))
    plain.close()
    kept.close()


def test_pipeline_rejects_bad_arguments(cuda):
    with pytest.raises(B.BmfrError):
        B.Plan(16, 16)
    # Widths 33..46 leave the mirrored margin beyond one image size; 32 and
    # 47 are the limits on either side (the same rule for heights).
    for w, h in ((33, 64), (46, 64), (64, 46)):
        with pytest.raises(B.BmfrError):
            B.Plan(w, h)
    for w, h in ((32, 64), (47, 64), (64, 47)):
        B.Plan(w, h).close()
    plan = B.Plan(64, 64)
    with pytest.raises(ValueError):
        plan.denoise_frame(np.zeros(15), np.zeros(2))
    plan.close()


@pytest.mark.parametrize("half_history", [0, 1])
def test_three_stream_frame_loop(cuda, half_history):
    """Uploads, frames and downloads issued on three streams, each frame's
    upload and the previous frame's download overlapping the denoising: the
    plan's own ordering must give every frame exactly the output of the
    one-stream loop."""
    import torch
    W, H, frames = 160, 96, 7
    sc = B.Scene(23, W, H, 10)
    data = [sc.render(f) for f in range(frames)]
    pin = lambda a: torch.from_numpy(a).pin_memory()
    host = [{k: pin(d[k]) for k in ("albedo", "normals", "positions", "noisy")} for d in data]
    kw = dict(half_history=half_history, fp32_qr=1 if half_history else 0,
              position_limit_squared=sc.position_limit_squared, normal_limit_squared=sc.normal_limit_squared)
    one = B.Plan(W, H, **kw)
    want = []
    for f in range(frames):
        h = host[f]
        one.upload_frame(h["albedo"], h["normals"], h["positions"], h["noisy"])
        one.denoise_frame(sc.prev_camera(f), sc.pixel_offset(f))
        want.append(one.download_result())
    three = B.Plan(W, H, **kw)
    up, comp, down = (torch.cuda.Stream(device=cuda) for _ in range(3))
    outs = [torch.empty((H, W, 3), dtype=torch.float32).pin_memory() for _ in range(frames)]
    for f in range(frames):
        h = host[f]
        three.upload_frame(h["albedo"], h["normals"], h["positions"], h["noisy"], stream=up)
        three.denoise_frame(sc.prev_camera(f), sc.pixel_offset(f), stream=comp)
        three.download_result(outs[f], stream=down)
    torch.cuda.synchronize()
    for f in range(frames):
        np.testing.assert_array_equal(outs[f].numpy(), want[f], err_msg=f"frame {f}")
    one.close()
    three.close()
