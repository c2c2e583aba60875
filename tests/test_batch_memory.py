"""Per-stream device memory of the many-stream engine, on the host.

bmfr_batch_stream_bytes is what admission against the memory budget charges
for a stream (the batch, the request server and the multi-GPU router all
use it).  It must equal the stream's buffers as the engine lays them out:
the six double-buffered histories of opencl/bmfr.cpp:316-347 (accumulated
noisy colour, accumulated filtered colour, TAA result, spp), the per-frame
buffers (reprojected positions, accept mask, tone-mapped frame, float32
result, weights, min/max, the fitter's noise table, tmp_data for the staged
pipeline) and, for streams that keep their own inputs, two G-buffers plus
albedo and noisy colour; each piece starts on a 256-byte boundary.  No GPU
is needed: the size is a host computation.
"""
import pytest

import bmfr_b200 as B

SIZES = [(640, 360), (1280, 720), (1920, 1080), (3840, 2160), (197, 131)]


def up256(n):
    return (n + 255) // 256 * 256


def expected_bytes(w, h, half_history, half_tmp, staged, own_inputs):
    """The engine's layout restated: what each piece holds, in order."""
    px = w * h
    ww, wh = 32 * -(-w // 32), 32 * -(-h // 32)
    mw, mh = ww + 32, wh + 32
    blocks = (mw // 32) * (mh // 32)
    hist = px * 3 * (2 if half_history else 4)
    pieces = [hist, hist, hist, px] * 2                 # noisy_acc, acc_filt, result, spp (x2)
    pieces += [px * 8, px, px * 12, px * 12]            # prev_pix, accept, tone_mapped, result_f32
    pieces += [blocks * 10 * 3 * 4, blocks * 6 * 2 * 4]  # weights, mins_maxs
    pieces += [9 * 4 * 256 * 4]                         # noise table: features 1..9 x 4 rows x 256 threads
    if staged:
        pieces += [mw * mh * 13 * (2 if half_tmp else 4)]
    if own_inputs:
        pieces += [px * 12] * 6                         # normals x2, positions x2, albedo, noisy
    return sum(up256(n) for n in pieces)


@pytest.mark.parametrize("w,h", SIZES)
@pytest.mark.parametrize("half_history", [0, 1])
@pytest.mark.parametrize("pipeline", [B.PIPELINE_STAGED, B.PIPELINE_FUSED])
@pytest.mark.parametrize("own_inputs", [False, True])
def test_stream_bytes_follow_the_layout(w, h, half_history, pipeline, own_inputs):
    p = B.default_params(half_history=half_history, pipeline=pipeline)
    got = B.Batch.stream_bytes(p, w, h, own_inputs)
    want = expected_bytes(w, h, half_history, p.use_half_precision_in_tmp_data, pipeline == B.PIPELINE_STAGED,
                          own_inputs)
    assert got == want


def test_stream_bytes_at_4k_with_binary16_histories():
    """71 bytes per pixel and 168 per block, plus the staged pipeline's
    binary16 tmp_data (26 bytes per margin pixel) and the 36 KB noise
    table: the figures the memory budget and the server's admission use."""
    w, h = 3840, 2160
    px, mpx, blocks = w * h, 3872 * 2208, 121 * 69
    fused = B.Batch.stream_bytes(B.default_params(half_history=1, pipeline=B.PIPELINE_FUSED), w, h)
    staged = B.Batch.stream_bytes(B.default_params(half_history=1, pipeline=B.PIPELINE_STAGED), w, h)
    assert abs(fused - (71 * px + 168 * blocks + 36864)) < 256 * 20
    assert staged - fused == up256(26 * mpx)
    assert round(fused / 2**20) == 563 and round(staged / 2**20) == 775
