"""End-to-end parity of the plan-managed frame pipeline (staged and fused
forms) with the oracle's frame loop, through host-buffer uploads."""
import numpy as np
import pytest

import bmfr_b200 as B
from oracle.oracle import Oracle, OraclePipeline

from test_parity_stages import assert_close

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("pipeline", [B.PIPELINE_STAGED, B.PIPELINE_FUSED])
@pytest.mark.parametrize("W,H,frames", [(128, 96, 6), (256, 256, 8)])
def test_pipeline_matches_oracle(cuda, pipeline, W, H, frames):
    import torch
    sc = B.Scene(21, W, H, 12)
    plan = B.Plan(W, H, pipeline=pipeline, position_limit_squared=sc.position_limit_squared,
                  normal_limit_squared=sc.normal_limit_squared)
    ref = OraclePipeline(Oracle(W, H, sc.position_limit_squared, sc.normal_limit_squared))
    for f in range(frames):
        d = sc.render(f)
        plan.upload_frame(d["albedo"], d["normals"], d["positions"], d["noisy"])
        plan.denoise_frame(sc.prev_camera(f), sc.pixel_offset(f))
        got = plan.download_result()
        want = ref.step(d["albedo"], d["normals"], d["positions"], d["noisy"], sc.prev_camera(f),
                        sc.pixel_offset(f))
        assert_close(got, want, f"result frame {f}", rtol=1e-4)
    torch.cuda.synchronize()
    assert plan.frame_number == frames
    plan.close()


def test_pipeline_rejects_bad_arguments(cuda):
    with pytest.raises(B.BmfrError):
        B.Plan(16, 16)
    with pytest.raises(B.BmfrError):
        B.Plan(33, 64)   # too small for the mirrored margin
    plan = B.Plan(64, 64)
    with pytest.raises(ValueError):
        plan.denoise_frame(np.zeros(15), np.zeros(2))
    plan.close()
