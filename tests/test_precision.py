"""The precision form: binary16 histories and an FP32 QR, checked against the
fitter in double precision.

bmfr_fitter_fp64 (the only FP64 code on the device) must equal the oracle's
fp64 fitter bit for bit; the precision form's weights and output pixels are
then measured against that fp64 reference (the tolerances below are written
for the seeded scenes used here).
"""
import numpy as np
import pytest

import bmfr_b200 as B
from oracle.oracle import FITTER_FP64, Oracle, OraclePipeline

pytestmark = pytest.mark.gpu


def rel_err(got, want, floor=1e-2):
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    return np.abs(got - want) / np.maximum(np.abs(want), floor)


def test_fp64_fitter_matches_oracle(cuda):
    import torch
    W, H = 192, 128
    sc = B.Scene(13, W, H, 16)
    o = Oracle(W, H, sc.position_limit_squared, sc.normal_limit_squared)
    pipe = OraclePipeline(o)
    plan = B.Plan(W, H)
    nb = plan.sizes.blocks
    for f in range(3):
        d = sc.render(f)
        pipe.step(d["albedo"], d["normals"], d["positions"], d["noisy"], sc.prev_camera(f), sc.pixel_offset(f))
        tmp = pipe.tmp_after_accumulate
        want_w = np.zeros(nb * 30)
        want_mm = np.zeros(nb * 12, np.float32)
        o.fitter_fp64(want_w, want_mm, tmp, f)
        w = torch.zeros(nb * 30, dtype=torch.float64, device=cuda)
        mm = torch.zeros(nb * 12, dtype=torch.float32, device=cuda)
        B.fitter_fp64(plan, w, mm, torch.from_numpy(tmp).to(cuda), f)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(w.cpu().numpy(), want_w)
        np.testing.assert_array_equal(mm.cpu().numpy(), want_mm)
    plan.close()


# 1280x720: more blocks than the persistent fitter's CTAs (each CTA fits
# several blocks through both tile buffers); 1920x1080: the precision
# workload's size.
@pytest.mark.parametrize("W,H", [(256, 192), (1280, 720), (1920, 1080)])
@pytest.mark.parametrize("qr", [B.QR_CHOLESKY2, B.QR_HOUSEHOLDER])
def test_fp32_qr_weights_against_fp64(cuda, qr, W, H):
    import torch
    sc = B.Scene(17, W, H, 24)
    o = Oracle(W, H, sc.position_limit_squared, sc.normal_limit_squared)
    pipe = OraclePipeline(o)
    plan = B.Plan(W, H, fp32_qr=qr)
    nb = plan.sizes.blocks
    for f in range(3):
        d = sc.render(f)
        pipe.step(d["albedo"], d["normals"], d["positions"], d["noisy"], sc.prev_camera(f), sc.pixel_offset(f))
        tmp = torch.from_numpy(pipe.tmp_after_accumulate).to(cuda)
        w64 = torch.zeros(nb * 30, dtype=torch.float64, device=cuda)
        w32 = torch.zeros(nb * 30, dtype=torch.float32, device=cuda)
        mm = torch.zeros(nb * 12, dtype=torch.float32, device=cuda)
        B.fitter_fp64(plan, w64, mm, tmp, f)
        B.fitter(plan, w32, mm, tmp, f)
        torch.cuda.synchronize()
        e = rel_err(w32.cpu().numpy(), w64.cpu().numpy(), floor=1e-3)
        assert e.mean() < 1e-4, e.mean()
        assert np.quantile(e, 0.999) < 1e-2
    plan.close()


@pytest.mark.parametrize("qr", [B.QR_CHOLESKY2, B.QR_HOUSEHOLDER])
@pytest.mark.parametrize("pipeline", [B.PIPELINE_STAGED, B.PIPELINE_FUSED])
def test_precision_form_output_against_fp64(cuda, pipeline, qr):
    """Binary16 histories + FP32 QR vs the pipeline with the fp64 fitter and
    float histories: mean relative error per frame below 2e-4, at most 0.1 %
    of pixels above 1e-3, no pixel above 2e-2."""
    W, H = 320, 180
    sc = B.Scene(19, W, H, 24)
    ref = OraclePipeline(Oracle(W, H, sc.position_limit_squared, sc.normal_limit_squared), fitter_mode=FITTER_FP64)
    plan = B.Plan(W, H, fp32_qr=qr, half_history=1, pipeline=pipeline,
                  position_limit_squared=sc.position_limit_squared, normal_limit_squared=sc.normal_limit_squared)
    for f in range(6):
        d = sc.render(f)
        want = ref.step(d["albedo"], d["normals"], d["positions"], d["noisy"], sc.prev_camera(f),
                        sc.pixel_offset(f))
        plan.upload_frame(d["albedo"], d["normals"], d["positions"], d["noisy"])
        plan.denoise_frame(sc.prev_camera(f), sc.pixel_offset(f))
        e = rel_err(plan.download_result(), want)
        assert e.mean() < 2e-4, (f, e.mean())
        assert (e > 1e-3).mean() <= 1e-3, (f, (e > 1e-3).mean())
        assert e.max() < 2e-2, (f, e.max())
    plan.close()


@pytest.mark.parametrize("pipeline", [B.PIPELINE_STAGED, B.PIPELINE_FUSED])
def test_precision_form_at_1080p_against_fp64(cuda, pipeline):
    """The precision workload (1920x1080, 24 spheres, its own seed): binary16
    histories and CholeskyQR2 against the pipeline with the fp64 fitter and
    float histories, with the bounds above."""
    W, H = 1920, 1080
    sc = B.Scene(20240603, W, H, 24)
    ref = OraclePipeline(Oracle(W, H, sc.position_limit_squared, sc.normal_limit_squared), fitter_mode=FITTER_FP64)
    plan = B.Plan(W, H, fp32_qr=B.QR_CHOLESKY2, half_history=1, pipeline=pipeline,
                  position_limit_squared=sc.position_limit_squared, normal_limit_squared=sc.normal_limit_squared)
    for f in range(3):
        d = sc.render(f)
        want = ref.step(d["albedo"], d["normals"], d["positions"], d["noisy"], sc.prev_camera(f),
                        sc.pixel_offset(f))
        plan.upload_frame(d["albedo"], d["normals"], d["positions"], d["noisy"])
        plan.denoise_frame(sc.prev_camera(f), sc.pixel_offset(f))
        e = rel_err(plan.download_result(), want)
        assert e.mean() < 2e-4, (f, e.mean())
        assert (e > 1e-3).mean() <= 1e-3, (f, (e > 1e-3).mean())
        assert e.max() < 2e-2, (f, e.max())
    plan.close()
