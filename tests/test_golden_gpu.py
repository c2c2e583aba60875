"""The CUDA path against the reference's own outputs.

tests/golden/ref_*.npz hold outputs of the reference's OpenCL kernels
(opencl/bmfr.cl compiled for the CPU, tests/golden/make_golden.py) with the
inputs that produced them: a three-frame run of the procedural scene (with
binary16 and with float32 tmp_data), and one frame of edge inputs for every
stage (NaN, infinities, values beyond
binary16, spp 0 and 255, degenerate blocks, reprojections on and beyond the
image edges).  The plan pipeline (staged and fused) and the five drop-in
entry points are run on the stored inputs.  Integer outputs, tmp_data, the
fitted weights and the accumulations must be bit-identical (NaN equal to
NaN); tone mapping (powr on the special function unit) and TAA within 1e-5.
"""
from pathlib import Path

import numpy as np
import pytest

import bmfr_b200 as B

from test_parity_pipeline import device_array
from test_parity_stages import assert_close

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


def same(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, what
    eq = (a == b) | (np.isnan(a) & np.isnan(b)) if a.dtype.kind == "f" else a == b
    assert eq.all(), f"{what}: {int((~eq).sum())} of {eq.size} values differ"


def weights_match(got, want, what):
    same(got, want, what)


@pytest.mark.parametrize("fixture,use_half", [("ref_pipeline.npz", 1), ("ref_pipeline_f32.npz", 0)])
@pytest.mark.parametrize("pipeline", [B.PIPELINE_STAGED, B.PIPELINE_FUSED])
def test_plan_pipeline_matches_reference_fixture(cuda, pipeline, fixture, use_half):
    """tmp_data in binary16 (the reference's default) and in float32 (its
    USE_HALF_PRECISION_IN_TMP_DATA=0), on the same scene frames."""
    inp = np.load(GOLDEN / "ref_pipeline.npz")
    g = np.load(GOLDEN / fixture)
    frames = sum(1 for k in g.files if k.endswith("_result"))
    H, W = inp["in0_albedo"].shape[:2]
    lim = g["limits"]
    plan = B.Plan(W, H, pipeline=pipeline, position_limit_squared=float(lim[0]),
                  normal_limit_squared=float(lim[1]), use_half_precision_in_tmp_data=use_half)
    plan.keep_intermediates(True)   # the tone-mapped frame is checked below
    for f in range(frames):
        plan.upload_frame(inp[f"in{f}_albedo"], inp[f"in{f}_normals"], inp[f"in{f}_positions"], inp[f"in{f}_noisy"])
        plan.denoise_frame(inp[f"in{f}_matrix"], inp[f"in{f}_offset"])
        got = plan.download_result()
        bufs = plan.buffers()
        same(device_array(bufs.accept, (H, W), np.uint8), g[f"out{f}_accept"], f"accept {f}")
        same(device_array(bufs.spp, (H, W), np.uint8), g[f"out{f}_spp"], f"spp {f}")
        same(device_array(bufs.prev_frame_pixel, (H, W, 2), np.float32), g[f"out{f}_prev_pix"], f"prev pix {f}")
        same(device_array(bufs.mins_maxs, g[f"out{f}_mins_maxs"].shape, np.float32), g[f"out{f}_mins_maxs"],
             f"mins_maxs {f}")
        weights_match(device_array(bufs.weights, g[f"out{f}_weights"].shape, np.float32), g[f"out{f}_weights"],
                      f"weights {f}")
        same(device_array(bufs.accumulated_noisy, (H, W, 3), np.float32), g[f"out{f}_noisy_acc"],
             f"accumulated noisy {f}")
        assert_close(device_array(bufs.tone_mapped, (H, W, 3), np.float32), g[f"out{f}_tone_mapped"],
                     f"tone mapped {f}", rtol=1e-5)
        assert_close(got, g[f"out{f}_result"], f"result {f}", rtol=1e-4)
    plan.close()


def test_dropin_stages_match_reference_edge_fixture(cuda):
    _check_dropin_stages(cuda, np.load(GOLDEN / "ref_stages.npz"))


def _oracle_stage_case(seed, frame):
    """The stage fixture's kinds of edge inputs drawn for (seed, frame)
    (tests/golden/cases.py) with the oracle's output of every stage, under
    the fixture's names.  The oracle equals the compiled reference bit for
    bit on these same cases (tests/test_reference_pin.py)."""
    import sys
    if str(GOLDEN) not in sys.path:
        sys.path.insert(0, str(GOLDEN))
    import cases
    from oracle.oracle import Oracle
    d = cases.stage_inputs(seed=seed, frame=frame)
    w, h = cases.STAGE_SIZE
    o = Oracle(w, h, float(d["limits"][0]), float(d["limits"][1]))
    g = {f"in_{k}": v for k, v in d.items()}
    pp = np.zeros((h, w, 2), np.float32)
    acc = np.zeros((h, w), np.uint8)
    spp = np.zeros((h, w), np.uint8)
    noisy = d["cur_noisy"].copy()
    tmp = o.new_tmp()
    o.accumulate_noisy_data(pp, acc, d["cur_normals"], d["prev_normals"], d["cur_positions"], d["prev_positions"],
                            noisy, d["prev_noisy"], d["prev_spp"], spp, tmp, d["matrix"], d["offset"], frame)
    g.update(out_acc_prev_pix=pp, out_acc_accept=acc, out_acc_spp=spp, out_acc_noisy=noisy, out_acc_tmp=tmp.copy())
    fit_in = cases.patch_fit_blocks(tmp.copy(), d["fit_blocks"], rng_seed=seed)
    weights = np.zeros(o.blocks * 30, np.float32)
    mm = np.zeros(o.blocks * 12, np.float32)
    o.fitter(weights, mm, fit_in.copy(), frame)
    g.update(in_fit_tmp=fit_in, out_fit_weights=weights, out_fit_mins_maxs=mm)
    filt = np.zeros((h, w, 3), np.float32)
    o.weighted_sum(weights, mm, filt, d["cur_normals"], d["cur_positions"], frame)
    tone = np.zeros((h, w, 3), np.float32)
    acc_cur = np.zeros((h, w, 3), np.float32)
    o.accumulate_filtered_data(filt, d["prev_pix"], d["accept"], d["albedo"], tone, d["cur_spp"], d["acc_prev"],
                               acc_cur, frame)
    res = np.zeros((h, w, 3), np.float32)
    o.taa(d["taa_prev_pix"], tone, res, d["taa_prev"], frame)
    g.update(out_ws_filtered=filt, out_af_tone_mapped=tone, out_af_accumulated=acc_cur, out_taa_result=res)
    return g


@pytest.mark.parametrize("offset", range(16))
def test_dropin_stages_match_oracle_on_edge_inputs(cuda, offset):
    """Edge inputs drawn anew for each of the 16 block offsets (frame
    16 + offset) through the five drop-in entry points."""
    _check_dropin_stages(cuda, _oracle_stage_case(1000 + offset, 16 + offset))


def _check_dropin_stages(cuda, g):
    """The five drop-in entry points on stage inputs `g`, each against the
    expected output of its stage under the stage fixture's names."""
    import torch
    H, W = g["in_albedo"].shape[:2]
    px = W * H
    f = int(g["in_frame"][0])
    plan = B.Plan(W, H, position_limit_squared=float(g["in_limits"][0]),
                  normal_limit_squared=float(g["in_limits"][1]))
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda)
    n = lambda x: x.detach().cpu().numpy()
    blocks = g["out_fit_weights"].size // 30

    # accumulate_noisy_data
    g_pp = torch.zeros(px * 2, dtype=torch.float32, device=cuda)
    g_acc = torch.zeros(px, dtype=torch.uint8, device=cuda)
    g_spp = torch.zeros(px, dtype=torch.uint8, device=cuda)
    g_tmp = torch.zeros(blocks * 13 * 1024, dtype=torch.float16, device=cuda)
    g_noisy = t(g["in_cur_noisy"])
    B.accumulate_noisy_data(plan, g_pp, g_acc, t(g["in_cur_normals"]), t(g["in_prev_normals"]),
                            t(g["in_cur_positions"]), t(g["in_prev_positions"]), g_noisy, t(g["in_prev_noisy"]),
                            t(g["in_prev_spp"]), g_spp, g_tmp, g["in_matrix"], g["in_offset"], f)
    torch.cuda.synchronize()
    same(n(g_pp).reshape(H, W, 2), g["out_acc_prev_pix"], "prev_frame_pixel")
    same(n(g_acc).reshape(H, W), g["out_acc_accept"], "accept")
    same(n(g_spp).reshape(H, W), g["out_acc_spp"], "spp")
    same(n(g_tmp).view(np.uint16), g["out_acc_tmp"].view(np.uint16), "tmp_data")
    same(n(g_noisy).reshape(H, W, 3), g["out_acc_noisy"], "accumulated noisy")

    # fitter (constant, all-zero and +-65504 blocks among the scene's)
    g_w = torch.zeros(blocks * 30, dtype=torch.float32, device=cuda)
    g_mm = torch.zeros(blocks * 12, dtype=torch.float32, device=cuda)
    B.fitter(plan, g_w, g_mm, t(g["in_fit_tmp"]), f)
    torch.cuda.synchronize()
    same(n(g_mm), g["out_fit_mins_maxs"], "mins_maxs")
    weights_match(n(g_w), g["out_fit_weights"], "weights")

    # weighted_sum on the reference's weights (NaN blocks included)
    g_out = torch.zeros(px * 3, dtype=torch.float32, device=cuda)
    B.weighted_sum(plan, t(g["out_fit_weights"]), t(g["out_fit_mins_maxs"]), g_out, t(g["in_cur_normals"]),
                   t(g["in_cur_positions"]), None, f)
    torch.cuda.synchronize()
    same(n(g_out).reshape(H, W, 3), g["out_ws_filtered"], "weighted sum")

    # accumulate_filtered_data (spp 0, taps on every edge)
    g_tm = torch.zeros(px * 3, dtype=torch.float32, device=cuda)
    g_acc_cur = torch.zeros(px * 3, dtype=torch.float32, device=cuda)
    B.accumulate_filtered_data(plan, t(g["out_ws_filtered"]), t(g["in_prev_pix"]), t(g["in_accept"]),
                               t(g["in_albedo"]), g_tm, t(g["in_cur_spp"]), t(g["in_acc_prev"]), g_acc_cur, f)
    torch.cuda.synchronize()
    same(n(g_acc_cur).reshape(H, W, 3), g["out_af_accumulated"], "accumulated filtered")
    assert_close(n(g_tm).reshape(H, W, 3), g["out_af_tone_mapped"], "tone mapped", rtol=1e-5)

    # taa (history positions NaN, infinite, at -1 and on the last row)
    g_res = torch.zeros(px * 3, dtype=torch.float32, device=cuda)
    B.taa(plan, t(g["in_taa_prev_pix"]), t(g["out_af_tone_mapped"]), g_res, t(g["in_taa_prev"]), f)
    torch.cuda.synchronize()
    assert_close(n(g_res).reshape(H, W, 3), g["out_taa_result"], "taa", rtol=1e-5)
    plan.close()

