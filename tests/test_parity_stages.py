"""Parity of the five CUDA stages with the CPU oracle on identical inputs.

Each stage is fed the SAME inputs on both sides (the oracle's own outputs of
the previous stage), frame after frame with real history, so a mismatch is
attributed to exactly one stage.  Integer outputs (reprojected pixel
positions, accept masks, spp, the block-major tmp_data layout) must be
bit-exact; float outputs must match within the relative tolerance below.
"""
import numpy as np
import pytest

import bmfr_b200 as B
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

# Float tolerance: |cuda - oracle| <= RTOL * max(|oracle|, FLOOR).  The CUDA
# kernels keep the reference's operation order, so the fit and the
# accumulations are bit-identical; pow() in the tone map (and so TAA) may
# differ in the last bits.
RTOL = 1e-3
FLOOR = 1e-2


def _t(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _np(t):
    return t.detach().cpu().numpy()


def assert_close(got, want, what, rtol=RTOL, floor=FLOOR):
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    assert got.shape == want.shape, what
    both_nan = np.isnan(got) & np.isnan(want)
    err = np.abs(got - want)
    lim = rtol * np.maximum(np.abs(want), floor)
    bad = ~both_nan & ~(err <= lim)
    assert not bad.any(), (f"{what}: {bad.sum()} of {bad.size} values off, worst "
                           f"{np.nanmax(np.where(bad, err / np.maximum(np.abs(want), floor), 0)):.3e}")


# 1280x720: 984 blocks, more than the persistent fitter's CTAs.
SIZES = [(64, 64), (100, 70), (256, 256), (1280, 720), (32, 32), (47, 63)]   # the last two: smallest accepted


@pytest.mark.parametrize("W,H", SIZES)
def test_stage_parity_over_frames(cuda, W, H):
    import torch
    sc = B.Scene(11, W, H, 12)
    plan = B.Plan(W, H, position_limit_squared=sc.position_limit_squared,
                  normal_limit_squared=sc.normal_limit_squared)
    o = Oracle(W, H, sc.position_limit_squared, sc.normal_limit_squared)
    px = W * H
    z3 = lambda: np.zeros((H, W, 3), np.float32)
    # Oracle-side histories.
    o_n, o_p, o_noisy, o_acc, o_res = [z3(), z3()], [z3(), z3()], [z3(), z3()], [z3(), z3()], [z3(), z3()]
    o_spp = [np.zeros((H, W), np.uint8), np.zeros((H, W), np.uint8)]
    pp, acc = np.zeros((H, W, 2), np.float32), np.zeros((H, W), np.uint8)
    tmp = o.new_tmp()
    weights = np.zeros(o.blocks * 30, np.float32)
    mm = np.zeros(o.blocks * 12, np.float32)
    filt, tm = z3(), z3()
    for f in list(range(4)) + [17]:
        d = sc.render(f)
        c, p = f & 1, (f & 1) ^ 1
        o_n[c][...], o_p[c][...], o_noisy[c][...] = d["normals"], d["positions"], d["noisy"]
        mat, off = sc.prev_camera(f), sc.pixel_offset(f)

        # --- accumulate_noisy_data: identical history on both sides
        g_pp = torch.zeros(px * 2, dtype=torch.float32, device=cuda)
        g_acc = torch.zeros(px, dtype=torch.uint8, device=cuda)
        g_spp = torch.zeros(px, dtype=torch.uint8, device=cuda)
        g_tmp = torch.zeros(o.blocks * 13 * 1024, dtype=torch.float16, device=cuda)
        g_noisy = _t(o_noisy[c], cuda)
        B.accumulate_noisy_data(plan, g_pp, g_acc, _t(o_n[c], cuda), _t(o_n[p], cuda), _t(o_p[c], cuda),
                                _t(o_p[p], cuda), g_noisy, _t(o_noisy[p], cuda), _t(o_spp[p], cuda), g_spp,
                                g_tmp, mat, off, f)
        o.accumulate_noisy_data(pp, acc, o_n[c], o_n[p], o_p[c], o_p[p], o_noisy[c], o_noisy[p], o_spp[p],
                                o_spp[c], tmp, mat, off, f)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(_np(g_pp).reshape(H, W, 2), pp, err_msg=f"prev_frame_pixel f={f}")
        np.testing.assert_array_equal(_np(g_acc).reshape(H, W), acc, err_msg=f"accept f={f}")
        np.testing.assert_array_equal(_np(g_spp).reshape(H, W), o_spp[c], err_msg=f"spp f={f}")
        np.testing.assert_array_equal(_np(g_tmp).view(np.uint16), tmp.view(np.uint16), err_msg=f"tmp f={f}")
        assert_close(_np(g_noisy).reshape(H, W, 3), o_noisy[c], f"accumulated noisy f={f}", rtol=1e-6)

        # --- fitter on the oracle's tmp
        g_w = torch.zeros(o.blocks * 30, dtype=torch.float32, device=cuda)
        g_mm = torch.zeros(o.blocks * 12, dtype=torch.float32, device=cuda)
        B.fitter(plan, g_w, g_mm, _t(tmp, cuda), f)
        o.fitter(weights, mm, tmp, f)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(_np(g_mm), mm, err_msg=f"mins_maxs f={f}")
        np.testing.assert_array_equal(_np(g_w), weights, err_msg=f"weights f={f}")

        # --- weighted_sum with the oracle's weights
        g_out = torch.zeros(px * 3, dtype=torch.float32, device=cuda)
        B.weighted_sum(plan, _t(weights, cuda), _t(mm, cuda), g_out, _t(o_n[c], cuda), _t(o_p[c], cuda), None, f)
        o.weighted_sum(weights, mm, filt, o_n[c], o_p[c], f)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(_np(g_out).reshape(H, W, 3), filt, err_msg=f"weighted_sum f={f}")

        # --- accumulate_filtered_data
        g_tm = torch.zeros(px * 3, dtype=torch.float32, device=cuda)
        g_acc_cur = torch.zeros(px * 3, dtype=torch.float32, device=cuda)
        B.accumulate_filtered_data(plan, _t(filt, cuda), _t(pp, cuda), _t(acc, cuda), _t(d["albedo"], cuda), g_tm,
                                   _t(o_spp[c], cuda), _t(o_acc[p], cuda), g_acc_cur, f)
        o.accumulate_filtered_data(filt, pp, acc, d["albedo"], tm, o_spp[c], o_acc[p], o_acc[c], f)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(_np(g_acc_cur).reshape(H, W, 3), o_acc[c], err_msg=f"acc filtered f={f}")
        assert_close(_np(g_tm).reshape(H, W, 3), tm, f"tone mapped f={f}", rtol=1e-5)

        # --- taa
        g_res = torch.zeros(px * 3, dtype=torch.float32, device=cuda)
        B.taa(plan, _t(pp, cuda), _t(tm, cuda), g_res, _t(o_res[p], cuda), f)
        o.taa(pp, tm, o_res[c], o_res[p], f)
        torch.cuda.synchronize()
        assert_close(_np(g_res).reshape(H, W, 3), o_res[c], f"taa f={f}", rtol=1e-5)
    plan.close()


def test_in_place_accumulation_matches_out_of_place(cuda):
    """The drop-in entry updates current_noisy in place like the reference;
    mirrored margin rows must equal their in-image pixel's row."""
    import torch
    W, H = 96, 64
    sc = B.Scene(2, W, H, 8)
    plan = B.Plan(W, H)
    px = W * H
    d0, d1 = sc.render(0), sc.render(1)
    args = []
    outs = []
    for _ in range(2):
        g_pp = torch.zeros(px * 2, dtype=torch.float32, device=cuda)
        g_acc = torch.zeros(px, dtype=torch.uint8, device=cuda)
        g_spp = torch.zeros(px, dtype=torch.uint8, device=cuda)
        g_tmp = torch.zeros(plan.sizes.blocks * 13 * 1024, dtype=torch.float16, device=cuda)
        g_noisy = _t(d1["noisy"], cuda)
        B.accumulate_noisy_data(plan, g_pp, g_acc, _t(d1["normals"], cuda), _t(d0["normals"], cuda),
                                _t(d1["positions"], cuda), _t(d0["positions"], cuda), g_noisy,
                                _t(d0["noisy"], cuda), torch.ones(px, dtype=torch.uint8, device=cuda), g_spp, g_tmp,
                                sc.camera(0), sc.pixel_offset(1), 1)
        outs.append((g_tmp.clone(), g_noisy.clone()))
    torch.cuda.synchronize()
    assert torch.equal(outs[0][0], outs[1][0])
    assert torch.equal(outs[0][1], outs[1][1])
    plan.close()
