"""Known-answer tests of the CPU oracle (no GPU).

The reference ships no golden vectors, so these pin the oracle against
independent restatements written here in Python and against hand-derived
properties of opencl/bmfr.cl.
"""
import numpy as np
import pytest

from oracle.oracle import FITTER_FP32, FITTER_FP64, FITTER_REFERENCE, Oracle, OraclePipeline, lib

BLOCK_OFFSETS = [(-14, -14), (4, -6), (-8, 14), (8, 0), (-10, -8), (2, 12), (12, -12), (-10, 0),
                 (12, 14), (-8, -16), (6, 6), (-2, -2), (6, -14), (-16, 12), (14, -4), (-6, 4)]


def py_hash(a: int) -> float:
    """random() of opencl/bmfr.cl:162-171 in Python integers."""
    m = 0xFFFFFFFF
    a &= m
    a = ((a + 0x7ed55d16) + (a << 12)) & m
    a = ((a ^ 0xc761c23c) ^ (a >> 19)) & m
    a = ((a + 0x165667b1) + (a << 5)) & m
    a = ((a + 0xd3a2646c) ^ (a << 9)) & m
    a = ((a + 0xfd7046c5) + (a << 3)) & m
    a = ((a ^ 0xb55a4f09) ^ (a >> 16)) & m
    return float(np.float32(np.float32(a) / np.float32(4294967296.0)))


@pytest.mark.parametrize("a", [0, 1, 2, 255, 256, 1023, 13 * 1024, 13 * 1024 * 59 + 777, 2**31 - 1, 2**32 - 1])
def test_hash_known_answers(a):
    assert lib.orc_random(a) == py_hash(a)


def test_hash_range_and_spread():
    vals = np.array([lib.orc_random(i) for i in range(4096)])
    assert vals.min() >= 0.0 and vals.max() <= 1.0
    assert abs(vals.mean() - 0.5) < 0.02


def test_add_random_is_double_rounded_once():
    # value + NOISE_AMOUNT * 2.f * (random(i) - 0.5f) with NOISE_AMOUNT a double
    # literal (opencl/bmfr.cpp:58, bmfr.cl:179-181).
    rng = np.random.default_rng(0)
    for _ in range(200):
        v = float(np.float32(rng.normal()))
        idv, sv, fb, fr = (int(x) for x in rng.integers(0, [256, 4, 10, 100]))
        idx = idv + sv * 256 + fb * 1024 + fr * 13 * 1024
        r = np.float32(np.float32(py_hash(idx)) - np.float32(0.5))
        expect = np.float32(np.float64(v) + (1e-2 * 2.0) * np.float64(r))
        assert lib.orc_add_random(v, idv, sv, fb, fr, 1e-2) == expect


@pytest.mark.parametrize("i,n,expect", [(-1, 64, 0), (-16, 64, 15), (-32, 64, 31), (0, 64, 0), (63, 64, 63),
                                        (64, 64, 63), (79, 64, 48), (95, 64, 32)])
def test_mirror(i, n, expect):
    assert lib.orc_mirror(i, n) == expect


@pytest.mark.parametrize("v", [0.0, 1.0, 1.0 + 2**-11, 1.0 + 3 * 2**-11, 65504.0, 65519.0, 65520.0, 5.96e-8,
                               2.98e-8, -2.5e-5, 3.14159])
def test_half_rounding_is_round_to_nearest_even(v):
    assert lib.orc_round_half(v) == float(np.float16(np.float32(v)))


def _scene_inputs(W, H, seed=3, frames=2):
    import bmfr_b200 as B
    sc = B.Scene(seed, W, H, 12)
    return sc, [sc.render(f) for f in range(frames)]


def test_tmp_layout_and_block_offsets():
    """tmp_data[((by*MWb + bx)*13 + k)*1024 + y*32 + x] holds feature k of pixel
    mirror(g - 16 + BLOCK_OFFSETS[f % 16]) (opencl/bmfr.cl:314-317, 455-476)."""
    W, H = 96, 64
    sc, fr = _scene_inputs(W, H, frames=1)
    o = Oracle(W, H, sc.position_limit_squared, sc.normal_limit_squared)
    for frame in (0, 5, 17):
        d = fr[0]
        tmp = o.new_tmp()
        pp = np.zeros((H, W, 2), np.float32)
        acc = np.zeros((H, W), np.uint8)
        spp = np.zeros((H, W), np.uint8)
        noisy = d["noisy"].copy()
        # frame > 0 needs history; reuse this frame's buffers as the previous ones.
        o.accumulate_noisy_data(pp, acc, d["normals"], d["normals"], d["positions"], d["positions"], noisy,
                                d["noisy"].copy(), np.ones((H, W), np.uint8), spp, tmp, sc.camera(0),
                                sc.pixel_offset(0), frame)
        t = tmp.reshape(o.margin_height // 32, o.margin_width // 32, 13, 32, 32)
        ox, oy = BLOCK_OFFSETS[frame % 16]
        rng = np.random.default_rng(frame)
        for gx, gy in rng.integers(0, [o.margin_width, o.margin_height], size=(64, 2)):
            px = lib.orc_mirror(int(gx) - 16 + ox, W)
            py = lib.orc_mirror(int(gy) - 16 + oy, H)
            blk = t[gy // 32, gx // 32, :, gy % 32, gx % 32]
            p = d["positions"][py, px]
            n = d["normals"][py, px]
            assert blk[0] == 1.0
            np.testing.assert_array_equal(blk[1:4], n.astype(np.float16))
            np.testing.assert_array_equal(blk[4:7], p.astype(np.float16))
            np.testing.assert_array_equal(blk[7:10], (p * p).astype(np.float16))


def test_frame0_accumulation_is_identity():
    """At frame 0 blend_alpha is 1: colour passes through, spp = 1, accept = 0,
    prev_frame_pixel = the pixel itself (opencl/bmfr.cl:324-336, 433-445)."""
    W, H = 64, 64
    sc, fr = _scene_inputs(W, H, frames=1)
    o = Oracle(W, H)
    d = fr[0]
    tmp, pp = o.new_tmp(), np.zeros((H, W, 2), np.float32)
    acc, spp = np.full((H, W), 9, np.uint8), np.zeros((H, W), np.uint8)
    noisy = d["noisy"].copy()
    o.accumulate_noisy_data(pp, acc, d["normals"], None, d["positions"], None, noisy, None, None, spp, tmp,
                            sc.camera(0), sc.pixel_offset(0), 0)
    np.testing.assert_array_equal(noisy, d["noisy"])
    assert (spp == 1).all() and (acc == 0).all()
    yy, xx = np.mgrid[0:H, 0:W]
    np.testing.assert_array_equal(pp[..., 0], xx)
    np.testing.assert_array_equal(pp[..., 1], yy)


def test_static_camera_reprojects_to_itself():
    """With a static camera and pixel offsets (0.5, 0.5) every visible pixel
    reprojects onto itself, accepts its own tap and doubles its spp."""
    W, H = 128, 96
    import bmfr_b200 as B
    sc = B.Scene(5, W, H, 12, orbit_degrees_per_frame=0.0)
    d = sc.render(0)
    o = Oracle(W, H, sc.position_limit_squared, sc.normal_limit_squared)
    tmp, pp = o.new_tmp(), np.zeros((H, W, 2), np.float32)
    acc, spp = np.zeros((H, W), np.uint8), np.zeros((H, W), np.uint8)
    noisy = d["noisy"].copy()
    o.accumulate_noisy_data(pp, acc, d["normals"], d["normals"], d["positions"], d["positions"], noisy,
                            d["noisy"].copy(), np.ones((H, W), np.uint8), spp, tmp, sc.camera(0),
                            sc.pixel_offset(1), 1)
    hit = np.linalg.norm(d["normals"], axis=-1) > 0.5
    yy, xx = np.mgrid[0:H, 0:W]
    err = np.maximum(np.abs(pp[..., 0] - xx), np.abs(pp[..., 1] - yy))
    assert err[hit].max() < 2e-3
    # The tap nearest to the pixel itself is always accepted.
    own_bit = np.where(pp[..., 0] - np.floor(pp[..., 0]) < 0.5, 1, 2) * np.where(
        pp[..., 1] - np.floor(pp[..., 1]) < 0.5, 1, 4)
    own_bit = np.where(own_bit == 8, 8, own_bit)
    assert ((acc[hit] & own_bit[hit]) != 0).mean() > 0.999
    assert (spp[hit] == 2).mean() > 0.99


def _fit_single_block(true_w, seed=0):
    """Builds one 32x32 block of tmp data whose colour is exactly linear in the
    (scaled) features and returns (weights, mins_maxs, features)."""
    rng = np.random.default_rng(seed)
    W = H = 64
    o = Oracle(W, H, use_half=False)
    tmp = o.new_tmp().reshape(o.blocks, 13, 1024)
    n = rng.normal(size=(1024, 3))
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    p = rng.uniform(-3, 3, size=(1024, 3))
    feats = np.concatenate([np.ones((1024, 1)), n, p, p * p], axis=1).astype(np.float32)
    mn, mx = feats[:, 4:].min(0), feats[:, 4:].max(0)
    scaled = feats.copy()
    rngmm = mx - mn
    scaled[:, 4:] = np.where(np.abs(rngmm) > 1, (feats[:, 4:] - mn) / rngmm, feats[:, 4:] - mn)
    colour = scaled.astype(np.float64) @ true_w
    for b in range(o.blocks):
        tmp[b, :10] = feats.T
        tmp[b, 10:] = colour.T
    w = np.zeros(o.blocks * 30, np.float32)
    mm = np.zeros(o.blocks * 12, np.float32)
    return o, tmp, w, mm, scaled, colour


def test_fitter_recovers_linear_model():
    rng = np.random.default_rng(1)
    true_w = rng.uniform(-1, 1, size=(10, 3))
    o, tmp, w, mm, scaled, colour = _fit_single_block(true_w)
    o.fitter(w, mm, tmp.reshape(-1), frame=3, mode=FITTER_FP64)
    wb = w.reshape(o.blocks, 10, 3)[0]
    pred = scaled @ wb
    rel = np.abs(pred - colour).max() / np.abs(colour).max()
    assert rel < 0.05, rel   # the fitter's +-1e-2 feature noise biases the fit slightly


def test_fitter_modes_agree():
    W = H = 128
    sc, fr = _scene_inputs(W, H, frames=1)
    o = Oracle(W, H, sc.position_limit_squared, sc.normal_limit_squared)
    d = fr[0]
    tmp, pp = o.new_tmp(), np.zeros((H, W, 2), np.float32)
    acc, spp = np.zeros((H, W), np.uint8), np.zeros((H, W), np.uint8)
    o.accumulate_noisy_data(pp, acc, d["normals"], None, d["positions"], None, d["noisy"].copy(), None, None, spp,
                            tmp, sc.camera(0), sc.pixel_offset(0), 0)
    outs = {}
    for mode in (FITTER_REFERENCE, FITTER_FP32, FITTER_FP64):
        w = np.zeros(o.blocks * 30, np.float32)
        mm = np.zeros(o.blocks * 12, np.float32)
        o.fitter(w, mm, tmp.copy(), 0, mode)
        out = np.zeros((H, W, 3), np.float32)
        o.weighted_sum(w, mm, out, d["normals"], d["positions"], 0)
        outs[mode] = out
    scale = np.abs(outs[FITTER_FP64]).mean()
    assert np.abs(outs[FITTER_FP32] - outs[FITTER_FP64]).mean() < 1e-3 * scale
    assert np.abs(outs[FITTER_REFERENCE] - outs[FITTER_FP64]).mean() < 3e-2 * scale


def test_oracle_pipeline_denoises():
    W = H = 128
    import bmfr_b200 as B
    sc = B.Scene(7, W, H, 12)
    pipe = OraclePipeline(Oracle(W, H, sc.position_limit_squared, sc.normal_limit_squared))
    psnr = []
    for f in range(6):
        d = sc.render(f, clean=True)
        out = pipe.step(d["albedo"], d["normals"], d["positions"], d["noisy"], sc.prev_camera(f),
                        sc.pixel_offset(f))
        noisy_tm = np.clip(np.maximum(0, d["albedo"] * d["noisy"]) ** 0.454545, 0, 1)
        mse = lambda a: np.mean((a - d["clean"]) ** 2)
        psnr.append((10 * np.log10(1 / mse(noisy_tm)), 10 * np.log10(1 / mse(out))))
        assert np.isfinite(out).all()
    assert psnr[-1][1] > psnr[-1][0] + 8.0
    assert psnr[-1][1] > psnr[0][1]
