"""The oracle pinned to the reference itself.

The reference's OpenCL kernels (opencl/bmfr.cl) are compiled for the CPU by
oracle/ref_cl and run through oracle.ref.RefKernels.  Their outputs are kept
as fixtures (tests/golden/ref_*.npz, written by tests/golden/make_golden.py),
so the first two tests pin the oracle even where the reference source is
absent; the others run the compiled reference live when it can be built.
Every comparison is bit for bit (NaN equal to NaN).
"""
import hashlib
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import Oracle, OraclePipeline
from oracle import ref as REF

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))


def same(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape and a.dtype == b.dtype, what
    if a.dtype.kind == "f":
        eq = (a == b) | (np.isnan(a) & np.isnan(b))
    else:
        eq = a == b
    assert eq.all(), f"{what}: {int((~eq).sum())} of {eq.size} values differ"


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("fixture,use_half", [("ref_pipeline.npz", True), ("ref_pipeline_f32.npz", False)])
def test_oracle_reproduces_reference_pipeline_fixture(fixture, use_half):
    """binary16 tmp_data (the reference's default) and float32 tmp_data
    (its USE_HALF_PRECISION_IN_TMP_DATA=0), on the same scene frames."""
    inp = np.load(GOLDEN / "ref_pipeline.npz")
    g = np.load(GOLDEN / fixture)
    frames = sum(1 for k in g.files if k.endswith("_result"))
    H, W = inp["in0_albedo"].shape[:2]
    lim = g["limits"]
    pipe = OraclePipeline(Oracle(W, H, float(lim[0]), float(lim[1]), use_half=use_half))
    for f in range(frames):
        res = pipe.step(*(inp[f"in{f}_{k}"] for k in ("albedo", "normals", "positions", "noisy", "matrix", "offset")))
        c = f & 1
        same(res, g[f"out{f}_result"], f"result {f}")
        same(pipe.tone_mapped, g[f"out{f}_tone_mapped"], f"tone mapped {f}")
        same(pipe.weights, g[f"out{f}_weights"], f"weights {f}")
        same(pipe.mins_maxs, g[f"out{f}_mins_maxs"], f"mins_maxs {f}")
        same(pipe.accept, g[f"out{f}_accept"], f"accept {f}")
        same(pipe.spp[c], g[f"out{f}_spp"], f"spp {f}")
        same(pipe.prev_pix, g[f"out{f}_prev_pix"], f"prev_frame_pixel {f}")
        same(pipe.noisy[c], g[f"out{f}_noisy_acc"], f"accumulated noisy {f}")
        tmp_bits = pipe.tmp_after_accumulate.view(np.uint16 if use_half else np.uint32)
        assert sha(tmp_bits) == str(g[f"sha{f}_tmp"]), f"tmp_data {f}"
        assert sha(pipe.filtered) == str(g[f"sha{f}_filtered"]), f"filtered {f}"
        assert sha(pipe.acc[c]) == str(g[f"sha{f}_acc"]), f"accumulated filtered {f}"


def run_stages(k, g):
    """The five stages of kernel set `k` (Oracle or RefKernels) on the stage
    fixture's inputs; returns the outputs under the fixture's names."""
    H, W = g["in_albedo"].shape[:2]
    f = int(g["in_frame"][0])
    o = k(W, H, float(g["in_limits"][0]), float(g["in_limits"][1]))
    out = {}
    pp = np.zeros((H, W, 2), np.float32)
    acc = np.zeros((H, W), np.uint8)
    spp = np.zeros((H, W), np.uint8)
    noisy = g["in_cur_noisy"].copy()
    tmp = o.new_tmp()
    o.accumulate_noisy_data(pp, acc, g["in_cur_normals"], g["in_prev_normals"], g["in_cur_positions"],
                            g["in_prev_positions"], noisy, g["in_prev_noisy"], g["in_prev_spp"], spp, tmp,
                            g["in_matrix"], g["in_offset"], f)
    out.update(out_acc_prev_pix=pp, out_acc_accept=acc, out_acc_spp=spp, out_acc_noisy=noisy, out_acc_tmp=tmp)
    weights = np.zeros(o.blocks * 30, np.float32)
    mm = np.zeros(o.blocks * 12, np.float32)
    t = g["in_fit_tmp"].copy()
    o.fitter(weights, mm, t, f)
    out.update(out_fit_weights=weights, out_fit_mins_maxs=mm)
    out["sha_fit_tmp_after"] = sha(t.view(np.uint16))
    filt = np.zeros((H, W, 3), np.float32)
    o.weighted_sum(g["out_fit_weights"], g["out_fit_mins_maxs"], filt, g["in_cur_normals"], g["in_cur_positions"], f)
    out["out_ws_filtered"] = filt
    tone = np.zeros((H, W, 3), np.float32)
    acc_cur = np.zeros((H, W, 3), np.float32)
    o.accumulate_filtered_data(g["out_ws_filtered"], g["in_prev_pix"], g["in_accept"], g["in_albedo"], tone,
                               g["in_cur_spp"], g["in_acc_prev"], acc_cur, f)
    out.update(out_af_tone_mapped=tone, out_af_accumulated=acc_cur)
    res = np.zeros((H, W, 3), np.float32)
    o.taa(g["in_taa_prev_pix"], g["out_af_tone_mapped"], res, g["in_taa_prev"], f)
    out["out_taa_result"] = res
    return out


def test_oracle_reproduces_reference_stage_fixture():
    """Edge inputs (NaN, infinities, values beyond binary16, spp 0 and 255,
    degenerate blocks, reprojections on and beyond the image edges)."""
    g = np.load(GOLDEN / "ref_stages.npz")
    out = run_stages(Oracle, g)
    for name, v in out.items():
        if name.startswith("sha_"):
            assert v == str(g[name]), name
        else:
            same(v, g[name], name)
    # The fixture does reach the edge branches it is meant for.
    assert np.isnan(g["out_fit_weights"]).any() and np.isfinite(g["out_fit_weights"]).mean() > 0.5
    assert (g["out_acc_spp"] == 255).any() and (g["in_cur_spp"] == 0).any()
    assert np.isnan(g["out_acc_prev_pix"]).any() and (g["out_acc_accept"] > 0).mean() > 0.2


needs_ref = pytest.mark.skipif(not REF.available(), reason="reference kernel source and oracle/_ref library absent")


@needs_ref
@pytest.mark.parametrize("W,H,frames,half", [(128, 96, 17, True), (200, 120, 4, True), (160, 96, 4, False),
                                             (32, 32, 17, True), (47, 63, 17, True), (64, 48, 17, False)])
def test_oracle_matches_compiled_reference(W, H, frames, half):
    """Frame loops over the oracle and over the reference's kernels: every
    intermediate buffer identical, tmp_data after the fitter included (the
    QR intermediates the reference leaves there).  17 frames cover all 16
    block offsets.  32x32 and 47x63 are the smallest images whose mirrored
    margin stays within one image size (mirror, bmfr.cl:209-216): there the
    margin reaches the last valid index."""
    import bmfr_b200 as B
    sc = B.Scene(21, W, H, 12)
    kw = dict(position_limit_squared=sc.position_limit_squared, normal_limit_squared=sc.normal_limit_squared,
              use_half=half)
    po, pr = OraclePipeline(Oracle(W, H, **kw)), OraclePipeline(REF.RefKernels(W, H, **kw))
    for f in range(frames):
        d = sc.render(f)
        args = (d["albedo"], d["normals"], d["positions"], d["noisy"], sc.prev_camera(f), sc.pixel_offset(f))
        same(po.step(*args), pr.step(*args), f"result {f}")
        c = f & 1
        for name in ("tmp_after_accumulate", "tmp", "prev_pix", "accept", "mins_maxs", "weights", "filtered",
                     "tone_mapped"):
            same(getattr(po, name), getattr(pr, name), f"{name} {f}")
        for name in ("spp", "noisy", "acc", "result"):
            same(getattr(po, name)[c], getattr(pr, name)[c], f"{name} {f}")


@needs_ref
@pytest.mark.parametrize("half", [True, False])
def test_oracle_matches_compiled_reference_with_edge_frames(half):
    """17 consecutive frames (all 16 block offsets) of the scene with edge
    values written into every fourth frame, so NaN and overflowing values
    pass through the spp, colour and TAA histories: every buffer of the
    oracle and of the compiled reference equal bit for bit, frame after
    frame."""
    import bmfr_b200 as B
    import cases
    W, H = 64, 48
    sc = B.Scene(41, W, H, 12)
    rng = np.random.default_rng(41)
    kw = dict(position_limit_squared=sc.position_limit_squared, normal_limit_squared=sc.normal_limit_squared,
              use_half=half)
    po, pr = OraclePipeline(Oracle(W, H, **kw)), OraclePipeline(REF.RefKernels(W, H, **kw))
    nan_hist = False
    for f in range(17):
        d = sc.render(f)
        if f % 4 == 1:   # edge values every fourth frame; the histories carry them between
            d = cases.edge_frame(d, rng, W, H)
        args = (d["albedo"], d["normals"], d["positions"], d["noisy"], sc.prev_camera(f), sc.pixel_offset(f))
        same(po.step(*args), pr.step(*args), f"result {f}")
        c = f & 1
        for name in ("tmp_after_accumulate", "tmp", "prev_pix", "accept", "mins_maxs", "weights", "filtered",
                     "tone_mapped"):
            same(getattr(po, name), getattr(pr, name), f"{name} {f}")
        for name in ("spp", "noisy", "acc", "result"):
            same(getattr(po, name)[c], getattr(pr, name)[c], f"{name} {f}")
        nan_hist = nan_hist or bool(np.isnan(pr.acc[c]).any())
    # NaN reached the accumulated filtered history (whose bilinear reads
    # spread it, as the reference's do), and the last frame still has lit
    # pixels of the scene.
    assert nan_hist and (pr.result[16 & 1] > 0).mean() > 0.05


@needs_ref
def test_stage_fixture_is_the_reference_output():
    """The committed edge-case fixture is what the compiled reference gives
    on its inputs today (the fixture and the runner agree)."""
    g = np.load(GOLDEN / "ref_stages.npz")
    out = run_stages(REF.RefKernels, g)
    for name, v in out.items():
        if name.startswith("sha_"):
            assert v == str(g[name]), name
        else:
            same(v, g[name], name)


def stage_chain(k, d, seed):
    """The five stages of kernel set `k` on stage inputs `d`
    (cases.stage_inputs), each fed by the previous stage's outputs and the
    fitter by the accumulation's tmp_data with the adversarial blocks
    written in; returns every output."""
    import cases
    w, h = cases.STAGE_SIZE
    f = int(d["frame"][0])
    o = k(w, h, float(d["limits"][0]), float(d["limits"][1]))
    out = {}
    pp = np.zeros((h, w, 2), np.float32)
    acc = np.zeros((h, w), np.uint8)
    spp = np.zeros((h, w), np.uint8)
    noisy = d["cur_noisy"].copy()
    tmp = o.new_tmp()
    o.accumulate_noisy_data(pp, acc, d["cur_normals"], d["prev_normals"], d["cur_positions"], d["prev_positions"],
                            noisy, d["prev_noisy"], d["prev_spp"], spp, tmp, d["matrix"], d["offset"], f)
    out.update(prev_pix=pp, accept=acc, spp=spp, noisy=noisy, tmp=tmp.copy())
    t = cases.patch_fit_blocks(tmp, d["fit_blocks"], rng_seed=seed)
    weights = np.zeros(o.blocks * 30, np.float32)
    mm = np.zeros(o.blocks * 12, np.float32)
    o.fitter(weights, mm, t, f)
    out.update(weights=weights, mins_maxs=mm, tmp_after_fit=t)
    filt = np.zeros((h, w, 3), np.float32)
    o.weighted_sum(weights, mm, filt, d["cur_normals"], d["cur_positions"], f)
    tone = np.zeros((h, w, 3), np.float32)
    acc_cur = np.zeros((h, w, 3), np.float32)
    o.accumulate_filtered_data(filt, d["prev_pix"], d["accept"], d["albedo"], tone, d["cur_spp"], d["acc_prev"],
                               acc_cur, f)
    res = np.zeros((h, w, 3), np.float32)
    o.taa(d["taa_prev_pix"], tone, res, d["taa_prev"], f)
    out.update(filtered=filt, tone_mapped=tone, accumulated=acc_cur, result=res)
    return out


@needs_ref
@pytest.mark.parametrize("offset", range(16))
def test_oracle_matches_compiled_reference_on_edge_inputs(offset):
    """The stage fixture's kinds of edge inputs (NaN, infinities, values
    beyond binary16, spp 0 and 255, constant, zero and +-65504 blocks,
    history positions on and beyond every edge) drawn anew for each of the
    16 block offsets (frame 16 + offset), through the oracle and the
    reference's compiled kernels: every output equal bit for bit."""
    import cases
    seed = 1000 + offset
    d = cases.stage_inputs(seed=seed, frame=16 + offset)
    a = stage_chain(Oracle, d, seed)
    b = stage_chain(REF.RefKernels, d, seed)
    for name in a:   # in stage order: the first difference names its stage
        same(a[name], b[name], f"{name} (block offset {offset})")
    # The case reaches the edge branches it is drawn for.
    assert np.isnan(b["weights"]).any() and (b["spp"] == 255).any() and np.isnan(b["prev_pix"]).any()
    assert 0.2 < (b["accept"] > 0).mean() < 1.0


def test_prepare_rules_fail_loudly():
    """The source preparation rewrites exactly the constructs it expects."""
    sys.path.insert(0, str(Path(REF.__file__).resolve().parent / "ref_cl"))
    import prepare
    src = ("__kernel void k(__local float *a,\n      __local float3 *b) {\n"
           "   __local float u, v;\n   local float3 d;\n   c = c < 0.f ? 0.f : c;\n}\n")
    out = prepare.prepare(src, "x.cl")
    assert "CLC_KERNEL_LOCAL float u, v;" in out and "CLC_KERNEL_LOCAL float3 d;" in out
    assert "clc_vselect(c < 0.f, 0.f, c)" in out and "__local float *a," in out
    with pytest.raises(SystemExit):
        prepare.prepare(src.replace("local float3 d;", "float3 d;"), "x.cl")
