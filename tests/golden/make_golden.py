"""Writes the reference fixtures tests/golden/ref_pipeline.npz,
tests/golden/ref_pipeline_f32.npz and tests/golden/ref_stages.npz.

The outputs come from the reference's own OpenCL kernels (opencl/bmfr.cl),
compiled for the CPU by oracle/ref_cl (oracle.ref.RefKernels), run on the
seeded inputs of tests/golden/cases.py; the inputs are stored beside them so
the fixtures do not depend on the scene generator staying unchanged.  Needs
the reference source (or a built oracle/_ref/libbmfr_ref.so):

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE))

import cases  # noqa: E402
from oracle.oracle import OraclePipeline  # noqa: E402
from oracle.ref import RefKernels  # noqa: E402


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def run_pipeline(use_half=True):
    """The scene frames through the reference's kernels; with use_half=False
    (tmp_data in float32, the reference's USE_HALF_PRECISION_IN_TMP_DATA=0)
    only the outputs are kept: the inputs are ref_pipeline.npz's."""
    frames, pos_lim, nrm_lim = cases.pipeline_inputs()
    w, h = cases.PIPELINE_SIZE
    pipe = OraclePipeline(RefKernels(w, h, pos_lim, nrm_lim, use_half=use_half))
    out = {"limits": np.array([pos_lim, nrm_lim], np.float32)}
    for f, d in enumerate(frames):
        res = pipe.step(d["albedo"], d["normals"], d["positions"], d["noisy"], d["matrix"], d["offset"])
        c = f & 1
        if use_half:
            for k in ("albedo", "normals", "positions", "noisy", "matrix", "offset"):
                out[f"in{f}_{k}"] = d[k]
        out[f"out{f}_result"] = res.copy()
        out[f"out{f}_tone_mapped"] = pipe.tone_mapped.copy()
        out[f"out{f}_weights"] = pipe.weights.copy()
        out[f"out{f}_mins_maxs"] = pipe.mins_maxs.copy()
        out[f"out{f}_accept"] = pipe.accept.copy()
        out[f"out{f}_spp"] = pipe.spp[c].copy()
        out[f"out{f}_prev_pix"] = pipe.prev_pix.copy()
        out[f"out{f}_noisy_acc"] = pipe.noisy[c].copy()
        out[f"sha{f}_tmp"] = np.array(sha(pipe.tmp_after_accumulate.view(np.uint16 if use_half else np.uint32)))
        out[f"sha{f}_filtered"] = np.array(sha(pipe.filtered))
        out[f"sha{f}_acc"] = np.array(sha(pipe.acc[c]))
    return out


def run_stages():
    d = cases.stage_inputs()
    w, h = cases.STAGE_SIZE
    f = int(d["frame"][0])
    ref = RefKernels(w, h, float(d["limits"][0]), float(d["limits"][1]))
    px = w * h
    out = {f"in_{k}": v for k, v in d.items()}

    pp = np.zeros((h, w, 2), np.float32)
    acc = np.zeros((h, w), np.uint8)
    spp = np.zeros((h, w), np.uint8)
    noisy = d["cur_noisy"].copy()
    tmp = ref.new_tmp()
    ref.accumulate_noisy_data(pp, acc, d["cur_normals"], d["prev_normals"], d["cur_positions"], d["prev_positions"],
                              noisy, d["prev_noisy"], d["prev_spp"], spp, tmp, d["matrix"], d["offset"], f)
    out.update(out_acc_prev_pix=pp, out_acc_accept=acc, out_acc_spp=spp, out_acc_noisy=noisy, out_acc_tmp=tmp.copy())

    fit_in = cases.patch_fit_blocks(tmp.copy(), d["fit_blocks"])
    weights = np.zeros(ref.blocks * 30, np.float32)
    mm = np.zeros(ref.blocks * 12, np.float32)
    t = fit_in.copy()
    ref.fitter(weights, mm, t, f)
    out.update(in_fit_tmp=fit_in, out_fit_weights=weights, out_fit_mins_maxs=mm)
    out["sha_fit_tmp_after"] = np.array(sha(t.view(np.uint16)))

    filt = np.zeros((h, w, 3), np.float32)
    ref.weighted_sum(weights, mm, filt, d["cur_normals"], d["cur_positions"], f)
    out["out_ws_filtered"] = filt

    tone = np.zeros((h, w, 3), np.float32)
    acc_cur = np.zeros((h, w, 3), np.float32)
    ref.accumulate_filtered_data(filt, d["prev_pix"], d["accept"], d["albedo"], tone, d["cur_spp"], d["acc_prev"],
                                 acc_cur, f)
    out.update(out_af_tone_mapped=tone, out_af_accumulated=acc_cur)

    res = np.zeros((h, w, 3), np.float32)
    ref.taa(d["taa_prev_pix"], tone, res, d["taa_prev"], f)
    out["out_taa_result"] = res
    assert px == h * w
    return out


def main():
    for name, fn in (("ref_pipeline.npz", run_pipeline), ("ref_pipeline_f32.npz", lambda: run_pipeline(False)),
                     ("ref_stages.npz", run_stages)):
        data = fn()
        np.savez_compressed(HERE / name, **data)
        print(f"{name}: {(HERE / name).stat().st_size / 1024:.0f} KiB, {len(data)} arrays")


if __name__ == "__main__":
    main()
