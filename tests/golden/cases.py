"""Seeded inputs of the reference fixtures (tests/golden/*.npz).

Two kinds of case:

* `pipeline_inputs` — consecutive frames of the procedural scene, run through
  the reference host program's frame loop;
* `stage_inputs` — one frame's inputs for each of the five kernels, taken
  from the scene and then pushed into the kernels' edge branches: NaN, +-inf
  and values beyond binary16 in the noisy colour and the positions (the NaN
  test and the +-65504 clamp of bmfr.cl:461-468, reprojections that leave
  the image), spp up to 255 (the saturation of bmfr.cl:436-441) and 0 (a
  division by zero in bmfr.cl:837), tmp_data blocks with constant, all-zero
  and +-65504 features (the two branches of scale(), bmfr.cl:200-205, and a
  degenerate QR), bilinear positions on and beyond every image edge.

Every array the kernels read is consistent with what the reference's own
pipeline can hand them where an inconsistent value would make a kernel read
outside its buffers (the accept bits of accumulate_filtered_data select
taps that exist), so the same inputs are safe for the CUDA kernels.
"""
from __future__ import annotations

import numpy as np

PIPELINE_SIZE = (72, 48)      # margin grid 128 x 96: 4 x 3 blocks
PIPELINE_FRAMES = 3
PIPELINE_SEED = 5
STAGE_SIZE = (56, 48)         # margin grid 96 x 96: 3 x 3 blocks
STAGE_FRAME = 23              # block offset 7
STAGE_SEED = 17


def geometry(w, h):
    ww, wh = 32 * ((w + 31) // 32), 32 * ((h + 31) // 32)
    mw, mh = ww + 32, wh + 32
    return mw, mh, (mw // 32) * (mh // 32)


def pipeline_inputs():
    """Frames of a 12-sphere scene: list of dicts (albedo, normals, positions,
    noisy, matrix, offset) plus the two test limits."""
    import bmfr_b200 as B
    w, h = PIPELINE_SIZE
    sc = B.Scene(PIPELINE_SEED, w, h, 12)
    frames = []
    for f in range(PIPELINE_FRAMES):
        d = sc.render(f)
        frames.append({k: d[k] for k in ("albedo", "normals", "positions", "noisy")}
                      | {"matrix": sc.prev_camera(f).astype(np.float32),
                         "offset": sc.pixel_offset(f).astype(np.float32)})
    return frames, float(sc.position_limit_squared), float(sc.normal_limit_squared)


def _pick(rng, n, k):
    return rng.choice(n, size=k, replace=False)


def stage_inputs(seed=STAGE_SEED, frame=STAGE_FRAME):
    """One frame's adversarial inputs for every stage (dict of arrays).  The
    defaults give the committed fixture; other seeds and frames (>= 1) give
    further cases of the same kinds, frame % 16 picking the block offset."""
    import bmfr_b200 as B
    w, h = STAGE_SIZE
    px = w * h
    mw, mh, blocks = geometry(w, h)
    rng = np.random.default_rng(seed)
    sc = B.Scene(seed, w, h, 16)
    prev, cur = sc.render(frame - 1), sc.render(frame)
    d = {"limits": np.array([sc.position_limit_squared, sc.normal_limit_squared], np.float32),
         "frame": np.array([frame], np.int32),
         "matrix": sc.prev_camera(frame).astype(np.float32),
         "offset": sc.pixel_offset(frame).astype(np.float32)}

    # accumulate_noisy_data.  The extreme values sit in the top 12 rows only:
    # one value clamped to 65504 overflows the binary16 QR of its whole block
    # (NaN weights), so the blocks below stay on the ordinary path.
    top = 12 * w
    noisy = cur["noisy"].reshape(px, 3).copy()
    idx = _pick(rng, top, 36)
    noisy[idx[:4]] = np.nan
    noisy[idx[4:6]] = np.inf
    noisy[idx[6:8]] = -np.inf
    noisy[idx[8:14]] = rng.uniform(7e4, 1e6, (6, 3))
    noisy[idx[14:26]] = rng.uniform(-3.0, -0.01, (12, 3))
    noisy[idx[26:]] = 0.0
    pos = cur["positions"].reshape(px, 3).copy()
    idx = _pick(rng, top, 16)
    pos[idx[:4]] = np.nan
    pos[idx[4:8]] = rng.uniform(260.0, 400.0, (4, 3))       # x*x beyond 65504
    pos[idx[8:12], 0] = np.inf
    idx = _pick(rng, px, 40)
    pos[idx] = pos[idx] + 1e-4                                # moved within the limit
    d.update(cur_normals=cur["normals"], prev_normals=prev["normals"], cur_positions=pos.reshape(h, w, 3),
             prev_positions=prev["positions"], cur_noisy=noisy.reshape(h, w, 3),
             prev_noisy=np.abs(rng.normal(0.5, 0.5, (h, w, 3))).astype(np.float32),
             prev_spp=rng.integers(0, 256, (h, w), dtype=np.uint8))
    d["prev_spp"].reshape(-1)[_pick(rng, px, 200)] = 255

    # fitter: a tmp_data of the scene frame (filled by the caller's
    # accumulate) is replaced block-wise by these patterns.
    d["fit_blocks"] = np.array([0, 4, 8], np.int32)         # constant / zero / +-65504 blocks

    # weighted_sum: the fitter's outputs are used (NaN weights included).

    # accumulate_filtered_data: prev positions around every edge; accept bits
    # only for taps inside the image.
    ppx = rng.uniform(-2.5, w + 1.5, px).astype(np.float32)
    ppy = rng.uniform(-2.5, h + 1.5, px).astype(np.float32)
    edge = _pick(rng, px, 60)
    ppx[edge[:10]] = -1.0
    ppx[edge[10:20]] = np.float32(w - 1)
    ppy[edge[20:30]] = -1.0
    ppy[edge[30:40]] = np.float32(h - 1)
    ppx[edge[40:50]] = np.nan
    ppy[edge[50:]] = np.inf
    prev_pix = np.stack([ppx, ppy], -1)
    fx = np.floor(np.nan_to_num(ppx, nan=-1e9, posinf=1e9, neginf=-1e9))
    fy = np.floor(np.nan_to_num(ppy, nan=-1e9, posinf=1e9, neginf=-1e9))
    accept = np.zeros(px, np.uint8)
    for bit, (dx, dy) in enumerate(((0, 0), (1, 0), (0, 1), (1, 1))):
        inside = (fx + dx >= 0) & (fx + dx < w) & (fy + dy >= 0) & (fy + dy < h)
        keep = inside & (rng.random(px) < 0.8)
        accept |= (keep.astype(np.uint8) << bit)
    spp = rng.integers(1, 256, px, dtype=np.uint8)
    spp[_pick(rng, px, 30)] = 0
    d.update(prev_pix=prev_pix.reshape(h, w, 2), accept=accept.reshape(h, w), cur_spp=spp.reshape(h, w),
             albedo=cur["albedo"], acc_prev=np.abs(rng.normal(0.4, 0.4, (h, w, 3))).astype(np.float32))

    # taa: previous result; its own prev positions (NaN and far outside included)
    tpx = rng.uniform(-3.0, w + 2.0, px).astype(np.float32)
    tpy = rng.uniform(-3.0, h + 2.0, px).astype(np.float32)
    e = _pick(rng, px, 40)
    tpx[e[:10]] = np.nan
    tpy[e[10:20]] = -np.inf
    tpx[e[20:30]] = -1.0
    tpy[e[30:]] = np.float32(h - 1)
    d.update(taa_prev_pix=np.stack([tpx, tpy], -1).reshape(h, w, 2),
             taa_prev=np.abs(rng.normal(0.5, 0.3, (h, w, 3))).astype(np.float32))
    return d


def patch_fit_blocks(tmp: np.ndarray, blocks, rng_seed=STAGE_SEED):
    """Writes the three adversarial block patterns into tmp_data (block-major,
    13 columns of 1024 values per block): constant features, an all-zero
    block, and features at +-65504."""
    rng = np.random.default_rng(rng_seed + 1)
    t = tmp.reshape(-1, 13, 1024)
    b0, b1, b2 = (int(b) for b in blocks)
    t[b0, :10] = t.dtype.type(0.75)                 # every feature constant: max - min = 0
    t[b0, 4:7] = t.dtype.type(300.0)                # scaled columns constant above 1
    t[b1] = 0
    t[b2, 1:10] = rng.choice(np.array([-65504.0, 65504.0, 0.0], np.float32), (9, 1024)).astype(t.dtype)
    return tmp


def edge_frame(d, rng, w, h):
    """A scene frame with a few edge values written in at random pixels:
    NaN, +-inf and beyond-binary16 colours, NaN and out-of-range positions
    (the stage fixture's kinds, here carried through the histories of the
    following frames)."""
    px = w * h
    noisy = d["noisy"].reshape(px, 3).copy()
    pos = d["positions"].reshape(px, 3).copy()
    idx = rng.choice(px, size=8, replace=False)
    noisy[idx[:2]] = np.nan
    noisy[idx[2]] = np.inf
    noisy[idx[3]] = -np.inf
    noisy[idx[4:6]] = rng.uniform(7e4, 1e6, (2, 3))
    pos[idx[6]] = np.nan
    pos[idx[7]] = rng.uniform(260.0, 400.0, 3)
    return dict(d, noisy=noisy.reshape(h, w, 3), positions=pos.reshape(h, w, 3))
