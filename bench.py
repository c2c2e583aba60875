"""Benchmark of the BMFR per-frame denoising pipeline on B200.

Workload: the plain BMFR pipeline at 1280x720 (five stages per frame) over a
seeded 12-sphere procedural scene of 60 frames, replayed forwards and
backwards.  One step = one denoised frame.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Our arm prints one JSON line with
  value      frames/s of the fused pipeline, inputs resident in HBM (all ranks),
  e2e        frames/s through the C ABI from pinned host buffers, with the
             four input uploads and the result download inside the timed region,
  stages     ms per stage (the reference's per-kernel profile, bmfr.cpp:488-517),
  roofline   the dominant kernel's achieved HBM bandwidth against the measured
             copy bandwidth,
  cpu_baseline  the CPU oracle (a port of the reference's kernels) on a bounded
             sample of frames on this host's cores.
--impl reference times that CPU port alone (the reference's OpenCL kernels
have no runnable platform here).  Under torchrun every rank denoises its own
stream (replicas, no collective on the data path); rank 0 prints.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WIDTH, HEIGHT, FRAMES, SPHERES, SEED = 1280, 720, 60, 12, 20240601
METRIC = "720p frames/s, full BMFR pipeline (accumulate, fitter, weighted sum, filtered accumulation, TAA)"


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def geometry(w, h):
    ww, wh = 32 * ((w + 31) // 32), 32 * ((h + 31) // 32)
    mw, mh = ww + 32, wh + 32
    return mw * mh, (mw // 32) * (mh // 32)


def stage_bytes(w, h):
    """Algorithmic HBM bytes per launch of each stage (fp32 buffers, half tmp)."""
    P = w * h
    Pm, B = geometry(w, h)
    return {
        "accumulate_noisy_data": 95 * P + 26 * Pm,
        "fitter": 26 * Pm + 168 * B,
        "weighted_sum": 36 * P,
        "accumulate_filtered_data": 70 * P,
        "weighted_sum+accumulate_filtered_data": 82 * P,
        "taa": 44 * P,
        "noise_table": 9 * 4 * 256 * 4,
        # accumulate (95 B/px + 26 B read per margin pixel from the inputs, no
        # tmp_data) + weighted sum and filtered accumulation (82 B/px less the
        # 24 B/px of N, P re-read from L2) -> counted once per byte of HBM.
        "block_kernel": 95 * P + 24 * (Pm - P) + 168 * B + 58 * P,
    }


def frame_order(i, n):
    """Triangle wave over 0..n-1 so the camera never jumps."""
    period = 2 * (n - 1)
    k = i % period
    return k if k < n else period - k


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            out, _ = self.proc.communicate(timeout=10)
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            try:
                sm.append(float(f[0]))
                mx = max(mx, float(f[1]))
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, f[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def render_frames(seed, w, h, n):
    import bmfr_b200 as B
    sc = B.Scene(seed, w, h, SPHERES)
    frames = [sc.render(f) for f in range(n)]
    return sc, frames


def cpu_port_frames_per_s(w, h, frames, sc, budget_s=12.0, min_frames=3, threads=0):
    """The oracle pipeline over the first frames until the time budget ends."""
    from oracle.oracle import Oracle, OraclePipeline
    pipe = OraclePipeline(Oracle(w, h, sc.position_limit_squared, sc.normal_limit_squared, threads=threads))
    # Frame 0 has no history; time frames 1.. as the reference's stats do.
    d = frames[0]
    pipe.step(d["albedo"], d["normals"], d["positions"], d["noisy"], sc.prev_camera(0), sc.pixel_offset(0))
    n, t0 = 0, time.perf_counter()
    while n < len(frames) - 1:
        f = n + 1
        d = frames[f]
        pipe.step(d["albedo"], d["normals"], d["positions"], d["noisy"], sc.prev_camera(f), sc.pixel_offset(f))
        n += 1
        if n >= min_frames and time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return n / dt, n, dt


def run_reference(args, world, rank):
    """CPU port of the reference's kernels on all host cores."""
    if rank != 0:
        return
    cores = os.cpu_count()
    sc, frames = render_frames(SEED, WIDTH, HEIGHT, min(FRAMES, args.steps + args.warmup + 1))
    from oracle.oracle import Oracle, OraclePipeline
    pipe = OraclePipeline(Oracle(WIDTH, HEIGHT, sc.position_limit_squared, sc.normal_limit_squared))
    nf = len(frames)
    for i in range(args.warmup):
        f = frame_order(i, nf)
        d = frames[f]
        pipe.step(d["albedo"], d["normals"], d["positions"], d["noisy"], sc.prev_camera(f), sc.pixel_offset(f))
    t0 = time.perf_counter()
    for i in range(args.warmup, args.warmup + args.steps):
        f = frame_order(i, nf)
        d = frames[f]
        pipe.step(d["albedo"], d["normals"], d["positions"], d["noisy"], sc.prev_camera(f), sc.pixel_offset(f))
    dt = time.perf_counter() - t0
    v = args.steps / dt
    sample = f"{args.steps} full 1280x720 frames of the oracle pipeline (5 stages), OpenMP over {cores} threads"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "frames/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "BMFR plain pipeline 1280x720, 12-sphere procedural scene", "width": WIDTH,
                   "height": HEIGHT, "frames": FRAMES, "parallelism": "host cores"},
        "cpu_baseline": {"value": v, "unit": "frames/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's OpenCL kernels have no runnable platform on this box; this is the oracle port",
    }), flush=True)


BATCH_STREAMS = [(640, 360)] * 8 + [(1280, 720)] * 8 + [(1920, 1080)] * 6 + [(3840, 2160)] * 2
BATCH_FRAMES = 30


def batch_scenes(rank):
    """The batched form's 24 streams: own seed, U{8..32} spheres, U[0.2,1.0] deg/frame."""
    import bmfr_b200 as B
    rng = np.random.default_rng(SEED + 17 + rank)
    return [B.Scene(SEED + 1000 * rank + k, w, h, int(rng.integers(8, 33)),
                    orbit_degrees_per_frame=float(rng.uniform(0.2, 1.0)))
            for k, (w, h) in enumerate(BATCH_STREAMS)]


def run_batched(args, world, rank, local, dev, barrier, pg):
    """Batched form: 24 streams of uneven size, one graph-captured step per
    frame of every stream, binary16 histories and FP32 QR, autotuned; next to
    the plain per-frame path on the same streams."""
    import torch
    import bmfr_b200 as B
    scenes = batch_scenes(rank)
    nfr = max(2, min(args.frames, BATCH_FRAMES))
    stream = torch.cuda.Stream(device=dev)
    frames = []
    for sc in scenes:
        px = sc.width * sc.height * 3
        fl = []
        for f in range(nfr):
            d = {k: torch.empty(px, dtype=torch.float32, device=dev) for k in ("albedo", "normals", "positions", "noisy")}
            sc.render_device(f, d["albedo"], d["normals"], d["positions"], d["noisy"], stream=stream)
            fl.append(d)
        frames.append(fl)
    stream.synchronize()
    n = len(scenes)
    params = B.default_params(pipeline=B.PIPELINE_FUSED, fp32_qr=1, half_history=1)
    batch = B.Batch(params)
    slots = [batch.add_stream(sc.width, sc.height) for sc in scenes]

    def step_args(i):
        f = frame_order(i, nfr)
        pf = frame_order(i - 1, nfr) if i > 0 else f
        io = []
        for k in range(n):
            d, p = frames[k][f], frames[k][pf]
            io.append(B.Batch.frame_io(d["albedo"], d["normals"], d["positions"], d["noisy"], p["normals"],
                                       p["positions"]))
        mats = np.concatenate([sc.camera(pf) for sc in scenes])
        offs = np.concatenate([sc.pixel_offset(f) for sc in scenes])
        return io, mats, offs

    io0, m0, o0 = step_args(0)
    tuning, tuned_ms = batch.autotune(slots, m0, o0, io=io0, steps=2, stream=stream)
    for sl in slots:
        batch.reset_stream(sl)
    for i in range(args.warmup):
        io, m, o = step_args(i)
        batch.step(slots, m, o, io=io, stream=stream)
    stream.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        e0.record(stream)
        for i in range(args.warmup, args.warmup + args.steps):
            io, m, o = step_args(i)
            batch.step(slots, m, o, io=io, stream=stream)
        e1.record(stream)
        e1.synchronize()
    ms = e0.elapsed_time(e1)
    if pg is not None:
        t = torch.tensor([ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
    value = world * n * args.steps / (ms / 1e3)
    batch.close()

    # The plain path (reference arithmetic, float histories, staged pipeline)
    # on the same streams, one frame at a time.
    plans = [B.Plan(sc.width, sc.height, position_limit_squared=sc.position_limit_squared,
                    normal_limit_squared=sc.normal_limit_squared) for sc in scenes]
    plain_steps = min(args.steps, 10)

    def plain_step(i):
        f = frame_order(i, nfr)
        pf = frame_order(i - 1, nfr) if i > 0 else f
        for k, (sc, pl) in enumerate(zip(scenes, plans)):
            d, p = frames[k][f], frames[k][pf]
            pl.denoise_frame_io(d["albedo"], d["normals"], d["positions"], d["noisy"], p["normals"], p["positions"],
                                sc.camera(pf), sc.pixel_offset(f), stream=stream)

    for i in range(3):
        plain_step(i)
    stream.synchronize()
    e0.record(stream)
    for i in range(3, 3 + plain_steps):
        plain_step(i)
    e1.record(stream)
    e1.synchronize()
    plain_ms = e0.elapsed_time(e1)
    plain_value = n * plain_steps / (plain_ms / 1e3)
    for pl in plans:
        pl.close()
    pixels = sum(w * h for w, h in BATCH_STREAMS)
    if rank == 0:
        print(json.dumps({
            "form": "batched", "metric": "multi-stream frames/s (24 streams: 8x640x360, 8x1280x720, 6x1920x1080, 2x3840x2160)",
            "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 math, f16 histories", "data": "synthetic (device-rendered, 30 frames per stream)",
            "config": {"workload": "batched form, 24 streams", "streams": len(BATCH_STREAMS),
                       "pixels_per_step": pixels, "frames": nfr, "tuning": {
                           "block_ctas_per_sm": tuning.block_ctas_per_sm, "taa_tile": [tuning.taa_tile_w, tuning.taa_tile_h],
                           "staging_depth": tuning.staging_depth}, "tuned_ms_per_step": tuned_ms},
            "plain_path": {"value": plain_value, "unit": "frames/s", "ms_per_round": plain_ms / plain_steps,
                           "how": "one plan per stream, staged pipeline, reference arithmetic, frames in turn"},
            "speedup_vs_plain": value / plain_value / world,
            "clocks": clocks.summary(), "gpu_launches": 3 * args.steps,
        }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=240)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--pipeline", default="staged", choices=["fused", "staged"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--frames", type=int, default=FRAMES, help="distinct scene frames held in HBM")
    ap.add_argument("--form", default="plain", choices=["plain", "batched", "served", "precision"])
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world, rank, local = dist_setup()

    if args.impl == "reference":
        run_reference(args, world, rank)
        return

    import torch
    import bmfr_b200 as B

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
        pg = dist

    def barrier():
        if pg is not None:
            pg.barrier()

    if args.form == "batched":
        run_batched(args, world, rank, local, dev, barrier, pg)
        if pg is not None:
            pg.destroy_process_group()
        return

    # Inputs: every rank denoises its own stream (replicas).
    nfr = max(2, min(args.frames, FRAMES))
    sc, frames = render_frames(SEED + rank, WIDTH, HEIGHT, nfr)
    mats = [sc.camera(f) for f in range(nfr)]
    off = sc.pixel_offset(0)
    stack = lambda k: torch.from_numpy(np.stack([f[k] for f in frames])).pin_memory()
    host = {k: stack(k) for k in ("albedo", "normals", "positions", "noisy")}
    devf = {k: v.to(dev) for k, v in host.items()}
    pipeline = B.PIPELINE_FUSED if args.pipeline == "fused" else B.PIPELINE_STAGED
    plan = B.Plan(WIDTH, HEIGHT, pipeline=pipeline, position_limit_squared=sc.position_limit_squared,
                  normal_limit_squared=sc.normal_limit_squared)
    stream = torch.cuda.Stream(device=dev)

    def step_resident(i):
        f = frame_order(i, nfr)
        pf = frame_order(i - 1, nfr) if i > 0 else f
        plan.denoise_frame_io(devf["albedo"][f], devf["normals"][f], devf["positions"][f], devf["noisy"][f],
                              devf["normals"][pf], devf["positions"][pf], mats[pf], off, stream=stream)

    # ---- value: device-resident inputs ---------------------------------------
    with torch.cuda.stream(stream):
        for i in range(args.warmup):
            step_resident(i)
    stream.synchronize()
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        ev0.record(stream)
        for i in range(args.warmup, args.warmup + args.steps):
            step_resident(i)
        ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    barrier()
    elapsed_ms = ev0.elapsed_time(ev1)
    if pg is not None:
        t = torch.tensor([elapsed_ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        elapsed_ms = float(t.item())
    value = world * args.steps / (elapsed_ms / 1e3)
    # noise table, block kernel, taa (fused); noise table, accumulate, fitter,
    # weighted_sum, accumulate_filtered, taa (staged)
    launches_per_frame = 3 if pipeline == B.PIPELINE_FUSED else 6

    # ---- per-stage profile (same workload, events between stages) ------------
    plan.enable_profiling(True)
    stage_ms = {}
    base = args.warmup + args.steps
    nprof = min(args.steps, 60)
    for i in range(base, base + nprof):
        step_resident(i)
        for k, v in plan.stage_times().items():
            stage_ms.setdefault(k, []).append(v)
    plan.enable_profiling(False)
    stages = {k: float(np.mean(v)) for k, v in stage_ms.items() if v}
    sb = stage_bytes(WIDTH, HEIGHT)
    dominant = max(stages, key=stages.get)
    hbm_peak, peak_kind = peaks()
    achieved = sb[dominant] / (stages[dominant] * 1e-3) / 1e9
    roofline = {"kernel": dominant, "bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                "frac": achieved / hbm_peak, "peak_source": peak_kind, "bytes_per_launch": sb[dominant],
                "traffic": None}
    stage_gbs = {k: sb[k] / (v * 1e-3) / 1e9 for k, v in stages.items() if v > 0}

    # ---- e2e: host buffers through the C ABI --------------------------------
    plan.reset()
    out_host = torch.empty((HEIGHT, WIDTH, 3), dtype=torch.float32).pin_memory()

    def step_e2e(i):
        f = frame_order(i, nfr)
        pf = frame_order(i - 1, nfr) if i > 0 else f
        plan.upload_frame(host["albedo"][f], host["normals"][f], host["positions"][f], host["noisy"][f],
                          stream=stream)
        plan.denoise_frame(mats[pf], off, stream=stream)
        plan.download_result(out_host, stream=stream)

    for i in range(args.warmup):
        step_e2e(i)
    stream.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_steps = min(args.steps, 120)
    e0.record(stream)
    for i in range(args.warmup, args.warmup + e2e_steps):
        step_e2e(i)
    e1.record(stream)
    e1.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    if pg is not None:
        t = torch.tensor([e2e_ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e = {"value": world * e2e_steps / (e2e_ms / 1e3), "unit": "frames/s",
           "h2d_bytes_per_step": 4 * WIDTH * HEIGHT * 12, "d2h_bytes_per_step": WIDTH * HEIGHT * 12}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        fps, n, dt = cpu_port_frames_per_s(WIDTH, HEIGHT, frames, sc)
        cpu = {"value": fps, "unit": "frames/s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"{n} consecutive 1280x720 frames of the oracle pipeline ({dt:.1f} s)"}

    plan.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "BMFR plain pipeline 1280x720, 12-sphere procedural scene, 60 frames replayed",
                       "width": WIDTH, "height": HEIGHT, "frames": nfr, "pipeline": args.pipeline,
                       "tmp_data": "binary16", "parallelism": f"replicas x{world}",
                       "l2": "no flush: per-frame working set ~180 MB (inputs + histories) exceeds the 126 MB L2"},
            "stages_ms": stages, "stages_gbs": stage_gbs,
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "clocks": clocks.summary(), "gpu_launches": launches_per_frame * args.steps,
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
