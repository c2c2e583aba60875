"""Benchmark of the BMFR per-frame denoising pipeline on B200.

Workload: the plain BMFR pipeline at 1280x720 (five stages per frame) over a
seeded 12-sphere procedural scene of 60 frames, replayed forwards and
backwards.  One step = one denoised frame.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Our arm prints one JSON line with
  value      frames/s of the plan pipeline (staged by default), inputs
             resident in HBM (all ranks); the K-step loop repeats until at
             least 0.5 s have passed and its median gives the step time,
  e2e        frames/s through the C ABI from pinned host buffers, with the
             four input uploads and the result download inside the timed region,
  stages     ms per stage (the reference's per-kernel profile, bmfr.cpp:488-517),
  roofline   the dominant kernel against its bound: the fitter's warp-
             instruction rate against the SMs' issue rate (it is issue-bound),
             with its HBM figures beside it; an HBM-bound kernel's bandwidth
             against the measured copy bandwidth,
  batched    the multi-stream half of the metric: 24 streams of uneven size
             per step, frames/s, step latency p50/p99, and the ratios to the
             plain path and to plans of the same arithmetic,
  served     64 Poisson render streams through the request server: frames/s
             and frame latency p50/p99, beside the plain path on the same
             trace, and the capacity of both,
  cpu_baseline  the reference's own OpenCL kernels compiled for the CPU
             (oracle/_ref) on a bounded sample of frames on this host's cores,
             with the oracle port's figure beside it.
--impl reference times the reference's kernels alone (the port where they
are not built).  --gpus N starts N ranks, one process per GPU, unless a
launcher already did (a rank count other than N is an error); every rank
denoises its own streams (replicas, no collective on the data path) and
rank 0 prints.
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


def max_over_ranks(value, device=None):
    """The slowest rank's value (bmfr_b200.replicas; imported here so that the
    reference arm maps no pipeline code)."""
    from bmfr_b200.replicas import max_over_ranks as m
    return m(value, device=device)

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
        # one pass: N, P, prev_pix, accept, albedo, spp, acc_prev read; acc_cur
        # and tone_mapped written (float histories; the filtered colour stays
        # on chip)
        "weighted_sum+accumulate_filtered_data": 82 * P,
        "taa": 44 * P,
        "noise_table": 9 * 4 * 256 * 4,
        # accumulate (95 B/px, and the margin-only pixels' 24 B of N, P read
        # again from their mirror) and the fit's weights and min/max; no
        # tmp_data
        "block_kernel": 95 * P + 24 * (Pm - P) + 168 * B,
    }


# DRAM bytes (read + write) per launch at 1280x720 from one ncu capture of
# the kernel (`bench.py --form probe --frames 6 --qr 0`, frame 3's launch;
# profiles/k_fitter_720p.md, k_taa_720p.md).
NCU_TRAFFIC_720P = {"fitter": 26.78e6, "taa": 25.94e6}
# Warp instructions per launch at 1280x720 (smsp__inst_executed.sum of the
# same captures): the numerator of the issue-rate roofline of a kernel that
# is bound by instruction issue rather than by HBM.
NCU_WARP_INST_720P = {"fitter": 47.24e6, "taa": 11.43e6}
SMS, SCHEDULERS_PER_SM = 148, 4
# Kernels bound by instruction issue rather than by HBM or tensor cores.
ISSUE_BOUND = {"fitter": "the fitter is a sequence of small dependent reductions and rank-one updates kept "
                         "bit-identical to the reference (no FMA contraction, correctly rounded quotients, binary16 "
                         "rounding at every store): bound by instruction issue, not by HBM (it reads its 26 MB "
                         "once) or tensor cores; stages_gbs shows the HBM-bound stages"}


MIN_TIMED_SECONDS = 0.5   # each timed region repeats its K-step loop at least this long


def timed_loops(run_steps, stream, dev, min_seconds=MIN_TIMED_SECONDS, max_loops=2000):
    """Times `run_steps(loop)` (one loop = K steps launched on `stream`) with
    CUDA events on `stream`, repeating the loop until `min_seconds` of device
    time have passed, so that the clock sampler sees the run.  The first loop
    sets the count, the largest over ranks, so every rank takes the same
    collective steps.  Returns the device milliseconds of every loop."""
    import torch
    evs = []

    def one(loop):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run_steps(loop)
        e1.record(stream)
        evs.append((e0, e1))

    one(0)
    evs[0][1].synchronize()
    first = evs[0][0].elapsed_time(evs[0][1])
    loops = int(min(max_loops, max(1, -(-min_seconds * 1e3 // max(first, 1e-3)))))
    loops = int(max_over_ranks(float(loops), device=dev))
    for loop in range(1, loops):
        one(loop)
    evs[-1][1].synchronize()
    return [a.elapsed_time(b) for a, b in evs]


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


def launch_command(gpus, argv, port=None):
    """The command that runs this benchmark as `gpus` ranks on this node, one
    process per GPU, rendezvous on 127.0.0.1."""
    if port is None:
        import socket
        with socket.socket() as so:
            so.bind(("127.0.0.1", 0))
            port = so.getsockname()[1]
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={gpus}",
            "--master-addr", "127.0.0.1", "--master-port", str(port), str(Path(__file__).resolve()), *argv]


def check_world(world, gpus):
    """A run whose rank count differs from --gpus is an error, not a silent
    one-GPU measurement."""
    if world != gpus:
        raise SystemExit(f"bench.py: --gpus {gpus} but the launcher started {world} rank(s)")


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def render_frames(seed, w, h, n):
    from bmfr_scene import Scene   # the input source alone: no pipeline library
    sc = Scene(seed, w, h, SPHERES)
    frames = [sc.render(f) for f in range(n)]
    return sc, frames


def host_threads():
    """Host threads this process may run on.  Passed to the CPU kernels
    explicitly: under torchrun OMP_NUM_THREADS is 1 in every rank, while the
    CPU arms run on rank 0 alone and should use the whole host."""
    try:
        return len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def cpu_kernels(kind, w, h, sc, threads=0):
    """The CPU implementations of the five kernels: "reference" = the
    reference's own OpenCL kernels compiled for the CPU (oracle/_ref, a fiber
    per work-item at the fitter's barriers), "port" = the oracle restatement
    (bit-identical outputs, one loop per kernel)."""
    from oracle.oracle import Oracle
    if kind == "reference":
        from oracle.ref import RefKernels
        return RefKernels(w, h, sc.position_limit_squared, sc.normal_limit_squared, threads=threads)
    return Oracle(w, h, sc.position_limit_squared, sc.normal_limit_squared, threads=threads)


def reference_available():
    try:
        from oracle import ref
        return ref.available()
    except Exception:
        return False


def cpu_frames_per_s(kind, w, h, frames, sc, budget_s=12.0, min_frames=3, max_frames=None, threads=0, warmup=1):
    """The frame loop over CPU kernels: `warmup` untimed frames (at least
    frame 0, which has no history; the reference's own statistics start at
    frame 1 too), then timed frames until the time budget ends; frames replay
    forwards and backwards."""
    from oracle.oracle import OraclePipeline
    pipe = OraclePipeline(cpu_kernels(kind, w, h, sc, threads))
    nf = len(frames)
    warmup = max(1, warmup)
    for i in range(warmup):
        f = frame_order(i, nf)
        d = frames[f]
        pipe.step(d["albedo"], d["normals"], d["positions"], d["noisy"], sc.prev_camera(f), sc.pixel_offset(f))
    n, t0, stage_s = 0, time.perf_counter(), {}
    while max_frames is None or n < max_frames:
        f = frame_order(n + warmup, nf)
        d = frames[f]
        pipe.step(d["albedo"], d["normals"], d["positions"], d["noisy"], sc.prev_camera(f), sc.pixel_offset(f))
        for k, v in pipe.stage_seconds.items():
            stage_s[k] = stage_s.get(k, 0.0) + v
        n += 1
        if n >= min_frames and time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return n / dt, n, dt, {k: 1e3 * v / n for k, v in stage_s.items()}


def cpu_baseline(frames, sc, ref_budget_s, port_budget_s):
    """cpu_baseline object: the reference's kernels on this host's cores when
    they are built, else the port; the port's figure rides along."""
    cores = host_threads()
    fps_p, n_p, dt_p, st_p = cpu_frames_per_s("port", WIDTH, HEIGHT, frames, sc, budget_s=port_budget_s,
                                              threads=cores)
    port = {"value": fps_p, "unit": "frames/s", "cores": cores, "kind": "port",
            "sample": f"{n_p} consecutive 1280x720 frames of the oracle pipeline ({dt_p:.1f} s)", "stages_ms": st_p}
    if not reference_available():
        return port
    fps, n, dt, st = cpu_frames_per_s("reference", WIDTH, HEIGHT, frames, sc, budget_s=ref_budget_s,
                                      threads=cores)
    return {"value": fps, "unit": "frames/s", "cores": cores, "kind": "reference",
            "sample": f"{n} consecutive 1280x720 frames of the reference's OpenCL kernels compiled for the CPU "
                      f"(oracle/_ref), OpenMP over {cores} threads ({dt:.1f} s)",
            "stages_ms": st, "port": port}


def run_reference(args, world, rank):
    """The reference's own kernels (oracle/_ref) on all host cores, on a
    bounded sample: min(--warmup, 3) warm-up frames, then up to --steps
    frames within a 90 s budget.  Falls back to the oracle port when the reference kernels
    are not built."""
    if rank != 0:
        return
    cores = host_threads()
    kind = "reference" if reference_available() else "port"
    warm = min(max(args.warmup, 1), 3)
    sc, frames = render_frames(SEED, WIDTH, HEIGHT, min(FRAMES, args.steps + warm + 1))
    fps, n, dt, stages = cpu_frames_per_s(kind, WIDTH, HEIGHT, frames, sc, budget_s=90.0,
                                          min_frames=min(3, args.steps), max_frames=args.steps, warmup=warm,
                                          threads=cores)
    what = ("the reference's OpenCL kernels (opencl/bmfr.cl) compiled for the CPU, a fiber per work-item "
            "at the fitter's barriers" if kind == "reference" else "the oracle port of the reference's kernels")
    sample = (f"{n} of {args.steps} requested full 1280x720 frames (90 s budget) of {what}, "
              f"OpenMP over {cores} threads; {warm} warm-up frames")
    line = {
        "impl": "reference", "metric": METRIC, "value": fps, "unit": "frames/s", "n_gpus": args.gpus,
        "steps": n, "steps_requested": args.steps, "warmup": warm, "warmup_requested": args.warmup_requested,
        "ms_per_step": 1e3 * dt / n,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "BMFR plain pipeline 1280x720, 12-sphere procedural scene", "width": WIDTH,
                   "height": HEIGHT, "frames": FRAMES, "parallelism": "host cores"},
        "cpu_baseline": {"value": fps, "unit": "frames/s", "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": fps, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "stages_ms": stages,
    }
    if kind == "reference":
        fps_p, n_p, dt_p, st_p = cpu_frames_per_s("port", WIDTH, HEIGHT, frames, sc, budget_s=20.0,
                                                  max_frames=args.steps, warmup=warm, threads=cores)
        line["port"] = {"value": fps_p, "unit": "frames/s", "cores": cores, "kind": "port", "frames": n_p,
                        "stages_ms": st_p,
                        "note": "the oracle restatement: bit-identical outputs, one loop per kernel"}
    else:
        line["note"] = "the reference kernels are not built here (oracle/_ref); this is the oracle port"
    print(json.dumps(line), flush=True)


BATCH_STREAMS = [(640, 360)] * 8 + [(1280, 720)] * 8 + [(1920, 1080)] * 6 + [(3840, 2160)] * 2
BATCH_FRAMES = 30


def batch_scenes(rank):
    """The batched form's 24 streams: own seed, U{8..32} spheres, U[0.2,1.0] deg/frame."""
    import bmfr_b200 as B
    rng = np.random.default_rng(SEED + 17 + rank)
    return [B.Scene(SEED + 1000 * rank + k, w, h, int(rng.integers(8, 33)),
                    orbit_degrees_per_frame=float(rng.uniform(0.2, 1.0)))
            for k, (w, h) in enumerate(BATCH_STREAMS)]


def measure_batched(args, world, rank, local, dev, barrier, steps, warmup):
    """Batched form: 24 streams of uneven size, one step per frame of every
    stream (staged: each stream's plan kernels on eight worker CUDA streams;
    fused: one graph-captured launch over all streams' blocks), binary16
    histories and FP32 QR (CholeskyQR2).  Beside it, the same streams one
    frame at a time through (a) the plain path (reference arithmetic, float
    histories: the drop-in path the batched form is compared with) and (b) plans with the batch's own
    arithmetic and histories (the gain of batching alone).  Returns the
    measurement as a dict."""
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
    pipeline = B.PIPELINE_FUSED if args.pipeline == "fused" else B.PIPELINE_STAGED
    params = B.default_params(pipeline=pipeline, fp32_qr=1, half_history=1)
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
    # Step arguments prepared up front: the timed loop only launches.
    prepared = [step_args(i) for i in range(2 * (nfr - 1))]
    for i in range(warmup):
        io, m, o = prepared[i % len(prepared)]
        batch.step(slots, m, o, io=io, stream=stream)
    stream.synchronize()
    barrier()
    step_events = []

    def k_steps(loop):
        for i in range(steps):
            io, m, o = prepared[(warmup + loop * steps + i) % len(prepared)]
            batch.step(slots, m, o, io=io, stream=stream)
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(stream)
            step_events.append(ev)

    with ClockSampler(local) as clocks:
        loop_ms = timed_loops(k_steps, stream, dev)
    stream.synchronize()
    # Device time of each step: between the events that close it and the
    # step before it (the first step of each loop is left out).
    per_step = [step_events[j - 1].elapsed_time(step_events[j]) for j in range(1, len(step_events))
                if j % steps != 0]
    ms = max_over_ranks(statistics.median(loop_ms), device=dev)   # the slowest rank
    value = world * n * steps / (ms / 1e3)
    batch.close()

    def plans_in_turn(plan_kw, rounds):
        """The same streams one frame at a time through their own plans."""
        plans = [B.Plan(sc.width, sc.height, position_limit_squared=sc.position_limit_squared,
                        normal_limit_squared=sc.normal_limit_squared, **plan_kw) for sc in scenes]

        def one_round(i):
            f = frame_order(i, nfr)
            pf = frame_order(i - 1, nfr) if i > 0 else f
            for k, (sc, pl) in enumerate(zip(scenes, plans)):
                d, p = frames[k][f], frames[k][pf]
                pl.denoise_frame_io(d["albedo"], d["normals"], d["positions"], d["noisy"], p["normals"],
                                    p["positions"], sc.camera(pf), sc.pixel_offset(f), stream=stream)

        for i in range(3):
            one_round(i)
        stream.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(3, 3 + rounds):
            one_round(i)
        e1.record(stream)
        e1.synchronize()
        t = e0.elapsed_time(e1)
        for pl in plans:
            pl.close()
        return n * rounds / (t / 1e3), t / rounds

    rounds = max(3, min(steps, 10))
    plain_value, plain_round_ms = plans_in_turn({}, rounds)
    prec_value, prec_round_ms = plans_in_turn(dict(fp32_qr=1, half_history=1, pipeline=pipeline), rounds)
    pixels = sum(w * h for w, h in BATCH_STREAMS)
    return {
        "metric": "multi-stream frames/s (24 streams: 8x640x360, 8x1280x720, 6x1920x1080, 2x3840x2160)",
        "value": value, "unit": "frames/s", "steps": steps, "timed_loops": len(loop_ms),
        "ms_per_step": ms / steps,
        "step_latency_ms": {"p50": float(np.percentile(per_step, 50)), "p99": float(np.percentile(per_step, 99)),
                            "how": "device time of each step (every stream's frame is done when its step ends)"},
        "dtype": "f32 math, f16 histories", "data": "synthetic (device-rendered, 30 frames per stream)",
        "config": {"workload": "batched form, 24 streams", "streams": len(BATCH_STREAMS), "pipeline": args.pipeline,
                   "qr": "CholeskyQR2 (FP32)", "pixels_per_step": pixels, "frames": nfr, "tuning": {
                       "block_ctas_per_sm": tuning.block_ctas_per_sm, "taa_tile": [tuning.taa_tile_w, tuning.taa_tile_h],
                       "staging_depth": tuning.staging_depth}, "tuned_ms_per_step": tuned_ms},
        "plain_path": {"value": plain_value, "unit": "frames/s", "ms_per_round": plain_round_ms,
                       "how": "one plan per stream, staged pipeline, reference arithmetic, float histories, "
                              "frames in turn"},
        "same_arithmetic_plans": {"value": prec_value, "unit": "frames/s", "ms_per_round": prec_round_ms,
                                  "how": "one plan per stream with the batch's parameters (CholeskyQR2, binary16 "
                                         "histories, same pipeline), frames in turn"},
        "speedup_vs_plain": value / plain_value / world,
        "speedup_vs_same_arithmetic_plans": value / prec_value / world,
        "clocks": clocks.summary(),
        # per step: noise table, block kernel, (pixel pass,) TAA (fused); per
        # stream noise table, accumulation, fitter, weighted sum + filtered
        # accumulation, TAA (staged)
        "gpu_launches": (3 + tuning.pixel_pass if pipeline == B.PIPELINE_FUSED else 5 * n) * steps
                        * len(loop_ms),
    }


def run_batched(args, world, rank, local, dev, barrier, pg):
    """--form batched: the batched measurement as its own JSON line."""
    r = measure_batched(args, world, rank, local, dev, barrier, args.steps, args.warmup)
    if rank == 0:
        r.update({"form": "batched", "n_gpus": world, "warmup": args.warmup, "higher_is_better": True,
                  "scaling": "weak", "vs_baseline": None})
        print(json.dumps(r), flush=True)


SERVED_SEATS = 64
SERVED_MIX = [((640, 360), 0.4), ((1280, 720), 0.4), ((1920, 1080), 0.15), ((3840, 2160), 0.05)]
SERVED_BUDGET = 120 * 10**9
SERVED_POOL = 16          # distinct rendered frames per resolution class
SERVED_LIFETIME = 300     # mean frames a stream lives


def served_trace(seed, seconds):
    """Arrival trace of the served form.  64 seats; the stream on a seat
    draws its size from the resolution mix and its rate from {30, 60} Hz,
    lives Geometric(1/300) frames whose requests arrive as a Poisson process,
    then leaves, and a new stream joins the seat after an exponential pause
    (mean 50 ms).  Events: (t, kind 0 open / 1 frame / 2 close, stream, a)."""
    rng = np.random.default_rng(seed)
    probs = [p for _, p in SERVED_MIX]
    period = 2 * (SERVED_POOL - 1)
    events, streams = [], []
    for seat in range(SERVED_SEATS):
        t = float(rng.uniform(0.0, 0.05))
        while t < seconds:
            sid = len(streams)
            cls = int(rng.choice(len(SERVED_MIX), p=probs))
            rate = float(rng.choice([30.0, 60.0]))
            life = int(rng.geometric(1.0 / SERVED_LIFETIME))
            streams.append({"cls": cls, "rate": rate, "phase": int(rng.integers(0, period))})
            events.append((t, 0, sid, 0))
            for f in range(life):
                t += float(rng.exponential(1.0 / rate))
                if t >= seconds:
                    break
                events.append((t, 1, sid, f))
            t += 1e-4
            events.append((t, 2, sid, 0))
            t += float(rng.exponential(0.05))
    events.sort()
    return events, streams


def drive_trace(events, t0, on_event):
    """Plays the trace in real time from t0 (perf_counter seconds)."""
    for ev in events:
        dt = t0 + ev[0] - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        on_event(ev)


def measure_served(args, world, rank, local, dev, barrier, seconds):
    """Served form: 64 render streams with Poisson frame requests at 30/60 Hz,
    joining and leaving, histories resident in HBM, admission against a
    120 GB budget; the request server (continuous batching) next to the
    plain per-frame path fed the same trace, and the capacity of both (every
    stream always ready).  Returns the measurement as a dict."""
    import queue
    import threading
    from concurrent.futures import ThreadPoolExecutor
    import torch
    import bmfr_b200 as B
    stream = torch.cuda.Stream(device=dev)
    period = 2 * (SERVED_POOL - 1)
    # Input pools: SERVED_POOL rendered frames per resolution class, walked
    # forwards and backwards by each stream from its own phase.
    pools = []
    for cls, ((w, h), _) in enumerate(SERVED_MIX):
        sc = B.Scene(SEED + 4000 + 100 * rank + cls, w, h, 8 + 8 * cls)
        px = w * h * 3
        fr = []
        for f in range(SERVED_POOL):
            d = {k: torch.empty(px, dtype=torch.float32, device=dev) for k in ("albedo", "normals", "positions", "noisy")}
            sc.render_device(f, d["albedo"], d["normals"], d["positions"], d["noisy"], stream=stream)
            fr.append(d)
        tab = []
        for i in range(period):
            f, pf = frame_order(i, SERVED_POOL), frame_order(i - 1, SERVED_POOL)
            d, p = fr[f], fr[pf]
            tab.append((B.Batch.frame_io(d["albedo"], d["normals"], d["positions"], d["noisy"], p["normals"],
                                         p["positions"]), sc.camera(pf), sc.pixel_offset(f), d, p))
        pools.append({"w": w, "h": h, "sc": sc, "frames": fr, "tab": tab})
    stream.synchronize()
    params = B.default_params(pipeline=B.PIPELINE_FUSED if args.pipeline == "fused" else B.PIPELINE_STAGED,
                              fp32_qr=1, half_history=1,
                              position_limit_squared=pools[0]["sc"].position_limit_squared,
                              normal_limit_squared=pools[0]["sc"].normal_limit_squared)
    seconds = float(seconds)
    warm_s = min(1.0, seconds / 4)
    events, streams = served_trace(SEED + 4242 + rank, seconds)
    n_req = sum(1 for e in events if e[1] == 1 and e[0] >= warm_s)

    # ---- capacity: every seat's first stream, one frame each per step --------
    first = {}
    for e in events:
        if e[1] == 0 and len(first) < SERVED_SEATS and e[2] not in first:
            first[e[2]] = streams[e[2]]
    cap_streams = list(first.values())[:SERVED_SEATS]
    batch = B.Batch(params)
    slots = [batch.add_stream(pools[st["cls"]]["w"], pools[st["cls"]]["h"]) for st in cap_streams]

    def cap_args(i):
        io, mats, offs = [], [], []
        for st in cap_streams:
            e = pools[st["cls"]]["tab"][(st["phase"] + i) % period]
            io.append(e[0])
            mats.append(e[1])
            offs.append(e[2])
        return io, np.concatenate(mats), np.concatenate(offs)

    io0, m0, o0 = cap_args(0)
    tuning, _ = batch.autotune(slots, m0, o0, io=io0, steps=2, stream=stream)
    cap_steps = 20
    for i in range(3):
        batch.step(slots, *cap_args(i)[1:], io=cap_args(i)[0], stream=stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(3, 3 + cap_steps):
        io, m, o = cap_args(i)
        batch.step(slots, m, o, io=io, stream=stream)
    e1.record(stream)
    e1.synchronize()
    cap_batched = len(cap_streams) * cap_steps / (e0.elapsed_time(e1) / 1e3)
    batch.close()

    plain_params = dict(position_limit_squared=params.position_limit_squared,
                        normal_limit_squared=params.normal_limit_squared)

    def capacity_of_plans(kw):
        cap_plans = [B.Plan(pools[st["cls"]]["w"], pools[st["cls"]]["h"], **plain_params, **kw)
                     for st in cap_streams]

        def plain_round(i):
            for st, pl in zip(cap_streams, cap_plans):
                _, m, o, d, p = pools[st["cls"]]["tab"][(st["phase"] + i) % period]
                pl.denoise_frame_io(d["albedo"], d["normals"], d["positions"], d["noisy"], p["normals"],
                                    p["positions"], m, o, stream=stream)

        for i in range(3):
            plain_round(i)
        plain_rounds = 5
        e0.record(stream)
        for i in range(3, 3 + plain_rounds):
            plain_round(i)
        e1.record(stream)
        e1.synchronize()
        v = len(cap_streams) * plain_rounds / (e0.elapsed_time(e1) / 1e3)
        for pl in cap_plans:
            pl.close()
        torch.cuda.synchronize()
        return v

    cap_plain = capacity_of_plans({})
    cap_same = capacity_of_plans(dict(fp32_qr=params.fp32_qr, half_history=params.half_history,
                                      pipeline=params.pipeline))

    # ---- the server saturated: every capacity stream's next frames queued at
    # once, so that each step takes a frame of every stream -------------------
    sat_frames = 8
    sat = B.Server(params)
    sat.set_tuning(tuning)
    sat_ids = [sat.open_stream(pools[st["cls"]]["w"], pools[st["cls"]]["h"]) for st in cap_streams]
    for i in range(2):   # warm-up frames
        for st, sid in zip(cap_streams, sat_ids):
            io, m, o = pools[st["cls"]]["tab"][(st["phase"] + i) % period][:3]
            sat.submit(sid, m, o, io=io)
    sat.drain(120000)
    sat.reset_stats()
    ts = time.perf_counter()
    for i in range(2, 2 + sat_frames):
        for st, sid in zip(cap_streams, sat_ids):
            io, m, o = pools[st["cls"]]["tab"][(st["phase"] + i) % period][:3]
            sat.submit(sid, m, o, io=io)
    sat.drain(120000)
    sat_s = time.perf_counter() - ts
    sst = sat.stats()
    for sid in sat_ids:
        sat.close_stream(sid)
    sat.close()
    torch.cuda.synchronize()
    saturated = {"value": len(cap_streams) * sat_frames / sat_s, "unit": "frames/s",
                 "frames_per_step": sst["mean_frames_per_step"], "steps": int(sst["steps"]),
                 "latency_ms": {"p50": sst["p50_latency_ms"], "p99": sst["p99_latency_ms"]},
                 "how": f"{len(cap_streams)} streams, {sat_frames} frames each submitted at once through the "
                        f"server (wall clock from the first submit to the drain); latency here is mostly "
                        f"queueing"}

    # Peak stream memory and peak open streams per class over the trace:
    # both paths reserve them before the trace starts.
    live, peak_bytes, per_cls, peak_cls = 0, 0, [0] * len(SERVED_MIX), [0] * len(SERVED_MIX)
    for t, kind, sid, a in events:
        c = streams[sid]["cls"]
        nbytes = B.Batch.stream_bytes(params, pools[c]["w"], pools[c]["h"])
        if kind == 0:
            live += nbytes
            per_cls[c] += 1
        elif kind == 2:
            live -= nbytes
            per_cls[c] -= 1
        peak_bytes = max(peak_bytes, live)
        peak_cls = [max(x, y) for x, y in zip(peak_cls, per_cls)]

    # ---- served: the request server on the trace -----------------------------
    server = B.Server(params, memory_budget_bytes=SERVED_BUDGET,
                      reserve_bytes=min(SERVED_BUDGET, int(peak_bytes * 1.25)))
    server.set_tuning(tuning)
    # Streams are opened and closed on helper threads, as separate render
    # clients would: a stream's frames are submitted once it is admitted
    # (frames that arrive while its admission is pending are not sent).
    opening = {}
    closer = ThreadPoolExecutor(max_workers=8)
    closes = []
    reset_done = [False]
    submitted = []          # (seconds into the trace, request id)
    open_ms = []
    not_admitted_yet = [0]

    def do_open(w, h):
        ta = time.perf_counter()
        try:
            sid_ = server.open_stream(w, h)
        except B.BmfrError as err:
            if err.status != B._native.BMFR_E_BUDGET:
                raise
            sid_ = None
        open_ms.append(1e3 * (time.perf_counter() - ta))
        return sid_

    def do_close(fut):
        sid_ = fut.result()
        if sid_ is not None:
            server.close_stream(sid_)

    def on_event_batched(ev):
        t, kind, sid, a = ev
        if not reset_done[0] and t >= warm_s:
            server.reset_stats()
            reset_done[0] = True
        st = streams[sid]
        pool = pools[st["cls"]]
        if kind == 0:
            opening[sid] = closer.submit(do_open, pool["w"], pool["h"])
        elif kind == 1:
            fut = opening[sid]
            if not fut.done():
                not_admitted_yet[0] += 1
            elif fut.result() is not None:
                io, m, o = pool["tab"][(st["phase"] + a) % period][:3]
                rid = server.submit(fut.result(), m, o, io=io)
                if reset_done[0]:
                    submitted.append((t, rid))
        else:
            closes.append(closer.submit(do_close, opening[sid]))

    barrier()
    with ClockSampler(local) as clocks:
        t0 = time.perf_counter()
        drive_trace(events, t0, on_event_batched)
        server.drain(120000)
        t_end = time.perf_counter()
    for c in closes:
        c.result()
    closer.shutdown()
    st = server.stats()
    by_second = {}
    for t, rid in submitted:
        ok, ms = server.poll(rid)
        by_second.setdefault(int(t), []).append(ms)
    server.close()
    served_fps = st["requests_completed"] / max(st["elapsed_seconds"], 1e-9)

    # ---- the plain per-frame path on the same trace ----------------------------
    # One plan per stream, made (or taken from the plans of closed streams) on
    # helper threads as the server's streams are; one worker launches the
    # frames in arrival order.
    work = queue.SimpleQueue()
    done = queue.SimpleQueue()
    free_plans = {k: [] for k in range(len(SERVED_MIX))}
    free_mu = threading.Lock()
    plan_of = {}
    lat = []
    plan_ms = []
    plain_not_admitted = [0]
    helper = ThreadPoolExecutor(max_workers=8)
    for c, n in enumerate(peak_cls):
        free_plans[c] = [B.Plan(pools[c]["w"], pools[c]["h"], **plain_params) for _ in range(n)]
    torch.cuda.synchronize()

    def make_plan(cls):
        ta = time.perf_counter()
        with free_mu:
            pl = free_plans[cls].pop() if free_plans[cls] else None
        if pl is None:
            pl = B.Plan(pools[cls]["w"], pools[cls]["h"], **plain_params)
        pl.reset()
        plan_ms.append(1e3 * (time.perf_counter() - ta))
        return pl

    def worker():
        while True:
            item = work.get()
            if item is None:
                done.put(None)
                return
            kind, sid, a, t_arr = item
            stt = streams[sid]
            pool = pools[stt["cls"]]
            if kind == 1:
                _, m, o, d, p = pool["tab"][(stt["phase"] + a) % period]
                plan_of[sid].result().denoise_frame_io(d["albedo"], d["normals"], d["positions"], d["noisy"],
                                                       p["normals"], p["positions"], m, o, stream=stream)
                ev = torch.cuda.Event()
                ev.record(stream)
                done.put((ev, t_arr))
            else:   # close: later frames of a new stream on this plan are ordered after these on `stream`
                pl = plan_of[sid].result()
                with free_mu:
                    free_plans[stt["cls"]].append(pl)

    def completer():
        while True:
            item = done.get()
            if item is None:
                return
            ev, t_arr = item
            ev.synchronize()
            lat.append((t_arr, time.perf_counter() - t_arr))

    def on_event_plain(ev):
        t, kind, sid, a = ev
        if kind == 0:
            plan_of[sid] = helper.submit(make_plan, streams[sid]["cls"])
        elif kind == 1:
            if plan_of[sid].done():
                work.put((kind, sid, a, time.perf_counter()))
            else:
                plain_not_admitted[0] += 1
        else:
            work.put((kind, sid, a, time.perf_counter()))

    th = [threading.Thread(target=worker), threading.Thread(target=completer)]
    for x in th:
        x.start()
    t0p = time.perf_counter()
    drive_trace(events, t0p, on_event_plain)
    work.put(None)
    for x in th:
        x.join()
    t_endp = time.perf_counter()
    helper.shutdown()
    torch.cuda.synchronize()
    for fl in free_plans.values():
        for pl in fl:
            pl.close()
    kept = np.array([l for (ta, l) in lat if ta - t0p >= warm_s]) * 1e3
    plain_by_second = {}
    for ta, l in lat:
        if ta - t0p >= warm_s:
            plain_by_second.setdefault(int(ta - t0p), []).append(1e3 * l)
    plain_fps = len(kept) / max(t_endp - (t0p + warm_s), 1e-9)

    return {
            "metric": "served form: aggregate frames/s with p50/p99 frame latency, 64 Poisson streams",
            "value": world * served_fps, "unit": "frames/s", "steps": int(st["steps"]),
            "ms_per_step": 1e3 * st["busy_seconds"] / max(st["steps"], 1),
            "dtype": "f32 math, f16 histories", "data": "synthetic (device-rendered frame pools)",
            "config": {"workload": "served form, 64 Poisson streams", "seats": SERVED_SEATS, "pipeline": args.pipeline,
                       "mix": [[w, h, p] for (w, h), p in SERVED_MIX], "rates_hz": [30, 60],
                       "mean_lifetime_frames": SERVED_LIFETIME, "budget_bytes": SERVED_BUDGET,
                       "trace_seconds": seconds, "warm_seconds": warm_s, "requests_after_warmup": n_req,
                       "streams_in_trace": len(streams), "input_pool_frames": SERVED_POOL,
                       "reserved_bytes": min(SERVED_BUDGET, int(peak_bytes * 1.25)), "peak_streams_per_class": peak_cls,
                       "tuning": {"block_ctas_per_sm": tuning.block_ctas_per_sm,
                                  "taa_tile": [tuning.taa_tile_w, tuning.taa_tile_h],
                                  "staging_depth": tuning.staging_depth}},
            "latency_ms": {"p50": st["p50_latency_ms"], "p99": st["p99_latency_ms"], "max": st["max_latency_ms"],
                           "mean": st["mean_latency_ms"]},
            "latency_p99_by_second_ms": [round(float(np.percentile(v, 99)), 3) for _, v in sorted(by_second.items())],
            "open_stream_ms": {"max": max(open_ms), "mean": float(np.mean(open_ms))} if open_ms else None,
            "frames_before_admission": not_admitted_yet[0],
            "server": {k: st[k] for k in ("requests_submitted", "requests_completed", "steps", "mean_frames_per_step",
                                          "streams_admitted", "streams_rejected", "busy_seconds", "elapsed_seconds")},
            "plain_path": {"value": plain_fps, "unit": "frames/s",
                           "latency_ms": {"p50": float(np.percentile(kept, 50)) if len(kept) else None,
                                          "p99": float(np.percentile(kept, 99)) if len(kept) else None,
                                          "max": float(kept.max()) if len(kept) else None},
                           "latency_p99_by_second_ms": [round(float(np.percentile(v, 99)), 3)
                                                        for _, v in sorted(plain_by_second.items())],
                           "open_stream_ms": {"max": max(plan_ms), "mean": float(np.mean(plan_ms))} if plan_ms else None,
                           "frames_before_admission": plain_not_admitted[0],
                           "how": "one staged plan per stream (reference arithmetic, float histories), "
                                  "requests in arrival order on one CUDA stream, plans reused across streams"},
            "saturated_server": saturated,
            "capacity": {"batched": cap_batched, "plain": cap_plain, "ratio": cap_batched / cap_plain,
                         "same_arithmetic_plans": cap_same, "ratio_vs_same_arithmetic": cap_batched / cap_same,
                         "unit": "frames/s", "streams": len(cap_streams),
                         "how": "every seat's first stream with a frame ready at every step; batched: one "
                                "step per frame of all streams (staged: each stream's plan kernels on eight "
                                "worker CUDA streams; fused: one graph-captured block-queue launch); plain: "
                                "their plans in turn"},
            # per step: 5 kernels per listed stream (staged) or noise, block kernel, (pixel pass,) TAA (fused)
            "clocks": clocks.summary(),
            "gpu_launches": (5 * int(st.get("frames", 0)) if args.pipeline == "staged"
                             else (3 + tuning.pixel_pass) * int(st["steps"])),
        }


def run_served(args, world, rank, local, dev, barrier, pg):
    """--form served: the served measurement as its own JSON line."""
    r = measure_served(args, world, rank, local, dev, barrier, args.seconds)
    if rank == 0:
        r.update({"form": "served", "n_gpus": world, "warmup": 0, "higher_is_better": True, "scaling": "weak",
                  "vs_baseline": None})
        print(json.dumps(r), flush=True)


PRECISION_W, PRECISION_H, PRECISION_FRAMES, PRECISION_SPHERES = 1920, 1080, 60, 24


def rel_err(got, want, floor):
    return (got - want).abs() / want.abs().clamp_min(floor)


def run_precision(args, world, rank, local, dev, barrier, pg):
    """Precision form at 1920x1080 over 60 frames: binary16 histories and the
    FP32 QR against the FP64 fitter (float histories), per frame.  Weights:
    the FP32-QR fitter and the FP64 fitter on the same tmp_data (relative
    error, floor 1e-3).  Pixels: the precision pipeline's output against the
    pipeline with the FP64 fitter (relative error, floor 1e-2), plus PSNR of
    both against the noise-free image."""
    import torch
    import bmfr_b200 as B
    W, H, F = PRECISION_W, PRECISION_H, max(2, min(args.frames, PRECISION_FRAMES))
    sc = B.Scene(SEED + 2, W, H, PRECISION_SPHERES)
    stream = torch.cuda.Stream(device=dev)
    px = W * H * 3
    fr = []
    for f in range(F):
        d = {k: torch.empty(px, dtype=torch.float32, device=dev)
             for k in ("albedo", "normals", "positions", "noisy", "clean")}
        sc.render_device(f, d["albedo"], d["normals"], d["positions"], d["noisy"], clean=d["clean"], stream=stream)
        fr.append(d)
    stream.synchronize()
    lim = dict(position_limit_squared=sc.position_limit_squared, normal_limit_squared=sc.normal_limit_squared)
    prec = B.Plan(W, H, fp32_qr=B.QR_CHOLESKY2, half_history=1, **lim)
    prec_hh = B.Plan(W, H, fp32_qr=B.QR_HOUSEHOLDER, half_history=1, **lim)
    plain = B.Plan(W, H, **lim)
    ref = B.Plan(W, H, **lim)          # stage calls of the FP64 pipeline
    qr = B.Plan(W, H, fp32_qr=B.QR_CHOLESKY2, **lim)
    qr_hh = B.Plan(W, H, fp32_qr=B.QR_HOUSEHOLDER, **lim)
    nb = ref.sizes.blocks
    z = lambda n, dt=torch.float32: torch.zeros(n, dtype=dt, device=dev)
    noisy_acc, acc, result = [z(px), z(px)], [z(px), z(px)], [z(px), z(px)]
    spp = [z(W * H, torch.uint8), z(W * H, torch.uint8)]
    tmp = z(ref.sizes.tmp_data_bytes, torch.uint8)
    tmp_copy = torch.empty_like(tmp)
    prev_pix, accept = z(W * H * 2), z(W * H, torch.uint8)
    w64, w32ref, w32, w32hh = z(nb * 30, torch.float64), z(nb * 30), z(nb * 30), z(nb * 30)
    mm, mm2 = z(nb * 12), z(nb * 12)
    filtered, tone = z(px), z(px)
    out_prec, out_hh = z(px), z(px)
    per_frame = []

    def psnr(x, clean):
        mse = float(((x.clamp(0, 1) - clean) ** 2).mean())
        return 10 * np.log10(1.0 / mse) if mse > 0 else float("inf")

    with torch.cuda.stream(stream):
        for f in range(F):
            d, p = fr[f], fr[max(f - 1, 0)]
            c, q = f & 1, (f & 1) ^ 1
            mat, off = sc.prev_camera(f), sc.pixel_offset(f)
            prec.denoise_frame_io(d["albedo"], d["normals"], d["positions"], d["noisy"], p["normals"],
                                  p["positions"], mat, off, result=out_prec, stream=stream)
            prec_hh.denoise_frame_io(d["albedo"], d["normals"], d["positions"], d["noisy"], p["normals"],
                                     p["positions"], mat, off, result=out_hh, stream=stream)
            noisy_acc[c].copy_(d["noisy"])
            B.accumulate_noisy_data(ref, prev_pix, accept, d["normals"], p["normals"], d["positions"],
                                    p["positions"], noisy_acc[c], noisy_acc[q], spp[q], spp[c], tmp, mat, off, f,
                                    stream=stream)
            tmp_copy.copy_(tmp)
            B.fitter_fp64(ref, w64, mm, tmp, f, stream=stream)
            w32ref.copy_(w64)
            B.fitter(qr, w32, mm2, tmp_copy, f, stream=stream)
            B.fitter(qr_hh, w32hh, mm2, tmp_copy, f, stream=stream)
            B.weighted_sum(ref, w32ref, mm, filtered, d["normals"], d["positions"], noisy_acc[c], f, stream=stream)
            B.accumulate_filtered_data(ref, filtered, prev_pix, accept, d["albedo"], tone, spp[c], acc[q], acc[c],
                                       f, stream=stream)
            B.taa(ref, prev_pix, tone, result[c], result[q], f, stream=stream)
            ew = rel_err(w32.double(), w64, 1e-3)
            ep = rel_err(out_prec.double(), result[c].double(), 1e-2)
            ewh = rel_err(w32hh.double(), w64, 1e-3)
            eph = rel_err(out_hh.double(), result[c].double(), 1e-2)
            per_frame.append({
                "frame": f, "weights_max": float(ew.max()), "weights_mean": float(ew.mean()),
                "pixels_max": float(ep.max()), "pixels_mean": float(ep.mean()),
                "pixels_over_1e-3": float((ep > 1e-3).double().mean()),
                "hh_weights_max": float(ewh.max()), "hh_weights_mean": float(ewh.mean()),
                "hh_pixels_max": float(eph.max()), "hh_pixels_mean": float(eph.mean()),
                "hh_pixels_over_1e-3": float((eph > 1e-3).double().mean()),
                "psnr_precision": psnr(out_prec, d["clean"]), "psnr_fp64": psnr(result[c], d["clean"])})
    stream.synchronize()
    if args.dump_pfm:
        # The last frame as float images for quality regression: the precision
        # form, the pipeline with the FP64 fitter, and the noise-free image.
        out_dir = Path(args.dump_pfm)
        out_dir.mkdir(parents=True, exist_ok=True)
        last = F - 1
        for name, img in (("precision", out_prec), ("fp64", result[last & 1]), ("clean", fr[last]["clean"])):
            B.write_pfm(out_dir / f"precision_1080p_frame{last}_{name}.pfm", img.cpu().numpy().reshape(H, W, 3))

    # Throughput of the precision form and of the plain drop-in at 1080p.
    def time_plan(pl, steps):
        pl.reset()
        for i in range(3):
            f, pf = frame_order(i, F), frame_order(i - 1, F) if i else 0
            pl.denoise_frame_io(fr[f]["albedo"], fr[f]["normals"], fr[f]["positions"], fr[f]["noisy"],
                                fr[pf]["normals"], fr[pf]["positions"], sc.camera(pf), sc.pixel_offset(f),
                                stream=stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(3, 3 + steps):
            f, pf = frame_order(i, F), frame_order(i - 1, F)
            pl.denoise_frame_io(fr[f]["albedo"], fr[f]["normals"], fr[f]["positions"], fr[f]["noisy"],
                                fr[pf]["normals"], fr[pf]["positions"], sc.camera(pf), sc.pixel_offset(f),
                                stream=stream)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / steps

    with ClockSampler(local) as clocks:
        ms_prec = time_plan(prec, args.steps)
    ms_hh = time_plan(prec_hh, args.steps)
    ms_plain = time_plan(plain, args.steps)
    prec.enable_profiling(True)
    time_plan(prec, 1)
    stages_prec = prec.stage_times()
    for pl in (prec, prec_hh, plain, ref, qr, qr_hh):
        pl.close()
    key = lambda k: [r[k] for r in per_frame]
    if rank == 0:
        print(json.dumps({
            "form": "precision", "metric": "1080p frames/s of the precision form with per-frame error against the FP64 fitter",
            "value": world * 1e3 / ms_prec, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": 3, "ms_per_step": ms_prec, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f16 storage, f32 QR", "data": "synthetic (device-rendered)",
            "config": {"workload": "precision form 1920x1080, 24-sphere scene", "width": W, "height": H,
                       "frames": F, "pipeline": "staged"},
            "plain_path": {"value": 1e3 / ms_plain, "ms_per_frame": ms_plain, "unit": "frames/s"},
            "householder32_path": {"value": 1e3 / ms_hh, "ms_per_frame": ms_hh, "unit": "frames/s"},
            "stages_ms": stages_prec,
            "qr": "CholeskyQR2 in FP32 (householder32_path and hh_* errors: the Householder sequence in FP32)",
            "errors": {
                "weights_rel_floor": 1e-3, "pixels_rel_floor": 1e-2,
                "weights_max": max(key("weights_max")), "weights_mean": float(np.mean(key("weights_mean"))),
                "pixels_max": max(key("pixels_max")), "pixels_mean": float(np.mean(key("pixels_mean"))),
                "pixels_over_1e-3": max(key("pixels_over_1e-3")),
                "hh_weights_max": max(key("hh_weights_max")), "hh_weights_mean": float(np.mean(key("hh_weights_mean"))),
                "hh_pixels_max": max(key("hh_pixels_max")), "hh_pixels_mean": float(np.mean(key("hh_pixels_mean"))),
                "hh_pixels_over_1e-3": max(key("hh_pixels_over_1e-3")),
                "psnr_precision_mean": float(np.mean(key("psnr_precision"))),
                "psnr_fp64_mean": float(np.mean(key("psnr_fp64")))},
            "per_frame": per_frame,
            "clocks": clocks.summary(), "gpu_launches": 6 * args.steps,
        }), flush=True)


def dropin_stage_ms(B, torch, dev, stream, params, frames, mats, off, nframes):
    """Each of the five drop-in stage entry points (the reference's kernels,
    opencl/bmfr.cl) timed alone with events around its call, on the same
    frames, buffers allocated by the caller as in opencl/bmfr.cpp:315-347."""
    plan = B.Plan(WIDTH, HEIGHT, params=params)
    px = WIDTH * HEIGHT
    z = lambda n, dt=torch.float32: torch.zeros(n, dtype=dt, device=dev)
    noisy, acc, res = [z(px * 3), z(px * 3)], [z(px * 3), z(px * 3)], [z(px * 3), z(px * 3)]
    spp = [z(px, torch.uint8), z(px, torch.uint8)]
    prev_pix, accept = z(px * 2), z(px, torch.uint8)
    tmp = z(plan.sizes.tmp_data_bytes, torch.uint8)
    nb = plan.sizes.blocks
    w, mm, filt, tone = z(nb * 30), z(nb * 12), z(px * 3), z(px * 3)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
    names = ("accumulate_noisy_data", "fitter", "weighted_sum", "accumulate_filtered_data", "taa")
    out = {k: [] for k in names}
    nfr = frames["albedo"].shape[0]
    with torch.cuda.stream(stream):
        for i in range(nframes + 3):
            f = frame_order(i, nfr)
            pf = frame_order(i - 1, nfr) if i > 0 else f
            c, q = i & 1, (i & 1) ^ 1
            noisy[c].copy_(frames["noisy"][f].reshape(-1))
            ev[0].record(stream)
            B.accumulate_noisy_data(plan, prev_pix, accept, frames["normals"][f], frames["normals"][pf],
                                    frames["positions"][f], frames["positions"][pf], noisy[c], noisy[q], spp[q],
                                    spp[c], tmp, mats[pf], off, i, stream=stream)
            ev[1].record(stream)
            B.fitter(plan, w, mm, tmp, i, stream=stream)
            ev[2].record(stream)
            B.weighted_sum(plan, w, mm, filt, frames["normals"][f], frames["positions"][f], noisy[c], i,
                           stream=stream)
            ev[3].record(stream)
            B.accumulate_filtered_data(plan, filt, prev_pix, accept, frames["albedo"][f], tone, spp[c], acc[q],
                                       acc[c], i, stream=stream)
            ev[4].record(stream)
            B.taa(plan, prev_pix, tone, res[c], res[q], i, stream=stream)
            ev[5].record(stream)
            ev[5].synchronize()
            if i >= 3:
                for k, n in enumerate(names):
                    out[n].append(ev[k].elapsed_time(ev[k + 1]))
    plan.close()
    return {k: float(np.mean(v)) for k, v in out.items()}


def run_probe(args, dev):
    """A few 1280x720 frames of the plan pipeline and nothing else: the
    workload that profiler captures of single kernels run on (frames
    rendered on the device; --qr selects the fitter arithmetic, precision
    methods with binary16 histories)."""
    import torch
    import bmfr_b200 as B
    sc = B.Scene(1, WIDTH, HEIGHT, SPHERES)
    px = WIDTH * HEIGHT * 3
    fr = []
    for f in range(max(1, args.frames)):
        d = {k: torch.empty(px, dtype=torch.float32, device=dev) for k in ("albedo", "normals", "positions", "noisy")}
        sc.render_device(f, d["albedo"], d["normals"], d["positions"], d["noisy"])
        fr.append(d)
    plan = B.Plan(WIDTH, HEIGHT, fp32_qr=args.qr, half_history=1 if args.qr else 0,
                  pipeline=B.PIPELINE_FUSED if args.pipeline == "fused" else B.PIPELINE_STAGED,
                  position_limit_squared=sc.position_limit_squared, normal_limit_squared=sc.normal_limit_squared)
    for f in range(len(fr)):
        d, p = fr[f], fr[max(f - 1, 0)]
        plan.denoise_frame_io(d["albedo"], d["normals"], d["positions"], d["noisy"], p["normals"], p["positions"],
                              sc.prev_camera(f), sc.pixel_offset(f))
    torch.cuda.synchronize()
    plan.close()
    print(json.dumps({"form": "probe", "frames": len(fr), "qr": args.qr, "pipeline": args.pipeline}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=240)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--pipeline", default="staged", choices=["fused", "staged"])
    ap.add_argument("--frame-loop", default="sequence", choices=["sequence", "single"],
                    help="plain form: the K frames of a timed loop through one bmfr_denoise_frames call "
                         "(sequence) or one bmfr_denoise_frame_io call each (single)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--frames", type=int, default=FRAMES, help="distinct scene frames held in HBM")
    ap.add_argument("--form", default="plain", choices=["plain", "batched", "served", "precision", "probe"])
    ap.add_argument("--qr", type=int, default=0, help="probe form: fp32_qr of the plan (0, 1 or 2)")
    ap.add_argument("--seconds", type=float, default=10.0, help="served form: length of the arrival trace")
    ap.add_argument("--dump-pfm", default="", help="precision form: write the last frame's images (PFM) here")
    ap.add_argument("--no-multistream", action="store_true",
                    help="plain form: leave out the batched and served objects of the line")
    ap.add_argument("--served-seconds", type=float, default=4.0,
                    help="plain form: length of the served object's arrival trace")
    args = ap.parse_args()
    args.warmup_requested = args.warmup
    args.warmup = max(args.warmup, 3)   # at least three untimed steps
    if args.gpus < 1:
        ap.error("--gpus must be at least 1")
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # One process per GPU: start N ranks of this same command.
        sys.exit(subprocess.call(launch_command(args.gpus, sys.argv[1:])))
    world, rank, local = dist_setup()
    check_world(world, args.gpus)

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

    if args.form == "probe":
        run_probe(args, dev)
        return
    if args.form != "plain":
        run = {"batched": run_batched, "served": run_served, "precision": run_precision}[args.form]
        run(args, world, rank, local, dev, barrier, pg)
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

    # Frames i0 .. i0+n-1 as one bmfr_denoise_frames call (raw device
    # addresses, so that building the call costs the host little).
    addr = {k: [devf[k][f].data_ptr() for f in range(nfr)] for k in devf}

    def steps_as_sequence(i0, n):
        ios, ms = [], []
        for i in range(i0, i0 + n):
            f = frame_order(i, nfr)
            pf = frame_order(i - 1, nfr) if i > 0 else f
            ios.append({"albedo": addr["albedo"][f], "normals": addr["normals"][f],
                        "positions": addr["positions"][f], "noisy": addr["noisy"][f],
                        "previous_normals": addr["normals"][pf], "previous_positions": addr["positions"][pf]})
            ms.append(mats[pf])
        plan.denoise_frames(ios, ms, [off] * n, stream=stream)

    def steps_one_by_one(i0, n):
        for i in range(i0, i0 + n):
            step_resident(i)

    run_steps = {"sequence": steps_as_sequence, "single": steps_one_by_one}

    # ---- value: device-resident inputs ---------------------------------------
    # Warm-up through both loops (the first overlapped call allocates the
    # plan's second set of per-frame buffers).
    with torch.cuda.stream(stream):
        steps_one_by_one(0, args.warmup)
        steps_as_sequence(args.warmup, args.warmup)
    stream.synchronize()
    barrier()
    torch.cuda.synchronize()
    # The K-step loop repeats until at least MIN_TIMED_SECONDS have passed;
    # the loop's median time, the slowest rank's, gives the step time.
    base0 = 2 * args.warmup
    base_next = [base0]

    def k_steps_of(kind):
        def k_steps(loop):
            run_steps[kind](base_next[0], args.steps)
            base_next[0] += args.steps
        return k_steps

    with ClockSampler(local) as clocks:
        loop_ms = timed_loops(k_steps_of(args.frame_loop), stream, dev)
    torch.cuda.synchronize()
    barrier()
    elapsed_ms = max_over_ranks(statistics.median(loop_ms), device=dev)   # the slowest rank
    value = world * args.steps / (elapsed_ms / 1e3)
    # The other frame loop on the same plan and frames, beside the line's.
    other_loop = "single" if args.frame_loop == "sequence" else "sequence"
    other_loop_ms = max_over_ranks(statistics.median(timed_loops(k_steps_of(other_loop), stream, dev,
                                                                 min_seconds=0.2)), device=dev)
    torch.cuda.synchronize()
    frame_loop_line = {
        "frame_loop": other_loop, "value": world * args.steps / (other_loop_ms / 1e3), "unit": "frames/s",
        "ms_per_step": other_loop_ms / args.steps,
        "how": "sequence: the K frames of a loop in one bmfr_denoise_frames call, each frame's accumulation "
               "overlapping the previous frame's fitter, weighted sum and TAA (same outputs bit for bit); "
               "single: one bmfr_denoise_frame_io call per frame, stages in stream order"}
    # noise table, block kernel, weighted sum + filtered accumulation, taa
    # (fused); noise table, accumulate, fitter, weighted sum + filtered
    # accumulation, taa (staged)
    launches_per_frame = 4 if pipeline == B.PIPELINE_FUSED else 5

    # ---- per-stage profile (same workload, events between stages) ------------
    plan.enable_profiling(True)
    stage_ms = {}
    base = base_next[0]
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
    hbm = {"achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
           "peak_source": peak_kind, "bytes_per_launch": sb[dominant], "traffic": NCU_TRAFFIC_720P.get(dominant)}
    clk = clocks.summary()
    sm_mhz = clk.get("sm_mhz") or 1965.0
    issue_peak = SMS * SCHEDULERS_PER_SM * sm_mhz * 1e6 / 1e9          # G warp-instructions/s
    issue = None
    if dominant in NCU_WARP_INST_720P:
        got = NCU_WARP_INST_720P[dominant] / (stages[dominant] * 1e-3) / 1e9
        issue = {"achieved": got, "peak": issue_peak, "unit": "G warp-instructions/s",
                 "frac": got / issue_peak, "instructions_per_launch": NCU_WARP_INST_720P[dominant],
                 "peak_source": f"{SMS} SMs x {SCHEDULERS_PER_SM} schedulers x 1 instruction/cycle at "
                                f"the sampled SM clock ({sm_mhz:.0f} MHz)"}
    if dominant in ISSUE_BOUND and issue is not None:
        # An issue-bound kernel: the issue rate leads, the HBM figures ride along.
        roofline = {"kernel": dominant, "bound": "issue", **{k: issue[k] for k in ("achieved", "peak", "unit", "frac")},
                    "peak_source": issue["peak_source"], "instructions_per_launch": issue["instructions_per_launch"],
                    "traffic": NCU_TRAFFIC_720P.get(dominant), "hbm": hbm,
                    "note": ISSUE_BOUND[dominant]}
    else:
        roofline = {"kernel": dominant, "bound": "hbm", **{k: hbm[k] for k in hbm}}
        if issue is not None:
            roofline["issue"] = issue
    stage_gbs = {k: sb[k] / (v * 1e-3) / 1e9 for k, v in stages.items() if v > 0}
    dropin = dropin_stage_ms(B, torch, dev, stream, plan.params, devf, mats, off, min(args.steps, 30))

    # ---- the other plan pipeline on the same frames, beside the bench's ----
    other = B.PIPELINE_STAGED if pipeline == B.PIPELINE_FUSED else B.PIPELINE_FUSED
    oplan = B.Plan(WIDTH, HEIGHT, pipeline=other, position_limit_squared=sc.position_limit_squared,
                   normal_limit_squared=sc.normal_limit_squared)

    def other_steps(loop):
        for i in range(args.steps):
            k = loop * args.steps + i
            f = frame_order(k, nfr)
            pf = frame_order(k - 1, nfr) if k > 0 else f
            oplan.denoise_frame_io(devf["albedo"][f], devf["normals"][f], devf["positions"][f], devf["noisy"][f],
                                   devf["normals"][pf], devf["positions"][pf], mats[pf], off, stream=stream)

    other_steps(0)
    stream.synchronize()
    other_ms = max_over_ranks(statistics.median(timed_loops(other_steps, stream, dev, min_seconds=0.2)), device=dev)
    oplan.close()
    other_line = {"pipeline": "fused" if other == B.PIPELINE_FUSED else "staged",
                  "value": world * args.steps / (other_ms / 1e3), "unit": "frames/s",
                  "ms_per_step": other_ms / args.steps,
                  "how": "fused: accumulate + fit in one kernel per 32x32 block (tmp_data stays on chip), then "
                         "weighted sum + filtered accumulation, then TAA; staged: the four-kernel plan pipeline"}

    # ---- e2e: host buffers through the C ABI --------------------------------
    # Uploads, frames and downloads on three streams: the plan orders them,
    # so frame i+1's upload and frame i-1's download overlap frame i.
    plan.reset()
    out_host = torch.empty((HEIGHT, WIDTH, 3), dtype=torch.float32).pin_memory()
    up_stream, down_stream = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)

    def step_e2e(i):
        f = frame_order(i, nfr)
        pf = frame_order(i - 1, nfr) if i > 0 else f
        plan.upload_frame(host["albedo"][f], host["normals"][f], host["positions"][f], host["noisy"][f],
                          stream=up_stream)
        plan.denoise_frame(mats[pf], off, stream=stream)
        plan.download_result(out_host, stream=down_stream)

    for i in range(args.warmup):
        step_e2e(i)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_steps = min(max(args.steps, 100), 300)   # ~0.1-0.3 s of PCIe-bound frames
    e0.record(up_stream)
    for i in range(args.warmup, args.warmup + e2e_steps):
        step_e2e(i)
    e1.record(down_stream)
    e1.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    e2e_ms = max_over_ranks(e2e_ms, device=dev)   # the slowest rank
    e2e = {"value": world * e2e_steps / (e2e_ms / 1e3), "unit": "frames/s",
           "h2d_bytes_per_step": 4 * WIDTH * HEIGHT * 12, "d2h_bytes_per_step": WIDTH * HEIGHT * 12}

    plan.close()
    del devf
    torch.cuda.synchronize()

    # ---- the multi-stream half of the metric: batched and served forms -------
    multi = {}
    if not args.no_multistream:
        mst = max(args.steps, 10)
        multi["batched"] = measure_batched(args, world, rank, local, dev, barrier, mst, args.warmup)
        torch.cuda.synchronize()
        multi["served"] = measure_served(args, world, rank, local, dev, barrier, args.served_seconds)
        torch.cuda.synchronize()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(frames, sc, ref_budget_s=15.0, port_budget_s=10.0)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "BMFR plain pipeline 1280x720, 12-sphere procedural scene, 60 frames replayed",
                       "width": WIDTH, "height": HEIGHT, "frames": nfr, "pipeline": args.pipeline,
                       "frame_loop": args.frame_loop,
                       "tmp_data": "binary16", "parallelism": f"replicas x{world}",
                       "l2": "no flush: per-frame working set ~180 MB (inputs + histories) exceeds the 126 MB L2"},
            "stages_ms": stages, "stages_gbs": stage_gbs, "other_pipeline": other_line,
            "other_frame_loop": frame_loop_line,
            "dropin_stages_ms": dropin,
            "dropin_stages_gbs": {k: sb[k] / (v * 1e-3) / 1e9 for k, v in dropin.items() if v > 0},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "clocks": clk, "timed_loops": len(loop_ms), "launches_per_step": launches_per_frame,
            "gpu_launches": launches_per_frame * args.steps * len(loop_ms),
        }
        if multi:
            line.update(multi)
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
