"""Streams across GPUs: one process per GPU, whole streams placed on ranks.

BMFR's per-frame path does not shard within a frame (accumulation and TAA
gather from arbitrary reprojected positions of the previous frame), so more
GPUs denoise more streams: each rank owns whole streams and their histories
in its HBM, and no collective runs on the data path.  This module holds the
host-side pieces: the placement of streams on ranks (largest first onto the
least-loaded rank, within each rank's memory budget) and the reductions
used to report a multi-GPU run (the slowest rank's time, totals).
"""
from __future__ import annotations


def place_streams(sizes, world: int, stream_bytes=None, budget_bytes: int = 0):
    """Assigns streams of the given (width, height) sizes to `world` ranks.

    Largest stream first onto the rank with the fewest pixels so far; with a
    budget, a rank whose streams would exceed it is skipped (a stream that
    fits nowhere raises).  stream_bytes(w, h) gives a stream's memory.
    Every rank computes the same answer.  Returns one list of stream indices
    per rank."""
    if world < 1:
        raise ValueError("world must be at least 1")
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i][0] * sizes[i][1], i))
    pixels = [0] * world
    used = [0] * world
    out = [[] for _ in range(world)]
    for i in order:
        w, h = sizes[i]
        need = stream_bytes(w, h) if stream_bytes else 0
        ranks = sorted(range(world), key=lambda r: (pixels[r], r))
        for r in ranks:
            if budget_bytes and used[r] + need > budget_bytes:
                continue
            out[r].append(i)
            pixels[r] += w * h
            used[r] += need
            break
        else:
            raise MemoryError(f"stream {i} ({w}x{h}) fits in no rank's budget")
    return [sorted(x) for x in out]


def max_over_ranks(value: float, device=None) -> float:
    """The largest value over the ranks of the default process group (the
    time of the slowest rank); the value itself without a group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    """Sum over the ranks of the default process group (totals of a run)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
