"""Multi-GPU host logic (bmfr_b200/replicas.py) on CPU: stream placement
and the cross-rank reductions, the latter with two gloo ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from bmfr_b200.replicas import max_over_ranks, place_streams, sum_over_ranks

SIZES = [(640, 360)] * 8 + [(1280, 720)] * 8 + [(1920, 1080)] * 6 + [(3840, 2160)] * 2


def test_place_streams_balances_pixels():
    for world in (1, 2, 4, 8):
        parts = place_streams(SIZES, world)
        assert sorted(i for p in parts for i in p) == list(range(len(SIZES)))
        load = [sum(SIZES[i][0] * SIZES[i][1] for i in p) for p in parts]
        biggest = max(w * h for w, h in SIZES)
        assert max(load) - min(load) <= biggest   # greedy, largest first


def test_place_streams_respects_budget():
    nbytes = lambda w, h: w * h * 100
    parts = place_streams(SIZES, 4, stream_bytes=nbytes, budget_bytes=1_400_000_000)
    for p in parts:
        assert sum(nbytes(*SIZES[i]) for i in p) <= 1_400_000_000
    with pytest.raises(MemoryError):
        place_streams(SIZES, 2, stream_bytes=nbytes, budget_bytes=500_000_000)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, results):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        slowest = max_over_ranks(1.5 + rank)
        total = sum_over_ranks(10.0 * (rank + 1))
        parts = place_streams(SIZES, world)
        results[rank] = (slowest, total, parts)
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_agree():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        results = mgr.dict()
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, results)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        got = dict(results)
    assert got[0][0] == got[1][0] == 2.5
    assert got[0][1] == got[1][1] == 30.0
    assert got[0][2] == got[1][2]   # every rank places the streams the same way


def test_reductions_without_a_group():
    assert max_over_ranks(3.0) == 3.0
    assert sum_over_ranks(3.0) == 3.0
