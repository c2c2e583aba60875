"""The host-side router over per-GPU servers (bmfr_b200/router.py) and the
benchmark's multi-GPU launch, on CPU: placement by memory budget with fake
servers, migration, the static assignment two gloo ranks agree on, and the
launch command / rank-count check of bench.py."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

from bmfr_b200.router import BMFR_E_BUDGET, BMFR_E_NOT_FOUND, Router, RouterError

ROOT = Path(__file__).resolve().parent.parent


class FakeServer:
    """The Server interface on host memory: a stream's 'history' is its frame
    counter, so a migration that loses or repeats a frame shows."""

    def __init__(self):
        self.streams, self.next, self.requests = {}, 0, []

    def open_stream(self, w, h):
        sid = self.next
        self.next += 1
        self.streams[sid] = {"w": w, "h": h, "frame": 0}
        return sid

    def close_stream(self, sid):
        del self.streams[sid]

    def submit(self, sid, matrix, offset, io=None):
        self.streams[sid]["frame"] += 1
        self.requests.append((sid, self.streams[sid]["frame"]))
        return len(self.requests) - 1

    def poll(self, rid):
        return True, 0.1

    def drain(self, timeout_ms=60000.0):
        pass

    def snapshot_bytes(self, sid):
        return 16

    def snapshot_stream(self, sid, out, stream=None):
        s = self.streams[sid]
        out[:] = 0
        out[0], out[1], out[2] = s["w"] % 256, s["h"] % 256, s["frame"]
        self.snap_meta = (s["w"], s["h"])
        return out

    def restore_stream(self, snap, stream=None):
        sid = self.next
        self.next += 1
        self.streams[sid] = {"w": None, "h": None, "frame": int(snap[2])}
        return sid


def nbytes(w, h):
    return w * h * 100


def test_new_streams_go_to_the_least_loaded_gpu_with_room():
    servers = [FakeServer() for _ in range(3)]
    r = Router(servers, budget_bytes=1_100_000_000, stream_bytes=nbytes)
    ids = [r.open_stream(1920, 1080) for _ in range(3)]
    assert sorted(r.gpu_of(i) for i in ids) == [0, 1, 2]      # one per GPU
    small = r.open_stream(640, 360)
    assert r.gpu_of(small) == 0                                # ties go to the lowest index
    big = r.open_stream(3840, 2160)                            # 829 MB: GPU 1 or 2 (fewest pixels)
    assert r.gpu_of(big) == 1
    load = r.load()
    assert load[1][2] == nbytes(1920, 1080) + nbytes(3840, 2160)
    assert all(b <= 1_100_000_000 for _, _, b in load)
    assert [r.gpu_of(r.open_stream(3840, 2160)) for _ in range(2)] == [2, 0]
    with pytest.raises(RouterError):                           # every GPU now holds a 4K stream
        r.open_stream(3840, 2160)


def test_a_stream_that_fits_nowhere_is_refused_and_closing_frees_room():
    servers = [FakeServer() for _ in range(2)]
    r = Router(servers, budget_bytes=900_000_000, stream_bytes=nbytes)
    a = r.open_stream(3840, 2160)
    b = r.open_stream(3840, 2160)
    with pytest.raises(RouterError) as e:
        r.open_stream(3840, 2160)
    assert e.value.status == BMFR_E_BUDGET
    r.close_stream(a)
    c = r.open_stream(3840, 2160)
    assert r.gpu_of(c) != r.gpu_of(b)
    with pytest.raises(RouterError) as e:
        r.submit(a, None, None)
    assert e.value.status == BMFR_E_NOT_FOUND


def test_requests_follow_the_stream_and_migration_keeps_its_history():
    servers = [FakeServer() for _ in range(2)]
    r = Router(servers, budget_bytes=0, stream_bytes=nbytes)
    s = r.open_stream(1280, 720)
    for _ in range(3):
        gpu, req = r.submit(s, None, None)
        assert gpu == r.gpu_of(s) and r.poll((gpu, req))[0]
    src = r.gpu_of(s)
    dst = r.migrate(s)
    assert dst != src and r.gpu_of(s) == dst
    assert servers[src].streams == {}                          # closed at the source
    gpu, _ = r.submit(s, None, None)
    assert gpu == dst
    # frames 1..3 on the source, frame 4 continues on the target
    assert servers[dst].requests[-1][1] == 4
    assert r.load()[src] == (0, 0, 0) and r.load()[dst][0] == 1
    r.close()
    assert r.load() == [(0, 0, 0), (0, 0, 0)]


def test_migration_respects_the_target_budget():
    servers = [FakeServer() for _ in range(2)]
    r = Router(servers, budget_bytes=900_000_000, stream_bytes=nbytes)
    a = r.open_stream(3840, 2160)
    r.open_stream(3840, 2160)
    with pytest.raises(RouterError):
        r.migrate(a, to=1 - r.gpu_of(a))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


SIZES = [(640, 360)] * 8 + [(1280, 720)] * 8 + [(1920, 1080)] * 6 + [(3840, 2160)] * 2


def _rank_main(rank, world, port, results):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        parts = Router.assign(SIZES, world, stream_bytes=nbytes, budget_bytes=2_000_000_000)
        mine = parts[rank]
        # Each rank serves its own list through a router over its one server.
        r = Router([FakeServer()], budget_bytes=2_000_000_000, stream_bytes=nbytes)
        for i in mine:
            r.open_stream(*SIZES[i])
        owned = torch.zeros(len(SIZES), dtype=torch.int64)
        owned[mine] = 1
        dist.all_reduce(owned)
        results[rank] = (parts, owned.tolist(), r.load()[0][2])
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_split_the_streams_exactly_once():
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
    assert got[0][0] == got[1][0]                  # the same placement on every rank
    assert got[0][1] == [1] * len(SIZES)            # every stream served by exactly one rank
    for rank in range(world):
        assert got[rank][2] <= 2_000_000_000


def _bench():
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_bench_launches_one_rank_per_gpu_and_checks_the_count():
    b = _bench()
    cmd = b.launch_command(4, ["--gpus", "4", "--steps", "20"], port=29555)
    assert cmd[:3] == [sys.executable, "-m", "torch.distributed.run"]
    assert "--nproc-per-node=4" in cmd and "--nnodes=1" in cmd
    assert cmd[cmd.index("--master-addr") + 1] == "127.0.0.1"
    assert cmd[cmd.index("--master-port") + 1] == "29555"
    assert cmd[-4:] == ["--gpus", "4", "--steps", "20"] and cmd[-5].endswith("bench.py")
    b.check_world(2, 2)
    with pytest.raises(SystemExit):
        b.check_world(1, 2)


def test_bench_reference_arm_as_two_ranks():
    """`bench.py --impl reference --gpus 2` starts two ranks itself; rank 0
    alone runs the CPU reference and prints one line, the other exits 0.
    torchrun sets OMP_NUM_THREADS=1 in every rank, so the arm passes its
    thread count to the CPU kernels itself: all the host's threads."""
    import json
    import subprocess
    env = dict(os.environ)
    env.pop("WORLD_SIZE", None)
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
                        "--warmup", "1"], capture_output=True, text=True, timeout=600, env=env, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["cores"] == len(os.sched_getaffinity(0))
