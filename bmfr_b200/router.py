"""Host-side router over per-GPU request servers.

BMFR's per-frame path does not shard within a frame, so more GPUs serve more
streams: each GPU runs its own request server (bmfr_server_*, continuous
batching of that GPU's streams, histories resident in its HBM) and a router
on the host decides which GPU a new stream joins.  The policy is the online
form of replicas.place_streams: a stream goes to the GPU with the fewest
open pixels among those whose memory budget still holds the stream's bytes;
a stream that fits nowhere is refused (BMFR_E_BUDGET, as one server refuses
it).  A stream can move between GPUs between frames (snapshot of its
histories on one server, restore on another), which is how a host rebalances
or drains a GPU.

The router holds no device memory and launches nothing itself.  In one
process it drives one Server per device (`Router.for_devices`); with one
process per GPU, every rank computes the same static placement
(`Router.assign`) and serves only its own streams.
"""
from __future__ import annotations

from dataclasses import dataclass

from .replicas import place_streams

BMFR_E_BUDGET = -5
BMFR_E_NOT_FOUND = -6


class RouterError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(msg)
        self.status = status


@dataclass
class _Route:
    gpu: int
    sid: int          # the stream's id on that GPU's server
    width: int
    height: int
    nbytes: int


class Router:
    """Streams across servers, one per GPU.

    servers: objects with the Server interface (open_stream, close_stream,
    submit, poll, drain, snapshot_stream, restore_stream);
    budget_bytes: per-GPU budget for stream histories (0: unlimited);
    stream_bytes(w, h): a stream's device memory (Batch.stream_bytes for the
    servers' parameters)."""

    def __init__(self, servers, budget_bytes: int = 0, stream_bytes=None):
        if not servers:
            raise ValueError("a router needs at least one server")
        self.servers = list(servers)
        self.budget = int(budget_bytes)
        self.stream_bytes = stream_bytes or (lambda w, h: 0)
        self.used = [0] * len(self.servers)
        self.pixels = [0] * len(self.servers)
        self.routes: dict[int, _Route] = {}
        self._next = 0

    @classmethod
    def for_devices(cls, devices, params=None, budget_bytes: int = 0, **server_kw):
        """One Server per CUDA device index, created with that device current."""
        import torch

        from . import Batch, Server, default_params
        params = params if params is not None else default_params()
        servers = []
        for d in devices:
            with torch.cuda.device(d):
                servers.append(Server(params, memory_budget_bytes=budget_bytes, **server_kw))
        return cls(servers, budget_bytes, lambda w, h: Batch.stream_bytes(params, w, h))

    @staticmethod
    def assign(sizes, gpus: int, stream_bytes=None, budget_bytes: int = 0):
        """Static placement of known streams for one process per GPU: every
        rank computes the same answer and opens only its own list."""
        return place_streams(sizes, gpus, stream_bytes=stream_bytes, budget_bytes=budget_bytes)

    def _pick(self, nbytes: int, exclude=None) -> int:
        order = sorted(range(len(self.servers)), key=lambda g: (self.pixels[g], g))
        for g in order:
            if g == exclude:
                continue
            if self.budget and self.used[g] + nbytes > self.budget:
                continue
            return g
        raise RouterError(BMFR_E_BUDGET, f"no GPU has {nbytes} bytes left in its budget")

    def _take(self, g: int, w: int, h: int, nbytes: int):
        self.used[g] += nbytes
        self.pixels[g] += w * h

    def _give(self, r: _Route):
        self.used[r.gpu] -= r.nbytes
        self.pixels[r.gpu] -= r.width * r.height

    def open_stream(self, width: int, height: int) -> int:
        """Admits a stream on the least-loaded GPU with room; returns the
        router's id for it."""
        nbytes = int(self.stream_bytes(width, height))
        g = self._pick(nbytes)
        sid = self.servers[g].open_stream(width, height)
        self._take(g, width, height, nbytes)
        rid = self._next
        self._next += 1
        self.routes[rid] = _Route(g, sid, width, height, nbytes)
        return rid

    def _route(self, rid: int) -> _Route:
        r = self.routes.get(rid)
        if r is None:
            raise RouterError(BMFR_E_NOT_FOUND, f"unknown stream {rid}")
        return r

    def gpu_of(self, rid: int) -> int:
        return self._route(rid).gpu

    def close_stream(self, rid: int) -> None:
        r = self._route(rid)
        self.servers[r.gpu].close_stream(r.sid)
        self._give(r)
        del self.routes[rid]

    def submit(self, rid: int, matrix, offset, io=None):
        """Forwards a frame request to the stream's GPU; returns (gpu, request id)."""
        r = self._route(rid)
        return r.gpu, self.servers[r.gpu].submit(r.sid, matrix, offset, io=io)

    def poll(self, ticket):
        gpu, req = ticket
        return self.servers[gpu].poll(req)

    def drain(self, timeout_ms: float = 60000.0) -> None:
        for s in self.servers:
            s.drain(timeout_ms)

    def migrate(self, rid: int, to: int | None = None, staging=None) -> int:
        """Moves a stream to GPU `to` (default: the least-loaded other GPU with
        room) between frames: drains its server, snapshots its histories into
        `staging` (host memory when None), restores them on the target and
        closes it at the source.  Its next frame continues exactly as it
        would have.  Returns the GPU it now lives on."""
        r = self._route(rid)
        if to is None:
            to = self._pick(r.nbytes, exclude=r.gpu)
        if to == r.gpu:
            return to
        if self.budget and self.used[to] + r.nbytes > self.budget:
            raise RouterError(BMFR_E_BUDGET, f"GPU {to} has no room for stream {rid}")
        src = self.servers[r.gpu]
        src.drain()
        snap = src.snapshot_stream(r.sid, staging if staging is not None else self._host_buffer(src, r))
        new_sid = self.servers[to].restore_stream(snap)
        src.close_stream(r.sid)
        self._give(r)
        self._take(to, r.width, r.height, r.nbytes)
        self.routes[rid] = _Route(to, new_sid, r.width, r.height, r.nbytes)
        return to

    @staticmethod
    def _host_buffer(server, r: _Route):
        nbytes = server.snapshot_bytes(r.sid)
        import numpy as np
        return np.empty(nbytes, dtype=np.uint8)

    def load(self):
        """Per GPU: (open streams, pixels, bytes)."""
        count = [0] * len(self.servers)
        for r in self.routes.values():
            count[r.gpu] += 1
        return [(count[g], self.pixels[g], self.used[g]) for g in range(len(self.servers))]

    def close(self) -> None:
        for rid in list(self.routes):
            self.close_stream(rid)
