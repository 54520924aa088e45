"""Continuous-batching serving loop for DIM solve requests.

Requests (a grid, its initial state and a step budget) arrive over time.  The
server admits them first-come-first-served as long as their device
footprint fits the HBM budget and a slot is free, keeps every admitted
solve's state resident on the GPU, and advances all admitted solves together
in quanta of a few steps through the batched form (one ``Batch`` per material
count and dimension).  A request that arrives while others run joins at the
next quantum; a finished request is downloaded and its memory returned at
once, which is what lets the queue drain into the freed room.

Every solve's arithmetic is the single-grid step's, so a result does not
depend on what else was in flight (tests/test_gpu_serving.py).
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from .abi import PRECISION_MIXED, Desc
from .batch import Batch

# Device doubles per cell: two state copies plus the staged-sweep scratch
# (csrc/dimgpu_api.cu staged_scratch_doubles).
def _staged_doubles(nmat: int, dim: int) -> int:
    pv, v, fv = 2 * nmat + dim + 1, 2 * nmat + dim, 2 * nmat + dim + 2
    return 5 * pv + nmat + 2 * v + fv


def footprint_bytes(desc: Desc, steps: int) -> int:
    """Device bytes a solve holds while admitted."""
    per_cell = 2 * desc.nvar + _staged_doubles(desc.nmat, desc.dim)
    return 8 * (per_cell * desc.ncell + max(steps, 1))


@dataclass
class Request:
    rid: int
    desc: Desc
    U: np.ndarray
    steps: int
    cfl: float = 0.6
    dt_max: float = 1e300
    arrival: float = 0.0          # seconds after the start of the run


@dataclass
class Result:
    rid: int
    U: np.ndarray
    dts: np.ndarray
    arrival: float
    admitted: float
    finished: float

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


@dataclass
class ServerStats:
    results: list = field(default_factory=list)
    elapsed: float = 0.0
    peak_bytes: int = 0
    peak_slots: int = 0
    quanta: int = 0

    def latency_percentiles(self):
        lat = np.array([r.latency for r in self.results])
        return float(np.percentile(lat, 50)), float(np.percentile(lat, 99))

    @property
    def solves_per_s(self) -> float:
        return len(self.results) / self.elapsed if self.elapsed > 0 else 0.0


class Server:
    """Admission, resident state and batched stepping of DIM solves."""

    def __init__(self, hbm_budget_bytes: float = 150e9, max_slots: int = 128, quantum: int = 8,
                 stream_handle: int | None = None):
        self.budget = float(hbm_budget_bytes)
        self.max_slots = max_slots
        self.quantum = quantum
        self.stream = stream_handle
        self.batches: dict[tuple[int, int], Batch] = {}
        self.pending: deque[Request] = deque()
        self.active: dict[int, tuple[Request, int, float]] = {}  # rid -> (request, instance id, admitted)
        self.used = 0
        self.cancelled: set[int] = set()

    def close(self):
        for b in self.batches.values():
            b.close()
        self.batches.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _batch(self, desc: Desc) -> Batch:
        key = (desc.nmat, desc.dim)
        if key not in self.batches:
            b = Batch(*key)
            if self.stream:
                b.set_stream(self.stream)
            self.batches[key] = b
        return self.batches[key]

    def submit(self, req: Request) -> None:
        if footprint_bytes(req.desc, req.steps) > self.budget:
            raise ValueError(f"request {req.rid} needs more device memory than the whole budget")
        self.pending.append(req)

    def cancel(self, rid: int) -> bool:
        """Drop a queued or running request; True if it was found."""
        for r in list(self.pending):
            if r.rid == rid:
                self.pending.remove(r)
                return True
        if rid in self.active:
            req, iid, _ = self.active.pop(rid)
            self._batch(req.desc).remove(iid)
            self.used -= footprint_bytes(req.desc, req.steps)
            self.cancelled.add(rid)
            return True
        return False

    def _admit(self, now: float) -> None:
        while self.pending and len(self.active) < self.max_slots:
            req = self.pending[0]
            need = footprint_bytes(req.desc, req.steps)
            if self.used + need > self.budget:
                break
            self.pending.popleft()
            iid = self._batch(req.desc).add(req.desc, req.U, req.steps, req.cfl, req.dt_max)
            self.active[req.rid] = (req, iid, now)
            self.used += need

    def _retire(self, now_fn) -> list[Result]:
        out = []
        for rid in list(self.active):
            req, iid, admitted = self.active[rid]
            b = self._batch(req.desc)
            done, left = b.status(iid)
            if left > 0:
                continue
            U, dts = b.download(iid)
            b.remove(iid)
            self.used -= footprint_bytes(req.desc, req.steps)
            del self.active[rid]
            out.append(Result(rid, U, dts, req.arrival, admitted, now_fn()))
        return out

    def serve(self, requests: list[Request], clock=time.perf_counter) -> ServerStats:
        """Run the event loop until every request has finished.  Arrivals
        follow each request's `arrival` offset in wall-clock time."""
        stats = ServerStats()
        reqs = sorted(requests, key=lambda r: r.arrival)
        t0 = clock()
        now_fn = lambda: clock() - t0  # noqa: E731
        i = 0
        total = len(reqs)
        while len(stats.results) + len(self.cancelled) < total:
            now = now_fn()
            while i < total and reqs[i].arrival <= now:
                self.submit(reqs[i])
                i += 1
            self._admit(now)
            stats.peak_bytes = max(stats.peak_bytes, self.used)
            stats.peak_slots = max(stats.peak_slots, len(self.active))
            if not self.active:
                if i < total:
                    time.sleep(max(0.0, min(0.002, reqs[i].arrival - now_fn())))
                continue
            for b in self.batches.values():
                if len(b):
                    b.run(self.quantum)
            stats.quanta += 1
            stats.results.extend(self._retire(now_fn))
        stats.elapsed = now_fn()
        return stats


def sequential(requests: list[Request], clock=time.perf_counter, stream_handle=None) -> ServerStats:
    """The plain path: one Session per request, first come first served."""
    from .dim import Session
    stats = ServerStats()
    reqs = sorted(requests, key=lambda r: r.arrival)
    t0 = clock()
    for r in reqs:
        while clock() - t0 < r.arrival:
            time.sleep(max(0.0, min(0.002, r.arrival - (clock() - t0))))
        start = clock() - t0
        with Session(r.desc, r.U) as s:
            if stream_handle:
                s.set_stream(stream_handle)
            dts = s.steps(r.steps, r.cfl, r.dt_max)
            U = s.download()
        stats.results.append(Result(r.rid, U, dts, r.arrival, start, clock() - t0))
    stats.elapsed = clock() - t0
    return stats


def make_requests(n: int, rate: float, seed: int = 0, steps_range=(100, 2000), share_1d: float = 0.4,
                  n1d_range=(256, 8192), side2d_range=(128, 2048), share_mixed: float = 0.5) -> list[Request]:
    """Config 4 request stream: Poisson arrivals at `rate` per second; 40 %
    1D tubes (N log-uniform in n1d_range), 60 % 2D grids (sides log-uniform
    in side2d_range), steps uniform in steps_range, config-0/1 style seeded
    initial conditions, a share_mixed fraction of them in the mixed-precision
    form."""
    from . import workloads as W
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(n):
        t += rng.exponential(1.0 / rate) if rate > 0 else 0.0
        s = int(rng.integers(0, 2**31 - 1))
        steps = int(rng.integers(steps_range[0], steps_range[1] + 1))
        if rng.uniform() < share_1d:
            N = int(round(math.exp(rng.uniform(math.log(n1d_range[0]), math.log(n1d_range[1])))))
            d, U = W.riemann(seed=s, N=(N,))
        else:
            N = tuple(int(round(math.exp(rng.uniform(math.log(side2d_range[0]), math.log(side2d_range[1])))))
                      for _ in range(2))
            d, U = W.riemann(seed=s, N=N, axis=int(rng.integers(0, 2))) if rng.uniform() < 0.5 \
                else W.single_bubble_2d(N, seed=s)
        if rng.uniform() < share_mixed:
            d.precision = PRECISION_MIXED
        out.append(Request(k, d, U, steps, 0.6, 1e300, t))
    return out
