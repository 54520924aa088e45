"""Continuous-batching serving loop for DIM solve requests.

Requests (a grid, its initial state and a step budget) arrive over time.  The
server (dimgpu_server_* in libdimgpu.so, a native server thread) admits them
first-come-first-served as long as their device footprint fits the HBM
budget and a slot is free, keeps every admitted solve's state resident on the
GPU in device memory reserved once (admission allocates and synchronises
nothing), and advances all admitted solves together in quanta of a few steps
through the batched form, one batch per material count and dimension, each
on its own stream so that they overlap.  A request that arrives while others
run joins at the next quantum; a finished request is downloaded and its
memory returned at once, which is what lets the queue drain into the freed
room.

Every solve's arithmetic is the single-grid step's, so a result does not
depend on what else was in flight (tests/test_gpu_serving.py).
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import abi
from .abi import PRECISION_MIXED, Desc, dptr
from .native import DimGpuError, lib

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
    """The continuous-batching server (dimgpu_server_* in libdimgpu.so): a
    native server thread admits, steps and retires solves; this class submits
    requests at their arrival times and collects the results."""

    def __init__(self, hbm_budget_bytes: float = 150e9, max_slots: int = 128, quantum: int = 8,
                 dim_share=(0.1, 0.4, 0.0), max_steps_per_solve: int = 4096, solo_min_cells: int = 1 << 18,
                 solo_share: float = 0.5, solo_slots: int = 4):
        cfg = abi.ServerConfig()
        cfg.hbm_budget_bytes = float(hbm_budget_bytes)
        for k in range(3):
            cfg.dim_share[k] = float(dim_share[k])
        cfg.max_slots = max_slots
        cfg.quantum = quantum
        cfg.max_steps_per_solve = max_steps_per_solve
        cfg.solo_min_cells = solo_min_cells
        cfg.solo_share = float(solo_share)
        cfg.solo_slots = solo_slots
        h = C.c_void_p()
        self._check(lib().dimgpu_server_create(C.byref(cfg), C.byref(h)), None)
        self._h = h
        self.budget = float(hbm_budget_bytes)
        self.ids: dict[int, int] = {}        # request rid -> server request id
        self.reqs: dict[int, Request] = {}

    def _check(self, rc: int, h=...) -> None:
        if rc != 0:
            handle = self._h if h is ... else h
            msg = lib().dimgpu_server_last_error(handle) if handle else lib().dimgpu_last_error(None)
            raise DimGpuError(rc, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "_h", None):
            lib().dimgpu_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, req: Request) -> None:
        U = np.ascontiguousarray(req.U, dtype=np.float64)
        nid = C.c_longlong()
        self._check(lib().dimgpu_server_submit(self._h, C.byref(req.desc), dptr(U), req.steps, req.cfl, req.dt_max,
                                               C.byref(nid)))
        self.ids[req.rid] = nid.value
        self.reqs[req.rid] = req

    def state(self, rid: int) -> int:
        st = C.c_int()
        self._check(lib().dimgpu_server_poll(self._h, self.ids[rid], C.byref(st), None, 0, None, None))
        return st.value

    def cancel(self, rid: int) -> bool:
        """Drop a queued or running request; True if it was still known."""
        if rid not in self.ids:
            return False
        return lib().dimgpu_server_cancel(self._h, self.ids[rid]) == 0

    def collect(self, rid: int):
        """(state, U, dts, latency) of a request; U / dts are meaningful only
        when it is done (the request is then forgotten by the server)."""
        req = self.reqs[rid]
        st, lat = C.c_int(), C.c_double()
        U = np.empty((req.desc.nvar, req.desc.ncell))
        dts = np.zeros(max(req.steps, 1))
        self._check(lib().dimgpu_server_poll(self._h, self.ids[rid], C.byref(st), dptr(U), U.size, dptr(dts),
                                             C.byref(lat)))
        if st.value in (abi.REQ_DONE, abi.REQ_CANCELLED):
            del self.ids[rid]
        return st.value, U, dts[:req.steps], lat.value

    def drain(self) -> None:
        self._check(lib().dimgpu_server_drain(self._h))

    def counters(self) -> abi.ServerCounters:
        out = abi.ServerCounters()
        self._check(lib().dimgpu_server_stats(self._h, C.byref(out)))
        return out

    def serve(self, requests: list[Request], clock=time.perf_counter) -> ServerStats:
        """Submit every request at its `arrival` offset (wall clock) and
        collect the results as they finish."""
        stats = ServerStats()
        reqs = sorted(requests, key=lambda r: r.arrival)
        t0 = clock()
        now_fn = lambda: clock() - t0  # noqa: E731
        submit_at: dict[int, float] = {}
        outstanding: list[int] = []
        i = 0
        while i < len(reqs) or outstanding:
            now = now_fn()
            while i < len(reqs) and reqs[i].arrival <= now:
                self.submit(reqs[i])
                submit_at[reqs[i].rid] = now_fn()
                outstanding.append(reqs[i].rid)
                i += 1
            still = []
            for rid in outstanding:
                if self.state(rid) != abi.REQ_DONE:
                    still.append(rid)
                    continue
                _, U, dts, lat = self.collect(rid)
                r = self.reqs[rid]
                stats.results.append(Result(rid, U, dts, r.arrival, submit_at[rid], submit_at[rid] + lat))
            outstanding = still
            if outstanding or i < len(reqs):
                nxt = reqs[i].arrival - now_fn() if i < len(reqs) else 0.002
                time.sleep(max(0.0, min(0.002, nxt)))
        stats.elapsed = now_fn()
        c = self.counters()
        stats.peak_bytes = int(c.peak_bytes)
        stats.peak_slots = int(c.peak_resident)
        stats.quanta = int(c.quanta)
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
