"""Autotuner for the sweep schedule and tile shape, and for the batch grid.

For every sweep axis the tuner times, on a throw-away session holding a copy
of the caller's state, the staged schedule (one kernel per stage) against the
fused tiled kernel with several tile shapes, and keeps the fastest.  Results
do not depend on the choice (the tests check bit equality across schedules
and tiles), only the speed does.  Choices are cached per key
(nmat, dim, precision, axis, log2 line length, log2 line count) in memory and
in a JSON file (``DIMGPU_TUNE_CACHE``, default ``~/.cache/dimgpu/tune.json``),
so a shape class is measured once.

For a ``Batch`` the tuner picks the persistent grid size (CTAs per launch)
from a few multiples of the SM count by timing one step of a throw-away batch
built from a sample of the instances.
"""
from __future__ import annotations

import json
import math
import os
import time

import numpy as np

from . import abi
from .abi import Desc

FUSED_X = [(128, 1), (256, 1), (64, 1)]
FUSED_YZ = [(64, 4), (32, 8), (128, 2)]

_memory: dict[str, dict] = {}


def cache_path() -> str:
    return os.environ.get("DIMGPU_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "dimgpu",
                                                            "tune.json"))


def _load() -> dict:
    p = cache_path()
    try:
        with open(p) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(key: str, value: dict) -> None:
    _memory[key] = value
    p = cache_path()
    try:
        os.makedirs(os.path.dirname(p), exist_ok=True)
        data = _load()
        data[key] = value
        tmp = p + f".{os.getpid()}"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, p)
    except OSError:
        pass


def key_for(desc: Desc, direction: int) -> str:
    n = desc.N[direction]
    lines = desc.ncell // n
    return (f"nm{desc.nmat}-d{desc.dim}-p{desc.precision}-dir{direction}-"
            f"n{int(round(math.log2(max(n, 1))))}-l{int(round(math.log2(max(lines, 1))))}")


def candidates(desc: Desc, direction: int):
    """(schedule, T, W) triples worth timing for one axis."""
    out = [(abi.SCHEDULE_STAGED, 0, 0)]
    if desc.precision == abi.PRECISION_FP64:
        for T, W in (FUSED_X if direction == 0 else FUSED_YZ):
            if direction != 0 and desc.N[0] < W:
                continue
            out.append((abi.SCHEDULE_FUSED, T, W))
    return out


def _apply(session, direction: int, choice) -> None:
    sched, T, W = choice
    session.set_schedule(direction, sched)
    if sched == abi.SCHEDULE_FUSED:
        session.set_tile(direction, T, W)


def tune(desc: Desc, U: np.ndarray, cfl: float = 0.6, repeats: int = 2, force: bool = False) -> dict:
    """Best (schedule, T, W) per axis for this grid; measured or cached."""
    from .dim import Session
    result = {}
    disk = None
    todo = []
    for direction in range(desc.dim):
        if desc.N[direction] <= 1:
            continue
        k = key_for(desc, direction)
        if not force:
            if k not in _memory:
                disk = _load() if disk is None else disk
                if k in disk:
                    _memory[k] = disk[k]
            if k in _memory:
                result[direction] = tuple(_memory[k]["choice"])
                continue
        todo.append(direction)
    if not todo:
        return result
    with Session(desc, U) as s:
        dt = s.compute_dt_cfl(cfl, 1e300)
        for direction in todo:
            timings = []
            for choice in candidates(desc, direction):
                _apply(s, direction, choice)
                s.upload(U)
                s.sweep_direction(direction, dt)  # first touch (scratch allocation, caches)
                s.upload(U)
                s.profile(True)
                for _ in range(repeats):
                    s.sweep_direction(direction, dt)
                ms = s.profile_read()["sweep"]["ms"] / repeats
                s.profile(False)
                timings.append((ms, choice))
            timings.sort(key=lambda x: x[0])
            best = timings[0][1]
            result[direction] = best
            _store(key_for(desc, direction), {"choice": list(best),
                                              "ms": {f"{c[0]}:{c[1]}x{c[2]}": m for m, c in timings},
                                              "when": time.strftime("%Y-%m-%dT%H:%M:%S")})
    return result


def apply(session, choices: dict) -> None:
    """Set a session's schedule and tiles from tune()'s result."""
    for direction, choice in choices.items():
        _apply(session, direction, choice)


def tune_batch_grid(instances, nmat: int, dim: int, cfl: float = 0.6, multiples=(2, 4, 8)) -> int:
    """Persistent grid size (CTAs) for batches like `instances` (a list of
    (desc, U)); times one step of a throw-away batch per candidate."""
    from .batch import Batch
    dev_sms = 148
    try:
        import torch
        dev_sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    except Exception:
        pass
    best = None
    for m in multiples:
        with Batch(nmat, dim) as b:
            b.set_grid(m * dev_sms)
            for d, U in instances:
                b.add(d, U, 2, cfl)
            b.run(1)                       # tables, scratch, first launch
            t0 = time.perf_counter()
            b.run(1)
            el = time.perf_counter() - t0
        if best is None or el < best[0]:
            best = (el, m * dev_sms)
    return best[1]
