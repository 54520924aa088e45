"""Python face of the DIM step, mirroring the reference's call surface.

The reference (src/dim/solver/advance_step.hpp:29-149) exposes
``dim::advance_one_step<DIM>(U, N, dx, params, cfg, cfl, dt_max) ->
StepResult{U_new, dt, phase_timings}`` with ``compute_dt_cfl``,
``sweep_direction_dispatch`` and ``apply_boundary_conditions`` beneath it.
Here the state is a NumPy SoA array ``(V, ncell)`` (include/dimgpu.h) and every
call goes through the C-ABI of libdimgpu.so; errors raise DimGpuError where
the reference throws std::runtime_error.

``Session`` keeps the state resident on the GPU between steps (the form the
reference's time loop in src/app/solver/run_dim.hpp:88-154 needs);
``advance_one_step`` is the stateless drop-in (host arrays in and out).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

from . import abi
from .abi import Desc, PhaseTimes, dptr
from .native import DimGpuError, check, lib

__all__ = ["Session", "StepResult", "advance_one_step", "DimGpuError"]


@dataclass
class StepResult:
    """dim::StepResult (src/dim/solver/advance_step.hpp:20-25); times in seconds."""
    U_new: np.ndarray
    dt: float
    phase_timings: dict = field(default_factory=dict)


def _times_dict(t: PhaseTimes) -> dict:
    return {"cfl_seconds": t.cfl_ms * 1e-3, "sweep_seconds": t.sweep_ms * 1e-3,
            "boundary_seconds": t.boundary_ms * 1e-3}


class CsvWriter:
    """An asynchronous CSV snapshot (dimgpu_csv_write_async)."""

    def __init__(self, handle):
        self._h = handle

    def wait(self) -> None:
        if self._h:
            h, self._h = self._h, None
            check(lib().dimgpu_csv_wait(h))

    def __del__(self):
        try:
            self.wait()
        except Exception:
            pass


class Session:
    """Device-resident DIM state with the reference's step operations."""

    def __init__(self, desc: Desc, U: np.ndarray | None = None):
        self.desc = desc.copy()
        h = C.c_void_p()
        check(lib().dimgpu_create(C.byref(self.desc), C.byref(h)))
        self._h = h
        if U is not None:
            self.upload(U)

    # ---- lifetime
    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().dimgpu_destroy(self._h)
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

    def _check(self, rc: int) -> None:
        check(rc, self._h)

    @property
    def count(self) -> int:
        return self.desc.nvar * self.desc.ncell

    # ---- data movement
    def upload(self, U: np.ndarray) -> None:
        U = np.ascontiguousarray(U, dtype=np.float64)
        if U.size != self.count:
            raise DimGpuError(abi.E_INVALID_ARG, "dim::advance_one_step: grid size mismatch")
        self._check(lib().dimgpu_upload(self._h, dptr(U), U.size))

    def download(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty((self.desc.nvar, self.desc.ncell))
        self._check(lib().dimgpu_download(self._h, dptr(out), out.size))
        return out

    # ---- the reference's operations
    def compute_dt_cfl(self, cfl: float, dt_max: float) -> float:
        """dim::compute_dt_cfl (src/dim/solver/cfl.hpp:16-66)."""
        dt = C.c_double()
        self._check(lib().dimgpu_compute_dt_cfl(self._h, cfl, dt_max, C.byref(dt)))
        return dt.value

    def sweep_direction(self, direction: int, dt: float) -> None:
        """dim::sweep_direction_dispatch (src/dim/solver/advance/sweep_core.hpp:151-202)."""
        self._check(lib().dimgpu_sweep_direction(self._h, direction, dt))

    def apply_boundary_conditions(self) -> None:
        """dim::apply_boundary_conditions (src/dim/solver/advance/boundary.hpp:165-226)."""
        self._check(lib().dimgpu_apply_boundary_conditions(self._h))

    def step(self, cfl: float, dt_max: float, timings: bool = False):
        """One dim::advance_one_step on the resident state; returns (dt, phase_timings)."""
        dt = C.c_double()
        t = PhaseTimes()
        self._check(lib().dimgpu_step(self._h, cfl, dt_max, C.byref(dt), C.byref(t) if timings else None))
        return dt.value, (_times_dict(t) if timings else {})

    def steps(self, n: int, cfl: float, dt_max: float) -> np.ndarray:
        """n steps with constant cfl / dt_max and no host synchronisation; the dts."""
        dts = np.zeros(max(n, 1))
        self._check(lib().dimgpu_steps(self._h, n, cfl, dt_max, dptr(dts)))
        return dts[:n]

    def enqueue_steps(self, n: int, cfl: float, dt_max: float) -> None:
        """Enqueue n steps on the session's stream without waiting."""
        self._check(lib().dimgpu_enqueue_steps(self._h, n, cfl, dt_max))

    def collect(self) -> np.ndarray:
        """Wait for the enqueued steps; their dts (raises on any step's error)."""
        dts = np.zeros(4096)
        cnt = C.c_int()
        self._check(lib().dimgpu_collect(self._h, dptr(dts), dts.size, C.byref(cnt)))
        return dts[:cnt.value].copy()

    def totals(self) -> np.ndarray:
        """{material_mass[nmat], mass, momentum[dim], energy} (conservation_report.hpp:188-218)."""
        out = np.zeros(self.desc.nmat + self.desc.dim + 2)
        self._check(lib().dimgpu_totals(self._h, dptr(out)))
        return out

    def boundary_flux(self) -> np.ndarray:
        """The boundary flux integrand, laid out as totals()
        (app_io::compute_dim_boundary_flux, src/app/io/conservation_report.hpp:253-305)."""
        out = np.zeros(self.desc.nmat + self.desc.dim + 2)
        self._check(lib().dimgpu_boundary_flux(self._h, dptr(out)))
        return out

    # ---- initial fields on the device, CSV snapshots
    def init_shock_bubble(self, ic: dict) -> None:
        """Write the shock-bubble field (workloads.shock_bubble_2d_setup's
        parameters) into the device state: the same bits as the host
        generator workloads.shock_bubble_2d."""
        st = abi.fill_struct(abi.ShockBubbleIC(), ic)
        self._check(lib().dimgpu_init_shock_bubble(self._h, C.byref(st)))

    def init_bubble_cloud(self, ic: dict, bubbles) -> None:
        """Write the bubble-cloud field (workloads.bubble_cloud_3d_setup's
        parameters and bubbles) into the device state: the same bits as the
        host generator workloads.bubble_cloud_3d."""
        st = abi.fill_struct(abi.BubbleCloudIC(), ic)
        arr = (abi.BubbleIC * max(1, len(bubbles)))()
        for b, (c, r, lo, hi) in enumerate(bubbles):
            abi.fill_struct(arr[b], {"center": c, "radius": r, "box_lo": lo, "box_hi": hi})
        self._check(lib().dimgpu_init_bubble_cloud(self._h, C.byref(st), arr, len(bubbles)))

    def write_csv_async(self, filename: str, domain_min, domain_max, threads: int = 0) -> "CsvWriter":
        """Start writing the current state as dim::write_csv does
        (src/io/dim_write_csv.hpp:15-125); the session may keep stepping.
        Call .wait() on the result."""
        lo = np.zeros(3)
        hi = np.zeros(3)
        lo[:len(domain_min)] = domain_min
        hi[:len(domain_max)] = domain_max
        h = C.c_void_p()
        self._check(lib().dimgpu_csv_write_async(self._h, os.fsencode(filename), dptr(lo), dptr(hi), threads,
                                                 C.byref(h)))
        return CsvWriter(h)

    # ---- tuning and measurement
    def set_stream(self, stream_handle: int | None) -> None:
        self._check(lib().dimgpu_set_stream(self._h, C.c_void_p(stream_handle or 0)))

    def set_tile(self, direction: int, T: int, W: int) -> None:
        self._check(lib().dimgpu_set_tile(self._h, direction, T, W))

    def set_schedule(self, direction: int, schedule: int) -> None:
        """abi.SCHEDULE_FUSED (one tiled kernel) or abi.SCHEDULE_STAGED (a kernel per stage)."""
        self._check(lib().dimgpu_set_schedule(self._h, direction, schedule))

    def profile(self, enable: bool) -> None:
        self._check(lib().dimgpu_profile(self._h, 1 if enable else 0))

    def profile_read(self) -> dict:
        out = np.zeros(8)
        self._check(lib().dimgpu_profile_read(self._h, dptr(out)))
        kinds = ("sweep", "cfl", "boundary", "other")
        return {k: {"ms": float(out[2 * i]), "launches": int(out[2 * i + 1])} for i, k in enumerate(kinds)}


def compute_dt_cfl_noalloc(desc: Desc, device_ptr: int, cfl: float, dt_max: float,
                           stream_handle: int | None = None) -> float:
    """CFL dt of a state the caller keeps in its own device memory
    (device_ptr: address of the SoA array), without any device allocation.

    For callers that manage all GPU memory themselves and cannot have the
    library allocate mid-loop.  At most 4 194 304 cells; the library's one
    static scratch array per GPU is shared by all calls, so overlapping calls
    on the same device race."""
    dt = C.c_double()
    check(lib().dimgpu_compute_dt_cfl_noalloc(C.byref(desc), C.cast(C.c_void_p(device_ptr), abi.DPTR), cfl,
                                              dt_max, C.byref(dt), C.c_void_p(stream_handle or 0)))
    return dt.value


def advance_one_step(U: np.ndarray, desc: Desc, cfl: float, dt_max: float,
                     timings: bool = False) -> StepResult:
    """Stateless drop-in for dim::advance_one_step: host SoA in, StepResult out."""
    U = np.ascontiguousarray(U, dtype=np.float64)
    out = np.empty_like(U)
    dt = C.c_double()
    t = PhaseTimes()
    check(lib().dimgpu_advance_one_step(C.byref(desc), dptr(U), dptr(out), cfl, dt_max, C.byref(dt),
                                        C.byref(t) if timings else None))
    return StepResult(out, dt.value, _times_dict(t) if timings else {})


class Slabs:
    """One grid decomposed into slabs along its slowest axis, one slab per
    listed device (dimgpu_slabs_*): bit-identical to a Session on the whole
    grid.  devices may repeat a device."""

    def __init__(self, desc: Desc, devices, U: np.ndarray | None = None):
        self.desc = desc.copy()
        devs = (C.c_int * len(devices))(*devices)
        h = C.c_void_p()
        check(lib().dimgpu_slabs_create(C.byref(self.desc), len(devices), devs, C.byref(h)))
        self._h = h
        if U is not None:
            self.upload(U)

    def _check(self, rc: int) -> None:
        if rc != 0:
            msg = lib().dimgpu_slabs_last_error(self._h)
            raise DimGpuError(rc, msg.decode() if msg else "")

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().dimgpu_slabs_destroy(self._h)
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

    def upload(self, U: np.ndarray) -> None:
        U = np.ascontiguousarray(U, dtype=np.float64)
        self._check(lib().dimgpu_slabs_upload(self._h, dptr(U), U.size))

    def download(self) -> np.ndarray:
        out = np.empty((self.desc.nvar, self.desc.ncell))
        self._check(lib().dimgpu_slabs_download(self._h, dptr(out), out.size))
        return out

    def step(self, cfl: float, dt_max: float) -> float:
        dt = C.c_double()
        self._check(lib().dimgpu_slabs_step(self._h, cfl, dt_max, C.byref(dt)))
        return dt.value

    def steps(self, n: int, cfl: float, dt_max: float) -> np.ndarray:
        return np.array([self.step(cfl, dt_max) for _ in range(n)])
