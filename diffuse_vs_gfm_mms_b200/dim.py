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
