"""Python face of the single-material Euler step (model MODEL_EULER).

The reference's sharp-interface solver advances a step with
``advance_one_step<DIM, EOS>(U, ctx) -> StepResult{U_new, phi_list_new, dt,
rgfm_diagnostic_rows, phase_timings}`` (src/sim/solver/advance_step.hpp:
489-866).  With no level set (``ctx.phi_list`` empty) and one material the
step reduces to its single-material fast path (advance_line,
src/sim/solver/advance/sweep_core.hpp:65-111): the CFL dt, MUSCL-Hancock +
HLLC sweeps and the boundary fill, which is what this module runs on the GPU.
Steps with level sets or several materials are the reference's rGFM path and
stay on the reference's CPU code; ``advance_one_step`` refuses them.

State: NumPy SoA ``(2 + DIM, ncell)``, components rho, mom[0..DIM-1], E.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

from . import abi
from .abi import Desc
from .dim import DimGpuError, Session

__all__ = ["SolverContext", "StepResult", "advance_one_step", "desc_from_context"]


@dataclass
class SolverContext:
    """The fields of SolverContext<DIM> (src/sim/solver/solver_context.hpp:
    21-60) that the single-material step reads."""
    N: Sequence[int]
    dx: Sequence[float]
    material_params: Sequence[tuple]            # [(kind, gamma, p_inf)]
    cfl: float = 0.5
    dt_max: float = 1e-3
    bc_lo: Sequence = ()
    bc_hi: Sequence = ()
    time_update: str = "split"
    phi_list: Sequence = ()
    completed_steps: int = 0


@dataclass
class StepResult:
    U_new: np.ndarray
    phi_list_new: list
    dt: float
    rgfm_diagnostic_rows: list = field(default_factory=list)
    phase_timings: dict = field(default_factory=dict)


def desc_from_context(ctx: SolverContext) -> Desc:
    if len(ctx.phi_list) != 0 or len(ctx.material_params) != 1:
        raise ValueError("level sets or several materials: that step is the reference's rGFM path, "
                         "which stays on its CPU code")
    dim = len(ctx.N)
    return abi.make_desc(dim, ctx.N, ctx.dx, list(ctx.material_params),
                         bc_lo=list(ctx.bc_lo) or None, bc_hi=list(ctx.bc_hi) or None,
                         time_update=ctx.time_update, model=abi.MODEL_EULER)


_cache: dict = {}


def advance_one_step(U: np.ndarray, ctx: SolverContext) -> StepResult:
    """Drop-in for the reference's single-material advance_one_step: host SoA
    in, StepResult out (a cached device session per grid shape)."""
    d = desc_from_context(ctx)
    key = bytes(d)
    s = _cache.get(key)
    if s is None:
        for old in _cache.values():
            old.close()
        _cache.clear()
        s = _cache[key] = Session(d)
    s.upload(U)
    dt, times = s.step(ctx.cfl, ctx.dt_max, timings=True)
    ctx.completed_steps += 1
    return StepResult(s.download(), [], dt, [], times)
