"""ctypes mirror of include/dimgpu.h (the library's C-ABI).

The structs and enums here are byte-for-byte the ones the header declares, so
Python callers, the tests and the CPU checkers all speak the same descriptor.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

MAX_MATERIALS = 4

# status codes
OK = 0
E_INVALID_ARG = 1
E_UNSUPPORTED_EOS = 2
E_NONFINITE = 3
E_TIMEOUT = 4
E_OOM = 5
E_CUDA = 6
E_UNSUPPORTED = 7

STATUS_NAMES = {
    OK: "DIMGPU_OK", E_INVALID_ARG: "DIMGPU_E_INVALID_ARG",
    E_UNSUPPORTED_EOS: "DIMGPU_E_UNSUPPORTED_EOS", E_NONFINITE: "DIMGPU_E_NONFINITE",
    E_TIMEOUT: "DIMGPU_E_TIMEOUT", E_OOM: "DIMGPU_E_OOM", E_CUDA: "DIMGPU_E_CUDA",
    E_UNSUPPORTED: "DIMGPU_E_UNSUPPORTED",
}

# EoS kinds, numbered like the reference's EOSKind (src/euler/eos_params.hpp:8-15)
EOS_KINDS = {
    "ideal_gas": 0, "stiffened_gas": 1, "noble_abel": 2, "real_gas": 2, "noble_abel_gas": 2,
    "peng_robinson": 3, "peng-robinson": 3, "tait": 4, "mie_gruneisen": 5,
    "mie-gruneisen": 5, "mie_gruneisen_fluid": 5,
}
EOS_IDEAL_GAS = 0
EOS_STIFFENED_GAS = 1

BC_TRANSMISSIVE = 0
BC_REFLECTIVE = 1
BC_NONREFLECTIVE = 2

LAMBDA_KAPILA = 0
LAMBDA_ALLAIRE = 1
LAMBDA_EQUAL_VELOCITY = 2
LAMBDA_MODELS = {"kapila": 0, "": 0, "allaire": 1, "equal_velocity": 2}

PRECISION_FP64 = 0
PRECISION_MIXED = 1
PRECISION_MIXED_FP64 = 2   # the mixed algorithm in FP64 throughout (its FP64 twin)

SCHEDULE_FUSED = 0
SCHEDULE_STAGED = 1

TIME_SPLIT = 0
TIME_UNSPLIT = 1

MODEL_DIM = 0     # the five-equation diffuse-interface step
MODEL_EULER = 1   # the single-material Euler step (one material, no level set)


class Material(C.Structure):
    _fields_ = [("kind", C.c_int), ("gamma", C.c_double), ("p_inf", C.c_double)]


class Desc(C.Structure):
    _fields_ = [
        ("dim", C.c_int),
        ("N", C.c_int * 3),
        ("dx", C.c_double * 3),
        ("nmat", C.c_int),
        ("mat", Material * MAX_MATERIALS),
        ("bc_lo", C.c_int * 3),
        ("bc_hi", C.c_int * 3),
        ("lambda_model", C.c_int),
        ("alpha_source_floor", C.c_double),
        ("precision", C.c_int),
        ("time_update", C.c_int),
        ("model", C.c_int),
    ]

    @property
    def ncell(self) -> int:
        n = 1
        for a in range(self.dim):
            n *= self.N[a]
        return n

    @property
    def nvar(self) -> int:
        return 2 * self.nmat + self.dim

    def shape(self):
        return tuple(self.N[a] for a in range(self.dim))

    def copy(self) -> "Desc":
        d = Desc()
        C.memmove(C.byref(d), C.byref(self), C.sizeof(Desc))
        return d


class ShockBubbleIC(C.Structure):
    """dimgpu_ic_shock_bubble."""
    _fields_ = [("center", C.c_double * 2), ("radius", C.c_double), ("thickness", C.c_double),
                ("sharpness", C.c_double), ("shock_x", C.c_double), ("zero_below", C.c_double),
                ("rho_post", C.c_double), ("u_post", C.c_double), ("p_post", C.c_double),
                ("rho_pre", C.c_double), ("p_pre", C.c_double), ("rho_bubble", C.c_double),
                ("p_bubble", C.c_double)]


class BubbleIC(C.Structure):
    """dimgpu_ic_bubble."""
    _fields_ = [("center", C.c_double * 3), ("radius", C.c_double), ("box_lo", C.c_int * 3),
                ("box_hi", C.c_int * 3)]


class BubbleCloudIC(C.Structure):
    """dimgpu_ic_bubble_cloud."""
    _fields_ = [("thickness", C.c_double), ("sharpness", C.c_double), ("zero_below", C.c_double),
                ("pulse_width", C.c_double), ("rho_liquid", C.c_double), ("rho_gas", C.c_double),
                ("p_ambient", C.c_double), ("p_pulse", C.c_double)]


class ServerConfig(C.Structure):
    """dimgpu_server_config."""
    _fields_ = [("hbm_budget_bytes", C.c_double), ("dim_share", C.c_double * 3), ("max_slots", C.c_int),
                ("quantum", C.c_int), ("max_steps_per_solve", C.c_int), ("solo_min_cells", C.c_longlong),
                ("solo_share", C.c_double), ("solo_slots", C.c_int)]


class ServerCounters(C.Structure):
    """dimgpu_server_counters."""
    _fields_ = [("submitted", C.c_longlong), ("completed", C.c_longlong), ("cancelled", C.c_longlong),
                ("failed", C.c_longlong), ("quanta", C.c_longlong), ("queued", C.c_longlong),
                ("resident", C.c_int), ("peak_resident", C.c_int), ("peak_bytes", C.c_double)]


REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_CANCELLED, REQ_FAILED = 0, 1, 2, 3, 4


def fill_struct(st: C.Structure, values: dict) -> C.Structure:
    """Set the fields of a ctypes structure from a dict (sequences for arrays)."""
    for name, _ in st._fields_:
        v = values[name]
        if isinstance(v, (tuple, list)):
            arr = getattr(st, name)
            for i, x in enumerate(v):
                arr[i] = x
        else:
            setattr(st, name, v)
    return st


class PhaseTimes(C.Structure):
    _fields_ = [("cfl_ms", C.c_double), ("sweep_ms", C.c_double), ("boundary_ms", C.c_double)]


def bc_code(name) -> int:
    if isinstance(name, int):
        return name
    name = str(name).strip().lower()
    if name == "reflective":
        return BC_REFLECTIVE
    if name in ("nonreflective", "non_reflective"):
        return BC_NONREFLECTIVE
    return BC_TRANSMISSIVE


def make_desc(dim: int, N: Sequence[int], dx: Sequence[float],
              materials: Sequence[tuple], bc_lo=None, bc_hi=None,
              lambda_model="kapila", alpha_source_floor: float = 0.0,
              precision: int = PRECISION_FP64, time_update="split", model: int = MODEL_DIM) -> Desc:
    """Build a descriptor.  materials: (kind, gamma, p_inf) with kind a name or code."""
    if dim not in (1, 2, 3):
        raise ValueError("dim must be 1, 2 or 3")
    if len(N) != dim or len(dx) != dim:
        raise ValueError("N and dx need one entry per axis")
    if not 1 <= len(materials) <= MAX_MATERIALS:
        raise ValueError(f"1..{MAX_MATERIALS} materials supported")
    d = Desc()
    d.dim = dim
    for a in range(3):
        d.N[a] = int(N[a]) if a < dim else 1
        d.dx[a] = float(dx[a]) if a < dim else 1.0
    d.nmat = len(materials)
    for k, (kind, gamma, p_inf) in enumerate(materials):
        d.mat[k].kind = EOS_KINDS[kind] if isinstance(kind, str) else int(kind)
        d.mat[k].gamma = float(gamma)
        d.mat[k].p_inf = float(p_inf)
    bc_lo = bc_lo or ["transmissive"] * dim
    bc_hi = bc_hi or ["transmissive"] * dim
    for a in range(3):
        d.bc_lo[a] = bc_code(bc_lo[a]) if a < dim else 0
        d.bc_hi[a] = bc_code(bc_hi[a]) if a < dim else 0
    d.lambda_model = LAMBDA_MODELS[lambda_model] if isinstance(lambda_model, str) else int(lambda_model)
    d.alpha_source_floor = float(alpha_source_floor)
    d.precision = int(precision)
    if isinstance(time_update, str):
        time_update = TIME_UNSPLIT if time_update.lower() == "unsplit" else TIME_SPLIT
    d.time_update = int(time_update)
    d.model = int(model)
    return d


DPTR = C.POINTER(C.c_double)


def dptr(a) -> "C._Pointer":
    """Pointer to a C-contiguous float64 numpy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data_as(DPTR)
