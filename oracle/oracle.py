"""TEST INFRASTRUCTURE ONLY — ctypes front end of the CPU checkers.

Two interchangeable back ends with the same functions:

* ``port``      — oracle/_build/libdimoracle.so, the C restatement of the
                  reference algorithm (oracle/dim_oracle.c);
* ``reference`` — oracle/_ref/libdimref.so, the reference's own header-only
                  code compiled from its sources (oracle/ref_harness.cpp).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the product package never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from diffuse_vs_gfm_mms_b200.abi import Desc, dptr

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "_build", "libdimoracle.so")
REF_SO = os.path.join(HERE, "_ref", "libdimref.so")


def build(quiet: bool = True, ref_src: str | None = None) -> None:
    """Compile the C restatement, and the reference from its sources when
    `ref_src` (or $DIMGPU_REFERENCE_SRC) names a checkout of it."""
    ref_src = ref_src or os.environ.get("DIMGPU_REFERENCE_SRC", "")
    cmd = ["make", "-C", HERE] + ([f"REF={ref_src}"] if ref_src else [])
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


class Checker:
    def __init__(self, kind: str = "port"):
        self.kind = kind
        path = PORT_SO if kind == "port" else REF_SO
        if not os.path.exists(path):
            raise FileNotFoundError(f"{kind} checker not built: {path}")
        self.lib = C.CDLL(path)
        self.prefix = "oracle_" if kind == "port" else "ref_"
        self._err = getattr(self.lib, self.prefix + "last_error")
        self._err.restype = C.c_char_p

    def _fn(self, name):
        f = getattr(self.lib, self.prefix + name)
        f.restype = C.c_int
        return f

    def _check(self, rc, name):
        if rc != 0:
            raise RuntimeError(f"{self.kind}.{name}: status {rc}: {self._err().decode()}")

    def set_threads(self, n: int) -> None:
        if self.kind == "port":
            self.lib.oracle_set_threads(C.c_int(n))
        else:
            self.lib.ref_set_threads(C.c_int(n))

    def max_threads(self) -> int:
        if self.kind == "port":
            return int(self.lib.oracle_set_threads(C.c_int(0)))
        return int(self.lib.ref_max_threads())

    # ---- field level ----
    def advance(self, d: Desc, soa: np.ndarray, cfl: float, dt_max: float, nsteps: int = 1):
        soa = np.ascontiguousarray(soa, dtype=np.float64)
        out = np.empty_like(soa)
        dts = np.zeros(max(nsteps, 1))
        if self.kind == "port":
            rc = self._fn("advance")(C.byref(d), dptr(soa), dptr(out), C.c_double(cfl),
                                     C.c_double(dt_max), C.c_int(nsteps), dptr(dts))
        else:
            rc = self._fn("advance")(C.byref(d), dptr(soa), dptr(out), C.c_double(cfl),
                                     C.c_double(dt_max), C.c_int(nsteps), dptr(dts), None)
        self._check(rc, "advance")
        return out, dts[:nsteps]

    def compute_dt_cfl(self, d: Desc, soa, cfl, dt_max) -> float:
        soa = np.ascontiguousarray(soa, dtype=np.float64)
        dt = C.c_double(0.0)
        self._check(self._fn("compute_dt_cfl")(C.byref(d), dptr(soa), C.c_double(cfl),
                                               C.c_double(dt_max), C.byref(dt)), "cfl")
        return dt.value

    def sweep_direction(self, d: Desc, direction: int, dt: float, soa):
        soa = np.ascontiguousarray(soa, dtype=np.float64)
        out = np.empty_like(soa)
        self._check(self._fn("sweep_direction")(C.byref(d), C.c_int(direction), C.c_double(dt),
                                                dptr(soa), dptr(out)), "sweep")
        return out

    def apply_boundary_conditions(self, d: Desc, soa):
        out = np.array(soa, dtype=np.float64, copy=True)
        self._check(self._fn("apply_boundary_conditions")(C.byref(d), dptr(out)), "bc")
        return out

    def write_csv(self, d: Desc, soa, domain_min, domain_max, filename: str) -> None:
        """dim::write_csv (src/io/dim_write_csv.hpp:15-125) of a SoA field."""
        soa = np.ascontiguousarray(soa, dtype=np.float64)
        lo = np.zeros(3)
        hi = np.zeros(3)
        lo[:len(domain_min)] = domain_min
        hi[:len(domain_max)] = domain_max
        self._check(self._fn("write_csv")(C.byref(d), dptr(soa), dptr(lo), dptr(hi), os.fsencode(filename)),
                    "write_csv")

    def boundary_flux(self, d: Desc, soa) -> np.ndarray:
        """compute_dim_boundary_flux: nmat + dim + 2 values, laid out as totals."""
        soa = np.ascontiguousarray(soa, dtype=np.float64)
        out = np.zeros(d.nmat + d.dim + 2)
        self._check(self._fn("boundary_flux")(C.byref(d), dptr(soa), dptr(out)), "boundary_flux")
        return out

    # ---- record level (record-major arrays) ----
    def _records(self, name, d, inp, out_width, *extra):
        inp = np.ascontiguousarray(inp, dtype=np.float64)
        n = inp.shape[0]
        out = np.zeros((n, out_width))
        self._check(self._fn(name)(C.byref(d), C.c_int(n), *extra, dptr(inp), dptr(out)), name)
        return out

    def cons_to_prim(self, d, U):
        return self._records("cons_to_prim", d, U, 2 * d.nmat + d.dim + 1)

    def prim_to_cons(self, d, P):
        return self._records("prim_to_cons", d, P, 2 * d.nmat + d.dim)

    def repair_state(self, d, U):
        U = np.array(U, dtype=np.float64, copy=True, order="C")
        self._check(self._fn("repair_state")(C.byref(d), C.c_int(U.shape[0]), dptr(U)), "repair")
        return U

    def mixture_pressure(self, d, rec):
        return self._records("mixture_pressure", d, rec, 1)[:, 0]

    def mixture_sound_speed(self, d, rec):
        return self._records("mixture_sound_speed", d, rec, 1)[:, 0]

    def alpha_rhs(self, d, P):
        return self._records("alpha_rhs", d, P, d.nmat)

    def hllc(self, d, direction, UL, UR):
        UL = np.ascontiguousarray(UL, dtype=np.float64)
        UR = np.ascontiguousarray(UR, dtype=np.float64)
        n = UL.shape[0]
        out = np.zeros((n, d.nmat + d.dim + 2))
        self._check(self._fn("hllc")(C.byref(d), C.c_int(n), C.c_int(direction), dptr(UL),
                                     dptr(UR), dptr(out)), "hllc")
        return out

    def solve_line(self, d, direction, dt, dx, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        out = np.zeros_like(U)
        self._check(self._fn("solve_line")(C.byref(d), C.c_int(U.shape[0]), C.c_int(direction),
                                           C.c_double(dt), C.c_double(dx), dptr(U), dptr(out)),
                    "solve_line")
        return out


def port() -> Checker:
    return Checker("port")


def reference() -> Checker:
    return Checker("reference")


def reference_available() -> bool:
    return os.path.exists(REF_SO)


EREF_SO = os.path.join(HERE, "_ref", "libeulerref.so")


class EulerChecker:
    """The single-material Euler step: ``port`` (oracle/euler_oracle.c, in
    libdimoracle.so) or ``reference`` (oracle/_ref/libeulerref.so, the
    reference's own advance_one_step<DIM, MaterialEOS> with no level set).
    SoA state: rho, mom[0..dim-1], E per cell."""

    def __init__(self, kind: str = "port"):
        self.kind = kind
        path = PORT_SO if kind == "port" else EREF_SO
        if not os.path.exists(path):
            raise FileNotFoundError(f"{kind} Euler checker not built: {path}")
        self.lib = C.CDLL(path)
        self.prefix = "euler_oracle_" if kind == "port" else "eref_"

    def _fn(self, name):
        f = getattr(self.lib, self.prefix + name)
        f.restype = C.c_int
        return f

    def _check(self, rc, name):
        if rc != 0:
            msg = ""
            if self.kind == "reference":
                f = self.lib.eref_last_error
                f.restype = C.c_char_p
                msg = f().decode()
            raise RuntimeError(f"euler {self.kind}.{name}: status {rc} {msg}")

    def set_threads(self, n: int) -> None:
        if self.kind == "reference":
            self.lib.eref_set_threads(C.c_int(n))

    def advance(self, d: Desc, soa: np.ndarray, cfl: float, dt_max: float, nsteps: int = 1):
        soa = np.ascontiguousarray(soa, dtype=np.float64)
        out = np.empty_like(soa)
        dts = np.zeros(max(nsteps, 1))
        rc = self._fn("advance")(C.byref(d), dptr(soa), dptr(out), C.c_double(cfl), C.c_double(dt_max),
                                 C.c_int(nsteps), dptr(dts))
        self._check(rc, "advance")
        return out, dts[:nsteps]

    def compute_dt_cfl(self, d: Desc, soa: np.ndarray, cfl: float, dt_max: float) -> float:
        soa = np.ascontiguousarray(soa, dtype=np.float64)
        dt = C.c_double(0.0)
        rc = self._fn("compute_dt_cfl")(C.byref(d), dptr(soa), C.c_double(cfl), C.c_double(dt_max), C.byref(dt))
        self._check(rc, "compute_dt_cfl")
        return dt.value

    def hllc(self, d: Desc, direction: int, UL: np.ndarray, UR: np.ndarray) -> np.ndarray:
        """Rows of (rho, mom, E) face states -> rows of fluxes."""
        UL = np.ascontiguousarray(UL, dtype=np.float64)
        UR = np.ascontiguousarray(UR, dtype=np.float64)
        out = np.empty_like(UL)
        rc = self._fn("hllc")(C.byref(d), C.c_int(len(UL)), C.c_int(direction), dptr(UL), dptr(UR), dptr(out))
        self._check(rc, "hllc")
        return out

    # port only: the sub-calls of one step
    def sweep_direction(self, d: Desc, direction: int, dt: float, soa: np.ndarray, out: np.ndarray | None = None):
        soa = np.ascontiguousarray(soa, dtype=np.float64)
        out = np.zeros_like(soa) if out is None else np.ascontiguousarray(out, dtype=np.float64).copy()
        rc = self.lib.euler_oracle_sweep_direction(C.byref(d), C.c_int(direction), C.c_double(dt), dptr(soa),
                                                   dptr(out))
        self._check(rc, "sweep_direction")
        return out

    def apply_boundary_conditions(self, d: Desc, soa: np.ndarray) -> np.ndarray:
        out = np.ascontiguousarray(soa, dtype=np.float64).copy()
        self._check(self.lib.euler_oracle_apply_boundary_conditions(C.byref(d), dptr(out)), "boundary")
        return out
