"""The single-material Euler step on the CPU: the C restatement
(oracle/euler_oracle.c) against the reference's golden vectors and the
compiled reference, and the device arithmetic (csrc/euler_physics.h, built
for the host with g++) against the restatement, bit for bit."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from diffuse_vs_gfm_mms_b200 import abi, workloads as W
from diffuse_vs_gfm_mms_b200.abi import dptr
from helpers import bitwise_equal, desc_from_array, load, ndiff

GOLD = load("euler_steps.npz")
CASES = sorted({k.rsplit("_desc", 1)[0] for k in GOLD.files if k.endswith("_desc") and not k.startswith("hllc_")})


def _case(name):
    d = desc_from_array(GOLD[f"{name}_desc"])
    cfl, n = GOLD[f"{name}_meta"]
    return d, GOLD[f"{name}_in"], float(cfl), int(n)


@pytest.fixture(scope="module")
def host():
    from conftest import build_host_harness
    return C.CDLL(build_host_harness())


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_golden(euler_port, name):
    d, U, cfl, n = _case(name)
    out, dts = euler_port.advance(d, U, cfl, 1e300, n)
    assert ndiff(out, GOLD[f"{name}_out"]) == 0
    assert bitwise_equal(dts, GOLD[f"{name}_dt"])


@pytest.mark.parametrize("seed", [21, 22, 23])
def test_oracle_matches_reference_on_fresh_inputs(euler_port, euler_reference, seed):
    for d, U in (W.euler_tube(seed=seed, N=(257,)), W.euler_blast(N=(29, 31), seed=seed),
                 W.euler_blast(N=(9, 11, 7), seed=seed, bc=["reflective", "nonreflective", "transmissive"])):
        a, da = euler_port.advance(d, U, 0.7, 1e300, 12)
        b, db = euler_reference.advance(d, U, 0.7, 1e300, 12)
        assert ndiff(a, b) == 0 and bitwise_equal(da, db)
    d, U = W.euler_blast(N=(24, 20), seed=seed)
    for dt_max in (1e-7, 3e-6):
        a, da = euler_port.advance(d, U, 0.7, dt_max, 5)
        b, db = euler_reference.advance(d, U, 0.7, dt_max, 5)
        assert ndiff(a, b) == 0 and bitwise_equal(da, db)


@pytest.mark.parametrize("tag", ["ideal", "water"])
def test_hllc_records(euler_port, host, tag):
    d = desc_from_array(GOLD[f"hllc_{tag}_desc"])
    UL, UR = GOLD[f"hllc_{tag}_UL"], GOLD[f"hllc_{tag}_UR"]
    for axis in (0, 1):
        want = GOLD[f"hllc_{tag}_F{axis}"]
        assert bitwise_equal(euler_port.hllc(d, axis, UL, UR), want)
        got = np.empty_like(UL)
        assert host.host_euler_hllc(C.byref(d), C.c_int(len(UL)), C.c_int(axis), dptr(UL), dptr(UR), dptr(got)) == 0
        assert bitwise_equal(got, want)


def test_hllc_reports_where_the_reference_throws(euler_port, host):
    d = abi.make_desc(1, [4], [0.1], [("ideal_gas", 1.4, 0.0)], model=abi.MODEL_EULER)
    UL = np.array([[np.nan, 0.0, 2.5]])
    UR = np.array([[1.0, 0.0, 2.5]])
    with pytest.raises(RuntimeError):
        euler_port.hllc(d, 0, UL, UR)
    out = np.empty_like(UL)
    assert host.host_euler_hllc(C.byref(d), 1, 0, dptr(UL), dptr(UR), dptr(out)) == abi.E_NONFINITE


@pytest.mark.parametrize("name", CASES)
def test_device_arithmetic_sweeps(euler_port, host, name):
    """Every axis of every golden input, both end-cell conventions."""
    d, U, cfl, _ = _case(name)
    dt = euler_port.compute_dt_cfl(d, U, cfl, 1e300)
    for direction in range(d.dim):
        for ends_copy in (0, 1):
            want = euler_port.sweep_direction(d, direction, dt, U, out=U if ends_copy else None)
            got = np.empty_like(U)
            rc = host.host_euler_sweep_direction(C.byref(d), direction, C.c_double(dt), dptr(U), dptr(got), ends_copy)
            assert rc == 0
            assert ndiff(got, want) == 0, (name, direction, ends_copy)


def test_restatement_rejects_what_the_reference_rejects(euler_port):
    d, U = W.euler_tube(seed=0, N=(2,))
    with pytest.raises(RuntimeError):
        euler_port.advance(d, U, 0.5, 1e300, 1)   # reconstruct_line_interfaces needs 3 cells
    d, U = W.euler_tube(seed=0, N=(10,))
    with pytest.raises(RuntimeError):
        euler_port.advance(d, U, -0.5, 1e300, 1)
