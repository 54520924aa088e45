"""The single-material Euler step on the GPU (DIMGPU_MODEL_EULER): bit for
bit against the reference's golden vectors and the C restatement, through
the whole step, its sub-calls and the drop-in interface."""
from __future__ import annotations

import numpy as np
import pytest

from diffuse_vs_gfm_mms_b200 import abi, euler, workloads as W
from diffuse_vs_gfm_mms_b200.dim import DimGpuError, Session, compute_dt_cfl_noalloc
from helpers import bitwise_equal, desc_from_array, load, ndiff

pytestmark = pytest.mark.gpu

GOLD = load("euler_steps.npz")
CASES = sorted({k.rsplit("_desc", 1)[0] for k in GOLD.files if k.endswith("_desc") and not k.startswith("hllc_")})


@pytest.mark.parametrize("name", CASES)
def test_golden_steps(name):
    d = desc_from_array(GOLD[f"{name}_desc"])
    cfl, n = GOLD[f"{name}_meta"]
    with Session(d, GOLD[f"{name}_in"]) as s:
        dts = s.steps(int(n), float(cfl), 1e300)
        out = s.download()
    assert ndiff(out, GOLD[f"{name}_out"]) == 0
    assert bitwise_equal(dts, GOLD[f"{name}_dt"])


@pytest.mark.parametrize("gen,steps", [
    (lambda: W.euler_tube(seed=31, N=(4096,)), 40),
    (lambda: W.euler_blast(N=(300, 200), seed=32), 20),
    (lambda: W.euler_blast(N=(130, 3), seed=33, bc=["reflective", "nonreflective"]), 10),
    (lambda: W.euler_blast(N=(48, 40, 36), seed=34, bc=["reflective", "transmissive", "nonreflective"]), 8),
    (lambda: W.euler_blast(N=(64, 64), seed=35, material=("stiffened_gas", 4.4, 6e8)), 20),
    (lambda: W.euler_blast(N=(40, 44, 30), seed=36, time_update="unsplit"), 6),
])
def test_against_oracle(euler_port, gen, steps):
    d, U = gen()
    ref, rdts = euler_port.advance(d, U, 0.6, 1e300, steps)
    with Session(d, U) as s:
        dts = s.steps(steps, 0.6, 1e300)
        out = s.download()
    assert ndiff(out, ref) == 0 and bitwise_equal(dts, rdts)


def test_subcalls(euler_port):
    d, U = W.euler_blast(N=(70, 50), seed=37, bc=["reflective", "nonreflective"])
    with Session(d, U) as s:
        dt = s.compute_dt_cfl(0.6, 1e300)
        assert dt == euler_port.compute_dt_cfl(d, U, 0.6, 1e300)
        ref = U
        for direction in range(2):
            s.sweep_direction(direction, dt)
            ref = euler_port.sweep_direction(d, direction, dt, ref)
            assert ndiff(s.download(), ref) == 0
            s.apply_boundary_conditions()
            ref = euler_port.apply_boundary_conditions(d, ref)
            assert ndiff(s.download(), ref) == 0


def test_tiles_do_not_change_results():
    d, U = W.euler_blast(N=(90, 70, 20), seed=38)
    outs = []
    for tiles in ((128, 1, 64, 4), (64, 1, 32, 8), (256, 1, 128, 2)):
        with Session(d, U) as s:
            s.set_tile(0, tiles[0], tiles[1])
            s.set_tile(1, tiles[2], tiles[3])
            s.set_tile(2, tiles[2], tiles[3])
            s.steps(4, 0.6, 1e300)
            outs.append(s.download())
    assert ndiff(outs[0], outs[1]) == 0 and ndiff(outs[0], outs[2]) == 0


def test_drop_in_interface(euler_port):
    d, U = W.euler_blast(N=(40, 30), seed=39, bc=["reflective", "transmissive"])
    ctx = euler.SolverContext(N=(40, 30), dx=(d.dx[0], d.dx[1]), material_params=[("ideal_gas", 1.4, 0.0)],
                              cfl=0.6, dt_max=1e300, bc_lo=["reflective", "transmissive"],
                              bc_hi=["reflective", "transmissive"])
    ref, rdts = euler_port.advance(d, U, 0.6, 1e300, 3)
    cur = U
    dts = []
    for _ in range(3):
        r = euler.advance_one_step(cur, ctx)
        cur = r.U_new
        dts.append(r.dt)
    assert ndiff(cur, ref) == 0 and bitwise_equal(np.array(dts), rdts) and ctx.completed_steps == 3
    with pytest.raises(ValueError):
        euler.advance_one_step(U, euler.SolverContext(N=(40, 30), dx=(0.1, 0.1), phi_list=[np.zeros(1200)],
                                                      material_params=[("ideal_gas", 1.4, 0.0)]))


def test_noalloc_cfl_for_euler(euler_port):
    import torch
    d, U = W.euler_blast(N=(64, 48), seed=40)
    t = torch.from_numpy(U).cuda()
    dt = compute_dt_cfl_noalloc(d, t.data_ptr(), 0.6, 1e300)
    assert dt == euler_port.compute_dt_cfl(d, U, 0.6, 1e300)
    bad = U.copy()
    bad[0, 17] = np.nan
    t = torch.from_numpy(bad).cuda()
    with pytest.raises(DimGpuError) as e:
        compute_dt_cfl_noalloc(d, t.data_ptr(), 0.6, 1e300)
    assert e.value.status == abi.E_NONFINITE


def test_errors_are_statuses():
    d, U = W.euler_tube(seed=0, N=(2,))
    with pytest.raises(DimGpuError) as e:
        Session(d)
    assert e.value.status == abi.E_INVALID_ARG
    d = abi.make_desc(1, [10], [0.1], [("ideal_gas", 1.4, 0.0), ("ideal_gas", 1.6, 0.0)], model=abi.MODEL_EULER)
    with pytest.raises(DimGpuError):
        Session(d)
    d, U = W.euler_tube(seed=0, N=(50,))
    d.precision = abi.PRECISION_MIXED
    with pytest.raises(DimGpuError) as e:
        Session(d)
    assert e.value.status == abi.E_UNSUPPORTED
    d, U = W.euler_tube(seed=0, N=(50,))
    bad = U.copy()
    bad[0, 20] = np.nan
    with Session(d, bad) as s:
        with pytest.raises(DimGpuError) as e:
            s.step(0.5, 1e300)
        assert e.value.status == abi.E_NONFINITE
