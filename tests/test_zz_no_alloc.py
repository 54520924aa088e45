"""The allocation-free CFL entry point, dimgpu_compute_dt_cfl_noalloc.

Who it is for: host programs that manage all of the GPU's memory themselves —
a serving process that has reserved the HBM budget for its resident solves,
or a solver that hands out device buffers from its own pool.  They cannot let
a library call cudaMalloc in the middle of a time loop: the memory may not be
available, and cudaMalloc / cudaFree synchronise the whole device.  So the
state stays in memory the caller owns (here a torch tensor) and the entry
point uses only the library's own static scratch array.

The checks: two calls in a row, on two different states, must return exactly
the dt that the ordinary session entry point (dimgpu_compute_dt_cfl) returns
for the same state — the same bit-for-bit bar as the other GPU tests — for
both precisions, 1D to 3D and one to four materials; a call made after the
first one on a device leaves the device's free memory unchanged; grids
beyond the limit are refused.  This file is collected last so a failure here
cannot hide the other results.
"""
from __future__ import annotations

import numpy as np
import pytest

from diffuse_vs_gfm_mms_b200 import abi, workloads as W
from diffuse_vs_gfm_mms_b200.dim import DimGpuError, Session, compute_dt_cfl_noalloc

pytestmark = pytest.mark.gpu


def _two_states(d, U, cfl):
    """Two different states of one grid and their dts from the session API."""
    with Session(d, U) as s:
        s.steps(3, cfl, 1e300)
        U1, dt1 = s.download(), s.compute_dt_cfl(cfl, 1e300)
        s.steps(2, cfl, 1e300)
        U2, dt2 = s.download(), s.compute_dt_cfl(cfl, 1e300)
    return (U1, dt1), (U2, dt2)


def _random_field(mats, N, seed):
    d = abi.make_desc(len(N), N, [1.0 / n for n in N], mats)
    U = W.random_states(d, d.ncell, seed=seed, edge_fraction=0.0).T.copy()
    return d, U


CASES = {
    "shock_bubble_256x128": lambda: W.shock_bubble_2d(N=(256, 128)),
    "shock_bubble_2048sq_at_limit": lambda: W.shock_bubble_2d(N=(2048, 2048)),
    "riemann_1d": lambda: W.riemann(seed=2, N=(1000,)),
    "cloud_3d": lambda: W.bubble_cloud_3d(N=(40, 36, 32), nbubbles=4),
    "one_material_2d": lambda: _random_field([("stiffened_gas", 4.4, 6e8)], (48, 40), 7),
    "three_materials_3d": lambda: _random_field(
        [("ideal_gas", 1.6, 0.0), ("stiffened_gas", 2.1, 3e8), ("ideal_gas", 1.4, 0.0)], (20, 18, 16), 8),
    "four_materials_2d": lambda: _random_field(
        [("stiffened_gas", 1.9, 5e8), ("ideal_gas", 1.3, 0.0), ("stiffened_gas", 5.5, 2e8), ("ideal_gas", 2.0, 0.0)],
        (40, 30), 9),
}


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
@pytest.mark.parametrize("case", list(CASES))
def test_two_calls_match_the_session_entry_point(case, precision):
    import torch

    d, U = CASES[case]()
    d.precision = precision
    cfl = 0.4 if "material" in case else (0.6 if d.dim == 3 else 0.8)
    (U1, dt1), (U2, dt2) = _two_states(d, U, cfl)
    assert not np.array_equal(U1, U2)
    buf = torch.from_numpy(U1.copy()).cuda()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream().cuda_stream
    got1 = compute_dt_cfl_noalloc(d, buf.data_ptr(), cfl, 1e300, stream)
    buf.copy_(torch.from_numpy(U2))
    torch.cuda.synchronize()
    got2 = compute_dt_cfl_noalloc(d, buf.data_ptr(), cfl, 1e300, stream)
    assert got1 == dt1
    assert got2 == dt2
    assert compute_dt_cfl_noalloc(d, buf.data_ptr(), cfl, 1e-9, stream) == 1e-9


def test_calls_after_the_first_leave_free_memory_unchanged():
    """After the first call on a device (which only looks up the static
    array's address), a call takes no device memory: cudaMemGetInfo reports
    the same free bytes before and after it."""
    import torch

    d, U = W.shock_bubble_2d(N=(512, 256))
    buf = torch.from_numpy(U).cuda()
    torch.cuda.synchronize()
    compute_dt_cfl_noalloc(d, buf.data_ptr(), 0.8, 1e300)
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        compute_dt_cfl_noalloc(d, buf.data_ptr(), 0.8, 1e300)
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before


def test_grids_beyond_the_limit_are_refused():
    import torch

    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    d = abi.make_desc(2, (2049, 2048), (1e-3, 1e-3), [("ideal_gas", 1.4, 0.0), ("ideal_gas", 1.67, 0.0)])
    with pytest.raises(DimGpuError) as e:
        compute_dt_cfl_noalloc(d, buf.data_ptr(), 0.8, 1e300)
    assert e.value.status == abi.E_INVALID_ARG
    assert "4194304" in str(e.value)
    # axes whose product overflows a 64-bit integer are refused, not wrapped
    d = abi.make_desc(3, (2**31 - 1, 2**31 - 1, 2**31 - 1), (1e-3, 1e-3, 1e-3),
                      [("ideal_gas", 1.4, 0.0), ("ideal_gas", 1.67, 0.0)])
    with pytest.raises(DimGpuError) as e:
        compute_dt_cfl_noalloc(d, buf.data_ptr(), 0.8, 1e300)
    assert e.value.status == abi.E_INVALID_ARG


def test_descriptors_the_session_refuses_are_refused():
    """Same descriptor checks as dimgpu_create: an unknown precision, an
    unknown time update, or a mixed-precision Euler descriptor."""
    import torch

    buf = torch.zeros(64, dtype=torch.float64, device="cuda")
    d = abi.make_desc(1, (8,), (0.1,), [("ideal_gas", 1.4, 0.0), ("ideal_gas", 1.67, 0.0)])
    d.precision = 7
    with pytest.raises(DimGpuError) as e:
        compute_dt_cfl_noalloc(d, buf.data_ptr(), 0.8, 1e300)
    assert e.value.status == abi.E_INVALID_ARG
    d.precision = abi.PRECISION_FP64
    d.time_update = 5
    with pytest.raises(DimGpuError) as e:
        compute_dt_cfl_noalloc(d, buf.data_ptr(), 0.8, 1e300)
    assert e.value.status == abi.E_INVALID_ARG
    d = abi.make_desc(1, (8,), (0.1,), [("ideal_gas", 1.4, 0.0)], model=abi.MODEL_EULER)
    d.precision = abi.PRECISION_MIXED
    with pytest.raises(DimGpuError) as e:
        compute_dt_cfl_noalloc(d, buf.data_ptr(), 0.8, 1e300)
    assert e.value.status == abi.E_UNSUPPORTED
