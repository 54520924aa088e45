"""The allocation-free CFL entry point, dimgpu_compute_dt_cfl_noalloc.

Who it is for: host programs that manage all of the GPU's memory themselves —
a serving process that has reserved the HBM budget for its resident solves,
or a solver that hands out device buffers from its own pool.  They cannot let
a library call cudaMalloc in the middle of a time loop: the memory may not be
available, and cudaMalloc / cudaFree synchronise the whole device.  So the
state stays in memory the caller owns (here a torch tensor) and the entry
point uses only the library's own static scratch array.

The check: two calls in a row, on two different states, must return exactly
the dt that the ordinary session entry point (dimgpu_compute_dt_cfl) returns
for the same state — the same bit-for-bit bar as the other GPU tests.  This
file is collected last so a failure here cannot hide the other results.
"""
from __future__ import annotations

import pytest

from diffuse_vs_gfm_mms_b200 import abi, workloads as W
from diffuse_vs_gfm_mms_b200.dim import DimGpuError, Session, compute_dt_cfl_noalloc

pytestmark = pytest.mark.gpu


def _states(N, cfl):
    """Two different states of one grid and their dts from the session API."""
    d, U = W.shock_bubble_2d(N=N)
    with Session(d, U) as s:
        s.steps(3, cfl, 1e300)
        U1, dt1 = s.download(), s.compute_dt_cfl(cfl, 1e300)
        s.steps(2, cfl, 1e300)
        U2, dt2 = s.download(), s.compute_dt_cfl(cfl, 1e300)
    return d, (U1, dt1), (U2, dt2)


@pytest.mark.parametrize("N", [(256, 128), (2048, 2048)])
def test_two_calls_match_the_session_entry_point(N):
    import torch

    d, (U1, dt1), (U2, dt2) = _states(N, 0.8)
    assert dt1 != dt2
    buf = torch.from_numpy(U1.copy()).cuda()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream().cuda_stream
    got1 = compute_dt_cfl_noalloc(d, buf.data_ptr(), 0.8, 1e300, stream)
    buf.copy_(torch.from_numpy(U2))
    torch.cuda.synchronize()
    got2 = compute_dt_cfl_noalloc(d, buf.data_ptr(), 0.8, 1e300, stream)
    assert got1 == dt1
    assert got2 == dt2
    assert compute_dt_cfl_noalloc(d, buf.data_ptr(), 0.8, 1e-9, stream) == 1e-9


def test_grids_beyond_the_limit_are_refused():
    import torch

    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    d = abi.make_desc(2, (2049, 2048), (1e-3, 1e-3), [("ideal_gas", 1.4, 0.0), ("ideal_gas", 1.67, 0.0)])
    with pytest.raises(DimGpuError) as e:
        compute_dt_cfl_noalloc(d, buf.data_ptr(), 0.8, 1e300)
    assert e.value.status == abi.E_INVALID_ARG
    assert "4194304" in str(e.value)
