"""The fused sweep schedule (one kernel per sweep, every stage in a
shared-memory tile) with its input tile staged by TMA: where the layout
allows a tensor map (even N[0] and cell count, even W for y / z sweeps) the
whole tile with its 3-cell halo arrives in one cp.async.bulk.tensor copy;
elsewhere each thread loads its own cell.  Either way the results are the
oracle's, bit for bit, for every tile shape and at ragged tile edges."""
from __future__ import annotations

import pytest

from diffuse_vs_gfm_mms_b200 import abi, workloads as W
from diffuse_vs_gfm_mms_b200.dim import Session
from helpers import bitwise_equal, ndiff

pytestmark = pytest.mark.gpu

TILES = {
    "x128x1_y64x4": [(128, 1), (64, 4), (64, 4)],
    "x64x4_y32x8": [(64, 4), (32, 8), (32, 8)],
    "x32x8_y16x16": [(32, 8), (16, 16), (16, 16)],
    "x128x2_y64x1_odd_w": [(128, 2), (64, 1), (128, 1)],
}

CASES = {
    "1d_even": lambda: W.riemann(seed=3, N=(300,)),
    "1d_odd": lambda: W.riemann(seed=4, N=(301,)),
    "2d_even": lambda: W.shock_bubble_2d(N=(130, 70)),
    "2d_odd": lambda: W.riemann(seed=5, N=(33, 17), axis=1),
    "3d_even": lambda: W.bubble_cloud_3d(N=(40, 36, 30), nbubbles=4),
    "3d_mixed_parity": lambda: W.bubble_cloud_3d(N=(24, 21, 18), nbubbles=2),
}


@pytest.mark.parametrize("tiles", list(TILES))
@pytest.mark.parametrize("case", list(CASES))
def test_fused_schedule_matches_oracle(port, case, tiles):
    d, U = CASES[case]()
    cfl = 0.6 if d.dim == 3 else 0.7
    with Session(d, U) as s:
        for direction in range(d.dim):
            s.set_schedule(direction, abi.SCHEDULE_FUSED)
            T, Wd = TILES[tiles][direction]
            s.set_tile(direction, T, Wd)
        dts = s.steps(4, cfl, 1e300)
        out = s.download()
    ref, rdts = port.advance(d, U, cfl, 1e300, 4)
    assert ndiff(out, ref) == 0 and bitwise_equal(dts, rdts)
