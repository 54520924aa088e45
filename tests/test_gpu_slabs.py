"""One grid decomposed into slabs along its slowest axis (dimgpu_slabs_*):
every step must give the same dt and the same state, bit for bit, as one
Session on the whole grid (which the oracle pins), however the planes are
split.  The slabs share cuda:0 here, so the ghost exchange runs as device
copies; across GPUs the same code issues peer copies of the same bytes."""
from __future__ import annotations

import numpy as np
import pytest

from diffuse_vs_gfm_mms_b200 import abi, workloads as W
from diffuse_vs_gfm_mms_b200.dim import Session, Slabs
from helpers import bitwise_equal, ndiff

pytestmark = pytest.mark.gpu


def _alone(d, U, steps, cfl):
    with Session(d, U) as s:
        dts = s.steps(steps, cfl, 1e300)
        return s.download(), dts


def _slabs(d, U, steps, cfl, nslabs):
    with Slabs(d, [0] * nslabs, U) as L:
        dts = L.steps(steps, cfl, 1e300)
        return L.download(), dts


def _cases():
    cases = []
    d, U = W.single_bubble_2d((96, 64), seed=3)
    cases.append(("bubble 96x64", d, U, 25, 0.6, (2, 4, 7)))
    d, U = W.riemann(seed=5, N=(16, 200), axis=1)
    d.bc_lo[1] = abi.BC_REFLECTIVE
    d.bc_hi[1] = abi.BC_REFLECTIVE
    cases.append(("riemann along y 16x200 reflective", d, U, 40, 0.7, (2, 3, 5)))
    d, U = W.riemann(seed=6, N=(10, 61), axis=1, position=0.37)
    d.bc_hi[1] = abi.BC_NONREFLECTIVE
    cases.append(("riemann along y 10x61 uneven", d, U, 30, 0.5, (4, 20)))
    d, U = W.single_bubble_2d((40, 9), seed=8)
    d.lambda_model = abi.LAMBDA_ALLAIRE
    cases.append(("bubble 40x9, three planes a slab", d, U, 20, 0.5, (3,)))
    d, U = W.bubble_cloud_3d(N=(24, 20, 18), nbubbles=3)
    cases.append(("cloud 24x20x18", d, U, 12, 0.6, (2, 3, 6)))
    d, U = W.riemann(seed=9, N=(6, 5, 40), axis=2, bc=abi.BC_TRANSMISSIVE)
    cases.append(("riemann along z 6x5x40", d, U, 25, 0.6, (4,)))
    return cases


CASES = _cases()


@pytest.mark.parametrize("name,d,U,steps,cfl,splits", CASES, ids=[c[0] for c in CASES])
def test_slabs_match_one_grid(name, d, U, steps, cfl, splits):
    ref, rdts = _alone(d, U, steps, cfl)
    for n in splits:
        out, dts = _slabs(d, U, steps, cfl, n)
        assert bitwise_equal(dts, rdts), (name, n)
        assert ndiff(out, ref) == 0, (name, n, ndiff(out, ref))


def test_slabs_match_the_oracle(port):
    d, U = W.riemann(seed=11, N=(8, 90), axis=1)
    ref, rdts = port.advance(d, U, 0.6, 1e300, 20)
    out, dts = _slabs(d, U, 20, 0.6, 3)
    assert ndiff(out, ref) == 0 and bitwise_equal(dts, rdts)


def test_mixed_slabs_match_one_mixed_grid():
    d, U = W.shock_bubble_2d((128, 64))
    d.precision = abi.PRECISION_MIXED
    ref, rdts = _alone(d, U, 30, 0.5)
    out, dts = _slabs(d, U, 30, 0.5, 4)
    assert bitwise_equal(dts, rdts) and ndiff(out, ref) == 0


def test_upload_between_runs_restarts_the_grid():
    d, U = W.single_bubble_2d((32, 48), seed=2)
    ref, rdts = _alone(d, U, 10, 0.6)
    with Slabs(d, [0, 0, 0]) as L:
        L.upload(U)
        L.steps(7, 0.6, 1e300)
        L.upload(U)
        dts = L.steps(10, 0.6, 1e300)
        assert bitwise_equal(dts, rdts) and ndiff(L.download(), ref) == 0
