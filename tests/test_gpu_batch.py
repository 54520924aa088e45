"""The batched form (dimgpu_batch_*): every instance of a batch must end bit
for bit where the same grid ends when run alone through a Session, and where
the CPU oracle ends, whatever else shares the batch and whenever instances
join or leave it."""
from __future__ import annotations

import numpy as np
import pytest

from diffuse_vs_gfm_mms_b200 import abi, workloads as W
from diffuse_vs_gfm_mms_b200.batch import Batch
from diffuse_vs_gfm_mms_b200.dim import DimGpuError, Session
from helpers import bitwise_equal, ndiff

pytestmark = pytest.mark.gpu


def _alone(d, U, steps, cfl):
    with Session(d, U) as s:
        dts = s.steps(steps, cfl, 1e300)
        return s.download(), dts


def _cases_2d():
    cases = []
    shapes = [(64, 80), (130, 70), (4, 200), (200, 4), (97, 33), (256, 64), (5, 5), (40, 1), (1, 40)]
    for k, N in enumerate(shapes):
        if k % 2:
            d, U = W.single_bubble_2d(N, seed=k) if min(N) > 1 else W.riemann(seed=k, N=N, axis=0 if N[0] > 1 else 1)
        else:
            d, U = W.riemann(seed=k, N=N, axis=k % 2 if N[k % 2] > 1 else 1 - k % 2)
        if k == 2:
            d.bc_lo[0] = abi.BC_REFLECTIVE
        if k == 4:
            d.bc_hi[1] = abi.BC_NONREFLECTIVE
        if k == 6:
            d.lambda_model = abi.LAMBDA_ALLAIRE
        cases.append((d, U, 3 + 5 * k, 0.5 + 0.04 * k))
    return cases


def test_batch_matches_alone_and_oracle(port):
    cases = _cases_2d()
    with Batch(2, 2) as b:
        ids = [b.add(d, U, steps, cfl) for d, U, steps, cfl in cases]
        for n in (5, 11, 2, 40):          # graph replays and single steps
            b.run(n)
        for iid, (d, U, steps, cfl) in zip(ids, cases):
            assert b.status(iid) == (steps, 0)
            out, dts = b.download(iid)
            ref, rdts = _alone(d, U, steps, cfl)
            assert ndiff(out, ref) == 0 and bitwise_equal(dts, rdts), (iid, d.shape())
        d, U, steps, cfl = cases[1]
        ref, rdts = port.advance(d, U, cfl, 1e300, steps)
        out, dts = b.download(ids[1])
        assert ndiff(out, ref) == 0 and bitwise_equal(dts, rdts)


def test_join_and_leave_mid_run():
    cases = _cases_2d()
    with Batch(2, 2) as b:
        first = [b.add(d, U, steps, cfl) for d, U, steps, cfl in cases[:4]]
        b.run(9)
        b.remove(first[0])                # finished (3 steps) and leaves
        late = [b.add(d, U, steps, cfl) for d, U, steps, cfl in cases[4:]]
        b.run(17)
        b.remove(first[1])
        b.run(30)
        for iid, (d, U, steps, cfl) in zip(first[2:] + late, cases[2:4] + cases[4:]):
            out, dts = b.download(iid)
            ref, rdts = _alone(d, U, steps, cfl)
            assert ndiff(out, ref) == 0 and bitwise_equal(dts, rdts)


@pytest.mark.parametrize("dim", [1, 3])
def test_other_dimensions(port, dim):
    if dim == 1:
        cases = [W.riemann(seed=s, N=(n,)) for s, n in ((1, 300), (2, 1000), (3, 57))]
    else:
        cases = [W.bubble_cloud_3d(N=(12, 10, 8), nbubbles=2), W.riemann(seed=4, N=(9, 6, 20), axis=2),
                 W.riemann(seed=5, N=(16, 1, 7), axis=0)]
    with Batch(2, dim) as b:
        ids = [b.add(d, U, 12, 0.6) for d, U in cases]
        b.run(12)
        for iid, (d, U) in zip(ids, cases):
            out, dts = b.download(iid)
            ref, rdts = port.advance(d, U, 0.6, 1e300, 12)
            assert ndiff(out, ref) == 0 and bitwise_equal(dts, rdts)


def test_same_alone_and_in_a_mix():
    """One grid's result does not depend on its batch-mates."""
    d0, U0 = W.single_bubble_2d((120, 90), seed=42)
    with Batch(2, 2) as b:
        i = b.add(d0, U0, 25, 0.7)
        b.run(25)
        alone, dt_alone = b.download(i)
    mates = _cases_2d()
    with Batch(2, 2) as b:
        ids = [b.add(d, U, steps, cfl) for d, U, steps, cfl in mates[:5]]
        i = b.add(d0, U0, 25, 0.7)
        ids += [b.add(d, U, steps, cfl) for d, U, steps, cfl in mates[5:]]
        b.run(7)
        b.run(30)
        mixed, dt_mixed = b.download(i)
    assert ndiff(alone, mixed) == 0 and bitwise_equal(dt_alone, dt_mixed)


def test_batch_rejects_what_it_does_not_run():
    with Batch(2, 2) as b:
        d, U = W.riemann(seed=1, N=(3, 10))
        with pytest.raises(DimGpuError):
            b.add(d, U, 5, 0.5)
        d, U = W.riemann(seed=1, N=(10, 10))
        d.time_update = abi.TIME_UNSPLIT
        with pytest.raises(DimGpuError):
            b.add(d, U, 5, 0.5)
        d3, U3 = W.riemann(seed=1, N=(10,))
        with pytest.raises(DimGpuError):
            b.add(d3, U3, 5, 0.5)
        assert len(b) == 0


def test_mixed_precision_instances(port):
    """Mixed-precision instances in a batch (alone and beside FP64 ones) end
    bit for bit where a mixed-precision Session ends."""
    cases = _cases_2d()[:6]
    mixed = []
    for k, (d, U, steps, cfl) in enumerate(cases):
        dm = d.copy()
        if k % 2 == 0:
            dm.precision = abi.PRECISION_MIXED
        mixed.append((dm, U, steps, cfl))
    with Batch(2, 2) as b:
        ids = [b.add(d, U, steps, cfl) for d, U, steps, cfl in mixed]
        b.run(40)
        for iid, (d, U, steps, cfl) in zip(ids, mixed):
            out, dts = b.download(iid)
            ref, rdts = _alone(d, U, steps, cfl)
            assert ndiff(out, ref) == 0 and bitwise_equal(dts, rdts), (iid, d.precision)


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_graphs_dropped_when_the_scratch_regrows_in_place(precision):
    """A leaves, a larger instance joins, runs from a captured graph, then a
    third joins and the scratch regrows: the regrown scratch can come back at
    the old address, so the captured graph (which bakes in the scratch
    capacity that strides every record) must be dropped on the capacity
    change too.  Every instance must still match its solve alone."""
    from diffuse_vs_gfm_mms_b200 import serve
    reqs = {r.rid: r for r in serve.make_requests(10, 200.0, seed=3, steps_range=(20, 60), n1d_range=(64, 512),
                                                  side2d_range=(16, 64))}
    for r in reqs.values():
        r.desc.precision = precision
    A, B, C = reqs[0], reqs[2], reqs[4]
    with Batch(2, 2) as b:
        ia = b.add(A.desc, A.U, A.steps, 0.6)
        for _ in range(4):
            b.run(8)
        b.remove(ia)
        ib = b.add(B.desc, B.U, B.steps, 0.6)
        for _ in range(3):
            b.run(8)
        ic = b.add(C.desc, C.U, C.steps, 0.6)
        b.run(8)
        for iid, r in ((ib, B), (ic, C)):
            done, _ = b.status(iid)
            out, dts = b.download(iid)
            ref, rdts = _alone(r.desc, r.U, done, 0.6)
            assert ndiff(out, ref) == 0 and bitwise_equal(dts, rdts), r.rid


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_arena_mode_joins_and_leaves_without_allocating(dim):
    """dimgpu_batch_reserve: after the one reservation, instances join and
    leave mid-run with no change of the device's free memory, instances that
    finished early stop being stepped, a full arena refuses with E_OOM, and
    every result is the instance's own (bit for bit as alone)."""
    import torch

    if dim == 1:
        cases = [W.riemann(seed=k, N=(60 + 37 * k,)) for k in range(6)]
    elif dim == 2:
        cases = [W.single_bubble_2d((20 + 7 * k, 30 + 5 * k), seed=k) if k % 2 else
                 W.riemann(seed=k, N=(24 + 9 * k, 18 + 4 * k), axis=k % 2) for k in range(6)]
    else:
        cases = [W.bubble_cloud_3d(N=(10 + k, 9 + 2 * k, 8 + k), nbubbles=1 + k % 2, seed=k) for k in range(6)]
    steps = [7, 19, 3, 26, 11, 16]
    cfl = 0.5
    total = sum(d.ncell for d, _ in cases)
    with Batch(2, dim) as b:
        b.reserve(max_cells=total // 2 + 64, max_instances=4, max_steps=200)
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        ids = {}
        for k in (0, 1):
            ids[k] = b.add(cases[k][0], cases[k][1], steps[k], cfl)
        b.run(5)
        for k in (2, 3):
            ids[k] = b.add(cases[k][0], cases[k][1], steps[k], cfl)
        b.run(9)                                   # instances 0 and 2 finish inside this run
        outs = {}
        for k in (0, 2):
            outs[k] = b.download(ids[k])
            b.remove(ids.pop(k))
        for k in (4, 5):
            try:
                ids[k] = b.add(cases[k][0], cases[k][1], steps[k], cfl)
            except DimGpuError as e:
                assert e.status == abi.E_OOM
        b.run(40)
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0
        for k, iid in ids.items():
            outs[k] = b.download(iid)
        used, _ = b.arena_used()
        assert used == sum(cases[k][0].ncell for k in ids)
    for k, (out, dts) in outs.items():
        d, U = cases[k]
        ref, rdts = _alone(d, U, steps[k], cfl)
        assert ndiff(out, ref) == 0 and bitwise_equal(dts, rdts), k
