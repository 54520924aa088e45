"""The serving loop: admission against an HBM budget and a slot cap,
continuous batching of requests that arrive while others run, retirement
that frees room for the queue — and every result the same as the request
run alone."""
from __future__ import annotations

import numpy as np
import pytest

from diffuse_vs_gfm_mms_b200 import abi, serve
from diffuse_vs_gfm_mms_b200.dim import DimGpuError, Session
from helpers import bitwise_equal, ndiff

pytestmark = pytest.mark.gpu


def _small_requests(n=10, rate=200.0, seed=3):
    return serve.make_requests(n, rate, seed=seed, steps_range=(20, 60), n1d_range=(64, 512),
                               side2d_range=(16, 64))


def _alone(r):
    with Session(r.desc, r.U) as s:
        dts = s.steps(r.steps, r.cfl, r.dt_max)
        return s.download(), dts


def test_results_same_alone_and_in_the_mix():
    reqs = _small_requests()
    budget = 4.0 * max(serve.footprint_bytes(r.desc, r.steps) for r in reqs)
    with serve.Server(hbm_budget_bytes=budget, max_slots=3, quantum=8) as srv:
        stats = srv.serve(reqs)
    assert len(stats.results) == len(reqs)
    assert stats.peak_bytes <= budget
    assert stats.peak_slots > 1                 # work overlapped on the device
    by_id = {r.rid: r for r in reqs}
    for res in stats.results:
        U, dts = _alone(by_id[res.rid])
        assert ndiff(res.U, U) == 0 and bitwise_equal(res.dts, dts), res.rid
        assert res.finished >= res.admitted >= 0.0
    p50, p99 = stats.latency_percentiles()
    assert 0 < p50 <= p99


def test_cancel_queued_and_running():
    """One slot: the first request runs (long), the others queue; cancelling
    the running one and a queued one leaves the rest to finish."""
    import time

    reqs = _small_requests(4, rate=0.0, seed=5)
    reqs[0].steps = 2000
    with serve.Server(max_slots=1, quantum=4, hbm_budget_bytes=4e9) as srv:
        for r in reqs:
            srv.submit(r)
        t0 = time.time()
        while srv.state(reqs[0].rid) != abi.REQ_RUNNING and time.time() - t0 < 10:
            time.sleep(0.001)
        assert srv.cancel(reqs[0].rid)          # running
        assert srv.cancel(reqs[-1].rid)         # still queued
        assert not srv.cancel(12345)
        srv.drain()
        assert srv.collect(reqs[0].rid)[0] == abi.REQ_CANCELLED
        assert srv.collect(reqs[-1].rid)[0] == abi.REQ_CANCELLED
        for r in reqs[1:-1]:
            st, U, dts, lat = srv.collect(r.rid)
            assert st == abi.REQ_DONE and lat > 0
            Ua, dta = _alone(r)
            assert ndiff(U, Ua) == 0 and bitwise_equal(dts, dta)
        c = srv.counters()
        assert c.cancelled == 2 and c.completed == 2 and c.resident == 0


def test_admission_waits_for_room_and_never_exceeds_the_budget():
    """A budget with room for about two of the requests at a time: every
    request still finishes, the arena is never over-committed, and the
    results are the solves' own."""
    reqs = _small_requests(8, rate=0.0, seed=9)
    one = max(serve.footprint_bytes(r.desc, 0) for r in reqs)
    budget = 2.2 * one / 0.4
    with serve.Server(hbm_budget_bytes=budget, max_slots=16, quantum=8, dim_share=(0.4, 0.6, 0.0),
                      solo_share=0.0, solo_slots=0) as srv:
        stats = srv.serve(reqs)
    assert len(stats.results) == len(reqs)
    assert stats.peak_bytes <= budget
    by_id = {r.rid: r for r in reqs}
    for res in stats.results:
        U, dts = _alone(by_id[res.rid])
        assert ndiff(res.U, U) == 0 and bitwise_equal(res.dts, dts), res.rid


def test_oversized_request_is_refused_at_submission():
    r = _small_requests(1, rate=0.0, seed=2)[0]
    with serve.Server(hbm_budget_bytes=1e3) as srv:
        with pytest.raises(DimGpuError) as e:
            srv.submit(r)
        assert e.value.status == abi.E_OOM


def test_solo_lanes_beside_batch_lanes():
    """Requests of at least solo_min_cells cells run alone on solo lanes
    (session shells over one arena), the rest in the batch lanes, all at
    once; every result is the solve's own.  The solo arena has room for
    about one big solve at a time, so the big ones also queue for room."""
    reqs = _small_requests(12, rate=0.0, seed=11)
    cut = sorted(r.desc.ncell for r in reqs)[len(reqs) // 2]
    big = [r for r in reqs if r.desc.ncell >= cut]
    small = [r for r in reqs if r.desc.ncell < cut]
    assert big and small
    one_big = max(serve.footprint_bytes(r.desc, 0) for r in big)
    budget = 64.0 * max(serve.footprint_bytes(r.desc, r.steps) for r in reqs)
    solo_share = 1.5 * one_big / budget
    with serve.Server(hbm_budget_bytes=budget, max_slots=16, quantum=8, dim_share=(0.2, 0.4, 0.0),
                      solo_min_cells=cut, solo_share=solo_share, solo_slots=2) as srv:
        stats = srv.serve(reqs)
    assert len(stats.results) == len(reqs)
    assert stats.peak_bytes <= budget
    by_id = {r.rid: r for r in reqs}
    for res in stats.results:
        U, dts = _alone(by_id[res.rid])
        assert ndiff(res.U, U) == 0 and bitwise_equal(res.dts, dts), res.rid


def test_cancel_a_running_solo_solve():
    import time

    reqs = _small_requests(3, rate=0.0, seed=13)
    reqs[0].steps = 3000
    with serve.Server(max_slots=4, quantum=4, hbm_budget_bytes=4e9, solo_min_cells=1, solo_slots=1) as srv:
        for r in reqs:
            srv.submit(r)
        t0 = time.time()
        while srv.state(reqs[0].rid) != abi.REQ_RUNNING and time.time() - t0 < 10:
            time.sleep(0.001)
        assert srv.cancel(reqs[0].rid)
        srv.drain()
        assert srv.collect(reqs[0].rid)[0] == abi.REQ_CANCELLED
        for r in reqs[1:]:
            st, U, dts, lat = srv.collect(r.rid)
            assert st == abi.REQ_DONE
            Ua, dta = _alone(r)
            assert ndiff(U, Ua) == 0 and bitwise_equal(dts, dta)
        c = srv.counters()
        assert c.cancelled == 1 and c.completed == 2 and c.resident == 0
