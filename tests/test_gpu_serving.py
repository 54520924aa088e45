"""The serving loop: admission against an HBM budget and a slot cap,
continuous batching of requests that arrive while others run, retirement
that frees room for the queue — and every result the same as the request
run alone."""
from __future__ import annotations

import numpy as np
import pytest

from diffuse_vs_gfm_mms_b200 import serve
from diffuse_vs_gfm_mms_b200.dim import Session
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
    budget = 2.5 * max(serve.footprint_bytes(r.desc, r.steps) for r in reqs)
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
    reqs = _small_requests(4, rate=0.0, seed=5)
    with serve.Server(max_slots=1, quantum=4) as srv:
        for r in reqs:
            srv.submit(r)
        srv._admit(0.0)
        running = next(iter(srv.active))
        assert srv.cancel(running)              # running
        assert srv.cancel(reqs[-1].rid)         # still queued
        assert not srv.cancel(12345)
        assert srv.used == 0
