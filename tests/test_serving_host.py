"""Host-side logic of the serving loop (no GPU): request streams and the
device-footprint model used for admission."""
from __future__ import annotations

import numpy as np

from diffuse_vs_gfm_mms_b200 import serve


def test_request_stream_follows_config_4():
    reqs = serve.make_requests(400, rate=50.0, seed=1, n1d_range=(256, 8192), side2d_range=(128, 256))
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) >= 0)
    gaps = np.diff(np.concatenate([[0.0], arr]))
    assert abs(gaps.mean() - 1 / 50.0) < 0.3 / 50.0       # Poisson at the requested rate
    share_1d = np.mean([r.desc.dim == 1 for r in reqs])
    assert 0.3 < share_1d < 0.5
    steps = np.array([r.steps for r in reqs])
    assert steps.min() >= 100 and steps.max() <= 2000
    for r in reqs:
        assert r.U.shape == (r.desc.nvar, r.desc.ncell)


def test_footprint_counts_state_scratch_and_dt_log():
    r = serve.make_requests(1, rate=0.0, seed=2, side2d_range=(64, 64), n1d_range=(100, 100))[0]
    fp = serve.footprint_bytes(r.desc, r.steps)
    assert fp >= 2 * r.U.nbytes + 8 * r.steps
    assert fp < 20 * r.U.nbytes
