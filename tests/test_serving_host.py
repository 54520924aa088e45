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


def _config(**kw):
    from diffuse_vs_gfm_mms_b200 import abi
    cfg = abi.ServerConfig()
    cfg.hbm_budget_bytes = kw.get("budget", 8e9)
    for k, v in enumerate(kw.get("dim_share", (0.1, 0.4, 0.0))):
        cfg.dim_share[k] = v
    cfg.max_slots = kw.get("max_slots", 8)
    cfg.quantum = kw.get("quantum", 8)
    cfg.max_steps_per_solve = kw.get("max_steps", 4096)
    cfg.solo_min_cells = kw.get("solo_min_cells", 1 << 18)
    cfg.solo_share = kw.get("solo_share", 0.5)
    cfg.solo_slots = kw.get("solo_slots", 4)
    return cfg


def test_server_config_validation_and_submit_refusals():
    """dimgpu_server_create checks its configuration, and submit refuses a
    solve larger than its lane's budget share before queueing it — both
    without touching a device (the lanes' memory is reserved on first
    admission)."""
    import ctypes as C

    from diffuse_vs_gfm_mms_b200 import abi
    from diffuse_vs_gfm_mms_b200.native import lib

    L = lib()

    def create(cfg):
        h = C.c_void_p()
        rc = L.dimgpu_server_create(C.byref(cfg), C.byref(h))
        return rc, h

    for bad in (dict(dim_share=(0.4, 0.6, 0.0), solo_share=0.5),    # shares above the budget
                dict(solo_share=-0.1), dict(solo_slots=-1), dict(solo_min_cells=-5),
                dict(max_steps=5000),                                  # solo lanes keep 4096 dts
                dict(quantum=0), dict(max_slots=0), dict(budget=0.0)):
        rc, h = create(_config(**bad))
        assert rc == abi.E_INVALID_ARG and not h.value, bad
    rc, h = create(_config(max_steps=5000, solo_slots=0))            # no solo lanes: no 4096 cap
    assert rc == abi.OK
    L.dimgpu_server_destroy(h)

    rc, h = create(_config(budget=1e3))
    assert rc == abi.OK
    try:
        small, big = serve.make_requests(2, rate=0.0, seed=4, n1d_range=(64, 64), side2d_range=(600, 600))
        for r in (small, big):
            rid = C.c_longlong()
            U = np.ascontiguousarray(r.U)
            rc = L.dimgpu_server_submit(h, C.byref(r.desc), U.ctypes.data_as(C.POINTER(C.c_double)),
                                        r.steps, r.cfl, r.dt_max, C.byref(rid))
            # 1e3 bytes hold neither a 64-cell batch solve (10 % share) nor a
            # 360 000-cell solo solve (50 %)
            assert rc == abi.E_OOM, (r.desc.ncell, rc)
        st = abi.ServerCounters()
        assert L.dimgpu_server_stats(h, C.byref(st)) == abi.OK
        assert st.submitted == 0 and st.queued == 0
    finally:
        L.dimgpu_server_destroy(h)
