"""Parity over the configurations as they are stated, at their step counts.

The records under tests/golden/long_*.npz were made by
tests/golden/make_long_runs.py from the reference's own DIM step (compiled
from its sources, oracle/_ref): the SHA-256 of the state at each checkpoint,
its per-variable sums and the full state of a fixed sample of cells, and
the dt of every step.  The CUDA path replays the same steps through the
C-ABI and must match bit for bit — the state's hash at every checkpoint and
every dt.  The relative L1 per conserved variable on the sampled cells and
the per-variable sums are checked first, so that a failure says by how much
it missed the 1e-10 target.

* config 0: the 1000-cell two-material tube over its full 2000 steps;
* config 1: the shock-bubble grid at its full 1024x512 size for 400 steps —
  the Mach 1.22 shock reaches the bubble's edge after about 230 steps, so
  the last checkpoints are well into the interaction;
* config 2: its generator (64 bubbles in the unit cube, 1e9 Pa slab) at
  64^3 and 128^3 for 100 steps.
"""
from __future__ import annotations

import hashlib
import os

import numpy as np
import pytest

from diffuse_vs_gfm_mms_b200 import workloads as W
from diffuse_vs_gfm_mms_b200.dim import Session
from helpers import GOLDEN, bitwise_equal, rel_l1

pytestmark = pytest.mark.gpu

REL_L1_TOL = 1e-10

GENERATORS = {
    "c0_riemann_1000": lambda: W.riemann(seed=0, N=(1000,)),
    "c1_shock_bubble_1024x512": lambda: W.shock_bubble_2d(N=(1024, 512)),
    "c2_cloud_64cubed": lambda: W.bubble_cloud_3d(N=(64, 64, 64)),
    "c2_cloud_128cubed": lambda: W.bubble_cloud_3d(N=(128, 128, 128)),
}


def sha256(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


@pytest.mark.parametrize("case", list(GENERATORS))
def test_long_run_matches_the_reference(case):
    path = os.path.join(GOLDEN, f"long_{case}.npz")
    if not os.path.exists(path):
        pytest.skip(f"{os.path.basename(path)} not generated")
    rec = np.load(path)
    d, U = GENERATORS[case]()
    assert sha256(U) == str(rec["in_sha256"]), "the seeded generator no longer gives the recorded input"
    cfl = float(rec["cfl"])
    idx = rec["sample_index"]
    dts = []
    with Session(d, U) as s:
        done = 0
        for c in rec["checkpoints"]:
            c = int(c)
            dts.append(s.steps(c - done, cfl, 1e300))
            done = c
            out = s.download()
            l1 = rel_l1(out[:, idx], rec[f"s{c}_sample"])
            assert np.all(l1 <= REL_L1_TOL), f"{case} step {c}: sampled relative L1 {l1}"
            sums = out.sum(axis=1)
            den = np.maximum(rec[f"s{c}_abs_sum"], 1e-300)
            assert np.all(np.abs(sums - rec[f"s{c}_sum"]) / den <= REL_L1_TOL), f"{case} step {c}: sums differ"
            assert bitwise_equal(out[:, idx], rec[f"s{c}_sample"]), f"{case} step {c}: sampled cells differ"
            assert sha256(out) == str(rec[f"s{c}_sha256"]), f"{case} step {c}: state differs from the reference"
    assert bitwise_equal(np.concatenate(dts), rec["dt"])


def test_slabs_reproduce_the_long_record():
    """The slab solver (four slabs of the c1 grid on one GPU, the ghost
    exchange as device copies) through the shock-bubble interaction: the
    same hash as the reference at every checkpoint and the same dts."""
    from diffuse_vs_gfm_mms_b200.dim import Slabs

    case = "c1_shock_bubble_1024x512"
    path = os.path.join(GOLDEN, f"long_{case}.npz")
    if not os.path.exists(path):
        pytest.skip(f"{os.path.basename(path)} not generated")
    rec = np.load(path)
    d, U = GENERATORS[case]()
    cfl = float(rec["cfl"])
    dts = []
    with Slabs(d, [0, 0, 0, 0], U) as L:
        done = 0
        for c in rec["checkpoints"]:
            c = int(c)
            dts.append(L.steps(c - done, cfl, 1e300))
            done = c
            assert sha256(L.download()) == str(rec[f"s{c}_sha256"]), f"slabs, step {c}"
    assert bitwise_equal(np.concatenate(dts), rec["dt"])


def test_server_solo_lane_reproduces_the_long_record():
    """A c1 solve submitted to the serving loop (a solo lane: a session shell
    over the server's arena) beside small batch-lane solves: its 100-step
    state is the reference's, bit for bit."""
    from diffuse_vs_gfm_mms_b200 import serve

    case = "c1_shock_bubble_1024x512"
    path = os.path.join(GOLDEN, f"long_{case}.npz")
    if not os.path.exists(path):
        pytest.skip(f"{os.path.basename(path)} not generated")
    rec = np.load(path)
    d, U = GENERATORS[case]()
    n = int(rec["checkpoints"][0])
    big = serve.Request(rid=0, desc=d, U=U, steps=n, cfl=float(rec["cfl"]), dt_max=1e300, arrival=0.0)
    small = serve.make_requests(6, rate=0.0, seed=21, steps_range=(20, 60), n1d_range=(64, 512),
                                side2d_range=(16, 64))
    for k, r in enumerate(small):
        r.rid = k + 1
    with serve.Server(hbm_budget_bytes=8e9, max_slots=16, quantum=8) as srv:
        stats = srv.serve([big] + small)
    res = {r.rid: r for r in stats.results}
    assert sha256(res[0].U) == str(rec[f"s{n}_sha256"])
    assert bitwise_equal(res[0].dts, rec["dt"][:n])
