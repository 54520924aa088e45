"""The long-run golden records (tests/golden/long_*.npz) on the CPU: each
record's input is what the seeded generator gives today, and the C
restatement of the step (oracle/dim_oracle.c) reproduces the reference's
record of the 1000-cell tube over all 2000 steps, bit for bit.  The c1 record
reaches into the shock-bubble interaction: the shock from x = 0.6 (about
1.44 length units per time unit) meets the bubble's edge at x = 0.75 near
t = 0.104, and the record's steps run to t > 0.12."""
from __future__ import annotations

import hashlib
import os

import numpy as np
import pytest

from diffuse_vs_gfm_mms_b200 import workloads as W
from helpers import GOLDEN, bitwise_equal


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def _rec(name):
    path = os.path.join(GOLDEN, f"long_{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"{os.path.basename(path)} not generated")
    return np.load(path)


def test_c0_record_reproduced_by_the_port(port):
    rec = _rec("c0_riemann_1000")
    d, U = W.riemann(seed=0, N=(1000,))
    assert _sha(U) == str(rec["in_sha256"])
    out, dts = port.advance(d, U, float(rec["cfl"]), 1e300, 2000)
    assert bitwise_equal(dts, rec["dt"])
    assert _sha(out) == str(rec["s2000_sha256"])


@pytest.mark.parametrize("name,gen", [("c1_shock_bubble_1024x512", lambda: W.shock_bubble_2d(N=(1024, 512))),
                                      ("c2_cloud_64cubed", lambda: W.bubble_cloud_3d(N=(64, 64, 64)))])
def test_record_inputs_match_the_generators(name, gen):
    rec = _rec(name)
    d, U = gen()
    assert _sha(U) == str(rec["in_sha256"])


def test_c1_record_reaches_the_interaction():
    rec = _rec("c1_shock_bubble_1024x512")
    assert float(np.sum(rec["dt"])) > 0.12
