"""The CSV snapshot format (dim::write_csv, src/io/dim_write_csv.hpp:15-125):
the C restatement's writer (oracle/dim_oracle.c) against the reference's own
writer compiled from its sources (oracle/_ref), byte for byte, on stepped
fields in 1D, 2D and 3D with two to four materials.  The CUDA writer is
checked against the same reference output in tests/test_gpu_io.py."""
from __future__ import annotations

import os

import pytest

from diffuse_vs_gfm_mms_b200 import abi, workloads as W

CASES = {
    "riemann_1d": (lambda: W.riemann(seed=3, N=(200,)), (0.0,), (1.0,)),
    "shock_bubble_2d": (lambda: W.shock_bubble_2d(N=(48, 24)), (0.0, 0.0), (2.0, 1.0)),
    "cloud_3d": (lambda: W.bubble_cloud_3d(N=(12, 10, 8), nbubbles=2), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0)),
    "four_materials_2d": (lambda: (abi.make_desc(2, (9, 7), (0.1, 0.2),
                                                 [("stiffened_gas", 1.9, 5e8), ("ideal_gas", 1.3, 0.0),
                                                  ("stiffened_gas", 5.5, 2e8), ("ideal_gas", 2.0, 0.0)]), None),
                          (-1.0, 0.5), (2.0, 3.0)),
}


def _field(name):
    gen, lo, hi = CASES[name]
    d, U = gen()
    if U is None:
        U = W.random_states(d, d.ncell, seed=4, edge_fraction=0.0).T.copy()
    return d, U, lo, hi


@pytest.mark.parametrize("name", list(CASES))
def test_port_csv_matches_reference_bytes(port, reference, tmp_path, name):
    d, U, lo, hi = _field(name)
    U, _ = port.advance(d, U, 0.5, 1e300, 3)
    a, b = os.path.join(tmp_path, "port.csv"), os.path.join(tmp_path, "ref.csv")
    port.write_csv(d, U, lo, hi, a)
    reference.write_csv(d, U, lo, hi, b)
    with open(a, "rb") as fa, open(b, "rb") as fb:
        pa, pb = fa.read(), fb.read()
    assert pa.splitlines()[0] == pb.splitlines()[0]
    assert len(pa.splitlines()) == d.ncell + 1
    assert pa == pb
