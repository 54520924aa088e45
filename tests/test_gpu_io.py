"""Device-side initial fields and the asynchronous CSV writer.

* The shock-bubble and bubble-cloud fields written by the device
  (dimgpu_init_shock_bubble / dimgpu_init_bubble_cloud) are the same bits as
  the host generator's (workloads.shock_bubble_2d / bubble_cloud_3d), which
  is what every parity record was made from.
* The CSV snapshot (dimgpu_csv_write_async) is byte for byte the file the
  reference's own dim::write_csv (src/io/dim_write_csv.hpp:15-125, compiled
  from its sources into oracle/_ref) writes for the same state, also while
  the session keeps stepping after the snapshot was taken.
"""
from __future__ import annotations

import os

import pytest

from diffuse_vs_gfm_mms_b200 import abi, workloads as W
from diffuse_vs_gfm_mms_b200.dim import Session
from helpers import bitwise_equal, ndiff

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N", [(96, 48), (1024, 512), (333, 129)])
def test_device_shock_bubble_field_is_the_host_field(N):
    d, U = W.shock_bubble_2d(N=N)
    d2, ic = W.shock_bubble_2d_setup(N)
    with Session(d2) as s:
        s.init_shock_bubble(ic)
        dev = s.download()
    assert ndiff(dev, U) == 0


@pytest.mark.parametrize("N,nb", [((32, 28, 24), 6), ((128, 128, 128), 64)])
def test_device_bubble_cloud_field_is_the_host_field(N, nb):
    d, U = W.bubble_cloud_3d(N=N, nbubbles=nb)
    d2, ic, bubbles = W.bubble_cloud_3d_setup(N, nbubbles=nb)
    with Session(d2) as s:
        s.init_bubble_cloud(ic, bubbles)
        dev = s.download()
    assert ndiff(dev, U) == 0


def _csv_case(name):
    if name == "shock_bubble":
        d, U = W.shock_bubble_2d(N=(64, 32))
        return d, U, (0.0, 0.0), (2.0, 1.0), 0.8
    if name == "cloud":
        d, U = W.bubble_cloud_3d(N=(16, 12, 10), nbubbles=2)
        return d, U, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), 0.6
    if name == "riemann_1d":
        d, U = W.riemann(seed=5, N=(300,))
        return d, U, (0.0,), (1.0,), 0.8
    d = abi.make_desc(2, (11, 9), (0.1, 0.2), [("ideal_gas", 1.6, 0.0), ("stiffened_gas", 2.1, 3e8),
                                               ("ideal_gas", 1.4, 0.0)])
    U = W.random_states(d, d.ncell, seed=6, edge_fraction=0.0).T.copy()
    return d, U, (-0.5, 0.0), (0.6, 1.8), 0.4


@pytest.mark.parametrize("name", ["shock_bubble", "cloud", "riemann_1d", "three_materials"])
def test_csv_snapshot_matches_the_reference_writer(reference, tmp_path, name):
    d, U, lo, hi, cfl = _csv_case(name)
    ours, ref = os.path.join(tmp_path, "gpu.csv"), os.path.join(tmp_path, "ref.csv")
    with Session(d, U) as s:
        s.steps(3, cfl, 1e300)
        state = s.download()
        w = s.write_csv_async(ours, lo, hi, threads=4)
        s.steps(2, cfl, 1e300)          # the session keeps stepping meanwhile
        w.wait()
        after = s.download()
    reference.write_csv(d, state, lo, hi, ref)
    with open(ours, "rb") as fa, open(ref, "rb") as fb:
        assert fa.read() == fb.read()
    assert not bitwise_equal(after, state)


def test_csv_snapshot_of_a_large_grid(reference, tmp_path):
    """More than one device -> host chunk (2^20 cells): 1100x1000 cells."""
    d, U = W.shock_bubble_2d(N=(1100, 1000))
    ours, ref = os.path.join(tmp_path, "gpu.csv"), os.path.join(tmp_path, "ref.csv")
    with Session(d, U) as s:
        s.write_csv_async(ours, (0.0, 0.0), (2.0, 1.0)).wait()
    reference.write_csv(d, U, (0.0, 0.0), (2.0, 1.0), ref)
    with open(ours, "rb") as fa, open(ref, "rb") as fb:
        assert fa.read() == fb.read()
