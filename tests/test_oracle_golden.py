"""The CPU oracle (C restatement) against golden vectors produced by the
reference itself, and against the live reference build when present."""
from __future__ import annotations

import numpy as np
import pytest

from diffuse_vs_gfm_mms_b200 import workloads as W
from helpers import bitwise_equal, desc_from_array, load, ndiff

KAT = load("kat_records.npz")
FIELDS = load("field_steps.npz")
KAT_KEYS = sorted({k.rsplit("_desc", 1)[0] for k in KAT.files if k.endswith("_desc")})
FIELD_KEYS = sorted({k.rsplit("_desc", 1)[0] for k in FIELDS.files if k.endswith("_desc")})


@pytest.mark.parametrize("key", KAT_KEYS)
def test_kat_records(port, key):
    d = desc_from_array(KAT[f"{key}_desc"])
    U, U2 = KAT[f"{key}_U"], KAT[f"{key}_U2"]
    P = port.cons_to_prim(d, U)
    assert bitwise_equal(P, KAT[f"{key}_cons_to_prim"])
    assert bitwise_equal(port.prim_to_cons(d, KAT[f"{key}_cons_to_prim"]), KAT[f"{key}_prim_to_cons"])
    assert bitwise_equal(port.repair_state(d, U), KAT[f"{key}_repair"])
    assert bitwise_equal(port.mixture_pressure(d, KAT[f"{key}_pressure_rec"]), KAT[f"{key}_pressure"])
    for lm in (0, 1, 2):
        d.lambda_model = lm
        assert bitwise_equal(port.alpha_rhs(d, P), KAT[f"{key}_alpha_rhs{lm}"])
        assert bitwise_equal(port.mixture_sound_speed(d, KAT[f"{key}_sound_rec"]), KAT[f"{key}_sound{lm}"])
        assert bitwise_equal(port.hllc(d, d.dim - 1, U, U2), KAT[f"{key}_hllc{lm}"])


@pytest.mark.parametrize("key", FIELD_KEYS)
def test_field_steps(port, key):
    d = desc_from_array(FIELDS[f"{key}_desc"])
    cfl, n = FIELDS[f"{key}_meta"]
    out, dts = port.advance(d, FIELDS[f"{key}_in"], float(cfl), 1e300, int(n))
    assert ndiff(out, FIELDS[f"{key}_out"]) == 0
    assert bitwise_equal(dts, FIELDS[f"{key}_dt"])


def test_port_matches_live_reference(port, reference):
    """Fresh seeds (not in the fixtures): oracle == reference, bit for bit."""
    for dim, N in ((1, (300,)), (2, (20, 16)), (3, (8, 8, 6))):
        d, U = W.riemann(seed=77 + dim, N=N, axis=dim - 1)
        a, da = port.advance(d, U, 0.7, 1e300, 6)
        b, db = reference.advance(d, U, 0.7, 1e300, 6)
        assert ndiff(a, b) == 0 and bitwise_equal(da, db)
        Ur = W.random_states(d, 3000, seed=dim)
        assert bitwise_equal(port.cons_to_prim(d, Ur), reference.cons_to_prim(d, Ur))
        assert bitwise_equal(port.repair_state(d, Ur), reference.repair_state(d, Ur))


def test_oracle_rejects_unsupported_eos(port):
    from diffuse_vs_gfm_mms_b200 import abi
    d = abi.make_desc(1, [8], [0.1], [("tait", 7.0, 0.0)])
    with pytest.raises(RuntimeError):
        port.cons_to_prim(d, np.zeros((1, 3)))


@pytest.mark.parametrize("gen", [
    lambda: W.riemann(seed=3, N=(200,)),
    lambda: W.shock_bubble_2d(N=(40, 20)),
    lambda: W.bubble_cloud_3d(N=(10, 9, 8), nbubbles=2),
    lambda: W.riemann(seed=7, N=(6, 14, 5), axis=1),
])
def test_boundary_flux_matches_reference(port, reference, gen):
    """compute_dim_boundary_flux (src/app/io/conservation_report.hpp:253-305):
    the restatement sums in the reference's order, so bit for bit."""
    d, U = gen()
    assert bitwise_equal(port.boundary_flux(d, U), reference.boundary_flux(d, U))
