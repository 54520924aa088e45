"""Generate the golden vectors under tests/golden/ from the reference itself.

    make -C oracle && python tests/golden/make_golden.py

Runs oracle/_ref/libdimref.so and oracle/_ref/libeulerref.so — the
reference's own header-only DIM step and single-material Euler step,
compiled from its sources by oracle/Makefile — on seeded inputs and stores
inputs and outputs as .npz fixtures.  The reference publishes no numeric
golden vectors of its own, so these pin the CPU restatement (and, through it,
the CUDA path) to the reference's exact double-precision results.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from diffuse_vs_gfm_mms_b200 import abi, workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

MATERIAL_SETS = {
    "water_air": [("stiffened_gas", 4.4, 6e8), ("ideal_gas", 1.4, 0.0)],
    "two_ideal": [("ideal_gas", 1.4, 0.0), ("ideal_gas", 1.67, 0.0)],
    "three": [("ideal_gas", 1.6, 0.0), ("stiffened_gas", 2.1, 3e8), ("ideal_gas", 1.4, 0.0)],
    "single": [("stiffened_gas", 6.1, 1e8)],
}


def desc_to_array(d: abi.Desc) -> np.ndarray:
    return np.frombuffer(bytes(d), dtype=np.uint8).copy()


def kat_records(ref: O.Checker):
    out = {}
    for dim in (1, 2, 3):
        for name, mats in MATERIAL_SETS.items():
            d = abi.make_desc(dim, [8] * dim, [0.1] * dim, mats)
            U = W.random_states(d, 80, seed=100 * dim + len(mats))
            U2 = W.random_states(d, 80, seed=100 * dim + len(mats) + 50)
            P = ref.cons_to_prim(d, U)
            key = f"d{dim}_{name}"
            out[f"{key}_desc"] = desc_to_array(d)
            out[f"{key}_U"] = U
            out[f"{key}_U2"] = U2
            out[f"{key}_cons_to_prim"] = P
            out[f"{key}_prim_to_cons"] = ref.prim_to_cons(d, P)
            out[f"{key}_repair"] = ref.repair_state(d, U)
            rec = np.concatenate([U[:, :d.nmat].sum(1, keepdims=True), P[:, -1:],
                                  P[:, d.nmat:2 * d.nmat], P[:, :d.nmat]], axis=1)
            out[f"{key}_sound_rec"] = rec
            for lm in (0, 1, 2):
                d.lambda_model = lm
                out[f"{key}_alpha_rhs{lm}"] = ref.alpha_rhs(d, P)
                out[f"{key}_sound{lm}"] = ref.mixture_sound_speed(d, rec)
                out[f"{key}_hllc{lm}"] = ref.hllc(d, dim - 1, U, U2)
            d.lambda_model = 0
            # mixture pressure records: rho_total, e, alpha[nmat], rho[nmat]
            rhot = np.maximum(U[:, :d.nmat].sum(1), 1e-12)
            vel = U[:, d.nmat:d.nmat + dim] / rhot[:, None]
            e = (U[:, d.nmat + dim] - 0.5 * rhot * (vel * vel).sum(1)) / rhot
            prec = np.concatenate([rhot[:, None], e[:, None], P[:, d.nmat:2 * d.nmat], P[:, :d.nmat]], axis=1)
            out[f"{key}_pressure_rec"] = prec
            out[f"{key}_pressure"] = ref.mixture_pressure(d, prec)
    return out


FIELD_CASES = {
    "c0_riemann_1d": (lambda: W.riemann(seed=1, N=(1000,)), 0.8, 20),
    "c1_shock_bubble_48x24": (lambda: W.shock_bubble_2d(N=(48, 24)), 0.8, 5),
    "c2_cloud_12cubed": (lambda: W.bubble_cloud_3d(N=(12, 12, 12), nbubbles=2), 0.6, 2),
}


def field_cases(ref: O.Checker):
    out = {}
    cases = dict(FIELD_CASES)
    for name, (gen, cfl, n) in cases.items():
        d, U = gen()
        outU, dts = ref.advance(d, U, cfl, 1e300, n)
        out[f"{name}_desc"] = desc_to_array(d)
        out[f"{name}_in"] = U
        out[f"{name}_out"] = outU
        out[f"{name}_dt"] = dts
        out[f"{name}_meta"] = np.array([cfl, n])
    # option coverage on small 2D fields
    extra = []
    d, U = W.riemann(seed=3, N=(16, 12), axis=1)
    d.time_update = abi.TIME_UNSPLIT
    extra.append(("unsplit_16x12", d, U, 0.5, 4))
    d, U = W.riemann(seed=4, N=(14, 16), axis=0, bc=["nonreflective", "reflective"])
    extra.append(("nonreflective_14x16", d, U, 0.5, 4))
    d, U = W.single_bubble_2d((14, 12), seed=5)
    d.lambda_model = abi.LAMBDA_ALLAIRE
    extra.append(("allaire_14x12", d, U, 0.5, 4))
    d, U = W.single_bubble_2d((14, 12), seed=6)
    d.lambda_model = abi.LAMBDA_EQUAL_VELOCITY
    d.alpha_source_floor = 1e-3
    extra.append(("equal_velocity_14x12", d, U, 0.5, 4))
    for name, d, U, cfl, n in extra:
        outU, dts = ref.advance(d, U, cfl, 1e300, n)
        out[f"{name}_desc"] = desc_to_array(d)
        out[f"{name}_in"] = U
        out[f"{name}_out"] = outU
        out[f"{name}_dt"] = dts
        out[f"{name}_meta"] = np.array([cfl, n])
    return out


EULER_CASES = {
    "sod_200": (lambda: W.euler_tube(seed=-1, N=(200,)), 0.8, 30),
    "tube_300_s0": (lambda: W.euler_tube(seed=0, N=(300,)), 0.8, 30),
    "tube_water_300": (lambda: W.euler_tube(seed=2, N=(300,)), 0.8, 30),
    "tube_2d_y": (lambda: W.euler_tube(seed=1, N=(12, 64), axis=1), 0.6, 20),
    "blast_2d": (lambda: W.euler_blast(N=(40, 36), seed=3), 0.6, 20),
    "blast_2d_reflective": (lambda: W.euler_blast(N=(36, 32), seed=4, bc=["reflective", "reflective"]), 0.6, 20),
    "blast_2d_nonreflective": (lambda: W.euler_blast(N=(36, 32), seed=5, bc=["nonreflective", "transmissive"]),
                               0.6, 20),
    "blast_2d_water": (lambda: W.euler_blast(N=(32, 32), seed=6, material=("stiffened_gas", 4.4, 6e8)), 0.6, 20),
    "blast_2d_unsplit": (lambda: W.euler_blast(N=(32, 30), seed=7, time_update="unsplit"), 0.5, 20),
    "blast_3d": (lambda: W.euler_blast(N=(14, 12, 10), seed=8), 0.6, 10),
    "nonreflective_n3": (lambda: W.euler_blast(N=(3, 24), seed=9, bc=["nonreflective", "nonreflective"]), 0.5, 10),
}


def euler_cases(eref: O.EulerChecker):
    """The single-material Euler step (oracle/_ref/libeulerref.so)."""
    out = {}
    for name, (gen, cfl, n) in EULER_CASES.items():
        d, U = gen()
        outU, dts = eref.advance(d, U, cfl, 1e300, n)
        out[f"{name}_desc"] = desc_to_array(d)
        out[f"{name}_in"] = U
        out[f"{name}_out"] = outU
        out[f"{name}_dt"] = dts
        out[f"{name}_meta"] = np.array([cfl, n])
    # HLLC records on random face pairs (ideal and stiffened), both axes of 2D
    for tag, mat in (("ideal", ("ideal_gas", 1.4, 0.0)), ("water", ("stiffened_gas", 4.4, 6e8))):
        d = abi.make_desc(2, [4, 4], [0.1, 0.1], [mat], model=abi.MODEL_EULER)
        rng = np.random.default_rng(11 if tag == "ideal" else 12)
        n = 200
        rho = np.exp(rng.uniform(np.log(0.1), np.log(1000.0), size=(2, n)))
        vel = rng.uniform(-300.0, 300.0, size=(2, 2, n))
        p = np.exp(rng.uniform(np.log(1e3), np.log(1e9), size=(2, n)))
        UL = W.euler_prim_to_cons(2, mat[0], mat[1], mat[2], rho[0], vel[0], p[0]).T.copy()
        UR = W.euler_prim_to_cons(2, mat[0], mat[1], mat[2], rho[1], vel[1], p[1]).T.copy()
        out[f"hllc_{tag}_desc"] = desc_to_array(d)
        out[f"hllc_{tag}_UL"] = UL
        out[f"hllc_{tag}_UR"] = UR
        for axis in (0, 1):
            out[f"hllc_{tag}_F{axis}"] = eref.hllc(d, axis, UL, UR)
    return out


def main():
    """python tests/golden/make_golden.py [dim | euler | all] (default all)."""
    which = sys.argv[1] if len(sys.argv) > 1 else "all"
    if which in ("dim", "all"):
        if not O.reference_available():
            raise SystemExit("oracle/_ref/libdimref.so missing: run make -C oracle where the reference sources exist")
        ref = O.reference()
        np.savez_compressed(os.path.join(HERE, "kat_records.npz"), **kat_records(ref))
        np.savez_compressed(os.path.join(HERE, "field_steps.npz"), **field_cases(ref))
    if which in ("euler", "all"):
        np.savez_compressed(os.path.join(HERE, "euler_steps.npz"), **euler_cases(O.EulerChecker("reference")))
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
