"""Operation counts of the split sweep per cell: mixture-pressure recoveries,
their doubling steps, bracket-decided bisection steps and literal residual
evaluations, repair_state calls and sound speeds.  The device arithmetic is
compiled for the host with counters (tests/native/physics_host.cpp) and run
over the shock-bubble and bubble-cloud fields at several times; the fields
are advanced between samples by the CPU oracle.

    python tests/native/bisection_counts.py [--nx 256] [--cloud 48]
"""
from __future__ import annotations

import argparse
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from conftest import build_host_harness  # noqa: E402
from diffuse_vs_gfm_mms_b200 import workloads as W  # noqa: E402
from diffuse_vs_gfm_mms_b200.abi import dptr  # noqa: E402

NAMES = ["recoveries", "doublings", "certain_steps", "literal_evals", "no_bracket", "repairs",
         "repair_recoveries", "repair_floors", "sound_speeds", "doublings_skipped"]


def counts(lib, d, U, dt):
    """Counts per cell of one sweep along each axis of the state U."""
    out = np.empty_like(U)
    rows = []
    for axis in range(d.dim):
        buf = (C.c_longlong * 16)()
        lib.host_opcounts(buf, 16, 1)
        assert lib.host_sweep_direction(C.byref(d), axis, C.c_double(dt), dptr(U), dptr(out)) == 0
        lib.host_opcounts(buf, 16, 1)
        rows.append(np.array(buf[:len(NAMES)], dtype=np.float64) / d.ncell)
    return rows


def table(title, samples):
    print(f"\n{title}")
    print(f"{'step':>5} {'axis':>4} " + " ".join(f"{n:>17}" for n in NAMES) + f" {'iters/recovery':>15}")
    for step, rows in samples:
        for axis, r in enumerate(rows):
            iters = (r[1] + r[2] + r[3] + r[9]) / max(r[0], 1e-30)
            print(f"{step:5d} {'xyz'[axis]:>4} " + " ".join(f"{v:17.3f}" for v in r) + f" {iters:15.2f}")


def run(name, d, U, port, lib, cfl, at):
    samples = []
    done = 0
    for step in at:
        if step > done:
            U, _ = port.advance(d, U, cfl, 1e300, step - done)
            done = step
        dt = port.compute_dt_cfl(d, U, cfl, 1e300)
        samples.append((step, counts(lib, d, U, dt)))
    table(name, samples)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=256, help="shock-bubble grid nx (ny = nx / 2)")
    ap.add_argument("--cloud", type=int, default=48, help="bubble-cloud grid side")
    args = ap.parse_args()
    from oracle import oracle as O
    if not os.path.exists(O.PORT_SO):
        O.build()
    port = O.port()
    lib = C.CDLL(build_host_harness())
    lib.host_opcounts.argtypes = [C.POINTER(C.c_longlong), C.c_int, C.c_int]
    lib.host_opcounts.restype = C.c_int
    nx = args.nx
    scale = nx / 1024
    d, U = W.shock_bubble_2d((nx, nx // 2))
    run(f"shock-bubble {nx}x{nx // 2}, CFL 0.8 (per cell and sweep)", d, U, port, lib, 0.8,
        [0, int(230 * scale), int(300 * scale), int(400 * scale)])
    n = args.cloud
    d, U = W.bubble_cloud_3d(N=(n, n, n))
    run(f"bubble cloud {n}^3, 64 bubbles, CFL 0.6 (per cell and sweep)", d, U, port, lib, 0.6, [0, 10, 40])
    d, U = W.riemann(seed=0, N=(1000,))
    run("two-material Riemann 1000, CFL 0.8 (per cell and sweep)", d, U, port, lib, 0.8, [0, 500, 2000])


if __name__ == "__main__":
    main()
