"""Generate the long-run golden records under tests/golden/ from the reference.

    make -C oracle && python tests/golden/make_long_runs.py [case ...]

Runs oracle/_ref/libdimref.so — the reference's own header-only DIM step
compiled from its sources — over the configurations as they are stated, at
the step counts where their physics happens, and stores a compact record of
each run (tests/golden/long_<case>.npz):

* the SHA-256 of the initial field's bytes (so a drift of the seeded
  generator is told apart from a difference of the step);
* the dt of every step;
* at every checkpoint: the SHA-256 of the state's bytes, the per-variable
  sum and sum of magnitudes, and the full state of a fixed sample of cells.

A field of 2.1M cells x 100 steps takes the reference tens of minutes on a
CPU; the GPU test replays the same steps in about a second and compares
bit for bit.  The records are small (a hash and a cell sample per
checkpoint), so they can be committed where the fields themselves could not.
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from diffuse_vs_gfm_mms_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

SAMPLE = 2048

# name -> (generator, cfl, checkpoints (cumulative step counts))
CASES = {
    # config 0 over its full 2000 steps
    "c0_riemann_1000": (lambda: W.riemann(seed=0, N=(1000,)), 0.8, (100, 500, 1000, 2000)),
    # config 1 at full size through the shock-bubble interaction (the shock
    # reaches the bubble's edge after about 230 steps)
    "c1_shock_bubble_1024x512": (lambda: W.shock_bubble_2d(N=(1024, 512)), 0.8, (100, 200, 300, 400)),
    # config 2's generator (64 bubbles in the unit cube) at 64^3 and 128^3
    "c2_cloud_64cubed": (lambda: W.bubble_cloud_3d(N=(64, 64, 64)), 0.6, (25, 50, 100)),
    "c2_cloud_128cubed": (lambda: W.bubble_cloud_3d(N=(128, 128, 128)), 0.6, (25, 50, 100)),
}


def sha256(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def sample_index(ncell: int) -> np.ndarray:
    """A fixed spread of cells: every k-th cell plus the first and last."""
    k = max(1, ncell // SAMPLE)
    return np.unique(np.concatenate([np.arange(0, ncell, k), [ncell - 1]]))


def record(name: str, ref: O.Checker) -> dict:
    gen, cfl, checkpoints = CASES[name]
    d, U = gen()
    idx = sample_index(U.shape[1])
    out = {"in_sha256": np.array(sha256(U)), "cfl": np.array(cfl), "checkpoints": np.array(checkpoints),
           "sample_index": idx}
    dts = []
    cur, done = U, 0
    for c in checkpoints:
        t0 = time.time()
        cur, dt = ref.advance(d, cur, cfl, 1e300, c - done)
        dts.append(dt)
        done = c
        out[f"s{c}_sha256"] = np.array(sha256(cur))
        out[f"s{c}_sum"] = cur.sum(axis=1)
        out[f"s{c}_abs_sum"] = np.abs(cur).sum(axis=1)
        out[f"s{c}_sample"] = cur[:, idx].copy()
        print(f"{name}: {c} steps ({time.time() - t0:.1f} s)", flush=True)
    out["dt"] = np.concatenate(dts)
    return out


def main():
    names = sys.argv[1:] or list(CASES)
    if not O.reference_available():
        raise SystemExit("oracle/_ref/libdimref.so missing: run make -C oracle where the reference sources exist")
    ref = O.reference()
    for name in names:
        np.savez_compressed(os.path.join(HERE, f"long_{name}.npz"), **record(name, ref))


if __name__ == "__main__":
    main()
