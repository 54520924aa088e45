"""Opt-in stress test (`-m slow`): the accelerated mixture-pressure bisection
of the kernels (csrc/dim_physics.h, compiled for the host) against the
literal bisection of the C restatement (oracle/dim_oracle.c, the reference's
MixtureEOS::pressure_from_internal_energy, src/dim/eos.hpp:77-143) on 10^8
seeded states, bit for bit.

The states are drawn to reach every branch of the reference's loop:

* the doubling phase — a stiffened component far below gamma * p_inf makes
  the per-material fallback pressure (the starting upper bound) much smaller
  than the root, so `hi` doubles before the bisection (about 9 % of the
  states double at least once, 0.1 % more than ten times);
* roots far below 1 (ideal gases at low pressure, where lo = 1e-12 and the
  1e-10 clamp of the residual matter) and far above 1e9;
* energies placed within a few termination thresholds of a recovery's
  stopping window, where the accelerated loop must evaluate the literal
  residual;
* one to four materials with random kinds, gamma in [1.05, 7] and p_inf up
  to 1e9, volume fractions down to 1e-13 and exact zeros, and non-finite /
  negative inputs.

Run with `python -m pytest tests -m slow`.  About a minute on 8 cores.
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from diffuse_vs_gfm_mms_b200 import abi

pytestmark = pytest.mark.slow

TOTAL = 100_000_000
CHUNK = 1_000_000


def _chunk(seed: int):
    """One chunk: a random material set and CHUNK pressure records
    (rho_total, e, alpha[nmat], rho[nmat])."""
    rng = np.random.default_rng(seed)
    nmat = int(rng.integers(1, 5))
    mats = []
    for _ in range(nmat):
        stiff = rng.uniform() < 0.6
        gamma = float(rng.uniform(1.05, 7.0))
        p_inf = float(np.exp(rng.uniform(np.log(1e5), np.log(1e9)))) if stiff else 0.0
        mats.append(("stiffened_gas" if stiff else "ideal_gas", gamma, p_inf))
    d = abi.make_desc(1, [8], [0.1], mats)
    n = CHUNK
    alpha = rng.dirichlet(np.full(nmat, 0.3), size=n).T if nmat > 1 else np.ones((1, n))
    tiny = rng.uniform(size=n) < 0.05
    if nmat > 1:
        k = rng.integers(0, nmat, size=n)
        alpha[k[tiny], np.nonzero(tiny)[0]] = np.exp(rng.uniform(np.log(1e-13), np.log(1e-6), size=tiny.sum()))
        alpha[:, rng.uniform(size=n) < 0.01] = 0.0
    rho = np.exp(rng.uniform(np.log(1e-4), np.log(1e4), size=(nmat, n)))
    p = np.exp(rng.uniform(np.log(1e-14), np.log(1e12), size=n))
    g = np.array([m[1] for m in mats])[:, None]
    pinf = np.array([m[2] for m in mats])[:, None]
    rho_e = (alpha * rho * ((p + g * pinf) / ((g - 1.0) * rho))).sum(axis=0)
    rho_t = (alpha * rho).sum(axis=0)
    rho_t = np.where(rng.uniform(size=n) < 0.02, np.exp(rng.uniform(np.log(1e-14), 0.0, size=n)), rho_t)
    e = rho_e / np.maximum(rho_t, 1e-12)
    near = rng.uniform(size=n) < 0.33
    e = np.where(near, e * (1.0 + rng.uniform(-5e-10, 5e-10, size=n)), e)
    bad = rng.uniform(size=n)
    e = np.where(bad < 0.002, -e, e)
    e = np.where((bad >= 0.002) & (bad < 0.003), np.nan, e)
    e = np.where((bad >= 0.003) & (bad < 0.004), np.inf, e)
    rho[:, (bad >= 0.004) & (bad < 0.005)] *= -1.0
    rec = np.concatenate([rho_t[:, None], e[:, None], alpha.T, rho.T], axis=1)
    return d, np.ascontiguousarray(rec)


def test_accelerated_bisection_on_1e8_states(port):
    from test_device_arithmetic_host import Host

    host = Host()
    nchunks = TOTAL // CHUNK

    def run(i):
        d, rec = _chunk(20_000 + i)
        a = host.mixture_pressure(d, rec)
        b = port.mixture_pressure(d, rec)
        same = (a == b) | (np.isnan(a) & np.isnan(b))
        return int((~same).sum())

    workers = min(8, os.cpu_count() or 1)
    with ThreadPoolExecutor(max_workers=workers) as ex:
        mism = list(ex.map(run, range(nchunks)))
    assert sum(mism) == 0, f"mismatching chunks: {[i for i, m in enumerate(mism) if m]}"
