"""The kernels' per-state arithmetic and five-stage line decomposition
(csrc/dim_physics.h, csrc/dim_line.h) compiled for the host with g++ and
checked bit for bit against the golden vectors and the oracle.  This covers
the accelerated bisection and the lazy repair_state on CPU, with no GPU."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from diffuse_vs_gfm_mms_b200 import abi, workloads as W
from diffuse_vs_gfm_mms_b200.abi import dptr
from helpers import bitwise_equal, desc_from_array, load, ndiff

KAT = load("kat_records.npz")
KAT_KEYS = sorted({k.rsplit("_desc", 1)[0] for k in KAT.files if k.endswith("_desc")})


class Host:
    """ctypes view of tests/_build/libphyshost.so with the oracle's API."""

    def __init__(self):
        from conftest import build_host_harness
        self.lib = C.CDLL(build_host_harness())

    def _rec(self, name, d, inp, width, *extra):
        inp = np.ascontiguousarray(inp, dtype=np.float64)
        out = np.zeros((inp.shape[0], width))
        rc = getattr(self.lib, "host_" + name)(C.byref(d), C.c_int(inp.shape[0]), *extra, dptr(inp), dptr(out))
        assert rc == 0
        return out

    def cons_to_prim(self, d, U):
        return self._rec("cons_to_prim", d, U, 2 * d.nmat + d.dim + 1)

    def prim_to_cons(self, d, P):
        return self._rec("prim_to_cons", d, P, 2 * d.nmat + d.dim)

    def repair_state(self, d, U):
        U = np.array(U, dtype=np.float64, copy=True)
        assert self.lib.host_repair_state(C.byref(d), C.c_int(U.shape[0]), dptr(U)) == 0
        return U

    def mixture_pressure(self, d, rec):
        return self._rec("mixture_pressure", d, rec, 1)[:, 0]

    def mixture_sound_speed(self, d, rec):
        return self._rec("mixture_sound_speed", d, rec, 1)[:, 0]

    def alpha_rhs(self, d, P):
        return self._rec("alpha_rhs", d, P, d.nmat)

    def hllc(self, d, direction, UL, UR):
        UL = np.ascontiguousarray(UL)
        UR = np.ascontiguousarray(UR)
        out = np.zeros((UL.shape[0], d.nmat + d.dim + 2))
        assert self.lib.host_hllc(C.byref(d), C.c_int(UL.shape[0]), C.c_int(direction), dptr(UL), dptr(UR),
                                  dptr(out)) == 0
        return out

    def sweep_direction(self, d, direction, dt, U):
        U = np.ascontiguousarray(U)
        out = np.empty_like(U)
        assert self.lib.host_sweep_direction(C.byref(d), C.c_int(direction), C.c_double(dt), dptr(U),
                                             dptr(out)) == 0
        return out


@pytest.fixture(scope="module")
def host():
    return Host()


@pytest.mark.parametrize("key", KAT_KEYS)
def test_kat_records(host, key):
    d = desc_from_array(KAT[f"{key}_desc"])
    U, U2 = KAT[f"{key}_U"], KAT[f"{key}_U2"]
    P = KAT[f"{key}_cons_to_prim"]
    assert bitwise_equal(host.cons_to_prim(d, U), P)
    assert bitwise_equal(host.prim_to_cons(d, P), KAT[f"{key}_prim_to_cons"])
    assert bitwise_equal(host.repair_state(d, U), KAT[f"{key}_repair"])
    assert bitwise_equal(host.mixture_pressure(d, KAT[f"{key}_pressure_rec"]), KAT[f"{key}_pressure"])
    for lm in (0, 1, 2):
        d.lambda_model = lm
        assert bitwise_equal(host.alpha_rhs(d, P), KAT[f"{key}_alpha_rhs{lm}"])
        assert bitwise_equal(host.mixture_sound_speed(d, KAT[f"{key}_sound_rec"]), KAT[f"{key}_sound{lm}"])
        assert bitwise_equal(host.hllc(d, d.dim - 1, U, U2), KAT[f"{key}_hllc{lm}"])


MATS = [
    [("stiffened_gas", 4.4, 6e8), ("ideal_gas", 1.4, 0.0)],
    [("ideal_gas", 1.4, 0.0), ("ideal_gas", 1.67, 0.0)],
    [("ideal_gas", 1.6, 0.0), ("stiffened_gas", 2.1, 3e8), ("ideal_gas", 1.4, 0.0)],
    [("stiffened_gas", 1.9, 5e8), ("ideal_gas", 1.3, 0.0), ("stiffened_gas", 5.5, 2e8), ("ideal_gas", 2.0, 0.0)],
]


@pytest.mark.parametrize("mi", range(len(MATS)))
@pytest.mark.parametrize("dim", (1, 2, 3))
def test_random_states_against_oracle(host, port, dim, mi):
    """40k random states per case (edge cases included): the accelerated
    bisection and the lazy repair return exactly the literal results."""
    d = abi.make_desc(dim, [8] * dim, [0.1] * dim, MATS[mi])
    U = W.random_states(d, 40000, seed=1000 + 10 * dim + mi)
    assert ndiff(host.cons_to_prim(d, U), port.cons_to_prim(d, U)) == 0
    assert ndiff(host.repair_state(d, U), port.repair_state(d, U)) == 0
    P = port.cons_to_prim(d, U)
    assert ndiff(host.prim_to_cons(d, P), port.prim_to_cons(d, P)) == 0


def test_pressure_near_termination_window(host, port):
    """States whose bisection stops within a few ulps of the termination
    threshold: the guard band must send them to the literal residual."""
    rng = np.random.default_rng(5)
    d = abi.make_desc(1, [8], [0.1], MATS[0])
    n = 20000
    a0 = rng.uniform(0, 1, n)
    rho = np.exp(rng.uniform(np.log(0.1), np.log(1000), (2, n)))
    p = np.exp(rng.uniform(np.log(1e-6), np.log(1e10), n))
    g, pinf = np.array([4.4, 1.4]), np.array([6e8, 0.0])
    ie = (a0 * (p + g[0] * pinf[0]) / (g[0] - 1) + (1 - a0) * p / (g[1] - 1))
    rt = a0 * rho[0] + (1 - a0) * rho[1]
    # perturb the energy by about one termination threshold
    e = ie / rt * (1 + rng.uniform(-3e-10, 3e-10, n))
    rec = np.stack([rt, e, a0, 1 - a0, rho[0], rho[1]], axis=1)
    assert ndiff(host.mixture_pressure(d, rec), port.mixture_pressure(d, rec)) == 0


SWEEP_CASES = [
    ("c0", lambda: W.riemann(seed=1, N=(1000,))),
    ("c1", lambda: W.shock_bubble_2d(N=(40, 20))),
    ("c2", lambda: W.bubble_cloud_3d(N=(10, 10, 10), nbubbles=2)),
    ("n2", lambda: W.riemann(seed=3, N=(2, 5), axis=1)),
    ("n1", lambda: W.riemann(seed=3, N=(3, 1, 4), axis=0)),
]


@pytest.mark.parametrize("name,gen", SWEEP_CASES)
def test_sweep_stages_against_oracle(host, port, name, gen):
    d, U = gen()
    U, _ = port.advance(d, U, 0.8, 1e300, 3)
    dt = port.compute_dt_cfl(d, U, 0.8, 1e300)
    for direction in range(d.dim):
        assert ndiff(host.sweep_direction(d, direction, dt, U), port.sweep_direction(d, direction, dt, U)) == 0


def _divisors():
    rng = np.random.default_rng(7)
    ds = {1, 2, 3, 5, 6, 7, 31, 518, 1030, 1024, 2048, (1 << 24) + 3, (1 << 31) - 1, 1 << 31,
          (1 << 31) + 1, (1 << 32) - 1}
    ds |= {(1 << k) + e for k in range(1, 32) for e in (-1, 0, 1) if 1 <= (1 << k) + e < (1 << 32)}
    ds |= set(int(v) for v in rng.integers(1, 1 << 32, 200, dtype=np.uint64))
    ds |= set(int(v) for v in rng.integers(1, 5000, 200))
    return sorted(ds)


def test_fastdiv_divides_every_index_exactly(host):
    """The staged kernels split item and line indices with FastDiv
    (csrc/fastdiv.h): quotient and remainder equal integer division for
    divisors over the whole 32-bit range and dividends at 0, 2^32 - 1, near
    multiples of the divisor and at random."""
    rng = np.random.default_rng(11)
    f = host.lib.host_fastdiv
    f.argtypes = [C.c_uint, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    for d in _divisors():
        k = rng.integers(0, (1 << 32) // d, 64, dtype=np.uint64)
        near = np.concatenate([k * d, k * d + d - 1, k * d - 1, k * d + 1])
        x = np.concatenate([near, rng.integers(0, 1 << 32, 2048, dtype=np.uint64),
                            np.array([0, 1, d - 1, d, (1 << 32) - 1], dtype=np.uint64)])
        x = x[x < (1 << 32)].astype(np.uint32)
        q = np.empty_like(x)
        r = np.empty_like(x)
        assert f(d, x.size, x.ctypes.data, q.ctypes.data, r.ctypes.data) == 0
        xx = x.astype(np.uint64)
        assert np.array_equal(q.astype(np.uint64), xx // d), d
        assert np.array_equal(r.astype(np.uint64), xx % d), d


@pytest.mark.parametrize("lam", (0, 1, 2))
@pytest.mark.parametrize("mi", range(len(MATS)))
def test_sound_speed_reuses_stage_a_speeds_bit_for_bit(host, mi, lam):
    """The fused CFL passes stage A's alpha-RHS material sound speeds into the
    mixture sound speed, which takes them where both evaluate
    material_sound_speed on the same arguments: the result must equal the
    one that evaluates every speed itself, bit for bit, for every λ-model,
    including densities and pressures at and around the two clamps' floors
    (1e-12, 1e-10), zero, negative and non-finite."""
    mats = MATS[mi]
    nm = len(mats)
    d = abi.make_desc(dim=1, N=(8,), dx=(1.0,), materials=mats, lambda_model=lam)
    rng = np.random.default_rng(100 + 10 * mi + lam)
    n = 20000
    edge = np.array([0.0, -1.0, 1e-13, 1e-12, 5e-11, 1e-10, np.nextafter(1e-10, 0), np.nextafter(1e-10, 1),
                     2e-10, np.inf, np.nan, 1.0])
    rec = np.empty((n, 2 + 2 * nm))
    rec[:, 0] = np.exp(rng.uniform(np.log(1e-3), np.log(2e3), n))
    rec[:, 1] = np.exp(rng.uniform(np.log(1e3), np.log(1e10), n))
    a = rng.dirichlet(np.ones(nm), n)
    rec[:, 2:2 + nm] = a
    rec[:, 2 + nm:] = np.exp(rng.uniform(np.log(1e-2), np.log(2e3), (n, nm)))
    pick = rng.random(n) < 0.3
    rec[pick, 1] = rng.choice(edge, pick.sum())
    for k in range(nm):
        pick = rng.random(n) < 0.2
        rec[pick, 2 + nm + k] = rng.choice(edge, pick.sum())
    rec = np.ascontiguousarray(rec)
    w = np.empty(n)
    wo = np.empty(n)
    f = host.lib.host_sound_ck
    assert f(C.byref(d), C.c_int(n), dptr(rec), dptr(w), dptr(wo)) == 0
    assert bitwise_equal(w, wo)
