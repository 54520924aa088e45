"""Parity of the CUDA DIM step with the CPU oracle and the reference's golden
vectors, through the C-ABI (libdimgpu.so).  The bar is bit-for-bit equality;
the parity target (1e-10 relative L1 per conserved variable after 100
steps) is asserted as well so a failure says by how much it missed."""
from __future__ import annotations

import numpy as np
import pytest

from diffuse_vs_gfm_mms_b200 import abi, workloads as W
from diffuse_vs_gfm_mms_b200.dim import DimGpuError, Session, advance_one_step
from helpers import bitwise_equal, desc_from_array, load, ndiff, rel_l1

pytestmark = pytest.mark.gpu

REL_L1_TOL = 1e-10
FIELDS = load("field_steps.npz")
FIELD_KEYS = sorted({k.rsplit("_desc", 1)[0] for k in FIELDS.files if k.endswith("_desc")})


@pytest.mark.parametrize("key", FIELD_KEYS)
def test_golden_field_steps(key):
    """Whole steps against the reference's own outputs (tests/golden)."""
    d = desc_from_array(FIELDS[f"{key}_desc"])
    cfl, n = FIELDS[f"{key}_meta"]
    with Session(d, FIELDS[f"{key}_in"]) as s:
        dts = s.steps(int(n), float(cfl), 1e300)
        out = s.download()
    assert bitwise_equal(dts, FIELDS[f"{key}_dt"])
    assert ndiff(out, FIELDS[f"{key}_out"]) == 0


def _run_both(port, d, U, cfl, n):
    with Session(d, U) as s:
        dts = s.steps(n, cfl, 1e300)
        out = s.download()
    ref, rdts = port.advance(d, U, cfl, 1e300, n)
    return out, dts, ref, rdts


def test_c0_riemann_100_steps(port):
    """Config 0 (1D two-material Riemann, 1000 cells) after 100 steps."""
    d, U = W.riemann(seed=0, N=(1000,))
    out, dts, ref, rdts = _run_both(port, d, U, 0.8, 100)
    assert np.all(rel_l1(out, ref) <= REL_L1_TOL)
    assert bitwise_equal(dts, rdts)
    assert ndiff(out, ref) == 0


@pytest.mark.parametrize("seed", [1, 2, 3, 4, 5])
def test_c0_seeds(port, seed):
    d, U = W.riemann(seed=seed, N=(1000,))
    out, dts, ref, rdts = _run_both(port, d, U, 0.8, 30)
    assert ndiff(out, ref) == 0 and bitwise_equal(dts, rdts)


def test_c1_shock_bubble_100_steps(port):
    """Config 1 geometry at 128x64, 100 steps."""
    d, U = W.shock_bubble_2d(N=(128, 64))
    out, dts, ref, rdts = _run_both(port, d, U, 0.8, 100)
    assert np.all(rel_l1(out, ref) <= REL_L1_TOL)
    assert ndiff(out, ref) == 0 and bitwise_equal(dts, rdts)


def test_c1_full_size_steps(port):
    """Config 1 at its full 1024x512 size, 3 steps, bit for bit."""
    d, U = W.shock_bubble_2d(N=(1024, 512))
    out, dts, ref, rdts = _run_both(port, d, U, 0.8, 3)
    assert ndiff(out, ref) == 0 and bitwise_equal(dts, rdts)


def test_c2_cloud_small(port):
    """Config 2's generator at 24^3 (64 bubbles scaled down to 6)."""
    d, U = W.bubble_cloud_3d(N=(24, 24, 24), nbubbles=6)
    out, dts, ref, rdts = _run_both(port, d, U, 0.6, 8)
    assert ndiff(out, ref) == 0 and bitwise_equal(dts, rdts)


@pytest.mark.parametrize("N,axis", [((37, 5), 0), ((5, 131), 1), ((7, 9, 130), 2), ((3, 4, 5), 0),
                                    ((1, 40), 1), ((40, 1), 0), ((2, 9), 1), ((9, 2), 0), ((1,), 0), ((2,), 0),
                                    ((3,), 0)])
def test_edge_shapes(port, N, axis):
    """Ragged tiles, lines of 1, 2 and 3 cells, degenerate axes."""
    d, U = W.riemann(seed=11, N=N, axis=axis)
    d.bc_lo[0] = abi.BC_REFLECTIVE
    out, dts, ref, rdts = _run_both(port, d, U, 0.5, 6)
    assert ndiff(out, ref) == 0 and bitwise_equal(dts, rdts)


@pytest.mark.parametrize("bc", ["transmissive", "reflective", "nonreflective"])
@pytest.mark.parametrize("N", [(3, 7), (4, 6), (12, 10)])
def test_boundary_kinds(port, bc, N):
    d, U = W.riemann(seed=21, N=N, axis=0, bc=[bc, "reflective"])
    out, dts, ref, rdts = _run_both(port, d, U, 0.5, 5)
    assert ndiff(out, ref) == 0 and bitwise_equal(dts, rdts)


def test_three_and_four_materials(port):
    for mats in ([("ideal_gas", 1.6, 0.0), ("stiffened_gas", 2.1, 3e8), ("ideal_gas", 1.4, 0.0)],
                 [("stiffened_gas", 1.9, 5e8), ("ideal_gas", 1.3, 0.0), ("stiffened_gas", 5.5, 2e8),
                  ("ideal_gas", 2.0, 0.0)]):
        d = abi.make_desc(2, (20, 14), (0.05, 0.07), mats)
        U = W.random_states(d, d.ncell, seed=len(mats), edge_fraction=0.0).T.copy()
        out, dts, ref, rdts = _run_both(port, d, U, 0.4, 4)
        assert ndiff(out, ref) == 0 and bitwise_equal(dts, rdts)


def test_operations_match_oracle(port):
    """compute_dt_cfl, sweep_direction and apply_boundary_conditions one by one."""
    d, U = W.bubble_cloud_3d(N=(20, 18, 16), nbubbles=3)
    U, _ = port.advance(d, U, 0.6, 1e300, 2)
    with Session(d, U) as s:
        dt = s.compute_dt_cfl(0.6, 1e300)
        assert dt == port.compute_dt_cfl(d, U, 0.6, 1e300)
        assert s.compute_dt_cfl(0.6, 1e-9) == 1e-9
        cur = U
        for direction in range(3):
            s.sweep_direction(direction, dt)
            cur = port.sweep_direction(d, direction, dt, cur)
            assert ndiff(s.download(), cur) == 0
            s.apply_boundary_conditions()
            cur = port.apply_boundary_conditions(d, cur)
            assert ndiff(s.download(), cur) == 0


def test_tile_shape_does_not_change_results():
    d, U = W.bubble_cloud_3d(N=(40, 36, 30), nbubbles=4)
    outs = []
    for tiles in ([(128, 1), (64, 4), (64, 4)], [(32, 1), (32, 8), (128, 2)], [(256, 1), (16, 16), (32, 4)]):
        with Session(d, U) as s:
            for direction, (T, Wd) in enumerate(tiles):
                s.set_tile(direction, T, Wd)
            s.steps(3, 0.6, 1e300)
            outs.append(s.download())
    assert ndiff(outs[0], outs[1]) == 0 and ndiff(outs[0], outs[2]) == 0


@pytest.mark.parametrize("N", [(33, 17, 9), (130, 3), (5, 70), (300,), (2, 9)])
def test_staged_schedule_matches_oracle(port, N):
    """The staged schedule (a kernel per stage, HBM scratch) on every axis."""
    d, U = W.riemann(seed=5, N=N, axis=len(N) - 1)
    with Session(d, U) as s:
        for direction in range(d.dim):
            s.set_schedule(direction, abi.SCHEDULE_STAGED)
        dts = s.steps(6, 0.5, 1e300)
        out = s.download()
    ref, rdts = port.advance(d, U, 0.5, 1e300, 6)
    assert ndiff(out, ref) == 0 and bitwise_equal(dts, rdts)


def test_schedules_agree_on_c1():
    d, U = W.shock_bubble_2d(N=(512, 256))
    outs = []
    for sched in ((abi.SCHEDULE_FUSED,) * 2, (abi.SCHEDULE_STAGED,) * 2,
                  (abi.SCHEDULE_STAGED, abi.SCHEDULE_FUSED)):
        with Session(d, U) as s:
            for direction, k in enumerate(sched):
                s.set_schedule(direction, k)
            s.steps(5, 0.8, 1e300)
            outs.append(s.download())
    assert ndiff(outs[0], outs[1]) == 0 and ndiff(outs[0], outs[2]) == 0


def test_large_3d_lines_match_oracle(port):
    """256^3 cloud, one x sweep, then y, then z: sampled lines against the
    oracle's solve_line (a size-independent check of the full-size grid)."""
    N = (256, 256, 256)
    d, U = W.bubble_cloud_3d(N=N, nbubbles=64)
    rng = np.random.default_rng(0)
    V = d.nvar
    with Session(d, U) as s:
        dt = s.compute_dt_cfl(0.6, 1e300)
        cur = U.reshape(V, N[2], N[1], N[0])
        for direction in range(3):
            s.sweep_direction(direction, dt)
            new = s.download().reshape(V, N[2], N[1], N[0])
            for _ in range(24):
                a, b = rng.integers(0, 256, size=2)
                if direction == 0:
                    line_in, line_out = cur[:, a, b, :], new[:, a, b, :]
                elif direction == 1:
                    line_in, line_out = cur[:, a, :, b], new[:, a, :, b]
                else:
                    line_in, line_out = cur[:, :, a, b], new[:, :, a, b]
                ref = port.solve_line(d, direction, dt, d.dx[direction], line_in.T.copy())
                assert ndiff(line_out.T, ref) == 0
            s.apply_boundary_conditions()
            cur = s.download().reshape(V, N[2], N[1], N[0])
        assert np.all(np.isfinite(cur))


def test_multi_chunk_3d_lines_match_oracle(port):
    """A grid above one scratch chunk (2^24 cells): 256 x 256 x 260, so each
    axis runs as two chunks of whole lines and the second chunk's items
    index lines from L0 > 0.  Lines on both sides of every chunk seam, the
    last line and random lines of each chunk against the oracle's
    solve_line."""
    N = (256, 256, 260)
    d, U = W.bubble_cloud_3d(N=N, nbubbles=64)
    rng = np.random.default_rng(1)
    V = d.nvar
    nlines = [N[1] * N[2], N[0] * N[2], N[0] * N[1]]
    with Session(d, U) as s:
        dt = s.compute_dt_cfl(0.6, 1e300)
        cur = U.reshape(V, N[2], N[1], N[0])
        for direction in range(3):
            s.sweep_direction(direction, dt)
            new = s.download().reshape(V, N[2], N[1], N[0])
            per = (1 << 24) // N[direction]
            assert per < nlines[direction]
            picks = [0, per - 1, per, per + 1, nlines[direction] - 1]
            picks += list(rng.integers(0, per, 6)) + list(rng.integers(per, nlines[direction], 6))
            for L in picks:
                L = int(L)
                if direction == 0:
                    z, y = divmod(L, N[1])
                    line_in, line_out = cur[:, z, y, :], new[:, z, y, :]
                elif direction == 1:
                    z, x = divmod(L, N[0])
                    line_in, line_out = cur[:, z, :, x], new[:, z, :, x]
                else:
                    y, x = divmod(L, N[0])
                    line_in, line_out = cur[:, :, y, x], new[:, :, y, x]
                ref = port.solve_line(d, direction, dt, d.dx[direction], line_in.T.copy())
                assert ndiff(line_out.T, ref) == 0, (direction, L)
            s.apply_boundary_conditions()
            cur = s.download().reshape(V, N[2], N[1], N[0])
        assert np.all(np.isfinite(cur))


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_multi_chunk_step_matches_separate_calls(precision):
    """A step on a grid of several scratch chunks (256 x 256 x 260: the CFL
    runs as its own pass, every sweep as two chunks of whole lines) must
    equal, bit for bit, the same step taken as separate calls (CFL, then
    each sweep with its boundary fill), whose sweeps match the oracle line
    by line (test_multi_chunk_3d_lines_match_oracle); FP64 and mixed."""
    N = (256, 256, 260)
    d, U = W.bubble_cloud_3d(N=N, nbubbles=64)
    d.precision = precision
    with Session(d, U) as s:
        dts = s.steps(2, 0.6, 1e300)
        out = s.download()
    ref_dts = []
    with Session(d, U) as s:
        for _ in range(2):
            dt = s.compute_dt_cfl(0.6, 1e300)
            ref_dts.append(dt)
            for direction in range(3):
                s.sweep_direction(direction, dt)
                s.apply_boundary_conditions()
        ref = s.download()
    assert bitwise_equal(np.asarray(dts), np.asarray(ref_dts))
    assert ndiff(out, ref) == 0


def test_repeatable():
    d, U = W.shock_bubble_2d(N=(256, 128))
    res = []
    for _ in range(2):
        with Session(d, U) as s:
            s.steps(10, 0.8, 1e300)
            res.append(s.download())
    assert ndiff(res[0], res[1]) == 0


def test_stateless_drop_in_matches_session(port):
    d, U = W.shock_bubble_2d(N=(64, 32))
    r = advance_one_step(U, d, 0.8, 1e300, timings=True)
    ref, rdt = port.advance(d, U, 0.8, 1e300, 1)
    assert r.dt == rdt[0] and ndiff(r.U_new, ref) == 0
    assert r.phase_timings["sweep_seconds"] > 0
    r2 = advance_one_step(r.U_new, d, 0.8, 1e-7)
    assert r2.dt == 1e-7


def test_dt_max_caps_the_step(port):
    d, U = W.riemann(seed=2, N=(200,))
    with Session(d, U) as s:
        dts = s.steps(5, 0.8, 1e-9)
    assert np.all(dts == 1e-9)


def test_totals_match_oracle(port):
    d, U = W.bubble_cloud_3d(N=(20, 20, 20), nbubbles=3)
    with Session(d, U) as s:
        got = s.totals()
    want = np.zeros_like(got)
    import ctypes as C
    from diffuse_vs_gfm_mms_b200.abi import dptr
    assert port.lib.oracle_totals(C.byref(d), dptr(np.ascontiguousarray(U)), dptr(want)) == 0
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-300)


def test_errors_are_statuses():
    with pytest.raises(DimGpuError) as e:
        Session(abi.make_desc(1, [8], [0.1], [("tait", 7.0, 0.0)]))
    assert e.value.status == abi.E_UNSUPPORTED_EOS
    d, U = W.riemann(seed=1, N=(50,))
    with Session(d) as s:
        with pytest.raises(DimGpuError) as e:
            s.upload(U[:, :10])
        assert e.value.status == abi.E_INVALID_ARG
        s.upload(U)
        with pytest.raises(DimGpuError):
            s.step(0.0, 1.0)
        with pytest.raises(DimGpuError):
            s.step(0.5, -1.0)
        with pytest.raises(DimGpuError):
            s.set_tile(0, 4, 1)
    bad = abi.make_desc(1, [8], [0.1], [("ideal_gas", 1.0, 0.0)])
    with pytest.raises(DimGpuError):
        Session(bad)


def test_autotuned_schedule_gives_the_same_result(tmp_path, monkeypatch):
    from diffuse_vs_gfm_mms_b200 import autotune
    monkeypatch.setenv("DIMGPU_TUNE_CACHE", str(tmp_path / "tune.json"))
    d, U = W.bubble_cloud_3d(N=(48, 40, 36), nbubbles=4)
    choice = autotune.tune(d, U, cfl=0.6, repeats=1, force=True)
    assert set(choice) == {0, 1, 2}
    assert autotune.tune(d, U, cfl=0.6) == choice          # served from the cache
    with Session(d, U) as s:
        autotune.apply(s, choice)
        s.steps(3, 0.6, 1e300)
        tuned = s.download()
    with Session(d, U) as s:
        s.steps(3, 0.6, 1e300)
        plain = s.download()
    assert ndiff(tuned, plain) == 0


@pytest.mark.parametrize("gen", [
    lambda: W.riemann(seed=3, N=(500,)),
    lambda: W.shock_bubble_2d(N=(160, 80)),
    lambda: W.bubble_cloud_3d(N=(24, 20, 16), nbubbles=3),
])
def test_boundary_flux_matches_oracle(port, gen):
    """The device boundary-flux integrand (parallel sums) against the
    reference-order sums of the oracle."""
    d, U = gen()
    with Session(d, U) as s:
        s.steps(3, 0.6, 1e300)
        got = s.boundary_flux()
        state = s.download()
    want = port.boundary_flux(d, state)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())
