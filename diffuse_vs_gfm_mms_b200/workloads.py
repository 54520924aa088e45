"""Seeded synthetic initial fields for the DIM step.

Each generator returns ``(desc, soa)``: a descriptor (include/dimgpu.h) and a
C-contiguous FP64 SoA field of shape (V, ncell), x-fastest.  Identical arrays
are fed to the GPU path and to the CPU checkers, so no initial-condition code
path can differ between them.

Shapes follow the reference's own validation precedents (Riemann tubes,
shock-bubble, bubble clouds); all values are drawn from ``numpy`` generators
seeded per call.  Diffuse interfaces use the reference's tanh indicator
``0.5 * (1 - tanh(a * s / thickness))`` (src/setup/dim_initial_conditions.hpp:
224-236) with thickness = 2 cells and a = 2.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .abi import Desc, make_desc

ALPHA_FLOOR = 1e-6


def prim_to_cons_np(dim: int, mats, alpha: np.ndarray, rho: np.ndarray,
                    vel: np.ndarray, p: np.ndarray) -> np.ndarray:
    """Vectorised primitive -> conservative map of one field.

    alpha, rho: (nmat, n); vel: (dim, n); p: (n,).  Same formulas as
    dim::prim_to_cons (src/dim/primitives.hpp:165-212) for ideal and
    stiffened gas; used only to build initial fields.
    """
    nmat = len(mats)
    n = p.shape[0]
    out = np.empty((2 * nmat + dim, n))
    m = alpha * rho
    rho_t = np.maximum(m.sum(axis=0), 1e-12)
    rho_e = np.zeros(n)
    for k, (kind, gamma, p_inf) in enumerate(mats):
        e_k = (p + gamma * p_inf) / ((gamma - 1.0) * rho[k])
        rho_e += alpha[k] * rho[k] * e_k
    ke = 0.5 * rho_t * (vel * vel).sum(axis=0)
    out[:nmat] = m
    out[nmat:nmat + dim] = rho_t * vel
    out[nmat + dim] = rho_e + ke
    out[nmat + dim + 1:] = alpha[:nmat - 1]
    return out


# ---- portable exp / tanh --------------------------------------------------------
#
# The initial fields are also generated on the device (csrc/dim_io.cuh), and
# both generators must give the same bits.  Library exp / tanh differ between
# numpy, libm and CUDA in the last bits, so the indicator uses its own exp
# from IEEE +, -, *, / and exact scaling only (Cody-Waite reduction with
# fdlibm's split of ln 2, then a degree-13 Taylor polynomial in Horner form,
# error below 1e-16 relative), evaluated in the same order on both sides.
LN2_HI = 6.93147180369123816490e-01
LN2_LO = 1.90821492927058770002e-10
INV_LN2 = 1.44269504088896338700e+00
EXP_COEF = [1.0 / math.factorial(n) for n in range(14)]   # 1/0! .. 1/13!


def portable_exp(x):
    """exp(x) for |x| <= 700 with the device generator's arithmetic."""
    x = np.asarray(x, dtype=np.float64)
    k = np.floor(x * INV_LN2 + 0.5)
    r = (x - k * LN2_HI) - k * LN2_LO
    p = np.full_like(r, EXP_COEF[13])
    for n in range(12, -1, -1):
        p = p * r + EXP_COEF[n]
    return np.ldexp(p, k.astype(np.int64))


def portable_tanh(y):
    """tanh(y) = (e - 1) / (e + 1) with e = exp(2|y|), odd; 1 beyond |y| = 20."""
    y = np.asarray(y, dtype=np.float64)
    a = np.minimum(np.abs(y), 20.0)
    e = portable_exp(2.0 * a)
    t = (e - 1.0) / (e + 1.0)
    t = np.where(np.abs(y) > 20.0, 1.0, t)
    return np.where(y < 0.0, -t, t)


def smooth_indicator(signed_distance, thickness, sharpness=2.0):
    """Reference tanh indicator (src/setup/dim_initial_conditions.hpp:224-236),
    1 inside (s <= 0), 0 outside, with the portable tanh."""
    return 0.5 * (1.0 - portable_tanh(max(sharpness, 1e-12) * signed_distance / thickness))


def _kind(p_inf: float) -> str:
    return "stiffened_gas" if p_inf > 0.0 else "ideal_gas"


@dataclass
class SideState:
    gamma: float
    p_inf: float
    rho: float
    p: float
    u: float


def draw_side(rng: np.random.Generator) -> SideState:
    """One side of the two-material Riemann problem (config-0 distributions)."""
    gamma = rng.uniform(1.4, 6.1)
    p_inf = 0.0 if rng.uniform() < 0.5 else rng.uniform(1e8, 6e8)
    rho = math.exp(rng.uniform(math.log(0.1), math.log(1000.0)))
    p = math.exp(rng.uniform(math.log(1e4), math.log(1e9)))
    u = rng.uniform(-100.0, 100.0)
    return SideState(gamma, p_inf, rho, p, u)


def riemann(seed: int = 0, N=(1000,), axis: int = 0, position: float = 0.5,
            lengths=None, bc=None) -> tuple[Desc, np.ndarray]:
    """Two-material Riemann problem (config 0 in 1D; any axis in 2D/3D).

    Left cells hold material 0 with alpha = 1 - 1e-6 and material 1 at
    alpha = 1e-6 (its own side's density); right cells the reverse.
    """
    rng = np.random.default_rng(seed)
    L, R = draw_side(rng), draw_side(rng)
    dim = len(N)
    lengths = lengths or [1.0] * dim
    dx = [lengths[a] / N[a] for a in range(dim)]
    mats = [(_kind(L.p_inf), L.gamma, L.p_inf), (_kind(R.p_inf), R.gamma, R.p_inf)]
    desc = make_desc(dim, N, dx, mats, bc_lo=bc, bc_hi=bc)
    coords = np.meshgrid(*[(np.arange(N[a]) + 0.5) * dx[a] for a in reversed(range(dim))],
                         indexing="ij")
    x = coords[dim - 1 - axis].reshape(-1)
    left = x < position * lengths[axis]
    n = x.size
    alpha = np.empty((2, n))
    alpha[0] = np.where(left, 1.0 - ALPHA_FLOOR, ALPHA_FLOOR)
    alpha[1] = 1.0 - alpha[0]
    rho = np.empty((2, n))
    rho[0] = L.rho
    rho[1] = R.rho
    vel = np.zeros((dim, n))
    vel[axis] = np.where(left, L.u, R.u)
    p = np.where(left, L.p, R.p)
    soa = prim_to_cons_np(dim, mats, alpha, rho, vel, p)
    return desc, np.ascontiguousarray(soa)


def rankine_hugoniot(mach: float, gamma: float, rho1: float, p1: float):
    """Post-shock (rho, u, p) of a shock of Mach `mach` running into rest."""
    m2 = mach * mach
    p2 = p1 * (1.0 + 2.0 * gamma / (gamma + 1.0) * (m2 - 1.0))
    rho2 = rho1 * (gamma + 1.0) * m2 / ((gamma - 1.0) * m2 + 2.0)
    c1 = math.sqrt(gamma * p1 / rho1)
    u2 = mach * c1 * (1.0 - rho1 / rho2)
    return rho2, u2, p2


def shock_bubble_2d_setup(N=(1024, 512)):
    """Descriptor and initial-field parameters of config 1 (the one definition
    the host generator below and the device generator,
    dimgpu_init_shock_bubble, both use)."""
    nx, ny = N
    dx = [2.0 / nx, 1.0 / ny]
    mats = [("ideal_gas", 1.4, 0.0), ("ideal_gas", 1.67, 0.0)]
    desc = make_desc(2, N, dx, mats, bc_lo=["transmissive", "reflective"],
                     bc_hi=["transmissive", "reflective"])
    rho2, u2, p2 = rankine_hugoniot(1.22, 1.4, 1.0, 1.0)
    ic = dict(center=(1.0, 0.5), radius=0.25, thickness=2.0 * max(dx), sharpness=2.0, shock_x=0.6,
              zero_below=1e-14, rho_post=rho2, u_post=u2, p_post=p2, rho_pre=1.0, p_pre=1.0,
              rho_bubble=0.138, p_bubble=1.0)
    return desc, ic


def shock_bubble_2d(N=(1024, 512), seed: int = 0) -> tuple[Desc, np.ndarray]:
    """Config 1: Mach 1.22 shock at x = 0.6 hitting a light bubble.

    Domain [0,2]x[0,1]; ambient gamma 1.4, rho 1, p 1; bubble gamma 1.67,
    rho 0.138, radius 0.25 at (1, 0.5); post-shock slab x < 0.6 moving +x.
    Transmissive in x, reflective in y.  (The seed is unused: the case is
    deterministic.)  dimgpu_init_shock_bubble builds the same bits on the
    device.
    """
    desc, ic = shock_bubble_2d_setup(N)
    nx, ny = N
    dx = [desc.dx[0], desc.dx[1]]
    mats = [(desc.mat[k].kind, desc.mat[k].gamma, desc.mat[k].p_inf) for k in range(2)]
    y, x = np.meshgrid((np.arange(ny) + 0.5) * dx[1], (np.arange(nx) + 0.5) * dx[0], indexing="ij")
    x = x.reshape(-1)
    y = y.reshape(-1)
    cx, cy = ic["center"]
    sd = np.sqrt((x - cx) * (x - cx) + (y - cy) * (y - cy)) - ic["radius"]
    ab = smooth_indicator(sd, ic["thickness"], ic["sharpness"])
    ab = np.where(ab <= ic["zero_below"], 0.0, ab)
    post = x < ic["shock_x"]
    rho_amb = np.where(post, ic["rho_post"], ic["rho_pre"])
    p_amb = np.where(post, ic["p_post"], ic["p_pre"])
    u_amb = np.where(post, ic["u_post"], 0.0)
    n = x.size
    alpha = np.stack([1.0 - ab, ab])
    rho = np.stack([rho_amb, np.full(n, ic["rho_bubble"])])
    vel = np.stack([(1.0 - ab) * u_amb, np.zeros(n)])
    p = (1.0 - ab) * p_amb + ab * ic["p_bubble"]
    soa = prim_to_cons_np(2, mats, alpha, rho, vel, p)
    return desc, np.ascontiguousarray(soa)


def bubble_cloud_3d_setup(N=(512, 512, 512), seed: int = 0, nbubbles: int = 64, pulse_width: float = 0.05):
    """Descriptor, field parameters and bubbles of config 2 (shared by the
    host generator below and dimgpu_init_bubble_cloud).  Each bubble is
    (centre, radius, box_lo, box_hi): its indicator is evaluated only in the
    box of cells within 6 interface thicknesses of its surface."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = N
    dx = [1.0 / nx, 1.0 / ny, 1.0 / nz]
    mats = [("stiffened_gas", 4.4, 6e8), ("ideal_gas", 1.4, 0.0)]
    desc = make_desc(3, N, dx, mats)
    bubbles = []
    tries = 0
    while len(bubbles) < nbubbles and tries < 100000:
        tries += 1
        r = rng.uniform(0.02, 0.06)
        c = rng.uniform(r + pulse_width, 1.0 - r, size=3)
        c[1:] = rng.uniform(r, 1.0 - r, size=2)
        if all(np.linalg.norm(c - b[0]) > r + b[1] + 2 * max(dx) for b in bubbles):
            bubbles.append((c, r))
    thick = 2.0 * max(dx)
    reach = 6.0 * thick
    out = []
    for c, r in bubbles:
        lo = [max(0, int((c[a] - r - reach) / dx[a])) for a in range(3)]
        hi = [min(N[a], int((c[a] + r + reach) / dx[a]) + 1) for a in range(3)]
        out.append((tuple(float(v) for v in c), float(r), lo, hi))
    ic = dict(thickness=thick, sharpness=2.0, zero_below=1e-14, pulse_width=pulse_width, rho_liquid=1000.0,
              rho_gas=1.2, p_ambient=1e5, p_pulse=1e9)
    return desc, ic, out


def bubble_cloud_3d(N=(512, 512, 512), seed: int = 0, nbubbles: int = 64,
                    pulse_width: float = 0.05) -> tuple[Desc, np.ndarray]:
    """Config 2: 64 seeded air bubbles in water, 1e9 Pa slab at x < 0.05.

    Water: stiffened gas gamma 4.4, p_inf 6e8, rho 1000, p 1e5.  Air: ideal
    gamma 1.4, rho 1.2, p 1e5.  Radii U[0.02, 0.06], rejection-sampled to be
    non-overlapping (with one cell of clearance).  Transmissive everywhere.
    dimgpu_init_bubble_cloud builds the same bits on the device.
    """
    desc, ic, bubbles = bubble_cloud_3d_setup(N, seed, nbubbles, pulse_width)
    nx, ny, nz = N
    dx = [desc.dx[0], desc.dx[1], desc.dx[2]]
    mats = [(desc.mat[k].kind, desc.mat[k].gamma, desc.mat[k].p_inf) for k in range(2)]
    ncell = nx * ny * nz
    air = np.zeros(ncell)
    air3 = air.reshape(nz, ny, nx)
    for c, r, lo, hi in bubbles:
        zs = (np.arange(lo[2], hi[2]) + 0.5) * dx[2]
        ys = (np.arange(lo[1], hi[1]) + 0.5) * dx[1]
        xs = (np.arange(lo[0], hi[0]) + 0.5) * dx[0]
        Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
        sd = np.sqrt((X - c[0]) * (X - c[0]) + (Y - c[1]) * (Y - c[1]) + (Z - c[2]) * (Z - c[2])) - r
        ind = smooth_indicator(sd, ic["thickness"], ic["sharpness"])
        sub = air3[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]]
        np.maximum(sub, ind, out=sub)
    air[air <= ic["zero_below"]] = 0.0
    out = np.empty((2 * 2 + 3, ncell))
    chunk = nx * ny * 16
    xs_all = (np.arange(nx) + 0.5) * dx[0]
    for s in range(0, ncell, chunk):
        e = min(ncell, s + chunk)
        a1 = air[s:e]
        n = e - s
        x = np.tile(xs_all, n // nx)
        p = np.where(x < ic["pulse_width"], ic["p_pulse"], ic["p_ambient"])
        alpha = np.stack([1.0 - a1, a1])
        rho = np.stack([np.full(n, ic["rho_liquid"]), np.full(n, ic["rho_gas"])])
        vel = np.zeros((3, n))
        out[:, s:e] = prim_to_cons_np(3, mats, alpha, rho, vel, p)
    return desc, out


def single_bubble_2d(N, seed: int = 0) -> tuple[Desc, np.ndarray]:
    """A config-0 material pair with one circular bubble of the second one."""
    rng = np.random.default_rng(seed)
    A, B = draw_side(rng), draw_side(rng)
    nx, ny = N
    dx = [1.0 / nx, 1.0 / ny]
    mats = [(_kind(A.p_inf), A.gamma, A.p_inf), (_kind(B.p_inf), B.gamma, B.p_inf)]
    desc = make_desc(2, N, dx, mats)
    cx, cy = rng.uniform(0.3, 0.7, size=2)
    r = rng.uniform(0.1, 0.25)
    y, x = np.meshgrid((np.arange(ny) + 0.5) * dx[1], (np.arange(nx) + 0.5) * dx[0], indexing="ij")
    sd = (np.sqrt((x - cx) * (x - cx) + (y - cy) * (y - cy)) - r).reshape(-1)
    ab = smooth_indicator(sd, 2.0 * max(dx))
    ab = np.clip(ab, ALPHA_FLOOR, 1.0 - ALPHA_FLOOR)
    n = sd.size
    alpha = np.stack([1.0 - ab, ab])
    rho = np.stack([np.full(n, A.rho), np.full(n, B.rho)])
    vel = np.zeros((2, n))
    vel[0] = (1.0 - ab) * A.u + ab * B.u
    p = (1.0 - ab) * A.p + ab * B.p
    soa = prim_to_cons_np(2, mats, alpha, rho, vel, p)
    return desc, np.ascontiguousarray(soa)


def random_states(desc: Desc, n: int, seed: int = 0, edge_fraction: float = 0.1) -> np.ndarray:
    """Record-major random conservative states, including edge cases
    (near-zero and zero fractions, tiny or negative masses, large momenta)."""
    rng = np.random.default_rng(seed)
    nmat, dim = desc.nmat, desc.dim
    mats = [(desc.mat[k].kind, desc.mat[k].gamma, desc.mat[k].p_inf) for k in range(nmat)]
    alpha = rng.dirichlet(np.ones(nmat), size=n).T
    rho = np.exp(rng.uniform(np.log(0.1), np.log(1000.0), size=(nmat, n)))
    p = np.exp(rng.uniform(np.log(1e-2), np.log(1e9), size=n))
    vel = rng.uniform(-300.0, 300.0, size=(dim, n))
    U = prim_to_cons_np(dim, mats, alpha, rho, vel, p).T.copy()
    ne = int(edge_fraction * n)
    if ne:
        idx = rng.choice(n, size=ne, replace=False)
        q = len(idx) // 5
        if nmat > 1:
            U[idx[:q], nmat + dim + 1] = 0.0                      # alpha_0 = 0
            U[idx[q:2 * q], nmat + dim + 1] = 1e-11               # alpha below inactive floor
        U[idx[2 * q:3 * q], 0] *= -1e-3                                # negative mass
        U[idx[3 * q:4 * q], nmat + dim] *= 1e-6                        # energy deficit
        U[idx[4 * q:], nmat:nmat + dim] *= 50.0                        # large momentum
    return U


def batch_instances(n: int = 256, seed: int = 0, side_range=(64, 1024)):
    """Config 3: n 2D instances, sides log-uniform in side_range per axis,
    each a config-0 two-material Riemann problem (random axis and interface
    position) or a single bubble, all with config-0 material draws."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log(side_range[0]), np.log(side_range[1])
    out = []
    for k in range(n):
        N = (int(round(np.exp(rng.uniform(lo, hi)))), int(round(np.exp(rng.uniform(lo, hi)))))
        s = int(rng.integers(0, 2**31 - 1))
        if rng.uniform() < 0.5:
            axis = int(rng.integers(0, 2))
            out.append(riemann(seed=s, N=N, axis=axis, position=float(rng.uniform(0.2, 0.8))))
        else:
            out.append(single_bubble_2d(N, seed=s))
    return out


# ---- the single-material Euler step (model MODEL_EULER) -------------------------
#
# SoA components rho, mom[0..dim-1], E.  Shapes follow the sharp-interface
# solver's single-material validation precedents (shock tubes, blast waves);
# values are drawn per seed.

def euler_prim_to_cons(dim: int, kind: str, gamma: float, p_inf: float, rho, vel, p) -> np.ndarray:
    """prim_to_cons of the Euler step (src/euler/primitives.hpp:7-34), vectorised,
    for building initial fields only."""
    rho = np.asarray(rho, dtype=np.float64)
    n = rho.shape[0]
    out = np.empty((dim + 2, n))
    out[0] = rho
    out[1:1 + dim] = rho * vel
    e = (p + (gamma * p_inf if kind == "stiffened_gas" else 0.0)) / ((gamma - 1.0) * rho)
    out[1 + dim] = rho * e + 0.5 * rho * (vel * vel).sum(axis=0)
    return out


def euler_tube(seed: int = 0, N=(1000,), axis: int = 0, position: float = 0.5, material=None,
               bc=None, time_update: str = "split") -> tuple[Desc, np.ndarray]:
    """Single-material Riemann tube along `axis`: left / right states drawn
    per seed (rho log-U[0.1, 10] ideal, log-U[100, 1000] stiffened; p
    log-U[1e4, 1e7]; u U[-50, 50]), or Sod's tube for seed < 0."""
    dim = len(N)
    rng = np.random.default_rng(seed if seed >= 0 else 0)
    if material is None:
        material = ("ideal_gas", 1.4, 0.0) if seed < 0 or seed % 3 != 2 else ("stiffened_gas", 4.4, 6e8)
    kind, gamma, p_inf = material
    if seed < 0:
        left, right = (1.0, 0.0, 1.0), (0.125, 0.0, 0.1)
    else:
        def side():
            if kind == "stiffened_gas":
                rho = math.exp(rng.uniform(math.log(100.0), math.log(1000.0)))
            else:
                rho = math.exp(rng.uniform(math.log(0.1), math.log(10.0)))
            return rho, rng.uniform(-50.0, 50.0), math.exp(rng.uniform(math.log(1e4), math.log(1e7)))
        left, right = side(), side()
    lengths = [1.0] * dim
    dx = [lengths[a] / N[a] for a in range(dim)]
    bc = bc or ["transmissive"] * dim
    d = make_desc(dim, N, dx, [material], bc_lo=bc, bc_hi=bc, time_update=time_update, model=1)
    n = int(np.prod(N))
    idx = np.unravel_index(np.arange(n), tuple(reversed(N)))
    coord = (idx[dim - 1 - axis] + 0.5) * dx[axis]
    is_left = coord < position * lengths[axis]
    rho = np.where(is_left, left[0], right[0])
    vel = np.zeros((dim, n))
    vel[axis] = np.where(is_left, left[1], right[1])
    p = np.where(is_left, left[2], right[2])
    return d, np.ascontiguousarray(euler_prim_to_cons(dim, kind, gamma, p_inf, rho, vel, p))


def euler_blast(N=(256, 256), seed: int = 0, material=("ideal_gas", 1.4, 0.0), bc=None,
                time_update: str = "split") -> tuple[Desc, np.ndarray]:
    """Blast wave: a high-pressure sphere (circle) of radius 0.1 at a seeded
    centre near the middle of the unit box, ambient rho = 1, p = 1e5 (1e5
    ambient, 1e9 inside for stiffened water), with seeded small velocity
    noise so no axis is symmetric."""
    dim = len(N)
    rng = np.random.default_rng(seed)
    kind, gamma, p_inf = material
    dx = [1.0 / N[a] for a in range(dim)]
    bc = bc or ["transmissive"] * dim
    d = make_desc(dim, N, dx, [material], bc_lo=bc, bc_hi=bc, time_update=time_update, model=1)
    n = int(np.prod(N))
    idx = np.unravel_index(np.arange(n), tuple(reversed(N)))
    centre = 0.5 + rng.uniform(-0.05, 0.05, size=dim)
    r2 = np.zeros(n)
    for a in range(dim):
        x = (idx[dim - 1 - a] + 0.5) * dx[a]
        r2 += (x - centre[a]) ** 2
    inside = r2 < 0.1 ** 2
    stiff = kind == "stiffened_gas"
    rho = np.where(inside, 1200.0 if stiff else 1.0, 1000.0 if stiff else 0.125)
    p = np.where(inside, 1e9 if stiff else 1e6, 1e5)
    vel = rng.uniform(-1.0, 1.0, size=(dim, n))
    return d, np.ascontiguousarray(euler_prim_to_cons(dim, kind, gamma, p_inf, rho, vel, p))
