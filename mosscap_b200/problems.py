"""Seeded synthetic initial conditions for the Euler-step workloads.

Each generator returns a :class:`Problem`: the grid/scheme description and a
conserved state ``Q`` of shape ``[var][zc][yc][xc]`` (the reference layout,
``source/State.hpp``) filled on every cell, ghosts included, from primitives
with the reference's ``prim_to_cons`` expression order (``source/Eos.hpp:81-99``),
the way the reference's problem generators do (e.g.
``source/ProblemGenerator/ShockTube2d.cpp:24-47``). Ghost cells still have to
be filled with the boundary conditions before the first step.

Cell centres follow ``State::get_pos`` (``source/State.hpp:123-134``):
``x = i*dx - (ng - 0.5)*dx + x_start``.
"""
from __future__ import annotations

from dataclasses import dataclass, field, replace
from typing import List, Optional, Sequence, Tuple

import numpy as np


@dataclass
class Problem:
    name: str
    num_dim: int
    nx: int
    ny: int = 1
    nz: int = 1
    ng: int = 3
    num_tracers: int = 0
    dx: float = 1.0
    loc: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    bc: Tuple[str, ...] = ("zerograd",) * 6
    bc_const: Optional[np.ndarray] = None
    reconstruction: str = "muscl"
    slope_limiter: str = "monotonizedcentral"
    riemann_solver: str = "hll"
    time_stepper: str = "ssprk3"
    gamma: float = 1.4
    max_cfl: float = 0.8
    max_time: float = 1.0
    output_delta: float = 0.1
    # acceleration of the gravity source term (sources.gravity.x/y/z of the
    # reference's configuration); None: no source term
    gravity: Optional[Tuple[float, float, float]] = None
    # equation of state (eos.type of the reference's configuration): "ideal",
    # "analyticlteh" or "tabulatedlteh"; eos.avg_mass,
    # eos.include_ionisation_energy and, for the tabulated kind, the table
    # (log_eint_rho_start, log_eint_rho_step, log_rho_start, log_rho_step,
    # y_table [n_rho, n_eint_rho], log_T_table [n_rho, n_eint_rho])
    eos: str = "ideal"
    eos_avg_mass: float = 1.0
    eos_ionisation: bool = False
    eos_table: Optional[tuple] = field(default=None, repr=False)
    Q: Optional[np.ndarray] = field(default=None, repr=False)

    @property
    def n_vars(self) -> int:
        return 2 + self.num_dim + self.num_tracers

    @property
    def shape(self) -> Tuple[int, int, int, int]:
        xc = self.nx + 2 * self.ng
        yc = self.ny + 2 * self.ng if self.num_dim > 1 else 1
        zc = self.nz + 2 * self.ng if self.num_dim > 2 else 1
        return (self.n_vars, zc, yc, xc)

    @property
    def interior_cells(self) -> int:
        n = self.nx
        if self.num_dim > 1:
            n *= self.ny
        if self.num_dim > 2:
            n *= self.nz
        return n

    def scheme_fields(self) -> dict:
        keys = ("num_dim", "nx", "ny", "nz", "ng", "num_tracers", "dx", "loc", "bc",
                "bc_const", "reconstruction", "slope_limiter", "riemann_solver",
                "time_stepper", "gamma", "max_cfl", "max_time", "output_delta")
        return {k: getattr(self, k) for k in keys}

    def with_scheme(self, **kw) -> "Problem":
        return replace(self, **kw)


def cell_centres(num_dim: int, n: int, ng: int, dx: float, start: float) -> np.ndarray:
    """Centres of all cells along one axis, ghosts included (State::get_pos)."""
    i = np.arange(n + 2 * ng, dtype=np.float64)
    ghost_offset = -(ng - 0.5) * dx
    return i * dx + ghost_offset + start


def prim_to_cons(num_dim: int, gamma: float, w: np.ndarray) -> np.ndarray:
    """Vectorised ``prim_to_cons`` (source/Eos.hpp:81-99) with the same
    evaluation order; tracer fields (beyond the hydro vars) become mass
    densities ``rho * s``."""
    q = np.empty_like(w)
    rho = w[0]
    q[0] = rho
    q[1] = rho * w[1]
    v2 = w[1] * w[1]
    if num_dim > 1:
        q[2] = rho * w[2]
        v2 = v2 + w[2] * w[2]
    if num_dim > 2:
        q[3] = rho * w[3]
        v2 = v2 + w[3] * w[3]
    e_kin = (0.5 * rho) * v2
    e_int = w[1 + num_dim] / (gamma - 1.0)
    q[1 + num_dim] = e_int + e_kin
    for t in range(2 + num_dim, w.shape[0]):
        q[t] = rho * w[t]
    return q


def sod_1d(n: int = 1024, ng: int = 3) -> Problem:
    """Sod shock tube on [0,1]: (rho,u,p) = (1,0,1) for x < 0.5 and
    (0.125,0,0.1) otherwise; gamma 1.4, MUSCL + minmod, HLLC, SSPRK2 (the
    reference's ``rk2``), CFL 0.8, zero-gradient ("outflow") ends, to t=0.2."""
    dx = 1.0 / n
    x = cell_centres(1, n, ng, dx, 0.0)
    w = np.zeros((3, 1, 1, x.size))
    left = x < 0.5
    w[0, 0, 0] = np.where(left, 1.0, 0.125)
    w[2, 0, 0] = np.where(left, 1.0, 0.1)
    p = Problem("sod_1d", 1, n, ng=ng, dx=dx, bc=("zerograd",) * 6, reconstruction="muscl",
                slope_limiter="minmod", riemann_solver="hllc", time_stepper="rk2", gamma=1.4,
                max_cfl=0.8, max_time=0.2, output_delta=0.1)
    p.Q = prim_to_cons(1, p.gamma, w)
    return p


def kelvin_helmholtz_2d(n: int = 2048, ng: int = 3, seed: int = 0, noise: float = 1e-3) -> Problem:
    """Periodic Kelvin-Helmholtz on [0,1]^2: rho = 2 and vx = +0.5 in the band
    |y - 0.5| < 0.25, rho = 1 and vx = -0.5 outside, p = 2.5, gamma = 5/3,
    vy = 0.01 sin(4 pi x) + noise * U(-1, 1) from ``seed``; WENO5-Z + HLLC,
    SSPRK3, CFL 0.4. max_time and the output interval are set large so that
    no output clamp shortens a step (the workload is a fixed step count)."""
    dx = 1.0 / n
    x = cell_centres(2, n, ng, dx, 0.0)
    y = cell_centres(2, n, ng, dx, 0.0)
    X, Y = np.meshgrid(x, y, indexing="xy")  # [j][i]
    band = np.abs(Y - 0.5) < 0.25
    rng = np.random.default_rng(seed)
    w = np.empty((4, 1, y.size, x.size))
    w[0, 0] = np.where(band, 2.0, 1.0)
    w[1, 0] = np.where(band, 0.5, -0.5)
    w[2, 0] = 0.01 * np.sin(4.0 * np.pi * X) + noise * rng.uniform(-1.0, 1.0, size=X.shape)
    w[3, 0] = 2.5
    gamma = 5.0 / 3.0
    p = Problem("kelvin_helmholtz_2d", 2, n, n, ng=ng, dx=dx, bc=("periodic",) * 6,
                reconstruction="weno5z", slope_limiter="monotonizedcentral",
                riemann_solver="hllc", time_stepper="ssprk3", gamma=gamma, max_cfl=0.4,
                max_time=1e30, output_delta=1e30)
    p.Q = prim_to_cons(2, gamma, w)
    return p


def sedov_3d(n: int = 512, ng: int = 3, e_blast: float = 1.0, max_cfl: float = 0.8 / 3.0) -> Problem:
    """Sedov-style blast on [-1,1]^3: rho = 1, ambient p = 1e-5, gamma = 1.4;
    energy ``e_blast`` deposited uniformly as internal energy in the cells whose
    centre lies within r < 3 dx. PPM (MC limiter) + HLL, SSPRK3, zero-gradient
    boundaries, to t = 0.05.

    The CFL number defaults to 0.8 / 3: the reference's CFL bound is
    per direction (source/Hydro.cpp:192-206) while its 3D update is unsplit,
    and at 0.8 the reference itself produces negative pressures in the first
    step and non-finite values from then on at every resolution >= 32^3."""
    dx = 2.0 / n
    c = cell_centres(3, n, ng, dx, -1.0)
    Z, Y, X = np.meshgrid(c, c, c, indexing="ij")
    r = np.sqrt(X * X + Y * Y + Z * Z)
    hot = r < 3.0 * dx
    ng3 = slice(ng, ng + n)
    n_in = int(np.count_nonzero(hot[ng3, ng3, ng3]))
    gamma = 1.4
    de = e_blast / (n_in * dx ** 3)
    w = np.zeros((5, c.size, c.size, c.size))
    w[0] = 1.0
    w[4] = np.where(hot, 1e-5 + (gamma - 1.0) * de, 1e-5)
    p = Problem("sedov_3d", 3, n, n, n, ng=ng, dx=dx, loc=(-1.0, -1.0, -1.0),
                bc=("zerograd",) * 6, reconstruction="ppm", slope_limiter="monotonizedcentral",
                riemann_solver="hll", time_stepper="ssprk3", gamma=gamma, max_cfl=max_cfl,
                max_time=0.05, output_delta=0.05)
    p.Q = prim_to_cons(3, gamma, w)
    return p


def riemann_batch(seed: int = 0, n1d: int = 2048, n2d: int = 2048, riemann_solver: str = "hllc",
                  min1d: int = 64, max1d: int = 4096, min2d: int = 64, max2d: int = 512,
                  max_cfl: float = 0.8, steps_time: float = 1e30, ng: int = 3) -> List[Problem]:
    """Independent Riemann problems of uneven size from one seed.

    1D: a shock tube with cell count log-uniform in [min1d, max1d] on [0,1],
    left / right states split at x = 0.5. 2D: a four-quadrant problem on
    [0,1]^2, side log-uniform in [min2d, max2d], one state per quadrant
    around (0.5, 0.5). Every state draws rho and p log-uniform in
    [1e-3, 10] and each velocity component uniform in [-2, 2]; gamma 1.4,
    MUSCL (minmod), ``riemann_solver``, SSPRK2 (``rk2``), zero-gradient
    boundaries, CFL ``max_cfl`` per problem (its own dt). The 2D CFL is
    ``max_cfl / 2``: the reference's CFL bound is per direction while its
    update is unsplit."""
    rng = np.random.default_rng(seed)
    out: List[Problem] = []

    def state(nd):
        rho = float(np.exp(rng.uniform(np.log(1e-3), np.log(10.0))))
        p = float(np.exp(rng.uniform(np.log(1e-3), np.log(10.0))))
        v = [float(x) for x in rng.uniform(-2.0, 2.0, size=nd)]
        return rho, v, p

    for _ in range(n1d):
        n = int(round(np.exp(rng.uniform(np.log(min1d), np.log(max1d)))))
        dx = 1.0 / n
        x = cell_centres(1, n, ng, dx, 0.0)
        (rl, vl, pl), (rr, vr, pr) = state(1), state(1)
        left = x < 0.5
        w = np.empty((3, 1, 1, x.size))
        w[0, 0, 0] = np.where(left, rl, rr)
        w[1, 0, 0] = np.where(left, vl[0], vr[0])
        w[2, 0, 0] = np.where(left, pl, pr)
        p = Problem(f"tube_{len(out)}", 1, n, ng=ng, dx=dx, bc=("zerograd",) * 6, reconstruction="muscl",
                    slope_limiter="minmod", riemann_solver=riemann_solver, time_stepper="rk2", gamma=1.4,
                    max_cfl=max_cfl, max_time=steps_time, output_delta=steps_time)
        p.Q = prim_to_cons(1, 1.4, w)
        out.append(p)
    for _ in range(n2d):
        n = int(round(np.exp(rng.uniform(np.log(min2d), np.log(max2d)))))
        dx = 1.0 / n
        c = cell_centres(2, n, ng, dx, 0.0)
        X, Y = np.meshgrid(c, c, indexing="xy")
        quad = (X >= 0.5).astype(int) + 2 * (Y >= 0.5).astype(int)
        w = np.empty((4, 1, c.size, c.size))
        for qd in range(4):
            rho, v, pr = state(2)
            m = quad == qd
            w[0, 0][m] = rho
            w[1, 0][m] = v[0]
            w[2, 0][m] = v[1]
            w[3, 0][m] = pr
        p = Problem(f"quadrant_{len(out)}", 2, n, n, ng=ng, dx=dx, bc=("zerograd",) * 6, reconstruction="muscl",
                    slope_limiter="minmod", riemann_solver=riemann_solver, time_stepper="rk2", gamma=1.4,
                    max_cfl=max_cfl / 2.0, max_time=steps_time, output_delta=steps_time)
        p.Q = prim_to_cons(2, 1.4, w)
        out.append(p)
    return out


def random_state(num_dim: int, nx: int, ny: int = 1, nz: int = 1, ng: int = 3,
                 num_tracers: int = 0, seed: int = 0, jumps: bool = True,
                 gamma: float = 1.4, vmax: float = 1.0) -> np.ndarray:
    """Smooth random fields plus (optionally) a few random discontinuities;
    positive density and pressure. Used by parity tests to exercise every
    branch of the limiters and Riemann solvers."""
    rng = np.random.default_rng(seed)
    shape = (1 if num_dim < 3 else nz + 2 * ng, 1 if num_dim < 2 else ny + 2 * ng, nx + 2 * ng)
    nv = 2 + num_dim + num_tracers
    w = np.empty((nv,) + shape)

    def smooth():
        zz, yy, xx = np.meshgrid(*[np.linspace(0, 1, s) for s in shape], indexing="ij")
        f = np.zeros(shape)
        for _ in range(3):
            k = rng.uniform(0.5, 4.0, size=3)
            ph = rng.uniform(0, 2 * np.pi, size=3)
            f += rng.uniform(0.2, 1.0) * np.sin(2 * np.pi * k[0] * xx + ph[0]) \
                * np.cos(2 * np.pi * k[1] * yy + ph[1]) * np.cos(2 * np.pi * k[2] * zz + ph[2])
        return f

    def jumpy():
        f = np.zeros(shape)
        if jumps:
            for _ in range(3):
                ax = rng.integers(0, num_dim)
                pos = rng.uniform(0.2, 0.8) * shape[2 - ax]
                idx = np.indices(shape)[2 - ax]
                f += np.where(idx < pos, rng.uniform(-0.5, 0.5), 0.0)
        return f

    w[0] = np.exp(0.5 * smooth() + jumpy())
    for d in range(num_dim):
        w[1 + d] = vmax * (0.5 * smooth() + jumpy())
    w[1 + num_dim] = np.exp(0.5 * smooth() + jumpy())
    for t in range(num_tracers):
        w[2 + num_dim + t] = 0.5 + 0.4 * np.tanh(smooth() + jumpy())
    return prim_to_cons(num_dim, gamma, w)


# ---------------------------------------------------------------------------
# Partially ionised hydrogen in local thermodynamic equilibrium (SI units), for
# the non-ideal EOS kinds (source/AnalyticLteH.hpp, source/TabulatedLteH.hpp)
# ---------------------------------------------------------------------------
H_MASS = 1.6737830080950003e-27  # [kg]
K_B = 1.380649e-23               # [J / K]
CHI_H = 2.178710282685096e-18    # [J]


def saha_y(nhtot, temp):
    """Ionisation fraction of hydrogen from the Saha equation (the
    reference's y_from_nhtot, source/AnalyticLteH.hpp:10-20)."""
    X = 2.4146830395719654e+21 * np.power(temp, 1.5) * np.exp(-157763.42386247337 / temp)
    return 0.5 * (-X + np.sqrt(X * X + 4 * nhtot * X)) / nhtot


def lte_internal_energy(rho, temp, gamma, avg_mass=1.0, ionisation=False):
    """Internal energy density [J / m^3] of LTE hydrogen at (rho, T)."""
    y = saha_y(rho / (H_MASS * avg_mass), temp)
    e = rho * (K_B / H_MASS) / avg_mass * (1.0 + y) * temp / (gamma - 1.0)
    if ionisation:
        e = e + y * rho * (CHI_H / H_MASS) / avg_mass
    return e


def lte_h_table(n_eint_rho: int = 96, n_rho: int = 48, gamma: float = 5.0 / 3.0,
                log_rho_range=(-10.0, -5.0), log_t_range=(3.4, 4.6)):
    """A tabulated LTE hydrogen EOS in the layout the reference reads
    (source/TabulatedLteH.hpp:30-58): y and log10 T on a grid uniform in
    log10(eint / rho) and log10(rho), eint including the ionisation energy.
    Each entry solves eint / rho = (k_B / m_H) (1 + y) T / (gamma - 1) +
    (chi_H / m_H) y with y from Saha, by bisection in log T."""
    log_rho = log_rho_range[0] + (log_rho_range[1] - log_rho_range[0]) * np.arange(n_rho) / (n_rho - 1)
    t_lo, t_hi = 10.0 ** log_t_range[0], 10.0 ** log_t_range[1]
    e_lo = lte_internal_energy(10.0 ** log_rho[-1], t_lo, gamma, ionisation=True) / 10.0 ** log_rho[-1]
    e_hi = lte_internal_energy(10.0 ** log_rho[0], t_hi, gamma, ionisation=True) / 10.0 ** log_rho[0]
    lx0, lx1 = np.log10(e_lo), np.log10(e_hi)
    log_e = lx0 + (lx1 - lx0) * np.arange(n_eint_rho) / (n_eint_rho - 1)
    R = 10.0 ** log_rho[:, None] * np.ones((1, n_eint_rho))
    target = 10.0 ** log_e[None, :] * np.ones((n_rho, 1))
    a = np.full(R.shape, np.log10(t_lo) - 1.0)
    b = np.full(R.shape, np.log10(t_hi) + 1.0)
    for _ in range(200):
        m = 0.5 * (a + b)
        f = lte_internal_energy(R, 10.0 ** m, gamma, ionisation=True) / R - target
        a = np.where(f < 0.0, m, a)
        b = np.where(f < 0.0, b, m)
    logt = 0.5 * (a + b)
    y = saha_y(R / H_MASS, 10.0 ** logt)
    return (float(lx0), float((lx1 - lx0) / (n_eint_rho - 1)), float(log_rho[0]),
            float((log_rho[-1] - log_rho[0]) / (n_rho - 1)), y, logt)


def lte_hydrogen(num_dim: int, n: int, seed: int = 0, eos: str = "analyticlteh", gamma: float = 5.0 / 3.0,
                 avg_mass: float = 1.0, ionisation: bool = False, ng: int = 3, table=None) -> Problem:
    """Partially ionised hydrogen in LTE: smooth seeded fields of density
    (1e-9 .. 1e-6 kg / m^3), temperature (5e3 .. 2e4 K) and velocity (up to
    5 km / s) on a periodic box of n cells per axis of 10 km; the energy
    includes the ionisation energy when the EOS does (ionisation for the
    analytic kind, always for the tabulated kind). MUSCL (MC) + HLLC, SSPRK3."""
    rng = np.random.default_rng(seed)
    dx = 1.0e4
    shape = tuple([n + 2 * ng] * num_dim)

    def smooth_field():
        c = (np.arange(n + 2 * ng) - ng + 0.5) / n
        grids = np.meshgrid(*([c] * num_dim), indexing="ij")
        f = np.zeros(shape)
        for _ in range(3):
            k = rng.integers(1, 4, size=num_dim)
            ph = rng.uniform(0, 2 * np.pi, size=num_dim)
            term = np.ones(shape)
            for a in range(num_dim):
                term = term * np.sin(2 * np.pi * k[a] * grids[a] + ph[a])
            f = f + rng.uniform(0.3, 1.0) * term
        return f / (np.abs(f).max() + 1e-300)

    rho = 10.0 ** (-7.5 + 1.5 * smooth_field())
    temp = 10.0 ** (4.0 + 0.3 * smooth_field())
    vel = [5.0e3 * smooth_field() for _ in range(num_dim)]
    with_ion = ionisation or eos == "tabulatedlteh"
    eint = lte_internal_energy(rho, temp, gamma, avg_mass, with_ion)
    ekin = 0.5 * rho * sum(v * v for v in vel)
    q = np.empty((2 + num_dim,) + shape)
    q[0] = rho
    for a in range(num_dim):
        q[1 + a] = rho * vel[a]
    q[1 + num_dim] = eint + ekin
    # [var][k][j][i] with the active axes last
    q = q.reshape((2 + num_dim,) + (1,) * (3 - num_dim) + shape)
    if eos == "tabulatedlteh" and table is None:
        table = lte_h_table(gamma=gamma)
    return Problem(f"lte_h_{num_dim}d", num_dim, n, n if num_dim > 1 else 1, n if num_dim > 2 else 1, ng=ng, dx=dx,
                   bc=("periodic",) * 6, reconstruction="muscl", slope_limiter="monotonizedcentral",
                   riemann_solver="hllc", time_stepper="ssprk3", gamma=gamma, max_cfl=0.4, max_time=1e30,
                   output_delta=1e30, eos=eos, eos_avg_mass=avg_mass, eos_ionisation=ionisation, eos_table=table,
                   Q=q)
