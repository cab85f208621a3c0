"""Generate the golden fixtures in tests/golden/ from the reference itself.

The reference's own hot-path sources (source/Hydro.cpp,
source/TimeStepping.cpp and the headers they include) are compiled by
``make -C oracle ref`` against the host Kokkos/YAKL shim into
``oracle/_ref/libmosscap_ref.so``; this script drives that build on seeded
synthetic inputs and records:

* ``<case>.npz`` -- the input state, the dt of every step and the final state
  for the three headline workloads at fixture size (Sod 1D at full size, KH 2D
  at 64^2, Sedov 3D at 12^3);
* ``sweep.json`` -- for every reconstruction x limiter x Riemann solver x
  stepper on small 1D / 2D / 3D grids with mixed boundary kinds, for the
  gravity source term with every stepper, and for two passive tracers in 3D,
  the SHA-256 of the input and of the final state and the dt sequence (bit
  patterns).

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import itertools
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import OracleConfig, OracleSim, build  # noqa: E402
from mosscap_b200 import problems as P  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def cfg_of(p: P.Problem) -> OracleConfig:
    return OracleConfig(**p.scheme_fields())


def run_case(p: P.Problem, steps: int, kind: str = "reference"):
    s = OracleSim(cfg_of(p), kind)
    if p.gravity is not None:
        s.set_gravity(p.gravity)
    s.set_Q(p.Q)
    s.fill_bcs()
    q0 = s.get_Q()
    dts = s.run(steps)
    return q0, dts, s.get_Q(), s.time


def headline_cases():
    sod = P.sod_1d(1024)
    kh = P.kelvin_helmholtz_2d(64, seed=0)
    # at 12^3 one CFL step already passes t = 0.05, so outputs every 0.004
    # make the clamp of every step matter instead
    sedov = P.sedov_3d(12).with_scheme(output_delta=0.004)
    return [("sod_1d", sod, 10 ** 6), ("kh_2d_64", kh, 20), ("sedov_3d_12", sedov, 10 ** 6)]


SWEEP_RECON = [("fog", "monotonizedcentral"), ("muscl", "vanleer"), ("muscl", "monotonizedcentral"),
               ("muscl", "minmod"), ("ppm", "vanleer"), ("ppm", "monotonizedcentral"), ("ppm", "minmod"),
               ("weno5z", "monotonizedcentral")]
SWEEP_BCS = {
    1: ("symmetricoutflowdiode", "wall", "zerograd", "zerograd", "zerograd", "zerograd"),
    2: ("wall", "symmetricoutflowdiode", "periodic", "periodic", "zerograd", "zerograd"),
    3: ("zerograd", "symmetric", "wall", "symmetricoutflowdiode", "periodic", "periodic"),
}
SWEEP_N = {1: 48, 2: 14, 3: 8}


def sweep_cases():
    """(name, Problem, steps) for the scheme sweep; inputs from random_state."""
    out = []
    for ndim in (1, 2, 3):
        n = SWEEP_N[ndim]
        for (rec, lim), rs, st in itertools.product(SWEEP_RECON, ("rusanov", "hll", "hllc"),
                                                    ("rk2", "ssprk3", "ssprk4")):
            ntr = 1 if (ndim < 3 and rs == "hllc" and st == "ssprk3") else 0
            seed = 1000 * ndim + 17 * SWEEP_RECON.index((rec, lim)) + 5 * ("rusanov", "hll", "hllc").index(rs) \
                + ("rk2", "ssprk3", "ssprk4").index(st)
            q = P.random_state(ndim, n, n, n, ng=3, num_tracers=ntr, seed=seed)
            p = P.Problem(f"sweep_{ndim}d_{rec}_{lim}_{rs}_{st}", ndim, n, n if ndim > 1 else 1,
                          n if ndim > 2 else 1, ng=3, num_tracers=ntr, dx=1.0 / n, bc=SWEEP_BCS[ndim],
                          reconstruction=rec, slope_limiter=lim, riemann_solver=rs, time_stepper=st,
                          gamma=1.4, max_cfl=0.6, max_time=0.04, output_delta=0.015, Q=q)
            out.append((p.name, p, 6, seed))
    # the gravity source term (source/SourceTerms/Gravity.cpp) with every
    # stepper in 1D / 2D / 3D
    for ndim, st in itertools.product((1, 2, 3), ("rk2", "ssprk3", "ssprk4")):
        n = SWEEP_N[ndim]
        seed = 5000 + 10 * ndim + ("rk2", "ssprk3", "ssprk4").index(st)
        rec, lim = [("muscl", "vanleer"), ("ppm", "monotonizedcentral"), ("weno5z", "monotonizedcentral")][ndim - 1]
        q = P.random_state(ndim, n, n, n, ng=3, seed=seed)
        p = P.Problem(f"gravity_{ndim}d_{rec}_{st}", ndim, n, n if ndim > 1 else 1, n if ndim > 2 else 1, ng=3,
                      dx=1.0 / n, bc=SWEEP_BCS[ndim], reconstruction=rec, slope_limiter=lim, riemann_solver="hllc",
                      time_stepper=st, gamma=1.4, max_cfl=0.6, max_time=0.04, output_delta=0.015,
                      gravity=(-1.5, 0.75, -0.5), Q=q)
        out.append((p.name, p, 6, seed))
    # passive tracers in 3D (two fields) with each reconstruction, HLL / HLLC
    # and rk2 / ssprk3
    for (rec, lim), rs, st in itertools.product([SWEEP_RECON[0], SWEEP_RECON[2], SWEEP_RECON[5], SWEEP_RECON[7]],
                                                 ("hll", "hllc"), ("rk2", "ssprk3")):
        n = SWEEP_N[3]
        seed = 7000 + 17 * SWEEP_RECON.index((rec, lim)) + 5 * ("hll", "hllc").index(rs) + ("rk2", "ssprk3").index(st)
        q = P.random_state(3, n, n, n, ng=3, num_tracers=2, seed=seed)
        p = P.Problem(f"tracer3d_{rec}_{lim}_{rs}_{st}", 3, n, n, n, ng=3, num_tracers=2, dx=1.0 / n,
                      bc=SWEEP_BCS[3], reconstruction=rec, slope_limiter=lim, riemann_solver=rs, time_stepper=st,
                      gamma=1.4, max_cfl=0.6, max_time=0.04, output_delta=0.015, Q=q)
        out.append((p.name, p, 6, seed))
    return out


def main():
    build("ref")
    for name, p, steps in headline_cases():
        q0, dts, q1, t = run_case(p, steps)
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), q0=q0, dts=dts, q1=q1, time=t)
        print(name, len(dts), "steps, t =", t)
    sweep = {}
    for name, p, steps, seed in sweep_cases():
        q0, dts, q1, t = run_case(p, steps)
        sweep[name] = {"seed": seed, "steps": int(len(dts)), "q0_sha256": sha(q0), "q1_sha256": sha(q1),
                       "dt_bits": [int(x) for x in np.asarray(dts).view(np.uint64)]}
    with open(os.path.join(OUT, "sweep.json"), "w") as f:
        json.dump(sweep, f, indent=0, sort_keys=True)
    print(len(sweep), "sweep cases")


if __name__ == "__main__":
    main()
