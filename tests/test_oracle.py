"""CPU tests of the oracle: the C restatement against the reference's own
build, both against the committed golden fixtures, and physics sanity checks
of the oracle itself."""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from mosscap_b200 import problems as P


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def _run(O, kind, p, steps):
    s = O.OracleSim(O.OracleConfig(**p.scheme_fields()), kind)
    if p.gravity is not None:
        s.set_gravity(p.gravity)
    s.set_Q(p.Q)
    s.fill_bcs()
    q0 = s.get_Q()
    dts = s.run(steps)
    return q0, dts, s.get_Q(), s.time


def _bits(a):
    return np.asarray(a, dtype=np.float64).view(np.uint64)


@pytest.mark.parametrize("name", ["sod_1d", "kh_2d_64", "sedov_3d_12"])
@pytest.mark.parametrize("kind", ["port", "reference"])
def test_headline_fixture(name, kind, request):
    O = request.getfixturevalue("oracle_port" if kind == "port" else "oracle_ref")
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    p = {"sod_1d": P.sod_1d(1024), "kh_2d_64": P.kelvin_helmholtz_2d(64, seed=0),
         "sedov_3d_12": P.sedov_3d(12).with_scheme(output_delta=0.004)}[name]
    q0, dts, q1, t = _run(O, kind, p, len(g["dts"]))
    assert np.array_equal(_bits(q0), _bits(g["q0"])), "input drifted from the fixture"
    assert np.array_equal(_bits(dts), _bits(g["dts"]))
    assert np.array_equal(_bits(q1), _bits(g["q1"]))
    assert t == float(g["time"])


@pytest.mark.parametrize("kind", ["port", "reference"])
def test_sweep_fixture(kind, request):
    """Every reconstruction x limiter x solver x stepper in 1D/2D/3D with mixed
    boundary kinds and tracers: final state and dt sequence bit-identical."""
    O = request.getfixturevalue("oracle_port" if kind == "port" else "oracle_ref")
    gold = json.load(open(os.path.join(GOLDEN, "sweep.json")))
    from make_golden import sweep_cases
    n = 0
    for name, p, steps, seed in sweep_cases():
        g = gold[name]
        q0, dts, q1, _ = _run(O, kind, p, steps)
        assert _sha(q0) == g["q0_sha256"], name
        assert [int(x) for x in _bits(dts)] == g["dt_bits"], name
        assert _sha(q1) == g["q1_sha256"], name
        n += 1
    assert n == len(gold) == 241


def test_constant_boundaries_port_vs_reference(oracle_port, oracle_ref):
    """Constant boundaries (Boundaries.hpp:111-115) incl. corners in 2D."""
    O = oracle_port
    bcc = np.zeros((6, 5))
    bcc[:, 0] = [1.0, 0.5, 2.0, 0.25, 1, 1]
    bcc[:, 1] = [0.1, -0.2, 0.0, 0.3, 0, 0]
    bcc[:, 2] = [0.0, 0.1, -0.1, 0.05, 0, 0]
    bcc[:, 3] = [2.5, 1.0, 3.0, 0.7, 0, 0]
    q = P.random_state(2, 16, 16, ng=3, seed=5)
    p = P.Problem("const", 2, 16, 16, ng=3, dx=1 / 16,
                  bc=("constant", "zerograd", "wall", "constant", "zerograd", "zerograd"),
                  bc_const=bcc, reconstruction="ppm", slope_limiter="vanleer", riemann_solver="hllc",
                  time_stepper="ssprk3", max_cfl=0.5, max_time=0.03, output_delta=0.01, Q=q)
    a = _run(O, "port", p, 50)
    b = _run(O, "reference", p, 50)
    for x, y in zip(a[:3], b[:3]):
        assert np.array_equal(_bits(x), _bits(y))


def test_sod_physics(oracle_port):
    """Sod at t=0.2 against the exact solution (Toro's exact Riemann solver):
    a sanity check of the oracle, not parity. L1 density error of a 1024-cell
    MUSCL/HLLC run is small."""
    p = P.sod_1d(1024)
    q0, dts, q1, t = _run(oracle_port, "port", p, 10 ** 6)
    assert abs(t - 0.2) < 1e-15
    rho = q1[0, 0, 0, 3:-3]
    x = (np.arange(1024) + 0.5) / 1024
    exact = _sod_exact_rho(x, 0.2)
    assert np.mean(np.abs(rho - exact)) < 5e-3
    # conservation with zero-gradient ends: the waves have not reached them
    assert abs(q1[0, 0, 0, 3:-3].sum() - q0[0, 0, 0, 3:-3].sum()) / 1024 < 1e-13


def _sod_exact_rho(x, t, g=1.4):
    rl, ul, pl, rr, ur, pr = 1.0, 0.0, 1.0, 0.125, 0.0, 0.1
    cl, cr = np.sqrt(g * pl / rl), np.sqrt(g * pr / rr)

    def f(p, rk, pk, ck):
        if p > pk:
            A, B = 2 / ((g + 1) * rk), (g - 1) / (g + 1) * pk
            return (p - pk) * np.sqrt(A / (p + B))
        return 2 * ck / (g - 1) * ((p / pk) ** ((g - 1) / (2 * g)) - 1)

    lo, hi = 1e-6, 5.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if f(mid, rl, pl, cl) + f(mid, rr, pr, cr) + ur - ul > 0:
            hi = mid
        else:
            lo = mid
    ps = 0.5 * (lo + hi)
    us = 0.5 * (ul + ur) + 0.5 * (f(ps, rr, pr, cr) - f(ps, rl, pl, cl))
    rsl = rl * (ps / pl) ** (1 / g)
    rsr = rr * ((ps / pr + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pr + 1))
    sr = ur + cr * np.sqrt((g + 1) / (2 * g) * ps / pr + (g - 1) / (2 * g))
    csl = cl * (ps / pl) ** ((g - 1) / (2 * g))
    xi = (x - 0.5) / t
    out = np.empty_like(x)
    for n, s in enumerate(xi):
        if s < ul - cl:
            out[n] = rl
        elif s < us - csl:
            u = 2 / (g + 1) * (cl + (g - 1) / 2 * ul + s)
            c = u - s
            out[n] = rl * (c / cl) ** (2 / (g - 1))
        elif s < us:
            out[n] = rsl
        elif s < sr:
            out[n] = rsr
        else:
            out[n] = rr
    return out


def _run_eos(O, kind, p, steps):
    s = O.OracleSim(O.OracleConfig(**p.scheme_fields()), kind)
    s.set_eos(p.eos, p.eos_avg_mass, p.eos_ionisation, p.eos_table)
    s.set_Q(p.Q)
    s.fill_bcs()
    s.update_eos()
    dts = s.run(steps)
    y, T = s.eos_fields()
    return s.get_Q(), dts, y, T


@pytest.mark.parametrize("eos,ion", [("analyticlteh", False), ("analyticlteh", True), ("tabulatedlteh", False)])
@pytest.mark.parametrize("ndim,n", [(1, 200), (2, 40), (3, 14)])
def test_eos_port_matches_reference(oracle_port, oracle_ref, eos, ion, ndim, n):
    """The non-ideal EOS updates (source/AnalyticLteH.hpp,
    source/TabulatedLteH.hpp) run ahead of every stage: the restatement
    equals the reference build bit for bit in the state, the dt sequence and
    the temperature / ionisation fields, and neither meets an abort."""
    p = P.lte_hydrogen(ndim, n, seed=ndim, eos=eos, ionisation=ion)
    a0 = oracle_ref.OracleSim(oracle_ref.OracleConfig(**p.scheme_fields()), "reference").abort_count()
    ref = _run_eos(oracle_ref, "reference", p, 5)
    port = _run_eos(oracle_port, "port", p, 5)
    for r, q in zip(ref, port):
        assert np.array_equal(_bits(r), _bits(q))
    assert oracle_ref.OracleSim(oracle_ref.OracleConfig(**p.scheme_fields()), "reference").abort_count() == a0
    y, T = ref[2], ref[3]
    assert (T > 1000.0).all() and (y > 0.0).all() and (y < 1.01).all()


def test_tabulated_eos_shifts_energy(oracle_port):
    """The tabulated kind changes the state (the ionisation-energy shift);
    the analytic kind leaves it to the ideal-gas step."""
    from dataclasses import replace
    p = P.lte_hydrogen(2, 32, seed=3, eos="tabulatedlteh")
    tab = _run_eos(oracle_port, "port", p, 4)[0]
    ideal = _run(oracle_port, "port", replace(p, eos="ideal"), 4)[2]
    assert not np.array_equal(tab, ideal)
    pa = replace(p, eos="analyticlteh", eos_table=None)
    ana = _run_eos(oracle_port, "port", pa, 4)[0]
    assert np.array_equal(_bits(ana), _bits(ideal))
