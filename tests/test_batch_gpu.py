"""GPU tests of the batched form (mc_batch_*): independent 1D and 2D Riemann
problems of uneven size advanced by one persistent launch per stage (or, in
the split form, one over the 2D tiles and one over the 1D tasks), each with
its own dt, replayed from a CUDA graph.

Every problem must match the reference algorithm (the oracle, run on that
problem alone) bit for bit while its state stays finite; the seeded set
contains a few high-Mach problems on which the reference itself produces
negative pressures, and those must be flagged instead. The result must not
depend on the schedule the autotuner picks."""
import numpy as np
import pytest

from mosscap_b200 import problems as P

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def _small_batch(rs, seed=7):
    return P.riemann_batch(seed=seed, n1d=24, n2d=10, riemann_solver=rs, min1d=40, max1d=700, min2d=24,
                           max2d=90)


def _oracle_run(O, p, steps):
    s = O.OracleSim(O.OracleConfig(**p.scheme_fields()), "port")
    s.set_Q(p.Q)
    s.fill_bcs()
    s.run(steps)
    return s.get_Q()


@pytest.mark.parametrize("rs", ["hllc", "rusanov"])
def test_batch_matches_oracle_per_problem(gpu_lib, oracle_port, rs):
    from mosscap_b200 import capi
    from mosscap_b200.hydro import BatchSim
    probs = _small_batch(rs)
    steps = 12
    b = BatchSim(probs)
    b.fill_bcs()
    b.advance(steps)
    times, nsteps, status = b.clocks()
    assert (nsteps == steps).all()
    checked = 0
    for k, p in enumerate(probs):
        ref = _oracle_run(oracle_port, p, steps)
        got = b.get_Q(k)
        if np.isfinite(ref).all():
            assert np.array_equal(_bits(got), _bits(ref)), f"problem {k} ({p.name}, {p.nx} cells) differs"
            checked += 1
        else:
            assert status[k] & (capi.FLAG_NONFINITE | capi.FLAG_NEG_PRESSURE | capi.FLAG_NEG_DENSITY), k
    assert checked >= len(probs) - 4


@pytest.mark.parametrize("stepper", ["ssprk3", "ssprk4"])
def test_batch_other_steppers_match_oracle(gpu_lib, oracle_port, stepper):
    """Three- and four-stage steppers: every stage's ghost cells are filled
    by each problem's last finishing tile or task of that stage (one count
    per stage and problem), bit-identical to the oracle per problem."""
    from mosscap_b200 import capi
    from mosscap_b200.hydro import BatchSim
    probs = [p.with_scheme(time_stepper=stepper) for p in _small_batch("hllc", seed=17)]
    steps = 6
    b = BatchSim(probs)
    b.fill_bcs()
    b.advance(steps)
    _, nsteps, status = b.clocks()
    checked = 0
    for k, p in enumerate(probs):
        ref = _oracle_run(oracle_port, p, steps)
        if np.isfinite(ref).all():
            assert nsteps[k] == steps, k
            assert np.array_equal(_bits(b.get_Q(k)), _bits(ref)), f"problem {k} ({p.name}) differs"
            checked += 1
        else:
            assert status[k] & (capi.FLAG_NONFINITE | capi.FLAG_NEG_PRESSURE | capi.FLAG_NEG_DENSITY), k
    assert checked >= len(probs) - 4


def test_batch_schedule_independent(gpu_lib):
    """Tuned and default schedules (static / dynamic, grid sizes, 1D task
    lengths) give bit-identical states and clocks."""
    from mosscap_b200.hydro import BatchSim
    probs = _small_batch("hllc", seed=11)
    a = BatchSim(probs)
    a.fill_bcs()
    sched_a = a.schedule()
    a.advance(8)
    b = BatchSim(probs)
    b.fill_bcs()
    sched_b = b.tune()
    b.advance(8)
    ta, _, _ = a.clocks()
    tb, _, _ = b.clocks()
    assert np.array_equal(_bits(ta), _bits(tb)), (sched_a, sched_b)
    for k in range(len(probs)):
        assert np.array_equal(_bits(a.get_Q(k)), _bits(b.get_Q(k))), (k, sched_a, sched_b)


def test_batch_one_and_two_launches_per_stage_agree(gpu_lib):
    """One launch per stage over the 2D tiles and the 1D tasks together (the
    default) and the split form give bit-identical states and clocks."""
    from mosscap_b200.hydro import BatchSim
    probs = _small_batch("hllc", seed=13)
    runs = []
    for n in (1, 2):
        b = BatchSim(probs)
        b.set_stage_launches(n)
        assert b.schedule()["launches_per_stage"] == n
        b.fill_bcs()
        b.advance(8)
        runs.append(b)
    ta, _, _ = runs[0].clocks()
    tb, _, _ = runs[1].clocks()
    assert np.array_equal(_bits(ta), _bits(tb))
    for k in range(len(probs)):
        assert np.array_equal(_bits(runs[0].get_Q(k)), _bits(runs[1].get_Q(k))), k


def test_batch_output_clamp_and_max_time(gpu_lib, oracle_port):
    """Per-problem output-time clamps and max_time: problems stop on their own."""
    from mosscap_b200.hydro import BatchSim
    probs = _small_batch("hllc", seed=3)[:6] + _small_batch("hllc", seed=3)[-3:]
    probs = [p.with_scheme(max_time=0.02 + 0.005 * k, output_delta=0.0041) for k, p in enumerate(probs)]
    b = BatchSim(probs)
    b.fill_bcs()
    b.advance(400)
    times, nsteps, status = b.clocks()
    for k, p in enumerate(probs):
        s = oracle_port.OracleSim(oracle_port.OracleConfig(**p.scheme_fields()), "port")
        s.set_Q(p.Q)
        s.fill_bcs()
        dts = s.run(400)
        ref = s.get_Q()
        if not np.isfinite(ref).all():
            continue
        assert times[k] == s.time == p.max_time, k
        assert nsteps[k] == len(dts), k
        assert np.array_equal(_bits(b.get_Q(k)), _bits(ref)), k


def test_batch_fp32_form(gpu_lib, oracle_port):
    from mosscap_b200.hydro import BatchSim
    probs = [p for p in _small_batch("hllc", seed=5)]
    b = BatchSim(probs, precision="fp32")
    b.fill_bcs()
    b.advance(10)
    worst = 0.0
    for k, p in enumerate(probs):
        ref = _oracle_run(oracle_port, p, 10)
        if not np.isfinite(ref).all():
            continue
        rho, rr = b.get_Q(k)[0], ref[0]
        worst = max(worst, float(np.abs(rho - rr).sum() / np.abs(rr).sum()))
    assert worst < 1e-5, worst
