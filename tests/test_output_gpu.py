"""GPU side of the NetCDF output: the primitive state W of mc_get_prim
(what the reference's State.W holds at output time) against the oracle bit
for bit, and HydroSim.run writing the reference's output files."""
import numpy as np
import pytest

from mosscap_b200 import netcdf as nc
from mosscap_b200 import output as out
from mosscap_b200 import problems as P

pytestmark = pytest.mark.gpu


def _same_bits(a, b, what):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    assert a.shape == b.shape, what
    bad = np.argwhere(a.view(np.uint64) != b.view(np.uint64))
    assert len(bad) == 0, f"{what}: {len(bad)} values differ, first {bad[:4]}"


def _problem(case):
    if case == "kh_ssprk3":
        return P.kelvin_helmholtz_2d(64, seed=3)
    if case == "sod_rk2":
        return P.sod_1d(700)
    if case == "tracers_ssprk4":
        q = P.random_state(2, 67, 45, ng=3, num_tracers=2, seed=5)
        return P.Problem("tracers", 2, 67, 45, ng=3, num_tracers=2, dx=1.0 / 67,
                         bc=("periodic", "periodic", "wall", "zerograd", "periodic", "periodic"),
                         reconstruction="muscl", slope_limiter="vanleer", riemann_solver="hllc",
                         time_stepper="ssprk4", gamma=1.4, max_cfl=0.3, max_time=1.0, output_delta=1.0, Q=q)
    return P.sedov_3d(12).with_scheme(output_delta=0.004)


@pytest.mark.parametrize("case", ["kh_ssprk3", "sod_rk2", "tracers_ssprk4", "sedov_3d"])
def test_get_W_matches_oracle(gpu_lib, oracle_port, case):
    from mosscap_b200.hydro import HydroSim
    p = _problem(case)
    o = oracle_port.OracleSim(oracle_port.OracleConfig(**p.scheme_fields()), "port")
    o.set_Q(p.Q)
    o.fill_bcs()
    sim = HydroSim(p)
    sim.fill_bcs()
    # before any step: the primitives of Q itself
    w0 = sim.get_W()
    assert np.all(np.isfinite(w0[0]))
    o.run(4)
    sim.run(4, device_loop=False)
    _same_bits(sim.get_Q(), o.get_Q(), "state")
    _same_bits(sim.get_W(), o.get_W(), "W after 4 steps")
    sim.close()


def test_run_writes_reference_outputs(gpu_lib, tmp_path):
    """KH 64^2 to t = 0.05 with output every 0.02: the initial output, one per
    due output and a final one, each record equal to the state then."""
    from mosscap_b200.hydro import HydroSim
    p = P.kelvin_helmholtz_2d(64, seed=1).with_scheme(max_time=0.05, output_delta=0.02)
    sim = HydroSim(p)
    sim.fill_bcs()
    cfg = out.OutputConfig.for_problem(p, directory=str(tmp_path))
    cfg.variables.primitive = True
    q0 = sim.get_Q()
    sim.run(device_loop=True, output=cfg)
    f = nc.read(str(tmp_path / f"output_{p.name}.nc"))
    t = f.variables["time"]
    # t = 0 (setup), 0.02 and 0.04 (due), 0.05 (after the loop; not due at 0.05)
    assert f.numrecs == cfg.output_count == 4
    assert t[0] == 0.0 and np.all(np.diff(t) > 0.0) and t[-1] == sim.time and np.isclose(sim.time, 0.05)
    assert np.isclose(t[1], 0.02) and np.isclose(t[2], 0.04)
    _same_bits(f.variables["Q"][0], q0, "initial record")
    _same_bits(f.variables["Q"][-1], sim.get_Q(), "final record")
    _same_bits(f.variables["W"][-1], sim.get_W(), "final W")
    sim.close()
