"""mc_step_host: compute_dt + time_step on a state held in host memory, with
the copies overlapping the step in 2D (stage 0's fluxes band by band as the
state arrives, dt applied once all of it is in, the last stage band by band
with each band copied back behind it).

Each case runs a few steps both ways from the same state: through
mc_step_host on a host buffer (the device copy filled with NaN beforehand,
so every value must come from the host), and through the serial calls
(mc_compute_dt, mc_time_step) on a device state. The dt sequences and the
states, ghost cells included, must be equal bit for bit; the last step of
each case is shortened by the output clamp."""
import numpy as np
import pytest
import torch

from mosscap_b200 import problems as P

pytestmark = pytest.mark.gpu

STEPS = 3


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def _problem(case):
    if case == "weno5z_hllc_ssprk3_periodic":
        p = P.kelvin_helmholtz_2d(130, seed=4)
        return P.Problem("kh_band_rows", 2, 130, 257, ng=3, dx=p.dx, bc=p.bc, reconstruction="weno5z",
                         riemann_solver="hllc", time_stepper="ssprk3", gamma=p.gamma, max_cfl=0.4,
                         Q=P.random_state(2, 130, 257, ng=3, seed=4, gamma=p.gamma)), "fp64"
    if case == "muscl_rusanov_rk2_gravity_tracers":
        q = P.random_state(2, 61, 95, ng=3, num_tracers=2, seed=8)
        return P.Problem("host_rk2", 2, 61, 95, ng=3, num_tracers=2, dx=1.0 / 95,
                         bc=("periodic", "periodic", "wall", "symmetricoutflowdiode", "zerograd", "zerograd"),
                         reconstruction="muscl", slope_limiter="minmod", riemann_solver="rusanov",
                         time_stepper="rk2", gamma=1.4, max_cfl=0.6, gravity=(0.2, -1.5, 0.0), Q=q), "fp64"
    if case == "ppm_hll_ssprk4_fp32":
        q = P.random_state(2, 88, 151, ng=3, seed=12)
        return P.Problem("host_fp32", 2, 88, 151, ng=3, dx=1.0 / 151,
                         bc=("zerograd", "wall", "periodic", "periodic", "zerograd", "zerograd"),
                         reconstruction="ppm", slope_limiter="monotonizedcentral", riemann_solver="hll",
                         time_stepper="ssprk4", gamma=1.4, max_cfl=0.5, Q=q), "fp32"
    if case == "weno5z_hllc_ssprk3_fp32_gravity":
        q = P.random_state(2, 72, 97, ng=3, seed=21)
        return P.Problem("host_fp32_gravity", 2, 72, 97, ng=3, dx=1.0 / 97,
                         bc=("periodic", "periodic", "wall", "zerograd", "zerograd", "zerograd"),
                         reconstruction="weno5z", riemann_solver="hllc", time_stepper="ssprk3", gamma=1.4,
                         max_cfl=0.4, gravity=(0.0, -2.0, 0.0), Q=q), "fp32"
    if case == "serial_2d_few_rows":
        q = P.random_state(2, 50, 24, ng=3, seed=3)
        return P.Problem("host_small", 2, 50, 24, ng=3, dx=1.0 / 50, bc=("zerograd",) * 6,
                         reconstruction="weno5z", riemann_solver="hllc", time_stepper="ssprk3", gamma=1.4,
                         max_cfl=0.4, Q=q), "fp64"
    if case == "serial_sod_1d":
        return P.sod_1d(300), "fp64"
    if case == "serial_3d":
        q = P.random_state(3, 14, 13, 12, ng=3, seed=5)
        return P.Problem("host_3d", 3, 14, 13, 12, ng=3, dx=1.0 / 14, bc=("zerograd",) * 6,
                         reconstruction="ppm", riemann_solver="hll", time_stepper="ssprk3", gamma=1.4, max_cfl=0.3,
                         Q=q), "fp64"
    raise KeyError(case)


def _serial(p, precision):
    from mosscap_b200.hydro import HydroSim
    sim = HydroSim(p, precision=precision)
    sim.fill_bcs()
    dts = []
    for _ in range(STEPS):
        dt = sim.compute_dt()
        sim.time_step(dt)
        dts.append(dt)
    q = sim.get_Q()
    sim.close()
    return np.array(dts), q


@pytest.mark.parametrize("pinned", [True, False])
@pytest.mark.parametrize("case", ["weno5z_hllc_ssprk3_periodic", "muscl_rusanov_rk2_gravity_tracers", "ppm_hll_ssprk4_fp32",
                                  "weno5z_hllc_ssprk3_fp32_gravity", "serial_2d_few_rows", "serial_sod_1d",
                                  "serial_3d"])
def test_step_host_matches_serial_calls(gpu_lib, case, pinned):
    from mosscap_b200.hydro import HydroSim
    if not pinned and case != "weno5z_hllc_ssprk3_periodic":
        pytest.skip("pageable memory: one case")
    p, precision = _problem(case)
    p = p.with_scheme(max_time=1e30, output_delta=1e30)
    # the output clamp shortens the last step: the next output time falls
    # inside it
    free_dts, _ = _serial(p, precision)
    p = p.with_scheme(output_delta=float(free_dts[:-1].sum() + 0.5 * free_dts[-1]))
    ref_dts, ref_q = _serial(p, precision)
    assert ref_dts[-1] < free_dts[-1]

    sim = HydroSim(p, precision=precision)
    sim.fill_bcs()
    host = torch.empty(tuple(sim.Q.shape), dtype=torch.float64, pin_memory=pinned)
    host.copy_(sim.Q)
    sim.Q.fill_(float("nan"))
    dts = np.array([sim.step_host(host) for _ in range(STEPS)])
    torch.cuda.synchronize()
    assert np.array_equal(_bits(dts), _bits(ref_dts)), (dts, ref_dts)
    hq = host.numpy()
    assert np.array_equal(_bits(hq), _bits(ref_q)), \
        f"{np.count_nonzero(_bits(hq) != _bits(ref_q))} host values differ"
    assert np.array_equal(_bits(sim.get_Q()), _bits(ref_q)), "device copy differs"
    assert sim.status() == 0
    sim.close()
