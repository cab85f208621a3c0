"""GPU tests of the non-ideal EOS updates (mc_set_eos / mc_update_eos /
mc_get_eos_fields) against the oracle.

The update runs ahead of every stage, as compute_hydro_fluxes does
(source/Hydro.cpp:326-328). The analytic LTE hydrogen kind only computes
the temperature and ionisation fields, so the state and the dt sequence
stay bit-identical to the oracle; its bisection stops within 0.1 K
(source/AnalyticLteH.hpp:104-107) and CUDA's pow / exp round differently
from the C library's, so a cell can take the other branch of one bisection
step: temperatures agree within 0.25 K, and ionisation fractions within the
change of the Saha fraction over that bracket. The tabulated kind feeds the
ionisation-energy shift back into the energy through log10, so the state
agrees to rounding (relative 1e-12), not bit for bit."""
import numpy as np
import pytest

from mosscap_b200 import problems as P

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def _oracle(O, p, steps):
    s = O.OracleSim(O.OracleConfig(**p.scheme_fields()), "port")
    s.set_eos(p.eos, p.eos_avg_mass, p.eos_ionisation, p.eos_table)
    s.set_Q(p.Q)
    s.fill_bcs()
    s.update_eos()
    dts = s.run(steps)
    y, T = s.eos_fields()
    return s.get_Q(), dts, y, T


def _gpu(p, steps, device_loop):
    from mosscap_b200.hydro import HydroSim
    sim = HydroSim(p)
    sim.fill_bcs()
    sim.update_eos()
    dts = sim.run(steps, device_loop=device_loop)
    y, T = sim.eos_fields()
    st = sim.status()
    return sim.get_Q(), np.asarray(dts), y, T, st


@pytest.mark.parametrize("ndim,n", [(1, 700), (2, 97), (3, 35)])
@pytest.mark.parametrize("ion", [False, True])
def test_analytic_lte_h(gpu_lib, oracle_port, ndim, n, ion):
    p = P.lte_hydrogen(ndim, n, seed=10 + ndim, eos="analyticlteh", ionisation=ion)
    q_ref, dts_ref, y_ref, T_ref = _oracle(oracle_port, p, 6)
    for loop in (False, True):
        q, dts, y, T, st = _gpu(p, 6, loop)
        assert st == 0
        assert np.array_equal(_bits(dts), _bits(dts_ref))
        assert np.array_equal(_bits(q), _bits(q_ref))
        dT = np.abs(T - T_ref)
        assert dT.max() <= 0.25, dT.max()
        assert (dT == 0.0).mean() > 0.95, (dT == 0.0).mean()
        # y is the Saha fraction at the last trial temperature, which lies
        # within the final bisection bracket: bound its difference by the
        # change of the Saha fraction over that bracket (plus the rounding
        # of the cancelling (sqrt(X^2 + 4 n X) - X) / (2 n))
        nh = q_ref[0] / (P.H_MASS * p.eos_avg_mass)
        X = 2.4146830395719654e+21 * np.power(T_ref, 1.5) * np.exp(-157763.42386247337 / T_ref)
        bound = np.abs(P.saha_y(nh, T_ref + 0.3) - P.saha_y(nh, T_ref - 0.3)) + 8e-16 * (1.0 + X / nh)
        assert (np.abs(y - y_ref) <= bound).all()


@pytest.mark.parametrize("ndim,n", [(1, 700), (2, 97), (3, 35)])
def test_tabulated_lte_h(gpu_lib, oracle_port, ndim, n):
    p = P.lte_hydrogen(ndim, n, seed=20 + ndim, eos="tabulatedlteh")
    q_ref, dts_ref, y_ref, T_ref = _oracle(oracle_port, p, 6)
    for loop in (False, True):
        q, dts, y, T, st = _gpu(p, 6, loop)
        assert st == 0
        assert np.allclose(dts, dts_ref, rtol=1e-12, atol=0.0)
        for v in range(q.shape[0]):
            scale = np.abs(q_ref[v]).max()
            assert np.abs(q[v] - q_ref[v]).max() <= 1e-12 * scale, v
        assert np.abs(y - y_ref).max() <= 1e-12
        assert np.allclose(T, T_ref, rtol=1e-12, atol=0.0)


def test_eos_flags_instead_of_abort(gpu_lib):
    """A cell with negative internal energy, on which the reference aborts,
    raises MC_FLAG_EOS; the context stays usable."""
    from mosscap_b200 import capi
    from mosscap_b200.hydro import HydroSim
    p = P.lte_hydrogen(2, 40, seed=5, eos="tabulatedlteh")
    q = p.Q.copy()
    q[-1, 0, 10, 10] = 0.25 * (q[1, 0, 10, 10] ** 2 + q[2, 0, 10, 10] ** 2) / q[0, 0, 10, 10]
    sim = HydroSim(p.with_scheme(Q=q))
    sim.update_eos()
    assert sim.status() & capi.FLAG_EOS
    sim2 = HydroSim(p)
    sim2.fill_bcs()
    sim2.update_eos()
    sim2.run(2)
    assert sim2.status() == 0
