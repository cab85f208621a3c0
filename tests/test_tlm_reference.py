"""CPU checks of the tangent-linear reference used by the adjoint tests: its
forward pass reproduces the oracle's KH run, and its directional derivative
agrees with central finite differences of its own forward pass."""
import numpy as np

import tlm_reference as T
from mosscap_b200 import problems as P


def test_tlm_forward_matches_oracle(oracle_port):
    n, steps = 16, 4
    p = P.kelvin_helmholtz_2d(n, seed=3)
    s = oracle_port.OracleSim(oracle_port.OracleConfig(**p.scheme_fields()), "port")
    s.set_Q(p.Q)
    s.fill_bcs()
    s.run(steps)
    ref = s.get_Q()[:, 0, 3:-3, 3:-3]
    vy = p.Q[2, 0, 3:-3, 3:-3] / p.Q[0, 0, 3:-3, 3:-3]
    q0 = T.kh_state(T.D(vy), T.D(p.gamma), n)
    q = T.run(q0, T.D(p.gamma), 1.0 / n, p.max_cfl, steps)
    assert np.max(np.abs(q.v - ref)) < 1e-12 * np.max(np.abs(ref))


def test_tlm_derivative_matches_finite_differences():
    n, steps = 12, 3
    p = P.kelvin_helmholtz_2d(n, seed=8)
    vy = p.Q[2, 0, 3:-3, 3:-3] / p.Q[0, 0, 3:-3, 3:-3]
    target = P.kelvin_helmholtz_2d(n, seed=9).Q[0, 0, 3:-3, 3:-3]
    rng = np.random.default_rng(1)
    d = rng.standard_normal((n, n))
    d /= np.linalg.norm(d)
    dg = 0.03
    tl, _ = T.directional_derivative(vy, d, p.gamma, dg, target, n, p.max_cfl, steps)
    # the CFL minimum of the uniform KH bands has near-ties: a step must stay
    # below the gap to the next arg-min candidate, where J has a kink
    eps = 1e-7
    _, jp = T.directional_derivative(vy + eps * d, d, p.gamma + eps * dg, dg, target, n, p.max_cfl, steps)
    _, jm = T.directional_derivative(vy - eps * d, d, p.gamma - eps * dg, dg, target, n, p.max_cfl, steps)
    fd = (jp - jm) / (2 * eps)
    assert abs(fd - tl) / abs(tl) < 1e-6, (fd, tl)
