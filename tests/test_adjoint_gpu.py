"""GPU tests of the discrete adjoint (mc_adjoint_* through EulerSteps).

Loss: J = 1/2 sum (rho_final - rho_target)^2 over the interior after n
SSPRK3 steps of 2D Kelvin-Helmholtz (WENO5-Z + HLLC, periodic), with the
target from a second seed. Gradient with respect to the initial vy field and
gamma, checked (1) against central finite differences along random
directions, and (2) against an independent FP64 forward-mode tangent-linear
reference (tests/tlm_reference.py)."""
import numpy as np
import pytest
import torch

from mosscap_b200 import problems as P

pytestmark = pytest.mark.gpu


def _setup(n, seed=0, target_seed=1):
    from mosscap_b200.adjoint import kh_vy
    p = P.kelvin_helmholtz_2d(n, seed=seed)
    vy = torch.tensor(kh_vy(p), device="cuda")
    pt = P.kelvin_helmholtz_2d(n, seed=target_seed)
    return p, vy, pt


def _loss_and_grad(p, vy0, gamma0, rho_target, steps, ckpt):
    from mosscap_b200.adjoint import EulerSteps, kh_initial_state
    vy = vy0.clone().requires_grad_(True)
    g = torch.tensor(gamma0, dtype=torch.float64, device="cuda", requires_grad=True)
    q0 = kh_initial_state(vy, g, p)
    q = EulerSteps.apply(q0, g, p, steps, ckpt)
    J = 0.5 * ((q[0] - rho_target) ** 2).sum()
    J.backward()
    return J.item(), vy.grad.detach().clone(), g.grad.item()


def _final_rho(p, vy, gamma, steps):
    from mosscap_b200.adjoint import EulerSteps, kh_initial_state
    with torch.no_grad():
        g = torch.tensor(gamma, dtype=torch.float64, device="cuda")
        return EulerSteps.apply(kh_initial_state(vy, g, p), g, p, steps, 1000)[0].clone()


def _central_difference(p, vy, gamma, d, dg, eps, rho_target, steps):
    """(J(x + eps d) - J(x - eps d)) / (2 eps) for J = 1/2 |rho - rho_t|^2,
    formed from the two final states as 1/2 sum (r+ - r-)(r+ + r- - 2 rho_t)
    so that the difference does not cancel at the level of J."""
    rp = _final_rho(p, vy + eps * d, gamma + eps * dg, steps)
    rm = _final_rho(p, vy - eps * d, gamma - eps * dg, steps)
    return float((0.5 * (rp - rm) * (rp + rm - 2.0 * rho_target)).sum()) / (2 * eps)


def _target_rho(p_target, gamma, steps):
    from mosscap_b200.adjoint import EulerSteps, kh_initial_state, kh_vy
    vy = torch.tensor(kh_vy(p_target), device="cuda")
    with torch.no_grad():
        g = torch.tensor(gamma, dtype=torch.float64, device="cuda")
        return EulerSteps.apply(kh_initial_state(vy, g, p_target), g, p_target, steps, 1000)[0].clone()


def test_adjoint_matches_finite_differences(gpu_lib):
    n, steps, ckpt = 48, 10, 4  # three segments, the last one partial
    p, vy, pt = _setup(n)
    gamma = p.gamma
    rho_t = _target_rho(pt, gamma, steps)
    J, gvy, gg = _loss_and_grad(p, vy, gamma, rho_t, steps, ckpt)
    assert J > 0 and np.isfinite(gvy.cpu().numpy()).all()
    rng = np.random.default_rng(2)
    worst = 0.0
    for k in range(8):
        d = torch.tensor(rng.standard_normal((n, n)), device="cuda")
        d = d / d.norm()
        dg = float(rng.standard_normal()) * 1e-2
        # The directional derivative is linear in (d, dg): difference the vy
        # part with a step below the gap between near-tied CFL arg-min
        # candidates of the KH bands (where J, a minimum over cells, has
        # kinks), and the gamma part with a step large enough to stay clear
        # of roundoff.
        fd = (_central_difference(p, vy, gamma, d, 0.0, 1e-7, rho_t, steps)
              + _central_difference(p, vy, gamma, 0.0 * d, dg, 1e-6, rho_t, steps))
        ad = float((gvy * d).sum()) + gg * dg
        rel = abs(fd - ad) / max(abs(fd), abs(ad), 1e-300)
        worst = max(worst, rel)
    assert worst < 1e-5, worst


def test_adjoint_matches_tangent_linear_reference(gpu_lib):
    import tlm_reference as T
    n, steps, ckpt = 24, 6, 4
    p, vy, pt = _setup(n, seed=4, target_seed=5)
    gamma = p.gamma
    rho_t = _target_rho(pt, gamma, steps)
    J, gvy, gg = _loss_and_grad(p, vy, gamma, rho_t, steps, ckpt)
    rng = np.random.default_rng(9)
    for k in range(3):
        d = rng.standard_normal((n, n))
        dg = float(rng.standard_normal()) * 0.05
        tl, jref = T.directional_derivative(vy.cpu().numpy(), d, gamma, dg, rho_t.cpu().numpy(), n, p.max_cfl,
                                            steps)
        ad = float((gvy.cpu().numpy() * d).sum()) + gg * dg
        assert abs(jref - J) / J < 1e-9, (jref, J)
        assert abs(tl - ad) / abs(tl) < 1e-8, (tl, ad)


def test_adjoint_checkpoint_interval_does_not_change_gradient(gpu_lib):
    n, steps = 32, 9
    p, vy, pt = _setup(n, seed=6, target_seed=7)
    rho_t = _target_rho(pt, p.gamma, steps)
    _, g1, gg1 = _loss_and_grad(p, vy, p.gamma, rho_t, steps, 1)
    _, g2, gg2 = _loss_and_grad(p, vy, p.gamma, rho_t, steps, 4)
    _, g3, gg3 = _loss_and_grad(p, vy, p.gamma, rho_t, steps, 100)
    assert torch.equal(g1, g2) and torch.equal(g2, g3)
    assert gg1 == gg2 == gg3


def test_reverse_reciprocal_error_bound(gpu_lib):
    """The reciprocal of the reverse sweep (rcp.approx.ftz.f64 refined by two
    Newton-Raphson steps) against IEEE 1/x: within 2 ulp over normal inputs of
    either sign whose reciprocal is normal (every denominator the sweep
    inverts is such a value)."""
    import ctypes
    from mosscap_b200 import capi
    rng = np.random.default_rng(0)
    n = 1 << 20
    x = rng.uniform(1.0, 10.0, n) * 10.0 ** rng.uniform(-300.0, 300.0, n) * rng.choice([-1.0, 1.0], n)
    x[:8] = [1.0, 2.0, 3.0, 1.0 / 3.0, 0.1, 1e-36, 1e20, 5.0 / 3.0 - 1.0]
    xt = torch.tensor(x, device="cuda")
    out = torch.empty_like(xt)
    capi.check(gpu_lib.mc_debug_reverse_reciprocal(ctypes.c_void_p(xt.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                                   n, None), "mc_debug_reverse_reciprocal")
    torch.cuda.synchronize()
    ref = 1.0 / x
    ulps = np.abs(out.cpu().numpy() - ref) / np.spacing(np.abs(ref))
    assert ulps.max() <= 2.0, ulps.max()


def test_gpu_tangent_linear_matches_numpy_reference(gpu_lib):
    """mc_tangent_linear (dual numbers through the forward kernels'
    arithmetic) against the numpy tangent-linear model: two independent
    forward-mode derivatives of the same discrete map."""
    import tlm_reference as T
    from mosscap_b200.adjoint import kh_directional_derivatives
    n, steps = 24, 6
    p, vy, pt = _setup(n, seed=4, target_seed=5)
    rho_t = _target_rho(pt, p.gamma, steps)
    rng = np.random.default_rng(9)
    dirs = [rng.standard_normal((n, n)) for _ in range(3)]
    dgs = [float(rng.standard_normal()) * 0.05 for _ in range(3)]
    J, dJ = kh_directional_derivatives(p, vy, p.gamma, torch.tensor(np.stack(dirs), device="cuda"), dgs, rho_t,
                                       steps)
    for k in range(3):
        tl, jref = T.directional_derivative(vy.cpu().numpy(), dirs[k], p.gamma, dgs[k], rho_t.cpu().numpy(), n,
                                            p.max_cfl, steps)
        assert abs(jref - J) / J < 1e-12, (jref, J)
        assert abs(tl - dJ[k]) / abs(tl) < 1e-10, (k, tl, dJ[k])


def test_gpu_tangent_linear_value_is_the_forward_state(gpu_lib):
    from mosscap_b200.adjoint import EulerSteps, kh_initial_state, tangent_linear
    n, steps = 40, 7
    p, vy, _ = _setup(n, seed=3)
    with torch.no_grad():
        g = torch.tensor(p.gamma, dtype=torch.float64, device="cuda")
        q0 = kh_initial_state(vy, g, p)
        qf = EulerSteps.apply(q0, g, p, steps, 1000)
        qt, _ = tangent_linear(p, q0, p.gamma, torch.zeros((1,) + tuple(q0.shape), dtype=torch.float64,
                                                                device="cuda"), [0.0], steps)
    assert torch.equal(qf, qt)


def test_adjoint_matches_gpu_tangent_linear(gpu_lib):
    """The reverse sweep against the tangent-linear model on 8 random
    directions (64^2, 40 steps, checkpoints every 20)."""
    from mosscap_b200.adjoint import kh_directional_derivatives
    n, steps, ckpt = 64, 40, 20
    p, vy, pt = _setup(n, seed=8, target_seed=9)
    rho_t = _target_rho(pt, p.gamma, steps)
    J, gvy, gg = _loss_and_grad(p, vy, p.gamma, rho_t, steps, ckpt)
    rng = np.random.default_rng(10)
    dirs = torch.tensor(rng.standard_normal((8, n, n)), device="cuda")
    dgs = [float(x) * 1e-2 for x in rng.standard_normal(8)]
    Jt, dJ = kh_directional_derivatives(p, vy, p.gamma, dirs, dgs, rho_t, steps)
    assert abs(Jt - J) / J < 1e-13, (Jt, J)
    for k in range(8):
        ad = float((gvy * dirs[k]).sum()) + gg * dgs[k]
        assert abs(ad - dJ[k]) / abs(dJ[k]) < 1e-9, (k, ad, dJ[k])


def test_adjoint_zero_steps_is_identity(gpu_lib):
    """A recorded run of 0 steps leaves the state alone and its reverse sweep
    returns the cotangent unchanged with dJ/dgamma = 0."""
    from mosscap_b200.adjoint import _Runner, pad_periodic
    p = P.kelvin_helmholtz_2d(32, seed=0)
    ng = p.ng
    q0 = torch.tensor(p.Q[:, 0, ng:-ng, ng:-ng], dtype=torch.float64, device="cuda")
    qpad = pad_periodic(q0, ng)
    before = qpad.clone()
    runner = _Runner(p, p.gamma, 4)
    runner.forward(qpad, 0)
    lam = torch.randn(qpad.shape, generator=torch.Generator().manual_seed(5), dtype=torch.float64).cuda()
    lam_in = lam.clone()
    dg = runner.backward(lam)
    torch.cuda.synchronize()
    assert torch.equal(qpad, before)
    assert torch.equal(lam, lam_in)
    assert dg == 0.0
