"""Test infrastructure: an FP64 forward-mode (tangent-linear) reference of the
2D Euler step, for checking the discrete adjoint.

The scheme of the reference (source/Reconstruct.hpp WENO5-Z, source/Riemann.hpp
HLLC, source/TimeStepping.cpp SSPRK3, source/Hydro.cpp CFL dt) is written
once, vectorised over a periodic grid, on dual numbers (value, derivative
along one direction). Branches follow the value, as in the adjoint. The
derivative it returns is the exact directional derivative of the discrete
map, independent of the adjoint code.
"""
from __future__ import annotations

import numpy as np


class D:
    __slots__ = ("v", "d")

    def __init__(self, v, d=None):
        self.v = np.asarray(v, dtype=np.float64)
        self.d = np.zeros_like(self.v) if d is None else np.asarray(d, dtype=np.float64)

    def _l(b):
        return b if isinstance(b, D) else D(b)

    def __add__(a, b):
        b = D._l(b)
        return D(a.v + b.v, a.d + b.d)

    __radd__ = __add__

    def __sub__(a, b):
        b = D._l(b)
        return D(a.v - b.v, a.d - b.d)

    def __rsub__(a, b):
        return D._l(b) - a

    def __mul__(a, b):
        b = D._l(b)
        return D(a.v * b.v, a.d * b.v + a.v * b.d)

    __rmul__ = __mul__

    def __truediv__(a, b):
        b = D._l(b)
        q = a.v / b.v
        return D(q, (a.d - q * b.d) / b.v)

    def __rtruediv__(a, b):
        return D._l(b) / a

    def __neg__(a):
        return D(-a.v, -a.d)

    def __getitem__(a, k):
        return D(a.v[k], a.d[k])


def sqrt(a):
    r = np.sqrt(a.v)
    return D(r, a.d / (2.0 * r))


def dabs(a):
    return D(np.abs(a.v), np.sign(a.v) * a.d)


def where(c, a, b):
    a, b = D._l(a), D._l(b)
    return D(np.where(c, a.v, b.v), np.where(c, a.d, b.d))


def smin(a, b):  # std::min(a, b)
    a, b = D._l(a), D._l(b)
    return where(b.v < a.v, b, a)


def smax(a, b):  # std::max(a, b)
    a, b = D._l(a), D._l(b)
    return where(a.v < b.v, b, a)


def roll(a, s, ax):
    return D(np.roll(a.v, s, axis=ax), np.roll(a.d, s, axis=ax))


def prim(q, g):
    rho = q[0]
    vx = q[1] / rho
    vy = q[2] / rho
    p = (g - 1.0) * (q[3] - 0.5 * rho * (vx * vx + vy * vy))
    return rho, vx, vy, p


def weno(s):
    sm2, sm1, c, sp1, sp2 = s
    ba, bb, eps = 13.0 / 12.0, 0.25, 1e-36
    b0 = ba * (sm2 - 2.0 * sm1 + c) * (sm2 - 2.0 * sm1 + c) + bb * (sm2 - 4.0 * sm1 + 3.0 * c) * (sm2 - 4.0 * sm1 + 3.0 * c)
    b1 = ba * (sm1 - 2.0 * c + sp1) * (sm1 - 2.0 * c + sp1) + bb * (sm1 - sp1) * (sm1 - sp1)
    b2 = ba * (c - 2.0 * sp1 + sp2) * (c - 2.0 * sp1 + sp2) + bb * (3.0 * c - 4.0 * sp1 + sp2) * (3.0 * c - 4.0 * sp1 + sp2)
    tau = dabs(b0 - b2)
    i0, i1, i2 = tau / (b0 + eps), tau / (b1 + eps), tau / (b2 + eps)
    a0, a1, a2 = 3.0 * (1.0 + i0 * i0), 6.0 * (1.0 + i1 * i1), 1.0 + i2 * i2
    wl = ((2.0 * c + 5.0 * sm1 - sm2) * a0 + (-sp1 + 5.0 * c + 2.0 * sm1) * a1
          + (2.0 * sp2 - 7.0 * sp1 + 11.0 * c) * a2) / (6.0 * (a0 + a1 + a2))
    a0, a1, a2 = 3.0 * (1.0 + i2 * i2), 6.0 * (1.0 + i1 * i1), 1.0 + i0 * i0
    wr = ((2.0 * c + 5.0 * sp1 - sp2) * a0 + (-sm1 + 5.0 * c + 2.0 * sp1) * a1
          + (2.0 * sm2 - 7.0 * sm1 + 11.0 * c) * a2) / (6.0 * (a0 + a1 + a2))
    return wl, wr


def hllc(wl, wr, g, axis):
    tiny = 1e-20
    rL, uxL, uyL, pL = wl
    rR, uxR, uyR, pR = wr
    vL, vR = (uxL, uxR) if axis == 0 else (uyL, uyR)
    csL, csR = sqrt(g * pL / rL), sqrt(g * pR / rR)
    qL3 = pL / (g - 1.0) + 0.5 * rL * (uxL * uxL + uyL * uyL)
    qR3 = pR / (g - 1.0) + 0.5 * rR * (uxR * uxR + uyR * uyR)
    pm = 0.5 * (pL + pR + (vL - vR) * (0.5 * (rL + rR)) * (0.5 * (csL + csR)))
    gf = (g + 1.0) / (2.0 * g)
    cLs = where(pm.v <= pL.v, D(np.ones_like(pm.v)), sqrt(1.0 + gf * (pm / pL - 1.0)))
    cRs = where(pm.v <= pR.v, D(np.ones_like(pm.v)), sqrt(1.0 + gf * (pm / pR - 1.0)))
    aL = vL - csL * cLs
    aR = vR + csR * cRs
    bM = smin(-tiny, aL)
    bP = smax(tiny, aR)
    uL, uR = vL - aL, vR - aR
    tL = pL + uL * (rL * vL)
    tR = pR + uR * (rR * vR)
    mL, mR = rL * uL, -(rR * uR)
    aM = (tL - tR) / (mL + mR)
    cp = smax((mL * tR + mR * tL) / (mL + mR), 0.0)
    zL, zR = vL - bM, vR - bP
    mfL, mfR = rL * zL, rR * zR
    fL = [mfL, mfL * uxL, mfL * uyL, qL3 * zL + pL * vL]
    fR = [mfR, mfR * uxR, mfR * uyR, qR3 * zR + pR * vR]
    fL[1 + axis] = fL[1 + axis] + pL
    fR[1 + axis] = fR[1 + axis] + pR
    pos = aM.v >= 0.0
    sL = where(pos, aM / (aM - bM), 0.0)
    sR = where(pos, 0.0, -aM / (bP - aM))
    sM = where(pos, -bM / (aM - bM), bP / (bP - aM))
    f = [sL * fL[k] + sR * fR[k] for k in range(4)]
    f[1 + axis] = f[1 + axis] + sM * cp
    f[3] = f[3] + sM * cp * aM
    return f


def rhs_div(q, g):
    """Sum over axes of F(i) - F(i+1) (the integrate_flux divergence)."""
    w = prim(q, g)
    out = [D(np.zeros_like(q.v[0])) for _ in range(4)]
    for axis, ax in ((0, 1), (1, 0)):  # x is the last array axis
        RL, RR = [], []
        for v in range(4):
            st = [roll(w[v], s, ax) for s in (2, 1, 0, -1, -2)]
            l, r = weno(st)
            RL.append(l)
            RR.append(r)
        left = [roll(RR[v], 1, ax) for v in range(4)]
        f = hllc(left, RL, g, axis)
        for v in range(4):
            out[v] = out[v] + (f[v] - roll(f[v], -1, ax))
    return out


def stack(parts):
    return D(np.stack([p.v for p in parts]), np.stack([p.d for p in parts]))


def cfl_min(q, g, dx):
    rho, vx, vy, p = prim(q, g)
    dtl = dx / (sqrt(g * p / rho) + sqrt(vx * vx + vy * vy))
    k = np.unravel_index(np.argmin(dtl.v), dtl.v.shape)
    return D(dtl.v[k], dtl.d[k])


def run(q0, g, dx, cfl, n_steps):
    q = q0
    for _ in range(n_steps):
        dt = cfl * cfl_min(q, g, dx)
        k = dt / dx
        d0 = stack(rhs_div(q, g))
        q1 = q + d0 * k
        d1 = stack(rhs_div(q1, g))
        q2 = 0.75 * q + 0.25 * (q1 + d1 * k)
        d2 = stack(rhs_div(q2, g))
        q = (1.0 / 3.0) * q + (2.0 / 3.0) * (q2 + d2 * k)
    return q


def kh_state(vy, g, n):
    dx = 1.0 / n
    y = (np.arange(n) + 0.5) * dx
    Y = np.repeat(y[:, None], n, axis=1)
    band = np.abs(Y - 0.5) < 0.25
    rho = np.where(band, 2.0, 1.0)
    vx = np.where(band, 0.5, -0.5)
    p = 2.5
    mx = D(rho * vx)
    my = D(rho) * vy
    e = p / (g - 1.0) + 0.5 * D(rho) * (D(vx * vx) + vy * vy)
    return stack([D(rho), mx, my, e])


def directional_derivative(vy, dvy, gamma, dgamma, rho_target, n, cfl, n_steps):
    """d/dt J(vy + t dvy, gamma + t dgamma) at t = 0, with
    J = 1/2 sum (rho_final - rho_target)^2."""
    g = D(gamma, dgamma)
    q0 = kh_state(D(vy, dvy), g, n)
    q = run(q0, g, 1.0 / n, cfl, n_steps)
    r = q[0] - rho_target
    return float(np.sum(r.v * r.d)), float(0.5 * np.sum(r.v * r.v))
