// Reverse-mode (vector-Jacobian) derivatives of the pointwise physics of
// physics.cuh, for the discrete adjoint of the 2D Euler step.
//
// Every function recomputes the forward intermediates it needs from its
// inputs (the forward expressions) and then runs the reverse sweep by hand.
// Branches (min / max, |x|, the HLLC shock-factor test and the contact-speed
// sign) are differentiated along the branch the forward computation takes.
// gamma enters through the sound speed, the ideal-gas energy and the HLLC
// shock-factor coefficient; its adjoint is accumulated in *gbar.
//
// The reverse sweep is a derivative, not a reproduction of the forward
// state, so it need not be bit-exact: every denominator is inverted once
// with arcp() and the quotients that share it become products.
#pragma once

#include "physics.cuh"

namespace mc {

// 1 / d for the reverse sweep: the PTX approximation rcp.approx.ftz.f64
// refined by two Newton-Raphson steps r <- r + r (1 - d r), each of which
// squares the relative error. For normal d with a normal reciprocal (every
// denominator here: densities, pressures, sound speeds, the WENO weight sums,
// regularised smoothness indicators and HLLC wave-speed differences).
__device__ __forceinline__ double arcp(double d) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
    double e = fma(-d, r, 1.0);
    r = fma(r, e, r);
    e = fma(-d, r, 1.0);
    return fma(r, e, r);
}

// Constants of the ideal gas shared by every face.
struct GasK {
    double gamma, gm1, rgm1;  // gamma, gamma - 1, 1 / (gamma - 1)
    double gfac;              // (gamma + 1) / (2 gamma), HLLC shock factor
    double dgfac;             // d gfac / d gamma = -1 / (2 gamma^2)
};

__host__ __device__ inline GasK gas_constants(double gamma) {
    GasK k;
    k.gamma = gamma;
    k.gm1 = gamma - 1.0;
    k.rgm1 = 1.0 / k.gm1;
    k.gfac = (gamma + 1.0) / (2.0 * gamma);
    k.dgfac = -1.0 / (2.0 * gamma * gamma);
    return k;
}

// cons_to_prim, 2D (source/Eos.hpp:61-79), for the reverse sweep.
__device__ __forceinline__ void prim_from_cons_rev2(double gm1, const double* q, double* w) {
    const double rr = arcp(q[0]);
    w[0] = q[0];
    w[1] = q[1] * rr;
    w[2] = q[2] * rr;
    w[3] = gm1 * (q[3] - 0.5 * q[0] * (w[1] * w[1] + w[2] * w[2]));
}

// cons_to_prim, 2D: w = (rho, m_x/rho, m_y/rho, (gamma-1)(E - rho |v|^2 / 2)).
// Given the cotangent wb of w, returns the cotangent qb of q.
__device__ __forceinline__ void prim_from_cons_vjp2(double gamma, const double* q, const double* wb, double* qb,
                                                    double* gbar) {
    const double rho = q[0];
    const double rr = arcp(rho);
    const double vx = q[1] * rr;
    const double vy = q[2] * rr;
    const double v2 = vx * vx + vy * vy;
    const double ekin = 0.5 * rho * v2;
    const double pb = wb[3];
    const double Eb = pb * (gamma - 1.0);
    const double ekb = -Eb;
    *gbar += pb * (q[3] - ekin);
    double rhob = wb[0] + ekb * 0.5 * v2;
    const double v2b = ekb * 0.5 * rho;
    const double vxb = wb[1] + v2b * 2.0 * vx;
    const double vyb = wb[2] + v2b * 2.0 * vy;
    qb[1] = vxb * rr;
    qb[2] = vyb * rr;
    rhob -= (vxb * vx + vyb * vy) * rr;
    qb[0] = rhob;
    qb[3] = Eb;
}

// Forward intermediates of the WENO5-Z face values (reconstruct<kWeno5z>,
// source/Reconstruct.hpp:217-274) on the stencil s[0..4] (offsets -2..2).
struct WenoZ {
    double t01, t02, t11, t12, t21, t22;  // the squared terms of the smoothness indicators
    double diff;                          // beta0 - beta2
    double r0, r1, r2;                    // 1 / (beta_k + eps)
    double ind0, ind1, ind2;              // tau5 / (beta_k + eps)
    double e0, e1, e2, f0, f1, f2;        // candidate values (x 6), left / right face
    double a0, a1, a2, b0, b1, b2;        // unnormalised weights, left / right face
    double rden, rdenR;                   // 1 / (6 sum of weights)
    double wl, wr;                        // the face values
};

__device__ __forceinline__ void wenoz_eval(const double* s, WenoZ& z) {
    const double c = s[2];
    const double b_a = 13.0 / 12.0, b_b = 0.25, eps = Consts<double>::weno_eps;
    z.t01 = s[0] - 2.0 * s[1] + c;
    z.t02 = s[0] - 4.0 * s[1] + 3.0 * c;
    z.t11 = s[1] - 2.0 * c + s[3];
    z.t12 = s[1] - s[3];
    z.t21 = c - 2.0 * s[3] + s[4];
    z.t22 = 3.0 * c - 4.0 * s[3] + s[4];
    const double beta0 = b_a * z.t01 * z.t01 + b_b * z.t02 * z.t02;
    const double beta1 = b_a * z.t11 * z.t11 + b_b * z.t12 * z.t12;
    const double beta2 = b_a * z.t21 * z.t21 + b_b * z.t22 * z.t22;
    z.diff = beta0 - beta2;
    const double tau5 = fabs(z.diff);
    z.r0 = arcp(beta0 + eps);
    z.r1 = arcp(beta1 + eps);
    z.r2 = arcp(beta2 + eps);
    z.ind0 = tau5 * z.r0;
    z.ind1 = tau5 * z.r1;
    z.ind2 = tau5 * z.r2;
    z.e0 = 2.0 * c + 5.0 * s[1] - s[0];
    z.e1 = -s[3] + 5.0 * c + 2.0 * s[1];
    z.e2 = 2.0 * s[4] - 7.0 * s[3] + 11.0 * c;
    z.f0 = 2.0 * c + 5.0 * s[3] - s[4];
    z.f1 = -s[1] + 5.0 * c + 2.0 * s[3];
    z.f2 = 2.0 * s[0] - 7.0 * s[1] + 11.0 * c;
    const double q0 = 1.0 + z.ind0 * z.ind0, q1 = 1.0 + z.ind1 * z.ind1, q2 = 1.0 + z.ind2 * z.ind2;
    z.a0 = 3.0 * q0;
    z.a1 = 6.0 * q1;
    z.a2 = q2;
    z.b0 = 3.0 * q2;
    z.b1 = z.a1;
    z.b2 = q0;
    z.rden = arcp(6.0 * (z.a0 + z.a1 + z.a2));
    z.rdenR = arcp(6.0 * (z.b0 + z.b1 + z.b2));
    z.wl = (z.e0 * z.a0 + z.e1 * z.a1 + z.e2 * z.a2) * z.rden;
    z.wr = (z.f0 * z.b0 + z.f1 * z.b1 + z.f2 * z.b2) * z.rdenR;
}

// WENO5-Z face values only.
__device__ __forceinline__ void weno5z_faces(const double* s, double& wl, double& wr) {
    WenoZ z;
    wenoz_eval(s, z);
    wl = z.wl;
    wr = z.wr;
}

// WENO5-Z vector-Jacobian product: given cotangents gl, gr of the left /
// right face values, adds the cotangent of stencil point k (offset k - 2) to
// sb[k].
__device__ __forceinline__ void weno5z_vjp(const double* s, double gl, double gr, double* sb) {
    WenoZ z;
    wenoz_eval(s, z);
    const double b_a = 13.0 / 12.0, b_b = 0.25;
    const double nLb = gl * z.rden, denb = -nLb * z.wl;
    const double nRb = gr * z.rdenR, denRb = -nRb * z.wr;
    const double e0b = nLb * z.a0, e1b = nLb * z.a1, e2b = nLb * z.a2;
    const double f0b = nRb * z.b0, f1b = nRb * z.b1, f2b = nRb * z.b2;
    const double a0b = nLb * z.e0 + 6.0 * denb, a1b = nLb * z.e1 + 6.0 * denb, a2b = nLb * z.e2 + 6.0 * denb;
    const double b0b = nRb * z.f0 + 6.0 * denRb, b1b = nRb * z.f1 + 6.0 * denRb, b2b = nRb * z.f2 + 6.0 * denRb;
    const double ind0b = (a0b * 6.0 + b2b * 2.0) * z.ind0;
    const double ind1b = (a1b + b1b) * 12.0 * z.ind1;
    const double ind2b = (a2b * 2.0 + b0b * 6.0) * z.ind2;
    const double tau5b = ind0b * z.r0 + ind1b * z.r1 + ind2b * z.r2;
    const double sg = z.diff > 0.0 ? 1.0 : (z.diff < 0.0 ? -1.0 : 0.0);
    const double beta0b = -ind0b * z.ind0 * z.r0 + sg * tau5b;
    const double beta1b = -ind1b * z.ind1 * z.r1;
    const double beta2b = -ind2b * z.ind2 * z.r2 - sg * tau5b;
    const double t01b = beta0b * 2.0 * b_a * z.t01, t02b = beta0b * 2.0 * b_b * z.t02;
    const double t11b = beta1b * 2.0 * b_a * z.t11, t12b = beta1b * 2.0 * b_b * z.t12;
    const double t21b = beta2b * 2.0 * b_a * z.t21, t22b = beta2b * 2.0 * b_b * z.t22;
    sb[0] += t01b + t02b - e0b + 2.0 * f2b;
    sb[1] += -2.0 * t01b - 4.0 * t02b + t11b + t12b + 5.0 * e0b + 2.0 * e1b - f1b - 7.0 * f2b;
    sb[2] += t01b + 3.0 * t02b - 2.0 * t11b + t21b + 3.0 * t22b + 2.0 * e0b + 5.0 * e1b + 11.0 * e2b + 2.0 * f0b +
             5.0 * f1b + 11.0 * f2b;
    sb[3] += t11b - t12b - 2.0 * t21b - 4.0 * t22b - e1b - 7.0 * e2b + 5.0 * f0b + 2.0 * f1b;
    sb[4] += t21b + t22b + 2.0 * e2b - f0b;
}

// HLLC interface flux (riemann<kHllc>, 2D; source/Riemann.hpp:75-176) along
// `axis`, returning the forward flux in f and, for the flux cotangent fb, the
// cotangents of the left / right primitive states in wLb / wRb (overwritten)
// and of gamma (added to *gbar).
__device__ __forceinline__ void hllc_vjp2(const GasK& K, int axis, const double* wL, const double* wR,
                                          const double* fb, double* f, double* wLb, double* wRb, double* gbar) {
    const double tiny = 1e-20;
    const double gamma = K.gamma, gfac = K.gfac, rgm1 = K.rgm1;
    const bool ax0 = axis == 0;  // normal velocity / momentum: index 1 (x) or 2 (y)
    const double rL = wL[0], uxL = wL[1], uyL = wL[2], pL = wL[3];
    const double rR = wR[0], uxR = wR[1], uyR = wR[2], pR = wR[3];
    const double vL = ax0 ? uxL : uyL;
    const double vR = ax0 ? uxR : uyR;
    // forward
    const double rrL = arcp(rL), rrR = arcp(rR);
    const double csL = sqrt(gamma * pL * rrL), csR = sqrt(gamma * pR * rrR);
    const double v2L = uxL * uxL + uyL * uyL, v2R = uxR * uxR + uyR * uyR;
    const double qL3 = pL * rgm1 + 0.5 * rL * v2L, qR3 = pR * rgm1 + 0.5 * rR * v2R;
    const double qLn = rL * vL, qRn = rR * vR;
    const double rho_avg = 0.5 * (rL + rR), cs_avg = 0.5 * (csL + csR);
    const double dv = vL - vR;
    const double p_mid = 0.5 * (pL + pR + dv * rho_avg * cs_avg);
    const bool shockL = !(p_mid <= pL), shockR = !(p_mid <= pR);
    const double rpL = shockL ? arcp(pL) : 0.0, rpR = shockR ? arcp(pR) : 0.0;
    const double xL = shockL ? 1.0 + gfac * (p_mid * rpL - 1.0) : 1.0;
    const double xR = shockR ? 1.0 + gfac * (p_mid * rpR - 1.0) : 1.0;
    const double cLs = shockL ? sqrt(xL) : 1.0, cRs = shockR ? sqrt(xR) : 1.0;
    const double aL = vL - csL * cLs, aR = vR + csR * cRs;
    const bool takeL = aL < -tiny, takeR = tiny < aR;
    const double bM = takeL ? aL : -tiny, bP = takeR ? aR : tiny;
    const double uL = vL - aL, uR = vR - aR;
    const double tL = pL + uL * qLn, tR = pR + uR * qRn;
    const double mL = rL * uL, mR = -(rR * uR);
    const double rS = arcp(mL + mR);
    const double aM = (tL - tR) * rS;
    const double cpr = (mL * tR + mR * tL) * rS;
    const bool cp_open = !(cpr < 0.0);
    const double cp = cp_open ? cpr : 0.0;
    const double zL = vL - bM, zR = vR - bP;
    const double mfL = rL * zL, mfR = rR * zR;
    double fL[4], fR[4];
    fL[0] = mfL;
    fR[0] = mfR;
    fL[1] = mfL * uxL;
    fR[1] = mfR * uxR;
    fL[2] = mfL * uyL;
    fR[2] = mfR * uyR;
    fL[1] += ax0 ? pL : 0.0;
    fL[2] += ax0 ? 0.0 : pL;
    fR[1] += ax0 ? pR : 0.0;
    fR[2] += ax0 ? 0.0 : pR;
    fL[3] = qL3 * zL + pL * vL;
    fR[3] = qR3 * zR + pR * vR;
    const bool pos = aM >= 0.0;
    const double rD = arcp(pos ? aM - bM : bP - aM);
    double sL, sR, sM;
    if (pos) {
        sL = aM * rD;
        sR = 0.0;
        sM = -bM * rD;
    } else {
        sL = 0.0;
        sR = -aM * rD;
        sM = bP * rD;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        f[k] = sL * fL[k] + sR * fR[k];
    }
    f[1] += ax0 ? sM * cp : 0.0;
    f[2] += ax0 ? 0.0 : sM * cp;
    f[3] += sM * cp * aM;

    // reverse
    const double fbn = ax0 ? fb[1] : fb[2];
    const double sMb = fb[3] * cp * aM + fbn * cp;
    const double cpb = fb[3] * sM * aM + fbn * sM;
    double aMb = fb[3] * sM * cp;
    double sLb = 0.0, sRb = 0.0;
    double fLb[4], fRb[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        sLb += fb[k] * fL[k];
        sRb += fb[k] * fR[k];
        fLb[k] = fb[k] * sL;
        fRb[k] = fb[k] * sR;
    }
    double bMb = 0.0, bPb = 0.0;
    if (pos) {
        const double Db = -(sLb * sL + sMb * sM) * rD;
        aMb += sLb * rD + Db;
        bMb += -sMb * rD - Db;
    } else {
        const double Db = -(sRb * sR + sMb * sM) * rD;
        aMb += -sRb * rD - Db;
        bPb += sMb * rD + Db;
    }
    // fluxes of the two sides
    double rLb = 0.0, rRb = 0.0, uxLb = 0.0, uxRb = 0.0, uyLb = 0.0, uyRb = 0.0, pLb = 0.0, pRb = 0.0;
    double vLb = 0.0, vRb = 0.0;
    const double mfLb = fLb[0] + fLb[1] * uxL + fLb[2] * uyL;
    const double mfRb = fRb[0] + fRb[1] * uxR + fRb[2] * uyR;
    uxLb += fLb[1] * mfL;
    uyLb += fLb[2] * mfL;
    uxRb += fRb[1] * mfR;
    uyRb += fRb[2] * mfR;
    pLb += (ax0 ? fLb[1] : fLb[2]) + fLb[3] * vL;
    pRb += (ax0 ? fRb[1] : fRb[2]) + fRb[3] * vR;
    const double qL3b = fLb[3] * zL, qR3b = fRb[3] * zR;
    const double zLb = fLb[3] * qL3 + mfLb * rL, zRb = fRb[3] * qR3 + mfRb * rR;
    vLb += fLb[3] * pL + zLb;
    vRb += fRb[3] * pR + zRb;
    rLb += mfLb * zL;
    rRb += mfRb * zR;
    bMb -= zLb;
    bPb -= zRb;
    // contact pressure and speed
    const double cprb = cp_open ? cpb : 0.0;
    const double Sb = -(cprb * cpr + aMb * aM) * rS;
    const double mLb = cprb * tR * rS + Sb, mRb = cprb * tL * rS + Sb;
    const double tRb = (cprb * mL - aMb) * rS, tLb = (cprb * mR + aMb) * rS;
    rLb += mLb * uL;
    const double uLb = mLb * rL + tLb * qLn;
    rRb += -mRb * uR;
    const double uRb = -mRb * rR + tRb * qRn;
    pLb += tLb;
    pRb += tRb;
    const double qLnb = tLb * uL, qRnb = tRb * uR;
    vLb += uLb;
    vRb += uRb;
    double aLb = -uLb, aRb = -uRb;
    if (takeL) {
        aLb += bMb;
    }
    if (takeR) {
        aRb += bPb;
    }
    // outer wave speeds
    vLb += aLb;
    vRb += aRb;
    double csLb = -aLb * cLs, csRb = aRb * cRs;
    const double cLsb = -aLb * csL, cRsb = aRb * csR;
    double p_midb = 0.0, gfacb = 0.0;
    if (shockL) {
        const double xb = 0.5 * cLsb * arcp(cLs);
        const double r = p_mid * rpL;
        gfacb += xb * (r - 1.0);
        const double rb = xb * gfac;
        p_midb += rb * rpL;
        pLb -= rb * r * rpL;
    }
    if (shockR) {
        const double xb = 0.5 * cRsb * arcp(cRs);
        const double r = p_mid * rpR;
        gfacb += xb * (r - 1.0);
        const double rb = xb * gfac;
        p_midb += rb * rpR;
        pRb -= rb * r * rpR;
    }
    pLb += 0.5 * p_midb;
    pRb += 0.5 * p_midb;
    const double dvb = 0.5 * p_midb * rho_avg * cs_avg;
    const double rho_avgb = 0.5 * p_midb * dv * cs_avg;
    const double cs_avgb = 0.5 * p_midb * dv * rho_avg;
    vLb += dvb;
    vRb -= dvb;
    rLb += 0.5 * rho_avgb;
    rRb += 0.5 * rho_avgb;
    csLb += 0.5 * cs_avgb;
    csRb += 0.5 * cs_avgb;
    // conserved normal momentum and total energy of the two sides
    rLb += qLnb * vL;
    vLb += qLnb * rL;
    rRb += qRnb * vR;
    vRb += qRnb * rR;
    pLb += qL3b * rgm1;
    pRb += qR3b * rgm1;
    double gb = -(qL3b * pL + qR3b * pR) * (rgm1 * rgm1);
    rLb += qL3b * 0.5 * v2L;
    rRb += qR3b * 0.5 * v2R;
    uxLb += qL3b * rL * uxL;
    uyLb += qL3b * rL * uyL;
    uxRb += qR3b * rR * uxR;
    uyRb += qR3b * rR * uyR;
    // sound speeds c = sqrt(gamma p / rho)
    {
        const double k = 0.5 * csLb * arcp(csL) * rrL;
        gb += k * pL;
        pLb += k * gamma;
        rLb -= k * gamma * pL * rrL;
    }
    {
        const double k = 0.5 * csRb * arcp(csR) * rrR;
        gb += k * pR;
        pRb += k * gamma;
        rRb -= k * gamma * pR * rrR;
    }
    gb += gfacb * K.dgfac;
    *gbar += gb;
    if (ax0) {
        uxLb += vLb;
        uxRb += vRb;
    } else {
        uyLb += vLb;
        uyRb += vRb;
    }
    wLb[0] = rLb;
    wLb[1] = uxLb;
    wLb[2] = uyLb;
    wLb[3] = pLb;
    wRb[0] = rRb;
    wRb[1] = uxRb;
    wRb[2] = uyRb;
    wRb[3] = pRb;
}

// CFL bound of one cell (dt_reducer, source/Hydro.cpp:192-206) from its
// conserved state, and its gradient: qb = dt_local / dq, *gbar += d/dgamma.
__device__ __forceinline__ double cfl_dt_grad2(double gamma, double dx, const double* q, double* qb, double* gbar) {
    double w[4];
    prim_from_cons<2>(gamma, q, w);
    const double cs = sqrt(gamma * w[3] / w[0]);
    const double vel = sqrt(w[1] * w[1] + w[2] * w[2]);
    const double den = cs + vel;
    const double dtl = dx / den;
    const double denb = -dx / (den * den);
    const double csb = denb, velb = denb;
    double wb[4];
    const double k = csb / (2.0 * cs * w[0]);
    double gb = k * w[3];
    wb[3] = k * gamma;
    wb[0] = -k * gamma * w[3] / w[0];
    wb[1] = vel > 0.0 ? velb * w[1] / vel : 0.0;
    wb[2] = vel > 0.0 ? velb * w[2] / vel : 0.0;
    prim_from_cons_vjp2(gamma, q, wb, qb, &gb);
    *gbar += gb;
    return dtl;
}

} // namespace mc
