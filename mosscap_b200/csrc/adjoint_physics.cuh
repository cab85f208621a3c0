// Reverse-mode (vector-Jacobian) derivatives of the pointwise physics of
// physics.cuh, for the discrete adjoint of the 2D Euler step.
//
// Every function recomputes the forward intermediates it needs from its
// inputs (same expressions as the forward code) and then runs the reverse
// sweep by hand. Branches (min / max, |x|, the HLLC shock-factor test and the
// contact-speed sign) are differentiated along the branch the forward
// computation takes. gamma enters through the sound speed, the ideal-gas
// energy and the HLLC shock-factor coefficient; its adjoint is accumulated
// in *gbar.
#pragma once

#include "physics.cuh"

namespace mc {

// cons_to_prim, 2D: w = (rho, m_x/rho, m_y/rho, (gamma-1)(E - rho |v|^2 / 2)).
// Given the cotangent wb of w, returns the cotangent qb of q.
__device__ __forceinline__ void prim_from_cons_vjp2(double gamma, const double* q, const double* wb, double* qb,
                                                    double* gbar) {
    const double rho = q[0];
    const double vx = q[1] / rho;
    const double vy = q[2] / rho;
    const double v2 = vx * vx + vy * vy;
    const double ekin = 0.5 * rho * v2;
    const double pb = wb[3];
    const double Eb = pb * (gamma - 1.0);
    const double ekb = -pb * (gamma - 1.0);
    *gbar += pb * (q[3] - ekin);
    double rhob = wb[0] + ekb * 0.5 * v2;
    const double v2b = ekb * 0.5 * rho;
    const double vxb = wb[1] + v2b * 2.0 * vx;
    const double vyb = wb[2] + v2b * 2.0 * vy;
    qb[1] = vxb / rho;
    qb[2] = vyb / rho;
    rhob -= (vxb * vx + vyb * vy) / rho;
    qb[0] = rhob;
    qb[3] = Eb;
}

// WENO5-Z face values (reconstruct<kWeno5z>) and their vector-Jacobian
// product: given cotangents gl, gr of the left / right face values, adds the
// cotangent of stencil point k (offset k - 2) to sb[k].
__device__ __forceinline__ void weno5z_vjp(const double* s, double gl, double gr, double* sb) {
    const double c = s[2];
    const double b_a = 13.0 / 12.0, b_b = 0.25, eps = 1e-36;
    const double t01 = s[0] - 2.0 * s[1] + c, t02 = s[0] - 4.0 * s[1] + 3.0 * c;
    const double t11 = s[1] - 2.0 * c + s[3], t12 = s[1] - s[3];
    const double t21 = c - 2.0 * s[3] + s[4], t22 = 3.0 * c - 4.0 * s[3] + s[4];
    const double beta0 = b_a * t01 * t01 + b_b * t02 * t02;
    const double beta1 = b_a * t11 * t11 + b_b * t12 * t12;
    const double beta2 = b_a * t21 * t21 + b_b * t22 * t22;
    const double diff = beta0 - beta2;
    const double tau5 = fabs(diff);
    const double d0 = beta0 + eps, d1 = beta1 + eps, d2 = beta2 + eps;
    const double ind0 = tau5 / d0, ind1 = tau5 / d1, ind2 = tau5 / d2;
    // left face
    const double e0 = 2.0 * c + 5.0 * s[1] - s[0];
    const double e1 = -s[3] + 5.0 * c + 2.0 * s[1];
    const double e2 = 2.0 * s[4] - 7.0 * s[3] + 11.0 * c;
    const double a0 = 3.0 * (1.0 + ind0 * ind0), a1 = 6.0 * (1.0 + ind1 * ind1), a2 = 1.0 + ind2 * ind2;
    const double den = 6.0 * (a0 + a1 + a2);
    const double wl = (e0 * a0 + e1 * a1 + e2 * a2) / den;
    // right face
    const double f0 = 2.0 * c + 5.0 * s[3] - s[4];
    const double f1 = -s[1] + 5.0 * c + 2.0 * s[3];
    const double f2 = 2.0 * s[0] - 7.0 * s[1] + 11.0 * c;
    const double b0 = 3.0 * (1.0 + ind2 * ind2), b1 = 6.0 * (1.0 + ind1 * ind1), b2 = 1.0 + ind0 * ind0;
    const double denR = 6.0 * (b0 + b1 + b2);
    const double wr = (f0 * b0 + f1 * b1 + f2 * b2) / denR;
    // reverse
    const double nLb = gl / den, denb = -gl * wl / den;
    const double nRb = gr / denR, denRb = -gr * wr / denR;
    const double e0b = nLb * a0, e1b = nLb * a1, e2b = nLb * a2;
    const double f0b = nRb * b0, f1b = nRb * b1, f2b = nRb * b2;
    const double a0b = nLb * e0 + 6.0 * denb, a1b = nLb * e1 + 6.0 * denb, a2b = nLb * e2 + 6.0 * denb;
    const double b0b = nRb * f0 + 6.0 * denRb, b1b = nRb * f1 + 6.0 * denRb, b2b = nRb * f2 + 6.0 * denRb;
    const double ind0b = a0b * 6.0 * ind0 + b2b * 2.0 * ind0;
    const double ind1b = a1b * 12.0 * ind1 + b1b * 12.0 * ind1;
    const double ind2b = a2b * 2.0 * ind2 + b0b * 6.0 * ind2;
    const double tau5b = ind0b / d0 + ind1b / d1 + ind2b / d2;
    const double sg = diff > 0.0 ? 1.0 : (diff < 0.0 ? -1.0 : 0.0);
    const double beta0b = -ind0b * ind0 / d0 + sg * tau5b;
    const double beta1b = -ind1b * ind1 / d1;
    const double beta2b = -ind2b * ind2 / d2 - sg * tau5b;
    const double t01b = beta0b * 2.0 * b_a * t01, t02b = beta0b * 2.0 * b_b * t02;
    const double t11b = beta1b * 2.0 * b_a * t11, t12b = beta1b * 2.0 * b_b * t12;
    const double t21b = beta2b * 2.0 * b_a * t21, t22b = beta2b * 2.0 * b_b * t22;
    sb[0] += t01b + t02b - e0b + 2.0 * f2b;
    sb[1] += -2.0 * t01b - 4.0 * t02b + t11b + t12b + 5.0 * e0b + 2.0 * e1b - f1b - 7.0 * f2b;
    sb[2] += t01b + 3.0 * t02b - 2.0 * t11b + t21b + 3.0 * t22b + 2.0 * e0b + 5.0 * e1b + 11.0 * e2b + 2.0 * f0b +
             5.0 * f1b + 11.0 * f2b;
    sb[3] += t11b - t12b - 2.0 * t21b - 4.0 * t22b - e1b - 7.0 * e2b + 5.0 * f0b + 2.0 * f1b;
    sb[4] += t21b + t22b + 2.0 * e2b - f0b;
}

// HLLC interface flux (riemann<kHllc>, 2D) along `axis`, returning the
// forward flux in f and, for the flux cotangent fb, the cotangents of the
// left / right primitive states in wLb / wRb (overwritten) and of gamma
// (added to *gbar).
__device__ __forceinline__ void hllc_vjp2(double gamma, int axis, const double* wL, const double* wR,
                                          const double* fb, double* f, double* wLb, double* wRb, double* gbar) {
    const double tiny = 1e-20;
    const double gfac = (gamma + 1.0) / (2.0 * gamma);
    const double gm1 = gamma - 1.0;
    const int iv = 1 + axis;  // index of the normal velocity / momentum
    const double rL = wL[0], uxL = wL[1], uyL = wL[2], pL = wL[3];
    const double rR = wR[0], uxR = wR[1], uyR = wR[2], pR = wR[3];
    const double vL = axis == 0 ? uxL : uyL;
    const double vR = axis == 0 ? uxR : uyR;
    // forward
    const double csL = sqrt(gamma * pL / rL), csR = sqrt(gamma * pR / rR);
    const double v2L = uxL * uxL + uyL * uyL, v2R = uxR * uxR + uyR * uyR;
    const double qL3 = pL / gm1 + 0.5 * rL * v2L, qR3 = pR / gm1 + 0.5 * rR * v2R;
    const double qLn = rL * vL, qRn = rR * vR;
    const double rho_avg = 0.5 * (rL + rR), cs_avg = 0.5 * (csL + csR);
    const double dv = vL - vR;
    const double p_mid = 0.5 * (pL + pR + dv * rho_avg * cs_avg);
    const bool shockL = !(p_mid <= pL), shockR = !(p_mid <= pR);
    const double xL = shockL ? 1.0 + gfac * (p_mid / pL - 1.0) : 1.0;
    const double xR = shockR ? 1.0 + gfac * (p_mid / pR - 1.0) : 1.0;
    const double cLs = shockL ? sqrt(xL) : 1.0, cRs = shockR ? sqrt(xR) : 1.0;
    const double aL = vL - csL * cLs, aR = vR + csR * cRs;
    const bool takeL = aL < -tiny, takeR = tiny < aR;
    const double bM = takeL ? aL : -tiny, bP = takeR ? aR : tiny;
    const double uL = vL - aL, uR = vR - aR;
    const double tL = pL + uL * qLn, tR = pR + uR * qRn;
    const double mL = rL * uL, mR = -(rR * uR);
    const double S = mL + mR;
    const double aM = (tL - tR) / S;
    const double cpr = (mL * tR + mR * tL) / S;
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
    fL[iv] += pL;
    fR[iv] += pR;
    fL[3] = qL3 * zL + pL * vL;
    fR[3] = qR3 * zR + pR * vR;
    const bool pos = aM >= 0.0;
    double sL, sR, sM, D;
    if (pos) {
        D = aM - bM;
        sL = aM / D;
        sR = 0.0;
        sM = -bM / D;
    } else {
        D = bP - aM;
        sL = 0.0;
        sR = -aM / D;
        sM = bP / D;
    }
    for (int k = 0; k < 4; ++k) {
        f[k] = sL * fL[k] + sR * fR[k];
    }
    f[iv] += sM * cp;
    f[3] += sM * cp * aM;

    // reverse
    double sMb = fb[3] * cp * aM + fb[iv] * cp;
    double cpb = fb[3] * sM * aM + fb[iv] * sM;
    double aMb = fb[3] * sM * cp;
    double sLb = 0.0, sRb = 0.0;
    double fLb[4], fRb[4];
    for (int k = 0; k < 4; ++k) {
        sLb += fb[k] * fL[k];
        sRb += fb[k] * fR[k];
        fLb[k] = fb[k] * sL;
        fRb[k] = fb[k] * sR;
    }
    double bMb = 0.0, bPb = 0.0;
    if (pos) {
        const double Db = -(sLb * sL + sMb * sM) / D;
        aMb += sLb / D + Db;
        bMb += -sMb / D - Db;
    } else {
        const double Db = -(sRb * sR + sMb * sM) / D;
        aMb += -sRb / D - Db;
        bPb += sMb / D + Db;
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
    pLb += fLb[iv] + fLb[3] * vL;
    pRb += fRb[iv] + fRb[3] * vR;
    double qL3b = fLb[3] * zL, qR3b = fRb[3] * zR;
    double zLb = fLb[3] * qL3 + mfLb * rL, zRb = fRb[3] * qR3 + mfRb * rR;
    vLb += fLb[3] * pL + zLb;
    vRb += fRb[3] * pR + zRb;
    rLb += mfLb * zL;
    rRb += mfRb * zR;
    bMb -= zLb;
    bPb -= zRb;
    // contact pressure and speed
    const double cprb = cp_open ? cpb : 0.0;
    const double Sb = -(cprb * cpr + aMb * aM) / S;
    const double mLb = cprb * tR / S + Sb, mRb = cprb * tL / S + Sb;
    const double tRb = cprb * mL / S - aMb / S, tLb = cprb * mR / S + aMb / S;
    rLb += mLb * uL;
    double uLb = mLb * rL + tLb * qLn;
    rRb += -mRb * uR;
    double uRb = -mRb * rR + tRb * qRn;
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
        const double xb = cLsb / (2.0 * cLs);
        const double r = p_mid / pL;
        gfacb += xb * (r - 1.0);
        const double rb = xb * gfac;
        p_midb += rb / pL;
        pLb -= rb * r / pL;
    }
    if (shockR) {
        const double xb = cRsb / (2.0 * cRs);
        const double r = p_mid / pR;
        gfacb += xb * (r - 1.0);
        const double rb = xb * gfac;
        p_midb += rb / pR;
        pRb -= rb * r / pR;
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
    pLb += qL3b / gm1;
    pRb += qR3b / gm1;
    double gb = -(qL3b * pL + qR3b * pR) / (gm1 * gm1);
    rLb += qL3b * 0.5 * v2L;
    rRb += qR3b * 0.5 * v2R;
    uxLb += qL3b * rL * uxL;
    uyLb += qL3b * rL * uyL;
    uxRb += qR3b * rR * uxR;
    uyRb += qR3b * rR * uyR;
    // sound speeds
    {
        const double k = csLb / (2.0 * csL * rL);
        gb += k * pL;
        pLb += k * gamma;
        rLb -= k * gamma * pL / rL;
    }
    {
        const double k = csRb / (2.0 * csR * rR);
        gb += k * pR;
        pRb += k * gamma;
        rRb -= k * gamma * pR / rR;
    }
    gb += gfacb * (-1.0 / (2.0 * gamma * gamma));
    *gbar += gb;
    if (axis == 0) {
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
