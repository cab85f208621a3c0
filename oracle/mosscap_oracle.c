/*
 * Oracle test infrastructure, not product code.
 *
 * Plain-C restatement of Mosscap's finite-volume Euler step (the hydro hot
 * path), used only as the correctness checker and as a CPU baseline. Every
 * floating-point expression keeps the reference's evaluation order so that
 * results are bit-identical to the reference compiled without FMA
 * contraction (build with -ffp-contract=off). Each function names the
 * reference file:line it restates. Enum ordinals and the data layout
 * ([var][k][j][i], i fastest, ng ghosts on every active axis) are the
 * reference's (source/State.hpp:10-29,101-106).
 */
#include "moracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

enum { FOG = 0, MUSCL = 1, PPM = 2, WENO5Z = 3 };
enum { VANLEER = 0, MONOTONIZED_CENTRAL = 1, MINMOD = 2 };
enum { RUSANOV = 0, HLL = 1, HLLC = 2 };
enum { RK2 = 0, SSPRK3 = 1, SSPRK4 = 2 };
enum { BC_WALL = 0, BC_PERIODIC, BC_SYMMETRIC, BC_DIODE, BC_ZEROGRAD, BC_CONSTANT, BC_USERFN };

#define MAXV 16

typedef struct {
    moracle_config c;
    int ndim, nhydro, nvar;
    int xc, yc, zc, ng;
    double *Q, *W, *RL, *RR, *F[3], *Qold;
    double time, prev_output_time;
    long long step;
    int gravity;
    double grav[3];
    /* non-ideal EOS (moracle_set_eos) */
    int eos_type, eos_ion;
    double avg_mass;
    double *y_space, *T_space;
    moracle_eos_table tab;
    double *ytab, *lTtab;
} osim;

/* std::min / std::max semantics (first argument wins ties and NaN compares). */
static inline double smin(double a, double b) { return (b < a) ? b : a; }
static inline double smax(double a, double b) { return (a < b) ? b : a; }
static inline double sq(double t) { return t * t; }

static inline long long at(const osim* s, int v, int k, int j, int i) {
    return (((long long)v * s->zc + k) * s->yc + j) * (long long)s->xc + i;
}

/* Index of the velocity / momentum along an axis: 1 + axis
 * (source/State.hpp:10-26, Velocity<> / Momentum<> :41-61). */
static inline int vel_idx(int axis) { return 1 + axis; }

/* ---- Eos.hpp ----------------------------------------------------------- */

/* sound_speed, source/Eos.hpp:54-59 */
static inline double sound_speed(int ndim, double gamma, const double* w) {
    return sqrt(gamma * w[1 + ndim] / w[0]);
}

/* cons_to_prim, source/Eos.hpp:61-79 */
static inline void cons_to_prim(int ndim, double gamma, const double* q, double* w) {
    w[0] = q[0];
    w[1] = q[1] / q[0];
    double v2 = sq(w[1]);
    if (ndim > 1) {
        w[2] = q[2] / q[0];
        v2 += sq(w[2]);
    }
    if (ndim > 2) {
        w[3] = q[3] / q[0];
        v2 += sq(w[3]);
    }
    const double e_kin = 0.5 * q[0] * v2;
    w[1 + ndim] = (gamma - 1.0) * (q[1 + ndim] - e_kin);
}

/* prim_to_cons, source/Eos.hpp:81-99 */
static inline void prim_to_cons(int ndim, double gamma, const double* w, double* q) {
    q[0] = w[0];
    q[1] = w[0] * w[1];
    double v2 = sq(w[1]);
    if (ndim > 1) {
        q[2] = w[0] * w[2];
        v2 += sq(w[2]);
    }
    if (ndim > 2) {
        q[3] = w[0] * w[3];
        v2 += sq(w[3]);
    }
    const double e_kin = 0.5 * w[0] * v2;
    const double e_int = w[1 + ndim] / (gamma - 1.0);
    q[1 + ndim] = e_int + e_kin;
}

/* prim_to_flux, source/Eos.hpp:101-131 */
static inline void prim_to_flux(int axis, int ndim, double gamma, const double* w, double* f) {
    const int iv = vel_idx(axis);
    const double mass_flux = w[0] * w[iv];
    double e_kin = 0.0;
    f[0] = mass_flux;
    f[1] = mass_flux * w[1];
    e_kin += sq(w[1]);
    if (ndim > 1) {
        f[2] = mass_flux * w[2];
        e_kin += sq(w[2]);
    }
    if (ndim > 2) {
        f[3] = mass_flux * w[3];
        e_kin += sq(w[3]);
    }
    e_kin *= 0.5 * w[0];
    f[iv] += w[1 + ndim];
    const double e_tot = w[1 + ndim] / (gamma - 1.0) + e_kin;
    f[1 + ndim] = (e_tot + w[1 + ndim]) * w[iv];
}

/* ---- Reconstruct.hpp ----------------------------------------------------- */

/* slope_limiter, source/Reconstruct.hpp:130-148 */
static inline double slope_limiter(int sl, double um, double up) {
    if (sl == VANLEER) {
        return (um * up > 0.0) ? 2.0 * um * up / (um + up) : 0.0;
    } else if (sl == MONOTONIZED_CENTRAL) {
        return (copysign(1.0, um) + copysign(1.0, up)) *
               smin(fabs(um), smin(0.25 * fabs(um + up), fabs(up)));
    } else if (sl == MINMOD) {
        return 0.5 * (copysign(1.0, um) + copysign(1.0, up)) * smin(fabs(um), fabs(up));
    }
    return 0.0;
}

/* reconstruct<>, source/Reconstruct.hpp:150-274. s points at the centre of a
 * stencil laid out with unit stride (s[-2] .. s[2]). */
static inline void reconstruct(int recon, int sl, const double* s, double* wL, double* wR) {
    if (recon == FOG) {
        *wL = s[0];
        *wR = s[0];
    } else if (recon == MUSCL) {
        const double dwL = s[0] - s[-1];
        const double dwR = s[1] - s[0];
        const double delta = slope_limiter(sl, dwL, dwR);
        *wL = s[0] - 0.5 * delta;
        *wR = s[0] + 0.5 * delta;
    } else if (recon == PPM) {
        const double dw_m = slope_limiter(sl, s[-1] - s[-2], s[0] - s[-1]);
        const double dw_0 = slope_limiter(sl, s[0] - s[-1], s[1] - s[0]);
        const double dw_p = slope_limiter(sl, s[1] - s[0], s[2] - s[1]);
        double l = 0.5 * (s[-1] + s[0]) - (1.0 / 6.0) * (dw_0 - dw_m);
        double r = 0.5 * (s[0] + s[1]) - (1.0 / 6.0) * (dw_p - dw_0);
        if ((r - s[0]) * (s[0] - l) <= 0.0) {
            l = s[0];
            r = s[0];
        }
        if (fabs(r - s[0]) >= 2.0 * fabs(l - s[0])) {
            r = 3.0 * s[0] - 2.0 * l;
        }
        if (fabs(l - s[0]) >= 2.0 * fabs(r - s[0])) {
            l = 3.0 * s[0] - 2.0 * r;
        }
        *wL = l;
        *wR = r;
    } else {
        const double c0 = 13.0 / 12.0, c1 = 0.25;
        const double beta0 = c0 * sq(s[-2] - 2.0 * s[-1] + s[0]) + c1 * sq(s[-2] - 4.0 * s[-1] + 3.0 * s[0]);
        const double beta1 = c0 * sq(s[-1] - 2.0 * s[0] + s[1]) + c1 * sq(s[-1] - s[1]);
        const double beta2 = c0 * sq(s[0] - 2.0 * s[1] + s[2]) + c1 * sq(3.0 * s[0] - 4.0 * s[1] + s[2]);
        const double eps = 1e-36;
        const double tau5 = fabs(beta0 - beta2);
        const double ind0 = tau5 / (beta0 + eps);
        const double ind1 = tau5 / (beta1 + eps);
        const double ind2 = tau5 / (beta2 + eps);
        double e0 = (2.0 * s[0] + 5.0 * s[-1] - s[-2]);
        double e1 = (-s[1] + 5.0 * s[0] + 2.0 * s[-1]);
        double e2 = (2.0 * s[2] - 7.0 * s[1] + 11.0 * s[0]);
        double a0 = 3.0 * (1.0 + sq(ind0));
        double a1 = 6.0 * (1.0 + sq(ind1));
        double a2 = 1.0 * (1.0 + sq(ind2));
        double den = 6.0 * (a0 + a1 + a2);
        *wL = (e0 * a0 + e1 * a1 + e2 * a2) / den;
        e0 = (2.0 * s[0] + 5.0 * s[1] - s[2]);
        e1 = (-s[-1] + 5.0 * s[0] + 2.0 * s[1]);
        e2 = (2.0 * s[-2] - 7.0 * s[-1] + 11.0 * s[0]);
        a0 = 3.0 * (1.0 + sq(ind2));
        a1 = 6.0 * (1.0 + sq(ind1));
        a2 = 1.0 * (1.0 + sq(ind0));
        den = 6.0 * (a0 + a1 + a2);
        *wR = (e0 * a0 + e1 * a1 + e2 * a2) / den;
    }
}

/* ---- Riemann.hpp --------------------------------------------------------- */

/* riemann_flux<>, source/Riemann.hpp:22-176. Hydro variables only. */
static void riemann(int rs, int axis, int ndim, double gamma, const double* wL, const double* wR,
                    double* flux) {
    const int nh = 2 + ndim;
    const int iv = vel_idx(axis);
    const int ie = 1 + ndim;
    const double tiny = 1e-20;
    double qL[5], qR[5], fL[5], fR[5];
    if (rs == RUSANOV) {
        const double vL = wL[iv], vR = wR[iv];
        prim_to_cons(ndim, gamma, wL, qL);
        prim_to_cons(ndim, gamma, wR, qR);
        prim_to_flux(axis, ndim, gamma, wL, fL);
        prim_to_flux(axis, ndim, gamma, wR, fR);
        const double csL = sound_speed(ndim, gamma, wL);
        const double csR = sound_speed(ndim, gamma, wR);
        const double max_c = 0.5 * (csL + fabs(vL) + csR + fabs(vR));
        for (int i = 0; i < nh; ++i) {
            flux[i] = 0.5 * (fL[i] + fR[i] - max_c * (qR[i] - qL[i]));
        }
    } else if (rs == HLL) {
        const double csL = sound_speed(ndim, gamma, wL);
        const double csR = sound_speed(ndim, gamma, wR);
        /* The right speed uses wL's velocity with csR, as the reference does. */
        const double sL = smin(-tiny, smin(wL[iv] - csL, wR[iv] - csR));
        const double sR = smax(-tiny, smax(wL[iv] + csL, wL[iv] + csR));
        const double sM = 1.0 / (sR - sL);
        prim_to_cons(ndim, gamma, wL, qL);
        prim_to_cons(ndim, gamma, wR, qR);
        prim_to_flux(axis, ndim, gamma, wL, fL);
        prim_to_flux(axis, ndim, gamma, wR, fR);
        for (int i = 0; i < nh; ++i) {
            flux[i] = sM * (sR * fL[i] - sL * fR[i] + sR * sL * (qR[i] - qL[i]));
        }
    } else {
        const double csL = sound_speed(ndim, gamma, wL);
        const double csR = sound_speed(ndim, gamma, wR);
        prim_to_cons(ndim, gamma, wL, qL);
        prim_to_cons(ndim, gamma, wR, qR);
        const double pL = wL[ie], pR = wR[ie];
        const double rho_avg = 0.5 * (wL[0] + wR[0]);
        const double cs_avg = 0.5 * (csL + csR);
        const double p_mid = 0.5 * (pL + pR + (wL[iv] - wR[iv]) * rho_avg * cs_avg);
        const double cLstar = (p_mid <= wL[ie])
                                  ? 1.0
                                  : sqrt(1.0 + (gamma + 1.0) / (2.0 * gamma) * (p_mid / wL[ie] - 1.0));
        const double cRstar = (p_mid <= wR[ie])
                                  ? 1.0
                                  : sqrt(1.0 + (gamma + 1.0) / (2.0 * gamma) * (p_mid / wR[ie] - 1.0));
        const double aL = wL[iv] - csL * cLstar;
        const double aR = wR[iv] + csR * cRstar;
        const double bM = smin(-tiny, aL);
        const double bP = smax(tiny, aR);
        double vxL = wL[iv] - aL;
        double vxR = wR[iv] - aR;
        const double tL = wL[ie] + vxL * qL[iv];
        const double tR = wR[ie] + vxR * qR[iv];
        const double mL = wL[0] * vxL;
        const double mR = -(wR[0] * vxR);
        const double aM = (tL - tR) / (mL + mR);
        const double cp = smax((mL * tR + mR * tL) / (mL + mR), 0.0);
        vxL = wL[iv] - bM;
        vxR = wR[iv] - bP;
        const double mfL = wL[0] * vxL;
        const double mfR = wR[0] * vxR;
        fL[0] = mfL;
        fR[0] = mfR;
        fL[1] = mfL * wL[1];
        fR[1] = mfR * wR[1];
        if (ndim > 1) {
            fL[2] = mfL * wL[2];
            fR[2] = mfR * wR[2];
        }
        if (ndim > 2) {
            fL[3] = mfL * wL[3];
            fR[3] = mfR * wR[3];
        }
        fL[iv] += wL[ie];
        fR[iv] += wR[ie];
        fL[ie] = qL[ie] * vxL + wL[ie] * wL[iv];
        fR[ie] = qR[ie] * vxR + wR[ie] * wR[iv];
        double sL, sR, sM;
        if (aM >= 0.0) {
            sL = aM / (aM - bM);
            sR = 0.0;
            sM = -bM / (aM - bM);
        } else {
            sL = 0.0;
            sR = -aM / (bP - aM);
            sM = bP / (bP - aM);
        }
        for (int v = 0; v < nh; ++v) {
            flux[v] = sL * fL[v] + sR * fR[v];
        }
        flux[iv] += sM * cp;
        flux[ie] += sM * cp * aM;
    }
}

/* ---- Hydro.cpp ------------------------------------------------------------ */

/* Interior loop bounds shared by recon / flux / integrate (Hydro.cpp:62-78,
 * :111-129, TimeStepping.cpp:11-20). */
typedef struct {
    int n[3];
    int s[3];
} range3;

static range3 interior_range(const osim* s) {
    range3 r;
    r.n[0] = s->xc - 2 * s->ng;
    r.n[1] = s->yc - 2 * s->ng > 1 ? s->yc - 2 * s->ng : 1;
    r.n[2] = s->zc - 2 * s->ng > 1 ? s->zc - 2 * s->ng : 1;
    r.s[0] = s->ng;
    r.s[1] = r.n[1] == 1 ? 0 : s->ng;
    r.s[2] = r.n[2] == 1 ? 0 : s->ng;
    return r;
}

/* global_cons_to_prim_impl, source/Hydro.cpp:8-53 (every cell, ghosts included) */
static void global_cons_to_prim(osim* s) {
    const long long plane = (long long)s->zc * s->yc * s->xc;
    const double gamma = s->c.gamma;
#pragma omp parallel for schedule(static)
    for (long long c = 0; c < plane; ++c) {
        double q[MAXV], w[MAXV];
        for (int v = 0; v < s->nhydro; ++v) {
            q[v] = s->Q[v * plane + c];
        }
        cons_to_prim(s->ndim, gamma, q, w);
        for (int v = 0; v < s->nhydro; ++v) {
            s->W[v * plane + c] = w[v];
        }
        const double inv_rho = 1.0 / q[0];
        for (int v = s->nhydro; v < s->nvar; ++v) {
            s->W[v * plane + c] = s->Q[v * plane + c] * inv_rho;
        }
    }
}

/* compute_recon_impl, source/Hydro.cpp:55-102 */
static void compute_recon(osim* s, int axis) {
    range3 r = interior_range(s);
    r.n[axis] += 2;
    r.s[axis] -= 1;
    const long long stride = axis == 0 ? 1 : axis == 1 ? s->xc : (long long)s->xc * s->yc;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = r.s[2]; k < r.s[2] + r.n[2]; ++k) {
        for (int j = r.s[1]; j < r.s[1] + r.n[1]; ++j) {
            for (int i = r.s[0]; i < r.s[0] + r.n[0]; ++i) {
                for (int v = 0; v < s->nvar; ++v) {
                    const long long id = at(s, v, k, j, i);
                    double st[5];
                    const int order = (s->c.reconstruction == PPM || s->c.reconstruction == WENO5Z) ? 2
                                      : s->c.reconstruction == MUSCL                                 ? 1
                                                                                                     : 0;
                    for (int o = -order; o <= order; ++o) {
                        st[2 + o] = s->W[id + o * stride];
                    }
                    double wl, wr;
                    reconstruct(s->c.reconstruction, s->c.slope_limiter, st + 2, &wl, &wr);
                    s->RL[id] = wl;
                    s->RR[id] = wr;
                }
            }
        }
    }
}

/* compute_flux_impl, source/Hydro.cpp:104-166 */
static void compute_flux(osim* s, int axis) {
    range3 r = interior_range(s);
    r.n[axis] += 1;
    const long long stride = axis == 0 ? 1 : axis == 1 ? s->xc : (long long)s->xc * s->yc;
    double* F = s->F[axis];
    const long long plane = (long long)s->zc * s->yc * s->xc;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = r.s[2]; k < r.s[2] + r.n[2]; ++k) {
        for (int j = r.s[1]; j < r.s[1] + r.n[1]; ++j) {
            for (int i = r.s[0]; i < r.s[0] + r.n[0]; ++i) {
                const long long id = at(s, 0, k, j, i);
                const long long idm = id - stride;
                double wl[MAXV], wr[MAXV], fl[MAXV];
                for (int v = 0; v < s->nhydro; ++v) {
                    wl[v] = s->RR[idm + v * plane];
                    wr[v] = s->RL[id + v * plane];
                }
                riemann(s->c.riemann_solver, axis, s->ndim, s->c.gamma, wl, wr, fl);
                for (int v = 0; v < s->nhydro; ++v) {
                    F[id + v * plane] = fl[v];
                }
                for (int v = s->nhydro; v < s->nvar; ++v) {
                    if (F[id] >= 0.0) {
                        F[id + v * plane] = F[id] * s->RR[idm + v * plane];
                    } else {
                        F[id + v * plane] = F[id] * s->RL[id + v * plane];
                    }
                }
            }
        }
    }
}

/* ---- Non-ideal EOS updates (Simulation::update_eos) ----------------------- */

static const double H_MASS = 1.6737830080950003e-27; /* [kg] */
static const double K_B = 1.380649e-23;              /* [J / K] */
static const double CHI_H = 2.178710282685096e-18;    /* [J] */

/* Conditions on which the reference aborts (moracle_abort_count). */
static long long g_port_aborts = 0;

/* saha_rhs_H, source/AnalyticLteH.hpp:10-14 */
static double saha_rhs_H(double temp) {
    return 2.4146830395719654e+21 * pow(temp, 1.5) * exp(-157763.42386247337 / temp);
}

/* y_from_nhtot, source/AnalyticLteH.hpp:16-20 */
static double y_from_nhtot(double nhtot, double temp) {
    const double X = saha_rhs_H(temp);
    return 0.5 * (-X + sqrt(sq(X) + 4 * nhtot * X)) / nhtot;
}

/* Kinetic energy and internal energy of cell id (both EOS updates). */
static void cell_energies(const osim* s, long long id, long long plane, double* rho, double* e_kin, double* eint) {
    double mom2_sum = sq(s->Q[id + plane]);
    if (s->ndim > 1) {
        mom2_sum += sq(s->Q[id + 2 * plane]);
    }
    if (s->ndim > 2) {
        mom2_sum += sq(s->Q[id + 3 * plane]);
    }
    *rho = s->Q[id];
    *e_kin = 0.5 * mom2_sum / *rho;
    *eint = s->Q[id + (1 + s->ndim) * plane] - *e_kin;
}

/* AnalyticLteH::update_eos, source/AnalyticLteH.hpp:49-120: temperature and
 * ionisation fraction by bisection, every cell including ghosts. */
static void eos_analytic(osim* s) {
    const long long plane = (long long)s->zc * s->yc * s->xc;
    const double gamma = s->c.gamma;
    const int ionisation_e = s->eos_ion;
    const double inv_avg_mass = 1.0 / s->avg_mass;
    long long aborts = 0;
#pragma omp parallel for schedule(static) reduction(+ : aborts)
    for (long long id = 0; id < plane; ++id) {
        double rho, e_kin, eint;
        cell_energies(s, id, plane, &rho, &e_kin, &eint);
        const double e_to_T = (gamma - 1.0) / (rho * (K_B / H_MASS) * inv_avg_mass);
#define TEMP_FROM_Y(yy) (e_to_T / (1.0 + (yy)) * (eint - ionisation_e * (yy) * rho * (CHI_H / H_MASS) * inv_avg_mass))
        const double rho_to_nhtot = (1.0 / H_MASS) * inv_avg_mass;
        const double min_temperature = 100.0;
        const double t1 = TEMP_FROM_Y(1.0);
        const double tb0 = smax(t1, min_temperature);
        const double tb1 = TEMP_FROM_Y(0.0);
        if (tb0 > tb1) {
            aborts += 1;
        }
        double temp_step = tb1 - tb0;
        double temp = tb0;
        double y = 0.0, test_temp, temp_err;
        for (int iter = 0; iter < 100; ++iter) {
            temp_step *= 0.5;
            test_temp = temp + temp_step;
            y = y_from_nhtot(rho * rho_to_nhtot, test_temp);
            temp_err = test_temp - TEMP_FROM_Y(y);
            if (temp_err <= 0.0) {
                temp = test_temp;
            }
            const double temp_err_bound = 1e-1;
            if (fabs(temp_step) < temp_err_bound || fabs(temp_err) < temp_err_bound) {
                break;
            }
        }
#undef TEMP_FROM_Y
        s->y_space[id] = y;
        s->T_space[id] = temp;
    }
    g_port_aborts += aborts;
}

/* TabulatedLteH::sample, source/TabulatedLteH.hpp:60-117 */
static void tab_sample(const osim* s, double log_eint_rho, double log_rho, double* out_y, double* out_log_T) {
    const moracle_eos_table* t = &s->tab;
    const double frac_eint_rho = (log_eint_rho - t->log_eint_rho_start) / t->log_eint_rho_step;
    int ix = (int)floor(frac_eint_rho);
    int ixp;
    double tx, txp;
    const int max_x = t->n_eint_rho - 1;
    const int max_y = t->n_rho - 1;
    if (frac_eint_rho < 0.0 || frac_eint_rho >= max_x) {
        ix = ix < 0 ? 0 : ix;
        ix = max_x < ix ? max_x : ix;
        ixp = ix;
        tx = 1.0;
        txp = 0.0;
    } else {
        ixp = ix + 1;
        txp = frac_eint_rho - ix;
        tx = 1.0 - txp;
    }
    const double frac_rho = (log_rho - t->log_rho_start) / t->log_rho_step;
    int iy = (int)floor(frac_rho);
    int iyp;
    double ty, typ;
    if (frac_rho < 0.0 || frac_rho >= max_y) {
        iy = iy < 0 ? 0 : iy;
        iy = max_y < iy ? max_y : iy;
        iyp = iy;
        ty = 1.0;
        typ = 0.0;
    } else {
        iyp = iy + 1;
        typ = frac_rho - iy;
        ty = 1.0 - typ;
    }
    const int nx = t->n_eint_rho;
    const double* Y = s->ytab;
    const double* L = s->lTtab;
    *out_y = (ty * (tx * Y[iy * nx + ix] + txp * Y[iy * nx + ixp]) +
              typ * (tx * Y[iyp * nx + ix] + txp * Y[iyp * nx + ixp]));
    *out_log_T = (ty * (tx * L[iy * nx + ix] + txp * L[iy * nx + ixp]) +
                  typ * (tx * L[iyp * nx + ix] + txp * L[iyp * nx + ixp]));
}

/* TabulatedLteH::update_eos, source/TabulatedLteH.hpp:119-163: y and T from
 * the table, and the internal energy shifted by the ionisation energy of the
 * change of y since the previous call, every cell including ghosts. */
static void eos_tabulated(osim* s) {
    const long long plane = (long long)s->zc * s->yc * s->xc;
    long long aborts = 0;
#pragma omp parallel for schedule(static) reduction(+ : aborts)
    for (long long id = 0; id < plane; ++id) {
        double rho, e_kin, eint;
        cell_energies(s, id, plane, &rho, &e_kin, &eint);
        const double log_rho = log10(rho);
        const double log_eint_rho = log10(eint) - log_rho;
        if (eint < 0.0 || log_eint_rho != log_eint_rho || log_rho != log_rho) {
            /* the reference aborts here (TabulatedLteH.hpp:142-144); the
             * restatement counts it and leaves the cell, whose NaN table
             * coordinates would index out of range */
            aborts += 1;
            continue;
        }
        double sy, slT;
        tab_sample(s, log_eint_rho, log_rho, &sy, &slT);
        const double prev_y = s->y_space[id];
        s->y_space[id] = sy;
        const double delta_eint = (prev_y < 0.0) ? 0.0 : rho * (CHI_H / H_MASS) * (sy - prev_y);
        s->T_space[id] = pow(10.0, slT);
        s->Q[id + (1 + s->ndim) * plane] += delta_eint;
    }
    g_port_aborts += aborts;
}

static void update_eos(osim* s) {
    if (s->eos_type == 1) {
        eos_analytic(s);
    } else if (s->eos_type == 2) {
        eos_tabulated(s);
    }
}

/* compute_hydro_fluxes, source/Hydro.cpp:325-343 (update_eos first) */
static void compute_hydro_fluxes(osim* s) {
    update_eos(s);
    global_cons_to_prim(s);
    for (int a = 0; a < s->ndim; ++a) {
        compute_recon(s, a);
        compute_flux(s, a);
    }
}

/* dt_reducer + compute_dt_impl, source/Hydro.cpp:192-242 (min over every cell) */
static double cfl_min(const osim* s) {
    const long long plane = (long long)s->zc * s->yc * s->xc;
    double result = DBL_MAX;
#pragma omp parallel
    {
        double local = DBL_MAX;
#pragma omp for schedule(static) nowait
        for (long long c = 0; c < plane; ++c) {
            double q[5], w[5];
            for (int v = 0; v < s->nhydro; ++v) {
                q[v] = s->Q[v * plane + c];
            }
            cons_to_prim(s->ndim, s->c.gamma, q, w);
            const double cs = sound_speed(s->ndim, s->c.gamma, w);
            double vel2 = sq(w[1]);
            if (s->ndim > 1) {
                vel2 += sq(w[2]);
            }
            if (s->ndim > 2) {
                vel2 += sq(w[3]);
            }
            const double vel = sqrt(vel2);
            const double dt_local = s->c.dx / (cs + vel);
            local = smin(dt_local, local);
        }
#pragma omp critical
        result = (local < result) ? local : result;
    }
    return result;
}

static double compute_dt(const osim* s) {
    double dt = cfl_min(s) * s->c.max_cfl;
    const double next_write = smin(s->c.max_time, s->prev_output_time + s->c.output_delta);
    if (s->time + dt >= next_write) {
        dt = next_write - s->time;
        while (s->time + dt < next_write) {
            dt = nextafter(dt, DBL_MAX);
        }
    }
    return dt;
}

/* ---- Boundaries.hpp ------------------------------------------------------- */

/* fill_one_bc_impl, source/Boundaries.hpp:11-119 */
static void fill_one_bc(osim* s, int axis) {
    const int ng = s->ng;
    const int dims[3] = {s->xc, s->yc, s->zc};
    int ld[3] = {s->xc, s->yc, s->zc};
    ld[axis] = 2 * ng;
    const int im = vel_idx(axis);
    const int ie = 1 + s->ndim;
    const int* bcs = s->c.bc;
#pragma omp parallel for collapse(2) schedule(static)
    for (int kk = 0; kk < ld[2]; ++kk) {
        for (int jj = 0; jj < ld[1]; ++jj) {
            for (int ii = 0; ii < ld[0]; ++ii) {
                int coord[3] = {ii, jj, kk};
                const int pencil = coord[axis];
                int cflip = (2 * ng - 1) - coord[axis];
                int cedge = ng;
                if (pencil >= ng) {
                    coord[axis] = (dims[axis] - 1) - (pencil - ng);
                    cflip = (dims[axis] - 1) - (2 * ng - 1) + (pencil - ng);
                    cedge = (dims[axis] - 1) - ng;
                }
                int flip[3] = {coord[0], coord[1], coord[2]};
                flip[axis] = cflip;
                int per[3] = {coord[0], coord[1], coord[2]};
                per[axis] += (pencil < ng ? 1 : -1) * (dims[axis] - 2 * ng);
                int edge[3] = {coord[0], coord[1], coord[2]};
                edge[axis] = cedge;
                const int start = coord[axis] < ng;
                const int bound = start ? bcs[2 * axis] : bcs[2 * axis + 1];
                const double* cv = start ? s->c.bc_const[2 * axis] : s->c.bc_const[2 * axis + 1];
#define QAT(v, c3) s->Q[at(s, (v), (c3)[2], (c3)[1], (c3)[0])]
                if (bound == BC_WALL) {
                    for (int v = 0; v < s->nvar; ++v) {
                        QAT(v, coord) = QAT(v, flip);
                    }
                    QAT(im, coord) = -QAT(im, coord);
                } else if (bound == BC_PERIODIC) {
                    for (int v = 0; v < s->nvar; ++v) {
                        QAT(v, coord) = QAT(v, per);
                    }
                } else if (bound == BC_SYMMETRIC) {
                    for (int v = 0; v < s->nvar; ++v) {
                        QAT(v, coord) = QAT(v, flip);
                    }
                } else if (bound == BC_DIODE) {
                    for (int v = 0; v < s->nvar; ++v) {
                        QAT(v, coord) = QAT(v, flip);
                    }
                    const double mom_pre = QAT(im, coord);
                    if (start) {
                        QAT(im, coord) = smin(mom_pre, 0.0);
                    } else {
                        QAT(im, coord) = smax(mom_pre, 0.0);
                    }
                    QAT(ie, coord) -= sq(QAT(im, coord) - mom_pre) / QAT(0, coord);
                } else if (bound == BC_ZEROGRAD) {
                    for (int v = 0; v < s->nvar; ++v) {
                        QAT(v, coord) = QAT(v, edge);
                    }
                } else if (bound == BC_CONSTANT) {
                    for (int v = 0; v < s->nvar; ++v) {
                        QAT(v, coord) = cv[v];
                    }
                }
#undef QAT
            }
        }
    }
}

/* fill_bcs, source/Boundaries.hpp:121-149 */
static void fill_bcs(osim* s) {
    for (int a = 0; a < s->ndim; ++a) {
        fill_one_bc(s, a);
    }
}

/* ---- TimeStepping.cpp ------------------------------------------------------ */

/* zero_source_terms + compute_source_terms (source/SourceTerms.hpp:8-16)
 * for one cell: S = 0, then the gravity source term if registered
 * (source/SourceTerms/Gravity.cpp:16-41): S(mom_a) += rho g_a,
 * S(E) += m_x g_x (+ m_y g_y (+ m_z g_z)). Computed from the stage input
 * before the cell is updated, as the reference's separate kernel is. */
static void cell_sources(const osim* s, int k, int j, int i, double* S) {
    for (int v = 0; v < s->nhydro; ++v) {
        S[v] = 0.0;
    }
    if (!s->gravity) {
        return;
    }
    const double rho = s->Q[at(s, 0, k, j, i)];
    S[1] += rho * s->grav[0];
    double energy_update = s->Q[at(s, 1, k, j, i)] * s->grav[0];
    if (s->ndim > 1) {
        S[2] += rho * s->grav[1];
        energy_update += s->Q[at(s, 2, k, j, i)] * s->grav[1];
    }
    if (s->ndim > 2) {
        S[3] += rho * s->grav[2];
        energy_update += s->Q[at(s, 3, k, j, i)] * s->grav[2];
    }
    S[1 + s->ndim] += energy_update;
}

/* integrate_flux + the stage updates, source/TimeStepping.cpp:10-35 and the
 * stage lambdas of rk2 (:60-67, :80-87), ssprk3 (:137-144, :157-164,
 * :177-184) and ssprk4 (:234-241, :254-261, :274-281, :294-301); the source
 * of hydro variable v is S(v) * dt. */
static void integrate(osim* s, int stepper, int stage, double dt) {
    const range3 r = interior_range(s);
    const int nz = r.n[2], ny = r.n[1], nx = r.n[0];
    const int ng = s->ng;
#pragma omp parallel for collapse(2) schedule(static)
    for (int ki = 0; ki < nz; ++ki) {
        for (int ji = 0; ji < ny; ++ji) {
            for (int ii = 0; ii < nx; ++ii) {
                const int k = nz == 1 ? ki : ki + ng;
                const int j = ny == 1 ? ji : ji + ng;
                const int i = ii + ng;
                double S[5];
                cell_sources(s, k, j, i, S);
                for (int v = 0; v < s->nvar; ++v) {
                    const long long id = at(s, v, k, j, i);
                    double qu = 0.0;
                    qu += s->F[0][id] - s->F[0][id + 1];
                    if (s->ndim > 1) {
                        qu += s->F[1][id] - s->F[1][id + s->xc];
                    }
                    if (s->ndim > 2) {
                        qu += s->F[2][id] - s->F[2][id + (long long)s->xc * s->yc];
                    }
                    qu *= dt / s->c.dx;
                    double source = 0.0;
                    if (v < s->nhydro) {
                        source = S[v] * dt;
                    }
                    double* Q = s->Q;
                    const double* Qo = s->Qold;
                    if (stepper == RK2) {
                        if (stage == 0) {
                            Q[id] += qu + source;
                        } else {
                            Q[id] = 0.5 * (Qo[id] + Q[id] + qu + source);
                        }
                    } else if (stepper == SSPRK3) {
                        if (stage == 0) {
                            Q[id] += qu + source;
                        } else if (stage == 1) {
                            Q[id] = 0.75 * Qo[id] + 0.25 * (Q[id] + qu + source);
                        } else {
                            Q[id] = (1.0 / 3.0) * Qo[id] + (2.0 / 3.0) * (Q[id] + qu + source);
                        }
                    } else {
                        if (stage == 2) {
                            Q[id] = (2.0 / 3.0) * Qo[id] + (1.0 / 3.0) * Q[id] + (1.0 / 6.0) * (qu + source);
                        } else {
                            Q[id] += 0.5 * (qu + source);
                        }
                    }
                }
            }
        }
    }
}

/* TimeStepper<>::time_step, source/TimeStepping.cpp:39-308 */
static void time_step(osim* s, double dt) {
    const int stepper = s->c.time_stepper;
    const int n_stages = stepper == RK2 ? 2 : stepper == SSPRK3 ? 3 : 4;
    const long long n = (long long)s->nvar * s->zc * s->yc * s->xc;
    memcpy(s->Qold, s->Q, sizeof(double) * n);
    for (int stage = 0; stage < n_stages; ++stage) {
        if (stage > 0) {
            fill_bcs(s);
        }
        compute_hydro_fluxes(s);
        integrate(s, stepper, stage, dt);
    }
    fill_bcs(s);
    s->time += dt;
    s->step += 1;
}

/* ---- C interface (moracle.h) ------------------------------------------------ */

void* moracle_create(const moracle_config* c) {
    if (c->num_dim < 1 || c->num_dim > 3) {
        return NULL;
    }
    const int min_ghost = c->reconstruction == FOG ? 1 : c->reconstruction == MUSCL ? 2 : 3;
    if (c->ng < min_ghost || 2 + c->num_dim + c->num_tracers > MAXV) {
        return NULL;
    }
    osim* s = (osim*)calloc(1, sizeof(osim));
    if (!s) {
        return NULL;
    }
    s->c = *c;
    s->ndim = c->num_dim;
    s->nhydro = 2 + c->num_dim;
    s->nvar = s->nhydro + c->num_tracers;
    s->ng = c->ng;
    s->xc = c->nx + 2 * c->ng;
    s->yc = c->num_dim > 1 ? c->ny + 2 * c->ng : 1;
    s->zc = c->num_dim > 2 ? c->nz + 2 * c->ng : 1;
    const long long n = (long long)s->nvar * s->zc * s->yc * s->xc;
    double** arrays[] = {&s->Q, &s->W, &s->RL, &s->RR, &s->F[0], &s->F[1], &s->F[2], &s->Qold};
    for (unsigned a = 0; a < sizeof(arrays) / sizeof(arrays[0]); ++a) {
        *arrays[a] = (double*)calloc((size_t)n, sizeof(double));
        if (!*arrays[a]) {
            moracle_destroy(s);
            return NULL;
        }
    }
    s->time = 0.0;
    s->prev_output_time = 0.0;
    return s;
}

void moracle_destroy(void* p) {
    osim* s = (osim*)p;
    if (!s) {
        return;
    }
    free(s->Q);
    free(s->W);
    free(s->RL);
    free(s->RR);
    free(s->F[0]);
    free(s->F[1]);
    free(s->F[2]);
    free(s->Qold);
    free(s->y_space);
    free(s->T_space);
    free(s->ytab);
    free(s->lTtab);
    free(s);
}

int64_t moracle_state_size(void* p) {
    const osim* s = (const osim*)p;
    return (int64_t)s->nvar * s->zc * s->yc * s->xc;
}

void moracle_set_Q(void* p, const double* q) {
    osim* s = (osim*)p;
    memcpy(s->Q, q, sizeof(double) * (size_t)moracle_state_size(p));
}

void moracle_get_Q(void* p, double* q) {
    osim* s = (osim*)p;
    memcpy(q, s->Q, sizeof(double) * (size_t)moracle_state_size(p));
}

void moracle_get_W(void* p, double* w) {
    osim* s = (osim*)p;
    memcpy(w, s->W, sizeof(double) * (size_t)moracle_state_size(p));
}

void moracle_fill_bcs(void* p) { fill_bcs((osim*)p); }

double moracle_compute_dt(void* p) { return compute_dt((const osim*)p); }

double moracle_cfl_min(void* p) { return cfl_min((const osim*)p); }

void moracle_time_step(void* p, double dt) { time_step((osim*)p, dt); }

int64_t moracle_run(void* p, int64_t max_steps, double* dt_log) {
    osim* s = (osim*)p;
    int64_t n = 0;
    while (s->time < s->c.max_time && n < max_steps) {
        const double dt = compute_dt(s);
        time_step(s, dt);
        if (dt_log) {
            dt_log[n] = dt;
        }
        ++n;
        if (s->time >= s->prev_output_time + s->c.output_delta) {
            s->prev_output_time = s->time;
        }
    }
    return n;
}

double moracle_get_time(void* p) { return ((osim*)p)->time; }

void moracle_set_clock(void* p, double time, double prev_output_time) {
    ((osim*)p)->time = time;
    ((osim*)p)->prev_output_time = prev_output_time;
}

void moracle_set_gravity(void* p, int enabled, double gx, double gy, double gz) {
    osim* s = (osim*)p;
    s->gravity = enabled ? 1 : 0;
    s->grav[0] = gx;
    s->grav[1] = gy;
    s->grav[2] = gz;
}

int moracle_set_eos(void* p, int type, double avg_mass, int include_ionisation_energy,
                    const moracle_eos_table* t) {
    osim* s = (osim*)p;
    const long long plane = (long long)s->zc * s->yc * s->xc;
    s->avg_mass = avg_mass;
    s->eos_ion = include_ionisation_energy != 0;
    if (type == 0) {
        s->eos_type = 0;
        return 0;
    }
    if (type != 1 && !(type == 2 && t && t->y_table && t->log_T_table)) {
        return -1;
    }
    if (!s->y_space) {
        s->y_space = (double*)calloc((size_t)plane, sizeof(double));
        s->T_space = (double*)calloc((size_t)plane, sizeof(double));
    }
    for (long long id = 0; id < plane; ++id) {
        s->y_space[id] = 0.0;
        s->T_space[id] = 0.0;
    }
    s->eos_type = type;
    if (type == 2) {
        /* Eos::init_tabulated_lte_h sets y_space = -1 (source/Eos.cpp:75) */
        const size_t n = (size_t)t->n_rho * (size_t)t->n_eint_rho;
        free(s->ytab);
        free(s->lTtab);
        s->ytab = (double*)malloc(n * sizeof(double));
        s->lTtab = (double*)malloc(n * sizeof(double));
        memcpy(s->ytab, t->y_table, n * sizeof(double));
        memcpy(s->lTtab, t->log_T_table, n * sizeof(double));
        s->tab = *t;
        for (long long id = 0; id < plane; ++id) {
            s->y_space[id] = -1.0;
        }
    }
    return 0;
}

void moracle_update_eos(void* p) {
    update_eos((osim*)p);
}

void moracle_get_eos_fields(void* p, double* y, double* T) {
    osim* s = (osim*)p;
    const long long plane = (long long)s->zc * s->yc * s->xc;
    for (long long id = 0; id < plane; ++id) {
        y[id] = s->y_space ? s->y_space[id] : 0.0;
        T[id] = s->T_space ? s->T_space[id] : 0.0;
    }
}

long long moracle_abort_count(void) {
    return g_port_aborts;
}

void moracle_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) {
        omp_set_num_threads(n);
    }
#else
    (void)n;
#endif
}
