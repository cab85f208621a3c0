// Pointwise physics of the Euler step: ideal-gas EOS conversions, slope
// limiters, face reconstruction and the three approximate Riemann solvers.
//
// Everything is templated on the compute type T. With T = double and the
// translation unit compiled with -fmad=false, every expression is evaluated in
// the same order as the reference (no reassociation, no contraction, IEEE
// division and square root), which makes the results bit-identical to the
// reference's CPU build. Each function cites the reference code it restates.
//
// Variable order (source/State.hpp:10-26): primitive w = [rho, v_x(, v_y(, v_z)), p],
// conserved q = [rho, m_x(, m_y(, m_z)), E]. The velocity / momentum along
// axis a sits at index 1 + a; pressure / energy at index 1 + NDIM.
#pragma once

#include <cstdint>

namespace mc {

enum Recon : int { kFog = 0, kMuscl = 1, kPpm = 2, kWeno5z = 3 };
enum Limiter : int { kVanLeer = 0, kMonotonizedCentral = 1, kMinmod = 2 };
enum Solver : int { kRusanov = 0, kHll = 1, kHllc = 2 };

// std::min / std::max semantics: the first argument is returned on ties and
// whenever the comparison is false (NaN).
template <class T>
__device__ __forceinline__ T smin(T a, T b) {
    return (b < a) ? b : a;
}
template <class T>
__device__ __forceinline__ T smax(T a, T b) {
    return (a < b) ? b : a;
}
template <class T>
__device__ __forceinline__ T sq(T a) {
    return a * a;
}
// a * b + c. For T = double in the exact translation units (compiled without
// contraction) this is the product and then the sum, as written.
template <class T>
__device__ __forceinline__ T madd(T a, T b, T c) {
    return a * b + c;
}

// Half-width of the reconstruction stencil: cells c-S..c+S are read to
// reconstruct the faces of cell c (source/Reconstruct.hpp:95-123, :150-274).
template <int REC>
__host__ __device__ constexpr int stencil_half() {
    return REC == kFog ? 0 : (REC == kMuscl ? 1 : 2);
}
// Ghost cells a reconstruction needs (source/Reconstruct.hpp:47-61): the face
// between cells c-1 and c uses both cells' reconstructions.
template <int REC>
__host__ __device__ constexpr int halo_of() {
    return stencil_half<REC>() + 1;
}

template <class T>
struct Consts;
template <>
struct Consts<double> {
    // WENO-Z regulariser (source/Reconstruct.hpp:238-242, double build)
    static constexpr double weno_eps = 1e-36;
};
template <>
struct Consts<float> {
    // WENO-Z regulariser of the reference's single-precision build
    static constexpr float weno_eps = 1e-15f;
};

// ---- EOS (source/Eos.hpp) ---------------------------------------------------

// sound_speed: sqrt(gamma p / rho)                                 Eos.hpp:54-59
template <int NDIM, class T>
__device__ __forceinline__ T sound_speed(T gamma, const T* w) {
    return sqrt(gamma * w[1 + NDIM] / w[0]);
}

// cons_to_prim                                                     Eos.hpp:61-79
template <int NDIM, class T>
__device__ __forceinline__ void prim_from_cons(T gamma, const T* q, T* w) {
    w[0] = q[0];
    w[1] = q[1] / q[0];
    T v2 = sq(w[1]);
    if constexpr (NDIM > 1) {
        w[2] = q[2] / q[0];
        v2 += sq(w[2]);
    }
    if constexpr (NDIM > 2) {
        w[3] = q[3] / q[0];
        v2 += sq(w[3]);
    }
    const T e_kin = T(0.5) * q[0] * v2;
    w[1 + NDIM] = (gamma - T(1)) * (q[1 + NDIM] - e_kin);
}

// prim_to_cons                                                     Eos.hpp:81-99
template <int NDIM, class T>
__device__ __forceinline__ void cons_from_prim(T gamma, const T* w, T* q) {
    q[0] = w[0];
    q[1] = w[0] * w[1];
    T v2 = sq(w[1]);
    if constexpr (NDIM > 1) {
        q[2] = w[0] * w[2];
        v2 += sq(w[2]);
    }
    if constexpr (NDIM > 2) {
        q[3] = w[0] * w[3];
        v2 += sq(w[3]);
    }
    const T e_kin = T(0.5) * w[0] * v2;
    const T e_int = w[1 + NDIM] / (gamma - T(1));
    q[1 + NDIM] = e_int + e_kin;
}

// Component 1 + axis of a small register array, for an axis that is
// uniform across the warp: the array stays in registers because every
// access below uses a compile-time index.
template <int NDIM, class T>
__device__ __forceinline__ T along(const T* a, int axis) {
    T r = a[1];
    if constexpr (NDIM > 1) {
        if (axis == 1) {
            r = a[2];
        }
    }
    if constexpr (NDIM > 2) {
        if (axis == 2) {
            r = a[3];
        }
    }
    return r;
}

// a[1 + axis] += x
template <int NDIM, class T>
__device__ __forceinline__ void add_along(T* a, int axis, T x) {
    if (axis == 0) {
        a[1] += x;
    } else if (NDIM > 1 && axis == 1) {
        a[NDIM > 1 ? 2 : 1] += x;
    } else if (NDIM > 2) {
        a[NDIM > 2 ? 3 : 1] += x;
    }
}

// prim_to_flux along `axis` (warp-uniform)                         Eos.hpp:101-131
template <int NDIM, class T>
__device__ __forceinline__ void flux_from_prim(T gamma, int axis, const T* w, T* f) {
    const T vn = along<NDIM>(w, axis);
    const T mass_flux = w[0] * vn;
    T e_kin = T(0);
    f[0] = mass_flux;
    f[1] = mass_flux * w[1];
    e_kin += sq(w[1]);
    if constexpr (NDIM > 1) {
        f[2] = mass_flux * w[2];
        e_kin += sq(w[2]);
    }
    if constexpr (NDIM > 2) {
        f[3] = mass_flux * w[3];
        e_kin += sq(w[3]);
    }
    e_kin *= T(0.5) * w[0];
    add_along<NDIM>(f, axis, w[1 + NDIM]);
    const T e_tot = w[1 + NDIM] / (gamma - T(1)) + e_kin;
    f[1 + NDIM] = (e_tot + w[1 + NDIM]) * vn;
}

// CFL time-step bound of one cell from its primitives (dt_reducer,
// source/Hydro.cpp:192-206): dx / (c_s + |v|).
template <int NDIM, class T>
__device__ __forceinline__ T cfl_dt(T gamma, T dx, const T* w) {
    const T cs = sound_speed<NDIM>(gamma, w);
    T vel2 = sq(w[1]);
    if constexpr (NDIM > 1) {
        vel2 += sq(w[2]);
    }
    if constexpr (NDIM > 2) {
        vel2 += sq(w[3]);
    }
    const T vel = sqrt(vel2);
    return dx / (cs + vel);
}

// ---- Reconstruction (source/Reconstruct.hpp) ---------------------------------

// slope_limiter<>, um = w_i - w_{i-1}, up = w_{i+1} - w_i      Reconstruct.hpp:130-148
template <int LIM, class T>
__device__ __forceinline__ T limited_slope(T um, T up) {
    if constexpr (LIM == kVanLeer) {
        return (um * up > T(0)) ? T(2) * um * up / (um + up) : T(0);
    } else if constexpr (LIM == kMonotonizedCentral) {
        return (copysign(T(1), um) + copysign(T(1), up)) *
               smin(fabs(um), smin(T(0.25) * fabs(um + up), fabs(up)));
    } else {
        return T(0.5) * (copysign(T(1), um) + copysign(T(1), up)) * smin(fabs(um), fabs(up));
    }
}

// Left / right face values of the cell at the centre of s (s[2]); s[k]
// holds the cell at offset k - 2.                          Reconstruct.hpp:150-274
template <int REC, int LIM, class T>
__device__ __forceinline__ void reconstruct(const T* s, T& wl, T& wr) {
    const T c = s[2];
    if constexpr (REC == kFog) {
        wl = c;
        wr = c;
    } else if constexpr (REC == kMuscl) {
        const T delta = limited_slope<LIM>(c - s[1], s[3] - c);
        wl = c - T(0.5) * delta;
        wr = c + T(0.5) * delta;
    } else if constexpr (REC == kPpm) {
        // limited-slope cubic with the Colella-Sekora / McCorquodale-Colella
        // monotonicity fixes; the clamp of the reference is disabled (:169-215)
        const T dw_m = limited_slope<LIM>(s[1] - s[0], c - s[1]);
        const T dw_0 = limited_slope<LIM>(c - s[1], s[3] - c);
        const T dw_p = limited_slope<LIM>(s[3] - c, s[4] - s[3]);
        T l = T(0.5) * (s[1] + c) - (T(1) / T(6)) * (dw_0 - dw_m);
        T r = T(0.5) * (c + s[3]) - (T(1) / T(6)) * (dw_p - dw_0);
        if ((r - c) * (c - l) <= T(0)) {
            l = c;
            r = c;
        }
        if (fabs(r - c) >= T(2) * fabs(l - c)) {
            r = T(3) * c - T(2) * l;
        }
        if (fabs(l - c) >= T(2) * fabs(r - c)) {
            l = T(3) * c - T(2) * r;
        }
        wl = l;
        wr = r;
    } else {
        // WENO5-Z (Borges et al. 2008) with the Z+ style indicator tau5 /
        // (beta_k + eps) squared; candidate stencils pre-multiplied by 6 (:217-274).
        // The reference's expression trees; madd(a, b, c) is a * b + c and
        // only commutes an addition's operands where it appears, so the
        // exact FP64 results are unchanged. 13 / 12 is the same correctly
        // rounded constant as the reference's T(13) / T(12).
        const T b_a = T(13.0 / 12.0);
        const T b_b = T(0.25);
        const T beta0 = madd(b_a, sq(s[0] - T(2) * s[1] + c), b_b * sq(s[0] - T(4) * s[1] + T(3) * c));
        const T beta1 = madd(b_a, sq(s[1] - T(2) * c + s[3]), b_b * sq(s[1] - s[3]));
        const T beta2 = madd(b_a, sq(c - T(2) * s[3] + s[4]), b_b * sq(T(3) * c - T(4) * s[3] + s[4]));
        const T eps = Consts<T>::weno_eps;
        const T tau5 = fabs(beta0 - beta2);
        const T ind0 = tau5 / (beta0 + eps);
        const T ind1 = tau5 / (beta1 + eps);
        const T ind2 = tau5 / (beta2 + eps);
        {
            const T e0 = (madd(T(2), c, T(5) * s[1]) - s[0]);
            const T e1 = (madd(T(2), s[1], -s[3] + T(5) * c));
            const T e2 = (madd(T(11), c, T(2) * s[4] - T(7) * s[3]));
            const T a0 = T(3) * madd(ind0, ind0, T(1));
            const T a1 = T(6) * madd(ind1, ind1, T(1));
            const T a2 = madd(ind2, ind2, T(1));
            const T den = T(6) * (a0 + a1 + a2);
            wl = madd(e2, a2, madd(e1, a1, e0 * a0)) / den;
        }
        {
            const T e0 = (madd(T(2), c, T(5) * s[3]) - s[4]);
            const T e1 = (madd(T(2), s[3], -s[1] + T(5) * c));
            const T e2 = (madd(T(11), c, T(2) * s[0] - T(7) * s[1]));
            const T a0 = T(3) * madd(ind2, ind2, T(1));
            const T a1 = T(6) * madd(ind1, ind1, T(1));
            const T a2 = madd(ind0, ind0, T(1));
            const T den = T(6) * (a0 + a1 + a2);
            wr = madd(e2, a2, madd(e1, a1, e0 * a0)) / den;
        }
    }
}

// ---- Riemann solvers (source/Riemann.hpp), hydro variables only ---------------

// Interface flux along `axis` (warp-uniform). gfac = (gamma + 1) / (2 gamma),
// the HLLC shock-factor coefficient, computed once by the caller with that
// same expression (the reference evaluates it per interface; the value is
// identical).
template <int RS, int NDIM, class T>
__device__ __forceinline__ void riemann(T gamma, T gfac, int axis, const T* wL, const T* wR, T* flux) {
    constexpr int nh = 2 + NDIM;
    constexpr int ie = 1 + NDIM;
    const T tiny = T(1e-20);
    T qL[nh], qR[nh], fL[nh], fR[nh];
    const T vL = along<NDIM>(wL, axis);
    const T vR = along<NDIM>(wR, axis);
    if constexpr (RS == kRusanov) {
        // local Lax-Friedrichs with the mean of both signal speeds   Riemann.hpp:22-46
        cons_from_prim<NDIM>(gamma, wL, qL);
        cons_from_prim<NDIM>(gamma, wR, qR);
        flux_from_prim<NDIM>(gamma, axis, wL, fL);
        flux_from_prim<NDIM>(gamma, axis, wR, fR);
        const T csL = sound_speed<NDIM>(gamma, wL);
        const T csR = sound_speed<NDIM>(gamma, wR);
        const T max_c = T(0.5) * (csL + fabs(vL) + csR + fabs(vR));
#pragma unroll
        for (int i = 0; i < nh; ++i) {
            flux[i] = T(0.5) * (fL[i] + fR[i] - max_c * (qR[i] - qL[i]));
        }
    } else if constexpr (RS == kHll) {
        // HLL with the reference's wave-speed estimates; the right estimate
        // pairs wL's velocity with csR                               Riemann.hpp:48-73
        const T csL = sound_speed<NDIM>(gamma, wL);
        const T csR = sound_speed<NDIM>(gamma, wR);
        const T sL = smin(-tiny, smin(vL - csL, vR - csR));
        const T sR = smax(-tiny, smax(vL + csL, vL + csR));
        const T sM = T(1) / (sR - sL);
        cons_from_prim<NDIM>(gamma, wL, qL);
        cons_from_prim<NDIM>(gamma, wR, qR);
        flux_from_prim<NDIM>(gamma, axis, wL, fL);
        flux_from_prim<NDIM>(gamma, axis, wR, fR);
#pragma unroll
        for (int i = 0; i < nh; ++i) {
            flux[i] = sM * (sR * fL[i] - sL * fR[i] + sR * sL * (qR[i] - qL[i]));
        }
    } else {
        // HLLC in the Athena arrangement: PVRS pressure estimate, shock
        // factors on the outer speeds, contact speed aM and pressure cp
        //                                                           Riemann.hpp:75-176
        const T csL = sound_speed<NDIM>(gamma, wL);
        const T csR = sound_speed<NDIM>(gamma, wR);
        cons_from_prim<NDIM>(gamma, wL, qL);
        cons_from_prim<NDIM>(gamma, wR, qR);
        const T pL = wL[ie];
        const T pR = wR[ie];
        const T rho_avg = T(0.5) * (wL[0] + wR[0]);
        const T cs_avg = T(0.5) * (csL + csR);
        const T p_mid = T(0.5) * (pL + pR + (vL - vR) * rho_avg * cs_avg);
        // both shock factors are evaluated and then selected: the lanes of a
        // warp disagree on the branch in most faces, and a straight-line
        // sequence lets the two square roots overlap (values unchanged)
        const T sqL = sqrt(T(1) + gfac * (p_mid / pL - T(1)));
        const T sqR = sqrt(T(1) + gfac * (p_mid / pR - T(1)));
        const T cLstar = (p_mid <= pL) ? T(1) : sqL;
        const T cRstar = (p_mid <= pR) ? T(1) : sqR;
        const T aL = vL - csL * cLstar;
        const T aR = vR + csR * cRstar;
        const T bM = smin(-tiny, aL);
        const T bP = smax(tiny, aR);
        T vxL = vL - aL;
        T vxR = vR - aR;
        const T tL = pL + vxL * along<NDIM>(qL, axis);
        const T tR = pR + vxR * along<NDIM>(qR, axis);
        const T mL = wL[0] * vxL;
        const T mR = -(wR[0] * vxR);
        const T aM = (tL - tR) / (mL + mR);
        const T cp = smax((mL * tR + mR * tL) / (mL + mR), T(0));
        vxL = vL - bM;
        vxR = vR - bP;
        const T mfL = wL[0] * vxL;
        const T mfR = wR[0] * vxR;
        fL[0] = mfL;
        fR[0] = mfR;
#pragma unroll
        for (int d = 1; d <= NDIM; ++d) {
            fL[d] = mfL * wL[d];
            fR[d] = mfR * wR[d];
        }
        add_along<NDIM>(fL, axis, pL);
        add_along<NDIM>(fR, axis, pR);
        fL[ie] = qL[ie] * vxL + pL * vL;
        fR[ie] = qR[ie] * vxR + pR * vR;
        // aM >= 0: sL = aM / (aM - bM), sR = 0, sM = -bM / (aM - bM);
        // otherwise sL = 0, sR = -aM / (bP - aM), sM = bP / (bP - aM):
        // the same two quotients, with their operands selected first
        const bool left = aM >= T(0);
        const T den = left ? (aM - bM) : (bP - aM);
        const T s_out = (left ? aM : -aM) / den;
        const T sM = (left ? -bM : bP) / den;
        const T sL = left ? s_out : T(0);
        const T sR = left ? T(0) : s_out;
#pragma unroll
        for (int i = 0; i < nh; ++i) {
            flux[i] = sL * fL[i] + sR * fR[i];
        }
        add_along<NDIM>(flux, axis, sM * cp);
        flux[ie] += sM * cp * aM;
    }
}

} // namespace mc
