// Non-ideal equations of state: the update_eos step that the reference runs
// ahead of every stage's sweep (compute_hydro_fluxes, source/Hydro.cpp:326-
// 328) and once at set-up (source/SetupModules.hpp:253-255). One thread per
// cell, ghosts included, as the reference's FlatLoop over zc x yc x xc.
//
//  * analytic LTE hydrogen (source/AnalyticLteH.hpp:49-120): temperature and
//    ionisation fraction of every cell by bisection on the Saha equation;
//    the state is not changed.
//  * tabulated LTE hydrogen (source/TabulatedLteH.hpp:60-163): y and
//    log10 T by bilinear interpolation in (log10(eint / rho), log10 rho),
//    and the energy shifted by the ionisation energy of the change of y
//    since the previous call.
//
// Compiled without contraction and with the reference's expression trees;
// pow, exp and log10 are CUDA's, whose last bits can differ from the C
// library's, so results agree with the reference to rounding, not bit for
// bit. A condition on which the reference aborts (bisection bounds flipped,
// negative internal energy) raises MC_FLAG_EOS in the status instead; the
// tabulated kind leaves such a cell (and any cell whose table coordinates
// are not numbers) unchanged.
#include <cuda_runtime.h>

#include "common.cuh"
#include "eos.h"

namespace mc {
namespace {

constexpr double kHMass = 1.6737830080950003e-27;  // [kg]
constexpr double kKB = 1.380649e-23;               // [J / K]
constexpr double kChiH = 2.178710282685096e-18;    // [J]

__device__ __forceinline__ double saha_rhs_H(double temp) {
    return 2.4146830395719654e+21 * pow(temp, 1.5) * exp(-157763.42386247337 / temp);
}

__device__ __forceinline__ double y_from_nhtot(double nhtot, double temp) {
    const double X = saha_rhs_H(temp);
    return 0.5 * (-X + sqrt(X * X + 4 * nhtot * X)) / nhtot;
}

template <int NDIM>
__device__ __forceinline__ void energies(const double* q, long long id, long long plane, double& rho, double& e_kin,
                                         double& eint) {
    double mom2_sum = q[id + plane] * q[id + plane];
    if constexpr (NDIM > 1) {
        mom2_sum += q[id + 2 * plane] * q[id + 2 * plane];
    }
    if constexpr (NDIM > 2) {
        mom2_sum += q[id + 3 * plane] * q[id + 3 * plane];
    }
    rho = q[id];
    e_kin = 0.5 * mom2_sum / rho;
    eint = q[id + (1 + NDIM) * plane] - e_kin;
}

template <int NDIM>
__global__ void __launch_bounds__(256) eos_analytic_kernel(EosLaunch L) {
    if (L.blk && L.skip_when_done && L.blk->done) {
        return;
    }
    const double gamma = L.gamma;
    const double ionisation_e = L.ionisation_e ? 1.0 : 0.0;
    const double inv_avg_mass = 1.0 / L.avg_mass;
    unsigned flags = 0;
    for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < L.plane;
         id += (long long)gridDim.x * blockDim.x) {
        double rho, e_kin, eint;
        energies<NDIM>(L.q_in, id, L.plane, rho, e_kin, eint);
        const double e_to_T = (gamma - 1.0) / (rho * (kKB / kHMass) * inv_avg_mass);
        auto temp_from_y = [&](double y) {
            return e_to_T / (1.0 + y) * (eint - ionisation_e * y * rho * (kChiH / kHMass) * inv_avg_mass);
        };
        const double rho_to_nhtot = (1.0 / kHMass) * inv_avg_mass;
        const double min_temperature = 100.0;
        const double t1 = temp_from_y(1.0);
        const double tb0 = (t1 < min_temperature) ? min_temperature : t1;  // std::max
        const double tb1 = temp_from_y(0.0);
        if (tb0 > tb1) {
            flags |= kFlagEos;
        }
        double temp_step = tb1 - tb0;
        double temp = tb0;
        double y = 0.0;
        for (int iter = 0; iter < 100; ++iter) {
            temp_step *= 0.5;
            const double test_temp = temp + temp_step;
            y = y_from_nhtot(rho * rho_to_nhtot, test_temp);
            const double temp_err = test_temp - temp_from_y(y);
            if (temp_err <= 0.0) {
                temp = test_temp;
            }
            if (fabs(temp_step) < 1e-1 || fabs(temp_err) < 1e-1) {
                break;
            }
        }
        L.y[id] = y;
        L.T[id] = temp;
    }
    if (flags && L.blk) {
        atomicOr(&L.blk->status, flags);
    }
}

struct Sample {
    double y, log_T;
};

__device__ __forceinline__ Sample table_sample(const EosLaunch& L, const double* Y, const double* LT,
                                              double log_eint_rho, double log_rho) {
    const double frac_eint_rho = (log_eint_rho - L.x_start) / L.x_step;
    int ix = int(floor(frac_eint_rho));
    int ixp;
    double tx, txp;
    const int max_x = L.nx_tab - 1;
    const int max_y = L.ny_tab - 1;
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
    const double frac_rho = (log_rho - L.y_start) / L.y_step;
    int iy = int(floor(frac_rho));
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
    const int n = L.nx_tab;
    Sample s;
    s.y = (ty * (tx * Y[iy * n + ix] + txp * Y[iy * n + ixp]) + typ * (tx * Y[iyp * n + ix] + txp * Y[iyp * n + ixp]));
    s.log_T = (ty * (tx * LT[iy * n + ix] + txp * LT[iy * n + ixp]) +
               typ * (tx * LT[iyp * n + ix] + txp * LT[iyp * n + ixp]));
    return s;
}

// With tables_in_smem, a persistent grid whose CTAs first copy both tables
// into shared memory: each cell then gathers its eight table values from
// shared memory instead of waiting on global loads after its state loads.
template <int NDIM>
__global__ void __launch_bounds__(256) eos_tabulated_kernel(EosLaunch L, int tables_in_smem) {
    if (L.blk && L.skip_when_done && L.blk->done) {
        return;
    }
    extern __shared__ __align__(16) double tab_smem[];
    const double* Y = L.y_table;
    const double* LT = L.log_T_table;
    if (tables_in_smem) {
        const int n = L.nx_tab * L.ny_tab;
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            tab_smem[k] = L.y_table[k];
            tab_smem[n + k] = L.log_T_table[k];
        }
        __syncthreads();
        Y = tab_smem;
        LT = tab_smem + n;
    }
    constexpr int ie = 1 + NDIM;
    constexpr int nh = 2 + NDIM;
    constexpr int U = 4;  // cells per thread whose loads are issued together
    const long long stride = (long long)gridDim.x * blockDim.x;
    unsigned flags = 0;
    for (long long base = blockIdx.x * (long long)blockDim.x + threadIdx.x; base < L.plane; base += U * stride) {
        double qv[U][nh], yp[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const long long id = base + u * stride;
            if (id < L.plane) {
#pragma unroll
                for (int v = 0; v < nh; ++v) {
                    qv[u][v] = L.q_in[id + v * L.plane];
                }
                yp[u] = L.y[id];
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const long long id = base + u * stride;
            if (id >= L.plane) {
                continue;
            }
            const double* q = qv[u];
            double mom2_sum = q[1] * q[1];
            if constexpr (NDIM > 1) {
                mom2_sum += q[2] * q[2];
            }
            if constexpr (NDIM > 2) {
                mom2_sum += q[3] * q[3];
            }
            const double rho = q[0];
            const double e_kin = 0.5 * mom2_sum / rho;
            const double eint = q[ie] - e_kin;
            const double log_rho = log10(rho);
            const double log_eint_rho = log10(eint) - log_rho;
            // The reference aborts on eint < 0 (TabulatedLteH.hpp:142-144); a
            // NaN coordinate (eint < 0, rho <= 0 or a non-finite state) would
            // also index the table out of range. Flag the cell and leave it.
            const double fx = (log_eint_rho - L.x_start) / L.x_step;
            const double fy = (log_rho - L.y_start) / L.y_step;
            if (eint < 0.0 || fx != fx || fy != fy) {
                flags |= kFlagEos;
                continue;
            }
            const Sample s = table_sample(L, Y, LT, log_eint_rho, log_rho);
            const double prev_y = yp[u];
            L.y[id] = s.y;
            const double delta_eint = (prev_y < 0.0) ? 0.0 : rho * (kChiH / kHMass) * (s.y - prev_y);
            L.T[id] = pow(10.0, s.log_T);
            // the state with the energy shifted: in place, or into a copy when
            // the input must stay as it is (the step-start state)
            if (L.q_out != L.q_in) {
                for (int v = 0; v < L.nvar; ++v) {
                    if (v != ie) {
                        L.q_out[id + v * L.plane] = L.q_in[id + v * L.plane];
                    }
                }
            }
            L.q_out[id + ie * L.plane] = q[ie] + delta_eint;
        }
    }
    if (flags && L.blk) {
        atomicOr(&L.blk->status, flags);
    }
}

constexpr size_t kTableSmemMax = 74 * 1024;  // three CTAs per SM (228 KB)

template <class K>
cudaError_t allow_table_smem(K kernel, size_t bytes) {
    if (bytes <= 48 * 1024) {
        return cudaSuccess;
    }
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

} // namespace

cudaError_t launch_eos_update(const EosLaunch& L, int ndim, cudaStream_t s) {
    const long long want = (L.plane + 255) / 256;
    const int blocks = (int)(want < 148 * 16 ? want : 148 * 16);
    if (L.type == kEosAnalytic) {
        if (ndim == 1) {
            eos_analytic_kernel<1><<<blocks, 256, 0, s>>>(L);
        } else if (ndim == 2) {
            eos_analytic_kernel<2><<<blocks, 256, 0, s>>>(L);
        } else {
            eos_analytic_kernel<3><<<blocks, 256, 0, s>>>(L);
        }
    } else if (L.type == kEosTabulated) {
        // both tables in shared memory when they fit three CTAs per SM
        const size_t tab_bytes = 2 * sizeof(double) * (size_t)L.nx_tab * (size_t)L.ny_tab;
        const bool smem = tab_bytes <= kTableSmemMax;
        const size_t sm = smem ? tab_bytes : 0;
        const int grid = smem ? (int)(want < 148 * 3 ? want : 148 * 3) : blocks;
        cudaError_t e = cudaSuccess;
        if (ndim == 1) {
            e = allow_table_smem(eos_tabulated_kernel<1>, sm);
            eos_tabulated_kernel<1><<<grid, 256, sm, s>>>(L, smem ? 1 : 0);
        } else if (ndim == 2) {
            e = allow_table_smem(eos_tabulated_kernel<2>, sm);
            eos_tabulated_kernel<2><<<grid, 256, sm, s>>>(L, smem ? 1 : 0);
        } else {
            e = allow_table_smem(eos_tabulated_kernel<3>, sm);
            eos_tabulated_kernel<3><<<grid, 256, sm, s>>>(L, smem ? 1 : 0);
        }
        if (e != cudaSuccess) {
            return e;
        }
    }
    return cudaGetLastError();
}

} // namespace mc
