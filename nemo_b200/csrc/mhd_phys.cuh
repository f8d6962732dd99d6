// mhd_phys.cuh -- GLM-MHD physics for the stage kernels, templated on the arithmetic type.
//
// R = double (plain path, compiled with -fmad=false): the reference's expressions in the
// reference's order, bit-identical to oracle/nemo_oracle.cpp.  R = float (FP32 form, fast math):
// the same formulas in FP32, with the logarithmic-mean switch widened to f^2 < 1e-2.
// All functions work in the frame rotated into the face normal: u = (rho, m_n, m_t1, m_t2, E,
// B_n, B_t1, B_t2, psi) (source/equations/mhd/equations_mod.f90:141-219).
#pragma once

#include "common.cuh"
#include "pmath64.cuh"

namespace nemo {

struct MhdK {
    double kappa, mu0;
};

template <typename R>
__device__ __forceinline__ R mlog(R x);
template <>
__device__ __forceinline__ double mlog<double>(double x) { return plog64(x); }
template <>
__device__ __forceinline__ float mlog<float>(float x) { return __logf(x); }

// pressure_elemental, source/equations/mhd/equations_mod.f90:223-234
template <typename R>
__device__ __forceinline__ R m_pressure(const R* u, R kappa, R mu0) {
    return (kappa - R(1.0)) * (u[4] - R(0.5) / u[0] * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) -
                               R(0.5) / mu0 * (u[5] * u[5] + u[6] * u[6] + u[7] * u[7] + u[8] * u[8]));
}

// xflux, equations_mod.f90:64-139
template <typename R>
__device__ __forceinline__ void m_xflux(const R* U, R* f, R kappa, R mu0, R ch) {
    const R smu_0 = R(1.0) / mu0, s2mu_0 = R(0.5) / mu0;
    const R kappaM1 = kappa - R(1.0), kappaM2 = kappa - R(2.0);
    const R Etotal = U[4] - R(0.5) * smu_0 * (U[8] * U[8]);
    const R srho = R(1.0) / U[0];
    const R v1 = U[1] * srho, v2 = U[2] * srho, v3 = U[3] * srho;
    const R v_2 = v1 * v1 + v2 * v2 + v3 * v3;
    const R bb2 = U[5] * U[5] + U[6] * U[6] + U[7] * U[7];
    const R vb = U[5] * v1 + U[6] * v2 + U[7] * v3;
    const R pt = kappaM1 * (Etotal - R(0.5) * U[0] * v_2) - kappaM2 * s2mu_0 * bb2;
    const R Ep = Etotal + pt;
    f[0] = U[1];
    f[1] = U[1] * v1 + pt - smu_0 * U[5] * U[5];
    f[2] = U[1] * v2 - smu_0 * U[5] * U[6];
    f[3] = U[1] * v3 - smu_0 * U[5] * U[7];
    f[4] = Ep * v1 - smu_0 * U[5] * vb;
    f[5] = R(0.0);
    f[6] = v1 * U[6] - U[5] * v2;
    f[7] = v1 * U[7] - U[5] * v3;
    f[4] = f[4] + smu_0 * ch * U[5] * U[8];
    f[5] = f[5] + ch * U[8];
    f[8] = ch * U[5];
}

// Fastest_Signal_Speed + xlambdaMax, equations_mod.f90:693-714, :522-531
template <typename R>
__device__ __forceinline__ R m_xlambda(const R* U, R kappa, R mu0) {
    const R pres = m_pressure(U, kappa, mu0);
    const R cs2 = kappa * pres / U[0];
    const R ca2 = U[5] * U[5] / U[0] / mu0;
    const R va2 = (U[6] * U[6] + U[7] * U[7]) / U[0] / mu0 + ca2;
    const R astar = sqrt((cs2 + va2) * (cs2 + va2) - R(4.0) * cs2 * ca2);
    const R c = sqrt(R(0.5) * (cs2 + va2 + astar));
    return fabs(U[1] / U[0]) + c;
}

template <typename R>
__device__ __forceinline__ bool m_isvalid(const R* u, R kappa, R mu0) {
    return (u[0] > R(0.0)) && (m_pressure(u, kappa, mu0) > R(0.0));
}

// Rusanov, source/equations/mhd/riemann/rusanov/riemann_mod.f90:7-24
template <typename R>
__device__ __forceinline__ void m_rusanov_x(const R* uL, const R* uR, R* F, R kappa, R mu0, R ch) {
    R FL[9], FR[9];
    m_xflux(uL, FL, kappa, mu0, ch);
    m_xflux(uR, FR, kappa, mu0, ch);
    const R lmax = fmax(m_xlambda(uL, kappa, mu0), m_xlambda(uR, kappa, mu0));
#pragma unroll
    for (int v = 0; v < 9; ++v) F[v] = R(0.5) * (FL[v] + FR[v] + lmax * (uL[v] - uR[v]));
}

// LN_MEAN, source/equations/mhd/two_point/ec/two_point_flux_mod.f90:203-219 (relative switch)
template <typename R>
__device__ __forceinline__ R ln_mean_rel(R aL, R aR) {
    const R Xi = aR / aL;
    const R u = (Xi * (Xi - R(2.0)) + R(1.0)) / (Xi * (Xi + R(2.0)) + R(1.0));
    const R eps = sizeof(R) == 8 ? R(1.0e-4) : R(1.0e-2);
    if (u < eps) return (aL + aR) * R(52.5) / (R(105.0) + u * (R(35.0) + u * (R(21.0) + u * R(15.0))));
    return (aR - aL) / mlog(Xi);
}

// EC (Derigs) flux, source/equations/mhd/two_point/ec/two_point_flux_mod.f90:13-86
template <typename R>
__device__ __forceinline__ void m_ec_x(const R* UL, const R* UR, R* F, R kappa, R mu0, R ch) {
    const R kappaM1 = kappa - R(1.0), skappaM1 = R(1.0) / (kappa - R(1.0)), smu_0 = R(1.0) / mu0;
    const R rho_L = UL[0], rho_R = UR[0];
    const R E_L = UL[4] - R(0.5) * smu_0 * (UL[8] * UL[8]), E_R = UR[4] - R(0.5) * smu_0 * (UR[8] * UR[8]);
    const R psi_L = UL[8], psi_R = UR[8];
    R v_L[3], v_R[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        v_L[c] = UL[1 + c] / rho_L;
        v_R[c] = UR[1 + c] / rho_R;
    }
    const R* B_L = UL + 5;
    const R* B_R = UR + 5;
    const R v2_L = v_L[0] * v_L[0] + v_L[1] * v_L[1] + v_L[2] * v_L[2];
    const R v2_R = v_R[0] * v_R[0] + v_R[1] * v_R[1] + v_R[2] * v_R[2];
    const R B2_L = B_L[0] * B_L[0] + B_L[1] * B_L[1] + B_L[2] * B_L[2];
    const R B2_R = B_R[0] * B_R[0] + B_R[1] * B_R[1] + B_R[2] * B_R[2];
    const R p_L = kappaM1 * (E_L - R(0.5) * (rho_L * v2_L + smu_0 * B2_L));
    const R p_R = kappaM1 * (E_R - R(0.5) * (rho_R * v2_R + smu_0 * B2_R));
    const R beta_L = R(0.5) * rho_L / p_L, beta_R = R(0.5) * rho_R / p_R;
    const R rhoLN = ln_mean_rel(rho_L, rho_R);
    const R betaLN = ln_mean_rel(beta_L, beta_R);
    R vAvg[3], BAvg[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        vAvg[c] = R(0.5) * (v_L[c] + v_R[c]);
        BAvg[c] = R(0.5) * (B_L[c] + B_R[c]);
    }
    const R v1_B2Avg = R(0.5) * (v_L[0] * B2_L + v_R[0] * B2_R);
    const R vB_Avg = R(0.5) * ((v_L[0] * B_L[0] + v_L[1] * B_L[1] + v_L[2] * B_L[2]) +
                               (v_R[0] * B_R[0] + v_R[1] * B_R[1] + v_R[2] * B_R[2]));
    const R pTilde = R(0.5) * ((rho_L + rho_R) / (beta_L + beta_R) + smu_0 * R(0.5) * (B2_L + B2_R));
    const R psiAvg = R(0.5) * (psi_L + psi_R);
    F[0] = rhoLN * vAvg[0];
    F[1] = F[0] * vAvg[0] - smu_0 * BAvg[0] * BAvg[0] + pTilde;
    F[2] = F[0] * vAvg[1] - smu_0 * BAvg[0] * BAvg[1];
    F[3] = F[0] * vAvg[2] - smu_0 * BAvg[0] * BAvg[2];
    F[6] = vAvg[0] * BAvg[1] - BAvg[0] * vAvg[1];
    F[7] = vAvg[0] * BAvg[2] - BAvg[0] * vAvg[2];
    F[5] = ch * psiAvg;
    F[8] = ch * BAvg[0];
    const R s1 = vAvg[0] * F[1] + vAvg[1] * F[2] + vAvg[2] * F[3];
    const R s2 = BAvg[0] * F[5] + BAvg[1] * F[6] + BAvg[2] * F[7];
    F[4] = F[0] * R(0.5) * (skappaM1 / betaLN - R(0.5) * (v2_L + v2_R)) + s1 +
           smu_0 * (s2 - R(0.5) * v1_B2Avg + BAvg[0] * vB_Avg + F[8] * psiAvg -
                    ch * R(0.5) * (psi_L * B_L[0] + psi_R * B_R[0]));
}

template <typename R>
__device__ __forceinline__ void m_central_x(const R* u, const R* v, R* F, R kappa, R mu0, R ch) {
    R fu[9], fv[9];
    m_xflux(u, fu, kappa, mu0, ch);
    m_xflux(v, fv, kappa, mu0, ch);
#pragma unroll
    for (int c = 0; c < 9; ++c) F[c] = R(0.5) * (fu[c] + fv[c]);
}

// Non_Conservative_two_point_xFlux (Powell + GLM), source/equations/mhd/non_conservative_flux_mod.f90:10-45
template <typename R>
__device__ __forceinline__ void m_nc_x(const R* UI, const R* UL, const R* UR, R* F, R mu0) {
    const R Bavg = R(0.5) * (UL[5] + UR[5]);
    const R Gavg = R(0.5) * (UL[8] + UR[8]);
    const R v[3] = {UI[1] / UI[0], UI[2] / UI[0], UI[3] / UI[0]};
    F[0] = R(0.0);
#pragma unroll
    for (int c = 0; c < 3; ++c) F[1 + c] = Bavg * UI[5 + c] / mu0;
    F[4] = Bavg * (UI[5] * v[0] + UI[6] * v[1] + UI[7] * v[2]) / mu0;
#pragma unroll
    for (int c = 0; c < 3; ++c) F[5 + c] = Bavg * v[c];
    F[8] = R(0.0);
    const R gv = Gavg * v[0];
    F[4] = F[4] + gv * (UI[8] / mu0);
    F[8] = F[8] + gv * R(1.0);
}

}  // namespace nemo
