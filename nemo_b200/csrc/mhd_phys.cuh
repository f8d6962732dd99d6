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

// HLLD (Miyoshi & Kusano, J. Comput. Phys. 208 (2005) 315-344) for mu0 = 1: the star and double-star
// states of source/equations/mhd/riemann/hlld/riemann_mod.f90:114-246 with the wave speeds of :83-97.
// That file is disabled in the reference (its line 1 is an #error: the GLM pair is not handled) and
// evaluates the fast speed on primitive variables; here the fast speed is taken from the conserved
// state, and the GLM pair (B_n, psi) is solved upwind first (characteristics B_n +- psi at speeds
// +-c_h, Dedner et al., J. Comput. Phys. 175 (2002)): both HLLD states use the upwind B_n*, the
// energy drops psi^2/2, and the GLM fluxes c_h psi*, c_h B_n*, c_h B_n* psi* are added at the end.
template <typename R>
__device__ __forceinline__ void m_hlld_x(const R* uL, const R* uR, R* F, R kappa, R ch) {
    const R half = R(0.5);
    // GLM pair: characteristics B_n + psi (speed +c_h) from the left, B_n - psi (speed -c_h) from the right
    const R bn = half * (uL[5] + uR[5]) - half * (uR[8] - uL[8]);
    const R psn = half * (uL[8] + uR[8]) - half * (uR[5] - uL[5]);
    const R bn2 = bn * bn;
    // primitive states; the pressure keeps the conserved state's own B_n, the energy E' drops psi
    R rho[2], un[2], vt1[2], vt2[2], bt1[2], bt2[2], pr[2], et[2], pt[2], cf[2];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const R* u = s ? uR : uL;
        rho[s] = u[0];
        un[s] = u[1] / u[0];
        vt1[s] = u[2] / u[0];
        vt2[s] = u[3] / u[0];
        bt1[s] = u[6];
        bt2[s] = u[7];
        pr[s] = (kappa - R(1.0)) * (u[4] - half / u[0] * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) -
                                    half * (u[5] * u[5] + u[6] * u[6] + u[7] * u[7] + u[8] * u[8]));
        const R bb = bn2 + bt1[s] * bt1[s] + bt2[s] * bt2[s];
        et[s] = pr[s] / (kappa - R(1.0)) + half * rho[s] * (un[s] * un[s] + vt1[s] * vt1[s] + vt2[s] * vt2[s]) + half * bb;
        pt[s] = pr[s] + half * bb;
        const R cs2 = kappa * pr[s] / rho[s];
        const R ca2 = bn2 / rho[s];
        const R va2 = bb / rho[s];
        cf[s] = sqrt(half * (cs2 + va2 + sqrt((cs2 + va2) * (cs2 + va2) - R(4.0) * cs2 * ca2)));
    }
    const R cmax = fmax(cf[0], cf[1]);
    const R SL = fmin(un[0], un[1]) - cmax;
    const R SR = fmax(un[0], un[1]) + cmax;
    // ideal-MHD fluxes of both states (GLM parts added at the end) and the states themselves
    R Fk[2][8], Uk[2][8];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const R vb = un[s] * bn + vt1[s] * bt1[s] + vt2[s] * bt2[s];
        const R m = rho[s] * un[s];
        Fk[s][0] = m;
        Fk[s][1] = m * un[s] + pt[s] - bn2;
        Fk[s][2] = m * vt1[s] - bn * bt1[s];
        Fk[s][3] = m * vt2[s] - bn * bt2[s];
        Fk[s][4] = (et[s] + pt[s]) * un[s] - bn * vb;
        Fk[s][5] = R(0.0);
        Fk[s][6] = un[s] * bt1[s] - bn * vt1[s];
        Fk[s][7] = un[s] * bt2[s] - bn * vt2[s];
        Uk[s][0] = rho[s];
        Uk[s][1] = m;
        Uk[s][2] = rho[s] * vt1[s];
        Uk[s][3] = rho[s] * vt2[s];
        Uk[s][4] = et[s];
        Uk[s][5] = bn;
        Uk[s][6] = bt1[s];
        Uk[s][7] = bt2[s];
    }
    if (SL > R(0.0)) {
#pragma unroll
        for (int v = 0; v < 8; ++v) F[v] = Fk[0][v];
    } else if (SR < R(0.0)) {
#pragma unroll
        for (int v = 0; v < 8; ++v) F[v] = Fk[1][v];
    } else {
        const R dL = rho[0] * (SL - un[0]), dR = rho[1] * (SR - un[1]);
        const R SM = (dR * un[1] - dL * un[0] - pt[1] + pt[0]) / (dR - dL);
        const R ptS = pt[0] + dL * (SM - un[0]);
        // single-star states
        R rs[2], ws1[2], ws2[2], cs1[2], cs2[2], es[2];
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const R S = s ? SR : SL;
            const R d = s ? dR : dL;
            rs[s] = d / (S - SM);
            const R den = d * (S - SM) - bn2;
            if (fabs(den) < R(1.0e-8)) {
                ws1[s] = vt1[s];
                ws2[s] = vt2[s];
                cs1[s] = bt1[s];
                cs2[s] = bt2[s];
            } else {
                const R fv = bn * (SM - un[s]) / den;
                const R fb = (d * (S - un[s]) - bn2) / den;
                ws1[s] = vt1[s] - fv * bt1[s];
                ws2[s] = vt2[s] - fv * bt2[s];
                cs1[s] = fb * bt1[s];
                cs2[s] = fb * bt2[s];
            }
            const R vb = un[s] * bn + vt1[s] * bt1[s] + vt2[s] * bt2[s];
            const R vbs = SM * bn + ws1[s] * cs1[s] + ws2[s] * cs2[s];
            es[s] = ((S - un[s]) * et[s] - pt[s] * un[s] + ptS * SM + bn * (vb - vbs)) / (S - SM);
        }
        const R sqL = sqrt(rs[0]), sqR = sqrt(rs[1]);
        const R SLs = SM - fabs(bn) / sqL, SRs = SM + fabs(bn) / sqR;
        // side s of the contact (0: left, 1: right) picked by selects, not by indexing with a run-time
        // index, which would put the two-sided arrays in local memory
        const bool sr = !(SM >= R(0.0));
        const R S = sr ? SR : SL;
        const R rsS = sr ? rs[1] : rs[0], ws1S = sr ? ws1[1] : ws1[0], ws2S = sr ? ws2[1] : ws2[0];
        const R cs1S = sr ? cs1[1] : cs1[0], cs2S = sr ? cs2[1] : cs2[0], esS = sr ? es[1] : es[0];
        R Us[8];
        Us[0] = rsS;
        Us[1] = rsS * SM;
        Us[2] = rsS * ws1S;
        Us[3] = rsS * ws2S;
        Us[4] = esS;
        Us[5] = bn;
        Us[6] = cs1S;
        Us[7] = cs2S;
        const bool outer = sr ? (SRs < R(0.0)) : (SLs >= R(0.0));
        if (outer) {
#pragma unroll
            for (int v = 0; v < 8; ++v) {
                const R FkS = sr ? Fk[1][v] : Fk[0][v], UkS = sr ? Uk[1][v] : Uk[0][v];
                F[v] = FkS + S * (Us[v] - UkS);
            }
        } else {
            // double-star state of side s (Alfven waves); it equals the single-star state if B_n = 0
            R Uss[8];
#pragma unroll
            for (int v = 0; v < 8; ++v) Uss[v] = Us[v];
            if (fabs(bn) >= R(1.0e-12)) {
                const R sg = bn < R(0.0) ? R(-1.0) : R(1.0);
                const R sden = R(1.0) / (sqL + sqR);
                const R w1 = (sqL * ws1[0] + sqR * ws1[1] + sg * (cs1[1] - cs1[0])) * sden;
                const R w2 = (sqL * ws2[0] + sqR * ws2[1] + sg * (cs2[1] - cs2[0])) * sden;
                const R c1 = (sqL * cs1[1] + sqR * cs1[0] + sg * sqL * sqR * (ws1[1] - ws1[0])) * sden;
                const R c2 = (sqL * cs2[1] + sqR * cs2[0] + sg * sqL * sqR * (ws2[1] - ws2[0])) * sden;
                const R wcs = ws1S * cs1S + ws2S * cs2S;
                const R wcss = w1 * c1 + w2 * c2;
                const R sq = sr ? sqR : sqL;
                Uss[2] = rsS * w1;
                Uss[3] = rsS * w2;
                Uss[4] = sr ? esS + sg * sq * (wcs - wcss) : esS - sg * sq * (wcs - wcss);
                Uss[6] = c1;
                Uss[7] = c2;
            }
            const R Ss = sr ? SRs : SLs;
#pragma unroll
            for (int v = 0; v < 8; ++v) {
                const R FkS = sr ? Fk[1][v] : Fk[0][v], UkS = sr ? Uk[1][v] : Uk[0][v];
                F[v] = FkS + Ss * Uss[v] - (Ss - S) * Us[v] - S * UkS;
            }
        }
    }
    F[4] = F[4] + ch * bn * psn;
    F[5] = ch * psn;
    F[8] = ch * bn;
}

template <typename R>
__device__ __forceinline__ void m_riemann_x(int kind, const R* uL, const R* uR, R* F, R kappa, R mu0, R ch) {
    if (kind == NEMO_SURFFLUX_HLLD) m_hlld_x(uL, uR, F, kappa, ch);
    else m_rusanov_x(uL, uR, F, kappa, mu0, ch);
}

// FAST: HLLD fixed at compile time (no run-time switch around every flux of the unrolled loops)
template <bool FAST, typename R>
__device__ __forceinline__ void m_riem(int kind, const R* uL, const R* uR, R* F, R kappa, R mu0, R ch) {
    if (FAST) m_hlld_x(uL, uR, F, kappa, ch);
    else m_riemann_x(kind, uL, uR, F, kappa, mu0, ch);
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
