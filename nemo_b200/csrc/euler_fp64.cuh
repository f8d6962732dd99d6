// euler_fp64.cuh -- Euler physics in FP64 for the plain path.
//
// Every function evaluates the reference's Fortran expressions in the same order (the Fortran
// files are cited per function); this header is compiled with -fmad=false so that each + - * /
// is one IEEE operation.  All functions work in the frame rotated into the face normal
// direction: u = (rho, m_n, m_t1, m_t2, E), which is how the reference's y/z wrappers call the
// x-direction kernels (source/equations/euler/equations_mod.f90:81-127).
#pragma once

#include "common.cuh"
#include "pmath64.cuh"

namespace nemo {

// pressure_elemental, source/equations/euler/equations_mod.f90:131-140
__device__ __forceinline__ double pressure64(const double* u, const OpConsts& k) {
    return k.km1 * (u[4] - 0.5 / u[0] * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]));
}

// xflux, source/equations/euler/equations_mod.f90:64-79
__device__ __forceinline__ void xflux64(const double* u, double pres, double* f) {
    double velx = u[1] / u[0];
    f[0] = u[1];
    f[1] = velx * u[1] + pres;
    f[2] = velx * u[2];
    f[3] = velx * u[3];
    f[4] = velx * (u[4] + pres);
}

// xlambdaMax, source/equations/euler/equations_mod.f90:384-393 (soundspeed :288-297)
__device__ __forceinline__ double xlambda64(const double* u, const OpConsts& k) {
    double c = sqrt(k.kappa * pressure64(u, k) / u[0]);
    return fabs(u[1] / u[0]) + c;
}

// HLLC/HLLE hybrid, source/equations/euler/riemann/hllc/riemann_mod.f90:7-104
__device__ __forceinline__ void hllc64(const double* UL, const double* UR, double* F, const OpConsts& k) {
    const double kappa = k.kappa;
    const double beta = k.hllc_beta;
    double VL = UL[1] / UL[0];
    double VR = UR[1] / UR[0];
    double pL = pressure64(UL, k);
    double pR = pressure64(UR, k);
    double cL = sqrt(kappa * pL / UL[0]);
    double cR = sqrt(kappa * pR / UR[0]);
    double HL = (UL[4] + pL) / UL[0];
    double HR = (UR[4] + pR) / UR[0];
    double sL = sqrt(UL[0]), sR = sqrt(UR[0]);
    double Ht = (sL * HL + sR * HR) / (sL + sR);
    double vt = (sL * VL + sR * VR) / (sL + sR);
    double at = sqrt(k.km1 * (Ht - 0.5 * (vt * vt)));
    double SL = fmin(fmin(vt - at, VL - beta * cL), 0.0);
    double SR = fmax(fmax(vt + at, VR + beta * cR), 0.0);
    // the supersonic cases (SL >= 0: the left flux, SR <= 0: the right flux) are selected at the
    // end instead of returned early: the same values, and no branch between the Riemann fluxes
    // of a line, which the compiler can then interleave (discarded values may be inf or NaN)
    double FL[5], FR[5];
    xflux64(UL, pL, FL);
    xflux64(UR, pR, FR);
    const bool supL = SL >= 0.0, supR = SR <= 0.0;
    double smooth = sqrt(fabs(pL - pR) / (pL + pR));
    double SS = (pR - pL + UL[1] * (SL - VL) - UR[1] * (SR - VR)) / (UL[0] * (SL - VL) - UR[0] * (SR - VR));
    const bool left = (SL <= 0.0 && 0.0 <= SS);
    const double* U = left ? UL : UR;
    const double* FU = left ? FL : FR;
    const double S = left ? SL : SR;
    const double V = left ? VL : VR;
    const double p = left ? pL : pR;
    double Q = U[0] * (S - V) / (S - SS);
    double Us[5];
    Us[0] = Q;
    Us[1] = Q * SS;
    Us[2] = Q * U[2] / U[0];
    Us[3] = Q * U[3] / U[0];
    Us[4] = Q * (U[4] / U[0] + (SS - V) * (SS + p / U[0] / (S - V)));
    const double oms = 1.0 - smooth;
    const double dS = SR - SL, SLSR = SL * SR;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        double FH = (SR * FL[v] - SL * FR[v] + SLSR * (UR[v] - UL[v])) / dS;
        const double Fm = smooth * FH + oms * (FU[v] + S * (Us[v] - U[v]));
        F[v] = supL ? FL[v] : (supR ? FR[v] : Fm);
    }
}

// Rusanov, source/equations/euler/riemann/rusanov/riemann_mod.f90:7-24
__device__ __forceinline__ void rusanov64(const double* uL, const double* uR, double* F, const OpConsts& k) {
    double FL[5], FR[5];
    double pL = pressure64(uL, k), pR = pressure64(uR, k);
    xflux64(uL, pL, FL);
    xflux64(uR, pR, FR);
    double lL = fabs(uL[1] / uL[0]) + sqrt(k.kappa * pL / uL[0]);
    double lR = fabs(uR[1] / uR[0]) + sqrt(k.kappa * pR / uR[0]);
    double lmax = fmax(lL, lR);
#pragma unroll
    for (int v = 0; v < 5; ++v) F[v] = 0.5 * (FL[v] + FR[v] + lmax * (uL[v] - uR[v]));
}

__device__ __forceinline__ void riemann64(int kind, const double* uL, const double* uR, double* F,
                                          const OpConsts& k) {
    if (kind == 1) rusanov64(uL, uR, F, k);
    else hllc64(uL, uR, F, k);
}

// FAST: the flux kinds fixed at compile time (HLLC faces and subcells, Chandrashekar pairs); a
// run-time switch inside the unrolled line loops is a branch around every flux
template <bool FAST>
__device__ __forceinline__ void riem64(int kind, const double* uL, const double* uR, double* F, const OpConsts& k) {
    if (FAST) hllc64(uL, uR, F, k);
    else riemann64(kind, uL, uR, F, k);
}

// logmean with the absolute switch, source/equations/euler/two_point/chandrashekar/
// two_point_flux_mod.f90:13-32
__device__ __forceinline__ double logmean64(double a, double b) {
    const double c1 = 1.0 / 6.0, c2 = 2.0 / 45.0, c3 = 22.0 / 945.0;
    double x = a / b;
    if (fabs(a - b) < 1e-4) {
        double u = (x * (x - 2.0) + 1.0) / (x * (x + 2.0) + 1.0);
        return (a + b) * (0.5 - u * (c1 - u * (c2 - c3 * u)));
    }
    return (a - b) / plog64(x);
}

// Per-node primitive data of the two-point flux: rho, normal/tangential velocities, beta.
struct Node5 {
    double rho, vn, vt1, vt2, beta;
};

// Chandrashekar EC/KEP flux, two_point_flux_mod.f90:34-77 (the per-node quantities pressure,
// beta = 0.5*rho/p and velocities are computed once per node with the same expressions).
__device__ __forceinline__ void chandrashekar64(const Node5& u, const Node5& v, double* f, const OpConsts& k) {
    double dens = logmean64(u.rho, v.rho);
    double velx = 0.5 * (u.vn + v.vn);
    double vely = 0.5 * (u.vt1 + v.vt1);
    double velz = 0.5 * (u.vt2 + v.vt2);
    double pres = 0.5 * (u.rho + v.rho) / (u.beta + v.beta);
    double ssum = (u.vn * u.vn + v.vn * v.vn) + (u.vt1 * u.vt1 + v.vt1 * v.vt1);
    ssum = ssum + (u.vt2 * u.vt2 + v.vt2 * v.vt2);
    double enth = k.c_enth / logmean64(u.beta, v.beta) + pres / dens + velx * velx + vely * vely +
                  velz * velz - 0.25 * ssum;
    f[0] = dens * velx;
    f[1] = f[0] * velx + pres;
    f[2] = f[0] * vely;
    f[3] = f[0] * velz;
    f[4] = f[0] * enth;
}

// central flux 0.5*(f(u)+f(v)), source/equations/euler/two_point/standard/two_point_flux_mod.f90:13-49
__device__ __forceinline__ void central64(const double* u, double pu, const double* v, double pv, double* f) {
    double fu[5], fv[5];
    xflux64(u, pu, fu);
    xflux64(v, pv, fv);
#pragma unroll
    for (int c = 0; c < 5; ++c) f[c] = 0.5 * (fu[c] + fv[c]);
}

__device__ __forceinline__ bool isvalid64(const double* u, const OpConsts& k) {
    return (u[0] > 0.0) && (pressure64(u, k) > 0.0);
}

// Barotropic cooling after a stage (hook_post_rk_timestep_200,
// source/physics/cooling/barotropic_cooling_mod.f90:39-53): the energy of the barotropic equation of
// state, isothermal at or below dens_critical, adiabatic above (rho^kappa = exp(kappa log rho)).
__device__ __forceinline__ double cooled_energy64(const double* q, const OpConsts& k) {
    const double kin = 0.5 / q[0] * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    if (q[0] <= k.cool_rho) return kin + k.cool_ci * q[0];
    return kin + k.cool_ca * pexp64(k.kappa * plog64(q[0]));
}

}  // namespace nemo
