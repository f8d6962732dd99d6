// stage_fp32.cu -- the FP32-bulk form of the fused LSRK stage (compiled with --use_fast_math).
//
// Same decomposition and thread mapping as stage_fp64.cu (one CTA = 8 elements, 48 threads per
// element, one per (direction, line)), with the precision split of the mixed-precision design:
//   FP64: the state and the RK register in HBM, the per-node primitive recovery (pressure from
//         conserved variables, where cancellation between total and kinetic energy lives), the
//         register/state update, the positivity repair and the CFL minimum;
//   FP32: all two-point fluxes, Riemann fluxes, FV subcells, the lift and the indicator.
// The logarithmic mean switches on the relative difference (Ismail-Roe form: f = (a-b)/(a+b),
// 4-term series for f^2 < 1e-2, else (a-b)/log(a/b)), because the reference's absolute switch
// |a-b| < 1e-4 is meaningless in FP32 for beta = rho/(2p) ~ 5e4.  The HBM traffic is that of the
// plain path (FP64 u in/out, FP64 register in/out); the arithmetic per node pair is a third.
#include "common.cuh"
#include "euler_fp64.cuh"
#include "kernels.h"
#include "repair64.cuh"

namespace nemo {

__constant__ OpConsts c_ops32;

namespace {

constexpr int EPC = 8;
constexpr int TPE = 48;
constexpr int NT = EPC * TPE;
constexpr int V = 5;

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ bool mbar_wait32(uint64_t* bar, unsigned phase) {
    unsigned addr = smem_u32(bar);
    for (int it = 0; it < (1 << 24); ++it) {
        unsigned ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok) : "r"(addr), "r"(phase) : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ bool tile_load32(double* su, const double* __restrict__ u, int64_t E, int64_t e0, int nel,
                                            uint64_t* bar, Control* ctrl) {
    if (threadIdx.x == 0) {
        unsigned b = smem_u32(bar);
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned b = smem_u32(bar);
        unsigned bytes = (unsigned)(nel * NP * 8);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes * V) : "memory");
        for (int v = 0; v < V; ++v) {
            const double* src = u + ((int64_t)v * E + e0) * NP;
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smem_u32(su + v * EPC * NP)),
                "l"(src), "r"(bytes), "r"(b)
                : "memory");
        }
    }
    bool ok = mbar_wait32(bar, 0);
    if (!ok) {
        atomicOr(&ctrl->error, 1);
        mbar_wait32(bar, 0);
    }
    return ok;
}

// Per-node FP32 primitives in the frame of direction d.
struct P32 {
    float rho, vn, vt1, vt2, p, E;
};

// Physical x-flux from primitives (equations_mod.f90:64-79 in primitive form).
__device__ __forceinline__ void xflux32(const P32& q, float* f) {
    const float mn = q.rho * q.vn;
    f[0] = mn;
    f[1] = mn * q.vn + q.p;
    f[2] = mn * q.vt1;
    f[3] = mn * q.vt2;
    f[4] = q.vn * (q.E + q.p);
}

// HLLC/HLLE hybrid (source/equations/euler/riemann/hllc/riemann_mod.f90:7-104) in FP32, on
// primitives recovered in FP64.
__device__ __forceinline__ void hllc32(const P32& L, const P32& R, float* F, const OpConsts& k) {
    const float kappa = (float)k.kappa;
    const float beta = (float)k.hllc_beta;
    const float km1 = (float)k.km1;
    const float cL = sqrtf(kappa * L.p / L.rho);
    const float cR = sqrtf(kappa * R.p / R.rho);
    const float HL = (L.E + L.p) / L.rho;
    const float HR = (R.E + R.p) / R.rho;
    const float sL = sqrtf(L.rho), sR = sqrtf(R.rho);
    const float isum = 1.0f / (sL + sR);
    const float Ht = (sL * HL + sR * HR) * isum;
    const float vt = (sL * L.vn + sR * R.vn) * isum;
    const float at = sqrtf(fmaxf(km1 * (Ht - 0.5f * vt * vt), 0.0f));
    const float SL = fminf(fminf(vt - at, L.vn - beta * cL), 0.0f);
    const float SR = fmaxf(fmaxf(vt + at, R.vn + beta * cR), 0.0f);
    float FL[5], FR[5];
    xflux32(L, FL);
    xflux32(R, FR);
    if (SL >= 0.0f) {
#pragma unroll
        for (int v = 0; v < 5; ++v) F[v] = FL[v];
        return;
    }
    if (SR <= 0.0f) {
#pragma unroll
        for (int v = 0; v < 5; ++v) F[v] = FR[v];
        return;
    }
    const float UL[5] = {L.rho, L.rho * L.vn, L.rho * L.vt1, L.rho * L.vt2, L.E};
    const float UR[5] = {R.rho, R.rho * R.vn, R.rho * R.vt1, R.rho * R.vt2, R.E};
    const float smooth = sqrtf(fabsf(L.p - R.p) / (L.p + R.p));
    const float aL = L.rho * (SL - L.vn), aR = R.rho * (SR - R.vn);
    const float SS = (R.p - L.p + UL[1] * (SL - L.vn) - UR[1] * (SR - R.vn)) / (aL - aR);
    const bool left = (0.0f <= SS);
    const P32& Q = left ? L : R;
    const float S = left ? SL : SR;
    const float qs = (left ? aL : aR) / (S - SS);
    const float Us[5] = {qs, qs * SS, qs * Q.vt1, qs * Q.vt2,
                         qs * (Q.E / Q.rho + (SS - Q.vn) * (SS + Q.p / (Q.rho * (S - Q.vn))))};
    const float idS = 1.0f / (SR - SL);
    const float oms = 1.0f - smooth;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        const float FH = (SR * FL[v] - SL * FR[v] + SL * SR * (UR[v] - UL[v])) * idS;
        const float Fu = left ? FL[v] : FR[v];
        const float Uu = left ? UL[v] : UR[v];
        F[v] = smooth * FH + oms * (Fu + S * (Us[v] - Uu));
    }
}

// Rusanov (source/equations/euler/riemann/rusanov/riemann_mod.f90:7-24) in FP32.
__device__ __forceinline__ void rusanov32(const P32& L, const P32& R, float* F, const OpConsts& k) {
    const float kappa = (float)k.kappa;
    float FL[5], FR[5];
    xflux32(L, FL);
    xflux32(R, FR);
    const float lm = fmaxf(fabsf(L.vn) + sqrtf(kappa * L.p / L.rho), fabsf(R.vn) + sqrtf(kappa * R.p / R.rho));
    const float UL[5] = {L.rho, L.rho * L.vn, L.rho * L.vt1, L.rho * L.vt2, L.E};
    const float UR[5] = {R.rho, R.rho * R.vn, R.rho * R.vt1, R.rho * R.vt2, R.E};
#pragma unroll
    for (int v = 0; v < 5; ++v) F[v] = 0.5f * (FL[v] + FR[v] + lm * (UL[v] - UR[v]));
}

__device__ __forceinline__ void riemann32(int kind, const P32& L, const P32& R, float* F, const OpConsts& k) {
    if (kind == 1) rusanov32(L, R, F, k);
    else hllc32(L, R, F, k);
}

// Logarithmic mean with a relative switch (Ismail-Roe): (a-b)/log(a/b) = (a+b)/2 / g(f^2),
// g(u) = atanh(sqrt u)/sqrt u = 1 + u/3 + u^2/5 + u^3/7 + ... for f = (a-b)/(a+b).
__device__ __forceinline__ float lnmean32(float a, float b) {
    const float s = a + b;
    const float f = (a - b) / s;
    const float u = f * f;
    if (u < 1e-2f) return 0.5f * s / (1.0f + u * (1.0f / 3.0f + u * (0.2f + u * (1.0f / 7.0f))));
    return (a - b) / __logf(a / b);
}

}  // namespace

// Node data in smem (FP32): rho, vx, vy, vz, p, E, beta, |v|^2 -> 8 arrays [8][EPC][64]
template <bool BLEND, bool RHS_ONLY>
__global__ void __launch_bounds__(NT, 2) k_stage_euler32(StageArgs a) {
    extern __shared__ __align__(128) double smem[];
    double* su = smem;                                  // [V][EPC][64] FP64 state
    float* sq = reinterpret_cast<float*>(su + V * EPC * NP);   // [8][EPC][64] FP32 node data
    float* sR = sq + 8 * EPC * NP;                       // [3][V][EPC][64] FP32 direction terms
    __shared__ uint64_t bar;
    __shared__ float s_alpha[EPC];
    __shared__ int s_bad[EPC];
    __shared__ unsigned s_lam[EPC][3];

    const OpConsts& k = c_ops32;
    Control* ctrl = a.ctrl;
    if (!RHS_ONLY && ctrl->done) return;
    const int tid = threadIdx.x;
    const int64_t E = a.E;
    const int64_t e0 = (int64_t)blockIdx.x * EPC;
    const int nel = (int)min((int64_t)EPC, E - e0);

    if (tid < EPC) {
        s_bad[tid] = 0;
        s_lam[tid][0] = s_lam[tid][1] = s_lam[tid][2] = 0u;
        float al = 0.0f;
        if (BLEND && tid < nel) {
            const int64_t e = e0 + tid;
            double ad = a.alpha_in[e];
            if (a.smooth) {
#pragma unroll
                for (int f = 0; f < 6; ++f) {
                    const int32_t ne = a.nbr[e * 6 + f];
                    if (ne >= 0) ad = fmax(ad, 0.5 * a.alpha_in[ne]);
                }
            }
            if (a.alpha_used) a.alpha_used[e] = ad;
            al = (float)ad;
        }
        s_alpha[tid] = al;
    }
    if (!tile_load32(su, a.u_in, E, e0, nel, &bar, ctrl)) return;

    auto SQ = [&](int q, int el, int n) -> float& { return sq[(q * EPC + el) * NP + n]; };
    // per-node primitives: recovered in FP64, stored in FP32
    for (int p = tid; p < nel * NP; p += NT) {
        const int el = p / NP, n = p % NP;
        const double r = su[(0 * EPC + el) * NP + n];
        const double mx = su[(1 * EPC + el) * NP + n], my = su[(2 * EPC + el) * NP + n];
        const double mz = su[(3 * EPC + el) * NP + n], en = su[(4 * EPC + el) * NP + n];
        const double ir = 1.0 / r;
        const double vx = mx * ir, vy = my * ir, vz = mz * ir;
        const double pr = k.km1 * (en - 0.5 * (mx * vx + my * vy + mz * vz));
        SQ(0, el, n) = (float)r;
        SQ(1, el, n) = (float)vx;
        SQ(2, el, n) = (float)vy;
        SQ(3, el, n) = (float)vz;
        SQ(4, el, n) = (float)pr;
        SQ(5, el, n) = (float)en;
        SQ(6, el, n) = (float)(0.5 * r / pr);
        SQ(7, el, n) = (float)(vx * vx + vy * vy + vz * vz);
    }
    __syncthreads();

    const int el = tid / TPE;
    const int rr = tid % TPE;
    const int d = rr / NF;
    const int ab = rr % NF;
    const int la = ab & 3, lb = ab >> 2;
    const bool active = el < nel;
    const int64_t e = e0 + el;
    const int c0 = d, c1 = (d + 1) % 3, c2 = (d + 2) % 3;

    auto node = [&](int elx, int n) {
        P32 q;
        q.rho = SQ(0, elx, n);
        q.vn = SQ(1 + c0, elx, n);
        q.vt1 = SQ(1 + c1, elx, n);
        q.vt2 = SQ(1 + c2, elx, n);
        q.p = SQ(4, elx, n);
        q.E = SQ(5, elx, n);
        return q;
    };

    float t[NN][V];
    if (active) {
        float Fs[2][V];
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const int f = 2 * d + side;
            const int own = line_node(d, la, lb, side ? NN - 1 : 0);
            const P32 qo = node(el, own);
            P32 qn = qo;
            const int32_t ne = a.nbr[e * 6 + f];
            if (ne >= 0) {
                const int nn = line_node(d, la, lb, side ? 0 : NN - 1);
                const int64_t nl = (int64_t)ne - e0;
                if (nl >= 0 && nl < nel) {
                    qn = node((int)nl, nn);
                } else {
                    const double* g = a.u_in;
                    const double r = __ldg(g + ((int64_t)0 * E + ne) * NP + nn);
                    const double m0 = __ldg(g + ((int64_t)(1 + c0) * E + ne) * NP + nn);
                    const double m1 = __ldg(g + ((int64_t)(1 + c1) * E + ne) * NP + nn);
                    const double m2 = __ldg(g + ((int64_t)(1 + c2) * E + ne) * NP + nn);
                    const double en = __ldg(g + ((int64_t)4 * E + ne) * NP + nn);
                    const double ir = 1.0 / r;
                    const double v0 = m0 * ir, v1 = m1 * ir, v2 = m2 * ir;
                    qn.rho = (float)r;
                    qn.vn = (float)v0;
                    qn.vt1 = (float)v1;
                    qn.vt2 = (float)v2;
                    qn.p = (float)(k.km1 * (en - 0.5 * (m0 * v0 + m1 * v1 + m2 * v2)));
                    qn.E = (float)en;
                }
            }
            if (side) riemann32(a.surface_flux, qo, qn, Fs[1], k);
            else riemann32(a.surface_flux, qn, qo, Fs[0], k);
        }
        int idx[NN];
#pragma unroll
        for (int i = 0; i < NN; ++i) idx[i] = line_node(d, la, lb, i);
#pragma unroll
        for (int i = 0; i < NN; ++i)
#pragma unroll
            for (int v = 0; v < V; ++v) t[i][v] = 0.0f;
        const float c_enth = (float)k.c_enth;
        const int PI_[6] = {0, 0, 0, 1, 1, 2};
        const int PM_[6] = {1, 2, 3, 2, 3, 3};
#pragma unroll
        for (int pq = 0; pq < 6; ++pq) {
            const int i = PI_[pq], m = PM_[pq];
            const int ni = idx[i], nm = idx[m];
            float F[V];
            if (a.volume_flux == NEMO_VOLFLUX_CENTRAL) {
                float fa[V], fb[V];
                xflux32(node(el, ni), fa);
                xflux32(node(el, nm), fb);
#pragma unroll
                for (int v = 0; v < V; ++v) F[v] = 0.5f * (fa[v] + fb[v]);
            } else {
                const float ru = SQ(0, el, ni), rv = SQ(0, el, nm);
                const float bu = SQ(6, el, ni), bv = SQ(6, el, nm);
                const float un = SQ(1 + c0, el, ni), vn = SQ(1 + c0, el, nm);
                const float u1 = SQ(1 + c1, el, ni), v1 = SQ(1 + c1, el, nm);
                const float u2 = SQ(1 + c2, el, ni), v2 = SQ(1 + c2, el, nm);
                const float dens = lnmean32(ru, rv);
                const float velx = 0.5f * (un + vn), vely = 0.5f * (u1 + v1), velz = 0.5f * (u2 + v2);
                const float pres = 0.5f * (ru + rv) / (bu + bv);
                const float enth = c_enth / lnmean32(bu, bv) + pres / dens + velx * velx + vely * vely + velz * velz -
                                   0.25f * (SQ(7, el, ni) + SQ(7, el, nm));
                F[0] = dens * velx;
                F[1] = F[0] * velx + pres;
                F[2] = F[0] * vely;
                F[3] = F[0] * velz;
                F[4] = F[0] * enth;
            }
            const float sim = (float)k.S[i * NN + m], smi = (float)k.S[m * NN + i];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                t[i][v] += sim * F[v];
                t[m][v] += smi * F[v];
            }
        }
        const float w0 = (float)k.winv[0], w3 = (float)k.winv[NN - 1];
#pragma unroll
        for (int v = 0; v < V; ++v) {
            t[0][v] -= w0 * Fs[0][v];
            t[NN - 1][v] += w3 * Fs[1][v];
        }
        if (BLEND) {
            const float al = s_alpha[el];
            if (al > 0.0f) {
                float Fl[V], Fr[V];
#pragma unroll
                for (int v = 0; v < V; ++v) Fl[v] = Fs[0][v];
#pragma unroll
                for (int i = 0; i < NN; ++i) {
                    if (i < NN - 1) {
                        riemann32(a.surface_flux, node(el, idx[i]), node(el, idx[i + 1]), Fr, k);
                    } else {
#pragma unroll
                        for (int v = 0; v < V; ++v) Fr[v] = Fs[1][v];
                    }
                    const float wi = (float)k.winv[i];
#pragma unroll
                    for (int v = 0; v < V; ++v) {
                        t[i][v] = (1.0f - al) * t[i][v] + al * (wi * (Fr[v] - Fl[v]));
                        Fl[v] = Fr[v];
                    }
                }
            }
        }
        const float cd = (float)a.cdel[e * 3 + d];
        float* R = sR + d * V * EPC * NP;
#pragma unroll
        for (int i = 0; i < NN; ++i) {
            const int n = idx[i];
            R[(0 * EPC + el) * NP + n] = cd * t[i][0];
            R[((1 + c0) * EPC + el) * NP + n] = cd * t[i][1];
            R[((1 + c1) * EPC + el) * NP + n] = cd * t[i][2];
            R[((1 + c2) * EPC + el) * NP + n] = cd * t[i][3];
            R[(4 * EPC + el) * NP + n] = cd * t[i][4];
        }
    }
    __syncthreads();

    // ---- FP64 register/state update
    const int st = a.stage;
    const double A = rk_a(st);
    const double Cdt = rk_c(st) * ctrl->dt[0];
    for (int p = tid; p < nel * NP; p += NT) {
        const int pel = p / NP, n = p % NP;
        const int64_t pe = e0 + pel;
        const double cdt = a.group ? rk_c(st) * ctrl->dt[a.group[pe]] : Cdt;
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const int s = (v * EPC + pel) * NP + n;
            const float R3 = (sR[s] + sR[V * EPC * NP + s]) + sR[2 * V * EPC * NP + s];
            const double rhs = -(double)R3;
            const int64_t g = ((int64_t)v * E + pe) * NP + n;
            if (RHS_ONLY) {
                a.rhs_out[g] = rhs;
            } else {
                const double r2 = st == 0 ? rhs : A * a.reg[g] + rhs;
                a.reg[g] = r2;
                su[s] = su[s] + cdt * r2;
            }
        }
        if (!RHS_ONLY && a.positivity) {
            double q[V];
#pragma unroll
            for (int v = 0; v < V; ++v) q[v] = su[(v * EPC + pel) * NP + n];
            if (!isvalid64(q, k)) s_bad[pel] = 1;
        }
    }
    if (RHS_ONLY) return;
    __syncthreads();
    if (a.positivity && tid < nel && s_bad[tid]) {
        // the repair of the plain path, on the FP64 state (rare)
        if (!repair_elem<EPC>(su, tid, k)) atomicAdd(&ctrl->nbad, 1ull);
    }
    __syncthreads();
    for (int p = tid; p < nel * NP; p += NT) {
        const int pel = p / NP, n = p % NP;
#pragma unroll
        for (int v = 0; v < V; ++v) a.u_out[((int64_t)v * E + e0 + pel) * NP + n] = su[(v * EPC + pel) * NP + n];
    }
    if (st == 4 && blockIdx.x == 0 && tid == 0) {
        for (int g = 0; g < ctrl->ngroups; ++g) ctrl->t[g] = ctrl->t[g] + ctrl->dt[g];
        ctrl->steps += 1;
    }

    // ---- epilogue on the new state: modal indicator (FP32) and CFL bound (FP32 speeds, FP64 min)
    const bool need_lam = a.epi_dt != 0;
    if (a.alpha_out || need_lam) {
        float* q = sR;                 // [EPC][64]
        float* t1 = sR + EPC * NP;
        float* t2 = sR + 2 * EPC * NP;
        for (int p = tid; p < nel * NP; p += NT) {
            const int pel = p / NP, n = p % NP;
            const double r = su[(0 * EPC + pel) * NP + n];
            const double mx = su[(1 * EPC + pel) * NP + n], my = su[(2 * EPC + pel) * NP + n];
            const double mz = su[(3 * EPC + pel) * NP + n], en = su[(4 * EPC + pel) * NP + n];
            const double ir = 1.0 / r;
            const double pr = k.km1 * (en - 0.5 * ir * (mx * mx + my * my + mz * mz));
            q[pel * NP + n] = (float)(r * pr);
            if (need_lam) {
                const float c = sqrtf((float)(k.kappa * pr * ir));
                const float vx = (float)(mx * ir), vy = (float)(my * ir), vz = (float)(mz * ir);
                atomicMax(&s_lam[pel][0], __float_as_uint(fabsf(vx) + c));
                atomicMax(&s_lam[pel][1], __float_as_uint(fabsf(vy) + c));
                atomicMax(&s_lam[pel][2], __float_as_uint(fabsf(vz) + c));
            }
        }
        __syncthreads();
        if (a.alpha_out) {
            for (int p = tid; p < nel * NP; p += NT) {
                const int pel = p / NP, n = p % NP;
                const int ai = n % NN, j = (n / NN) % NN, kk = n / NF;
                float s = 0.0f;
#pragma unroll
                for (int i = 0; i < NN; ++i) s += (float)k.Vinv[ai * NN + i] * q[pel * NP + nidx(i, j, kk)];
                t1[pel * NP + n] = s;
            }
            __syncthreads();
            for (int p = tid; p < nel * NP; p += NT) {
                const int pel = p / NP, n = p % NP;
                const int ai = n % NN, bj = (n / NN) % NN, kk = n / NF;
                float s = 0.0f;
#pragma unroll
                for (int j = 0; j < NN; ++j) s += (float)k.Vinv[bj * NN + j] * t1[pel * NP + nidx(ai, j, kk)];
                t2[pel * NP + n] = s;
            }
            __syncthreads();
            for (int p = tid; p < nel * NP; p += NT) {
                const int pel = p / NP, n = p % NP;
                const int ai = n % NN, bj = (n / NN) % NN, cc = n / NF;
                float s = 0.0f;
#pragma unroll
                for (int kk = 0; kk < NN; ++kk) s += (float)k.Vinv[cc * NN + kk] * t2[pel * NP + nidx(ai, bj, kk)];
                q[pel * NP + n] = s * s;  // modal energies
            }
            __syncthreads();
            // energies summed by the 64 modes of each element: one warp-sized group per element
            if (tid < nel * 32) {
                const int pel = tid / 32, lane = tid % 32;
                float tot = 0.f, c1s = 0.f, c2s = 0.f;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int n = lane + 32 * h;
                    const int ai = n % NN, bj = (n / NN) % NN, cc = n / NF;
                    const float e2 = q[pel * NP + n];
                    tot += e2;
                    if (ai < NN - 1 && bj < NN - 1 && cc < NN - 1) c1s += e2;
                    if (ai < NN - 2 && bj < NN - 2 && cc < NN - 2) c2s += e2;
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    tot += __shfl_xor_sync(0xffffffffu, tot, o);
                    c1s += __shfl_xor_sync(0xffffffffu, c1s, o);
                    c2s += __shfl_xor_sync(0xffffffffu, c2s, o);
                }
                if (lane == 0) {
                    const float energy = fmaxf((tot - c1s) / tot, (c1s - c2s) / c1s);
                    float al = 1.0f / (1.0f + __expf((float)k.ind_k * (energy - (float)k.ind_T)));
                    if (al < (float)k.alpha_min) al = 0.0f;
                    else if (al > (float)k.one_m_alpha_min) al = 1.0f;
                    a.alpha_out[e0 + pel] = (double)fminf((float)k.alpha_max, al);
                }
            }
        }
        if (need_lam && tid < nel) {
            const int64_t pe = e0 + tid;
            const double lf = (double)__uint_as_float(s_lam[tid][0]);
            const double lg = (double)__uint_as_float(s_lam[tid][1]);
            const double lh = (double)__uint_as_float(s_lam[tid][2]);
            const double dte = fmin(fmin(a.delta[pe * 3 + 0] / lf, a.delta[pe * 3 + 1] / lg), a.delta[pe * 3 + 2] / lh);
            const int g = a.group ? a.group[pe] : 0;
            atomicMin(&ctrl->dtmin_bits[g], (unsigned long long)__double_as_longlong(dte));
            atomicMax(&ctrl->lmax_bits[g], (unsigned long long)__double_as_longlong(fmax(fmax(lf, lg), lh)));
        }
    }
}

int stage_smem_bytes32() {
    return V * EPC * NP * (int)sizeof(double) + (8 + 3 * V) * EPC * NP * (int)sizeof(float);
}

cudaError_t launch_stage_euler32(const StageArgs& a, bool blend, bool rhs_only, cudaStream_t s) {
    const int grid = (int)((a.E + EPC - 1) / EPC);
    const int smem = stage_smem_bytes32();
    if (rhs_only) {
        if (blend) k_stage_euler32<true, true><<<grid, NT, smem, s>>>(a);
        else k_stage_euler32<false, true><<<grid, NT, smem, s>>>(a);
    } else {
        if (blend) k_stage_euler32<true, false><<<grid, NT, smem, s>>>(a);
        else k_stage_euler32<false, false><<<grid, NT, smem, s>>>(a);
    }
    return cudaGetLastError();
}

template <typename K>
static cudaError_t set_attrs32(K kernel, int smem) {
    cudaError_t err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (err != cudaSuccess) return err;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
}

cudaError_t setup_stage_euler32(const OpConsts& ops) {
    const int smem = stage_smem_bytes32();
    cudaError_t err;
    if ((err = set_attrs32(k_stage_euler32<true, true>, smem)) != cudaSuccess) return err;
    if ((err = set_attrs32(k_stage_euler32<false, true>, smem)) != cudaSuccess) return err;
    if ((err = set_attrs32(k_stage_euler32<true, false>, smem)) != cudaSuccess) return err;
    if ((err = set_attrs32(k_stage_euler32<false, false>, smem)) != cudaSuccess) return err;
    return cudaMemcpyToSymbol(c_ops32, &ops, sizeof(OpConsts));
}

}  // namespace nemo
