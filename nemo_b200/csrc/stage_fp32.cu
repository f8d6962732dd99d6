// stage_fp32.cu -- the FP32-bulk form of the fused LSRK stage (compiled with --use_fast_math).
//
// One CTA = 4, 8 or 16 consecutive elements of the Morton order (8: a 2x2x2 block of a brick, 16: a
// 4x2x2 block), 16 threads per element, thread (a,b) owning the three lines through (a,b); two
// kernels per tile size, a general one (flux kinds and indicator chosen at run time) and one
// specialised to HLLC + Chandrashekar + modal indicator; precision split of the mixed-precision design:
//   FP64: the state and the RK register in HBM, the per-node primitive recovery (pressure from
//         conserved variables, where cancellation between total and kinetic energy lives), the
//         register/state update, the positivity repair and the CFL minimum;
//   FP32: all two-point fluxes, Riemann fluxes, FV subcells, the lift and the indicator.
// The logarithmic mean switches on the relative difference (Ismail-Roe form: f = (a-b)/(a+b),
// 4-term series for f^2 < 1e-2, else (a-b)/log(a/b)), because the reference's absolute switch
// |a-b| < 1e-4 is meaningless in FP32 for beta = rho/(2p) ~ 5e4; the Chandrashekar pair is written
// in terms of g = atanh(f)/f, which leaves it three divisions.  The HBM traffic is that of the
// plain path (FP64 u in/out, FP64 register in/out); the arithmetic per node pair is a third.
#include "common.cuh"
#include "euler_fp64.cuh"
#include "kernels.h"
#include "mortar.cuh"
#include "repair64.cuh"

namespace nemo {

__constant__ OpConsts c_ops32;

namespace {

constexpr int EPC8 = 8;         // elements per CTA of the persistent kernel (the grid kernel takes 4, 8
                                // or 16 as a template parameter; the autotuner picks)
constexpr int TPE = 16;         // threads per element, one per line position (a,b): a warp holds
                                // exactly two elements
constexpr int V = 5;
constexpr int NQ = 6;           // FP32 node data: rho, vx, vy, vz, p, beta
// element stride of the FP32 shared-memory arrays (node data, rhs terms, epilogue scratch): the 6
// extra words move the second element of a warp onto other banks (fewer shared-memory conflicts
// in the line accesses; 2.4 % faster per stage than the unpadded 64 on B200)
constexpr int SP = NP + 6;

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

// Stage the tile's state into shared memory with 1D bulk copies (V arrays of nel*64 doubles,
// contiguous per variable), completing on the CTA's mbarrier (initialised once by mbar_init32; one
// phase per tile).  The RK register does not pass through shared memory: the update reads and
// writes it straight from global memory with coalesced accesses, after an L2 prefetch issued here.
template <int EPC>
__device__ __forceinline__ void tile_issue32(double* su, const double* __restrict__ u,
                                             const double* __restrict__ reg, int64_t E, int64_t e0, int nel,
                                             uint64_t* bar) {
    if (threadIdx.x == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        const unsigned bytes = (unsigned)(nel * NP * 8);
        const unsigned b0 = smem_u32(bar);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b0), "r"(bytes * V) : "memory");
        for (int v = 0; v < V; ++v) {
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smem_u32(su + v * EPC * NP)),
                "l"(u + ((int64_t)v * E + e0) * NP), "r"(bytes), "r"(b0)
                : "memory");
        }
        if (reg)
            for (int v = 0; v < V; ++v)
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(reg + ((int64_t)v * E + e0) * NP),
                             "r"(bytes)
                             : "memory");
    }
}

__device__ __forceinline__ bool tile_wait32(uint64_t* bar, unsigned phase, Control* ctrl) {
    bool ok = mbar_wait32(bar, phase);
    if (!ok) {
        atomicOr(&ctrl->error, 1);
        mbar_wait32(bar, phase);  // second bounded wait for the copies still in flight
    }
    return ok;
}

// Write the tile's new state back with 1D bulk copies from shared memory.  The calling thread waits
// until the copies have read shared memory before the CTA may reuse or leave it.
template <int EPC>
__device__ __forceinline__ void tile_store32(const double* su, double* __restrict__ u_out, int64_t E, int64_t e0,
                                             int nel) {
    const unsigned bytes = (unsigned)(nel * NP * 8);
    for (int v = 0; v < V; ++v)
        asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(u_out + ((int64_t)v * E + e0) * NP),
                     "r"(smem_u32(su + v * EPC * NP)), "r"(bytes)
                     : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

__device__ __forceinline__ void tile_store_wait32() {
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// 1/x in FP64 from the approximate FP32 reciprocal (about 1 ulp of FP32) by two Newton steps
// (relative error ~1e-16 for the positive, normal densities it is used on; the FP32 form needs no
// correctly rounded division here).  The correctly rounded FP32 seed was 0.5-1 % slower per stage.
__device__ __forceinline__ double rcp64(double x) {
    double y = (double)(1.0f / (float)x);   // the approximate FP32 reciprocal (fast-math) as the seed
    y = y * fma(-x, y, 2.0);
    return y * fma(-x, y, 2.0);
}

// Admissibility screen without a division: rho > 0 and rho E > |m|^2 / 2 (same sign as the
// pressure for rho > 0), with a small relative margin so borderline nodes go to the exact check.
__device__ __forceinline__ bool admissible_screen(const double* q) {
    return q[0] > 0.0 && q[0] * q[4] > 0.5 * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]) * (1.0 + 1e-12);
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
    const float kappa = k.kappa32;
    const float beta = k.hllc_beta32;
    const float km1 = k.km1_32;
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
    // the supersonic cases (SL >= 0: left flux, SR <= 0: right flux) by selection, not by early
    // returns: without branches the Riemann fluxes of a line are one straight-line block that the
    // compiler can interleave (the discarded intermediate values may be inf or NaN)
    const bool supL = SL >= 0.0f, supR = SR <= 0.0f;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        const float FH = (SR * FL[v] - SL * FR[v] + SL * SR * (UR[v] - UL[v])) * idS;
        const float Fu = left ? FL[v] : FR[v];
        const float Uu = left ? UL[v] : UR[v];
        const float Fm = smooth * FH + oms * (Fu + S * (Us[v] - Uu));
        F[v] = supL ? FL[v] : (supR ? FR[v] : Fm);
    }
}

// Rusanov (source/equations/euler/riemann/rusanov/riemann_mod.f90:7-24) in FP32.
__device__ __forceinline__ void rusanov32(const P32& L, const P32& R, float* F, const OpConsts& k) {
    const float kappa = k.kappa32;
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

// The specialised form (FAST) has its flux choices fixed at compile time: HLLC at the faces and in the
// subcells, the Chandrashekar pair, the modal indicator.  A run-time switch inside the unrolled line
// loops is a branch around every flux, which keeps the compiler from interleaving independent
// fluxes; the specialised kernel is 5-7 % faster per stage on B200 with bit-identical results.
template <bool FAST>
__device__ __forceinline__ void riem32(int kind, const P32& L, const P32& R, float* F, const OpConsts& k) {
    if (FAST) hllc32(L, R, F, k);
    else riemann32(kind, L, R, F, k);
}

// g(a, b) = atanh(f)/f for f = (a-b)/(a+b) (rs = 1/(a+b)), so that the logarithmic mean
// (a-b)/log(a/b) is (a+b)/(2g) and its inverse 2g/(a+b): the series 1 + u/3 + u^2/5 + u^3/7
// (u = f^2) below u = 1e-2 (Ismail-Roe), else log(a/b)/(2f).  Written this way the Chandrashekar
// pair needs three divisions instead of seven.  The log is computed to about 2e-7 relative from
// the exponent and a 5-term atanh series of the mantissa: the hardware approximation (__logf, up
// to 5e-7 relative for ratios near 2, the density jump of a shear layer) left the FP32 form at
// 1.03e-6 rel. L1 density against FP64 on the batched forest workload, this one at 9.7e-7, for 3 %
// more time per stage.
__device__ __forceinline__ float lngain32(float a, float b, float rs) {
    const float f = (a - b) * rs;
    const float u = f * f;
    if (u < 1e-2f) return 1.0f + u * (1.0f / 3.0f + u * (0.2f + u * (1.0f / 7.0f)));
    // log(a/b) = e ln2 + 2 atanh(t), t = (m-1)/(m+1) for the mantissa m in [1/sqrt2, sqrt2)
    const int bits = __float_as_int(a / b);
    int ex = ((bits >> 23) & 0xff) - 127;
    float m = __int_as_float((bits & 0x007fffff) | 0x3f800000);
    if (m > 1.41421356f) {
        m = 0.5f * m;
        ex += 1;
    }
    const float t = (m - 1.0f) / (m + 1.0f), t2 = t * t;
    const float lg = (float)ex * 0.69314718f +
                     2.0f * t * (1.0f + t2 * (1.0f / 3.0f + t2 * (0.2f + t2 * (1.0f / 7.0f + t2 * (1.0f / 9.0f)))));
    return 0.5f * lg / f;
}

// Epilogue on a state held in smem (FP64): the blending coefficient for the next stage (modal
// indicator, or the learned indicator with the modal one as fallback and judge) and, if requested,
// the per-element CFL bound.  16 threads per element; thread (a,b) starts from its x-line nodes.
__device__ __forceinline__ float hsum16(float v) {
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float hmax16(float v) {
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float hmin16(float v) {
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Transposed all-reduce over the 16 lanes of an element: lane l returns the sum over the 16 lanes
// of v[l] (15 shuffles for 16 sums instead of 64).
__device__ __forceinline__ float tsum16(float (&v)[16], int l) {
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) {
        const bool up = (l & o) != 0;
#pragma unroll
        for (int i = 0; i < o; ++i) {
            const float send = up ? v[i] : v[i + o];
            const float keep = up ? v[i + o] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
    return v[0];
}

template <int EPC, bool FAST>
__device__ __forceinline__ void epilogue32(const StageArgs& a, const double* su, float* scratch, const float* sw,
                                           int el, int ab, int la, int lb, bool active, int64_t e,
                                           const OpConsts& k) {
    Control* ctrl = a.ctrl;
    const bool need_lam = a.epi_dt != 0;
    const bool learned_form = !FAST && a.mlp32 != nullptr;
    if (!a.alpha_out && !need_lam) return;
    __shared__ int s_fb[EPC];
    __shared__ float s_jd[EPC];
    __shared__ double s_dt[EPC], s_lm[EPC];
    __shared__ int s_gr[EPC];
    if (threadIdx.x < EPC) s_fb[threadIdx.x] = 0;
    float qr[NN], qp[NN];
    float lx = 0.f, ly = 0.f, lz = 0.f;
#pragma unroll
    for (int i = 0; i < NN; ++i) {
        qr[i] = 1.f;
        qp[i] = 1.f;
    }
    if (active) {
#pragma unroll
        for (int i = 0; i < NN; ++i) {
            const int n = nidx(i, la, lb);
            const double r = su[(0 * EPC + el) * NP + n];
            const double mx = su[(1 * EPC + el) * NP + n], my = su[(2 * EPC + el) * NP + n];
            const double mz = su[(3 * EPC + el) * NP + n], en = su[(4 * EPC + el) * NP + n];
            const double ir = rcp64(r);
            const double prd = k.km1 * (en - 0.5 * ir * (mx * mx + my * my + mz * mz));
            qr[i] = (float)r;
            qp[i] = (float)prd;
            if (need_lam) {
                const float c = sqrtf((float)(k.kappa * prd * ir));
                lx = fmaxf(lx, fabsf((float)(mx * ir)) + c);
                ly = fmaxf(ly, fabsf((float)(my * ir)) + c);
                lz = fmaxf(lz, fabsf((float)(mz * ir)) + c);
            }
        }
    }
    if (a.alpha_out) {
        const bool learned = learned_form;
        const bool want_feat = !FAST && (learned || a.feat_out != nullptr);
        // modal transforms of rho*p (and, for the features, rho and p) fused over the quantities:
        // x in registers, y and z through shared memory [3][EPC][64] each
        float* t1 = scratch;                 // [3][EPC][64]
        float* t2 = scratch + 3 * EPC * SP;  // [3][EPC][64]
        float tot[3] = {0.f, 0.f, 0.f}, cl1 = 0.f, cl2 = 0.f, Eo[2][6];
#pragma unroll
        for (int w = 0; w < 2; ++w)
#pragma unroll
            for (int i = 0; i < 6; ++i) Eo[w][i] = 0.f;
        const int nq = want_feat ? 3 : 1;   // rho*p, then rho and p
        if (active) {
            for (int w = 0; w < nq; ++w) {
#pragma unroll
                for (int o = 0; o < NN; ++o) {
                    float s = 0.f;
#pragma unroll
                    for (int i = 0; i < NN; ++i) {
                        const float qv = w == 0 ? qr[i] * qp[i] : (w == 1 ? qr[i] : qp[i]);
                        s += k.Vinv32[o * NN + i] * qv;
                    }
                    t1[(w * EPC + el) * SP + nidx(o, la, lb)] = s;
                }
            }
        }
        __syncwarp();   // the element's 16 threads share one warp
        if (active) {
            for (int w = 0; w < nq; ++w) {
#pragma unroll
                for (int o = 0; o < NN; ++o) {
                    float s = 0.f;
#pragma unroll
                    for (int j = 0; j < NN; ++j) s += k.Vinv32[o * NN + j] * t1[(w * EPC + el) * SP + nidx(la, j, lb)];
                    t2[(w * EPC + el) * SP + nidx(la, o, lb)] = s;
                }
            }
        }
        __syncwarp();   // the element's 16 threads share one warp
        if (active) {
            for (int w = 0; w < nq; ++w) {
#pragma unroll
                for (int o = 0; o < NN; ++o) {
                    float s = 0.f;
#pragma unroll
                    for (int kk = 0; kk < NN; ++kk)
                        s += k.Vinv32[o * NN + kk] * t2[(w * EPC + el) * SP + nidx(la, lb, kk)];
                    const float e2 = s * s;
                    tot[w] += e2;
                    if (w == 0) {
                        if (la < NN - 1 && lb < NN - 1 && o < NN - 1) cl1 += e2;
                        if (la < NN - 2 && lb < NN - 2 && o < NN - 2) cl2 += e2;
                    } else {
                        const int ord[3] = {la, lb, o};
#pragma unroll
                        for (int d = 0; d < 3; ++d) {
                            if (ord[d] == NN - 1) Eo[w - 1][2 * d] += e2;
                            if (ord[d] == NN - 2) Eo[w - 1][2 * d + 1] += e2;
                        }
                    }
                }
            }
        }
        const float t0 = hsum16(tot[0]), c1 = hsum16(cl1), c2 = hsum16(cl2);
        float am;
        {
            const float energy = fmaxf((t0 - c1) / t0, (c1 - c2) / c1);
            float al = 1.0f / (1.0f + __expf(k.ind_k32 * (energy - k.ind_T32)));
            if (al < k.alpha_min32) al = 0.0f;
            else if (al > k.one_m_alpha_min32) al = 1.0f;
            am = fminf(k.alpha_max32, al);
        }
        float alpha = am;
        if (!FAST && a.feat_out) {
#pragma unroll
            for (int w = 0; w < 2; ++w) {
                const float tw = hsum16(tot[1 + w]);
#pragma unroll
                for (int i = 0; i < 6; ++i) {
                    const float f = __logf(hsum16(Eo[w][i]) / tw + 1e-12f);
                    if (active && ab == 0) a.feat_out[e * 12 + 6 * w + i] = f;
                }
            }
            if (active && ab == 0 && a.alpha_modal_out) a.alpha_modal_out[e] = (double)am;
        }
        if (learned) {
            // positivity-risk check and the 12 features: one transposed reduction over the 16 lanes
            // leaves lane i with the element total of quantity i (0..11 the order energies, 12/13
            // the rho and p energies, 14/15 the sums of rho and p), then each lane forms its feature
            float rs = 0.f, ps = 0.f, rmn = 3.4e38f, pmn = 3.4e38f;
#pragma unroll
            for (int i = 0; i < NN; ++i) {
                rs += qr[i];
                ps += qp[i];
                rmn = fminf(rmn, qr[i]);
                pmn = fminf(pmn, qp[i]);
            }
            float red[16];
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                red[i] = Eo[0][i];
                red[6 + i] = Eo[1][i];
            }
            red[12] = tot[1];
            red[13] = tot[2];
            red[14] = rs;
            red[15] = ps;
            const float mine = tsum16(red, ab);
            const float tq = __shfl_sync(0xffffffffu, mine, 12 + (ab >= 6 ? 1 : 0), 16);
            rs = __shfl_sync(0xffffffffu, mine, 14, 16);
            ps = __shfl_sync(0xffffffffu, mine, 15, 16);
            rmn = hmin16(rmn);
            pmn = hmin16(pmn);
            const float lo = sw[MLP_NW + (ab < 12 ? ab : 0)], hi = sw[MLP_NW + 12 + (ab < 12 ? ab : 0)];
            const float xm = __logf(mine / tq + 1e-12f) * 0.1f + 1.0f;
            const bool out_of_bounds = ab < 12 && (xm < lo || xm > hi);
            // the vote runs in every lane of the warp (the two elements of a warp may differ in fb)
            const unsigned oob = __ballot_sync(0xffffffffu, out_of_bounds) & (0xffffu << (threadIdx.x & 16));
            const bool fb = rmn < 0.1f * (rs / 64.0f) || pmn < 0.1f * (ps / 64.0f) || oob != 0u;
            float x[12];
#pragma unroll
            for (int i = 0; i < 12; ++i) x[i] = __shfl_sync(0xffffffffu, xm, i, 16);
            // sw: W1 transposed [12][32], b1[32], W2 transposed [32][32], b2[32], W3[32], b3
            const float* W1T = sw;
            const float* b1 = W1T + 12 * 32;
            const float* W2T = b1 + 32;
            const float* b2 = W2T + 32 * 32;
            const float* W3 = b2 + 32;
            const int j0 = 2 * ab;
            float2 sacc = *reinterpret_cast<const float2*>(b1 + j0);
#pragma unroll
            for (int i = 0; i < 12; ++i) {
                const float2 wv = *reinterpret_cast<const float2*>(W1T + i * 32 + j0);
                sacc.x += wv.x * x[i];
                sacc.y += wv.y * x[i];
            }
            const float h0 = sacc.x / (1.0f + __expf(-sacc.x)), h1v = sacc.y / (1.0f + __expf(-sacc.y));
            float2 uacc = *reinterpret_cast<const float2*>(b2 + j0);
#pragma unroll
            for (int src = 0; src < 16; ++src) {
                const float he = __shfl_sync(0xffffffffu, h0, src, 16);
                const float ho = __shfl_sync(0xffffffffu, h1v, src, 16);
                const float2 we = *reinterpret_cast<const float2*>(W2T + (2 * src) * 32 + j0);
                const float2 wo = *reinterpret_cast<const float2*>(W2T + (2 * src + 1) * 32 + j0);
                uacc.x += we.x * he + wo.x * ho;
                uacc.y += we.y * he + wo.y * ho;
            }
            const float g0 = uacc.x / (1.0f + __expf(-uacc.x)), g1 = uacc.y / (1.0f + __expf(-uacc.y));
            const float z = hsum16(W3[j0] * g0 + W3[j0 + 1] * g1) + W3[32];
            float al = k.alpha_max32 / (1.0f + __expf(-z));
            if (al < k.alpha_min32) al = 0.0f;
            if (fb) {
                alpha = am;
                if (active && ab == 0) s_fb[el] = 1;
            } else {
                alpha = al;
                if (active && ab == 0) s_jd[el] = fabsf(al - am);
            }
        }
        if (active && ab == 0) a.alpha_out[e] = (double)alpha;
    }
    if (need_lam) {
        lx = hmax16(lx);
        ly = hmax16(ly);
        lz = hmax16(lz);
        if (active && ab == 0) {
            const double dte = fmin(fmin(a.delta[e * 3 + 0] / (double)lx, a.delta[e * 3 + 1] / (double)ly),
                                    a.delta[e * 3 + 2] / (double)lz);
            s_dt[el] = dte;
            s_lm[el] = (double)fmaxf(fmaxf(lx, ly), lz);
            s_gr[el] = a.group ? a.group[e] : 0;
        }
    }
    // one set of atomics per CTA instead of per element: the counters and minima are single
    // addresses that every element of the launch would otherwise hit
    if (!(a.alpha_out && learned_form) && !need_lam) return;   // thread 0 would have nothing to add
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nel = (int)min((int64_t)EPC, a.E_own - (e - el));
        if (a.alpha_out && learned_form) {
            unsigned long long nfb = 0, nj = 0;
            double js = 0.0;
            for (int i = 0; i < nel; ++i) {
                if (s_fb[i]) nfb += 1;
                else {
                    js += (double)s_jd[i];
                    nj += 1;
                }
            }
            if (nfb) atomicAdd(&ctrl->fallback, nfb);
            if (nj) {
                atomicAdd(&ctrl->judge_sum, js);
                atomicAdd(&ctrl->judge_n, nj);
            }
        }
        if (need_lam) {
            int g = s_gr[0];
            double dmin = s_dt[0], lmx = s_lm[0];
            for (int i = 1; i <= nel; ++i) {
                if (i == nel || s_gr[i] != g) {
                    atomicMin(&ctrl->dtmin_bits[g], (unsigned long long)__double_as_longlong(dmin));
                    atomicMax(&ctrl->lmax_bits[g], (unsigned long long)__double_as_longlong(lmx));
                    if (i == nel) break;
                    g = s_gr[i];
                    dmin = s_dt[i];
                    lmx = s_lm[i];
                } else {
                    dmin = fmin(dmin, s_dt[i]);
                    lmx = fmax(lmx, s_lm[i]);
                }
            }
        }
    }
}

}  // namespace

// Shared-memory carve-up of one CTA of the FP32 stage.
struct Smem32 {
    double* su;        // [V][EPC][64] FP64 state
    float* sq;         // [NQ][EPC][64] FP32 node data
    float* sR;         // [V][EPC][64] FP32 rhs terms
    uint64_t* bar;     // TMA completion barrier of the state (initialised once per CTA)
    float* s_alpha;    // [EPC]
    int* s_bad;        // [EPC]
    const float* s_w;  // learned indicator, transposed layout (shared memory, or global through L1)
};

template <int EPC>
__device__ __forceinline__ void load_mlp32(const StageArgs& a, float* s_w) {
    constexpr int NT = EPC * TPE;
    if (a.mlp32t) {  // visible to the epilogue after the barriers of the stage
        const float4* src = reinterpret_cast<const float4*>(a.mlp32t);
        float4* dst = reinterpret_cast<float4*>(s_w);
        for (int i = threadIdx.x; i < MLP_NT / 4; i += NT) dst[i] = __ldg(src + i);
    }
}

template <int EPC>
__device__ __forceinline__ Smem32 smem32(double* smem, uint64_t* bar, float* s_alpha, int* s_bad, const float* s_w) {
    Smem32 S;
    S.su = smem;
    S.sq = reinterpret_cast<float*>(S.su + V * EPC * NP);
    S.sR = S.sq + NQ * EPC * SP;
    S.bar = bar;
    S.s_alpha = s_alpha;
    S.s_bad = s_bad;
    S.s_w = s_w;
    return S;
}

// Acquire a mortar's flux rows: wait (bounded) until its flag carries this launch's epoch.
__device__ __forceinline__ void mortar_acquire(const uint32_t* flag, uint32_t epoch, Control* ctrl) {
    for (int it = 0; it < (1 << 20); ++it) {
        uint32_t v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(flag) : "memory");
        if (v == epoch) return;
        __nanosleep(64);
    }
    atomicOr(&ctrl->error, 4);
}

// The positivity repair runs for few elements: out of line, so that the stage kernel's hot code
// stays smaller (about 1 % per stage on B200).
__device__ __noinline__ bool repair_call32(double* su, int el, int ab, int epc) {
    if (epc == 4) return repair_elem16<4>(su, el, ab, c_ops32);
    if (epc == 16) return repair_elem16<16>(su, el, ab, c_ops32);
    return repair_elem16<8>(su, el, ab, c_ops32);
}

__device__ __forceinline__ void mbar_init32(uint64_t* bar) {
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
}

// One tile of EPC elements (tile index `tile`, TMA barrier parity `phase`): thread (a,b) of an
// element owns the x-, y- and z-lines through (a,b) and processes them one direction after the
// other, accumulating into one shared rhs array (x, then y, then z).  A warp holds two elements.
template <int EPC, bool BLEND, bool RHS_ONLY, bool PERSIST, bool FAST>
__device__ __forceinline__ void tile32(const StageArgs& a, const Smem32& S, int64_t tile, unsigned phase,
                                       uint32_t epoch) {
    const OpConsts& k = c_ops32;
    Control* ctrl = a.ctrl;
    double* su = S.su;
    float* sq = S.sq;
    float* sR = S.sR;
    float* s_alpha = S.s_alpha;
    int* s_bad = S.s_bad;
    const float* s_w = S.s_w;
    const int tid = threadIdx.x;
    const int64_t E = a.E;
    const int64_t e0 = a.E_begin + tile * EPC;
    const int nel = (int)min((int64_t)EPC, a.E_own - e0);

    // the tile's bulk copy first, so that it is in flight while the blending coefficients are read
    const bool load_reg = !RHS_ONLY && !a.prep_only && a.stage > 0;
    tile_issue32<EPC>(su, a.u_in, load_reg ? a.reg : nullptr, E, e0, nel, S.bar);
    if (tid < EPC) {
        s_bad[tid] = 0;
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
    // s_alpha and s_bad become visible at the barrier after the primitives: the coefficient loads
    // overlap the bulk copy and the primitives instead of holding the whole CTA (1.5 % per stage)
    if (!tile_wait32(S.bar, phase, ctrl)) return;

    const int el = tid >> 4, ab = tid & 15, la = ab & 3, lb = ab >> 2;
    const bool active = el < nel;
    const int64_t e = e0 + el;
    if (a.prep_only) {
        __syncthreads();
        epilogue32<EPC, FAST>(a, su, sq, s_w, el, ab, la, lb, active, e, k);
        return;
    }
    auto SQ = [&](int q, int elx, int n) -> float& { return sq[(q * EPC + elx) * SP + n]; };

    // per-node primitives of the thread's x-line nodes: recovered in FP64, stored in FP32
    if (active) {
#pragma unroll
        for (int i = 0; i < NN; ++i) {
            const int n = nidx(i, la, lb);
            const double r = su[(0 * EPC + el) * NP + n];
            const double mx = su[(1 * EPC + el) * NP + n], my = su[(2 * EPC + el) * NP + n];
            const double mz = su[(3 * EPC + el) * NP + n], en = su[(4 * EPC + el) * NP + n];
            const double ir = rcp64(r);
            const double vx = mx * ir, vy = my * ir, vz = mz * ir;
            const double pr = k.km1 * (en - 0.5 * (mx * vx + my * vy + mz * vz));
            const float rf = (float)r, pf = (float)pr;
            SQ(0, el, n) = rf;
            SQ(1, el, n) = (float)vx;
            SQ(2, el, n) = (float)vy;
            SQ(3, el, n) = (float)vz;
            SQ(4, el, n) = pf;
            SQ(5, el, n) = 0.5f * rf / pf;
        }
    }
    __syncthreads();   // the primitives of the tile, s_alpha and s_bad visible

    const float ikm1 = k.ikm1_32;
    const float c_enth = k.c_enth32;
    for (int d = 0; d < 3; ++d) {
        if (active) {
            const int c0 = d, c1 = (d + 1) % 3, c2 = (d + 2) % 3;
            int idx[NN];
            float rho[NN], vn[NN], w1[NN], w2[NN], pr[NN], bt[NN];
#pragma unroll
            for (int i = 0; i < NN; ++i) {
                const int n = line_node(d, la, lb, i);
                idx[i] = n;
                rho[i] = SQ(0, el, n);
                vn[i] = SQ(1 + c0, el, n);
                w1[i] = SQ(1 + c1, el, n);
                w2[i] = SQ(1 + c2, el, n);
                pr[i] = SQ(4, el, n);
                bt[i] = SQ(5, el, n);
            }
            auto prim = [&](int i) {
                P32 q;
                q.rho = rho[i];
                q.vn = vn[i];
                q.vt1 = w1[i];
                q.vt2 = w2[i];
                q.p = pr[i];
                q.E = pr[i] * ikm1 + 0.5f * rho[i] * (vn[i] * vn[i] + w1[i] * w1[i] + w2[i] * w2[i]);
                return q;
            };
            // ---- surface fluxes at both ends of the line
            float Fs[2][V];
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                const int f = 2 * d + side;
                const P32 qo = prim(side ? NN - 1 : 0);
                P32 qn = qo;
                const int32_t ne = a.nbr[e * 6 + f];
                if (ne <= -2) {  // 2:1 mortar face: flux row of the mortar kernel / task (FP64)
                    if (PERSIST) mortar_acquire(a.mflag + (-2 - ne) / 5, epoch, ctrl);
                    const double* mf = a.mflux + (int64_t)(-2 - ne) * V * NF + ab;
#pragma unroll
                    for (int v = 0; v < V; ++v) Fs[side][v] = (float)mf[v * NF];
                    continue;
                }
                if (ne >= 0) {
                    const int nn = line_node(d, la, lb, side ? 0 : NN - 1);
                    const int64_t nl = (int64_t)ne - e0;
                    if (nl >= 0 && nl < nel) {
                        const int nli = (int)nl;
                        qn.rho = SQ(0, nli, nn);
                        qn.vn = SQ(1 + c0, nli, nn);
                        qn.vt1 = SQ(1 + c1, nli, nn);
                        qn.vt2 = SQ(1 + c2, nli, nn);
                        qn.p = SQ(4, nli, nn);
                        qn.E = qn.p * ikm1 + 0.5f * qn.rho * (qn.vn * qn.vn + qn.vt1 * qn.vt1 + qn.vt2 * qn.vt2);
                    } else {
                        const double* g = a.u_in;   // out-of-tile trace: L2 only, each node read once per CTA
                        const double r = __ldcg(g + ((int64_t)0 * E + ne) * NP + nn);
                        const double m0 = __ldcg(g + ((int64_t)(1 + c0) * E + ne) * NP + nn);
                        const double m1 = __ldcg(g + ((int64_t)(1 + c1) * E + ne) * NP + nn);
                        const double m2 = __ldcg(g + ((int64_t)(1 + c2) * E + ne) * NP + nn);
                        const double en = __ldcg(g + ((int64_t)4 * E + ne) * NP + nn);
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
                if (side) riem32<FAST>(a.surface_flux, qo, qn, Fs[1], k);
                else riem32<FAST>(a.surface_flux, qn, qo, Fs[0], k);
            }
            // ---- volume: 6 node pairs of the line from registers
            float t[NN][V];
#pragma unroll
            for (int i = 0; i < NN; ++i)
#pragma unroll
                for (int v = 0; v < V; ++v) t[i][v] = 0.0f;
#pragma unroll
            for (int i = 0; i < NN - 1; ++i) {
#pragma unroll
                for (int m = i + 1; m < NN; ++m) {
                    float F[V];
                    if (!FAST && a.volume_flux == NEMO_VOLFLUX_CENTRAL) {
                        float fa[V], fb[V];
                        xflux32(prim(i), fa);
                        xflux32(prim(m), fb);
#pragma unroll
                        for (int v = 0; v < V; ++v) F[v] = 0.5f * (fa[v] + fb[v]);
                    } else {
                        // logarithmic means as (a+b)/(2g): dens = {rho}_ln, p^ = {rho}/(2{beta}),
                        // p^/dens = g_rho/(beta_i+beta_m), 1/{beta}_ln = 2 g_beta/(beta_i+beta_m)
                        const float srho = rho[i] + rho[m];
                        const float rsb = 1.0f / (bt[i] + bt[m]);
                        const float gr = lngain32(rho[i], rho[m], 1.0f / srho);
                        const float gb = lngain32(bt[i], bt[m], rsb);
                        const float dens = 0.5f * srho / gr;
                        const float velx = 0.5f * (vn[i] + vn[m]), vely = 0.5f * (w1[i] + w1[m]);
                        const float velz = 0.5f * (w2[i] + w2[m]);
                        const float pres = 0.5f * srho * rsb;
                        const float vsq = (vn[i] * vn[i] + w1[i] * w1[i] + w2[i] * w2[i]) +
                                          (vn[m] * vn[m] + w1[m] * w1[m] + w2[m] * w2[m]);
                        const float enth = (2.0f * c_enth * gb + gr) * rsb + velx * velx + vely * vely + velz * velz -
                                           0.25f * vsq;
                        F[0] = dens * velx;
                        F[1] = F[0] * velx + pres;
                        F[2] = F[0] * vely;
                        F[3] = F[0] * velz;
                        F[4] = F[0] * enth;
                    }
                    const float sim = k.S32[i * NN + m], smi = k.S32[m * NN + i];
#pragma unroll
                    for (int v = 0; v < V; ++v) {
                        t[i][v] += sim * F[v];
                        t[m][v] += smi * F[v];
                    }
                }
            }
            // ---- lift
            const float w0 = k.winv32[0], w3 = k.winv32[NN - 1];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                t[0][v] -= w0 * Fs[0][v];
                t[NN - 1][v] += w3 * Fs[1][v];
            }
            // ---- FV subcells and the convex blend
            if (BLEND) {
                const float al = s_alpha[el];
                if (al > 0.0f) {
                    float Fl[V], Fr[V];
#pragma unroll
                    for (int v = 0; v < V; ++v) Fl[v] = Fs[0][v];
#pragma unroll
                    for (int i = 0; i < NN; ++i) {
                        if (i < NN - 1) {
                            riem32<FAST>(a.surface_flux, prim(i), prim(i + 1), Fr, k);
                        } else {
#pragma unroll
                            for (int v = 0; v < V; ++v) Fr[v] = Fs[1][v];
                        }
                        const float wi = k.winv32[i];
#pragma unroll
                        for (int v = 0; v < V; ++v) {
                            t[i][v] = (1.0f - al) * t[i][v] + al * (wi * (Fr[v] - Fl[v]));
                            Fl[v] = Fr[v];
                        }
                    }
                }
            }
            // ---- accumulate c_d * t into the element's rhs terms (x writes, y and z add)
            const float cd = (float)a.cdel[e * 3 + d];
            const int vo[V] = {0, 1 + c0, 1 + c1, 1 + c2, 4};
#pragma unroll
            for (int i = 0; i < NN; ++i)
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    float& R = sR[(vo[v] * EPC + el) * SP + idx[i]];
                    R = (d == 0 ? 0.0f : R) + cd * t[i][v];
                }
        }
        __syncwarp();   // the element's 16 threads share one warp
    }

    // ---- FP64 register/state update: thread ab of an element takes nodes ab + 16 q, so the register
    // moves between global memory and registers in coalesced 128-byte rows
    const int st = a.stage;
    const double A = rk_a(st);
    const double cdt = a.group ? (active ? rk_c(st) * ctrl->dt[a.group[e]] : 0.0) : rk_c(st) * ctrl->dt[0];
    if (active) {
        // the thread's 20 register values are loaded before any is stored: interleaved with the
        // stores (which the compiler cannot prove to be other addresses) each load would wait for
        // the previous store, 20 L2 round trips in a row.  L2 only (prefetched there at the tile
        // start): L1 stays for the neighbour traces.
        double rg[4][V];
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int v = 0; v < V; ++v)
                rg[q][v] = (RHS_ONLY || st == 0) ? 0.0 : __ldcg(a.reg + ((int64_t)v * E + e) * NP + ab + 16 * q);
        bool ok = true;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int n = ab + 16 * q;
            double qv[V];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int s = (v * EPC + el) * NP + n;
                const double rhs = -(double)sR[(v * EPC + el) * SP + n];
                const int64_t g = ((int64_t)v * E + e) * NP + n;
                if (RHS_ONLY) {
                    a.rhs_out[g] = rhs;
                } else {
                    const double r2 = st == 0 ? rhs : A * rg[q][v] + rhs;
                    a.reg[g] = r2;
                    su[s] = su[s] + cdt * r2;
                }
                qv[v] = su[s];
            }
            if (!RHS_ONLY && a.positivity) ok = ok && admissible_screen(qv);   // exact check in the repair
        }
        if (!ok) s_bad[el] = 1;
    }
    if (RHS_ONLY) return;
    __syncwarp();   // the element's 16 threads share one warp
    if (a.positivity && active && s_bad[el]) {   // the element's 16 threads together
        const bool repaired = repair_call32(su, el, ab, EPC);
        if (!repaired && ab == 0) atomicAdd(&ctrl->nbad, 1ull);
    }
    if (k.cool) {   // source term after the stage, on the element's own nodes (after its repair)
        __syncwarp();
        if (active) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int n = ab + 16 * q;
                double qv[V];
#pragma unroll
                for (int v = 0; v < V; ++v) qv[v] = su[(v * EPC + el) * NP + n];
                su[(4 * EPC + el) * NP + n] = cooled_energy64(qv, k);
            }
        }
    }
    // make the generic-proxy writes of su visible to the bulk copies, then store the tile
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) tile_store32<EPC>(su, a.u_out, E, e0, nel);
    if (st == 4 && a.tick && tile == 0 && tid == 0) {
        for (int g = 0; g < ctrl->ngroups; ++g) ctrl->t[g] = ctrl->t[g] + ctrl->dt[g];
        ctrl->steps += 1;
    }

    epilogue32<EPC, FAST>(a, su, sq, s_w, el, ab, la, lb, active, e, k);
    if (tid == 0) tile_store_wait32();
}


template <int EPC, bool BLEND, bool RHS_ONLY, bool FAST>
__global__ void __launch_bounds__(EPC * TPE, 32 / EPC) k_stage_euler32(StageArgs a) {
    extern __shared__ __align__(128) double smem[];
    __shared__ uint64_t bar[1];
    __shared__ float s_alpha[EPC];
    __shared__ int s_bad[EPC];
    if (!RHS_ONLY && !a.prep_only && a.ctrl->done) return;
    // the learned indicator's weights are read through L1 by the epilogue (a CTA handles one tile:
    // a shared-memory copy of the 6 KB per CTA would cost more L2 reads than it saves)
    const Smem32 S = smem32<EPC>(smem, bar, s_alpha, s_bad, a.mlp32t);
    mbar_init32(bar);
    tile32<EPC, BLEND, RHS_ONLY, false, FAST>(a, S, (int64_t)blockIdx.x, 0u, 0u);
}

// Persistent form: gridDim.x CTAs (a multiple of the SM count) take tasks from a device counter --
// first the pairs of 2:1 mortars (their flux rows, published with the launch's epoch), then the
// element tiles in Morton order.  Tiles that meet a mortar face acquire its flag; every mortar task
// was taken before any tile task, by a running CTA that waits on nothing, so the waits end.  The
// last CTA to finish resets the counter and advances the epoch for the next launch.
template <bool BLEND, bool FAST>
__global__ void __launch_bounds__(EPC8 * TPE, 4) k_stage_euler32p(StageArgs a, MortarArgs ma) {
    constexpr int EPC = EPC8;
    extern __shared__ __align__(128) double smem[];
    __shared__ uint64_t bar[1];
    __shared__ float s_alpha[EPC];
    __shared__ int s_bad[EPC];
    __shared__ __align__(16) float s_w[MLP_NT];
    __shared__ uint32_t s_task;
    Control* ctrl = a.ctrl;
    if (ctrl->done) return;
    const uint32_t epoch = ctrl->epoch;
    ma.epoch = epoch;
    load_mlp32<EPC>(a, s_w);
    const Smem32 S = smem32<EPC>(smem, bar, s_alpha, s_bad, s_w);
    mbar_init32(bar);
    const int64_t ntiles = (a.E_own - a.E_begin + EPC - 1) / EPC;
    const int64_t npairs = (ma.nm + mortar::MPB - 1) / mortar::MPB;
    unsigned phase = 0;
    for (;;) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic smem writes before TMA
        __syncthreads();   // the previous task is finished with shared memory and s_task
        if (threadIdx.x == 0) s_task = atomicAdd(&ctrl->work, 1u);
        __syncthreads();
        const int64_t task = s_task;
        if (task < npairs) {
            mortar::mortar_pair<false>(ma, task, smem, c_ops32);
            continue;
        }
        const int64_t tile = task - npairs;
        if (tile >= ntiles) break;
        tile32<EPC, BLEND, false, true, FAST>(a, S, tile, phase, epoch);
        phase ^= 1u;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned n = atomicAdd(&ctrl->exit_count, 1u);
        if (n == gridDim.x - 1) {
            ctrl->work = 0u;
            ctrl->exit_count = 0u;
            ctrl->epoch = epoch + 1u;
            __threadfence();
        }
    }
}

int stage_smem_bytes32(int epc) {
    return V * epc * NP * (int)sizeof(double) + (NQ + V) * epc * SP * (int)sizeof(float);
}

// The specialised kernel serves the configuration with HLLC faces, the Chandrashekar pair and the
// modal (or no) indicator without feature output; every other configuration takes the general one.
static bool fast_form(const StageArgs& a) {
    return a.surface_flux == NEMO_SURFFLUX_HLLC && a.volume_flux == NEMO_VOLFLUX_CHANDRASHEKAR && a.mlp32 == nullptr &&
           a.feat_out == nullptr;
}

template <int EPC>
static cudaError_t launch32(const StageArgs& a, bool blend, bool rhs_only, cudaStream_t s) {
    const int grid = (int)((a.E_own - a.E_begin + EPC - 1) / EPC);
    if (grid <= 0) return cudaSuccess;
    const int smem = stage_smem_bytes32(EPC), nt = EPC * TPE;
    if (rhs_only) {
        if (blend) k_stage_euler32<EPC, true, true, false><<<grid, nt, smem, s>>>(a);
        else k_stage_euler32<EPC, false, true, false><<<grid, nt, smem, s>>>(a);
    } else if (fast_form(a)) {
        if (blend) k_stage_euler32<EPC, true, false, true><<<grid, nt, smem, s>>>(a);
        else k_stage_euler32<EPC, false, false, true><<<grid, nt, smem, s>>>(a);
    } else {
        if (blend) k_stage_euler32<EPC, true, false, false><<<grid, nt, smem, s>>>(a);
        else k_stage_euler32<EPC, false, false, false><<<grid, nt, smem, s>>>(a);
    }
    return cudaGetLastError();
}

cudaError_t launch_stage_euler32(const StageArgs& a, bool blend, bool rhs_only, cudaStream_t s, int epc) {
    if (epc == 4) return launch32<4>(a, blend, rhs_only, s);
    if (epc == 16) return launch32<16>(a, blend, rhs_only, s);
    return launch32<8>(a, blend, rhs_only, s);
}

template <typename K>
static cudaError_t set_attrs32(K kernel, int smem) {
    cudaError_t err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (err != cudaSuccess) return err;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
}

cudaError_t launch_stage_euler32p(const StageArgs& a, const MortarArgs& ma, bool blend, int grid, cudaStream_t s) {
    const int smem = stage_smem_bytes32(EPC8);
    if (fast_form(a)) {
        if (blend) k_stage_euler32p<true, true><<<grid, EPC8 * TPE, smem, s>>>(a, ma);
        else k_stage_euler32p<false, true><<<grid, EPC8 * TPE, smem, s>>>(a, ma);
    } else {
        if (blend) k_stage_euler32p<true, false><<<grid, EPC8 * TPE, smem, s>>>(a, ma);
        else k_stage_euler32p<false, false><<<grid, EPC8 * TPE, smem, s>>>(a, ma);
    }
    return cudaGetLastError();
}

// CTAs per SM of the persistent kernel: the smaller of the general and the specialised form (the
// grid size is fixed before the configuration picks one of them)
cudaError_t stage32p_max_ctas_per_sm(bool blend, int* n) {
    const int smem = stage_smem_bytes32(EPC8);
    int n1 = 0, n2 = 0;
    cudaError_t err;
    if (blend) {
        if ((err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n1, k_stage_euler32p<true, false>, EPC8 * TPE, smem)))
            return err;
        err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n2, k_stage_euler32p<true, true>, EPC8 * TPE, smem);
    } else {
        if ((err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n1, k_stage_euler32p<false, false>, EPC8 * TPE, smem)))
            return err;
        err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n2, k_stage_euler32p<false, true>, EPC8 * TPE, smem);
    }
    *n = n1 < n2 ? n1 : n2;
    return err;
}

template <int EPC>
static cudaError_t setup32() {
    // the grid-schedule kernels leave the shared-memory carveout to the driver: it keeps 4 CTAs per
    // SM (8 elements per CTA) and more L1 than the largest carveout would (1 % faster per stage on B200)
    const auto dyn = cudaFuncAttributeMaxDynamicSharedMemorySize;
    const int smem = stage_smem_bytes32(EPC);
    cudaError_t err;
    if ((err = cudaFuncSetAttribute(k_stage_euler32<EPC, true, true, false>, dyn, smem)) != cudaSuccess) return err;
    if ((err = cudaFuncSetAttribute(k_stage_euler32<EPC, false, true, false>, dyn, smem)) != cudaSuccess) return err;
    if ((err = cudaFuncSetAttribute(k_stage_euler32<EPC, true, false, false>, dyn, smem)) != cudaSuccess) return err;
    if ((err = cudaFuncSetAttribute(k_stage_euler32<EPC, false, false, false>, dyn, smem)) != cudaSuccess) return err;
    if ((err = cudaFuncSetAttribute(k_stage_euler32<EPC, true, false, true>, dyn, smem)) != cudaSuccess) return err;
    return cudaFuncSetAttribute(k_stage_euler32<EPC, false, false, true>, dyn, smem);
}

cudaError_t setup_stage_euler32(const OpConsts& ops) {
    const int smem = stage_smem_bytes32(EPC8);
    cudaError_t err;
    if ((err = set_attrs32(k_stage_euler32p<true, false>, smem)) != cudaSuccess) return err;
    if ((err = set_attrs32(k_stage_euler32p<false, false>, smem)) != cudaSuccess) return err;
    if ((err = set_attrs32(k_stage_euler32p<true, true>, smem)) != cudaSuccess) return err;
    if ((err = set_attrs32(k_stage_euler32p<false, true>, smem)) != cudaSuccess) return err;
    if ((err = setup32<4>()) != cudaSuccess) return err;
    if ((err = setup32<8>()) != cudaSuccess) return err;
    if ((err = setup32<16>()) != cudaSuccess) return err;
    return cudaMemcpyToSymbol(c_ops32, &ops, sizeof(OpConsts));
}


// ---- GLM-MHD stage (float flux arithmetic)
#define NEMO_MHD_OPS c_ops32
}  // namespace nemo
#include "stage_mhd.cuh"
namespace nemo {
#undef NEMO_MHD_OPS

// state, rhs rows and the subcell interface fluxes of each thread's line
int stage_smem_bytes_mhd32() {
    return mhd::V * mhd::EPC * (NP * (int)sizeof(double) + mhd::SPM * (int)sizeof(float)) +
           (NN - 1) * mhd::V * mhd::NT * (int)sizeof(float);
}

cudaError_t setup_stage_mhd32() {
    const int smem = stage_smem_bytes_mhd32();
    cudaError_t err;
    const auto dyn = cudaFuncAttributeMaxDynamicSharedMemorySize;
    if ((err = cudaFuncSetAttribute(k_stage_mhd<float, true, true, false>, dyn, smem))) return err;
    if ((err = cudaFuncSetAttribute(k_stage_mhd<float, false, true, false>, dyn, smem))) return err;
    if ((err = cudaFuncSetAttribute(k_stage_mhd<float, true, false, false>, dyn, smem))) return err;
    if ((err = cudaFuncSetAttribute(k_stage_mhd<float, false, false, false>, dyn, smem))) return err;
    if ((err = cudaFuncSetAttribute(k_stage_mhd<float, true, false, true>, dyn, smem))) return err;
    return cudaFuncSetAttribute(k_stage_mhd<float, false, false, true>, dyn, smem);
}

cudaError_t launch_stage_mhd32(const StageArgs& a, bool blend, bool rhs_only, cudaStream_t s) {
    const int grid = (int)((a.E_own - a.E_begin + mhd::EPC - 1) / mhd::EPC);
    if (grid <= 0) return cudaSuccess;
    const int smem = stage_smem_bytes_mhd32();
    // the specialised kernel for HLLD faces and the EC pair flux, the general one for the rest
    const bool fast = a.surface_flux == NEMO_SURFFLUX_HLLD && a.volume_flux == NEMO_VOLFLUX_EC_MHD;
    if (rhs_only) {
        if (blend) k_stage_mhd<float, true, true, false><<<grid, mhd::NT, smem, s>>>(a);
        else k_stage_mhd<float, false, true, false><<<grid, mhd::NT, smem, s>>>(a);
    } else if (fast) {
        if (blend) k_stage_mhd<float, true, false, true><<<grid, mhd::NT, smem, s>>>(a);
        else k_stage_mhd<float, false, false, true><<<grid, mhd::NT, smem, s>>>(a);
    } else {
        if (blend) k_stage_mhd<float, true, false, false><<<grid, mhd::NT, smem, s>>>(a);
        else k_stage_mhd<float, false, false, false><<<grid, mhd::NT, smem, s>>>(a);
    }
    return cudaGetLastError();
}

}  // namespace nemo
