// stage_mhd.cuh -- fused LSRK stage for GLM-MHD (9 variables), templated on the flux arithmetic.
//
// Included by stage_fp64.cu (R = double, -fmad=false: bit-identical to the oracle) and by
// stage_fp32.cu (R = float, fast math; state, register, update, repair and reductions stay FP64).
// One CTA = EPC elements (8 for the FP32 form, 4 for the plain FP64 form), 16 threads per element;
// thread (a,b) owns the x-, y- and z-lines through (a,b) and adds its direction terms into one
// shared rhs array (x, then y, then z), which keeps the oracle's summation order.  Two kernels per
// form: a general one (flux kinds chosen at run time) and one specialised to HLLD + EC.  Per line:
// surface flux (HLLD or Rusanov) + the element's own-side
// non-conservative Powell/GLM term at both ends, 6 node pairs of EC flux (Derigs) + non-conservative
// term in flux-differencing form, the lift, and (alpha > 0) FV subcells with the same interface
// terms; then the GLM damping -glm_alpha psi, the RK register/state update (FP64) and the
// positivity repair.  The epilogue computes the blending coefficient for the next stage (modal
// indicator, or the learned one with the modal fallback) and, on the last stage, the CFL bound,
// the maximum wave speed and the maximum velocity for the GLM cleaning speed.
#pragma once

#include "common.cuh"
#include "kernels.h"
#include "mhd_phys.cuh"
#include "pmath64.cuh"
#include "repair64.cuh"

namespace nemo {
namespace mhd {

// Tile shape (compile-time knobs for tuning builds): elements per CTA (16 threads each) and, per
// form, the minimum number of resident CTAs per SM asked of the register allocator.
#ifndef NEMO_MHD_EPC
#define NEMO_MHD_EPC 8
#endif
#ifndef NEMO_MHD64_MINB
#define NEMO_MHD64_MINB 1
#endif
#ifndef NEMO_MHD32_MINB
#define NEMO_MHD32_MINB 3
#endif
constexpr int EPC = NEMO_MHD_EPC;
constexpr int NT = 16 * EPC;
constexpr int V = 9;
// element stride of the rhs array: 6 words of padding move the two elements of a warp onto
// different banks (as in the Euler FP32 stage; 0.7 % faster per FP32 stage at 64^3)
constexpr int SPM = NP + 6;

__device__ __forceinline__ unsigned su32(const void* p) { return static_cast<unsigned>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ bool mbar_wait_m(uint64_t* bar, unsigned phase) {
    const unsigned addr = su32(bar);
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

// The tile's bulk copy: issue (barrier set-up, thread 0 starts the copies), then, after other work,
// the wait.
__device__ __forceinline__ void tile_issue_m(double* su, const double* __restrict__ u, int64_t E, int64_t e0, int nel,
                                             uint64_t* bar) {
    if (threadIdx.x == 0) {
        const unsigned b = su32(bar);
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned b = su32(bar);
        const unsigned bytes = (unsigned)(nel * NP * 8);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes * V) : "memory");
        for (int v = 0; v < V; ++v)
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    su32(su + v * EPC * NP)),
                "l"(u + ((int64_t)v * E + e0) * NP), "r"(bytes), "r"(b)
                : "memory");
    }
}

__device__ __forceinline__ bool tile_wait_m(uint64_t* bar, Control* ctrl) {
    bool ok = mbar_wait_m(bar, 0);
    if (!ok) {
        atomicOr(&ctrl->error, 1);
        mbar_wait_m(bar, 0);
    }
    return ok;
}

// rotated state of node n of element el (momentum and field cyclically into direction d)
template <typename R>
__device__ __forceinline__ void load_rot(const double* su, int el, int n, int d, R* r) {
    r[0] = (R)su[(0 * EPC + el) * NP + n];
    r[4] = (R)su[(4 * EPC + el) * NP + n];
    r[8] = (R)su[(8 * EPC + el) * NP + n];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        r[1 + c] = (R)su[((1 + (d + c) % 3) * EPC + el) * NP + n];
        r[5 + c] = (R)su[((5 + (d + c) % 3) * EPC + el) * NP + n];
    }
}

// an out-of-tile neighbour's trace node, rotated into the frame of direction d (L2 only: each node
// is read once per CTA, so L1 is kept for the register rows)
template <typename R>
__device__ __forceinline__ void load_rot_global(const double* __restrict__ g, int64_t E, int64_t ne, int n, int d, R* r) {
    r[0] = (R)__ldcg(g + ((int64_t)0 * E + ne) * NP + n);
    r[4] = (R)__ldcg(g + ((int64_t)4 * E + ne) * NP + n);
    r[8] = (R)__ldcg(g + ((int64_t)8 * E + ne) * NP + n);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        r[1 + c] = (R)__ldcg(g + ((int64_t)(1 + (d + c) % 3) * E + ne) * NP + n);
        r[5 + c] = (R)__ldcg(g + ((int64_t)(5 + (d + c) % 3) * E + ne) * NP + n);
    }
}

// variable index of rotated component c in direction d
__device__ __forceinline__ int unrot(int d, int c) {
    if (c == 0 || c == 4 || c == 8) return c;
    if (c < 4) return 1 + (d + c - 1) % 3;
    return 5 + (d + c - 5) % 3;
}

__device__ __forceinline__ float hsum16m(float v) {
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float hmin16m(float v) {
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ double silu_m(double x) { return x / (1.0 + pexp64(-x)); }
__device__ __forceinline__ float silu_m(float x) { return x / (1.0f + __expf(-x)); }
__device__ __forceinline__ double expneg(double x) { return pexp64(x); }
__device__ __forceinline__ float expneg(float x) { return __expf(x); }

// Epilogue: modal (or learned) blending coefficient of the state in su and the CFL bound; sums in
// the oracle's serial order (one thread per element), MLP layers over 32 threads per element.
template <typename R>
__device__ void epilogue_mhd(const StageArgs& a, const double* su, R* scr, unsigned long long (*s_lam)[3],
                             unsigned long long* s_vmax, int nel, int64_t e0, int tid, const OpConsts& k) {
    __shared__ R s_am[EPC];
    __shared__ int s_fb[EPC];
    Control* ctrl = a.ctrl;
    const R kap = (R)k.kappa, mu0 = (R)k.mu0;
    if (a.alpha_out) {
        const R* W = nullptr;
        if (sizeof(R) == 8) W = reinterpret_cast<const R*>(a.mlp64);
        else W = reinterpret_cast<const R*>(a.mlp32);
        const bool learned = W != nullptr;
        R* q = scr;
        R* t1 = scr + EPC * NP;
        R* t2 = scr + 2 * EPC * NP;
        const int nq = learned ? 3 : 1;
        for (int w = 0; w < nq; ++w) {
            R* cm = scr + (3 + w) * EPC * NP;
            for (int p = tid; p < nel * NP; p += NT) {
                const int pel = p / NP, n = p % NP;
                R uu[V];
#pragma unroll
                for (int v = 0; v < V; ++v) uu[v] = (R)su[(v * EPC + pel) * NP + n];
                const R pr = m_pressure(uu, kap, mu0);
                q[pel * NP + n] = w == 0 ? uu[0] * pr : (w == 1 ? uu[0] : pr);
            }
            __syncthreads();
            for (int p = tid; p < nel * NP; p += NT) {
                const int pel = p / NP, n = p % NP;
                const int ai = n % NN, j = (n / NN) % NN, kk = n / NF;
                R s = R(0.0);
#pragma unroll
                for (int i = 0; i < NN; ++i) s = s + op_Vinv<R>(k, ai * NN + i) * q[pel * NP + nidx(i, j, kk)];
                t1[pel * NP + n] = s;
            }
            __syncthreads();
            for (int p = tid; p < nel * NP; p += NT) {
                const int pel = p / NP, n = p % NP;
                const int ai = n % NN, bj = (n / NN) % NN, kk = n / NF;
                R s = R(0.0);
#pragma unroll
                for (int j = 0; j < NN; ++j) s = s + op_Vinv<R>(k, bj * NN + j) * t1[pel * NP + nidx(ai, j, kk)];
                t2[pel * NP + n] = s;
            }
            __syncthreads();
            for (int p = tid; p < nel * NP; p += NT) {
                const int pel = p / NP, n = p % NP;
                const int ai = n % NN, bj = (n / NN) % NN, cc = n / NF;
                R s = R(0.0);
#pragma unroll
                for (int kk = 0; kk < NN; ++kk) s = s + op_Vinv<R>(k, cc * NN + kk) * t2[pel * NP + nidx(ai, bj, kk)];
                cm[pel * NP + n] = s;
            }
            __syncthreads();
        }
        R* feat = q;
        if constexpr (sizeof(R) == 4) {
            // FP32 form: the element's 16 threads share the sums (modes / nodes lane + 16 q)
            const int pel = tid >> 4, lane = tid & 15;
            const bool act = pel < nel;
            float total = 0.f, clip1 = 0.f, clip2 = 0.f;
            if (act) {
                const float* m = scr + 3 * EPC * NP + pel * NP;
#pragma unroll
                for (int qq = 0; qq < 4; ++qq) {
                    const int n = lane + 16 * qq, ai = n & 3, bj = (n >> 2) & 3, cc = n >> 4;
                    const float e2 = m[n] * m[n];
                    total += e2;
                    if (ai < NN - 1 && bj < NN - 1 && cc < NN - 1) clip1 += e2;
                    if (ai < NN - 2 && bj < NN - 2 && cc < NN - 2) clip2 += e2;
                }
            }
            total = hsum16m(total);
            clip1 = hsum16m(clip1);
            clip2 = hsum16m(clip2);
            const float energy = fmaxf((total - clip1) / total, (clip1 - clip2) / clip1);
            float al = 1.0f / (1.0f + __expf((float)k.ind_k * (energy - (float)k.ind_T)));
            if (al < (float)k.alpha_min) al = 0.0f;
            else if (al > (float)k.one_m_alpha_min) al = 1.0f;
            if (act && lane == 0) s_am[pel] = fminf((float)k.alpha_max, al);
            bool fb = false;
            if (learned) {
                float rs = 0.f, ps = 0.f, rmin = 3.4e38f, pmin = 3.4e38f;
                if (act) {
#pragma unroll
                    for (int qq = 0; qq < 4; ++qq) {
                        const int n = lane + 16 * qq;
                        float uu[V];
#pragma unroll
                        for (int v = 0; v < V; ++v) uu[v] = (float)su[(v * EPC + pel) * NP + n];
                        const float pr = m_pressure(uu, kap, mu0);
                        rs += uu[0];
                        ps += pr;
                        rmin = fminf(rmin, uu[0]);
                        pmin = fminf(pmin, pr);
                    }
                }
                rs = hsum16m(rs);
                ps = hsum16m(ps);
                rmin = hmin16m(rmin);
                pmin = hmin16m(pmin);
                fb = rmin < 0.1f * (rs / 64.0f) || pmin < 0.1f * (ps / 64.0f);
                float xmine = 0.f;
#pragma unroll
                for (int w = 0; w < 2; ++w) {
                    float tot = 0.f, Eo[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                    if (act) {
                        const float* mw = scr + (4 + w) * EPC * NP + pel * NP;
#pragma unroll
                        for (int qq = 0; qq < 4; ++qq) {
                            const int n = lane + 16 * qq;
                            const int ord[3] = {n & 3, (n >> 2) & 3, n >> 4};
                            const float ee = mw[n] * mw[n];
                            tot += ee;
#pragma unroll
                            for (int d = 0; d < 3; ++d) {
                                if (ord[d] == NN - 1) Eo[2 * d] += ee;
                                if (ord[d] == NN - 2) Eo[2 * d + 1] += ee;
                            }
                        }
                    }
                    tot = hsum16m(tot);
#pragma unroll
                    for (int i = 0; i < 6; ++i) {
                        const float Ei = hsum16m(Eo[i]);
                        if (lane == 6 * w + i) xmine = __logf(Ei / tot + 1e-12f);
                    }
                }
                const bool mine_out = lane < 12 && act &&
                                      (xmine / 10.0f + 1.0f < W[MLP_NW + (lane < 12 ? lane : 0)] ||
                                       xmine / 10.0f + 1.0f > W[MLP_NW + 12 + (lane < 12 ? lane : 0)]);
                if (act && lane < 12) feat[pel * 12 + lane] = xmine;
                // the vote runs in every lane of the warp
                const unsigned oob = __ballot_sync(0xffffffffu, mine_out) & (0xffffu << (threadIdx.x & 16));
                fb = fb || oob != 0u;
            }
            if (act && lane == 0) s_fb[pel] = fb ? 1 : 0;
        } else {
            if (tid < nel) {
                const R* m = scr + 3 * EPC * NP + tid * NP;
                R total = R(0.0), clip1 = R(0.0), clip2 = R(0.0);
                for (int cc = 0; cc < NN; ++cc)
                    for (int bj = 0; bj < NN; ++bj)
                        for (int ai = 0; ai < NN; ++ai) {
                            const R mv = m[nidx(ai, bj, cc)];
                            const R e2 = mv * mv;
                            total = total + e2;
                            if (ai < NN - 1 && bj < NN - 1 && cc < NN - 1) clip1 = clip1 + e2;
                            if (ai < NN - 2 && bj < NN - 2 && cc < NN - 2) clip2 = clip2 + e2;
                        }
                const R e1 = (total - clip1) / total;
                const R e2 = (clip1 - clip2) / clip1;
                const R energy = fmax(e1, e2);
                R al = R(1.0) / (R(1.0) + expneg((R)k.ind_k * (energy - (R)k.ind_T)));
                if (al < (R)k.alpha_min) al = R(0.0);
                else if (al > (R)k.one_m_alpha_min) al = R(1.0);
                s_am[tid] = fmin((R)k.alpha_max, al);
                int fb = 0;
                if (learned) {
                    R rs = R(0.0), ps = R(0.0), rmin = R(1e30), pmin = R(1e30);
                    for (int n = 0; n < NP; ++n) {
                        R uu[V];
    #pragma unroll
                        for (int v = 0; v < V; ++v) uu[v] = (R)su[(v * EPC + tid) * NP + n];
                        const R pr = m_pressure(uu, kap, mu0);
                        rs = rs + uu[0];
                        ps = ps + pr;
                        rmin = fmin(rmin, uu[0]);
                        pmin = fmin(pmin, pr);
                    }
                    if (rmin < R(0.1) * (rs / R(64.0)) || pmin < R(0.1) * (ps / R(64.0))) fb = 1;
                    for (int w = 0; w < 2; ++w) {
                        const R* mw = scr + (4 + w) * EPC * NP + tid * NP;
                        R tot = R(0.0), Eo[6] = {R(0), R(0), R(0), R(0), R(0), R(0)};
                        for (int cc = 0; cc < NN; ++cc)
                            for (int bj = 0; bj < NN; ++bj)
                                for (int ai = 0; ai < NN; ++ai) {
                                    const R mv = mw[nidx(ai, bj, cc)];
                                    const R ee = mv * mv;
                                    tot = tot + ee;
                                    const int ord[3] = {ai, bj, cc};
    #pragma unroll
                                    for (int d = 0; d < 3; ++d) {
                                        if (ord[d] == NN - 1) Eo[2 * d] = Eo[2 * d] + ee;
                                        if (ord[d] == NN - 2) Eo[2 * d + 1] = Eo[2 * d + 1] + ee;
                                    }
                                }
                        for (int i = 0; i < 6; ++i) {
                            const R f = mlog(Eo[i] / tot + R(1e-12));
                            feat[tid * 12 + 6 * w + i] = f;
                            const R x = f / R(10.0) + R(1.0);
                            if (x < W[MLP_NW + 6 * w + i] || x > W[MLP_NW + 12 + 6 * w + i]) fb = 1;
                        }
                    }
                }
                s_fb[tid] = fb;
            }
        }
        __syncthreads();
        if (learned) {
            const R* W1 = W;
            const R* b1 = W1 + 32 * 12;
            const R* W2 = b1 + 32;
            const R* b2 = W2 + 32 * 32;
            const R* W3 = b2 + 32;
            R* h1 = t1;
            R* h2 = t2;
            for (int p = tid; p < nel * 32; p += NT) {
                const int pel = p / 32, j = p % 32;
                R s = b1[j];
                for (int i = 0; i < 12; ++i) s = s + W1[j * 12 + i] * (feat[pel * 12 + i] / R(10.0) + R(1.0));
                h1[pel * 32 + j] = silu_m(s);
            }
            __syncthreads();
            for (int p = tid; p < nel * 32; p += NT) {
                const int pel = p / 32, j = p % 32;
                R s = b2[j];
                for (int i = 0; i < 32; ++i) s = s + W2[j * 32 + i] * h1[pel * 32 + i];
                h2[pel * 32 + j] = silu_m(s);
            }
            __syncthreads();
            if (tid < nel) {
                R z = W3[32];
                for (int j = 0; j < 32; ++j) z = z + W3[j] * h2[tid * 32 + j];
                R al = (R)k.alpha_max / (R(1.0) + expneg(-z));
                if (al < (R)k.alpha_min) al = R(0.0);
                const R am = s_am[tid];
                if (s_fb[tid]) {
                    atomicAdd(&ctrl->fallback, 1ull);
                    al = am;
                } else {
                    atomicAdd(&ctrl->judge_sum, (double)fabs(al - am));
                    atomicAdd(&ctrl->judge_n, 1ull);
                }
                a.alpha_out[e0 + tid] = (double)al;
            }
        } else if (tid < nel) {
            a.alpha_out[e0 + tid] = (double)s_am[tid];
        }
    }
    if (a.epi_dt) {
        for (int p = tid; p < nel * NP; p += NT) {
            const int pel = p / NP, n = p % NP;
            double uu[V];
#pragma unroll
            for (int v = 0; v < V; ++v) uu[v] = su[(v * EPC + pel) * NP + n];
            double rr[V];
#pragma unroll
            for (int dd = 0; dd < 3; ++dd) {
                rr[0] = uu[0];
                rr[4] = uu[4];
                rr[8] = uu[8];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    rr[1 + c] = uu[1 + (dd + c) % 3];
                    rr[5 + c] = uu[5 + (dd + c) % 3];
                }
                const double lam = m_xlambda(rr, k.kappa, k.mu0);
                atomicMax(&s_lam[pel][dd], (unsigned long long)__double_as_longlong(lam));
            }
            const double vm = fmax(fmax(fabs(uu[1] / uu[0]), fabs(uu[2] / uu[0])), fabs(uu[3] / uu[0]));
            atomicMax(s_vmax, (unsigned long long)__double_as_longlong(vm));
        }
        __syncthreads();
        if (tid < nel) {
            const int64_t pe = e0 + tid;
            const double lf = __longlong_as_double((long long)s_lam[tid][0]);
            const double lg = __longlong_as_double((long long)s_lam[tid][1]);
            const double lh = __longlong_as_double((long long)s_lam[tid][2]);
            const double dte = fmin(fmin(a.delta[pe * 3 + 0] / lf, a.delta[pe * 3 + 1] / lg), a.delta[pe * 3 + 2] / lh);
            const int g = a.group ? a.group[pe] : 0;
            atomicMin(&ctrl->dtmin_bits[g], (unsigned long long)__double_as_longlong(dte));
            atomicMax(&ctrl->lmax_bits[g], (unsigned long long)__double_as_longlong(fmax(fmax(lf, lg), lh)));
        }
        if (tid == 0) atomicMax(&ctrl->vmax_bits, *s_vmax);
    }
}

}  // namespace mhd

// FP32 form: 3 CTAs per SM (168 registers, a few hundred bytes of spills; 2 % faster on B200 than
// 4 CTAs at 128 registers with twice the spills, and 2 CTAs without spills is 14 % slower);
// plain FP64: 1 CTA per SM with the full register file.  The conserved state is read per node pair
// from the FP64 tile: a shared-memory array of per-node FP32 primitives (20 KB more per CTA) made the
// pair fluxes cheaper but the stage 4 % slower, as the larger carveout left L1 too small for the
// neighbour traces and register rows.
template <typename R, bool BLEND, bool RHS_ONLY, bool FAST>
__global__ void __launch_bounds__(mhd::NT, sizeof(R) == 4 ? NEMO_MHD32_MINB : NEMO_MHD64_MINB) k_stage_mhd(StageArgs a) {
    constexpr int MEPC = mhd::EPC, MV = mhd::V;
    using mhd::load_rot;
    using mhd::load_rot_global;
    using mhd::unrot;
    extern __shared__ __align__(128) double smem_m[];
    double* su = smem_m;                                    // [9][MEPC][64] FP64 state
    R* sR = reinterpret_cast<R*>(su + MV * MEPC * NP);        // [9][MEPC][64] rhs terms
    R* sFh = sR + MV * MEPC * mhd::SPM;                        // [NN-1][9][NT] subcell interface fluxes
    __shared__ uint64_t bar;
    __shared__ R s_alpha[MEPC];
    __shared__ int s_bad[MEPC];
    __shared__ unsigned long long s_lam[MEPC][3];
    __shared__ unsigned long long s_vmax;

    const OpConsts& k = NEMO_MHD_OPS;
    Control* ctrl = a.ctrl;
    if (!RHS_ONLY && !a.prep_only && ctrl->done) return;
    const int tid = threadIdx.x;
    const int64_t E = a.E;
    const int64_t e0 = a.E_begin + (int64_t)blockIdx.x * MEPC;
    const int nel = (int)min((int64_t)MEPC, a.E_own - e0);
    const R kap = (R)k.kappa, mu0 = (R)k.mu0;
    const R ch = (R)ctrl->glm_ch;

    // the tile's bulk copy first, so that it is in flight while the blending coefficients are read
    mhd::tile_issue_m(su, a.u_in, E, e0, nel, &bar);
    // the first thread of each element reads its blending coefficient; the element's 16 threads
    // share a warp, so a warp sync makes it visible (no CTA barrier: the loads overlap the bulk copy)
    if ((tid & 15) == 0) {
        const int te = tid >> 4;
        s_bad[te] = 0;
        s_lam[te][0] = s_lam[te][1] = s_lam[te][2] = 0ull;
        R al = R(0.0);
        if (BLEND && te < nel) {
            const int64_t e = e0 + te;
            double ad = a.alpha_in[e];
            if (a.smooth)
                for (int f = 0; f < 6; ++f) {
                    const int32_t ne = a.nbr[e * 6 + f];
                    if (ne >= 0) ad = fmax(ad, 0.5 * a.alpha_in[ne]);
                }
            if (a.alpha_used) a.alpha_used[e] = ad;
            al = (R)ad;
        }
        s_alpha[te] = al;
    }
    if (tid == 0) s_vmax = 0ull;
    __syncwarp();   // s_alpha, s_bad of the warp's elements; s_lam and s_vmax are read after CTA barriers
    if (!mhd::tile_wait_m(&bar, ctrl)) return;
    if (a.prep_only) {
        __syncthreads();
        mhd::epilogue_mhd<R>(a, su, sR, s_lam, &s_vmax, nel, e0, tid, k);
        return;
    }

    const int el = tid >> 4, ab = tid & 15, la = ab & 3, lb = ab >> 2;
    const bool active = el < nel;
    const int64_t e = e0 + el;
    for (int d = 0; d < 3; ++d) {
        if (active) {
            int idx[NN];
#pragma unroll
            for (int i = 0; i < NN; ++i) idx[i] = line_node(d, la, lb, i);
            // ---- surface flux + own-side non-conservative term at both ends
            // the flux at one end: side 0 the face 2d (neighbour on the left), side 1 the face 2d+1
            auto side_flux = [&](const int side, R* Fo) {
                const int f = 2 * d + side;
                R uo[MV], un[MV], F[MV], G[MV];
                load_rot(su, el, line_node(d, la, lb, side ? NN - 1 : 0), d, uo);
                const int32_t ne = a.nbr[e * 6 + f];
                if (ne <= -2) {  // 2:1 mortar face: flux row (incl. the own-side NC term) of the mortar kernel
                    const double* mf = a.mflux + (int64_t)(-2 - ne) * MV * NF + ab;
#pragma unroll
                    for (int v = 0; v < MV; ++v) Fo[v] = (R)mf[v * NF];
                    return;
                }
                if (ne >= 0) {
                    const int nn = line_node(d, la, lb, side ? 0 : NN - 1);
                    const int64_t nl = (int64_t)ne - e0;
                    if (nl >= 0 && nl < nel) load_rot(su, (int)nl, nn, d, un);
                    else load_rot_global(a.u_in, E, ne, nn, d, un);
                } else {
#pragma unroll
                    for (int v = 0; v < MV; ++v) un[v] = uo[v];
                }
                R uL[MV], uR[MV];
#pragma unroll
                for (int v = 0; v < MV; ++v) {
                    uL[v] = side ? uo[v] : un[v];
                    uR[v] = side ? un[v] : uo[v];
                }
                m_riem<FAST>(a.surface_flux, uL, uR, F, kap, mu0, ch);
                m_nc_x(uo, uL, uR, G, mu0);
#pragma unroll
                for (int v = 0; v < MV; ++v) Fo[v] = F[v] + G[v];
            };
            R Fs[2][MV];
            if constexpr (sizeof(R) == 8) {
                // plain form: both ends in a rolled loop (one inlined Riemann solver instead of two: 9 %
                // per stage); the fluxes pass through the thread's subcell slots (free until the
                // subcell fluxes) into registers.  The FP32 form keeps both ends inlined (its rolled
                // loop was 0.4 % slower).
#pragma unroll 1
                for (int side = 0; side < 2; ++side) {
                    R Fo[MV];
                    side_flux(side, Fo);
#pragma unroll
                    for (int v = 0; v < MV; ++v) sFh[(side * MV + v) * mhd::NT + tid] = Fo[v];
                }
#pragma unroll
                for (int side = 0; side < 2; ++side)
#pragma unroll
                    for (int v = 0; v < MV; ++v) Fs[side][v] = sFh[(side * MV + v) * mhd::NT + tid];
            } else {
#pragma unroll
                for (int side = 0; side < 2; ++side) {
                    const int f = 2 * d + side;
                    R uo[MV], un[MV], F[MV], G[MV];
                    load_rot(su, el, idx[side ? NN - 1 : 0], d, uo);
                    const int32_t ne = a.nbr[e * 6 + f];
                    if (ne <= -2) {  // 2:1 mortar face: flux row (incl. the own-side NC term) of the mortar kernel
                        const double* mf = a.mflux + (int64_t)(-2 - ne) * MV * NF + ab;
#pragma unroll
                        for (int v = 0; v < MV; ++v) Fs[side][v] = (R)mf[v * NF];
                        continue;
                    }
                    if (ne >= 0) {
                        const int nn = line_node(d, la, lb, side ? 0 : NN - 1);
                        const int64_t nl = (int64_t)ne - e0;
                        if (nl >= 0 && nl < nel) load_rot(su, (int)nl, nn, d, un);
                        else load_rot_global(a.u_in, E, ne, nn, d, un);
                    } else {
#pragma unroll
                        for (int v = 0; v < MV; ++v) un[v] = uo[v];
                    }
                    if (side) {
                        m_riem<FAST>(a.surface_flux, uo, un, F, kap, mu0, ch);
                        m_nc_x(uo, uo, un, G, mu0);
                    } else {
                        m_riem<FAST>(a.surface_flux, un, uo, F, kap, mu0, ch);
                        m_nc_x(uo, un, uo, G, mu0);
                    }
#pragma unroll
                    for (int v = 0; v < MV; ++v) Fs[side][v] = F[v] + G[v];
                }
            }
            // ---- volume: EC flux + non-conservative term, 6 pairs in the oracle's order
            R t[NN][MV];
#pragma unroll
            for (int i = 0; i < NN; ++i)
#pragma unroll
                for (int v = 0; v < MV; ++v) t[i][v] = R(0.0);
#pragma unroll
            for (int i = 0; i < NN - 1; ++i)
#pragma unroll
                for (int m = i + 1; m < NN; ++m) {
                    R ui[MV], um[MV], F[MV], Gi[MV], Gm[MV];
                    load_rot(su, el, idx[i], d, ui);
                    load_rot(su, el, idx[m], d, um);
                    if (!FAST && a.volume_flux == NEMO_VOLFLUX_CENTRAL) m_central_x(ui, um, F, kap, mu0, ch);
                    else m_ec_x(ui, um, F, kap, mu0, ch);
                    m_nc_x(ui, ui, um, Gi, mu0);
                    m_nc_x(um, ui, um, Gm, mu0);
                    const R sim = op_S<R>(k, i * NN + m), smi = op_S<R>(k, m * NN + i);
#pragma unroll
                    for (int v = 0; v < MV; ++v) {
                        t[i][v] = t[i][v] + sim * (F[v] + Gi[v]);
                        t[m][v] = t[m][v] + smi * (F[v] + Gm[v]);
                    }
                }
            // ---- lift
#pragma unroll
            for (int v = 0; v < MV; ++v) {
                t[0][v] = t[0][v] + op_winv<R>(k, 0) * (-Fs[0][v]);
                t[NN - 1][v] = t[NN - 1][v] + op_winv<R>(k, NN - 1) * Fs[1][v];
            }
            // ---- FV subcells and blend
            if (BLEND) {
                const R al = s_alpha[el];
                if (al > R(0.0)) {
                    // the three interface Riemann fluxes in a rolled loop (one inlined solver instead of
                    // three: less code), kept in the thread's shared-memory slots
#pragma unroll 1
                    for (int q = 0; q < NN - 1; ++q) {
                        R uq[MV], ur[MV], Fq[MV];
                        load_rot(su, el, line_node(d, la, lb, q), d, uq);
                        load_rot(su, el, line_node(d, la, lb, q + 1), d, ur);
                        m_riem<FAST>(a.surface_flux, uq, ur, Fq, kap, mu0, ch);
#pragma unroll
                        for (int v = 0; v < MV; ++v) sFh[(q * MV + v) * mhd::NT + tid] = Fq[v];
                    }
#pragma unroll
                    for (int i = 0; i < NN; ++i) {
                        R ui[MV], FR[MV], FL[MV], G[MV];
                        load_rot(su, el, idx[i], d, ui);
                        if (i > 0) {
                            R ul[MV];
                            load_rot(su, el, idx[i - 1], d, ul);
                            m_nc_x(ui, ul, ui, G, mu0);
#pragma unroll
                            for (int v = 0; v < MV; ++v) FL[v] = sFh[((i - 1) * MV + v) * mhd::NT + tid] + G[v];
                        } else {
#pragma unroll
                            for (int v = 0; v < MV; ++v) FL[v] = Fs[0][v];
                        }
                        if (i < NN - 1) {
                            R ur[MV];
                            load_rot(su, el, idx[i + 1], d, ur);
                            m_nc_x(ui, ui, ur, G, mu0);
#pragma unroll
                            for (int v = 0; v < MV; ++v) FR[v] = sFh[(i * MV + v) * mhd::NT + tid] + G[v];
                        } else {
#pragma unroll
                            for (int v = 0; v < MV; ++v) FR[v] = Fs[1][v];
                        }
                        const R wi = op_winv<R>(k, i);
#pragma unroll
                        for (int v = 0; v < MV; ++v) t[i][v] = (R(1.0) - al) * t[i][v] + al * (wi * (FR[v] - FL[v]));
                    }
                }
            }
            // ---- accumulate c_d * t (x writes, y and z add)
            const R cd = (R)a.cdel[e * 3 + d];
#pragma unroll
            for (int i = 0; i < NN; ++i)
#pragma unroll
                for (int c = 0; c < MV; ++c) {
                    R& Rv = sR[(unrot(d, c) * MEPC + el) * mhd::SPM + idx[i]];
                    Rv = (d == 0 ? cd * t[i][c] : Rv + cd * t[i][c]);
                }
        }
        __syncthreads();
    }

    // ---- FP64 register/state update and GLM damping
    const int st = a.stage;
    const double A = rk_a(st);
    const double cdt = rk_c(st) * ctrl->dt[0];
    const double galpha = ctrl->glm_alpha;
    if (active) {
        bool ok = true;
#pragma unroll
        for (int i = 0; i < NN; ++i) {
            const int n = nidx(i, la, lb);
            double uu[MV];
            // the node's register values are loaded before any is stored (interleaved, each load
            // would wait for the previous store); the FP32 form reads them from L2 only (0.7 %
            // faster; the FP64 form is not)
            double rgv[MV];
#pragma unroll
            for (int v = 0; v < MV; ++v) {
                const int64_t g = ((int64_t)v * E + e) * NP + n;
                rgv[v] = (RHS_ONLY || st == 0) ? 0.0 : (sizeof(R) == 4 ? __ldcg(a.reg + g) : a.reg[g]);
            }
#pragma unroll
            for (int v = 0; v < MV; ++v) {
                const int s = (v * MEPC + el) * NP + n;
                double rhs = -(double)sR[(v * MEPC + el) * mhd::SPM + n];
                if (v == 8) rhs = rhs - galpha * su[s];
                const int64_t g = ((int64_t)v * E + e) * NP + n;
                if (RHS_ONLY) {
                    a.rhs_out[g] = rhs;
                } else {
                    const double rg = rgv[v];
                    const double r2 = st == 0 ? rhs : A * rg + rhs;
                    a.reg[g] = r2;
                    su[s] = su[s] + cdt * r2;
                }
                uu[v] = su[s];
            }
            if (!RHS_ONLY && a.positivity) ok = ok && m_isvalid(uu, k.kappa, k.mu0);
        }
        if (!ok) s_bad[el] = 1;
    }
    if (RHS_ONLY) return;
    __syncthreads();
    if (a.positivity && active && s_bad[el]) {
        if constexpr (sizeof(R) == 4) {   // FP32 form: the element's 16 threads (a half-warp) together
            const bool repaired = repair_elem16_mhd<mhd::EPC>(su, el, ab, k);
            if (!repaired && ab == 0) atomicAdd(&ctrl->nbad, 1ull);
        } else if (ab == 0) {             // plain form: one thread (register budget of the FP64 kernel)
            if (!repair_elem_mhd<mhd::EPC>(su, el, k)) atomicAdd(&ctrl->nbad, 1ull);
        }
    }
    __syncthreads();
    if (active) {
#pragma unroll
        for (int v = 0; v < MV; ++v)
#pragma unroll
            for (int i = 0; i < NN; ++i) {
                const int n = nidx(i, la, lb);
                a.u_out[((int64_t)v * E + e) * NP + n] = su[(v * MEPC + el) * NP + n];
            }
    }
    if (st == 4 && a.tick && blockIdx.x == 0 && tid == 0) {
        for (int g = 0; g < ctrl->ngroups; ++g) ctrl->t[g] = ctrl->t[g] + ctrl->dt[g];
        ctrl->steps += 1;
    }
    __syncthreads();
    mhd::epilogue_mhd<R>(a, su, sR, s_lam, &s_vmax, nel, e0, tid, k);
}

}  // namespace nemo
