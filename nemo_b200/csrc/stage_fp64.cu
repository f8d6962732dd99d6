// stage_fp64.cu -- plain FP64 path: one fused kernel per LSRK stage (compiled with -fmad=false).
//
// One CTA owns EPC = 4 consecutive elements (a 2x2x1 block on a Morton-ordered brick) and runs
// 48 threads per element, one per (direction d, line (a,b)).  Per stage and element it does what
// the reference spreads over hook_pre_rk_timestep_300 and hook_mid_rk_timestep_500:
//   1. TMA bulk copy (cp.async.bulk, mbarrier) of the 8 elements' SoA state into shared memory;
//   2. per-node primitives (velocities, beta_d = rho/(2 p_d) per direction);
//   3. the two face fluxes at the ends of the thread's line (kernel_fill_faceflux,
//      source/kernel/mcfv/3d/kernel_flux_mod.f90:47-278; neighbour traces from shared memory
//      when the neighbour is in the CTA, else from global memory);
//   4. split-form flux differencing along the line, 6 node pairs in a fixed order, plus the
//      surface lift, plus (alpha > 0) first-order FV subcells and the convex blend;
//   5. the LSRK 5-4 register/state update (timedisc_probe, source/timedisc/rungekutta/
//      low-storage/4-5/timedisc_probe_mod.f90:7-39; rkstep_cb :19-49);
//   6. the positivity repair (dgfv_repair_3d, source/kernel/mcfv/3d/kernel_validate_mod.f90:159-272);
//   7. epilogue on the new state: the modal indicator for the next stage and, on the last
//      stage, the per-element CFL bound for the next time step (kernel_timestep_mod.f90:348-394).
// The arithmetic follows oracle/nemo_oracle.cpp expression by expression, so the two agree to
// the last bit except where log/exp enter.
#include "common.cuh"
#include "euler_fp64.cuh"
#include "kernels.h"
#include "repair64.cuh"

namespace nemo {

__constant__ OpConsts c_ops64;

namespace {

// Tile shape (compile-time knobs for tuning builds): elements per CTA and the minimum number of
// resident CTAs per SM that __launch_bounds__ asks the register allocator for.  Measured on B200
// (Sedov 32^3, plain FP64 stage, bit-identical results in every case): 8 elements x 1 CTA/SM at 168
// registers 0.890 ms; 4 x 3 CTAs/SM at 96 registers 0.735 ms; 2 x 6 at 96 registers 0.764 ms;
// 2 x 5 0.784 ms.  Three independent 192-thread CTAs per SM overlap one another's tile loads,
// barriers and epilogues, which one 384-thread CTA cannot (barrier stalls were 2.0 per issue).
#ifndef NEMO_FP64_EPC
#define NEMO_FP64_EPC 4
#endif
#ifndef NEMO_FP64_MINB
#define NEMO_FP64_MINB 3
#endif
constexpr int EPC = NEMO_FP64_EPC;   // elements per CTA
constexpr int TPE = 48;              // threads per element
constexpr int NT = EPC * TPE;        // 192 threads at 4 elements per CTA
constexpr int V = 5;
static_assert(NT / 32 >= EPC, "the repair runs one element per warp");

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

// Bounded wait on an mbarrier phase; returns false if the bound expired.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned phase) {
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

// Stage the tile's state (V arrays of nel*64 doubles, contiguous per variable) into smem: the issue
// (barrier set-up, then thread 0 starts the bulk copies) and, after other work, the wait.
__device__ __forceinline__ void tile_issue(double* su, const double* __restrict__ u, int64_t E, int64_t e0, int nel,
                                          uint64_t* bar) {
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
}

__device__ __forceinline__ bool tile_wait(uint64_t* bar, Control* ctrl) {
    bool ok = mbar_wait(bar, 0);
    if (!ok) {
        atomicOr(&ctrl->error, 1);
        mbar_wait(bar, 0);  // second bounded wait for the copies still in flight
    }
    return ok;
}


// Epilogue on a state held in smem (the new state of a stage, or the uploaded state of a prepare
// launch): the blending coefficient for the next stage (modal indicator, or learned indicator with
// the modal one as fallback and judge) and, if requested, the per-element CFL bound.
__device__ __forceinline__ double silu64(double x) { return x / (1.0 + pexp64(-x)); }

__device__ void epilogue64(const StageArgs& a, const double* su, double* sp, unsigned long long (*s_lam)[3],
                           int nel, int64_t e0, int tid, const OpConsts& k) {
    __shared__ double s_am[EPC];
    __shared__ int s_fb[EPC];
    Control* ctrl = a.ctrl;
    const int64_t E = a.E;
    (void)E;
    if (a.alpha_out) {
        const bool learned = a.mlp64 != nullptr;
        double* q = sp;
        double* t1 = sp + EPC * NP;
        double* t2 = sp + 2 * EPC * NP;
        const int nq = learned ? 3 : 1;   // modal coefficients of rho*p, then rho and p
        for (int w = 0; w < nq; ++w) {
            double* cm = sp + (3 + w) * EPC * NP;
            for (int p = tid; p < nel * NP; p += NT) {
                const int pel = p / NP, n = p % NP;
                double uu[V];
#pragma unroll
                for (int v = 0; v < V; ++v) uu[v] = su[(v * EPC + pel) * NP + n];
                q[pel * NP + n] = w == 0 ? uu[0] * pressure64(uu, k) : (w == 1 ? uu[0] : pressure64(uu, k));
            }
            __syncthreads();
            for (int p = tid; p < nel * NP; p += NT) {
                const int pel = p / NP, n = p % NP;
                const int ai = n % NN, j = (n / NN) % NN, kk = n / NF;
                double s = 0.0;
#pragma unroll
                for (int i = 0; i < NN; ++i) s = s + k.Vinv[ai * NN + i] * q[pel * NP + nidx(i, j, kk)];
                t1[pel * NP + n] = s;
            }
            __syncthreads();
            for (int p = tid; p < nel * NP; p += NT) {
                const int pel = p / NP, n = p % NP;
                const int ai = n % NN, bj = (n / NN) % NN, kk = n / NF;
                double s = 0.0;
#pragma unroll
                for (int j = 0; j < NN; ++j) s = s + k.Vinv[bj * NN + j] * t1[pel * NP + nidx(ai, j, kk)];
                t2[pel * NP + n] = s;
            }
            __syncthreads();
            for (int p = tid; p < nel * NP; p += NT) {
                const int pel = p / NP, n = p % NP;
                const int ai = n % NN, bj = (n / NN) % NN, cc = n / NF;
                double s = 0.0;
#pragma unroll
                for (int kk = 0; kk < NN; ++kk) s = s + k.Vinv[cc * NN + kk] * t2[pel * NP + nidx(ai, bj, kk)];
                cm[pel * NP + n] = s;
            }
            __syncthreads();
        }
        double* feat = q;   // [EPC][12], the nodal scratch is dead now
        if (tid < nel) {
            const double* m = sp + 3 * EPC * NP + tid * NP;
            double total = 0.0, clip1 = 0.0, clip2 = 0.0;
            for (int cc = 0; cc < NN; ++cc)
                for (int bj = 0; bj < NN; ++bj)
                    for (int ai = 0; ai < NN; ++ai) {
                        const double mv = m[nidx(ai, bj, cc)];
                        const double e2 = mv * mv;
                        total = total + e2;
                        if (ai < NN - 1 && bj < NN - 1 && cc < NN - 1) clip1 = clip1 + e2;
                        if (ai < NN - 2 && bj < NN - 2 && cc < NN - 2) clip2 = clip2 + e2;
                    }
            const double e1 = (total - clip1) / total;
            const double e2 = (clip1 - clip2) / clip1;
            const double energy = fmax(e1, e2);
            double al = 1.0 / (1.0 + pexp64(k.ind_k * (energy - k.ind_T)));
            if (al < k.alpha_min) al = 0.0;
            else if (al > k.one_m_alpha_min) al = 1.0;
            s_am[tid] = fmin(k.alpha_max, al);
            int fb = 0;
            if (learned) {
                // positivity-risk check: min nodal rho or p below a tenth of the element mean
                double rs = 0.0, ps = 0.0, rmin = 1e300, pmin = 1e300;
                for (int n = 0; n < NP; ++n) {
                    double uu[V];
#pragma unroll
                    for (int v = 0; v < V; ++v) uu[v] = su[(v * EPC + tid) * NP + n];
                    const double pr = pressure64(uu, k);
                    rs = rs + uu[0];
                    ps = ps + pr;
                    rmin = fmin(rmin, uu[0]);
                    pmin = fmin(pmin, pr);
                }
                if (rmin < 0.1 * (rs / 64.0) || pmin < 0.1 * (ps / 64.0)) fb = 1;
                for (int w = 0; w < 2; ++w) {
                    const double* mw = sp + (4 + w) * EPC * NP + tid * NP;
                    double tot = 0.0, Eo[6] = {0, 0, 0, 0, 0, 0};
                    for (int cc = 0; cc < NN; ++cc)
                        for (int bj = 0; bj < NN; ++bj)
                            for (int ai = 0; ai < NN; ++ai) {
                                const double mv = mw[nidx(ai, bj, cc)];
                                const double ee = mv * mv;
                                tot = tot + ee;
                                const int ord[3] = {ai, bj, cc};
#pragma unroll
                                for (int d = 0; d < 3; ++d) {
                                    if (ord[d] == NN - 1) Eo[2 * d] = Eo[2 * d] + ee;
                                    if (ord[d] == NN - 2) Eo[2 * d + 1] = Eo[2 * d + 1] + ee;
                                }
                            }
                    for (int i = 0; i < 6; ++i) {
                        const double f = plog64(Eo[i] / tot + 1e-12);
                        feat[tid * 12 + 6 * w + i] = f;
                        const double x = f / 10.0 + 1.0;
                        if (x < a.mlp64[MLP_NW + 6 * w + i] || x > a.mlp64[MLP_NW + 12 + 6 * w + i]) fb = 1;
                    }
                }
            }
            s_fb[tid] = fb;
        }
        __syncthreads();
        if (learned) {
            const double* W1 = a.mlp64;
            const double* b1 = W1 + 32 * 12;
            const double* W2 = b1 + 32;
            const double* b2 = W2 + 32 * 32;
            const double* W3 = b2 + 32;
            double* h1 = t1;   // [EPC][32]
            double* h2 = t2;
            for (int p = tid; p < nel * 32; p += NT) {
                const int pel = p / 32, j = p % 32;
                double s = b1[j];
                for (int i = 0; i < 12; ++i) s = s + W1[j * 12 + i] * (feat[pel * 12 + i] / 10.0 + 1.0);
                h1[pel * 32 + j] = silu64(s);
            }
            __syncthreads();
            for (int p = tid; p < nel * 32; p += NT) {
                const int pel = p / 32, j = p % 32;
                double s = b2[j];
                for (int i = 0; i < 32; ++i) s = s + W2[j * 32 + i] * h1[pel * 32 + i];
                h2[pel * 32 + j] = silu64(s);
            }
            __syncthreads();
            if (tid < nel) {
                double z = W3[32];
                for (int j = 0; j < 32; ++j) z = z + W3[j] * h2[tid * 32 + j];
                double al = k.alpha_max / (1.0 + pexp64(-z));
                if (al < k.alpha_min) al = 0.0;
                const double am = s_am[tid];
                if (s_fb[tid]) {
                    atomicAdd(&ctrl->fallback, 1ull);
                    al = am;
                } else {
                    atomicAdd(&ctrl->judge_sum, fabs(al - am));
                    atomicAdd(&ctrl->judge_n, 1ull);
                }
                a.alpha_out[e0 + tid] = al;
            }
        } else if (tid < nel) {
            a.alpha_out[e0 + tid] = s_am[tid];
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
                rr[1] = uu[1 + dd];
                rr[2] = uu[1 + (dd + 1) % 3];
                rr[3] = uu[1 + (dd + 2) % 3];
                rr[4] = uu[4];
                const double lam = xlambda64(rr, k);
                atomicMax(&s_lam[pel][dd], (unsigned long long)__double_as_longlong(lam));
            }
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
    }
}

}  // namespace

template <bool BLEND, bool IND, bool RHS_ONLY, bool FAST>
__global__ void __launch_bounds__(NT, NEMO_FP64_MINB) k_stage_euler64(StageArgs a) {
    extern __shared__ __align__(128) double smem[];
    double* su = smem;                    // [V][EPC][64] state, later the new state
    double* sp = su + V * EPC * NP;       // [6][EPC][64] vx,vy,vz,beta_x,beta_y,beta_z; later R_x
    double* sR = sp + 6 * EPC * NP;       // [2][V][EPC][64] R_y, R_z
    __shared__ uint64_t bar;
    __shared__ double s_alpha[EPC];
    __shared__ int s_bad[EPC];
    __shared__ unsigned long long s_lam[EPC][3];

    const OpConsts& k = c_ops64;
    Control* ctrl = a.ctrl;
    if (!RHS_ONLY && ctrl->done) return;

    const int tid = threadIdx.x;
    const int64_t E = a.E;
    const int64_t e0 = a.E_begin + (int64_t)blockIdx.x * EPC;
    const int nel = (int)min((int64_t)EPC, a.E_own - e0);

    // the tile's bulk copy first, so that it is in flight while the blending coefficients are read
    tile_issue(su, a.u_in, E, e0, nel, &bar);
    if (tid < EPC) {
        s_bad[tid] = 0;
        s_lam[tid][0] = s_lam[tid][1] = s_lam[tid][2] = 0ull;
        double al = 0.0;
        if (IND && tid < nel) {
            int64_t e = e0 + tid;
            al = a.alpha_in[e];
            if (a.smooth) {
#pragma unroll
                for (int f = 0; f < 6; ++f) {
                    int32_t ne = a.nbr[e * 6 + f];
                    if (ne >= 0) al = fmax(al, 0.5 * a.alpha_in[ne]);
                }
            }
            if (a.alpha_used) a.alpha_used[e] = al;
        }
        s_alpha[tid] = al;
    }
    // s_alpha, s_bad and s_lam become visible at the barrier after the primitives: the coefficient
    // loads overlap the bulk copy instead of holding the whole CTA
    if (!tile_wait(&bar, ctrl)) return;
    if (a.prep_only) {
        __syncthreads();
        epilogue64(a, su, smem + V * EPC * NP, s_lam, nel, e0, tid, k);
        return;
    }

    // per-node primitives: velocities and, per direction d, beta_d = rho/(2 p_d) where p_d is the
    // pressure of the state rotated into direction d (the reference evaluates the two-point flux on
    // the rotated state, so the kinetic-energy sum runs in the rotated component order)
    for (int p = tid; p < nel * NP; p += NT) {
        int el = p / NP, n = p % NP;
        double q[5];
#pragma unroll
        for (int v = 0; v < V; ++v) q[v] = su[(v * EPC + el) * NP + n];
        sp[(0 * EPC + el) * NP + n] = q[1] / q[0];
        sp[(1 * EPC + el) * NP + n] = q[2] / q[0];
        sp[(2 * EPC + el) * NP + n] = q[3] / q[0];
#pragma unroll
        for (int dd = 0; dd < 3; ++dd) {
            double r[5] = {q[0], q[1 + dd], q[1 + (dd + 1) % 3], q[1 + (dd + 2) % 3], q[4]};
            sp[((3 + dd) * EPC + el) * NP + n] = 0.5 * q[0] / pressure64(r, k);
        }
    }
    __syncthreads();

    const int el = tid / TPE;
    const int r = tid % TPE;
    const int d = r / NF;
    const int ab = r % NF;
    const int la = ab & 3, lb = ab >> 2;
    const bool active = el < nel;
    const int64_t e = e0 + el;
    // rotated component c (0..2) of the momentum/velocity -> original index (d + c) % 3
    const int c0 = d, c1 = (d + 1) % 3, c2 = (d + 2) % 3;

    double t[NN][V];  // direction-d contribution per line node, rotated frame
    if (active) {
        // ---- split-form volume flux differencing along the line
        int idx[NN];
#pragma unroll
        for (int i = 0; i < NN; ++i) idx[i] = line_node(d, la, lb, i);
#pragma unroll
        for (int i = 0; i < NN; ++i)
#pragma unroll
            for (int v = 0; v < V; ++v) t[i][v] = 0.0;
        const int PI_[6] = {0, 0, 0, 1, 1, 2};
        const int PM_[6] = {1, 2, 3, 2, 3, 3};
#pragma unroll
        for (int pq = 0; pq < 6; ++pq) {
            const int i = PI_[pq], m = PM_[pq];
            double F[V];
            if (!FAST && a.volume_flux == NEMO_VOLFLUX_CENTRAL) {
                double ui[V], um[V];
                ui[0] = su[(0 * EPC + el) * NP + idx[i]];
                ui[1] = su[((1 + c0) * EPC + el) * NP + idx[i]];
                ui[2] = su[((1 + c1) * EPC + el) * NP + idx[i]];
                ui[3] = su[((1 + c2) * EPC + el) * NP + idx[i]];
                ui[4] = su[(4 * EPC + el) * NP + idx[i]];
                um[0] = su[(0 * EPC + el) * NP + idx[m]];
                um[1] = su[((1 + c0) * EPC + el) * NP + idx[m]];
                um[2] = su[((1 + c1) * EPC + el) * NP + idx[m]];
                um[3] = su[((1 + c2) * EPC + el) * NP + idx[m]];
                um[4] = su[(4 * EPC + el) * NP + idx[m]];
                central64(ui, pressure64(ui, k), um, pressure64(um, k), F);
            } else {
                Node5 ni, nm;
                ni.rho = su[(0 * EPC + el) * NP + idx[i]];
                ni.vn = sp[(c0 * EPC + el) * NP + idx[i]];
                ni.vt1 = sp[(c1 * EPC + el) * NP + idx[i]];
                ni.vt2 = sp[(c2 * EPC + el) * NP + idx[i]];
                ni.beta = sp[((3 + d) * EPC + el) * NP + idx[i]];
                nm.rho = su[(0 * EPC + el) * NP + idx[m]];
                nm.vn = sp[(c0 * EPC + el) * NP + idx[m]];
                nm.vt1 = sp[(c1 * EPC + el) * NP + idx[m]];
                nm.vt2 = sp[(c2 * EPC + el) * NP + idx[m]];
                nm.beta = sp[((3 + d) * EPC + el) * NP + idx[m]];
                chandrashekar64(ni, nm, F, k);
            }
            const double sim = k.S[i * NN + m], smi = k.S[m * NN + i];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                t[i][v] = t[i][v] + sim * F[v];
                t[m][v] = t[m][v] + smi * F[v];
            }
        }
        // ---- surface fluxes at the two ends of the line (faces 2d, 2d+1 at (la,lb)), after the
        //      volume pairs so that they are not live during the pair loop (fewer registers)
        double Fs[2][V];
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const int f = 2 * d + side;
            const int own = line_node(d, la, lb, side ? NN - 1 : 0);
            double uo[V], un[V];
            uo[0] = su[(0 * EPC + el) * NP + own];
            uo[1] = su[((1 + c0) * EPC + el) * NP + own];
            uo[2] = su[((1 + c1) * EPC + el) * NP + own];
            uo[3] = su[((1 + c2) * EPC + el) * NP + own];
            uo[4] = su[(4 * EPC + el) * NP + own];
            const int32_t ne = a.nbr[e * 6 + f];
            if (ne <= -2) {  // 2:1 mortar face: flux row of the mortar kernel
                const double* mf = a.mflux + (int64_t)(-2 - ne) * V * NF + ab;
#pragma unroll
                for (int v = 0; v < V; ++v) Fs[side][v] = mf[v * NF];
                continue;
            }
            if (ne >= 0) {
                const int nn = line_node(d, la, lb, side ? 0 : NN - 1);
                const int64_t nl = (int64_t)ne - e0;
                if (nl >= 0 && nl < nel) {
                    const int nli = (int)nl;
                    un[0] = su[(0 * EPC + nli) * NP + nn];
                    un[1] = su[((1 + c0) * EPC + nli) * NP + nn];
                    un[2] = su[((1 + c1) * EPC + nli) * NP + nn];
                    un[3] = su[((1 + c2) * EPC + nli) * NP + nn];
                    un[4] = su[(4 * EPC + nli) * NP + nn];
                } else {
                    const double* g = a.u_in;
                    un[0] = __ldg(g + ((int64_t)0 * E + ne) * NP + nn);
                    un[1] = __ldg(g + ((int64_t)(1 + c0) * E + ne) * NP + nn);
                    un[2] = __ldg(g + ((int64_t)(1 + c1) * E + ne) * NP + nn);
                    un[3] = __ldg(g + ((int64_t)(1 + c2) * E + ne) * NP + nn);
                    un[4] = __ldg(g + ((int64_t)4 * E + ne) * NP + nn);
                }
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v) un[v] = uo[v];
            }
            if (side) riem64<FAST>(a.surface_flux, uo, un, Fs[1], k);
            else riem64<FAST>(a.surface_flux, un, uo, Fs[0], k);
        }

        // ---- surface lift at the line ends
#pragma unroll
        for (int v = 0; v < V; ++v) {
            t[0][v] = t[0][v] + k.winv[0] * (-Fs[0][v]);
            t[NN - 1][v] = t[NN - 1][v] + k.winv[NN - 1] * Fs[1][v];
        }
        // ---- FV subcells and convex blend
        if (BLEND) {
            const double al = s_alpha[el];
            if (al > 0.0) {
                double Fl[V], Fr[V];
#pragma unroll
                for (int v = 0; v < V; ++v) Fl[v] = Fs[0][v];
#pragma unroll
                for (int i = 0; i < NN; ++i) {
                    if (i < NN - 1) {
                        double uL[V], uR[V];
                        uL[0] = su[(0 * EPC + el) * NP + idx[i]];
                        uL[1] = su[((1 + c0) * EPC + el) * NP + idx[i]];
                        uL[2] = su[((1 + c1) * EPC + el) * NP + idx[i]];
                        uL[3] = su[((1 + c2) * EPC + el) * NP + idx[i]];
                        uL[4] = su[(4 * EPC + el) * NP + idx[i]];
                        uR[0] = su[(0 * EPC + el) * NP + idx[i + 1]];
                        uR[1] = su[((1 + c0) * EPC + el) * NP + idx[i + 1]];
                        uR[2] = su[((1 + c1) * EPC + el) * NP + idx[i + 1]];
                        uR[3] = su[((1 + c2) * EPC + el) * NP + idx[i + 1]];
                        uR[4] = su[(4 * EPC + el) * NP + idx[i + 1]];
                        riem64<FAST>(a.surface_flux, uL, uR, Fr, k);
                    } else {
#pragma unroll
                        for (int v = 0; v < V; ++v) Fr[v] = Fs[1][v];
                    }
#pragma unroll
                    for (int v = 0; v < V; ++v) {
                        double fv = k.winv[i] * (Fr[v] - Fl[v]);
                        t[i][v] = (1.0 - al) * t[i][v] + al * fv;
                        Fl[v] = Fr[v];
                    }
                }
            }
        }
    }
    __syncthreads();  // all reads of the primitives done: sp becomes R_x
    if (active) {
        const double cd = a.cdel[e * 3 + d];
        double* R = d == 0 ? sp : sR + (d - 1) * V * EPC * NP;
#pragma unroll
        for (int i = 0; i < NN; ++i) {
            const int n = line_node(d, la, lb, i);
            R[(0 * EPC + el) * NP + n] = cd * t[i][0];
            R[((1 + c0) * EPC + el) * NP + n] = cd * t[i][1];
            R[((1 + c1) * EPC + el) * NP + n] = cd * t[i][2];
            R[((1 + c2) * EPC + el) * NP + n] = cd * t[i][3];
            R[(4 * EPC + el) * NP + n] = cd * t[i][4];
        }
    }
    __syncthreads();

    // ---- rhs, LSRK register and state update
    const int st = a.stage;
    const double A = rk_a(st);
    const double Cdt = rk_c(st) * ctrl->dt[0];
    for (int p = tid; p < nel * NP; p += NT) {
        const int pel = p / NP, n = p % NP;
        const int64_t pe = e0 + pel;
        const double cdt = a.group ? rk_c(st) * ctrl->dt[a.group[pe]] : Cdt;
        bool ok = true;
        // the node's register values are loaded before any is stored (interleaved, each load would
        // wait for the previous store: the compiler cannot prove the addresses differ)
        double rg[V];
#pragma unroll
        for (int v = 0; v < V; ++v) rg[v] = (RHS_ONLY || st == 0) ? 0.0 : a.reg[((int64_t)v * E + pe) * NP + n];
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const int s = (v * EPC + pel) * NP + n;
            const double Rv = (sp[s] + sR[s]) + sR[V * EPC * NP + s];
            const double rhs = -Rv;
            const int64_t g = ((int64_t)v * E + pe) * NP + n;
            if (RHS_ONLY) {
                a.rhs_out[g] = rhs;
            } else {
                const double rr = st == 0 ? rhs : A * rg[v] + rhs;
                a.reg[g] = rr;
                su[s] = su[s] + cdt * rr;
            }
        }
        if (!RHS_ONLY && a.positivity) {
            double q[V];
#pragma unroll
            for (int v = 0; v < V; ++v) q[v] = su[(v * EPC + pel) * NP + n];
            ok = isvalid64(q, k);
            if (!ok) s_bad[pel] = 1;
        }
    }
    if (RHS_ONLY) return;
    __syncthreads();
    {   // element w is repaired by lanes 0..15 of warp w together (same arithmetic and order as the
        // serial dgfv_repair_3d, no call frame in this kernel)
        const int w = tid >> 5, lane = tid & 31;
        if (a.positivity && w < nel && lane < 16 && s_bad[w]) {
            const bool repaired = repair_elem16<EPC>(su, w, lane, k);
            if (!repaired && lane == 0) atomicAdd(&ctrl->nbad, 1ull);
        }
    }
    __syncthreads();
    // ---- source term after the stage, then store the new state
    for (int p = tid; p < nel * NP; p += NT) {
        const int pel = p / NP, n = p % NP;
        if (k.cool) {
            double q[V];
#pragma unroll
            for (int v = 0; v < V; ++v) q[v] = su[(v * EPC + pel) * NP + n];
            su[(4 * EPC + pel) * NP + n] = cooled_energy64(q, k);
        }
#pragma unroll
        for (int v = 0; v < V; ++v) a.u_out[((int64_t)v * E + e0 + pel) * NP + n] = su[(v * EPC + pel) * NP + n];
    }
    if (st == 4 && a.tick && blockIdx.x == 0 && tid == 0) {
        for (int g = 0; g < ctrl->ngroups; ++g) ctrl->t[g] = ctrl->t[g] + ctrl->dt[g];
        ctrl->steps += 1;
    }

    epilogue64(a, su, sp, s_lam, nel, e0, tid, k);
}

// Conserved totals: per-element weighted sums in the oracle's order, then a serial sum per
// variable (deterministic, bit-reproducible).
__global__ void k_totals_elem64(const double* __restrict__ u, const double* __restrict__ delta, int64_t E,
                                int64_t n, int nv, double* __restrict__ part) {
    const OpConsts& k = c_ops64;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const double vol = delta[e * 3 + 0] * delta[e * 3 + 1] * delta[e * 3 + 2];
    for (int v = 0; v < nv; ++v) {
        double s = 0.0;
        const double* ue = u + ((int64_t)v * E + e) * NP;
        for (int kk = 0; kk < NN; ++kk)
            for (int j = 0; j < NN; ++j)
                for (int i = 0; i < NN; ++i) s = s + k.wt[i] * k.wt[j] * k.wt[kk] * ue[nidx(i, j, kk)];
        part[(int64_t)v * n + e] = vol * s;
    }
}

__global__ void k_totals_sum64(const double* __restrict__ part, int64_t E, int nv, double* __restrict__ out) {
    const int v = threadIdx.x;
    if (v >= nv) return;
    double tot = 0.0;
    for (int64_t e = 0; e < E; ++e) tot = tot + part[(int64_t)v * E + e];
    out[v] = tot;
}

// ---------------------------------------------------------------------------------------------
// launchers

int stage_smem_bytes64() { return (V * EPC * NP + 6 * EPC * NP + 2 * V * EPC * NP) * (int)sizeof(double); }

cudaError_t launch_stage_euler64(const StageArgs& a, bool blend, bool ind, bool rhs_only, cudaStream_t s) {
    const int grid = (int)((a.E_own - a.E_begin + EPC - 1) / EPC);
    if (grid <= 0) return cudaSuccess;
    const int smem = stage_smem_bytes64();
    (void)ind;
    // the specialised kernel for HLLC faces and Chandrashekar pairs, the general one for the rest
    const bool fast = a.surface_flux == NEMO_SURFFLUX_HLLC && a.volume_flux == NEMO_VOLFLUX_CHANDRASHEKAR;
    if (rhs_only) {
        if (blend) k_stage_euler64<true, true, true, false><<<grid, NT, smem, s>>>(a);
        else k_stage_euler64<false, false, true, false><<<grid, NT, smem, s>>>(a);
    } else if (fast) {
        if (blend) k_stage_euler64<true, true, false, true><<<grid, NT, smem, s>>>(a);
        else k_stage_euler64<false, false, false, true><<<grid, NT, smem, s>>>(a);
    } else {
        if (blend) k_stage_euler64<true, true, false, false><<<grid, NT, smem, s>>>(a);
        else k_stage_euler64<false, false, false, false><<<grid, NT, smem, s>>>(a);
    }
    return cudaGetLastError();
}

cudaError_t setup_stage_euler64(const OpConsts& ops) {
    const int smem = stage_smem_bytes64();
    cudaError_t err;
    const auto dyn = cudaFuncAttributeMaxDynamicSharedMemorySize;
    if ((err = cudaFuncSetAttribute(k_stage_euler64<true, true, true, false>, dyn, smem)) != cudaSuccess) return err;
    if ((err = cudaFuncSetAttribute(k_stage_euler64<false, false, true, false>, dyn, smem)) != cudaSuccess) return err;
    if ((err = cudaFuncSetAttribute(k_stage_euler64<true, true, false, false>, dyn, smem)) != cudaSuccess) return err;
    if ((err = cudaFuncSetAttribute(k_stage_euler64<false, false, false, false>, dyn, smem)) != cudaSuccess) return err;
    if ((err = cudaFuncSetAttribute(k_stage_euler64<true, true, false, true>, dyn, smem)) != cudaSuccess) return err;
    if ((err = cudaFuncSetAttribute(k_stage_euler64<false, false, false, true>, dyn, smem)) != cudaSuccess) return err;
    return cudaMemcpyToSymbol(c_ops64, &ops, sizeof(OpConsts));
}

cudaError_t launch_totals64(const double* u, const double* delta, int64_t E, int64_t n, int nv, double* part,
                            double* out, cudaStream_t s) {
    k_totals_elem64<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(u, delta, E, n, nv, part);
    k_totals_sum64<<<1, 32, 0, s>>>(part, n, nv, out);
    return cudaGetLastError();
}


// ---- GLM-MHD stage (double flux arithmetic).  Tile of the plain form: 4 elements (64 threads) with
// at least 4 CTAs per SM at the full 255 registers (Orszag-Tang 64^3, B200: 12.81 ms per stage against
// 13.21 ms for 8 elements x 1-2 CTAs/SM; 2 elements x 8 CTAs 12.81 ms; 4 x 5 at 168 registers
// 15.89 ms; bit-identical results).  The FP32 form keeps its 8-element tile (stage_fp32.cu).
#ifndef NEMO_MHD_EPC
#define NEMO_MHD_EPC 4
#endif
#ifndef NEMO_MHD64_MINB
#define NEMO_MHD64_MINB 4
#endif
#define NEMO_MHD_OPS c_ops64
}  // namespace nemo
#include "stage_mhd.cuh"
namespace nemo {
#undef NEMO_MHD_OPS

// state, rhs rows and the subcell interface fluxes of each thread's line
int stage_smem_bytes_mhd64() {
    return mhd::V * mhd::EPC * (NP * (int)sizeof(double) + mhd::SPM * (int)sizeof(double)) +
           (NN - 1) * mhd::V * mhd::NT * (int)sizeof(double);
}

cudaError_t setup_stage_mhd64() {
    const int smem = stage_smem_bytes_mhd64();
    cudaError_t err;
    const auto dyn = cudaFuncAttributeMaxDynamicSharedMemorySize;
    if ((err = cudaFuncSetAttribute(k_stage_mhd<double, true, true, false>, dyn, smem))) return err;
    if ((err = cudaFuncSetAttribute(k_stage_mhd<double, false, true, false>, dyn, smem))) return err;
    if ((err = cudaFuncSetAttribute(k_stage_mhd<double, true, false, false>, dyn, smem))) return err;
    if ((err = cudaFuncSetAttribute(k_stage_mhd<double, false, false, false>, dyn, smem))) return err;
    if ((err = cudaFuncSetAttribute(k_stage_mhd<double, true, false, true>, dyn, smem))) return err;
    return cudaFuncSetAttribute(k_stage_mhd<double, false, false, true>, dyn, smem);
}

// Positivity repair of element states held outside the library (the per-quad kernel_repair of a
// host, source/kernel/mcfv/3d/kernel_validate_mod.f90:27-157): one warp per element [nv][64] (the
// Fortran state(n,n,n,nv) layout); if a node is inadmissible, lanes 0..15 run the cooperative
// dgfv_repair_3d of the stage kernels on it.  ok[e] = 1 if the element is admissible afterwards.
__global__ void __launch_bounds__(32) k_repair_states64(double* __restrict__ st, int64_t n, int nv, int is_mhd,
                                                        int32_t* __restrict__ ok) {
    __shared__ double su[VMAX * NP];
    const OpConsts& k = c_ops64;
    const int64_t e = blockIdx.x;
    const int lane = threadIdx.x;
    double* g = st + e * (int64_t)nv * NP;
    for (int p = lane; p < nv * NP; p += 32) su[p] = g[p];
    __syncwarp();
    bool valid = true;
    for (int p = lane; p < NP; p += 32) {
        double q[VMAX];
        for (int v = 0; v < nv; ++v) q[v] = su[v * NP + p];
        valid = valid && (is_mhd ? m_isvalid<double>(q, k.kappa, k.mu0) : isvalid64(q, k));
    }
    bool good = __all_sync(0xffffffffu, valid);
    if (!good) {
        bool rep = false;
        if (lane < 16) rep = is_mhd ? repair_elem16_mhd<1>(su, 0, lane, k) : repair_elem16<1>(su, 0, lane, k);
        good = __shfl_sync(0xffffffffu, rep, 0);
        __syncwarp();
        for (int p = lane; p < nv * NP; p += 32) g[p] = su[p];
    }
    if (lane == 0) ok[e] = good ? 1 : 0;
}

cudaError_t launch_repair_states64(double* st, int64_t n, int nv, int mhd, int32_t* ok, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    if (n > 0x7fffffffLL) return cudaErrorInvalidValue;
    k_repair_states64<<<(unsigned)n, 32, 0, s>>>(st, n, nv, mhd, ok);
    return cudaGetLastError();
}

cudaError_t launch_stage_mhd64(const StageArgs& a, bool blend, bool rhs_only, cudaStream_t s) {
    const int grid = (int)((a.E_own - a.E_begin + mhd::EPC - 1) / mhd::EPC);
    if (grid <= 0) return cudaSuccess;
    const int smem = stage_smem_bytes_mhd64();
    // the specialised kernel for HLLD faces and the EC pair flux, the general one for the rest
    const bool fast = a.surface_flux == NEMO_SURFFLUX_HLLD && a.volume_flux == NEMO_VOLFLUX_EC_MHD;
    if (rhs_only) {
        if (blend) k_stage_mhd<double, true, true, false><<<grid, mhd::NT, smem, s>>>(a);
        else k_stage_mhd<double, false, true, false><<<grid, mhd::NT, smem, s>>>(a);
    } else if (fast) {
        if (blend) k_stage_mhd<double, true, false, true><<<grid, mhd::NT, smem, s>>>(a);
        else k_stage_mhd<double, false, false, true><<<grid, mhd::NT, smem, s>>>(a);
    } else {
        if (blend) k_stage_mhd<double, true, false, false><<<grid, mhd::NT, smem, s>>>(a);
        else k_stage_mhd<double, false, false, false><<<grid, mhd::NT, smem, s>>>(a);
    }
    return cudaGetLastError();
}

}  // namespace nemo
