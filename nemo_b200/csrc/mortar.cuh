// mortar.cuh -- one pair of 2:1 mortars processed by 128 threads (64 per mortar, one per sub-face
// node): coarse trace staged in shared memory and prolonged (tensor product of the 1D interpolation
// matrices), Riemann flux against the fine quad's trace in the face's rotated frame (plus, for MHD,
// each side's non-conservative term), the fine rows written directly and the coarse row projected
// (1D projection matrices), sums in the oracle's order (oracle mortar_fluxes).  A prolonged sub-face
// trace with an inadmissible node (a strong shock on the coarse side) is replaced by the coarse face's
// mean, which is admissible; the reference interpolates without this guard.  Used by the mortar
// kernel (mortar.cu) and by the persistent FP32 stage kernel, which runs the mortar pairs as its
// first tasks and publishes each mortar with a release flag (epoch) that its element tiles acquire.
// Reference: the mortar part of kernel_fill_faceflux, source/kernel/mcfv/3d/kernel_flux_mod.f90:
// 100-118 and 252-269, with kernel_operators_interpolationMatrix / _projectionMatrix,
// source/kernel/dgsem/weakform/2d/kernel_operators_mod.f90:1010-1100.
#pragma once

#include "euler_fp64.cuh"
#include "kernels.h"
#include "mhd_phys.cuh"

namespace nemo {
namespace mortar {

constexpr int MPB = 2;          // mortars per 128-thread task
constexpr int SCRATCH_DOUBLES = MPB * 9 * NF + MPB * 4 * 9 * NF;

// LGL-weighted mean of a coarse face trace held as [V][NF] (out of line: taken only on a shock)
static __device__ __noinline__ void face_mean(const double* uc, int V, double* out, const OpConsts& k) {
    for (int v = 0; v < V; ++v) {
        double acc = 0.0;
        for (int bb = 0; bb < NN; ++bb)
            for (int aa = 0; aa < NN; ++aa) acc = acc + (k.wt[aa] * k.wt[bb]) * uc[v * NF + aa + NN * bb];
        out[v] = acc;
    }
}

template <bool MHD>
__device__ __forceinline__ void mortar_pair(const MortarArgs& a, int64_t pair, double* scratch, const OpConsts& k) {
    constexpr int V = MHD ? 9 : 5;
    auto s_uc = reinterpret_cast<double (*)[V][NF]>(scratch);                       // [MPB][V][NF]
    auto s_fs = reinterpret_cast<double (*)[4][V][NF]>(scratch + MPB * V * NF);      // [MPB][4][V][NF]
    const int ml = threadIdx.x >> 6, r = threadIdx.x & 63;
    const int64_t m = pair * MPB + ml;
    const bool act = m < a.nm;
    const int32_t* t = a.mortar + 6 * (act ? m : 0);
    const int64_t E = a.E;
    const int64_t qc = t[0];
    const int fc = t[1], ff = fc ^ 1, d = fc >> 1;
    const bool coarse_left = (fc & 1) != 0;
    if (act && r < NF) {
        const int n = line_node(d, r & 3, r >> 2, (fc & 1) ? NN - 1 : 0);
#pragma unroll
        for (int v = 0; v < V; ++v) s_uc[ml][v][r] = a.u_in[((int64_t)v * E + qc) * NP + n];
    }
    __syncthreads();
    const int kq = r >> 4, i = r & 3, j = (r >> 2) & 3;
    const int s = kq & 1, tt = kq >> 1;
    if (act) {
        const int64_t qf = t[2 + kq];
        const int nf = line_node(d, i, j, (ff & 1) ? NN - 1 : 0);
        double up[V], uf[V];
#pragma unroll
        for (int v = 0; v < V; ++v) {
            double acc = 0.0;
#pragma unroll
            for (int bb = 0; bb < NN; ++bb) {
                double in = 0.0;
#pragma unroll
                for (int aa = 0; aa < NN; ++aa) in = in + k.pro[s][i * NN + aa] * s_uc[ml][v][aa + NN * bb];
                acc = acc + k.pro[tt][j * NN + bb] * in;
            }
            up[v] = acc;
        }
        // a sub-face (16 lanes of this warp; act is warp-uniform) whose prolonged trace has an
        // inadmissible node takes the coarse face's mean instead, as the oracle does
        bool okn;
        if constexpr (MHD) okn = m_isvalid<double>(up, k.kappa, k.mu0);
        else okn = isvalid64(up, k);
        const unsigned badl = __ballot_sync(0xffffffffu, !okn);
        if (badl & (0xffffu << (16 * (kq & 1)))) face_mean(&s_uc[ml][0][0], V, up, k);
#pragma unroll
        for (int v = 0; v < V; ++v) uf[v] = a.u_in[((int64_t)v * E + qf) * NP + nf];
        // rotate into the face frame: component c of momentum (and field) -> original (d + c) % 3
        double rp[V], rf[V];
        rp[0] = up[0];
        rf[0] = uf[0];
        rp[4] = up[4];
        rf[4] = uf[4];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            rp[1 + c] = up[1 + (d + c) % 3];
            rf[1 + c] = uf[1 + (d + c) % 3];
        }
        if (MHD) {
            rp[8] = up[8];
            rf[8] = uf[8];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                rp[5 + c] = up[5 + (d + c) % 3];
                rf[5 + c] = uf[5 + (d + c) % 3];
            }
        }
        const double* uL = coarse_left ? rp : rf;
        const double* uR = coarse_left ? rf : rp;
        double F[V], Gf[V], Gc[V];
        double* out = a.mflux + ((5 * m + 1 + kq) * V) * NF + (i + NN * j);
        if (MHD) {
            const double ch = a.ctrl->glm_ch;
            m_riemann_x<double>(a.surface_flux, uL, uR, F, k.kappa, k.mu0, ch);
            m_nc_x<double>(rf, uL, uR, Gf, k.mu0);
            m_nc_x<double>(rp, uL, uR, Gc, k.mu0);
#pragma unroll
            for (int v = 0; v < V; ++v) {
                out[v * NF] = F[v] + Gf[v];
                s_fs[ml][kq][v][i + NN * j] = F[v] + Gc[v];
            }
        } else {
            riemann64(a.surface_flux, uL, uR, F, k);
#pragma unroll
            for (int v = 0; v < V; ++v) {
                out[v * NF] = F[v];
                s_fs[ml][kq][v][i + NN * j] = F[v];
            }
        }
    }
    __syncthreads();
    if (act && r < NF) {
        const int aa = r & 3, bb = r >> 2;
        double* out = a.mflux + (5 * m * V) * NF + r;
#pragma unroll
        for (int v = 0; v < V; ++v) {
            double acc = 0.0;
#pragma unroll
            for (int t2 = 0; t2 < 2; ++t2)
#pragma unroll
                for (int s2 = 0; s2 < 2; ++s2)
#pragma unroll
                    for (int jj = 0; jj < NN; ++jj) {
                        double in = 0.0;
#pragma unroll
                        for (int ii = 0; ii < NN; ++ii)
                            in = in + k.prj[s2][aa * NN + ii] * s_fs[ml][s2 + 2 * t2][v][ii + NN * jj];
                        acc = acc + k.prj[t2][bb * NN + jj] * in;
                    }
            out[v * NF] = acc;
        }
    }
    if (a.mflag) {  // publish: the mortar's five flux rows are complete for this epoch
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0 || threadIdx.x == 64) {
            if (act) {
                __threadfence();
                asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(a.mflag + m), "r"(a.epoch) : "memory");
            }
        }
    }
}

}  // namespace mortar
}  // namespace nemo
