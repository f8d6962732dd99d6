// mortar.cu -- 2:1 non-conforming faces (compiled with -fmad=false: bit-identical to the oracle).
//
// One mortar = one coarse face and the four fine faces behind it (fine quad k = s + 2t at half s of
// the face's first tangential axis and half t of the second).  64 threads per mortar, one per
// sub-face node: the coarse trace is staged in shared memory and prolonged to the node (tensor
// product of the 1D interpolation matrices), the Riemann flux is evaluated against the fine quad's
// trace in the face's rotated frame (with the MHD non-conservative term of each side), the fine
// quad's flux row is written directly, and the coarse row is the projection of the four sub-face
// fluxes (1D projection matrices).  The sums run in the oracle's order (oracle mortar_fluxes).
// Reference: the mortar part of kernel_fill_faceflux, source/kernel/mcfv/3d/kernel_flux_mod.f90:
// 100-118 and 252-269, with kernel_operators_interpolationMatrix / _projectionMatrix,
// source/kernel/dgsem/weakform/2d/kernel_operators_mod.f90:1010-1100.
#include "euler_fp64.cuh"
#include "kernels.h"
#include "mhd_phys.cuh"

namespace nemo {

namespace {

__constant__ OpConsts c_opsm;

constexpr int MPB = 2;          // mortars per block
constexpr int MT = 64 * MPB;    // threads per block

template <bool MHD>
__global__ void __launch_bounds__(MT) k_mortar(MortarArgs a) {
    constexpr int V = MHD ? 9 : 5;
    __shared__ double s_uc[MPB][V][NF];        // coarse trace, unrotated components
    __shared__ double s_fs[MPB][4][V][NF];     // coarse-side sub-face fluxes, rotated frame
    const OpConsts& k = c_opsm;
    if (a.skip_if_done && a.ctrl->done) return;
    const int ml = threadIdx.x >> 6, r = threadIdx.x & 63;
    const int64_t m = (int64_t)blockIdx.x * MPB + ml;
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
            uf[v] = a.u_in[((int64_t)v * E + qf) * NP + nf];
        }
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
}

}  // namespace

cudaError_t setup_mortar(const OpConsts& ops) { return cudaMemcpyToSymbol(c_opsm, &ops, sizeof(OpConsts)); }

cudaError_t launch_mortar(const MortarArgs& a, cudaStream_t s) {
    if (a.nm <= 0) return cudaSuccess;
    const unsigned grid = (unsigned)((a.nm + MPB - 1) / MPB);
    if (a.mhd) k_mortar<true><<<grid, MT, 0, s>>>(a);
    else k_mortar<false><<<grid, MT, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace nemo
