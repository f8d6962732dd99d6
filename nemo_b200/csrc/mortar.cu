// mortar.cu -- the 2:1 mortar kernel (compiled with -fmad=false: bit-identical to the oracle).
// One 128-thread block per pair of mortars; the arithmetic is mortar::mortar_pair (mortar.cuh).
#include "mortar.cuh"

namespace nemo {

namespace {

__constant__ OpConsts c_opsm;

template <bool MHD>
__global__ void __launch_bounds__(128) k_mortar(MortarArgs a) {
    __shared__ double scratch[mortar::SCRATCH_DOUBLES];
    if (a.skip_if_done && a.ctrl->done) return;
    mortar::mortar_pair<MHD>(a, (int64_t)blockIdx.x, scratch, c_opsm);
}

// Lagrange basis polynomial j of the nodes x at xi (the same product as the host's and the oracle's)
__device__ __forceinline__ double lagrange_dev(const double* x, int j, double xi) {
    double l = 1.0;
#pragma unroll
    for (int m = 0; m < NN; ++m)
        if (m != j) l = l * ((xi - x[m]) / (x[j] - x[m]));
    return l;
}

// Element data of an adapted forest from the old one, one thread per new node (all variables):
// copy; interpolation of an ancestor's polynomial at the new element's nodes (kernel_amr_refine,
// source/kernel/dgsem/weakform/2d/kernel_amr_mod.f90:12-31, as a 3D tensor product); or the sum over
// the 8 children of their projections (kernel_amr_coarsen, :53-73).  The sums run in the oracle's
// order (oracle or_remap).
__global__ void k_remap(const double* __restrict__ uo, int64_t Eo, double* __restrict__ un, int64_t En,
                        const int32_t* __restrict__ remap, int nv) {
    const OpConsts& k = c_opsm;
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= En * NP) return;
    const int64_t e = idx / NP;
    const int n = (int)(idx % NP);
    const int ii = n % NN, jj = (n / NN) % NN, kk = n / NF;
    const int kind = remap[e * 4 + 0];
    const int64_t src = remap[e * 4 + 1];
    if (kind == 0) {
        for (int v = 0; v < nv; ++v) un[((int64_t)v * En + e) * NP + n] = uo[((int64_t)v * Eo + src) * NP + n];
        return;
    }
    if (kind == 1) {
        const int depth = remap[e * 4 + 2];
        const int off = remap[e * 4 + 3];
        const int o[3] = {off & 0xff, (off >> 8) & 0xff, (off >> 16) & 0xff};
        const int nd[3] = {ii, jj, kk};
        double w[3][NN];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double xi = -1.0 + (2.0 * (double)o[d] + 1.0 + k.x[nd[d]]) / (double)(1 << depth);
#pragma unroll
            for (int a = 0; a < NN; ++a) w[d][a] = lagrange_dev(k.x, a, xi);
        }
        for (int v = 0; v < nv; ++v) {
            const double* ue = uo + ((int64_t)v * Eo + src) * NP;
            double acc = 0.0;
            for (int c = 0; c < NN; ++c)
                for (int b = 0; b < NN; ++b)
#pragma unroll
                    for (int a = 0; a < NN; ++a) acc = acc + ((w[0][a] * w[1][b]) * w[2][c]) * ue[nidx(a, b, c)];
            un[((int64_t)v * En + e) * NP + n] = acc;
        }
        return;
    }
    for (int v = 0; v < nv; ++v) {
        double acc = 0.0;
        for (int ch = 0; ch < 8; ++ch) {
            const double* px = k.prj[ch & 1];
            const double* py = k.prj[(ch >> 1) & 1];
            const double* pz = k.prj[ch >> 2];
            const double* ue = uo + ((int64_t)v * Eo + src + ch) * NP;
            for (int c = 0; c < NN; ++c)
                for (int b = 0; b < NN; ++b)
#pragma unroll
                    for (int a = 0; a < NN; ++a)
                        acc = acc + ((px[ii * NN + a] * py[jj * NN + b]) * pz[kk * NN + c]) * ue[nidx(a, b, c)];
        }
        un[((int64_t)v * En + e) * NP + n] = acc;
    }
}

// LGL-weighted sum of one element's 64 values, in the oracle's order (elem_mean)
__device__ __forceinline__ double elem_wsum(const double* w, const double* ue) {
    double acc = 0.0;
    for (int c = 0; c < NN; ++c)
        for (int b = 0; b < NN; ++b)
#pragma unroll
            for (int a = 0; a < NN; ++a) acc = acc + ((w[a] * w[b]) * w[c]) * ue[nidx(a, b, c)];
    return acc;
}

// Admissibility of the transferred elements (isvalid after setup_amr_replace_refine / _coarsen,
// source/setups/euler/3d/sedov/setup_amr_mod.f90:90 and :122), one warp per new element: an
// inadmissible refined element marks its ancestor (bad[src]), an inadmissible coarsened one itself
// (bad[Eo + e]).  The element index is warp-uniform, so the ballot sees all 32 lanes.
__global__ void __launch_bounds__(128) k_remap_check(const double* __restrict__ un, int64_t En,
                                                     const int32_t* __restrict__ remap, int nv, int64_t Eo,
                                                     int32_t* __restrict__ bad) {
    const OpConsts& k = c_opsm;
    const int64_t e = (int64_t)blockIdx.x * 4 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (e >= En) return;
    const int kind = remap[e * 4];
    if (kind == 0) return;
    bool ok = true;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int n = lane + 32 * h;
        double q[9];
        for (int v = 0; v < nv; ++v) q[v] = un[((int64_t)v * En + e) * NP + n];
        ok = ok && (nv == 9 ? m_isvalid<double>(q, k.kappa, k.mu0) : isvalid64(q, k));
    }
    const unsigned nbad = __ballot_sync(0xffffffffu, !ok);
    if (nbad != 0u && lane == 0) atomicOr(&bad[kind == 1 ? (int64_t)remap[e * 4 + 1] : Eo + e], 1);
}

// The lowest-order transfer where the check failed: every element refined from a marked ancestor takes
// the ancestor's mean, a marked coarsened element the mean of its 8 children (oracle or_remap).
__global__ void __launch_bounds__(128) k_remap_fallback(const double* __restrict__ uo, int64_t Eo,
                                                        double* __restrict__ un, int64_t En,
                                                        const int32_t* __restrict__ remap, int nv,
                                                        const int32_t* __restrict__ bad) {
    const OpConsts& k = c_opsm;
    const int64_t e = (int64_t)blockIdx.x * 4 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (e >= En) return;
    const int kind = remap[e * 4];
    const int64_t src = remap[e * 4 + 1];
    if (kind == 0 || !bad[kind == 1 ? src : Eo + e]) return;
    for (int v = 0; v < nv; ++v) {
        double m;
        if (kind == 1) {
            m = elem_wsum(k.w, uo + ((int64_t)v * Eo + src) * NP) * 0.125;
        } else {
            double acc = 0.0;
            for (int ch = 0; ch < 8; ++ch) acc = acc + elem_wsum(k.w, uo + ((int64_t)v * Eo + src + ch) * NP);
            m = acc * 0.015625;
        }
        un[((int64_t)v * En + e) * NP + lane] = m;
        un[((int64_t)v * En + e) * NP + lane + 32] = m;
    }
}

// Adapt flags from the density (setup_amr_probe_refine / setup_amr_probe_coarsen of the Sedov setup,
// source/setups/euler/3d/sedov/setup_amr_mod.f90:23-65), one warp per element: +1 where some node's
// density exceeds refine_thr, -1 where no node's density exceeds coarsen_thr (a family coarsens when
// all 8 members say so), else 0.  The element index is warp-uniform, so the shuffles see all lanes.
__global__ void __launch_bounds__(128) k_amr_flags(const double* __restrict__ u, int64_t E, double refine_thr,
                                                   double coarsen_thr, int32_t* __restrict__ flags) {
    const int64_t e = (int64_t)blockIdx.x * 4 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (e >= E) return;
    const double* d = u + e * NP;   // variable 0 (density) of element e
    const double a = d[lane], b = d[lane + 32];
    int up = (a > refine_thr) || (b > refine_thr);
    int keep = (a > coarsen_thr) || (b > coarsen_thr);
    up = __any_sync(0xffffffffu, up);
    keep = __any_sync(0xffffffffu, keep);
    if (lane == 0) flags[e] = up ? 1 : (keep ? 0 : -1);
}

}  // namespace

cudaError_t launch_remap(const double* uo, int64_t Eo, double* un, int64_t En, const int32_t* remap, int nv,
                         int32_t* bad, cudaStream_t s) {
    const int64_t total = En * NP;
    if (total <= 0) return cudaSuccess;
    k_remap<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(uo, Eo, un, En, remap, nv);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    const unsigned blocks = (unsigned)((En + 3) / 4);
    if ((err = cudaMemsetAsync(bad, 0, sizeof(int32_t) * (size_t)(Eo + En), s)) != cudaSuccess) return err;
    k_remap_check<<<blocks, 128, 0, s>>>(un, En, remap, nv, Eo, bad);
    k_remap_fallback<<<blocks, 128, 0, s>>>(uo, Eo, un, En, remap, nv, bad);
    return cudaGetLastError();
}

cudaError_t launch_amr_flags(const double* u, int64_t E, double refine_thr, double coarsen_thr, int32_t* flags,
                             cudaStream_t s) {
    if (E <= 0) return cudaSuccess;
    k_amr_flags<<<(unsigned)((E + 3) / 4), 128, 0, s>>>(u, E, refine_thr, coarsen_thr, flags);
    return cudaGetLastError();
}

cudaError_t setup_mortar(const OpConsts& ops) { return cudaMemcpyToSymbol(c_opsm, &ops, sizeof(OpConsts)); }

cudaError_t launch_mortar(const MortarArgs& a, cudaStream_t s) {
    if (a.nm <= 0) return cudaSuccess;
    const unsigned grid = (unsigned)((a.nm + mortar::MPB - 1) / mortar::MPB);
    if (a.mhd) k_mortar<true><<<grid, 128, 0, s>>>(a);
    else k_mortar<false><<<grid, 128, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace nemo
