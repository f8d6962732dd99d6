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

}  // namespace

cudaError_t setup_mortar(const OpConsts& ops) { return cudaMemcpyToSymbol(c_opsm, &ops, sizeof(OpConsts)); }

cudaError_t launch_mortar(const MortarArgs& a, cudaStream_t s) {
    if (a.nm <= 0) return cudaSuccess;
    const unsigned grid = (unsigned)((a.nm + mortar::MPB - 1) / mortar::MPB);
    if (a.mhd) k_mortar<true><<<grid, 128, 0, s>>>(a);
    else k_mortar<false><<<grid, 128, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace nemo
