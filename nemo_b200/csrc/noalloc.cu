// noalloc.cu -- conserved totals of a caller-owned device state, allocating nothing.
//
// Some hosts cannot allocate device memory at the point where they want the totals: a Fortran
// driver whose device arrays come from its own pool (OpenACC/CUDA Fortran data regions sized at
// start-up, with the rest of the device reserved), or a code that runs under a fixed device-memory
// budget where a cudaMalloc/cudaFree in mid-run would either fail or implicitly synchronise the
// device.  For them nemo_gpu_totals_noalloc reads the state and writes the totals in memory the
// caller owns, and keeps its per-element partial sums in the fixed array below, which is part of
// the library image: every GPU that loads the library holds it (4.5 MiB) until the process exits.
//
// The kernels are the same arithmetic as k_totals_elem64/k_totals_sum64 (stage_fp64.cu); like that
// file, this one is compiled with -fmad=false, so both entry points give identical totals.
#include <cstdio>
#include <cstring>

#include "kernels.h"

namespace nemo {

constexpr int64_t NOALLOC_MAX_ELEMS = 65536;
constexpr int NOALLOC_MAX_VARS = 9;

// Per-element partial sums [nvars][nelems] of the last call (shared by every call).
static __device__ __align__(256) double g_totals_scratch[NOALLOC_MAX_VARS * NOALLOC_MAX_ELEMS];

namespace {

struct Weights {
    double wt[NN];
};

// part[v][e] for the first n elements of a state with element stride E (n <= E; elements [n, E) are
// ghost copies of a partitioned run and are not summed)
__global__ void k_totals_elem64_static(const double* __restrict__ u, const double* __restrict__ delta, int64_t E,
                                       int64_t n, int nv, Weights w, double* __restrict__ part) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const double vol = delta[e * 3 + 0] * delta[e * 3 + 1] * delta[e * 3 + 2];
    for (int v = 0; v < nv; ++v) {
        double s = 0.0;
        const double* ue = u + ((int64_t)v * E + e) * NP;
        for (int kk = 0; kk < NN; ++kk)
            for (int j = 0; j < NN; ++j)
                for (int i = 0; i < NN; ++i) s = s + w.wt[i] * w.wt[j] * w.wt[kk] * ue[nidx(i, j, kk)];
        part[(int64_t)v * n + e] = vol * s;
    }
}

__global__ void k_totals_sum64_static(const double* __restrict__ part, int64_t E, int nv, double* __restrict__ out) {
    const int v = threadIdx.x;
    if (v >= nv) return;
    double tot = 0.0;
    for (int64_t e = 0; e < E; ++e) tot = tot + part[(int64_t)v * E + e];
    out[v] = tot;
}

constexpr int MAX_DEVICES = 64;
double* g_scratch_ptr[MAX_DEVICES] = {};
Weights g_weights;          // quadrature weights on [-1/2, 1/2], built with the first scratch look-up
bool g_have_weights = false;

}  // namespace

void set_last_error(const char* msg);  // nemo_gpu.cu: the message nemo_gpu_last_error returns

}  // namespace nemo

using namespace nemo;

extern "C" int nemo_gpu_operators(int32_t n, double* nodes, double* weights, double* dmat, double* smat,
                                  double* vinv);

extern "C" int nemo_gpu_totals_noalloc(const double* u_dev, const double* delta_dev, int64_t elem_stride,
                                       int64_t nelems, int32_t nvars, double* out_dev, uint64_t stream) {
    auto fail = [](int code, const char* msg) {
        set_last_error(msg);
        return code;
    };
    if (!u_dev || !delta_dev || !out_dev) return fail(NEMO_ERR_ARG, "nemo_gpu_totals_noalloc: NULL device pointer");
    if (nelems <= 0 || nelems > NOALLOC_MAX_ELEMS) {
        char buf[160];
        std::snprintf(buf, sizeof buf, "nemo_gpu_totals_noalloc: nelems = %lld outside [1, %lld] (the size of its fixed scratch)",
                      (long long)nelems, (long long)NOALLOC_MAX_ELEMS);
        return fail(NEMO_ERR_ARG, buf);
    }
    if (elem_stride < nelems) {
        char buf[160];
        std::snprintf(buf, sizeof buf, "nemo_gpu_totals_noalloc: elem_stride = %lld below nelems = %lld",
                      (long long)elem_stride, (long long)nelems);
        return fail(NEMO_ERR_ARG, buf);
    }
    if (nvars < 1 || nvars > NOALLOC_MAX_VARS) return fail(NEMO_ERR_ARG, "nemo_gpu_totals_noalloc: nvars outside [1, 9]");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES)
        return fail(NEMO_ERR_CUDA, "nemo_gpu_totals_noalloc: no current CUDA device");
    // set-up, once per device, with that device current: the device address of the fixed scratch
    if (!g_scratch_ptr[dev]) {
        double* ptr = nullptr;
        cudaError_t err = cudaGetSymbolAddress((void**)&ptr, g_totals_scratch);
        if (err != cudaSuccess || !ptr) return fail(NEMO_ERR_CUDA, "nemo_gpu_totals_noalloc: cudaGetSymbolAddress failed");
        g_scratch_ptr[dev] = ptr;
    }
    if (!g_have_weights) {
        double x[NN], wl[NN];
        if (nemo_gpu_operators(NN, x, wl, nullptr, nullptr, nullptr) != NEMO_OK)
            return fail(NEMO_ERR_ARG, "nemo_gpu_totals_noalloc: quadrature weights could not be built");
        for (int i = 0; i < NN; ++i) g_weights.wt[i] = 0.5 * wl[i];
        g_have_weights = true;
    }
    cudaStream_t s = (cudaStream_t)(uintptr_t)stream;
    k_totals_elem64_static<<<(unsigned)((nelems + 127) / 128), 128, 0, s>>>(u_dev, delta_dev, elem_stride, nelems,
                                                                           nvars, g_weights, g_scratch_ptr[dev]);
    k_totals_sum64_static<<<1, 32, 0, s>>>(g_scratch_ptr[dev], nelems, nvars, out_dev);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return fail(NEMO_ERR_CUDA, cudaGetErrorString(err));
    return NEMO_OK;
}
