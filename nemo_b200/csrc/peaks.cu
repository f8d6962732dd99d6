// peaks.cu -- measured FP64 and FP32 fused-multiply-add peaks of the current GPU.
//
// The stage kernels are graded against the binding one of two rooflines: HBM bandwidth and the
// arithmetic peak of the precision their flux arithmetic runs in (FP64 for the plain path, FP32 for
// the FP32-bulk form).  The bandwidth peak is a measured copy; this file measures the arithmetic
// peaks the same way, with the library's own kernels: every thread runs CHAINS independent FMA
// chains (x = x * a + b, a flop count of 2 per FMA), enough resident warps per SM to cover the FMA
// latency, and the best of a few timed launches is reported.  The chains converge to a fixed point
// (|a| < 1), so no value overflows; a comparison against an impossible value keeps the compiler
// from removing the arithmetic.
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/nemo_gpu.h"

namespace nemo {
void set_last_error(const char* msg);
}

namespace {

constexpr int CHAINS = 8;
constexpr int UNROLL = 16;

template <typename T>
__global__ void __launch_bounds__(256) k_fma_peak(int64_t iters, T a, T b, T* sink) {
    T x[CHAINS];
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) x[c] = (T)(threadIdx.x + c) * (T)1e-3;
    for (int64_t it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < UNROLL; ++u)
#pragma unroll
            for (int c = 0; c < CHAINS; ++c) x[c] = fma(x[c], a, b);
    }
    T s = 0;
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) s += x[c];
    if (s == (T)-12345.0) sink[threadIdx.x] = s;   // never true: keeps the chains alive
}

template <typename T>
cudaError_t time_peak(int64_t iters, int grid, cudaStream_t st, T* sink, double* tflops) {
    cudaEvent_t e0, e1;
    cudaError_t err;
    if ((err = cudaEventCreate(&e0)) != cudaSuccess) return err;
    if ((err = cudaEventCreate(&e1)) != cudaSuccess) {
        cudaEventDestroy(e0);
        return err;
    }
    const T a = (T)0.999, b = (T)1e-3;
    k_fma_peak<T><<<grid, 256, 0, st>>>(iters / 8, a, b, sink);   // warm-up
    double best = 0.0;
    for (int rep = 0; rep < 3 && err == cudaSuccess; ++rep) {
        cudaEventRecord(e0, st);
        k_fma_peak<T><<<grid, 256, 0, st>>>(iters, a, b, sink);
        cudaEventRecord(e1, st);
        if ((err = cudaEventSynchronize(e1)) != cudaSuccess) break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double flops = 2.0 * CHAINS * UNROLL * (double)iters * grid * 256.0;
        if (ms > 0.f && flops / (ms * 1e-3) > best) best = flops / (ms * 1e-3);
    }
    if (err == cudaSuccess) err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *tflops = best * 1e-12;
    return err;
}

}  // namespace

/* out[0] = FP64 FMA peak (TFLOP/s), out[1] = FP32 FMA peak (TFLOP/s), out[2] = SM count,
   out[3] = SM clock (MHz) the device reports as its maximum. */
extern "C" int nemo_gpu_measure_peaks(double* out) {
    if (!out) {
        nemo::set_last_error("nemo_gpu_measure_peaks: out is NULL");
        return NEMO_ERR_ARG;
    }
    int dev = 0, nsm = 0, clk = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err == cudaSuccess) err = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (err == cudaSuccess) err = cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, dev);
    cudaStream_t st = nullptr;
    if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    void* sink = nullptr;
    if (err == cudaSuccess) err = cudaMalloc(&sink, 256 * sizeof(double));
    const int grid = nsm * 8;   // 8 CTAs of 256 threads: 64 warps per SM, 16 per scheduler
    double p64 = 0.0, p32 = 0.0;
    if (err == cudaSuccess) err = time_peak<double>(1 << 12, grid, st, (double*)sink, &p64);
    if (err == cudaSuccess) err = time_peak<float>(1 << 13, grid, st, (float*)sink, &p32);
    if (sink) cudaFree(sink);
    if (st) cudaStreamDestroy(st);
    if (err != cudaSuccess) {
        nemo::set_last_error(cudaGetErrorString(err));
        return NEMO_ERR_CUDA;
    }
    out[0] = p64;
    out[1] = p32;
    out[2] = nsm;
    out[3] = clk * 1e-3;
    return NEMO_OK;
}
