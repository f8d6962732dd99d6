// mlp.cu -- training kernels of the learned shock indicator (forward, backward, Adam).
//
// Network: x = feat/10 + 1 (12 inputs), h1 = SiLU(W1 x + b1) (32), h2 = SiLU(W2 h1 + b2) (32),
// alpha = amax * sigmoid(W3 . h2 + b3); packed weights as in common.cuh (MLP_NW values, FP32
// master copy).  Loss: mean squared error of alpha against the modal indicator's alpha.
// One thread per sample: forward with the pre-activations kept in registers, backward on the fly;
// the per-sample gradient contributions are summed over the warp with shuffles and then over the
// block in shared memory before one atomic add per weight and block into the global gradient.
#include "kernels.h"

namespace nemo {

namespace {

constexpr int NI = 12, NH = 32;
constexpr int O_W1 = 0, O_B1 = NH * NI, O_W2 = O_B1 + NH, O_B2 = O_W2 + NH * NH, O_W3 = O_B2 + NH, O_B3 = O_W3 + NH;

__device__ __forceinline__ float sigm(float x) { return 1.0f / (1.0f + __expf(-x)); }

__device__ __forceinline__ void warp_add(float* sg, int k, float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&sg[k], v);
}

__global__ void __launch_bounds__(256) k_mlp_grad(const float* __restrict__ feat, const float* __restrict__ target,
                                                  const int32_t* __restrict__ idx, int64_t n,
                                                  const float* __restrict__ W, float amax, float inv_n,
                                                  float* __restrict__ grad, float* __restrict__ loss) {
    __shared__ float sg[MLP_NW];
    __shared__ float sl;
    for (int i = threadIdx.x; i < MLP_NW; i += blockDim.x) sg[i] = 0.f;
    if (threadIdx.x == 0) sl = 0.f;
    __syncthreads();
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool act = s < n;
    const int64_t row = act ? (idx ? (int64_t)idx[s] : s) : 0;
    float x[NI], p1[NH], p2[NH];
#pragma unroll
    for (int i = 0; i < NI; ++i) x[i] = act ? feat[row * NI + i] * 0.1f + 1.0f : 0.f;
#pragma unroll
    for (int j = 0; j < NH; ++j) {
        float a = W[O_B1 + j];
#pragma unroll
        for (int i = 0; i < NI; ++i) a += W[O_W1 + j * NI + i] * x[i];
        p1[j] = a;
    }
#pragma unroll 4
    for (int j = 0; j < NH; ++j) {
        float a = W[O_B2 + j];
#pragma unroll
        for (int i = 0; i < NH; ++i) a += W[O_W2 + j * NH + i] * (p1[i] * sigm(p1[i]));
        p2[j] = a;
    }
    float z = W[O_B3];
#pragma unroll
    for (int j = 0; j < NH; ++j) z += W[O_W3 + j] * (p2[j] * sigm(p2[j]));
    const float sz = sigm(z);
    const float out = amax * sz;
    const float r = act ? out - target[row] : 0.f;
    // loss
    {
        float v = r * r * inv_n;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(&sl, v);
    }
    const float dz = 2.0f * r * inv_n * amax * sz * (1.0f - sz);
    warp_add(sg, O_B3, dz);
    // layer 3 and dpre2
    float d2[NH];
#pragma unroll
    for (int j = 0; j < NH; ++j) {
        const float sj = sigm(p2[j]);
        const float h2 = p2[j] * sj;
        warp_add(sg, O_W3 + j, dz * h2);
        d2[j] = dz * W[O_W3 + j] * (sj * (1.0f + p2[j] * (1.0f - sj)));
        warp_add(sg, O_B2 + j, d2[j]);
    }
    // layer 2 weights
#pragma unroll 1
    for (int j = 0; j < NH; ++j)
#pragma unroll
        for (int i = 0; i < NH; ++i) warp_add(sg, O_W2 + j * NH + i, d2[j] * (p1[i] * sigm(p1[i])));
    // layer 1
#pragma unroll 1
    for (int i = 0; i < NH; ++i) {
        float dh = 0.f;
#pragma unroll
        for (int j = 0; j < NH; ++j) dh += d2[j] * W[O_W2 + j * NH + i];
        const float si = sigm(p1[i]);
        const float d1 = dh * (si * (1.0f + p1[i] * (1.0f - si)));
        warp_add(sg, O_B1 + i, d1);
#pragma unroll
        for (int q = 0; q < NI; ++q) warp_add(sg, O_W1 + i * NI + q, d1 * x[q]);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < MLP_NW; i += blockDim.x) atomicAdd(&grad[i], sg[i]);
    if (threadIdx.x == 0 && loss) atomicAdd(loss, sl);
}

__global__ void k_mlp_adam(float* __restrict__ W, const float* __restrict__ g, float* __restrict__ m,
                           float* __restrict__ v, float lr, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= MLP_NW) return;
    const float b1 = 0.9f, b2 = 0.999f;
    m[i] = b1 * m[i] + (1.0f - b1) * g[i];
    v[i] = b2 * v[i] + (1.0f - b2) * g[i] * g[i];
    W[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + 1e-8f);
}

__global__ void k_mlp_fwd(const float* __restrict__ feat, int64_t n, const float* __restrict__ W, float amax,
                          float* __restrict__ out) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float x[NI], h1[NH];
#pragma unroll
    for (int i = 0; i < NI; ++i) x[i] = feat[s * NI + i] * 0.1f + 1.0f;
#pragma unroll
    for (int j = 0; j < NH; ++j) {
        float a = W[O_B1 + j];
#pragma unroll
        for (int i = 0; i < NI; ++i) a += W[O_W1 + j * NI + i] * x[i];
        h1[j] = a * sigm(a);
    }
    float z = W[O_B3];
#pragma unroll 4
    for (int j = 0; j < NH; ++j) {
        float a = W[O_B2 + j];
#pragma unroll
        for (int i = 0; i < NH; ++i) a += W[O_W2 + j * NH + i] * h1[i];
        z += W[O_W3 + j] * (a * sigm(a));
    }
    out[s] = amax * sigm(z);
}

}  // namespace

cudaError_t mlp_grad_launch(const float* feat, const float* target, const int32_t* idx, int64_t n, const float* W,
                            float amax, float* grad, float* loss, cudaStream_t s) {
    const unsigned blocks = (unsigned)((n + 255) / 256);
    k_mlp_grad<<<blocks, 256, 0, s>>>(feat, target, idx, n, W, amax, 1.0f / (float)n, grad, loss);
    return cudaGetLastError();
}

cudaError_t mlp_adam_launch(float* W, const float* grad, float* m, float* v, int step, float lr, cudaStream_t s) {
    const float c1 = 1.0f - powf(0.9f, (float)step), c2 = 1.0f - powf(0.999f, (float)step);
    k_mlp_adam<<<(MLP_NW + 255) / 256, 256, 0, s>>>(W, grad, m, v, lr, c1, c2);
    return cudaGetLastError();
}

cudaError_t mlp_forward_launch(const float* feat, int64_t n, const float* W, float amax, float* out, cudaStream_t s) {
    k_mlp_fwd<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(feat, n, W, amax, out);
    return cudaGetLastError();
}

}  // namespace nemo
