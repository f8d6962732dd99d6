// control.cu -- small kernels that manage the device-side run control and the state layout.
#include "kernels.h"

namespace nemo {

namespace {

constexpr unsigned long long POS_INF_BITS = 0x7FF0000000000000ull;

__global__ void k_ctrl_reset(Control* c) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < c->ngroups) {
        c->dtmin_bits[g] = POS_INF_BITS;
        c->lmax_bits[g] = 0ull;
    }
    if (g == 0) c->vmax_bits = 0ull;
}

__global__ void k_ctrl_set_dt(Control* c, double dt) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < c->ngroups) c->dt[g] = dt;
    if (g == 0) c->done = 0;
}

// hook_calc_timestep for the next step, from the CFL bounds accumulated by the previous
// step's last stage (or by a prepare launch): dt = factor * min(delta/lambda), clamped to t_end.
__global__ void k_ctrl_step(Control* c) {
    __shared__ int s_live;
    if (threadIdx.x == 0) {
        s_live = 0;
        if (c->mhd) {  // GLM cleaning speed and damping of this step (kernel_timestep_mod.f90:338-344)
            const double lmax = __longlong_as_double((long long)c->lmax_bits[0]);
            const double vmax = __longlong_as_double((long long)c->vmax_bits);
            c->glm_ch = 2.0 * fabs(lmax - vmax);
            c->glm_alpha = c->glm_ch / 0.18;
            c->vmax_bits = 0ull;
        }
    }
    __syncthreads();
    for (int g = threadIdx.x; g < c->ngroups; g += blockDim.x) {
        const double dtmin = __longlong_as_double((long long)c->dtmin_bits[g]);
        double dt = c->dt_factor * dtmin;
        const double t = c->t[g];
        if (c->t_end > 0.0) {
            if (t >= c->t_end) dt = 0.0;
            else {
                if (t + dt > c->t_end) dt = c->t_end - t;
                atomicOr(&s_live, 1);
            }
        } else {
            atomicOr(&s_live, 1);
        }
        if (!(dt >= 0.0) || isinf(dt)) {
            atomicOr(&c->error, 2);
            dt = 0.0;
        }
        c->dt[g] = dt;
        c->dtmin_bits[g] = POS_INF_BITS;
        c->lmax_bits[g] = 0ull;
    }
    __syncthreads();
    if (threadIdx.x == 0) c->done = (s_live == 0 || c->error) ? 1 : 0;
}

// aos[e][v][n] <-> soa[v][e][n]
__global__ void k_aos_to_soa(const double* __restrict__ aos, double* __restrict__ soa, int64_t E, int nv) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t total = E * nv * NP;
    if (i >= total) return;
    const int64_t n = i % NP, v = (i / NP) % nv, e = i / ((int64_t)NP * nv);
    soa[(v * E + e) * NP + n] = aos[i];
}

__global__ void k_soa_to_aos(const double* __restrict__ soa, double* __restrict__ aos, int64_t E, int nv) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t total = E * nv * NP;
    if (i >= total) return;
    const int64_t n = i % NP, v = (i / NP) % nv, e = i / ((int64_t)NP * nv);
    aos[i] = soa[(v * E + e) * NP + n];
}

// element exchange buffers: per listed element its V x 64 state values and its raw indicator
__global__ void k_pack(const double* __restrict__ u, const double* __restrict__ alpha, const int32_t* __restrict__ idx,
                       int64_t n, int64_t E, int nv, double* __restrict__ buf) {
    const int64_t row = (int64_t)nv * NP + 1;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * row) return;
    const int64_t m = i / row, r = i % row;
    const int64_t e = idx[m];
    buf[i] = r < (int64_t)nv * NP ? u[((r / NP) * E + e) * NP + r % NP] : (alpha ? alpha[e] : 0.0);
}

__global__ void k_unpack(double* __restrict__ u, double* __restrict__ alpha, const int32_t* __restrict__ idx,
                         int64_t n, int64_t E, int nv, const double* __restrict__ buf) {
    const int64_t row = (int64_t)nv * NP + 1;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * row) return;
    const int64_t m = i / row, r = i % row;
    const int64_t e = idx[m];
    if (r < (int64_t)nv * NP) u[((r / NP) * E + e) * NP + r % NP] = buf[i];
    else if (alpha) alpha[e] = buf[i];
}

// face exchange buffers: per listed (element, face) the V x 16 trace values of that face (node order
// of line_node) and the element's raw indicator; entries outside [0, E) x [0, 6) are skipped
__device__ __forceinline__ int face_node(int f, int j) { return line_node(f >> 1, j & 3, j >> 2, (f & 1) ? NN - 1 : 0); }

__global__ void k_pack_faces(const double* __restrict__ u, const double* __restrict__ alpha,
                             const int32_t* __restrict__ idx, const int32_t* __restrict__ face, int64_t n, int64_t E,
                             int nv, double* __restrict__ buf) {
    const int64_t row = (int64_t)nv * NF + 1;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * row) return;
    const int64_t m = i / row, r = i % row;
    const int64_t e = idx[m];
    const int f = face[m];
    if (e < 0 || e >= E || f < 0 || f > 5) return;
    buf[i] = r < (int64_t)nv * NF ? u[((r / NF) * E + e) * NP + face_node(f, (int)(r % NF))] : (alpha ? alpha[e] : 0.0);
}

__global__ void k_unpack_faces(double* __restrict__ u, double* __restrict__ alpha, const int32_t* __restrict__ idx,
                               const int32_t* __restrict__ face, int64_t n, int64_t E, int nv,
                               const double* __restrict__ buf) {
    const int64_t row = (int64_t)nv * NF + 1;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * row) return;
    const int64_t m = i / row, r = i % row;
    const int64_t e = idx[m];
    const int f = face[m];
    if (e < 0 || e >= E || f < 0 || f > 5) return;
    if (r < (int64_t)nv * NF) u[((r / NF) * E + e) * NP + face_node(f, (int)(r % NF))] = buf[i];
    else if (alpha) alpha[e] = buf[i];
}

}  // namespace

cudaError_t launch_pack_faces(const double* u, const double* alpha, const int32_t* idx, const int32_t* face, int64_t n,
                              int64_t E, int nv, double* buf, cudaStream_t s) {
    const int64_t total = n * ((int64_t)nv * NF + 1);
    if (total > 0) k_pack_faces<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(u, alpha, idx, face, n, E, nv, buf);
    return cudaGetLastError();
}

cudaError_t launch_unpack_faces(double* u, double* alpha, const int32_t* idx, const int32_t* face, int64_t n, int64_t E,
                                int nv, const double* buf, cudaStream_t s) {
    const int64_t total = n * ((int64_t)nv * NF + 1);
    if (total > 0) k_unpack_faces<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(u, alpha, idx, face, n, E, nv, buf);
    return cudaGetLastError();
}

cudaError_t launch_pack(const double* u, const double* alpha, const int32_t* idx, int64_t n, int64_t E, int nv,
                        double* buf, cudaStream_t s) {
    const int64_t total = n * ((int64_t)nv * NP + 1);
    if (total > 0) k_pack<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(u, alpha, idx, n, E, nv, buf);
    return cudaGetLastError();
}

cudaError_t launch_unpack(double* u, double* alpha, const int32_t* idx, int64_t n, int64_t E, int nv,
                          const double* buf, cudaStream_t s) {
    const int64_t total = n * ((int64_t)nv * NP + 1);
    if (total > 0) k_unpack<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(u, alpha, idx, n, E, nv, buf);
    return cudaGetLastError();
}

cudaError_t launch_ctrl_reset(Control* c, cudaStream_t s) {
    k_ctrl_reset<<<MAX_GROUPS / 256, 256, 0, s>>>(c);
    return cudaGetLastError();
}

cudaError_t launch_ctrl_set_dt(Control* c, double dt, cudaStream_t s) {
    k_ctrl_set_dt<<<MAX_GROUPS / 256, 256, 0, s>>>(c, dt);
    return cudaGetLastError();
}

cudaError_t launch_ctrl_step(Control* c, cudaStream_t s) {
    k_ctrl_step<<<1, 256, 0, s>>>(c);
    return cudaGetLastError();
}

cudaError_t launch_aos_to_soa(const double* aos, double* soa, int64_t E, int nv, cudaStream_t s) {
    const int64_t total = E * nv * NP;
    k_aos_to_soa<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(aos, soa, E, nv);
    return cudaGetLastError();
}

cudaError_t launch_soa_to_aos(const double* soa, double* aos, int64_t E, int nv, cudaStream_t s) {
    const int64_t total = E * nv * NP;
    k_soa_to_aos<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(soa, aos, E, nv);
    return cudaGetLastError();
}

}  // namespace nemo
