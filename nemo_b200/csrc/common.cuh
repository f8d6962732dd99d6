// common.cuh -- layout, constants and small device helpers shared by the sm_100a kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace nemo {

constexpr int NN = 4;             // Gauss-Lobatto nodes per direction (N = 3)
constexpr int NP = NN * NN * NN;  // nodes per element
constexpr int NF = NN * NN;       // nodes per face
constexpr int VMAX = 9;

// Per-run control block in device memory.  One entry per group (independent run of an
// ensemble); group 0 only for a single run.
constexpr int MAX_GROUPS = 1024;

struct Control {
    double dt[MAX_GROUPS];                    // time step of the current step
    double t[MAX_GROUPS];                     // simulation time
    unsigned long long dtmin_bits[MAX_GROUPS];// min over elements of delta/lambda (positive double bits)
    unsigned long long lmax_bits[MAX_GROUPS]; // max wave speed (positive double bits)
    double t_end;                             // > 0: clamp the last step
    double dt_factor;                         // 0.5^(D-1) * cfl / (2*N_NODES - 1)
    int32_t ngroups;
    int32_t done;                             // all groups reached t_end
    int32_t error;                            // bit 0: bounded TMA wait expired; bit 1: non-finite dt;
                                              // bit 2: bounded wait on a mortar flag expired
    int32_t pad;
    unsigned long long nbad;                  // elements whose positivity repair failed
    unsigned long long steps;
    unsigned long long fallback;              // elements that used the modal fallback (learned indicator)
    double judge_sum;                         // sum |alpha_learned - alpha_modal| over judged elements
    unsigned long long judge_n;               // number of judged elements
    double glm_ch;                            // GLM cleaning speed of the current step (MHD)
    double glm_alpha;                         // GLM damping of the current step (MHD)
    unsigned long long vmax_bits;             // max |velocity component| (positive double bits, MHD)
    int32_t mhd;                              // 1: update glm_ch/glm_alpha from lmax/vmax each step
    int32_t pad2;
    uint32_t epoch;                           // persistent stage launches: current launch number (>= 1)
    uint32_t work;                            // persistent stage launches: next task (reset by the last CTA)
    uint32_t exit_count;                      // persistent stage launches: CTAs finished
    uint32_t pad3;
};

// Learned indicator: packed MLP weights (W1[32][12], b1[32], W2[32][32], b2[32], W3[32], b3)
// followed by the lower and upper bounds of the 12 normalised inputs.
constexpr int MLP_NW = 32 * 12 + 32 + 32 * 32 + 32 + 32 + 1;
constexpr int MLP_NPACK = MLP_NW + 24;
// FP32 form: the same weights with W1 and W2 transposed ([12][32], [32][32]) followed by the input
// bounds, padded to whole float4s, stored after the packed copy; a CTA copies them to shared memory
// with float4 loads.
constexpr int MLP_NT = (MLP_NPACK + 3) / 4 * 4;

// Operator constants (filled once by nemo_gpu_init from the host-built matrices).
struct OpConsts {
    double S[NN * NN];     // split-form matrix 2D - W^-1 B, zero diagonal
    double winv[NN];       // 1/w_i on [-1,1]
    double Vinv[NN * NN];  // nodal -> modal (normalised Legendre)
    double wt[NN];         // weights on [-1/2,1/2] (totals)
    double kappa, km1;     // kappa, kappa - 1
    double c_enth;         // 0.5/(kappa-1)
    double hllc_beta;      // sqrt(0.5*(kappa-1)/kappa)
    double ind_T, ind_k;   // indicator threshold T and -s/T
    double alpha_min, alpha_max, one_m_alpha_min;
    double repair_decr;
    double mu0;
    int cool;              // barotropic cooling after every stage
    double cool_rho;       // dens_critical
    double cool_ci;        // k_isothermal / (kappa - 1)
    double cool_ca;        // k_adiabatic / (kappa - 1)
    double x[NN];            // Gauss-Lobatto nodes on [-1,1] (adapt: interpolation to descendants)
    double w[NN];            // their weights (adapt: element means)
    double pro[2][NN * NN];  // 2:1 mortar prolongation to the lower/upper half, [s][fine i][coarse j]
    double prj[2][NN * NN];  // 2:1 mortar projection from the lower/upper half, [s][coarse a][fine i]
    // FP32 copies for the FP32 kernels (rounded once here instead of converted at every use)
    float S32[NN * NN], winv32[NN], Vinv32[NN * NN];
    float kappa32, km1_32, ikm1_32, c_enth32, hllc_beta32;
    float ind_k32, ind_T32, alpha_min32, alpha_max32, one_m_alpha_min32;
};

// Operator matrix entries in the arithmetic type R of a kernel (the FP32 copies for float)
template <typename R>
__device__ __forceinline__ R op_S(const OpConsts& k, int i) {
    if constexpr (sizeof(R) == 4) return k.S32[i];
    else return k.S[i];
}
template <typename R>
__device__ __forceinline__ R op_winv(const OpConsts& k, int i) {
    if constexpr (sizeof(R) == 4) return k.winv32[i];
    else return k.winv[i];
}
template <typename R>
__device__ __forceinline__ R op_Vinv(const OpConsts& k, int i) {
    if constexpr (sizeof(R) == 4) return k.Vinv32[i];
    else return k.Vinv[i];
}

__host__ __device__ inline int nidx(int i, int j, int k) { return i + NN * (j + NN * k); }

// node index of line position i on the line (a,b) of direction d
__host__ __device__ inline int line_node(int d, int a, int b, int i) {
    return d == 0 ? nidx(i, a, b) : (d == 1 ? nidx(a, i, b) : nidx(a, b, i));
}

// LSRK 5-4 coefficients (Kennedy-Carpenter 2N), source/timedisc/rungekutta/low-storage/4-5/
// timedisc_const_mod.f90:5-29; A = a_rk, C = c_rk (weights), B = b_rk (stage times).
__host__ __device__ inline double rk_a(int s) {
    switch (s) {
        case 1: return -567301805773.0 / 1357537059087.0;
        case 2: return -2404267990393.0 / 2016746695238.0;
        case 3: return -3550918686646.0 / 2091501179385.0;
        case 4: return -1275806237668.0 / 842570457699.0;
        default: return 0.0;
    }
}
__host__ __device__ inline double rk_c(int s) {
    switch (s) {
        case 0: return 1432997174477.0 / 9575080441755.0;
        case 1: return 5161836677717.0 / 13612068292357.0;
        case 2: return 1720146321549.0 / 2090206949498.0;
        case 3: return 3134564353537.0 / 4481467310338.0;
        default: return 2277821191437.0 / 14882151754819.0;
    }
}

}  // namespace nemo
