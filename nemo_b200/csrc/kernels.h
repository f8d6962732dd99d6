// kernels.h -- argument blocks and launchers of the device kernels (internal to the library).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/nemo_gpu.h"
#include "common.cuh"

namespace nemo {

struct StageArgs {
    int64_t E;                // element stride of the SoA arrays
    int64_t E_begin;          // first element of this launch (0, or the first partition-boundary element)
    int64_t E_own;            // end of this launch's elements, at most the owned count ([owned, E) are
                              // ghost copies: neighbour data only)
    const double* u_in;       // [V][E][64]
    double* u_out;            // [V][E][64]
    double* reg;              // [V][E][64] LSRK register (FP64)
    const int32_t* nbr;       // [E][6] conforming face neighbours, -1 domain boundary, <= -2 mortar row -2-nbr
    const double* cdel;       // [E][3] 2/delta
    const double* delta;      // [E][3]
    const double* alpha_in;   // raw indicator of u_in [E] (blended runs)
    double* alpha_out;        // raw indicator of u_out [E] (epilogue) or null
    double* alpha_used;       // alpha applied in this stage [E] or null
    const int32_t* group;     // [E] or null (single run)
    Control* ctrl;
    double* rhs_out;          // rhs-only launches
    int32_t stage;            // 0..4
    int32_t epi_dt;           // last stage: CFL bound of the new state
    int32_t smooth;           // alpha smoothing
    int32_t positivity;
    int32_t surface_flux;
    int32_t volume_flux;
    int32_t prep_only;        // only the epilogue on u_in (indicator and CFL bound of a state)
    int32_t tick;             // this launch advances t and the step counter after the last stage
    const double* mlp64;      // learned indicator (FP64 values of the BF16 weights) or null
    const float* mlp32;       // same, FP32
    const float* mlp32t;      // FP32, W1 and W2 transposed (MLP_NT floats, 16-byte aligned)
    float* feat_out;          // FP32 form, prepare launches: indicator features [E][12] or null
    double* alpha_modal_out;  // FP32 form, prepare launches: modal alpha [E] or null
    const double* mflux;      // [5 M][V][16] mortar face fluxes in the face's rotated frame (mortar.cu)
    const uint32_t* mflag;    // [M] persistent launches: epoch at which a mortar's rows are complete
};

// 2:1 mortars (mortar.cu): per mortar, the coarse face flux (row 5m) and the four fine face fluxes
// (rows 5m+1+k) of the state u_in, before the stage kernel that reads them.
struct MortarArgs {
    int64_t E;
    int64_t nm;
    const double* u_in;       // [V][E][64]
    const int32_t* mortar;    // [nm][6]: coarse quad, coarse face, fine quads k = s + 2t
    double* mflux;            // [5 nm][V][16]
    const Control* ctrl;      // GLM cleaning speed (MHD); done flag
    int32_t mhd;
    int32_t surface_flux;
    int32_t skip_if_done;     // stage launches: nothing to do once the run reached t_end
    uint32_t* mflag;          // [nm] or null: set to epoch (release) once a mortar's rows are written
    uint32_t epoch;
};
cudaError_t setup_mortar(const OpConsts& ops);
// adapt: new SoA state [V][En][64] from the old one [V][Eo][64] by remap rows (kind, src, depth,
// offsets) -- copy, interpolation from an ancestor, projection of 8 children
cudaError_t launch_remap(const double* uo, int64_t Eo, double* un, int64_t En, const int32_t* remap, int nv,
                         int32_t* bad, cudaStream_t s);
cudaError_t launch_amr_flags(const double* u, int64_t E, double refine_thr, double coarsen_thr, int32_t* flags,
                             cudaStream_t s);
cudaError_t launch_mortar(const MortarArgs& a, cudaStream_t s);

// plain FP64 Euler path (stage_fp64.cu)
cudaError_t setup_stage_euler64(const OpConsts& ops);
cudaError_t launch_stage_euler64(const StageArgs& a, bool blend, bool ind, bool rhs_only, cudaStream_t s);
// conserved totals of the first n elements of an SoA state with element stride E
cudaError_t launch_totals64(const double* u, const double* delta, int64_t E, int64_t n, int nv, double* part,
                            double* out, cudaStream_t s);
int stage_smem_bytes64();
// positivity repair of element states [n][nv][64] (one element per warp), ok[e] = admissible after
cudaError_t launch_repair_states64(double* st, int64_t n, int nv, int mhd, int32_t* ok, cudaStream_t s);

// FP32-bulk Euler path (stage_fp32.cu)
cudaError_t setup_stage_euler32(const OpConsts& ops);
// epc: elements per CTA of the grid schedule, 4, 8 or 16
cudaError_t launch_stage_euler32(const StageArgs& a, bool blend, bool rhs_only, cudaStream_t s, int epc = 8);
// persistent FP32 stage with the mortar pairs as its first tasks (grid = CTAs, <= SMs x resident)
cudaError_t launch_stage_euler32p(const StageArgs& a, const MortarArgs& ma, bool blend, int grid, cudaStream_t s);
cudaError_t stage32p_max_ctas_per_sm(bool blend, int* n);
int stage_smem_bytes32(int epc);

// GLM-MHD stages (stage_mhd.cuh instantiated in stage_fp64.cu / stage_fp32.cu)
cudaError_t setup_stage_mhd64();
cudaError_t setup_stage_mhd32();
cudaError_t launch_stage_mhd64(const StageArgs& a, bool blend, bool rhs_only, cudaStream_t s);
cudaError_t launch_stage_mhd32(const StageArgs& a, bool blend, bool rhs_only, cudaStream_t s);

// learned-indicator training (mlp.cu)
cudaError_t mlp_grad_launch(const float* feat, const float* target, const int32_t* idx, int64_t n, const float* W,
                            float amax, float* grad, float* loss, cudaStream_t s);
cudaError_t mlp_adam_launch(float* W, const float* grad, float* m, float* v, int step, float lr, cudaStream_t s);
cudaError_t mlp_forward_launch(const float* feat, int64_t n, const float* W, float amax, float* out, cudaStream_t s);

// control kernels (control.cu)
// element exchange (partitioned runs): buf[m] = (state of element idx[m], V x 64, then its raw alpha)
cudaError_t launch_pack_faces(const double* u, const double* alpha, const int32_t* idx, const int32_t* face, int64_t n,
                              int64_t E, int nv, double* buf, cudaStream_t s);
cudaError_t launch_unpack_faces(double* u, double* alpha, const int32_t* idx, const int32_t* face, int64_t n, int64_t E,
                                int nv, const double* buf, cudaStream_t s);
cudaError_t launch_pack(const double* u, const double* alpha, const int32_t* idx, int64_t n, int64_t E, int nv,
                        double* buf, cudaStream_t s);
cudaError_t launch_unpack(double* u, double* alpha, const int32_t* idx, int64_t n, int64_t E, int nv,
                          const double* buf, cudaStream_t s);
cudaError_t launch_ctrl_reset(Control* c, cudaStream_t s);
cudaError_t launch_ctrl_set_dt(Control* c, double dt, cudaStream_t s);
cudaError_t launch_ctrl_step(Control* c, cudaStream_t s);
cudaError_t launch_aos_to_soa(const double* aos, double* soa, int64_t E, int nv, cudaStream_t s);
cudaError_t launch_soa_to_aos(const double* soa, double* aos, int64_t E, int nv, cudaStream_t s);

}  // namespace nemo
