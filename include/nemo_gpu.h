/*
 * nemo_gpu.h -- C-ABI of the B200 spatial operator for nemo (jmark/nemo).
 *
 * The reference drives its spatial operator through Fortran hook modules that the
 * build registry wires together at compile time (scripts/nemo.py:245-305).  The GPU
 * module replaces three of them:
 *
 *   hook_calc_timestep_200   source/kernel/mcfv/3d/kernel_timestep_mod.f90:17-58
 *   hook_pre_rk_timestep_300 source/kernel/mcfv/3d/kernel_hooks_mod.f90:7-20
 *   hook_mid_rk_timestep_500 source/timedisc/rungekutta/low-storage/4-5/timedisc_hooks_mod.f90:51-58
 *
 * and calls this library through iso_c_binding interfaces in the style of the p4wrap
 * bindings (source/mesh/p4est/wrapper/p4wrap_interfaces_mod.f90).  Every entry point is
 * plain C: pointers, sizes and scalars only, and returns an int status (0 = OK).  No C++
 * exception crosses the boundary; on a non-zero status nemo_gpu_last_error() yields the
 * message, and the Fortran shim forwards it to raise_error (source/utils/status_mod.f90:7-21).
 *
 * Data conventions (match the reference's):
 *   - one element ("quad") holds N_NODES^3 Gauss-Lobatto nodes, Fortran order state(i,j,k,v),
 *     i fastest (x), then j (y), k (z), then the variable; variables rho, rho*u, rho*v, rho*w, E
 *     (source/equations/euler/equations_const_mod.f90:7-16) or the 9 GLM-MHD variables
 *     (source/equations/mhd/equations_const_mod.f90:7-29);
 *   - face ids NOR,SOU = x-/x+, WES,EAS = y-/y+, FRO,BAC = z-/z+ are 1..6 on the Fortran side
 *     (source/utils/constants_mod.f90:33-40) and 0..5 in this header;
 *   - du/dt = rhs, the time integrator is the 2N low-storage RK 5-4 of Kennedy-Carpenter
 *     (source/timedisc/rungekutta/low-storage/4-5/timedisc_const_mod.f90:5-29).
 *
 * Threading: call from one host thread; the library owns one CUDA stream and all device
 * memory.  The state on the device is authoritative between upload and download.
 */
#ifndef NEMO_GPU_H
#define NEMO_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- configuration ------------------------------------------------------------------ */

enum nemo_eqn        { NEMO_EQN_EULER = 0, NEMO_EQN_MHD = 1 };
/* two-point volume fluxes: source/equations/euler/two_point/{chandrashekar,standard},
   source/equations/mhd/two_point/ec */
enum nemo_volflux    { NEMO_VOLFLUX_CHANDRASHEKAR = 0, NEMO_VOLFLUX_CENTRAL = 1, NEMO_VOLFLUX_EC_MHD = 2 };
/* surface fluxes: source/equations/euler/riemann/{hllc,rusanov}, source/equations/mhd/riemann/{hlld,rusanov} */
enum nemo_surfflux   { NEMO_SURFFLUX_HLLC = 0, NEMO_SURFFLUX_RUSANOV = 1, NEMO_SURFFLUX_HLLD = 2 };
/* arithmetic of the flux bulk; conserved-variable RK registers are FP64 in every mode */
enum nemo_precision  { NEMO_PREC_FP64 = 0, NEMO_PREC_FP32 = 1 };
/* DG/FV blending coefficient alpha: none, modal-energy indicator, learned MLP (modal fallback) */
enum nemo_indicator  { NEMO_IND_NONE = 0, NEMO_IND_MODAL = 1, NEMO_IND_LEARNED = 2 };
/* source terms applied after every stage (hook_post_rk_timestep): barotropic cooling resets the
   energy to the barotropic equation of state, source/physics/cooling/barotropic_cooling_mod.f90:39-53 */
enum nemo_source     { NEMO_SOURCE_NONE = 0, NEMO_SOURCE_BAROTROPIC_COOLING = 1 };

enum nemo_face { NEMO_NOR = 0, NEMO_SOU = 1, NEMO_WES = 2, NEMO_EAS = 3, NEMO_FRO = 4, NEMO_BAC = 5 };

enum nemo_status {
    NEMO_OK = 0,
    NEMO_ERR_ARG = 1,          /* bad argument (size, null pointer, unsupported option) */
    NEMO_ERR_STATE = 2,        /* call out of order (no init / no mesh / no state) */
    NEMO_ERR_CUDA = 3,         /* a CUDA runtime call failed */
    NEMO_ERR_REPAIR = 4,       /* positivity repair failed on at least one element */
    NEMO_ERR_NONFINITE = 5     /* non-finite time step or state */
};

typedef struct nemo_cfg {
    int32_t n_nodes;          /* Gauss-Lobatto nodes per direction (N+1); 4 is compiled */
    int32_t n_vars;           /* 5 (Euler) or 9 (GLM-MHD) */
    int32_t eqn;              /* enum nemo_eqn */
    int32_t volume_flux;      /* enum nemo_volflux */
    int32_t surface_flux;     /* enum nemo_surfflux */
    int32_t precision;        /* enum nemo_precision */
    int32_t indicator;        /* enum nemo_indicator */
    int32_t alpha_smoothing;  /* 1: alpha_e = max(alpha_e, 0.5 * max over face neighbours) */
    int32_t positivity;       /* 1: element-tile squeeze repair after every stage
                                 (source/kernel/mcfv/3d/kernel_validate_mod.f90:159-272) */
    int32_t non_conservative; /* MHD: add the Powell/GLM non-conservative term */
    int32_t source;           /* enum nemo_source (Euler only) */
    int32_t pad_;
    double  kappa;            /* ratio of specific heats (setup_config_mod kappa) */
    double  mu0;              /* magnetic permeability (MHD) */
    double  cfl;              /* CFL number used by nemo_gpu_calc_timestep / run */
    double  alpha_max;        /* upper clip of alpha (0.5) */
    double  alpha_min;        /* alpha below this is set to 0 (0.001) */
    double  repair_decr;      /* squeeze decrement of the repair (0.01, kernel_config_mod.f90:5) */
    double  glm_ch;           /* GLM cleaning speed (MHD); updated by calc_timestep */
    double  glm_alpha;        /* GLM damping (MHD); updated by calc_timestep */
    double  dens_critical;    /* barotropic cooling: rho <= dens_critical is isothermal */
    double  k_isothermal;     /* barotropic cooling: p = k_isothermal rho below dens_critical */
    double  k_adiabatic;      /* barotropic cooling: p = k_adiabatic rho^kappa above it */
    double  reserved;
} nemo_cfg;

/* Fill *cfg with the defaults of the Euler DGSEM path (N=3, Chandrashekar, HLLC, FP64). */
int nemo_gpu_default_cfg(nemo_cfg* cfg);

/* hook_init_400 (source/kernel/dgsem/weakform/2d/kernel_hooks_mod.f90:7-13 ->
   kernel_share_mod.f90:56-151): build the Gauss-Lobatto operators and select the device. */
int nemo_gpu_init(const nemo_cfg* cfg);

/* Operator matrices as kernel_share_mod exports them, computed on the host without a GPU:
   nodes/weights on [-1,1] (n), D (n*n, row-major D[i*n+m] = l_m'(x_i)), the split-form
   matrix S = 2D - W^-1 B (n*n), the modal transform inverse Vandermonde Vinv (n*n). */
int nemo_gpu_operators(int32_t n, double* nodes, double* weights, double* dmat, double* smat,
                       double* vinv);

/* 2:1 mortar matrices (kernel_operators_interpolationMatrix and _projectionMatrix with Q = 2,
   source/kernel/dgsem/weakform/2d/kernel_operators_mod.f90:1010-1054, :1056-1100), computed on
   the host without a GPU: prolong[2][n][n] (lower/upper half, [s][fine node][coarse node]) and
   project[2][n][n] ([s][coarse node][fine node]); either pointer may be NULL. */
int nemo_gpu_mortar_operators(int32_t n, double* prolong, double* project);

/* Mesh in the reference's side form (source/mesh/p4est/mesh_types_mod.f90:57-77):
     delta[nelems*3], center[nelems*3]            element sizes and centres
     side_quads[nsides*2*4]                        0-based element ids, [side][iside][iquad]
     side_faceid[nsides*2]                         face id (0..5) of the side as seen by each element
     side_nquads[nsides*2]                         1, or 4 on the fine side of a 2:1 mortar, 0 at a boundary
     boundary[nsides]                              0 = interior, else 1 + face id of the domain face
   The element order is the order of the state arrays.  Sides with nquads 4 on one half are
   2:1 mortars (kernel_fill_faceflux, source/kernel/mcfv/3d/kernel_flux_mod.f90:100-118, 252-269):
   iquad k = s + 2t runs over the fine elements, s = lower/upper half along the face's first
   tangential axis (the lower-numbered of the two axes other than the face normal), t along the
   second -- the rfaceMat/rfaceTam pairing of source/kernel/mcfv/3d/kernel_share_mod.f90:36-60.
   All elements are axis-aligned in one frame (no tree rotations).  Each stage then runs a mortar
   kernel before the stage kernel: coarse trace prolonged to the four sub-faces, Riemann flux on
   every sub-face node, the fine faces take it and the coarse face takes its L2 projection. */
int nemo_gpu_set_mesh(int64_t nelems, const double* delta, const double* center, int64_t nsides,
                      const int32_t* side_quads, const int8_t* side_faceid,
                      const int8_t* side_nquads, const int32_t* boundary);

/* Independent runs batched in one mesh (ensembles): group id per element, 0..ngroups-1.
   Each group gets its own time step and simulation time.  Default: one group. */
int nemo_gpu_set_groups(int32_t ngroups, const int32_t* group_of_elem);

/* Element partition across processes (the reference partitions quads over MPI ranks with p4est and
   exchanges the partition-boundary payloads, source/mesh/p4est/mesh_utils_mod.f90:623-675, 1014-).
   Elements [0, n_owned) of this process's mesh are advanced; [n_owned, nelems) are ghost copies of
   other processes' elements that only serve as face neighbours (and mortar partners).  The caller
   refreshes the ghosts before every stage: nemo_gpu_pack_elements gathers the listed elements of the
   current state into buf_dev ([n][n_vars*64 + 1] doubles: the element's state, then its raw blending
   coefficient), nemo_gpu_unpack_elements scatters such a buffer into the listed (ghost) elements.
   idx_dev and buf_dev are device pointers; both calls return after the copy has completed.  The
   time step of a partitioned run is the minimum over processes of nemo_gpu_calc_timestep. */
int nemo_gpu_set_owned(int64_t n_owned);

/* AMR adapt between steps (mesh_adapt, source/mesh/p4est/mesh_utils_mod.f90:879-1010, called by a
   setup's hook_pre_timestep_300; payload transfer of kernel_amr_refine / kernel_amr_coarsen,
   source/kernel/dgsem/weakform/2d/kernel_amr_mod.f90:12-73, in 3D as in the replace callbacks of
   source/setups/euler/3d/sedov/setup_amr_mod.f90:67-125).  The host rebuilds the forest; the new mesh
   comes in set_mesh form, plus remap[nelems][4] int32 rows (kind, src, depth, offsets): kind 0 copies
   old element src; kind 1 interpolates the polynomial of old element src, an ancestor depth levels up
   (1..7), at the nodes of the new element, which sits at offsets ox | oy << 8 | oz << 16 inside it;
   kind 2 takes the sum of the DG projections of the 8 old children src .. src + 7 (child
   c = sx + 2 sy + 4 sz).  A transferred element that is not admissible falls back to the mean: all
   elements refined from that ancestor take its mean, a coarsened element the mean of its children
   (the reference steps down through lower orders, :82-95 and :114-124).  The state is remapped on the
   device, the mesh replaced, the simulation time kept; groups and ghost elements are not supported.
   Rows are checked before anything on the device changes (NEMO_ERR_ARG). */
int nemo_gpu_adapt(int64_t nelems, const double* delta, const double* center, int64_t nsides,
                   const int32_t* side_quads, const int8_t* side_faceid, const int8_t* side_nquads,
                   const int32_t* boundary, const int32_t* remap);
/* Adapt flags of the current state, computed on the device (the density probes of the Sedov setup,
   setup_amr_probe_refine / setup_amr_probe_coarsen, source/setups/euler/3d/sedov/setup_amr_mod.f90:
   23-65): flags[e] = +1 if some node's density exceeds refine_threshold, else -1 if no node's density
   exceeds coarsen_threshold, else 0.  flags is a host array of nelems int32; a family of 8 leaves
   coarsens when all of its members hold -1.  Only the flags cross to the host. */
int nemo_gpu_amr_flags(double refine_threshold, double coarsen_threshold, int32_t* flags);
int nemo_gpu_pack_elements(const int32_t* idx_dev, int64_t n, double* buf_dev);
int nemo_gpu_unpack_elements(const int32_t* idx_dev, int64_t n, const double* buf_dev);
/* The face form of the ghost refresh (the reference sends whole payloads; only the traces on the
   faces that a process's own elements or mortars touch, and the raw blending coefficient, are
   read from a ghost): for each listed (element idx_dev[i], face face_dev[i]) buf_dev holds a row of
   n_vars*16 + 1 doubles, the 16 face nodes of every variable (j = a + 4 b over the face's two
   tangential directions in increasing order) and then the element's raw blending coefficient.
   Entries outside [0, nelems) x [0, 6) are skipped.  Device pointers; both calls return after the
   copy has completed. */
int nemo_gpu_pack_faces(const int32_t* idx_dev, const int32_t* face_dev, int64_t n, double* buf_dev);
int nemo_gpu_unpack_faces(const int32_t* idx_dev, const int32_t* face_dev, int64_t n, const double* buf_dev);

/* A stage in two parts, so that a partitioned host overlaps its ghost exchange with work: with the
   owned elements ordered so that [0, n_interior) read no ghost data (neither a conforming neighbour
   nor a quad of a 2:1 mortar is a ghost), nemo_gpu_stage_interior enqueues the stage for those
   elements and returns at once; the host refreshes the ghosts (its own exchange, then
   nemo_gpu_unpack_faces / _elements), and nemo_gpu_stage_boundary advances the rest, waits, and
   reports as nemo_gpu_stage.  The two parts give the results of nemo_gpu_stage bit for bit (each
   element's update reads only its own state and its neighbours' traces).  n_interior = 0 (the
   default, and after nemo_gpu_set_owned) runs everything in the boundary part.  Needs the grid
   stage schedule.  The reference exchanges first and then computes
   (source/mesh/p4est/mesh_utils_mod.f90:650-664, source/timedisc/rungekutta/timedisc_evolve_mod.f90:20-84). */
int nemo_gpu_set_interior(int64_t n_interior);
int nemo_gpu_stage_interior(int32_t stage, double dt);
int nemo_gpu_stage_boundary(int32_t stage, double dt, int32_t* nbad_out);

/* GLM-MHD on partitioned hosts: the wave-speed and velocity maxima of the state's CFL evaluation
   (after nemo_gpu_calc_timestep) and the cleaning speed / damping of the coming step, which a
   partitioned host sets from the all-reduced maxima, c_h = 2 |lmax - vmax|, alpha = c_h / 0.18
   (source/kernel/mcfv/3d/kernel_timestep_mod.f90:48-52, :338-344). */
int nemo_gpu_glm_speeds(double* lmax_out, double* vmax_out);
int nemo_gpu_set_glm(double ch, double alpha);

/* Copy the conserved state host->device.  host points at the first element's state(1,1,1,1);
   consecutive elements are elem_stride_bytes apart (sizeof(quad_t) when the state sits in the
   reference's quad_t array, n^3*V*8 for a packed [E][V][n^3] array).  Resets the RK register. */
int nemo_gpu_upload_state(const double* host, int64_t elem_stride_bytes);
int nemo_gpu_download_state(double* host, int64_t elem_stride_bytes);

/* Asynchronous form of nemo_gpu_upload_state for hosts that stream independent states through the
   library (ensemble members, parameter sweeps, a state per step): the host->device copy runs on the
   library's upload stream into one of two staging slots and returns at once; the library stream
   takes the new state in stream order (work enqueued before the call still sees the old state, work
   enqueued after it the new one, as a new run: time 0, register cleared).  So the copy of the next
   state overlaps the stage work of the current one and, with nemo_gpu_download_state_async, the
   copy of its result.  host must be pinned (cudaHostAlloc or
   cudaHostRegister) for the copy to be asynchronous, and must not be modified before
   nemo_gpu_upload_wait returns (or before the second-next call of this function, which reuses the
   slot).  Same layout and stride rules as nemo_gpu_upload_state.  No reference counterpart: the
   reference's state lives in host memory. */
int nemo_gpu_upload_state_async(const double* host, int64_t elem_stride_bytes);

/* Wait until the host->device copies of every asynchronous upload have finished (their host
   buffers may then be reused). */
int nemo_gpu_upload_wait(void);

/* Asynchronous form of nemo_gpu_download_state: the state after all work enqueued so far is copied
   in stream order into one of two staging slots and from there to host on the library's download
   stream; the call returns at once (it waits only when the slot's copy of two calls ago is still
   running).  host should be pinned and must not be read before nemo_gpu_sync returns.  With
   nemo_gpu_upload_state_async and nemo_gpu_run_async the copies in both directions overlap the
   steps of other states.  No reference counterpart. */
int nemo_gpu_download_state_async(double* host, int64_t elem_stride_bytes);

/* Checkpoint staging (the state that hook_checkpoint_fill writes, source/checkpoint/flash/
   checkpoint_mod.f90:319-364, and the restart that source/nemo_prog.f90:107-114 leaves as a TODO).
   nemo_gpu_checkpoint_begin takes a snapshot of the state, of t (group 0) and of the step counter in
   stream order -- after everything enqueued before it -- into a library-owned device buffer, starts
   the device->host copy into host (layout as download_state) on a second stream and returns; later
   steps run while the copy proceeds.  host must stay valid, and should be page-locked for the copy
   to overlap, until nemo_gpu_checkpoint_wait returns the snapshot's t and step count.  A second
   begin first waits for the previous copy.  nemo_gpu_set_time restores t (every group) and the step
   counter after an upload_state, which resets both: upload + set_time is the restart.  alpha_host
   (optional, nelems doubles) receives the blending coefficients of the last stage (zeros without an
   indicator), copied with the state. */
int nemo_gpu_checkpoint_begin(double* host, int64_t elem_stride_bytes, double* alpha_host);
int nemo_gpu_checkpoint_wait(double* t_out, int64_t* steps_out);
int nemo_gpu_set_time(double t, int64_t steps);

/* hook_calc_timestep_200: dt = 0.5^(D-1) * cfl / (2*N_NODES-1) * min_e min_d (delta_d / lambda_d),
   lmax = max wave speed.  Device reduction in FP64.  dt_out/lmax_out are host pointers. */
int nemo_gpu_calc_timestep(double cfl, double* dt_out, double* lmax_out);

/* One RK stage (hook_pre_rk_timestep_300 + hook_mid_rk_timestep_500): rhs of the current
   state, register update, state update, positivity repair.  stage is 1..5 as rt%rkstage.
   nbad_out (may be NULL) receives the number of elements whose repair failed. */
int nemo_gpu_stage(int32_t stage, double dt, double t_stage, int32_t* nbad_out);

/* Enqueue nsteps full time steps with the device-side dt (as nemo_gpu_run without an end time) on
   the library stream and return without waiting: with nemo_gpu_upload_state_async before and
   nemo_gpu_download_state_async after it, a host streams states through the library with the
   copies of one state overlapping the steps of another.  Errors the device reports while these steps run
   (bounded waits, a non-finite dt) come back from the next nemo_gpu_sync or nemo_gpu_run; repair
   failures are counted in nemo_gpu_status.  Not in timing mode.  No reference counterpart. */
int nemo_gpu_run_async(int64_t nsteps);

/* Wait for all work the library has enqueued (steps, asynchronous uploads and downloads, checkpoint
   copies) and return the status the device reported for it. */
int nemo_gpu_sync(void);

/* One full time step (5 stages) with the given dt, replayed from a captured CUDA graph. */
int nemo_gpu_step(double dt);

/* Run nsteps time steps, or until t_end if t_end > 0 (the last step is clamped), with dt
   computed on the device before every step (hook_calc_timestep then hook_evolve).  The loop
   is captured as CUDA graphs; the host syncs once.  t_out, steps_out may be NULL. */
int nemo_gpu_run(int64_t nsteps, double t_end, double* t_out, int64_t* steps_out);

/* kernel_calc_flux for every element: rhs (packed [E][V][n^3] host array) of the current
   state, without updating it (source/kernel/mcfv/3d/kernel_flux_mod.f90:280-500). */
int nemo_gpu_rhs(double* rhs_host);

/* AMR operator matrices for hosts that transfer quad payloads themselves (the setups' replace
   callbacks, source/setups/euler/3d/sedov/setup_amr_mod.f90:67-125, through kernel_share_mod's
   refineMat / coarseMat): Fortran-layout arrays (n, n, 3, 8, 0:qmax), first index fastest.
   refine(:,:,d,f,q) maps a parent's nodal values along direction d to child f's (f = cx + 2 cy +
   4 cz, 0-based here, p4est child order) after truncating the parent to its Legendre modes 0..q
   in that direction; coarsen(:,:,d,f,q) maps child f's nodal values to its L2 projection onto the
   parent (Gauss-Lobatto quadrature), truncated the same way; summing blockmulXYZ(coarsen(..f..))
   over the 8 children gives the parent.  At q = n-1 these are the interpolation and projection of
   nemo_gpu_adapt; q = 0 gives element means.  0 <= qmax <= n-1; either output may be NULL. */
int nemo_gpu_amr_operators(int32_t n, int32_t qmax, double* refine, double* coarsen);

/* Positivity repair of n element states held by the host (kernel_repair of a per-quad host shim,
   source/kernel/mcfv/3d/kernel_validate_mod.f90:27-157): each element [n_vars][64] at a byte
   stride from the previous one (sizeof(quad_t) for quad%pld%hydro%state) is checked and, if a node
   is inadmissible, repaired on the device by the stage kernels' dgfv_repair_3d; the states are
   written back in place and ok_host[e] = 1 if element e is admissible afterwards.  Returns
   NEMO_ERR_REPAIR if any element stays inadmissible (as the reference raises an error).  Needs
   nemo_gpu_init; allocates and frees a device buffer per call (a slow path, not for the stage). */
int nemo_gpu_repair_states(double* host, int64_t n, int64_t elem_stride_bytes, int32_t* ok_host);

/* Blending coefficient alpha per element (host array [E]) of the current state. */
int nemo_gpu_alpha(double* alpha_host);

/* Conserved totals (sum of w_ijk * vol * u) per variable, out[10] (first n_vars used);
   source/setups/euler/3d/_common_/setup_analyze_mod.f90:28-150. */
int nemo_gpu_totals(double* out);

/* Simulation time of group 0 and the accumulated repair-failure count. */
int nemo_gpu_status(double* t_out, int64_t* nbad_total_out);

/* ---- learned shock indicator ---------------------------------------------------------------
   Network: x = feature/10 + 1 (12 inputs), h1 = SiLU(W1 x + b1) (32), h2 = SiLU(W2 h1 + b2) (32),
   alpha = alpha_max * sigmoid(W3 . h2 + b3), alpha < alpha_min -> 0.  Packed weights (1505 values):
   W1[32][12] b1[32] W2[32][32] b2[32] W3[32] b3.  Features per element: for q = rho then p, direction
   x, y, z and polynomial order N then N-1, log(E_q,d,o / E_q + 1e-12) with E the modal energies.  The
   modal indicator stays the fallback (inputs outside the training bounds, or an element whose minimum
   nodal rho or p is below a tenth of its mean) and the judge (mean |alpha_learned - alpha_modal|).
   No counterpart in the reference (its indicator module is absent from the snapshot). */

/* Load the weights (rounded to BF16; evaluated in FP32 by the FP32 form, in FP64 by the plain form)
   and the per-input bounds lo[12], hi[12] of the training data (normalised inputs). */
int nemo_gpu_set_mlp(const float* weights, int32_t nweights, const float* lo, const float* hi);

/* Features [E][12] (FP32) and the modal alpha [E] of the current state. */
int nemo_gpu_features(float* feat_host, double* alpha_modal_host);

/* Since the last upload: elements that fell back to the modal indicator, elements judged, and the
   mean |alpha_learned - alpha_modal| over the judged ones. */
int nemo_gpu_indicator_stats(int64_t* fallback_out, int64_t* judged_out, double* judge_mae_out);

/* Training on the GPU with the library's own forward/backward/Adam kernels (mini-batch Adam,
   mean squared error against target alphas).  weights: in = initial, out = trained (FP32, 1505).
   loss_out: per-epoch mean batch loss (epochs values) or NULL. */
int nemo_gpu_mlp_train(const float* feat, const float* target, int64_t nsamp, float* weights, float alpha_max,
                       int32_t epochs, int32_t batch, float lr, uint64_t seed, float* loss_out);

/* Loss and gradient of the mean squared error over all nsamp samples (one forward+backward). */
int nemo_gpu_mlp_grad(const float* feat, const float* target, int64_t nsamp, const float* weights, float alpha_max,
                      float* loss_out, float* grad_out);

/* Network output alpha_max * sigmoid(z) per sample (before the alpha_min clip). */
int nemo_gpu_mlp_forward(const float* feat, int64_t nsamp, const float* weights, float alpha_max, float* alpha_out);

/* Conserved totals (as nemo_gpu_totals) of a state held in device memory that the caller owns,
   without allocating anything.  No counterpart in the reference: it serves hosts that cannot
   allocate device memory at this point (device arrays owned by a Fortran/OpenACC pool sized at
   start-up, or a fixed device-memory budget where a cudaMalloc/cudaFree would fail or synchronise
   the device).  u_dev: [nvars][elem_stride][64] FP64 (the library's layout); delta_dev:
   [elem_stride][3]; only the first nelems elements are summed, so a partitioned state passes its
   element count as elem_stride and its owned count as nelems (its ghost copies after the owned
   elements are left out, as nemo_gpu_totals leaves them out); out_dev: nvars doubles; all device
   pointers.  stream: a cudaStream_t as an integer (0 = the legacy default stream); the call only
   enqueues work on it.  Limits: 1 <= nelems <= 65536, nelems <= elem_stride and 1 <= nvars <= 9
   (anything else is rejected with NEMO_ERR_ARG): the per-element partial sums live in a fixed
   4.5 MiB device array inside the library, held by every GPU that loads it until exit.  The first
   call on a device looks up that array's address with cudaGetSymbolAddress and caches it; under
   lazy module loading that look-up may load the library's device code, which can itself allocate,
   so make the first call at start-up (and before any stream capture).  The cached address belongs
   to the device context: after a cudaDeviceReset by the host it is stale, so do not call this
   entry point again in that process.  Every call overwrites the array, so calls that overlap on
   the GPU (other streams) race. */
int nemo_gpu_totals_noalloc(const double* u_dev, const double* delta_dev, int64_t elem_stride, int64_t nelems,
                            int32_t nvars, double* out_dev, uint64_t stream);

int nemo_gpu_finalize(void);

/* Copy the last error message (NUL terminated, truncated to len). */
int nemo_gpu_last_error(char* buf, int32_t len);

/* Stage schedule autotuner (no reference counterpart: the reference has one CPU loop).  For the
   FP32 Euler form it times nsteps full steps of each candidate from the current state -- one CTA per
   tile of 8, 4 or 16 elements plus the mortar kernel, and the persistent kernel (tiles of 8) with 1
   to 4 CTAs per SM (as many as fit) taking the mortar pairs and then the tiles from a device queue
   -- restores the state, the register, the indicator and the control block after each, and keeps
   the fastest.  mode_out (0 grid with 8 elements per CTA, 1 persistent, 2 grid with 4, 3 grid with
   16), ctas_out (persistent grid size) and ms_out[8] (ms per step: [0] grid 8, [1..4] persistent at
   1..4 CTAs per SM, [5] grid 4, [6] grid 16, [7] unused; -1 where not run) may be NULL.  Other forms
   have one schedule (mode 0). */
int nemo_gpu_autotune(int32_t nsteps, int32_t* mode_out, int32_t* ctas_out, double* ms_out);

/* Set the FP32 Euler stage schedule directly (mode as nemo_gpu_autotune's; ctas for mode 1). */
int nemo_gpu_set_schedule(int32_t mode, int32_t ctas);

/* Timing mode: when on, nemo_gpu_run issues its kernels as plain launches with a CUDA event
   between consecutive kernels on the library stream (instead of replaying CUDA graphs), and
   nemo_gpu_kernel_timing reports, for the last run, the summed device time and launch count of
   the stage kernels and of all kernels. */
int nemo_gpu_set_timing(int32_t on);
int nemo_gpu_kernel_timing(double* stage_ms, int64_t* stage_launches, double* total_ms, int64_t* total_launches);

/* The library's CUDA stream (cudaStream_t as an integer), for callers that record their own
   events on it. */
int nemo_gpu_stream(uint64_t* stream_out);

/* Measured arithmetic peaks of the current device for the roofline of the stage kernels (no
   counterpart in the reference, which reports only its wall-time performance index,
   source/driver_mod.f90:83): out[0] FP64 and out[1] FP32 fused-multiply-add throughput in
   TFLOP/s (2 flops per FMA, independent chains on every SM, best of 3 timed launches of about
   10 ms), out[2] the SM count, out[3] the maximum SM clock in MHz.  Allocates and frees a 2 KB
   buffer and a stream; call it outside timed regions. */
int nemo_gpu_measure_peaks(double* out);

#ifdef __cplusplus
}
#endif

#endif /* NEMO_GPU_H */
