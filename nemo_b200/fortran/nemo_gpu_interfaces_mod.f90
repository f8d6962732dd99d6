!! nemo_gpu_interfaces_mod -- iso_c_binding interfaces to libnemo_gpu.so (include/nemo_gpu.h).
!!
!! Written in the style of the reference's p4wrap bindings
!! (source/mesh/p4est/wrapper/p4wrap_interfaces_mod.f90): one bind(c) interface per C entry
!! point, value arguments for scalars, c_ptr for arrays that live in the quad/side structures.
!! Every function returns a C int status (0 = OK); nemo_gpu_check turns a non-zero status into
!! raise_error with the library's message (source/utils/status_mod.f90:7-21).

module nemo_gpu_interfaces_mod

use iso_c_binding

implicit none

integer(c_int), parameter :: NEMO_EQN_EULER = 0, NEMO_EQN_MHD = 1
integer(c_int), parameter :: NEMO_VOLFLUX_CHANDRASHEKAR = 0, NEMO_VOLFLUX_CENTRAL = 1
integer(c_int), parameter :: NEMO_SURFFLUX_HLLC = 0, NEMO_SURFFLUX_RUSANOV = 1
integer(c_int), parameter :: NEMO_PREC_FP64 = 0, NEMO_PREC_FP32 = 1
integer(c_int), parameter :: NEMO_IND_NONE = 0, NEMO_IND_MODAL = 1, NEMO_IND_LEARNED = 2
integer(c_int), parameter :: NEMO_SOURCE_NONE = 0, NEMO_SOURCE_BAROTROPIC_COOLING = 1

!! mirrors struct nemo_cfg (include/nemo_gpu.h)
type, bind(c) :: nemo_cfg_t
    integer(c_int)  :: n_nodes, n_vars, eqn, volume_flux, surface_flux, precision, indicator
    integer(c_int)  :: alpha_smoothing, positivity, non_conservative, source, pad_
    real(c_double)  :: kappa, mu0, cfl, alpha_max, alpha_min, repair_decr, glm_ch, glm_alpha
    real(c_double)  :: dens_critical, k_isothermal, k_adiabatic, reserved
end type

interface
    function nemo_gpu_default_cfg(cfg) result(st) bind(c, name="nemo_gpu_default_cfg")
        import :: c_int, nemo_cfg_t
        type(nemo_cfg_t), intent(out) :: cfg
        integer(c_int) :: st
    end function

    function nemo_gpu_init(cfg) result(st) bind(c, name="nemo_gpu_init")
        import :: c_int, nemo_cfg_t
        type(nemo_cfg_t), intent(in) :: cfg
        integer(c_int) :: st
    end function

    function nemo_gpu_operators(n, nodes, weights, dmat, smat, vinv) result(st) bind(c, name="nemo_gpu_operators")
        import :: c_int, c_double
        integer(c_int), value :: n
        real(c_double), intent(out) :: nodes(*), weights(*), dmat(*), smat(*), vinv(*)
        integer(c_int) :: st
    end function

    function nemo_gpu_set_mesh(nelems, delta, center, nsides, side_quads, side_faceid, side_nquads, boundary) &
            result(st) bind(c, name="nemo_gpu_set_mesh")
        import :: c_int, c_int8_t, c_int32_t, c_int64_t, c_double
        integer(c_int64_t), value :: nelems, nsides
        real(c_double), intent(in) :: delta(*), center(*)
        integer(c_int32_t), intent(in) :: side_quads(*), boundary(*)
        integer(c_int8_t), intent(in) :: side_faceid(*), side_nquads(*)
        integer(c_int) :: st
    end function

    function nemo_gpu_set_groups(ngroups, group_of_elem) result(st) bind(c, name="nemo_gpu_set_groups")
        import :: c_int, c_int32_t
        integer(c_int32_t), value :: ngroups
        integer(c_int32_t), intent(in) :: group_of_elem(*)
        integer(c_int) :: st
    end function

    function nemo_gpu_upload_state(host, elem_stride_bytes) result(st) bind(c, name="nemo_gpu_upload_state")
        import :: c_int, c_int64_t, c_ptr
        type(c_ptr), value :: host
        integer(c_int64_t), value :: elem_stride_bytes
        integer(c_int) :: st
    end function

    function nemo_gpu_download_state(host, elem_stride_bytes) result(st) bind(c, name="nemo_gpu_download_state")
        import :: c_int, c_int64_t, c_ptr
        type(c_ptr), value :: host
        integer(c_int64_t), value :: elem_stride_bytes
        integer(c_int) :: st
    end function

    function nemo_gpu_calc_timestep(cfl, dt, lmax) result(st) bind(c, name="nemo_gpu_calc_timestep")
        import :: c_int, c_double
        real(c_double), value :: cfl
        real(c_double), intent(out) :: dt, lmax
        integer(c_int) :: st
    end function

    function nemo_gpu_stage(stage, dt, t_stage, nbad) result(st) bind(c, name="nemo_gpu_stage")
        import :: c_int, c_int32_t, c_double
        integer(c_int32_t), value :: stage
        real(c_double), value :: dt, t_stage
        integer(c_int32_t), intent(out) :: nbad
        integer(c_int) :: st
    end function

    function nemo_gpu_step(dt) result(st) bind(c, name="nemo_gpu_step")
        import :: c_int, c_double
        real(c_double), value :: dt
        integer(c_int) :: st
    end function

    function nemo_gpu_run(nsteps, t_end, t_out, steps_out) result(st) bind(c, name="nemo_gpu_run")
        import :: c_int, c_int64_t, c_double
        integer(c_int64_t), value :: nsteps
        real(c_double), value :: t_end
        real(c_double), intent(out) :: t_out
        integer(c_int64_t), intent(out) :: steps_out
        integer(c_int) :: st
    end function

    function nemo_gpu_totals(out) result(st) bind(c, name="nemo_gpu_totals")
        import :: c_int, c_double
        real(c_double), intent(out) :: out(10)
        integer(c_int) :: st
    end function

    function nemo_gpu_finalize() result(st) bind(c, name="nemo_gpu_finalize")
        import :: c_int
        integer(c_int) :: st
    end function

    function nemo_gpu_last_error(buf, len) result(st) bind(c, name="nemo_gpu_last_error")
        import :: c_int, c_int32_t, c_char
        character(kind=c_char), intent(out) :: buf(*)
        integer(c_int32_t), value :: len
        integer(c_int) :: st
    end function

    !! Adapt flags of the current state from the device density probe (replaces the probe callbacks
    !! of mesh_adapt); flags(nquads): +1 refine, -1 coarsen (all 8 of a family), 0 keep.
    function nemo_gpu_amr_flags(refine_threshold, coarsen_threshold, flags) result(st) &
            bind(c, name="nemo_gpu_amr_flags")
        import :: c_int, c_int32_t, c_double
        real(c_double), value :: refine_threshold, coarsen_threshold
        integer(c_int32_t), intent(out) :: flags(*)
        integer(c_int) :: st
    end function

    !! The adapted forest in set_mesh form plus remap(4, nquads_new) rows (kind, src, depth, offsets)
    !! with 0-based src (replaces the replace callbacks of mesh_adapt).
    function nemo_gpu_adapt(nelems, delta, center, nsides, side_quads, side_faceid, side_nquads, boundary, &
            remap) result(st) bind(c, name="nemo_gpu_adapt")
        import :: c_int, c_int8_t, c_int32_t, c_int64_t, c_double
        integer(c_int64_t), value :: nelems, nsides
        real(c_double), intent(in) :: delta(*), center(*)
        integer(c_int32_t), intent(in) :: side_quads(*), boundary(*), remap(*)
        integer(c_int8_t), intent(in) :: side_faceid(*), side_nquads(*)
        integer(c_int) :: st
    end function

    !! Checkpoint staging: snapshot in stream order, device->host copy on a second stream
    !! (hook_checkpoint_fill); restart = upload_state + set_time.
    function nemo_gpu_checkpoint_begin(host, elem_stride_bytes, alpha_host) result(st) &
            bind(c, name="nemo_gpu_checkpoint_begin")
        import :: c_int, c_int64_t, c_ptr
        type(c_ptr), value :: host, alpha_host
        integer(c_int64_t), value :: elem_stride_bytes
        integer(c_int) :: st
    end function

    function nemo_gpu_checkpoint_wait(t_out, steps_out) result(st) bind(c, name="nemo_gpu_checkpoint_wait")
        import :: c_int, c_int64_t, c_double
        real(c_double), intent(out) :: t_out
        integer(c_int64_t), intent(out) :: steps_out
        integer(c_int) :: st
    end function

    function nemo_gpu_set_time(t, steps) result(st) bind(c, name="nemo_gpu_set_time")
        import :: c_int, c_int64_t, c_double
        real(c_double), value :: t
        integer(c_int64_t), value :: steps
        integer(c_int) :: st
    end function

    !! Element partition over MPI ranks: owned quads first, then ghosts; ghost refresh before every
    !! stage around the host's own exchange (mesh_exchange).  idx/face/buf are device pointers.
    function nemo_gpu_set_owned(n_owned) result(st) bind(c, name="nemo_gpu_set_owned")
        import :: c_int, c_int64_t
        integer(c_int64_t), value :: n_owned
        integer(c_int) :: st
    end function

    function nemo_gpu_pack_faces(idx_dev, face_dev, n, buf_dev) result(st) bind(c, name="nemo_gpu_pack_faces")
        import :: c_int, c_int64_t, c_ptr
        type(c_ptr), value :: idx_dev, face_dev, buf_dev
        integer(c_int64_t), value :: n
        integer(c_int) :: st
    end function

    function nemo_gpu_unpack_faces(idx_dev, face_dev, n, buf_dev) result(st) bind(c, name="nemo_gpu_unpack_faces")
        import :: c_int, c_int64_t, c_ptr
        type(c_ptr), value :: idx_dev, face_dev, buf_dev
        integer(c_int64_t), value :: n
        integer(c_int) :: st
    end function

    function nemo_gpu_pack_elements(idx_dev, n, buf_dev) result(st) bind(c, name="nemo_gpu_pack_elements")
        import :: c_int, c_int64_t, c_ptr
        type(c_ptr), value :: idx_dev, buf_dev
        integer(c_int64_t), value :: n
        integer(c_int) :: st
    end function

    function nemo_gpu_unpack_elements(idx_dev, n, buf_dev) result(st) bind(c, name="nemo_gpu_unpack_elements")
        import :: c_int, c_int64_t, c_ptr
        type(c_ptr), value :: idx_dev, buf_dev
        integer(c_int64_t), value :: n
        integer(c_int) :: st
    end function

    !! Blending coefficient per quad of the current state (host array alpha(nquads)).
    function nemo_gpu_alpha(alpha) result(st) bind(c, name="nemo_gpu_alpha")
        import :: c_int, c_double
        real(c_double), intent(out) :: alpha(*)
        integer(c_int) :: st
    end function

    !! refineMat / coarseMat (n, n, 3, 8, 0:qmax) of kernel_share_mod for the setups' replace callbacks.
    function nemo_gpu_amr_operators(n, qmax, refine, coarsen) result(st) bind(c, name="nemo_gpu_amr_operators")
        import :: c_int, c_int32_t, c_double
        integer(c_int32_t), value :: n, qmax
        real(c_double), intent(out) :: refine(*), coarsen(*)
        integer(c_int) :: st
    end function

    !! Positivity repair of host-held quad states (n of them, elem_stride_bytes apart), in place on the
    !! device; ok(e) = 1 if quad e is admissible afterwards (kernel_repair).
    function nemo_gpu_repair_states(host, n, elem_stride_bytes, ok) result(st) bind(c, name="nemo_gpu_repair_states")
        import :: c_int, c_int32_t, c_int64_t, c_ptr
        type(c_ptr), value :: host
        integer(c_int64_t), value :: n, elem_stride_bytes
        integer(c_int32_t), intent(out) :: ok(*)
        integer(c_int) :: st
    end function
end interface

contains

!! Forward a non-zero status to the reference's error path.
subroutine nemo_gpu_check(st, where)

    use status_mod, only: raise_error

    integer(c_int), intent(in) :: st
    character(len=*), intent(in) :: where

    character(kind=c_char) :: buf(512)
    character(len=512) :: msg
    integer :: i, rc

    if (st == 0) return
    rc = nemo_gpu_last_error(buf, 512_c_int32_t)
    msg = ''
    do i = 1, 512
        if (buf(i) == c_null_char) exit
        msg(i:i) = buf(i)
    end do
    call raise_error('nemo_gpu (' // where // '): ' // trim(msg))

end subroutine

end module
