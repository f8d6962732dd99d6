!! GPU kernel module, hook part: replaces kernel_hooks_mod of a CPU kernel directory
!! (source/kernel/mcfv/3d/kernel_hooks_mod.f90).  A setup's preproc.py selects it with
!!     kernel = home + '/source/kernel/dgsem-gpu/3d'
!! and links libnemo_gpu.so; nemo.py then wires these hooks into the generated dispatchers
!! (scripts/nemo.py:245-305) exactly as it wires the CPU kernel's.

module kernel_hooks_mod

use constants_mod

contains

!! hook_init_400: operators and device selection (kernel_share_mod::init on the CPU side).
subroutine hook_init_400

    use iso_c_binding
    use nemo_gpu_interfaces_mod
    use kernel_share_mod, only: nodes, weights, gpu_cfg, kernel_share_amr_operators
    use kernel_config_mod, only: repair_decr
    use setup_config_mod, only: kappa, CFL

    real(c_double) :: x(N_NODES), w(N_NODES), dmat(N_NODES**2), smat(N_NODES**2), vinv(N_NODES**2)

    call nemo_gpu_check(nemo_gpu_default_cfg(gpu_cfg), 'default_cfg')
    gpu_cfg%kappa = kappa
    gpu_cfg%cfl = CFL
    gpu_cfg%repair_decr = repair_decr
# ifdef PP_KERNEL_GPU_PRECISION
    gpu_cfg%precision = PP_KERNEL_GPU_PRECISION
# endif
# ifdef PP_KERNEL_GPU_INDICATOR
    gpu_cfg%indicator = PP_KERNEL_GPU_INDICATOR
    gpu_cfg%positivity = 1
# endif
    call nemo_gpu_check(nemo_gpu_init(gpu_cfg), 'init')

    !! nodes/weights on [-1/2,1/2] as the mesh layer expects (source/mesh/p4est/quad_utils_mod.f90:11)
    call nemo_gpu_check(nemo_gpu_operators(int(N_NODES,c_int), x, w, dmat, smat, vinv), 'operators')
    nodes = 0.5_dp * x
    weights = 0.5_dp * w

    call kernel_share_amr_operators()

end subroutine

!! hook_init_520 (after the mesh, hook_init_500/510): connectivity to the device.
subroutine hook_init_520

    use kernel_share_mod, only: kernel_share_set_mesh

    call kernel_share_set_mesh()

end subroutine

!! hook_init_815 (after the setup filled the initial state, hook_init_810): state to the device.
subroutine hook_init_815

    use kernel_share_mod, only: kernel_share_upload

    call kernel_share_upload()

end subroutine

!! Face fill and face flux are fused into the stage kernel: nothing to do before the stage.
subroutine hook_pre_rk_timestep_300

end subroutine

!! The setups' analyze and checkpoint hooks read quad%pld%hydro%state (and aux%hydro%blend): bring
!! them back first.
subroutine hook_analyze_100

    use kernel_share_mod, only: kernel_share_download

    call kernel_share_download()

end subroutine

subroutine hook_checkpoint_100

    use kernel_share_mod, only: kernel_share_download, kernel_share_blend

    call kernel_share_download()
    call kernel_share_blend()

end subroutine

# ifdef PP_KERNEL_GPU_AMR_SYNC
!! Setups that adapt the forest with their own replace callbacks on the host (hook_pre_timestep_300,
!! source/setups/euler/3d/sedov/setup_amr_mod.f90:7-21, every amr_each_ntimesteps steps): the state
!! comes back to the quads before, and the new forest and its state go to the device after.  Setups
!! that adapt through nemo_gpu_amr_flags / nemo_gpu_adapt leave PP_KERNEL_GPU_AMR_SYNC undefined.
subroutine hook_pre_timestep_290

    use share_mod, only: rt => runtime
    use setup_config_mod, only: amr_each_ntimesteps
    use kernel_share_mod, only: kernel_share_download

    if (mod(rt%timesteps,amr_each_ntimesteps) == 0) call kernel_share_download()

end subroutine

subroutine hook_pre_timestep_310

    use iso_c_binding
    use share_mod, only: rt => runtime
    use setup_config_mod, only: amr_each_ntimesteps
    use kernel_share_mod, only: kernel_share_set_mesh, kernel_share_upload
    use nemo_gpu_interfaces_mod

    if (mod(rt%timesteps,amr_each_ntimesteps) == 0) then
        call kernel_share_set_mesh()
        call kernel_share_upload()
        !! the upload starts a new run on the device: carry the time over
        call nemo_gpu_check(nemo_gpu_set_time(real(rt%simtime,c_double), int(rt%timesteps,c_int64_t)), 'set_time')
    end if

end subroutine
# endif

end module
