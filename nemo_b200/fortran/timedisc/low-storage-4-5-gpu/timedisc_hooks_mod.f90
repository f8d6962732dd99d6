!! GPU time integrator hooks: replaces source/timedisc/rungekutta/low-storage/4-5/timedisc_hooks_mod.f90.
!! The register lives on the device (FP64); one call runs face fluxes, the element operator, the
!! register/state update and the positivity repair of every quad for stage rt%rkstage.
!! timedisc_const_mod, timedisc_evolve_mod and timedisc_types_mod of the CPU directory are reused
!! unchanged (the stage loop of hook_evolve_500 and its per-stage status check stay as they are).

module timedisc_hooks_mod

use constants_mod

contains

subroutine hook_mid_rk_timestep_500

    use iso_c_binding
    use share_mod, only: rt => runtime
    use nemo_gpu_interfaces_mod

    integer(c_int32_t) :: nbad

    call nemo_gpu_check(nemo_gpu_stage(int(rt%rkstage,c_int32_t), real(rt%timestep,c_double), &
        real(rt%rksimtime,c_double), nbad), 'stage')

end subroutine

end module
