!! GPU kernel module, time step: hook_calc_timestep_200 as in
!! source/kernel/mcfv/3d/kernel_timestep_mod.f90:17-58, the reduction running on the device.

module kernel_timestep_mod

use constants_mod

contains

subroutine hook_calc_timestep_200

    use iso_c_binding
    use share_mod, only: rt => runtime
    use setup_config_mod, only: CFL
    use kernel_share_mod, only: dtmin, lmax
    use nemo_gpu_interfaces_mod

    real(c_double) :: dt, lm

    call nemo_gpu_check(nemo_gpu_calc_timestep(real(CFL,c_double), dt, lm), 'calc_timestep')
    rt%maxtimestep = dt
    dtmin = dt
    lmax = lm

end subroutine

end module
