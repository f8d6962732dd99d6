!! GPU kernel module, tunables of the positivity repair.  The device repair reads repair_decr from
!! the library configuration (nemo_cfg%repair_decr, filled by hook_init_400 from here); lofactor is
!! exported for setups that import it from a CPU kernel directory.

module kernel_config_mod

use constants_mod

!! squeeze step of dgfv_repair_3d towards the tile mean (source/kernel/mcfv/3d/kernel_config_mod.f90)
real(dp), parameter :: repair_decr = 0.01_dp

real(dp), parameter :: lofactor = 1e-3_dp

end module
