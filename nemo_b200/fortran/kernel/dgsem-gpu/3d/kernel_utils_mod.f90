!! GPU kernel module, helpers the setups' checkpoint callbacks import from kernel_utils_mod
!! (source/setups/euler/3d/_common_/setup_checkpoint_mod.f90:309-320).
!!
!! inflate: the GPU kernel blends DG and FV with one coefficient per quad (aux%hydro%blend); the
!! blend datasets of the FLASH checkpoint have one value per node and blending level, so the
!! coefficient is broadcast to that shape, blend(N_NODES,N_NODES,N_NODES,lo:hi).

module kernel_utils_mod

use constants_mod

contains

pure function inflate(x, lo, hi) result(out)

    real(dp), intent(in) :: x
    integer, intent(in) :: lo, hi
    real(dp) :: out(N_NODES,N_NODES,N_NODES,lo:hi)

    out = x

end function

end module
