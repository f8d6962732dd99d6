!! GPU kernel module, constants: the symbols the setups import from kernel_const_mod.
!!
!! DGFV_QMAX is the highest modal order index of refineMat/coarseMat (kernel_share_mod); the
!! setups' replace callbacks step q down from DGFV_QMAX-2 to 0 until the transferred state is
!! admissible (source/setups/euler/3d/sedov/setup_amr_mod.f90:82-95) and size their checkpoint
!! blend datasets with it (source/setups/euler/3d/_common_/setup_checkpoint_mod.f90:36-51).  A
!! setup's preproc.py sets PP_KERNEL_DGFV_QMAX (3 in the Euler 3D setups); without it the value is
!! the polynomial degree N = N_NODES-1, the most the operators resolve.

module kernel_const_mod

use constants_mod

# ifdef PP_KERNEL_DGFV_QMAX
integer, parameter :: DGFV_QMAX = min(PP_KERNEL_DGFV_QMAX, N_NODES-1)
# else
integer, parameter :: DGFV_QMAX = N_NODES-1
# endif

end module
