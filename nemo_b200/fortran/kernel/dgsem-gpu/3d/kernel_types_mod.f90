!! GPU kernel module, payload types composed into quad_t by nemo.py (scripts/nemo.py:307-362).
!!
!! The state keeps the reference's layout, state(N_NODES,N_NODES,N_NODES,N_VARS) per quad, so the
!! library uploads and downloads it with one strided copy over the quad array.  The auxiliary part
!! holds no face buffers (face traces and fluxes live on the device, inside the stage kernel); it
!! carries the quad's blending coefficient, copied back from the device at the sync points
!! (analyze, checkpoint) for the setups' output.

module kernel_types_mod

use constants_mod

type :: payload_hydro_t

    real(dp) :: state(N_NODES,N_NODES,N_NODES,N_VARS)

end type

type :: auxiliary_hydro_t

    real(dp) :: blend = 0.0_dp

end type

end module
