!! GPU kernel module, admissibility: kernel_validate and the per-quad kernel_repair of
!! source/kernel/mcfv/3d/kernel_validate_mod.f90 (same interfaces) for host code that holds quad
!! states between sync points.  The repair itself runs on the device (nemo_gpu_repair_states: the
!! stage kernels' dgfv_repair_3d, the squeeze of 2x2x2 tiles towards their means in repair_decr
!! steps); a quad that stays inadmissible goes to raise_error, as on the CPU.

module kernel_validate_mod

use constants_mod

private
public :: kernel_repair
public :: kernel_validate

interface kernel_repair
    procedure :: repair_quad
    procedure :: repair_quad_state
end interface

contains

function repair_quad(quad) result(ok)

    use mesh_types_mod, only: quad_t

    type(quad_t), intent(inout) :: quad
    logical :: ok

    ok = repair_quad_state(quad, quad%pld%hydro%state)

end function

function repair_quad_state(quad, state) result(ok)

    use iso_c_binding
    use mesh_types_mod, only: quad_t
    use equations_mod, only: isvalid
    use nemo_gpu_interfaces_mod

    type(quad_t), intent(inout) :: quad
    real(dp), intent(inout), target :: state(N_NODES,N_NODES,N_NODES,N_VARS)
    logical :: ok

    integer(c_int32_t) :: okc(1)

    ok = isvalid(state)
    if (ok) return
    call nemo_gpu_check(nemo_gpu_repair_states(c_loc(state), 1_c_int64_t, &
        int(8*N_NODES**3*N_VARS, c_int64_t), okc), 'repair_states')
    ok = okc(1) == 1

end function

pure function kernel_validate(state) result(ok)

    use equations_mod, only: isvalid

    real(dp), intent(in) :: state(N_NODES,N_NODES,N_NODES,N_VARS)
    logical :: ok

    ok = isvalid(state)

end function

end module
