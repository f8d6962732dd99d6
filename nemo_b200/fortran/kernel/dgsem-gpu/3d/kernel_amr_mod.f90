!! GPU kernel module, per-quad AMR transfer for setups that call it from their replace callbacks
!! (source/setups/mhd/3d/_common_/setup_amr_mod.f90:52-113): the interfaces of
!! source/kernel/mcfv/3d/kernel_amr_mod.f90 with the full-order operators of kernel_share_mod
!! (q = DGFV_QMAX).  These run on the host, between the state download before the adapt and the
!! upload after it (kernel_hooks_mod); the device-side transfer of a whole forest is nemo_gpu_adapt.

module kernel_amr_mod

use constants_mod

interface kernel_amr_coarsen
    procedure :: amr_coarsen_var
    procedure :: amr_coarsen_state
end interface

contains

!! Tensor-product application along x, y, z: out(i,j,k) = sum A(i,a) B(j,b) C(k,c) x(a,b,c).
pure function apply_xyz(A, B, C, x) result(out)

    real(dp), intent(in) :: A(N_NODES,N_NODES), B(N_NODES,N_NODES), C(N_NODES,N_NODES)
    real(dp), intent(in) :: x(N_NODES,N_NODES,N_NODES)
    real(dp) :: out(N_NODES,N_NODES,N_NODES), t1(N_NODES,N_NODES,N_NODES), t2(N_NODES,N_NODES,N_NODES)

    integer :: j, k

    do k = 1,N_NODES
        t1(:,:,k) = matmul(A, x(:,:,k))
    end do
    do k = 1,N_NODES
        t2(:,:,k) = matmul(t1(:,:,k), transpose(B))
    end do
    do j = 1,N_NODES
        out(:,j,:) = matmul(t2(:,j,:), transpose(C))
    end do

end function

!! parent state -> the 8 children (p4est child order)
subroutine kernel_amr_refine(incoming, outgoing)

    use kernel_share_mod, only: refineMat
    use kernel_const_mod, only: DGFV_QMAX
    use mesh_const_mod, only: MESH_CHILDREN

    real(dp), intent(in)  :: incoming(N_NODES,N_NODES,N_NODES,N_VARS)
    real(dp), intent(out) :: outgoing(N_NODES,N_NODES,N_NODES,N_VARS,MESH_CHILDREN)

    integer :: f, h

    do f = 1,MESH_CHILDREN
        do h = 1,N_VARS
            outgoing(:,:,:,h,f) = apply_xyz(refineMat(:,:,1,f,DGFV_QMAX), refineMat(:,:,2,f,DGFV_QMAX), &
                refineMat(:,:,3,f,DGFV_QMAX), incoming(:,:,:,h))
        end do
    end do

end subroutine

!! 8 children of one variable -> the parent (sum of the children's projections)
subroutine amr_coarsen_var(incoming, outgoing)

    use kernel_share_mod, only: coarseMat
    use kernel_const_mod, only: DGFV_QMAX
    use mesh_const_mod, only: MESH_CHILDREN

    real(dp), intent(in)  :: incoming(N_NODES,N_NODES,N_NODES,MESH_CHILDREN)
    real(dp), intent(out) :: outgoing(N_NODES,N_NODES,N_NODES)

    integer :: f

    outgoing = 0.0_dp
    do f = 1,MESH_CHILDREN
        outgoing = outgoing + apply_xyz(coarseMat(:,:,1,f,DGFV_QMAX), coarseMat(:,:,2,f,DGFV_QMAX), &
            coarseMat(:,:,3,f,DGFV_QMAX), incoming(:,:,:,f))
    end do

end subroutine

subroutine amr_coarsen_state(incoming, outgoing)

    use mesh_const_mod, only: MESH_CHILDREN

    real(dp), intent(in)  :: incoming(N_NODES,N_NODES,N_NODES,N_VARS,MESH_CHILDREN)
    real(dp), intent(out) :: outgoing(N_NODES,N_NODES,N_NODES,N_VARS)

    integer :: h

    do h = 1,N_VARS
        call amr_coarsen_var(incoming(:,:,:,h,:), outgoing(:,:,:,h))
    end do

end subroutine

end module
