!! GPU kernel module, shared data: the symbols other modules import from kernel_share_mod
!! (nodes, weights, dtmin, lmax, refineMat, coarseMat) plus the host<->device synchronisation of the
!! quad states.

module kernel_share_mod

use constants_mod
use kernel_const_mod, only: DGFV_QMAX
use nemo_gpu_interfaces_mod, only: nemo_cfg_t

real(dp), save :: nodes(N_NODES)
real(dp), save :: weights(N_NODES)

!! AMR transfer operators of the setups' replace callbacks (nemo_gpu_amr_operators): for child f
!! (p4est order) and direction d, refineMat(:,:,d,f,q) maps the parent's nodal values to the child's
!! after truncating the parent to its Legendre modes 0..q; coarseMat(:,:,d,f,q) maps the child's
!! nodal values to its projection onto the parent, truncated the same way.
real(dp), save :: refineMat(N_NODES,N_NODES,3,8,0:DGFV_QMAX)
real(dp), save :: coarseMat(N_NODES,N_NODES,3,8,0:DGFV_QMAX)

real(dp), save :: dtmin
real(dp), save :: lmax

type(nemo_cfg_t), save :: gpu_cfg

contains

subroutine kernel_share_amr_operators

    use iso_c_binding
    use nemo_gpu_interfaces_mod

    call nemo_gpu_check(nemo_gpu_amr_operators(int(N_NODES,c_int32_t), int(DGFV_QMAX,c_int32_t), &
        refineMat, coarseMat), 'amr_operators')

end subroutine

!! The quads' blending coefficients (aux%hydro%blend) from the device, for the setups' output.
subroutine kernel_share_blend

    use iso_c_binding
    use share_mod, only: mesh
    use nemo_gpu_interfaces_mod

    real(c_double), allocatable :: alpha(:)
    integer(kind=8) :: i

    allocate(alpha(mesh%nquads))
    call nemo_gpu_check(nemo_gpu_alpha(alpha), 'alpha')
    do i = 1,mesh%nquads
        mesh%quads(i)%aux%hydro%blend = alpha(i)
    end do

end subroutine

!! side_t / quad_t -> the C side arrays (0-based ids and face ids, source/mesh/p4est/mesh_types_mod.f90:30-77)
subroutine kernel_share_set_mesh

    use iso_c_binding
    use share_mod, only: mesh
    use mesh_const_mod, only: MESH_HALF
    use nemo_gpu_interfaces_mod

    real(c_double), allocatable :: delta(:,:), center(:,:)
    integer(c_int32_t), allocatable :: quads(:,:,:), boundary(:)
    integer(c_int8_t), allocatable :: faceid(:,:), nquads(:,:)
    integer(kind=8) :: i
    integer :: iside, iquad

    allocate(delta(3,mesh%nquads), center(3,mesh%nquads))
    allocate(quads(4,2,mesh%nsides), faceid(2,mesh%nsides), nquads(2,mesh%nsides), boundary(mesh%nsides))

    do i = 1,mesh%nquads
        delta(:,i) = mesh%quads(i)%delta
        center(:,i) = mesh%quads(i)%center
    end do

    quads = -1
    do i = 1,mesh%nsides
        associate(side => mesh%sides(i))
        do iside = 1,2
            nquads(iside,i) = int(side%nquads(iside), c_int8_t)
            faceid(iside,i) = int(side%faceid(iside) - 1, c_int8_t)
            do iquad = 1,side%nquads(iside)
                quads(iquad,iside,i) = int(side%iquads(iquad,iside) - 1, c_int32_t)
            end do
        end do
        boundary(i) = int(side%boundary, c_int32_t)
        end associate
    end do

    call nemo_gpu_check(nemo_gpu_set_mesh(int(mesh%nquads,c_int64_t), delta, center, &
        int(mesh%nsides,c_int64_t), quads, faceid, nquads, boundary), 'set_mesh')

end subroutine

!! quad%pld%hydro%state of all quads, strided by sizeof(quad_t)
subroutine kernel_share_upload

    use iso_c_binding
    use share_mod, only: mesh
    use nemo_gpu_interfaces_mod

    integer(c_int64_t) :: stride

    stride = transfer(c_loc(mesh%quads(2)), 0_c_int64_t) - transfer(c_loc(mesh%quads(1)), 0_c_int64_t)
    call nemo_gpu_check(nemo_gpu_upload_state(c_loc(mesh%quads(1)%pld%hydro%state), stride), 'upload_state')

end subroutine

subroutine kernel_share_download

    use iso_c_binding
    use share_mod, only: mesh
    use nemo_gpu_interfaces_mod

    integer(c_int64_t) :: stride

    stride = transfer(c_loc(mesh%quads(2)), 0_c_int64_t) - transfer(c_loc(mesh%quads(1)), 0_c_int64_t)
    call nemo_gpu_check(nemo_gpu_download_state(c_loc(mesh%quads(1)%pld%hydro%state), stride), 'download_state')

end subroutine

end module
