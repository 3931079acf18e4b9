! globalHdnnps_gpu.f90 -- Fortran drop-in for module globalHdnnps
! (src/potentials/globalHdnnps.f90 of the reference): a committee of
! potentials evaluated on the GPU through hdnnp_committee_energy_and_forces
! (include/hdnnp_gpu.h).  A caller replaces `use globalHdnnps` by
! `use globalHdnnps_gpu` and keeps its calls:
!   call initGlobalHdnnpsFromInputFile()                         ! :13 (reads nnps.txt)
!   call globalHdnnpEnergyAndForces(ats, energy, forces, dEdLat, std)  ! :31
! As in the reference, the first potential provides the neighbour lists and
! the scaled symmetry functions; energy, forces and dEdLat are member means
! and std the population standard deviation of the member energies.
!
! Not compiled in this image (no Fortran compiler); it compiles after
! hdnnps_gpu.f90 and the reference's precision and atomicStructure modules.
module globalHdnnps_gpu
    use iso_c_binding
    use precision
    use atomicStructure
    use hdnnps_gpu
    implicit none

    integer :: nGlobalHdnnps = 0
    type(hdnnp), allocatable, target :: globalHdnnpHandles(:)

    interface
        function c_committee_energy_and_forces(ctx, members, nmembers, nat, z, pos, periodic, lat, energy, force, &
                                               dEdLat, std) bind(C, name='hdnnp_committee_energy_and_forces') &
                                               result(code)
            import :: c_int, c_ptr, c_double, c_int32_t
            type(c_ptr), value :: ctx
            type(c_ptr), intent(in) :: members(*)
            integer(c_int), value :: nmembers, nat
            integer(c_int32_t), intent(in) :: z(*)
            real(c_double), intent(in) :: pos(*)
            integer(c_int), value :: periodic
            real(c_double), intent(in) :: lat(9)
            real(c_double), intent(out) :: energy
            real(c_double), intent(out) :: force(*)
            type(c_ptr), value :: dEdLat, std
            integer(c_int) :: code
        end function
    end interface

contains

    ! initGlobalHdnnpsFromInputFile (globalHdnnps.f90:13-29): nnps.txt holds
    ! the number of potentials and then one RuNNer directory per line.
    subroutine initGlobalHdnnpsFromInputFile()
        integer :: nnunit, i
        character(len=256) :: txt

        open(newunit=nnunit, file='nnps.txt', action='read')
        read(nnunit, *) nGlobalHdnnps
        allocate(globalHdnnpHandles(nGlobalHdnnps))
        do i = 1, nGlobalHdnnps
            read(nnunit, '(A)') txt
            call parseRuNNerInput(globalHdnnpHandles(i), trim(txt))
        end do
        close(nnunit)
    end subroutine initGlobalHdnnpsFromInputFile

    ! globalHdnnpEnergyAndForces (globalHdnnps.f90:31-70).
    subroutine globalHdnnpEnergyAndForces(ats, energy, forces, dEdLat, std)
        type(atStruct), intent(in) :: ats
        real(dp), intent(out) :: forces(3, ats%nat), energy
        real(dp), intent(out), optional, target :: std, dEdLat(3,3)
        type(c_ptr), allocatable :: members(:)
        integer(c_int32_t), allocatable :: el(:)
        real(c_double) :: lat(9)
        integer(c_int) :: code, periodic
        type(c_ptr) :: pdl, psd
        integer :: i

        allocate(members(nGlobalHdnnps), el(ats%nat))
        do i = 1, nGlobalHdnnps
            members(i) = globalHdnnpHandles(i)%model
        end do
        el = int(ats%el, c_int32_t)
        periodic = 0
        lat = [1._dp, 0._dp, 0._dp, 0._dp, 1._dp, 0._dp, 0._dp, 0._dp, 1._dp]
        if (ats%periodic) then
            periodic = 1
            lat = reshape(ats%lat, [9])
        end if
        pdl = c_null_ptr
        psd = c_null_ptr
        if (present(dEdLat)) pdl = c_loc(dEdLat)
        if (present(std)) psd = c_loc(std)
        code = c_committee_energy_and_forces(globalHdnnpHandles(1)%ctx, members, int(nGlobalHdnnps, c_int), &
                                             int(ats%nat, c_int), el, ats%ats, periodic, lat, energy, forces, pdl, psd)
        if (code /= 0) then
            print*, 'hdnnp committee error', code
            stop
        end if
    end subroutine globalHdnnpEnergyAndForces

end module globalHdnnps_gpu
