! hdnnps_gpu.f90 -- Fortran drop-in for the potential API of module hdnnps
! (src/potentials/hdnnps.f90 of the reference) on top of the C ABI in
! include/hdnnp_gpu.h (libhdnnp_b200.so).
!
! A caller replaces `use hdnnps` by `use hdnnps_gpu` and keeps its calls:
!   call parseRuNNerInput(handle, './hdnnp-params/')          ! hdnnps.f90:34
!   call hdnnpEnergyAndForces(handle, ats, epot, forces)      ! hdnnps.f90:333
!   call hdnnpEnergyAndForces(handle, ats, epot, forces, dEdLat)
! with the same argument types (type(atStruct) from module atomicStructure,
! real(dp) = c_double).  Errors print the library's message and stop, as the
! reference does.  The evaluation runs on the GPU given by HDNNP_DEVICE
! (default 0).
!
! This image has no Fortran compiler, so this file is not compiled here; it
! compiles against the reference's modules precision and atomicStructure:
!   gfortran -c hdnnps_gpu.f90 (after precision.f90, atomicStructure.f90 ...)
!   link with -L<lib dir> -lhdnnp_b200
module hdnnps_gpu
    use iso_c_binding
    use precision
    use atomicStructure
    implicit none

    private
    public :: hdnnp, parseRuNNerInput, hdnnpEnergyAndForces, hdnnpFree

    type hdnnp
        type(c_ptr) :: model = c_null_ptr
        type(c_ptr) :: ctx = c_null_ptr
        real(dp) :: maxRc = 0._dp
    end type hdnnp

    interface
        function c_last_error() bind(C, name='hdnnp_last_error') result(p)
            import :: c_ptr
            type(c_ptr) :: p
        end function

        function c_model_load_runner(path, device, model) bind(C, name='hdnnp_model_load_runner') result(code)
            import :: c_char, c_int, c_ptr
            character(kind=c_char), dimension(*), intent(in) :: path
            integer(c_int), value :: device
            type(c_ptr), intent(out) :: model
            integer(c_int) :: code
        end function

        function c_model_info(model, nelem, z, nsf, max_rc) bind(C, name='hdnnp_model_info') result(code)
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: model
            integer(c_int), intent(out) :: nelem
            integer(c_int), intent(out) :: z(118), nsf(118)
            real(c_double), intent(out) :: max_rc
            integer(c_int) :: code
        end function

        function c_ctx_create(model, ctx) bind(C, name='hdnnp_ctx_create') result(code)
            import :: c_int, c_ptr
            type(c_ptr), value :: model
            type(c_ptr), intent(out) :: ctx
            integer(c_int) :: code
        end function

        subroutine c_ctx_free(ctx) bind(C, name='hdnnp_ctx_free')
            import :: c_ptr
            type(c_ptr), value :: ctx
        end subroutine

        subroutine c_model_free(model) bind(C, name='hdnnp_model_free')
            import :: c_ptr
            type(c_ptr), value :: model
        end subroutine

        function c_energy_and_forces(ctx, nat, z, pos, periodic, lat, energy, force, dEdLat) &
                bind(C, name='hdnnp_energy_and_forces') result(code)
            import :: c_int, c_ptr, c_double, c_int32_t
            type(c_ptr), value :: ctx
            integer(c_int), value :: nat
            integer(c_int32_t), intent(in) :: z(*)
            real(c_double), intent(in) :: pos(*)
            integer(c_int), value :: periodic
            real(c_double), intent(in) :: lat(9)
            real(c_double), intent(out) :: energy
            real(c_double), intent(out) :: force(*)
            type(c_ptr), value :: dEdLat
            integer(c_int) :: code
        end function
    end interface

contains

    subroutine fail_stop(code)
        integer(c_int), intent(in) :: code
        character(kind=c_char), pointer :: msg(:)
        character(len=512) :: txt
        integer :: i
        call c_f_pointer(c_last_error(), msg, [512])
        txt = ''
        do i = 1, 512
            if (msg(i) == c_null_char) exit
            txt(i:i) = msg(i)
        end do
        print*, 'hdnnp error', code, ': ', trim(txt)
        stop
    end subroutine

    ! parseRuNNerInput (hdnnps.f90:34): reads input.nn, scaling.data and
    ! weights.NNN.data from `path` and uploads the potential to the GPU.
    subroutine parseRuNNerInput(handle, path)
        type(hdnnp), intent(inout) :: handle
        character(len=*) :: path
        integer(c_int) :: code, nelem, device, stat
        integer(c_int) :: z(118), nsf(118)
        character(len=16) :: env
        real(c_double) :: rc

        device = 0
        call get_environment_variable('HDNNP_DEVICE', env, status=stat)
        if (stat == 0) read(env, *) device
        code = c_model_load_runner(trim(path) // c_null_char, device, handle%model)
        if (code /= 0) call fail_stop(code)
        code = c_ctx_create(handle%model, handle%ctx)
        if (code /= 0) call fail_stop(code)
        code = c_model_info(handle%model, nelem, z, nsf, rc)
        if (code /= 0) call fail_stop(code)
        handle%maxRc = rc
    end subroutine parseRuNNerInput

    ! hdnnpEnergyAndForces (hdnnps.f90:333): energy, forces and optionally
    ! dE/dlattice of one structure.
    subroutine hdnnpEnergyAndForces(handle, ats, energy, force, dEdLat)
        type(hdnnp), intent(inout) :: handle
        type(atStruct), intent(inout) :: ats
        real(dp), intent(out) :: energy
        real(dp), intent(out) :: force(3, ats%nat)
        real(dp), intent(out), optional, target :: dEdLat(3,3)
        integer(c_int32_t), allocatable :: el(:)
        real(c_double) :: lat(9)
        integer(c_int) :: code, periodic
        type(c_ptr) :: pdl

        allocate(el(ats%nat))
        el = int(ats%el, c_int32_t)
        periodic = 0
        lat = [1._dp, 0._dp, 0._dp, 0._dp, 1._dp, 0._dp, 0._dp, 0._dp, 1._dp]
        if (ats%periodic) then
            periodic = 1
            lat = reshape(ats%lat, [9])
        end if
        pdl = c_null_ptr
        if (present(dEdLat)) pdl = c_loc(dEdLat)
        code = c_energy_and_forces(handle%ctx, int(ats%nat, c_int), el, ats%ats, periodic, lat, energy, force, pdl)
        if (code /= 0) call fail_stop(code)
    end subroutine hdnnpEnergyAndForces

    subroutine hdnnpFree(handle)
        type(hdnnp), intent(inout) :: handle
        if (c_associated(handle%ctx)) call c_ctx_free(handle%ctx)
        if (c_associated(handle%model)) call c_model_free(handle%model)
        handle%ctx = c_null_ptr
        handle%model = c_null_ptr
    end subroutine hdnnpFree

end module hdnnps_gpu
