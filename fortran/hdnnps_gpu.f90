! hdnnps_gpu.f90 -- Fortran drop-in for the potential API of module hdnnps
! (src/potentials/hdnnps.f90 of the reference) on top of the C ABI in
! include/hdnnp_gpu.h (libhdnnp_b200.so).
!
! A caller replaces `use hdnnps` by `use hdnnps_gpu` and keeps its calls:
!   call parseRuNNerInput(handle, './hdnnp-params/')          ! hdnnps.f90:34
!   call hdnnpEnergyAndForces(handle, ats, epot, forces)      ! hdnnps.f90:333
!   call hdnnpEnergyAndForces(handle, ats, epot, forces, dEdLat)
!   call hdnnpCalcNeighborLists(handle, ats, neiLists)        ! hdnnps.f90:373
!   call hdnnpCalcSymfunctions(handle, ats, neiLists, sfs)    ! hdnnps.f90:390
!   call hdnnpCalcNNs(handle, ats, neiLists, sfs, e, f, dl)   ! hdnnps.f90:487
! with the same argument types (type(atStruct) from module atomicStructure,
! type(neighborList) from neighborLists, type(symFunctionContainer) from
! symmetryFunctions, real(dp) = c_double).  type(hdnnp) keeps the
! reference's components (sfLists, nnList, maxRc, emin, emax, atomenergies,
! scalesf, centersf), filled by parseRuNNerInput from the parsed potential,
! plus the C handles.  Errors print the library's message and stop, as the
! reference does.  The evaluation runs on the GPU given by HDNNP_DEVICE
! (default 0).
!
! The stage routines keep the lists and symmetry functions on the GPU, in the
! context of the handle that built them.  neiLists comes back in the
! reference's layout; sfs carries the values (sfs(iat)%sfs(isf)%sf and
! nNeis) but no dsf: hdnnpCalcNNs recomputes the derivatives on the GPU.  As
! in the reference's committee (globalHdnnps.f90:47-57), hdnnpCalcNNs of any
! handle uses the symmetry functions of the last hdnnpCalcSymfunctions call.
!
! This image has no Fortran compiler, so this file is not compiled here; it
! compiles against the reference's modules precision, constants,
! atomicStructure, symmetryFunctions, neighborLists and neuralNetworks:
!   gfortran -c hdnnps_gpu.f90 (after those modules)
!   link with -L<lib dir> -lhdnnp_b200
module hdnnps_gpu
    use iso_c_binding
    use precision
    use constants, only: maxElemNum
    use atomicStructure
    use symmetryFunctions, only: symFunctionList, symFunctionContainer
    use neighborLists, only: neighborList
    use neuralNetworks, only: neuralNetwork, nn_new
    implicit none

    private
    public :: hdnnp, parseRuNNerInput, hdnnpEnergyAndForces, hdnnpFree, &
              hdnnpCalcNeighborLists, hdnnpCalcSymfunctions, hdnnpCalcNNs

    type hdnnp
        type(symFunctionList) :: sfLists(maxElemNum)
        type(neuralNetwork) :: nnList(maxElemNum)
        real(dp) :: maxRc = 0._dp
        real(dp) :: emin = 0._dp, emax = 0._dp
        real(dp) :: atomenergies(maxElemNum) = 0._dp
        logical :: scalesf = .false.
        logical :: centersf = .false.
        type(c_ptr) :: model = c_null_ptr
        type(c_ptr) :: ctx = c_null_ptr
        integer :: nsfMax = 0      ! largest sfLists(:)%nsf of the potential's elements
    end type hdnnp

    ! context holding the symmetry functions of the last hdnnpCalcSymfunctions
    type(c_ptr), save :: stage_ctx = c_null_ptr

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

        function c_model_flags(model, scalesf, centersf, emin, emax, ae) bind(C, name='hdnnp_model_flags') result(code)
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: model
            integer(c_int), intent(out) :: scalesf, centersf
            real(c_double), intent(out) :: emin, emax
            real(c_double), intent(out) :: ae(118)
            integer(c_int) :: code
        end function

        function c_model_symfunctions(model, z, nsf, params) bind(C, name='hdnnp_model_symfunctions') result(code)
            import :: c_int, c_ptr
            type(c_ptr), value :: model
            integer(c_int), value :: z
            integer(c_int), intent(out) :: nsf
            type(c_ptr), value :: params
            integer(c_int) :: code
        end function

        function c_model_network(model, z, nlayers, dims, acts, vals) bind(C, name='hdnnp_model_network') result(code)
            import :: c_int, c_ptr
            type(c_ptr), value :: model
            integer(c_int), value :: z
            integer(c_int), intent(out) :: nlayers
            type(c_ptr), value :: dims, acts, vals
            integer(c_int) :: code
        end function

        function c_calc_neighbor_lists(ctx, nat, z, pos, periodic, lat, nentries) &
                bind(C, name='hdnnp_calc_neighbor_lists') result(code)
            import :: c_int, c_ptr, c_double, c_int32_t
            type(c_ptr), value :: ctx
            integer(c_int), value :: nat
            integer(c_int32_t), intent(in) :: z(*)
            real(c_double), intent(in) :: pos(*)
            integer(c_int), value :: periodic
            real(c_double), intent(in) :: lat(9)
            integer(c_int), intent(out) :: nentries
            integer(c_int) :: code
        end function

        function c_neighbor_lists_fetch(ctx, nneis, ineis, neis) bind(C, name='hdnnp_neighbor_lists_fetch') &
                result(code)
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
            integer(c_int), intent(out) :: nneis(*)
            type(c_ptr), value :: ineis, neis
            integer(c_int) :: code
        end function

        function c_calc_symfunctions(ctx, g) bind(C, name='hdnnp_calc_symfunctions') result(code)
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx, g
            integer(c_int) :: code
        end function

        function c_calc_nns(ctx, nn, energy, force, dEdLat) bind(C, name='hdnnp_calc_nns') result(code)
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx, nn
            real(c_double), intent(out) :: energy
            real(c_double), intent(out) :: force(*)
            type(c_ptr), value :: dEdLat
            integer(c_int) :: code
        end function

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
        handle%nsfMax = maxval(nsf(1:nelem))
        call fill_components(handle, nelem, z)
    end subroutine parseRuNNerInput

    ! The components of type(hdnnp) (hdnnps.f90:13-21) from the parsed
    ! potential: symmetry functions in the reference's sorted order, networks
    ! (weights(nOut, nInp), bias, activation), scaling flags, atom energies.
    subroutine fill_components(handle, nelem, z)
        type(hdnnp), intent(inout) :: handle
        integer(c_int), intent(in) :: nelem, z(118)
        integer(c_int) :: code, sc, ce, nsf, nl, e, s, l, o
        real(c_double) :: ae(118)
        real(c_double), allocatable, target :: par(:), vals(:)
        integer(c_int), allocatable, target :: dims(:)
        character(kind=c_char), allocatable, target :: acts(:)
        integer, allocatable :: nodes(:)
        character, allocatable :: act(:)

        code = c_model_flags(handle%model, sc, ce, handle%emin, handle%emax, ae)
        if (code /= 0) call fail_stop(code)
        handle%scalesf = sc /= 0
        handle%centersf = ce /= 0
        handle%atomenergies = ae
        do e = 1, nelem
            code = c_model_symfunctions(handle%model, z(e), nsf, c_null_ptr)
            if (code /= 0) call fail_stop(code)
            allocate(par(11 * nsf))
            code = c_model_symfunctions(handle%model, z(e), nsf, c_loc(par))
            if (code /= 0) call fail_stop(code)
            handle%sfLists(z(e))%nsf = nsf
            if (allocated(handle%sfLists(z(e))%sfs)) deallocate(handle%sfLists(z(e))%sfs)
            allocate(handle%sfLists(z(e))%sfs(nsf))
            do s = 1, nsf
                o = 11 * (s - 1)
                handle%sfLists(z(e))%sfs(s)%name = nint(par(o + 1))
                handle%sfLists(z(e))%sfs(s)%sfEls = [nint(par(o + 2)), nint(par(o + 3))]
                handle%sfLists(z(e))%sfs(s)%rcut = par(o + 4)
                handle%sfLists(z(e))%sfs(s)%eta = par(o + 5)
                handle%sfLists(z(e))%sfs(s)%lambda = par(o + 6)
                handle%sfLists(z(e))%sfs(s)%zeta = par(o + 7)
                handle%sfLists(z(e))%sfs(s)%Rs = par(o + 8)
                handle%sfLists(z(e))%sfs(s)%sfmin = par(o + 9)
                handle%sfLists(z(e))%sfs(s)%sfmax = par(o + 10)
                handle%sfLists(z(e))%sfs(s)%sfmean = par(o + 11)
            end do
            deallocate(par)
            code = c_model_network(handle%model, z(e), nl, c_null_ptr, c_null_ptr, c_null_ptr)
            if (code /= 0) call fail_stop(code)
            allocate(dims(2 * nl), acts(nl), nodes(nl), act(nl))
            code = c_model_network(handle%model, z(e), nl, c_loc(dims), c_loc(acts), c_null_ptr)
            if (code /= 0) call fail_stop(code)
            allocate(vals(sum(dims(1::2) * dims(2::2) + dims(2::2))))
            code = c_model_network(handle%model, z(e), nl, c_loc(dims), c_loc(acts), c_loc(vals))
            if (code /= 0) call fail_stop(code)
            do l = 1, nl
                nodes(l) = dims(2 * l)
                act(l) = acts(l)
            end do
            call nn_new(handle%nnList(z(e)), dims(1), nl, nodes, act)
            o = 0
            do l = 1, nl
                handle%nnList(z(e))%layers(l)%weights = reshape(vals(o + 1:o + dims(2 * l - 1) * dims(2 * l)), &
                                                                 [dims(2 * l), dims(2 * l - 1)])
                o = o + dims(2 * l - 1) * dims(2 * l)
                handle%nnList(z(e))%layers(l)%bias = vals(o + 1:o + dims(2 * l))
                o = o + dims(2 * l)
            end do
            deallocate(dims, acts, nodes, act, vals)
        end do
    end subroutine fill_components

    subroutine struct_args(ats, el, periodic, lat)
        type(atStruct), intent(in) :: ats
        integer(c_int32_t), allocatable, intent(out) :: el(:)
        integer(c_int), intent(out) :: periodic
        real(c_double), intent(out) :: lat(9)
        allocate(el(ats%nat))
        el = int(ats%el, c_int32_t)
        periodic = 0
        lat = [1._dp, 0._dp, 0._dp, 0._dp, 1._dp, 0._dp, 0._dp, 0._dp, 1._dp]
        if (ats%periodic) then
            periodic = 1
            lat = reshape(ats%lat, [9])
        end if
    end subroutine struct_args

    ! hdnnpCalcNeighborLists (hdnnps.f90:373): lists on the GPU, returned in
    ! the reference's layout (entry 1 = the atom itself; 1-based indices).
    subroutine hdnnpCalcNeighborLists(handle, ats, neiLists)
        type(hdnnp), intent(in) :: handle
        type(atStruct), intent(in) :: ats
        type(neighborList), intent(out) :: neiLists(ats%nat)
        integer(c_int32_t), allocatable :: el(:)
        integer(c_int) :: code, periodic, nent
        integer(c_int), allocatable, target :: nneis(:), ineis(:)
        real(c_double), allocatable, target :: neis(:)
        real(c_double) :: lat(9)
        integer :: i, o

        call struct_args(ats, el, periodic, lat)
        code = c_calc_neighbor_lists(handle%ctx, int(ats%nat, c_int), el, ats%ats, periodic, lat, nent)
        if (code /= 0) call fail_stop(code)
        allocate(nneis(ats%nat))
        code = c_neighbor_lists_fetch(handle%ctx, nneis, c_null_ptr, c_null_ptr)
        if (code /= 0) call fail_stop(code)
        allocate(ineis(sum(nneis)), neis(3 * sum(nneis)))
        code = c_neighbor_lists_fetch(handle%ctx, nneis, c_loc(ineis), c_loc(neis))
        if (code /= 0) call fail_stop(code)
        o = 0
        do i = 1, ats%nat
            neiLists(i)%nNeis = nneis(i)
            neiLists(i)%maxNeis = nneis(i)
            allocate(neiLists(i)%ineis(nneis(i)), neiLists(i)%neis(3, nneis(i)))
            neiLists(i)%ineis = ineis(o + 1:o + nneis(i)) + 1
            neiLists(i)%neis = reshape(neis(3 * o + 1:3 * (o + nneis(i))), [3, nneis(i)])
            o = o + nneis(i)
        end do
    end subroutine hdnnpCalcNeighborLists

    ! hdnnpCalcSymfunctions (hdnnps.f90:390): the scaled values of the
    ! structure of the last hdnnpCalcNeighborLists of this handle; dsf is not
    ! allocated (the derivatives stay implicit, see hdnnpCalcNNs).
    subroutine hdnnpCalcSymfunctions(handle, ats, neiLists, sfs, calcSfsTogether)
        type(hdnnp), intent(in) :: handle
        type(atStruct), intent(in) :: ats
        type(neighborList), intent(in) :: neiLists(ats%nat)
        type(symFunctionContainer), intent(out) :: sfs(ats%nat)
        logical, intent(in), optional :: calcSfsTogether
        real(c_double), allocatable, target :: g(:, :)
        integer(c_int) :: code
        integer :: iat, isf

        allocate(g(handle%nsfMax, ats%nat))  ! the C layout: nat rows of nsf_max
        code = c_calc_symfunctions(handle%ctx, c_loc(g))
        if (code /= 0) call fail_stop(code)
        stage_ctx = handle%ctx
        do iat = 1, ats%nat
            sfs(iat)%nsf = handle%sfLists(ats%el(iat))%nsf
            allocate(sfs(iat)%sfs(sfs(iat)%nsf))
            do isf = 1, sfs(iat)%nsf
                sfs(iat)%sfs(isf)%nNeis = neiLists(iat)%nNeis
                sfs(iat)%sfs(isf)%sf = g(isf, iat)
            end do
        end do
    end subroutine hdnnpCalcSymfunctions

    ! hdnnpCalcNNs (hdnnps.f90:487): this handle's networks on the symmetry
    ! functions of the last hdnnpCalcSymfunctions (of any handle, as the
    ! reference's committee does) and the force / dEdLat contraction.
    subroutine hdnnpCalcNNs(handle, ats, neiLists, sfs, energy, force, dEdLat)
        type(hdnnp), intent(inout) :: handle
        type(atStruct), intent(in) :: ats
        type(neighborList), intent(in) :: neiLists(ats%nat)
        type(symFunctionContainer), intent(in) :: sfs(ats%nat)
        real(dp), intent(out) :: energy
        real(dp), intent(out) :: force(3, ats%nat)
        real(dp), intent(out), optional, target :: dEdLat(3,3)
        integer(c_int) :: code
        type(c_ptr) :: pdl

        if (.not. c_associated(stage_ctx)) then
            print*, 'hdnnpCalcNNs: no symmetry functions (call hdnnpCalcSymfunctions first)'
            stop
        end if
        pdl = c_null_ptr
        if (present(dEdLat)) pdl = c_loc(dEdLat)
        code = c_calc_nns(stage_ctx, handle%model, energy, force, pdl)
        if (code /= 0) call fail_stop(code)
    end subroutine hdnnpCalcNNs

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

        call struct_args(ats, el, periodic, lat)
        pdl = c_null_ptr
        if (present(dEdLat)) pdl = c_loc(dEdLat)
        code = c_energy_and_forces(handle%ctx, int(ats%nat, c_int), el, ats%ats, periodic, lat, energy, force, pdl)
        if (code /= 0) call fail_stop(code)
    end subroutine hdnnpEnergyAndForces

    subroutine hdnnpFree(handle)
        type(hdnnp), intent(inout) :: handle
        if (c_associated(handle%ctx) .and. c_associated(stage_ctx, handle%ctx)) stage_ctx = c_null_ptr
        if (c_associated(handle%ctx)) call c_ctx_free(handle%ctx)
        if (c_associated(handle%model)) call c_model_free(handle%model)
        handle%ctx = c_null_ptr
        handle%model = c_null_ptr
    end subroutine hdnnpFree

end module hdnnps_gpu
