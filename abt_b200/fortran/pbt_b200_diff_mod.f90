! pbt_b200_diff_mod.f90 -- Fortran side of the drop-in boundary.
!
! Provides diff_main, diffraction and finalise with the reference's argument
! lists (src/diff_mod.f90:674, :446 and src/outputs_mod.f90:63) and forwards
! them to libpbt_b200.so through iso_c_binding.  A build links this module
! in place of diff_mod.o / the finalise routine and adds -lpbt_b200.
!
! The reference's outbeamtype is not bind(C); diff_main packs the fields that
! diffraction reads (ampl, vk7, prop_out, fov, fi) into pbt_outbeam records
! and the facet vertex lists of geometry_type into a CSR.
!
! Build: compile this module with the reference's sources in place of
! diff_mod.f90 and link libpbt_b200.so (e.g. gfortran -c pbt_b200_diff_mod.f90
! after types_mod.o; link with -L<dir> -lpbt_b200).  It has not been compiled
! on the machine that built the library, which has no Fortran compiler.
module pbt_b200_diff_mod

    use, intrinsic :: iso_c_binding
    use types_mod

    implicit none

    integer(c_int), parameter :: PBT_PREC_FP64 = 0, PBT_PREC_FP32 = 1

    type, bind(C) :: pbt_outbeam
        real(c_double) :: ampl(8)      ! ampl(1:2,1:2) complex(8), column-major, re/im
        real(c_double) :: vk7(3)
        real(c_double) :: prop_out(3)
        real(c_double) :: fov
        integer(c_int64_t) :: fi
    end type

    type, bind(C) :: pbt_output_params
        real(c_double) :: abs, scatt, ext, albedo, asymmetry, abs_eff, scatt_eff, ext_eff, &
                          geo_cross_sec, back_scatt, beam_energy_out, ext_energy_out, &
                          scatt_beam, scatt_ext_diff, asymmetry_beam, asymmetry_ext_diff, &
                          scatt_eff_beam, scatt_eff_ext_diff
    end type

    type(c_ptr), save :: pbt_ctx = c_null_ptr
    integer(c_int), save :: pbt_precision = PBT_PREC_FP64
    ! device of the context: -1 (PBT_DEVICE_LOCAL_RANK) takes the node-local rank of
    ! an MPI launcher modulo the visible devices, so that the reference's MPI build
    ! spreads its ranks over a node's GPUs; set it before the first call to pin one
    integer(c_int), save :: pbt_device = -1_c_int

    interface
        integer(c_int) function pbt_ctx_create(device, ctx) bind(C, name="pbt_ctx_create")
            import :: c_int, c_ptr
            integer(c_int), value :: device
            type(c_ptr) :: ctx
        end function
        type(c_ptr) function pbt_last_error_string() bind(C, name="pbt_last_error_string")
            import :: c_ptr
        end function
        integer(c_int) function pbt_diff_main_c(ctx, beam, nbeam, ext, next, verts, nverts, &
                face_off, face_vi, nfaces, theta, ntheta, phi, nphi, lambda, is_fast_diff, &
                precision, ampl_far_beam, ampl_far_ext_diff) bind(C, name="pbt_diff_main_c")
            import :: c_int, c_int32_t, c_int64_t, c_double, c_double_complex, c_ptr, pbt_outbeam
            type(c_ptr), value :: ctx
            type(pbt_outbeam), intent(in) :: beam(*), ext(*)
            integer(c_int64_t), value :: nbeam, next, nverts, nfaces, ntheta, nphi
            real(c_double), intent(in) :: verts(*), theta(*), phi(*)
            integer(c_int64_t), intent(in) :: face_off(*), face_vi(*)
            real(c_double), value :: lambda
            integer(c_int32_t), value :: is_fast_diff, precision
            complex(c_double_complex), intent(out) :: ampl_far_beam(*), ampl_far_ext_diff(*)
        end function
        integer(c_int) function pbt_diffraction_c(ctx, outbeam, verts, nverts, face_off, face_vi, &
                nfaces, theta, ntheta, phi, nphi, lambda, is_fast_diff, amplC) &
                bind(C, name="pbt_diffraction_c")
            import :: c_int, c_int32_t, c_int64_t, c_double, c_double_complex, c_ptr, pbt_outbeam
            type(c_ptr), value :: ctx
            type(pbt_outbeam), intent(in) :: outbeam
            integer(c_int64_t), value :: nverts, nfaces, ntheta, nphi
            real(c_double), intent(in) :: verts(*), theta(*), phi(*)
            integer(c_int64_t), intent(in) :: face_off(*), face_vi(*)
            real(c_double), value :: lambda
            integer(c_int32_t), value :: is_fast_diff
            complex(c_double_complex), intent(out) :: amplC(*)
        end function
        integer(c_int) function pbt_finalise_c(ctx, ampl_far_beam, ampl_far_ext_diff, theta, &
                ntheta, phi, nphi, lambda, scaling, params, mueller, mueller_1d, accumulate) &
                bind(C, name="pbt_finalise_c")
            import :: c_int, c_int32_t, c_int64_t, c_double, c_double_complex, c_ptr, pbt_output_params
            type(c_ptr), value :: ctx
            complex(c_double_complex), intent(in) :: ampl_far_beam(*), ampl_far_ext_diff(*)
            real(c_double), intent(in) :: theta(*), phi(*)
            integer(c_int64_t), value :: ntheta, nphi
            real(c_double), value :: lambda
            integer(c_int32_t), value :: scaling, accumulate
            type(pbt_output_params), intent(inout) :: params
            real(c_double), intent(out) :: mueller(*), mueller_1d(*)
        end function
        integer(c_int) function pbt_beamlist_writer_open(path, theta, ntheta, phi, nphi, nverts, &
                                                         face_off, face_vi, nfaces, lambda, w) &
                                                         bind(C, name="pbt_beamlist_writer_open")
            import :: c_int, c_char, c_double, c_int64_t, c_ptr
            character(kind=c_char), dimension(*), intent(in) :: path
            real(c_double), intent(in) :: theta(*), phi(*)
            integer(c_int64_t), value :: ntheta, nphi, nverts, nfaces
            integer(c_int64_t), intent(in) :: face_off(*), face_vi(*)
            real(c_double), value :: lambda
            type(c_ptr), intent(out) :: w
        end function
        integer(c_int) function pbt_beamlist_writer_add(w, beam, nbeam, ext, next, verts, params_in) &
                                                        bind(C, name="pbt_beamlist_writer_add")
            import :: c_int, c_int64_t, c_double, c_ptr, pbt_outbeam, pbt_output_params
            type(c_ptr), value :: w
            type(pbt_outbeam), intent(in) :: beam(*), ext(*)
            integer(c_int64_t), value :: nbeam, next
            real(c_double), intent(in) :: verts(*)
            type(pbt_output_params), intent(in) :: params_in
        end function
        integer(c_int) function pbt_make_far_field_bins_c(theta, ntheta, phi, nphi, x, y, z) &
                                                          bind(C, name="pbt_make_far_field_bins_c")
            import :: c_int, c_int64_t, c_double
            real(c_double), intent(in) :: theta(*), phi(*)
            integer(c_int64_t), value :: ntheta, nphi
            real(c_double), intent(out) :: x(*), y(*), z(*)
        end function
        integer(c_int) function pbt_beamlist_writer_close(w) bind(C, name="pbt_beamlist_writer_close")
            import :: c_int, c_ptr
            type(c_ptr), value :: w
        end function
    end interface

    type(c_ptr), save :: pbt_dump = c_null_ptr

    contains

    subroutine pbt_check(status, what)
        integer(c_int), intent(in) :: status
        character(*), intent(in) :: what
        character(kind=c_char), pointer :: msg(:)
        integer :: n
        if (status == 0) return
        call c_f_pointer(pbt_last_error_string(), msg, [1024])
        n = 0
        do while (n < 1024)
            if (msg(n + 1) == c_null_char) exit
            n = n + 1
        end do
        print *, what, ' failed: ', msg(1:n)
        error stop
    end subroutine

    subroutine pbt_init()
        if (.not. c_associated(pbt_ctx)) call pbt_check(pbt_ctx_create(pbt_device, pbt_ctx), 'pbt_ctx_create')
    end subroutine

    ! facet vertex CSR of the geometry (geometry%f(:)%vi), 0-based offsets
    subroutine pack_faces(geometry, face_off, face_vi)
        type(geometry_type), intent(in) :: geometry
        integer(c_int64_t), allocatable, intent(out) :: face_off(:), face_vi(:)
        integer(8) :: f, n
        allocate(face_off(geometry%nf + 1))
        face_off(1) = 0
        do f = 1, geometry%nf
            face_off(f + 1) = face_off(f) + geometry%f(f)%nv
        end do
        allocate(face_vi(face_off(geometry%nf + 1)))
        do f = 1, geometry%nf
            n = geometry%f(f)%nv
            face_vi(face_off(f) + 1:face_off(f) + n) = geometry%f(f)%vi(1:n)
        end do
    end subroutine

    subroutine pack_outbeam(ob, p)
        type(outbeamtype), intent(in) :: ob
        type(pbt_outbeam), intent(out) :: p
        p%ampl = [real(ob%ampl(1,1)), aimag(ob%ampl(1,1)), real(ob%ampl(2,1)), aimag(ob%ampl(2,1)), &
                  real(ob%ampl(1,2)), aimag(ob%ampl(1,2)), real(ob%ampl(2,2)), aimag(ob%ampl(2,2))]
        p%vk7 = ob%vk7
        p%prop_out = ob%prop_out
        p%fov = ob%fov
        p%fi = ob%fi
    end subroutine

    ! same argument list as diff_main, src/diff_mod.f90:674-680
    subroutine diff_main(beam_outbeam_tree, beam_outbeam_tree_counter, ampl_far_beam, &
                         ext_diff_outbeam_tree, ampl_far_ext_diff, job_params, geometry)
        type(outbeamtype), dimension(:), allocatable, intent(inout) :: beam_outbeam_tree
        integer(8), intent(inout) :: beam_outbeam_tree_counter
        complex(8), dimension(:,:,:,:), allocatable, intent(out) :: ampl_far_beam
        type(outbeamtype), dimension(:), allocatable, intent(in) :: ext_diff_outbeam_tree
        complex(8), dimension(:,:,:,:), allocatable, intent(out) :: ampl_far_ext_diff
        type(job_parameters_type), intent(in) :: job_params
        type(geometry_type), intent(in) :: geometry

        type(pbt_outbeam), allocatable :: pb(:), pe(:)
        integer(c_int64_t), allocatable :: face_off(:), face_vi(:)
        integer(8) :: j, nphi, ntheta, next
        integer(c_int32_t) :: fast

        call pbt_init()
        nphi = size(job_params%phi_vals, 1)
        ntheta = size(job_params%theta_vals, 1)
        next = size(ext_diff_outbeam_tree, 1)
        allocate(ampl_far_beam(nphi, ntheta, 2, 2), ampl_far_ext_diff(nphi, ntheta, 2, 2))
        allocate(pb(max(1_8, beam_outbeam_tree_counter)), pe(max(1_8, next)))
        do j = 1, beam_outbeam_tree_counter
            call pack_outbeam(beam_outbeam_tree(j), pb(j))
        end do
        do j = 1, next
            call pack_outbeam(ext_diff_outbeam_tree(j), pe(j))
        end do
        call pack_faces(geometry, face_off, face_vi)
        fast = merge(1_c_int32_t, 0_c_int32_t, job_params%is_fast_diff)
        call pbt_check(pbt_diff_main_c(pbt_ctx, pb, int(beam_outbeam_tree_counter, c_int64_t), pe, &
                       int(next, c_int64_t), geometry%v, int(size(geometry%v, 1), c_int64_t), &
                       face_off, face_vi, int(geometry%nf, c_int64_t), job_params%theta_vals, &
                       int(ntheta, c_int64_t), job_params%phi_vals, int(nphi, c_int64_t), &
                       job_params%la, fast, pbt_precision, ampl_far_beam, ampl_far_ext_diff), &
                       'pbt_diff_main_c')
    end subroutine

    ! same argument list as diffraction, src/diff_mod.f90:446-455 (the -memory path)
    subroutine diffraction(xfar, yfar, zfar, lambda, amplC, phi_vals, theta_vals, job_params, &
                           outbeam, geometry)
        real(8), dimension(:,:), allocatable, intent(in) :: xfar, yfar, zfar  ! recomputed by the library
        real(8), intent(in) :: lambda
        complex(8), dimension(:,:,:,:), allocatable, intent(inout) :: amplC
        real(8), dimension(:), allocatable, intent(in) :: phi_vals, theta_vals
        type(job_parameters_type), intent(in) :: job_params
        type(outbeamtype), intent(in) :: outbeam
        type(geometry_type), intent(in) :: geometry

        type(pbt_outbeam) :: p
        integer(c_int64_t), allocatable :: face_off(:), face_vi(:)
        integer(c_int32_t) :: fast

        call pbt_init()
        call pack_outbeam(outbeam, p)
        call pack_faces(geometry, face_off, face_vi)
        fast = merge(1_c_int32_t, 0_c_int32_t, job_params%is_fast_diff)
        call pbt_check(pbt_diffraction_c(pbt_ctx, p, geometry%v, int(size(geometry%v, 1), c_int64_t), &
                       face_off, face_vi, int(geometry%nf, c_int64_t), theta_vals, &
                       int(size(theta_vals), c_int64_t), phi_vals, int(size(phi_vals), c_int64_t), &
                       lambda, fast, amplC), 'pbt_diffraction_c')
    end subroutine

    ! same argument list as make_far_field_bins, src/diff_mod.f90:827-836
    subroutine make_far_field_bins(x, y, z, theta_vals, phi_vals)
        real(8), dimension(:,:), allocatable, intent(out) :: x, y, z
        real(8), dimension(:), allocatable, intent(in) :: theta_vals
        real(8), dimension(:), allocatable, intent(in) :: phi_vals
        integer(8) :: nphi, ntheta
        nphi = size(phi_vals, 1)
        ntheta = size(theta_vals, 1)
        allocate(x(nphi, ntheta), y(nphi, ntheta), z(nphi, ntheta))
        call pbt_check(pbt_make_far_field_bins_c(theta_vals, int(ntheta, c_int64_t), phi_vals, &
                       int(nphi, c_int64_t), x, y, z), 'pbt_make_far_field_bins_c')
    end subroutine

    ! Beam-list dump: open once before the orientation loop, call
    ! pbt_dump_orientation beside diff_main (src/pbt_seq_mod.f90:212) with the
    ! same outbeam lists and the rotated geometry, close after the loop.  The
    ! file replays through pbt_diff_batch_c (abt_b200.beamlist in Python).
    subroutine pbt_dump_open(path, job_params, geometry)
        character(len=*), intent(in) :: path
        type(job_parameters_type), intent(in) :: job_params
        type(geometry_type), intent(in) :: geometry
        integer(c_int64_t), allocatable :: face_off(:), face_vi(:)
        call pack_faces(geometry, face_off, face_vi)
        call pbt_check(pbt_beamlist_writer_open(trim(path) // c_null_char, job_params%theta_vals, &
                       int(size(job_params%theta_vals), c_int64_t), job_params%phi_vals, &
                       int(size(job_params%phi_vals), c_int64_t), int(size(geometry%v, 1), c_int64_t), &
                       face_off, face_vi, int(geometry%nf, c_int64_t), job_params%la, pbt_dump), &
                       'pbt_beamlist_writer_open')
    end subroutine

    subroutine pbt_dump_orientation(beam_outbeam_tree, beam_outbeam_tree_counter, &
                                    ext_diff_outbeam_tree, geometry, params_in)
        type(outbeamtype), dimension(:), allocatable, intent(in) :: beam_outbeam_tree
        integer(8), intent(in) :: beam_outbeam_tree_counter
        type(outbeamtype), dimension(:), allocatable, intent(in) :: ext_diff_outbeam_tree
        type(geometry_type), intent(in) :: geometry
        type(pbt_output_params), intent(in) :: params_in   ! abs, geo_cross_sec, energies
        type(pbt_outbeam), allocatable :: pb(:), pe(:)
        integer(8) :: j, next
        next = size(ext_diff_outbeam_tree, 1)
        allocate(pb(max(1_8, beam_outbeam_tree_counter)), pe(max(1_8, next)))
        do j = 1, beam_outbeam_tree_counter
            call pack_outbeam(beam_outbeam_tree(j), pb(j))
        end do
        do j = 1, next
            call pack_outbeam(ext_diff_outbeam_tree(j), pe(j))
        end do
        call pbt_check(pbt_beamlist_writer_add(pbt_dump, pb, int(beam_outbeam_tree_counter, c_int64_t), &
                       pe, int(next, c_int64_t), geometry%v, params_in), 'pbt_beamlist_writer_add')
    end subroutine

    subroutine pbt_dump_close()
        call pbt_check(pbt_beamlist_writer_close(pbt_dump), 'pbt_beamlist_writer_close')
        pbt_dump = c_null_ptr
    end subroutine

end module pbt_b200_diff_mod
