! mps_linsolve_c.f90 -- ISO_C_BINDING interface to libmps3d_b200 (the C ABI
! of include/mps_linsolve.h) for the reference's Fortran host.
!
! A maintainer adds this module to mgridlib and links -lmps3d_b200 -lcudart.
! The derived types are bind(C), so a Fortran compiler lays them out with
! the companion C compiler's rules; their component order and kinds follow
! the structs of mps_linsolve.h one for one (mps_solver.cu static_asserts
! the offsets this module relies on, and tests/test_fortran_binding.py
! checks this file's types and interfaces against the header).
!
! Array arguments are type(c_ptr), value: pass c_loc() of the reference's
! target arrays (host entry points) or of device arrays (the *_dev entry
! points: CUDA Fortran device arrays, or host_data use_device under
! OpenACC).  Streams are type(c_ptr), value: c_null_ptr is the handle's
! own stream; the legacy default stream is transfer(1_c_intptr_t, c_null_ptr).
!
! Entry points and the reference code they replace:
!   mps_linsolve / mps_linsolve_dev : the loop "do i=1,nvcycles; call
!       perform_vcycle(...); if(resnorm .le. err_tol) exit" of
!       plasma_pde/poissoneq.f90:427-450 (and edeneq, ionseq, eenergyeq,
!       neutralseq, generic_pde/pdedefs.f90:304-328)
!   mps_vcycle_once  : one perform_vcycle call, mgridlib/mgridsteps.f90:384-417
!   mps_apply_A_dev  : find_AX, mgridlib/discretepde.f90:672-1119
!   mps_find_bvec_dev: find_bvec, mgridlib/discretepde.f90:382-618
!   mps_fill_ghosts_dev: update_boundary_ghostvalues, discretepde.f90:1121-1267
module mps_linsolve_c
    use iso_c_binding
    implicit none

    integer(c_int), parameter :: MPS_OK = 0, MPS_ERR_NOT_CONVERGED = 1, MPS_ERR_NAN = 2, &
                                 MPS_ERR_BREAKDOWN = 3, MPS_ERR_BAD_ARG = 4, MPS_ERR_TIMEOUT = 5, &
                                 MPS_ERR_CUDA = 6, MPS_ERR_NOMEM = 7, MPS_ERR_TOO_LARGE = 8
    integer(c_int), parameter :: MPS_BC_DIRC = 1, MPS_BC_FLUX = 2, MPS_BC_ZGRD = 3, &
                                 MPS_BC_PERI = 4, MPS_BC_DZGD = 5
    integer(c_int), parameter :: MPS_HIER_CELL = 0, MPS_HIER_GEOM = 1
    integer(c_int), parameter :: MPS_PREC_FP64 = 0, MPS_PREC_MIXED = 1
    integer(c_int), parameter :: MPS_KRYLOV_NONE = 0, MPS_KRYLOV_FGMRES = 1
    integer(c_int), parameter :: MPS_FLUX_UPWIND = 0, MPS_FLUX_SG = 1
    integer(c_int), parameter :: MPS_TOL_RMS_ABS = 0, MPS_TOL_REL_L2 = 1
    integer(c_int), parameter :: MPS_NOALLOC_MAX_CELLS = 262144

    type, bind(C) :: mps_grid
        integer(c_int) :: lx, ly, lz
        real(c_double) :: llenx, lleny, llenz
    end type

    type, bind(C) :: mps_solver_opts
        real(c_double) :: tol
        integer(c_int) :: tol_kind, maxit, nu1, nu2, hierarchy
        integer(c_int) :: ranks(3)
        integer(c_int) :: max_coarse, precision, inner_cycles, krylov, restart
        integer(c_int) :: fill_ghosts, use_graph, transpose, flux
    end type

    type, bind(C) :: mps_solve_info
        integer(c_int) :: status, iters, vcycles, levels
        real(c_double) :: rel_res, rms_res, rel_res0, time_ms
        integer(c_int) :: launches
    end type

    type, bind(C) :: mps_profile
        integer(c_int) :: count(8)
        real(c_double) :: ms(8)
        integer(c_int) :: precision_bytes, coeff_field
        integer(c_long_long) :: cells
    end type

    type, bind(C) :: mps_problem
        type(mps_grid) :: g
        integer(c_int) :: timederiv
        real(c_double) :: dt
        type(c_ptr) :: vel, dcoeff, reac, source
        integer(c_int) :: bc_code(6)
        type(c_ptr) :: bcval(6)
        type(c_ptr) :: mgridsterm, soln
    end type

    ! the fields of one implicit potential + electron step (device pointers)
    type, bind(C) :: mps_plasma_step
        type(mps_grid) :: g
        integer(c_int) :: phi_bc(6)
        type(c_ptr) :: phi_bcval(6)
        type(c_ptr) :: eps, phi
        real(c_double) :: rho_scale
        integer(c_int) :: nion
        type(c_ptr) :: n_ion, ion_charge, phi_source
        integer(c_int) :: ne_bc(6)
        type(c_ptr) :: ne_bcval(6)
        type(c_ptr) :: n_e, mu_e, d_e, te, prod_e
        real(c_double) :: dt, nemin, efield_scale
        integer(c_int) :: limiter
        real(c_double) :: vel_scaling, dcoeff_scaling, source_scaling
        type(c_ptr) :: efield, vel, dcoeff, source
    end type

    interface
        subroutine mps_default_opts(o) bind(C, name="mps_default_opts")
            import :: mps_solver_opts
            type(mps_solver_opts), intent(out) :: o
        end subroutine

        type(c_ptr) function mps_version() bind(C, name="mps_version")
            import :: c_ptr
        end function

        integer(c_int) function mps_create(h, device) bind(C, name="mps_create")
            import :: c_ptr, c_int
            type(c_ptr), intent(out) :: h
            integer(c_int), value :: device
        end function

        integer(c_int) function mps_destroy(h) bind(C, name="mps_destroy")
            import :: c_ptr, c_int
            type(c_ptr), value :: h
        end function

        type(c_ptr) function mps_stream(h) bind(C, name="mps_stream")
            import :: c_ptr
            type(c_ptr), value :: h
        end function

        type(c_ptr) function mps_last_error(h) bind(C, name="mps_last_error")
            import :: c_ptr
            type(c_ptr), value :: h
        end function

        integer(c_int) function mps_linsolve(h, g, timederiv, dt, vel, dcoeff, reac, source, &
                bc_code, bcval, mgridsterm, soln, opts, info) bind(C, name="mps_linsolve")
            import :: c_ptr, c_int, c_double, mps_grid, mps_solver_opts, mps_solve_info
            type(c_ptr), value :: h
            type(mps_grid), intent(in) :: g
            integer(c_int), value :: timederiv
            real(c_double), value :: dt
            type(c_ptr), value :: vel, dcoeff, reac, source
            integer(c_int), intent(in) :: bc_code(6)
            type(c_ptr), intent(in) :: bcval(6)
            type(c_ptr), value :: mgridsterm, soln
            type(mps_solver_opts), intent(in) :: opts
            type(mps_solve_info), intent(out) :: info
        end function

        integer(c_int) function mps_linsolve_dev(h, g, timederiv, dt, vel, dcoeff, reac, source, &
                bc_code, bcval, mgridsterm, soln, opts, info, stream) bind(C, name="mps_linsolve_dev")
            import :: c_ptr, c_int, c_double, mps_grid, mps_solver_opts, mps_solve_info
            type(c_ptr), value :: h
            type(mps_grid), intent(in) :: g
            integer(c_int), value :: timederiv
            real(c_double), value :: dt
            type(c_ptr), value :: vel, dcoeff, reac, source
            integer(c_int), intent(in) :: bc_code(6)
            type(c_ptr), intent(in) :: bcval(6)
            type(c_ptr), value :: mgridsterm, soln
            type(mps_solver_opts), intent(in) :: opts
            type(mps_solve_info), intent(out) :: info
            type(c_ptr), value :: stream
        end function

        integer(c_int) function mps_vcycle_once(h, g, timederiv, dt, vel, dcoeff, reac, source, &
                bc_code, bcval, mgridsterm, soln, resnorm, opts) bind(C, name="mps_vcycle_once")
            import :: c_ptr, c_int, c_double, mps_grid
            type(c_ptr), value :: h
            type(mps_grid), intent(in) :: g
            integer(c_int), value :: timederiv
            real(c_double), value :: dt
            type(c_ptr), value :: vel, dcoeff, reac, source
            integer(c_int), intent(in) :: bc_code(6)
            type(c_ptr), intent(in) :: bcval(6)
            type(c_ptr), value :: mgridsterm, soln
            real(c_double), intent(out) :: resnorm
            type(c_ptr), value :: opts          ! c_null_ptr: reference hierarchy, 2/2 sweeps
        end function

        integer(c_int) function mps_apply_A_dev(h, g, timederiv, dt, vel, dcoeff, reac, bc_code, &
                soln, ax, opts, stream) bind(C, name="mps_apply_A_dev")
            import :: c_ptr, c_int, c_double, mps_grid
            type(c_ptr), value :: h
            type(mps_grid), intent(in) :: g
            integer(c_int), value :: timederiv
            real(c_double), value :: dt
            type(c_ptr), value :: vel, dcoeff, reac
            integer(c_int), intent(in) :: bc_code(6)
            type(c_ptr), value :: soln, ax
            type(c_ptr), value :: opts          ! c_null_ptr: upwind flux, no transpose
            type(c_ptr), value :: stream
        end function

        integer(c_int) function mps_find_bvec_dev(h, g, vel, dcoeff, source, bc_code, bcval, &
                mgridsterm, b, opts, stream) bind(C, name="mps_find_bvec_dev")
            import :: c_ptr, c_int, mps_grid
            type(c_ptr), value :: h
            type(mps_grid), intent(in) :: g
            type(c_ptr), value :: vel, dcoeff, source
            integer(c_int), intent(in) :: bc_code(6)
            type(c_ptr), intent(in) :: bcval(6)
            type(c_ptr), value :: mgridsterm, b
            type(c_ptr), value :: opts          ! c_null_ptr: upwind flux
            type(c_ptr), value :: stream
        end function

        integer(c_int) function mps_set_profile(h, on) bind(C, name="mps_set_profile")
            import :: c_ptr, c_int
            type(c_ptr), value :: h
            integer(c_int), value :: on
        end function

        integer(c_int) function mps_get_profile(h, p, reset) bind(C, name="mps_get_profile")
            import :: c_ptr, c_int, mps_profile
            type(c_ptr), value :: h
            type(mps_profile), intent(out) :: p
            integer(c_int), value :: reset
        end function

        integer(c_int) function mps_fill_ghosts_dev(h, g, bc_code, bcval, soln, stream) &
                bind(C, name="mps_fill_ghosts_dev")
            import :: c_ptr, c_int, mps_grid
            type(c_ptr), value :: h
            type(mps_grid), intent(in) :: g
            integer(c_int), intent(in) :: bc_code(6)
            type(c_ptr), intent(in) :: bcval(6)
            type(c_ptr), value :: soln
            type(c_ptr), value :: stream
        end function

        integer(c_int) function mps_linsolve_batched_dev(h, nprob, probs, opts, infos, stream) &
                bind(C, name="mps_linsolve_batched_dev")
            import :: c_ptr, c_int, mps_problem, mps_solver_opts, mps_solve_info
            type(c_ptr), value :: h
            integer(c_int), value :: nprob
            type(mps_problem), intent(in) :: probs(nprob)
            type(mps_solver_opts), intent(in) :: opts
            type(mps_solve_info), intent(out) :: infos(nprob)
            type(c_ptr), value :: stream
        end function

        integer(c_int) function mps_operator_vjp_dev(g, vel, dcoeff, bc_code, lam, u, opts, &
                gvel, gdcoeff, greac, stream) bind(C, name="mps_operator_vjp_dev")
            import :: c_ptr, c_int, mps_grid
            type(mps_grid), intent(in) :: g
            type(c_ptr), value :: vel, dcoeff
            integer(c_int), intent(in) :: bc_code(6)
            type(c_ptr), value :: lam, u
            type(c_ptr), value :: opts          ! c_null_ptr: upwind flux
            type(c_ptr), value :: gvel, gdcoeff, greac
            type(c_ptr), value :: stream
        end function

        ! update_efield, plasma_pde/poissoneq.f90:565-680
        integer(c_int) function mps_efield_dev(g, phi_bc, phi_bcval, phi, scale, limiter, efield, stream) &
                bind(C, name="mps_efield_dev")
            import :: c_ptr, c_int, c_double, mps_grid
            type(mps_grid), intent(in) :: g
            integer(c_int), intent(in) :: phi_bc(6)
            type(c_ptr), intent(in) :: phi_bcval(6)
            type(c_ptr), value :: phi
            real(c_double), value :: scale
            integer(c_int), value :: limiter
            type(c_ptr), value :: efield
            type(c_ptr), value :: stream
        end function

        ! eden_update_transport, plasma_pde/edeneq.f90:360-444
        integer(c_int) function mps_eden_transport_dev(g, efield, mu_e, dco, te, prod, n_old, timederiv, dt, &
                scaling, vel, dcoeff, source, stream) bind(C, name="mps_eden_transport_dev")
            import :: c_ptr, c_int, c_double, mps_grid
            type(mps_grid), intent(in) :: g
            type(c_ptr), value :: efield, mu_e, dco, te, prod, n_old
            integer(c_int), value :: timederiv
            real(c_double), value :: dt
            real(c_double), intent(in) :: scaling(3)
            type(c_ptr), value :: vel, dcoeff, source
            type(c_ptr), value :: stream
        end function

        ! poisson_update_transport, plasma_pde/poissoneq.f90:335-385
        integer(c_int) function mps_poisson_source_dev(g, n_e, nspec, n_ion, charge, scale, phi_old, dt, &
                source, stream) bind(C, name="mps_poisson_source_dev")
            import :: c_ptr, c_int, c_double, mps_grid
            type(mps_grid), intent(in) :: g
            type(c_ptr), value :: n_e
            integer(c_int), value :: nspec
            type(c_ptr), value :: n_ion, charge
            real(c_double), value :: scale
            type(c_ptr), value :: phi_old
            real(c_double), value :: dt
            type(c_ptr), value :: source
            type(c_ptr), value :: stream
        end function

        ! potential + electron part of the time step, solve_manager.f90:363-502
        integer(c_int) function mps_plasma_step_dev(hp, he, step, opts_phi, opts_e, info_phi, info_e, stream) &
                bind(C, name="mps_plasma_step_dev")
            import :: c_ptr, c_int, mps_plasma_step, mps_solver_opts, mps_solve_info
            type(c_ptr), value :: hp, he
            type(mps_plasma_step), intent(in) :: step
            type(mps_solver_opts), intent(in) :: opts_phi, opts_e
            type(mps_solve_info), intent(out) :: info_phi, info_e
            type(c_ptr), value :: stream
        end function

        ! VTK output, mgridlib/cartwrite.f90 (names: trim(name)//c_null_char)
        integer(c_int) function mps_write_vtr_dev(filename, g, off, nscalars, names, fields, stream) &
                bind(C, name="mps_write_vtr_dev")
            import :: c_ptr, c_int, c_char, c_double, mps_grid
            character(kind=c_char), intent(in) :: filename(*)
            type(mps_grid), intent(in) :: g
            real(c_double), intent(in) :: off(3)
            integer(c_int), value :: nscalars
            type(c_ptr), intent(in) :: names(*)
            type(c_ptr), intent(in) :: fields(*)
            type(c_ptr), value :: stream
        end function

        integer(c_int) function mps_write_vtr_piece_dev(dirname, rank, pind, g, off, nscalars, names, fields, &
                stream) bind(C, name="mps_write_vtr_piece_dev")
            import :: c_ptr, c_int, c_char, c_double, mps_grid
            character(kind=c_char), intent(in) :: dirname(*)
            integer(c_int), value :: rank
            integer(c_int), intent(in) :: pind(3)
            type(mps_grid), intent(in) :: g
            real(c_double), intent(in) :: off(3)
            integer(c_int), value :: nscalars
            type(c_ptr), intent(in) :: names(*)
            type(c_ptr), intent(in) :: fields(*)
            type(c_ptr), value :: stream
        end function

        integer(c_int) function mps_write_pvtr(dirname, lxyz, pxyz, nscalars, names) bind(C, name="mps_write_pvtr")
            import :: c_ptr, c_int, c_char
            character(kind=c_char), intent(in) :: dirname(*)
            integer(c_int), intent(in) :: lxyz(3), pxyz(3)
            integer(c_int), value :: nscalars
            type(c_ptr), intent(in) :: names(*)
        end function

        ! no handle, no device allocation; stream c_null_ptr is the legacy
        ! default stream here (there is no handle stream)
        integer(c_int) function mps_apply_A_noalloc(g, timederiv, dt, vel, dcoeff, reac, bc_code, &
                soln, ax, opts, stream) bind(C, name="mps_apply_A_noalloc")
            import :: c_ptr, c_int, c_double, mps_grid
            type(mps_grid), intent(in) :: g
            integer(c_int), value :: timederiv
            real(c_double), value :: dt
            type(c_ptr), value :: vel, dcoeff, reac
            integer(c_int), intent(in) :: bc_code(6)
            type(c_ptr), value :: soln, ax
            type(c_ptr), value :: opts          ! c_null_ptr: upwind flux, no transpose
            type(c_ptr), value :: stream
        end function
    end interface

contains

    ! the reference's character(4) codes (globalvars.f90:11-17, discretepde.f90)
    integer(c_int) function bc_int(code)
        character(len=4), intent(in) :: code
        select case (code)
        case ('DIRC'); bc_int = MPS_BC_DIRC
        case ('FLUX'); bc_int = MPS_BC_FLUX
        case ('ZGRD'); bc_int = MPS_BC_ZGRD
        case ('PERI'); bc_int = MPS_BC_PERI
        case default;  bc_int = MPS_BC_DZGD
        end select
    end function

end module mps_linsolve_c
