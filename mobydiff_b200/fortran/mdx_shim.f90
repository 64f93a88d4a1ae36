! mdx_shim.f90 -- drop-in replacements for mobydiff's OpenMP-offload modules
! gpu_runtime, step, boundary and pressure_solver, with the same module and
! procedure names and argument lists (src/modules/gpu_runtime.f90,
! step.f90, boundary.f90, pressure_solver.f90).  Each body hands the call to
! libmobyb200.so through mdx_bindings.  init.f90, config.f90, ibm.f90 (host
! geometry) and field_hdf5.c stay unchanged; io.f90's `!$omp target update`
! lines become calls to mdx_update_host / mdx_update_device.  Not compiled in
! this repository (no Fortran compiler); tests/test_gpu_shim_replay.py replays
! the call sequence of every body below through the same C entry points.

module mdx_state
    use, intrinsic :: iso_c_binding
    implicit none
    type(C_PTR), save :: ctx = C_NULL_PTR
    ! host addresses of the IBM coefficient arrays last uploaded, and whether
    ! they must be sent again (no upload yet, or marked changed)
    type(C_PTR), save :: ibm_sent(3) = C_NULL_PTR
    logical, save :: ibm_stale = .true.
end module mdx_state

! The reference computes the IBM coefficients on the host (set_ibm_coeff,
! main.f90:57-60) and maps them with enter_ibm_data (ibm.f90:57-68), which
! stays unchanged and holds only OpenMP directives.  The shim therefore sends
! ibm%coef_u/v/w to the device itself: before the first predictor or
! projection, again when the arrays are reallocated (new addresses), and
! again after ibm_coefficients_changed() -- the call for a program that
! rewrites the coefficients in place (main.f90 never does).
module mdx_ibm_sync
    use, intrinsic :: iso_c_binding
    use :: ibmm, only: ibm_type
    use :: mdx_bindings
    use :: mdx_state
    implicit none
    private
    public :: sync_ibm, ibm_coefficients_changed
contains
    subroutine sync_ibm(ibm)
        type(ibm_type), intent(in), target :: ibm
        type(C_PTR) :: p(3)
        if (.not. (allocated(ibm%coef_u) .and. allocated(ibm%coef_v) .and. allocated(ibm%coef_w))) then
            print *, "ERROR: IBM coefficients not allocated (init_ibm and set_ibm_coeff come first)."
            error stop 1
        end if
        p(1) = c_loc(ibm%coef_u)
        p(2) = c_loc(ibm%coef_v)
        p(3) = c_loc(ibm%coef_w)
        if (.not. ibm_stale) then
            if (c_associated(p(1), ibm_sent(1)) .and. c_associated(p(2), ibm_sent(2)) .and. &
                c_associated(p(3), ibm_sent(3))) return
        end if
        call mdx_check(mdx_enter_ibm_data(ctx, p(1), p(2), p(3)), ctx, "enter_ibm_data")
        ibm_sent = p
        ibm_stale = .false.
    end subroutine sync_ibm

    subroutine ibm_coefficients_changed()
        ibm_stale = .true.
    end subroutine ibm_coefficients_changed
end module mdx_ibm_sync

module gpu_runtime
    use, intrinsic :: iso_c_binding
    use :: init, only: grid_type, field_type
    use :: mdx_bindings
    use :: mdx_state
    implicit none
contains
    subroutine init_openmp_offload()
        integer(C_INT) :: n, rc
        n = 0
        rc = mdx_device_count(n)
        if (rc /= MDX_OK .or. n <= 0) then
            print *, "ERROR: no CUDA device available for mobydiff_b200 (mdx_device_count status", rc, ")."
            error stop 1
        end if
        print *, "CUDA devices available:", n
    end subroutine init_openmp_offload

    subroutine enter_field_data(f, g)
        type(field_type), intent(inout), target :: f
        type(grid_type),  intent(in)    :: g
        type(mdx_grid_t) :: cg
        type(mdx_bc_t) :: cb
        cg%nx = g%nx; cg%ny = g%ny; cg%nz = g%nz; cg%nsteps = g%nsteps
        cg%lx = g%lx; cg%ly = g%ly; cg%lz = g%lz; cg%dx = g%dx; cg%dy = g%dy; cg%dz = g%dz
        cg%re = g%re; cg%dt = g%dt; cg%t_final = g%t_final; cg%t_current = g%t_current
        cg%cfl = g%cfl; cg%cflmax = g%cflmax; cg%dtmax = g%dtmax
        cg%forcing_x = g%forcing_x; cg%forcing_y = g%forcing_y; cg%forcing_z = g%forcing_z
        cb%is_periodic = 1; cb%bc_type = 0; cb%bc_value = 0.0d0       ! init_bc defaults
        call mdx_check(mdx_create(0_C_INT, cg, cb, ctx), ctx, "mdx_create")
        call mdx_check(mdx_enter_field_data(ctx, c_loc(f%un), c_loc(f%us), c_loc(f%oldrhsu), &
            c_loc(f%vn), c_loc(f%vs), c_loc(f%oldrhsv), c_loc(f%wn), c_loc(f%ws), c_loc(f%oldrhsw), &
            c_loc(f%pn)), ctx, "enter_field_data")
    end subroutine enter_field_data

    subroutine exit_field_data(f, g)
        type(field_type), intent(inout) :: f
        type(grid_type),  intent(in)    :: g
        call mdx_check(mdx_exit_field_data(ctx), ctx, "exit_field_data")
        call mdx_check(mdx_destroy(ctx), ctx, "mdx_destroy")
        ctx = C_NULL_PTR
        ibm_sent = C_NULL_PTR
        ibm_stale = .true.
    end subroutine exit_field_data
end module gpu_runtime

module boundary
    use, intrinsic :: iso_c_binding
    use :: init, only: grid_type, field_type
    use :: mdx_bindings
    use :: mdx_state
    implicit none

    type :: boundary_type                      ! unchanged, boundary.f90:6-10
        logical(C_BOOL) :: isPeriodic(1:3)
        integer(C_INT) :: bcType(1:3,0:1,0:3)
        real(C_DOUBLE) :: bcValue(1:3,0:1,0:3)
    end type boundary_type

    type(mdx_bc_t), save, private :: last_bc
    logical, save, private :: have_bc = .false.
contains
    subroutine init_bc(bc)                     ! unchanged, boundary.f90:14-20
        type(boundary_type), intent(inout) :: bc
        bc%isPeriodic(1:3) = .True.
        bc%bcType(:,:,:) = 0
        bc%bcValue(:,:,:) = 0
    end subroutine init_bc

    ! hand bc to the context when it differs from the last one sent
    subroutine sync_bc(bc)
        type(boundary_type), intent(in) :: bc
        type(mdx_bc_t) :: cb
        integer :: t
        do t = 1, 3
            cb%is_periodic(t) = merge(1_C_INT, 0_C_INT, logical(bc%isPeriodic(t)))
        end do
        cb%bc_type = reshape(bc%bcType, [24])
        cb%bc_value = reshape(bc%bcValue, [24])
        if (have_bc) then
            if (all(cb%is_periodic == last_bc%is_periodic) .and. all(cb%bc_type == last_bc%bc_type) .and. &
                all(cb%bc_value == last_bc%bc_value)) return
        end if
        call mdx_check(mdx_set_bc(ctx, cb), ctx, "mdx_set_bc")
        last_bc = cb
        have_bc = .true.
    end subroutine sync_bc

    subroutine apply_bc(f, g)
        type(field_type), intent(inout) :: f
        type(grid_type),  intent(in)    :: g
        call mdx_check(mdx_apply_bc(ctx), ctx, "apply_bc")
    end subroutine apply_bc

    subroutine apply_bc_redblack(f, g, bc)
        type(field_type), intent(inout)  :: f
        type(grid_type),  intent(in)     :: g
        type(boundary_type),  intent(in) :: bc
        call sync_bc(bc)
        call mdx_check(mdx_apply_bc_redblack(ctx), ctx, "apply_bc_redblack")
    end subroutine apply_bc_redblack
end module boundary

module step
    use, intrinsic :: iso_c_binding
    use :: init, only: grid_type, field_type
    use :: ibmm, only: ibm_type
    use :: boundary, only: boundary_type, sync_bc
    use :: mdx_ibm_sync, only: sync_ibm
    use :: mdx_bindings
    use :: mdx_state
    implicit none
    real(C_DOUBLE), parameter :: rk_alpha(3) = [64.0d0/120.0d0,  50.0d0/120.0d0,  90.0d0/120.0d0]
    real(C_DOUBLE), parameter :: rk_beta(3)  = [ 0.0d0,         -34.0d0/120.0d0, -50.0d0/120.0d0]
    real(C_DOUBLE), parameter :: rk_gamma(3) = [64.0d0/120.0d0,  16.0d0/120.0d0,  40.0d0/120.0d0]
contains
    subroutine momentum(f, g, dt_alpha, dt_beta, dt_gamma, ibm, bc)
        type(field_type), intent(inout) :: f
        type(grid_type),  intent(in)    :: g
        real(C_DOUBLE),   intent(in)    :: dt_alpha, dt_beta, dt_gamma
        type(ibm_type),   intent(in), target :: ibm
        type(boundary_type), intent(in) :: bc
        call sync_bc(bc)
        call sync_ibm(ibm)
        call mdx_check(mdx_momentum(ctx, dt_alpha, dt_beta, dt_gamma), ctx, "momentum")
    end subroutine momentum

    real(C_DOUBLE) function get_cfl(f, g)
        type(field_type), intent(inout) :: f
        type(grid_type),  intent(in)    :: g
        call mdx_check(mdx_get_cfl(ctx, get_cfl), ctx, "get_cfl")
    end function get_cfl
end module step

module pressure_solver
    use, intrinsic :: iso_c_binding
    use :: init, only: grid_type, field_type
    use :: pressure_workspace, only: pressure_solver_type
    use :: ibmm, only: ibm_type
    use :: boundary, only: boundary_type, sync_bc
    use :: mdx_ibm_sync, only: sync_ibm
    use :: mdx_bindings
    use :: mdx_state
    implicit none
    private
    public :: pressure_solver_type, init_pressure_solver, pressure_projection, destroy_pressure_solver
contains
    subroutine init_pressure_solver(ps, g)
        type(pressure_solver_type), intent(inout) :: ps
        type(grid_type), intent(in) :: g
        type(mdx_solver_opts_t) :: o
        call mdx_default_solver_opts(o)
#ifdef USE_REDBLACK
        o%solver = MDX_SOLVER_REDBLACK
        o%n_iter = ps%nIter
        o%sor = ps%sor
#else
        o%solver = MDX_SOLVER_FFT
#endif
        call mdx_check(mdx_init_pressure_solver(ctx, o), ctx, "init_pressure_solver")
    end subroutine init_pressure_solver

    subroutine pressure_projection(ps, f, g, dt_gamma, ibm, bc)
        type(pressure_solver_type), intent(inout) :: ps
        type(field_type), intent(inout) :: f
        type(grid_type), intent(in) :: g
        real(C_DOUBLE), intent(in) :: dt_gamma
        type(ibm_type), intent(in), target :: ibm
        type(boundary_type), intent(in) :: bc
        call sync_bc(bc)
        call sync_ibm(ibm)
        call mdx_check(mdx_pressure_projection(ctx, dt_gamma, C_NULL_PTR), ctx, "pressure_projection")
    end subroutine pressure_projection

    subroutine destroy_pressure_solver(ps)
        type(pressure_solver_type), intent(inout) :: ps
        call mdx_check(mdx_destroy_pressure_solver(ctx), ctx, "destroy_pressure_solver")
    end subroutine destroy_pressure_solver
end module pressure_solver
