! mdx_bindings.f90 -- iso_c_binding interfaces to libmobyb200.so
! (include/mobydiff_b200.h).  Part of the Fortran drop-in for mobydiff's
! OpenMP-offload modules; see mdx_shim.f90 for the module bodies.
! Not compiled in this repository (no Fortran compiler in its build image).
module mdx_bindings
    use, intrinsic :: iso_c_binding
    implicit none

    integer(C_INT), parameter :: MDX_OK = 0
    integer(C_INT), parameter :: MDX_SOLVER_FFT = 0, MDX_SOLVER_REDBLACK = 1

    ! grid_type with C layout (src/modules/init.f90:5-12 component order)
    type, bind(C) :: mdx_grid_t
        integer(C_INT) :: nx, ny, nz, nsteps
        real(C_DOUBLE) :: lx, ly, lz, dx, dy, dz
        real(C_DOUBLE) :: re, dt, t_final, t_current, cfl, cflmax, dtmax
        real(C_DOUBLE) :: forcing_x, forcing_y, forcing_z
    end type mdx_grid_t

    ! boundary_type with C layout; bc_type/bc_value keep bcType(1:3,0:1,0:3) order
    type, bind(C) :: mdx_bc_t
        integer(C_INT) :: is_periodic(3)
        integer(C_INT) :: bc_type(24)
        real(C_DOUBLE) :: bc_value(24)
    end type mdx_bc_t

    type, bind(C) :: mdx_solver_opts_t
        integer(C_INT) :: solver, n_iter
        real(C_DOUBLE) :: sor, tol
        integer(C_INT) :: max_iter, check_every, precision
        integer(C_INT) :: sor_variant, sor_kz
        integer(C_INT) :: check_mode
        integer(C_INT) :: fft_kernel
        integer(C_INT) :: inner_form
        integer(C_INT) :: reserved_i(2)
        real(C_DOUBLE) :: atol
        real(C_DOUBLE) :: inner_sor
        real(C_DOUBLE) :: reserved_d(6)
    end type mdx_solver_opts_t

    type, bind(C) :: mdx_solve_stats_t
        integer(C_INT) :: iterations, status
        real(C_DOUBLE) :: residual, residual0, atol
        integer(C_INT) :: variant, guessed
    end type mdx_solve_stats_t

    ! ibm_type geometry parameters (mdx_ibm_geom_t)
    type, bind(C) :: mdx_ibm_geom_t
        integer(C_INT) :: geometry, n_wave_x
        real(C_DOUBLE) :: amp, phase, lambda, y0, height
    end type mdx_ibm_geom_t

    interface
        function mdx_device_count(count) bind(C, name="mdx_device_count") result(rc)
            import :: C_INT
            integer(C_INT), intent(out) :: count
            integer(C_INT) :: rc
        end function
        function mdx_last_error(ctx) bind(C, name="mdx_last_error") result(msg)
            import :: C_PTR
            type(C_PTR), value :: ctx
            type(C_PTR) :: msg
        end function
        subroutine mdx_default_solver_opts(o) bind(C, name="mdx_default_solver_opts")
            import :: mdx_solver_opts_t
            type(mdx_solver_opts_t), intent(out) :: o
        end subroutine
        function mdx_create(device, g, bc, ctx) bind(C, name="mdx_create") result(rc)
            import :: C_INT, C_PTR, mdx_grid_t, mdx_bc_t
            integer(C_INT), value :: device
            type(mdx_grid_t), intent(in) :: g
            type(mdx_bc_t), intent(in) :: bc
            type(C_PTR), intent(out) :: ctx
            integer(C_INT) :: rc
        end function
        function mdx_set_bc(ctx, bc) bind(C, name="mdx_set_bc") result(rc)
            import :: C_INT, C_PTR, mdx_bc_t
            type(C_PTR), value :: ctx
            type(mdx_bc_t), intent(in) :: bc
            integer(C_INT) :: rc
        end function
        function mdx_destroy(ctx) bind(C, name="mdx_destroy") result(rc)
            import :: C_INT, C_PTR
            type(C_PTR), value :: ctx
            integer(C_INT) :: rc
        end function
        function mdx_enter_field_data(ctx, un, us, oldrhsu, vn, vs, oldrhsv, wn, ws, oldrhsw, pn) &
                bind(C, name="mdx_enter_field_data") result(rc)
            import :: C_INT, C_PTR
            type(C_PTR), value :: ctx, un, us, oldrhsu, vn, vs, oldrhsv, wn, ws, oldrhsw, pn
            integer(C_INT) :: rc
        end function
        function mdx_exit_field_data(ctx) bind(C, name="mdx_exit_field_data") result(rc)
            import :: C_INT, C_PTR
            type(C_PTR), value :: ctx
            integer(C_INT) :: rc
        end function
        function mdx_update_host(ctx, un, vn, wn, pn) bind(C, name="mdx_update_host") result(rc)
            import :: C_INT, C_PTR
            type(C_PTR), value :: ctx, un, vn, wn, pn
            integer(C_INT) :: rc
        end function
        function mdx_update_device(ctx, un, vn, wn, pn) bind(C, name="mdx_update_device") result(rc)
            import :: C_INT, C_PTR
            type(C_PTR), value :: ctx, un, vn, wn, pn
            integer(C_INT) :: rc
        end function
        function mdx_enter_ibm_data(ctx, cu, cv, cw) bind(C, name="mdx_enter_ibm_data") result(rc)
            import :: C_INT, C_PTR
            type(C_PTR), value :: ctx, cu, cv, cw
            integer(C_INT) :: rc
        end function
        function mdx_enter_ibm_geometry(ctx, geom) bind(C, name="mdx_enter_ibm_geometry") result(rc)
            import :: C_INT, C_PTR, mdx_ibm_geom_t
            type(C_PTR), value :: ctx
            type(mdx_ibm_geom_t), intent(in) :: geom
            integer(C_INT) :: rc
        end function
        function mdx_exit_ibm_data(ctx) bind(C, name="mdx_exit_ibm_data") result(rc)
            import :: C_INT, C_PTR
            type(C_PTR), value :: ctx
            integer(C_INT) :: rc
        end function
        function mdx_momentum(ctx, dt_alpha, dt_beta, dt_gamma) bind(C, name="mdx_momentum") result(rc)
            import :: C_INT, C_PTR, C_DOUBLE
            type(C_PTR), value :: ctx
            real(C_DOUBLE), value :: dt_alpha, dt_beta, dt_gamma
            integer(C_INT) :: rc
        end function
        function mdx_apply_bc(ctx) bind(C, name="mdx_apply_bc") result(rc)
            import :: C_INT, C_PTR
            type(C_PTR), value :: ctx
            integer(C_INT) :: rc
        end function
        function mdx_apply_bc_redblack(ctx) bind(C, name="mdx_apply_bc_redblack") result(rc)
            import :: C_INT, C_PTR
            type(C_PTR), value :: ctx
            integer(C_INT) :: rc
        end function
        function mdx_init_pressure_solver(ctx, o) bind(C, name="mdx_init_pressure_solver") result(rc)
            import :: C_INT, C_PTR, mdx_solver_opts_t
            type(C_PTR), value :: ctx
            type(mdx_solver_opts_t), intent(in) :: o
            integer(C_INT) :: rc
        end function
        function mdx_destroy_pressure_solver(ctx) bind(C, name="mdx_destroy_pressure_solver") result(rc)
            import :: C_INT, C_PTR
            type(C_PTR), value :: ctx
            integer(C_INT) :: rc
        end function
        function mdx_pressure_projection(ctx, dt_gamma, stats) bind(C, name="mdx_pressure_projection") result(rc)
            import :: C_INT, C_PTR, C_DOUBLE
            type(C_PTR), value :: ctx
            real(C_DOUBLE), value :: dt_gamma
            type(C_PTR), value :: stats
            integer(C_INT) :: rc
        end function
        function mdx_get_cfl(ctx, cfl) bind(C, name="mdx_get_cfl") result(rc)
            import :: C_INT, C_PTR, C_DOUBLE
            type(C_PTR), value :: ctx
            real(C_DOUBLE), intent(out) :: cfl
            integer(C_INT) :: rc
        end function
        function mdx_center_vel(ctx, uc, vc, wc) bind(C, name="mdx_center_vel") result(rc)
            import :: C_INT, C_PTR
            type(C_PTR), value :: ctx, uc, vc, wc
            integer(C_INT) :: rc
        end function
        ! warm starts and the learned warm start (no counterpart in the reference)
        function mdx_set_pressure_guess(ctx, mode, record) bind(C, name="mdx_set_pressure_guess") result(rc)
            import :: C_INT, C_PTR
            type(C_PTR), value :: ctx
            integer(C_INT), value :: mode, record
            integer(C_INT) :: rc
        end function
        function mdx_unet_create(ctx, opts) bind(C, name="mdx_unet_create") result(rc)
            import :: C_INT, C_PTR
            type(C_PTR), value :: ctx, opts     ! NULL: default options
            integer(C_INT) :: rc
        end function
        function mdx_unet_record(ctx, on) bind(C, name="mdx_unet_record") result(rc)
            import :: C_INT, C_PTR
            type(C_PTR), value :: ctx
            integer(C_INT), value :: on
            integer(C_INT) :: rc
        end function
        function mdx_unet_train(ctx, iters, lr, loss_first, loss_last) bind(C, name="mdx_unet_train") result(rc)
            import :: C_INT, C_PTR, C_DOUBLE
            type(C_PTR), value :: ctx
            integer(C_INT), value :: iters
            real(C_DOUBLE), value :: lr
            real(C_DOUBLE), intent(out) :: loss_first, loss_last
            integer(C_INT) :: rc
        end function
        function mdx_unet_param_count(ctx) bind(C, name="mdx_unet_param_count") result(n)
            import :: C_PTR, C_LONG_LONG
            type(C_PTR), value :: ctx
            integer(C_LONG_LONG) :: n
        end function
        function mdx_unet_get_params(ctx, host, n) bind(C, name="mdx_unet_get_params") result(rc)
            import :: C_INT, C_PTR, C_LONG_LONG
            type(C_PTR), value :: ctx, host
            integer(C_LONG_LONG), value :: n
            integer(C_INT) :: rc
        end function
        function mdx_unet_set_params(ctx, host, n) bind(C, name="mdx_unet_set_params") result(rc)
            import :: C_INT, C_PTR, C_LONG_LONG
            type(C_PTR), value :: ctx, host
            integer(C_LONG_LONG), value :: n
            integer(C_INT) :: rc
        end function
        function mdx_unet_get_out_scale(ctx, scale) bind(C, name="mdx_unet_get_out_scale") result(rc)
            import :: C_INT, C_PTR, C_DOUBLE
            type(C_PTR), value :: ctx
            real(C_DOUBLE), intent(out) :: scale
            integer(C_INT) :: rc
        end function
        function mdx_unet_set_out_scale(ctx, scale) bind(C, name="mdx_unet_set_out_scale") result(rc)
            import :: C_INT, C_PTR, C_DOUBLE
            type(C_PTR), value :: ctx
            real(C_DOUBLE), value :: scale
            integer(C_INT) :: rc
        end function
    end interface

contains

    ! error stop with the library message, as check_cufft does
    ! (src/modules/pressure/cufft_bindings.f90:56-74)
    subroutine mdx_check(rc, ctx, what)
        integer(C_INT), intent(in) :: rc
        type(C_PTR), intent(in) :: ctx
        character(len=*), intent(in) :: what
        character(kind=C_CHAR), pointer :: msg(:)
        integer :: n
        if (rc == MDX_OK) return
        call c_f_pointer(mdx_last_error(ctx), msg, [1024])
        n = 0
        do while (n < 1024)
            if (msg(n + 1) == C_NULL_CHAR) exit
            n = n + 1
        end do
        print *, "mobydiff_b200: ", what, " failed: ", msg(1:n)
        error stop 1
    end subroutine mdx_check

end module mdx_bindings
