! MOD_paraclaws_b200.f90 -- iso_c_binding interfaces of the paraclaws_b200 C ABI
! (include/paraclaws_b200.h) for the reference's Fortran host.
!
! Not compiled here: this image has no Fortran compiler.  tests/test_fortran_binding.py checks
! on the CPU that every bind(C) interface below names a function of include/paraclaws_b200.h
! with the same number of arguments and matching kinds (int <-> integer(c_int), double <->
! real(c_double), long long <-> integer(c_long_long), pointers by reference or type(c_ptr)
! by value), and that the two bind(C) derived types have the C structs' fields in order.
!
! Put this file, MOD_solve.f90 and SMOD_boundary_conditions.f90 into the reference's USER_DIR:
! mk/generate_source_list.py:53-134 appends a file whose module is new and swaps in the ones
! that redeclare a base module or submodule.  Link with
!   -L<repo>/paraclaws_b200 -lparaclaws_b200 -Wl,-rpath,<repo>/paraclaws_b200
! (reference Makefile:80-84 for gfortran, :116-120 for ifx).

module MOD_paraclaws_b200
    use iso_c_binding
    implicit none

    ! status codes (PCL_OK, PCL_ERR_*)
    integer(c_int), parameter :: PCL_OK = 0, PCL_ERR_NAN = -1, PCL_ERR_NEG_DEPTH = -2, PCL_ERR_TIMEOUT = -3
    integer(c_int), parameter :: PCL_ERR_OOM = -4, PCL_ERR_BADARG = -5, PCL_ERR_CUDA = -6, PCL_ERR_FATAL_DT = -7

    ! struct pcl_solver_control: control.in's records in utility/MOD_IO.f90:61-94 order, then custom.in
    type, bind(C) :: pcl_solver_control
        integer(c_int) :: num_equations, num_dimensions, num_ghost, num_aux, num_waves
        integer(c_int) :: number_of_snapshots
        integer(c_int) :: adaptive_timestepping
        integer(c_int) :: higher_order_flux_correction
        integer(c_int) :: use_limiter
        integer(c_int) :: limiter_method
        integer(c_int) :: m_xi, m_eta
        integer(c_int) :: bc_xi_lower, bc_xi_upper, bc_eta_lower, bc_eta_upper
        integer(c_int) :: precision_mode
        integer(c_int) :: initial_condition
        real(c_double) :: t_start, t_final, dt_initial, cfl_limit, dt_min, dt_max
        real(c_double) :: dt_max_growth_ratio, dt_min_shrink_ratio
        real(c_double) :: xi_min, xi_max, eta_min, eta_max
        real(c_double) :: grav
        real(c_double) :: dam_radius, dam_h_in, dam_h_out, dam_x0, dam_y0
        integer(c_long_long) :: max_accepted_steps
    end type

    ! struct pcl_run_stats
    type, bind(C) :: pcl_run_stats
        integer(c_long_long) :: attempts, accepted, rejected
        integer(c_long_long) :: launches
        real(c_double) :: time, dt, dt_previous, cfl
        integer(c_int) :: snapshot_index, done, status, last_ierr
    end type

    interface
        integer(c_int) function pcl_read_solver_control(control_in, custom_in, ctl) bind(C)
            import :: c_int, c_char, pcl_solver_control
            character(kind=c_char), dimension(*), intent(in) :: control_in
            character(kind=c_char), dimension(*), intent(in) :: custom_in
            type(pcl_solver_control), intent(out) :: ctl
        end function

        integer(c_int) function pcl_create(ctl, device, ctx) bind(C)
            import :: c_int, c_ptr, pcl_solver_control
            type(pcl_solver_control), intent(in) :: ctl
            integer(c_int), value :: device
            type(c_ptr), intent(out) :: ctx
        end function

        integer(c_int) function pcl_destroy(ctx) bind(C)
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
        end function

        integer(c_int) function pcl_upload_state(ctx, vars) bind(C)
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            real(c_double), dimension(*), intent(in) :: vars
        end function

        integer(c_int) function pcl_download_state(ctx, vars) bind(C)
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            real(c_double), dimension(*), intent(out) :: vars
        end function

        integer(c_int) function pcl_set_mesh_metrics(ctx, capacity, length_ratio_xi, length_ratio_eta) bind(C)
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            real(c_double), dimension(*), intent(in) :: capacity
            real(c_double), dimension(*), intent(in) :: length_ratio_xi
            real(c_double), dimension(*), intent(in) :: length_ratio_eta
        end function

        integer(c_int) function pcl_set_equation(ctx, eq_module, params, nparams) bind(C)
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            integer(c_int), value :: eq_module
            real(c_double), dimension(*), intent(in) :: params
            integer(c_int), value :: nparams
        end function

        ! schedule of the FP64 eta sweep (PCL_SHAPE_AUTO 0, _WINDOW 1, _BAND 2); results unchanged
        integer(c_int) function pcl_set_sweep_shape(ctx, eta_shape) bind(C)
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
            integer(c_int), value :: eta_shape
        end function

        integer(c_int) function pcl_get_sweep_shape(ctx, eta_shape) bind(C)
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
            integer(c_int), intent(out) :: eta_shape
        end function

        integer(c_int) function pcl_update_rank_boundaries(ctx) bind(C)
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
        end function

        integer(c_int) function pcl_solve_dimensional_split(ctx, ierr) bind(C)
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
            integer(c_int), intent(out) :: ierr
        end function

        integer(c_int) function pcl_restore_solution(ctx) bind(C)
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
        end function

        integer(c_int) function pcl_integrate_source_term(ctx) bind(C)
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
        end function

        integer(c_int) function pcl_update_time(ctx, step_valid) bind(C)
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
            integer(c_int), value :: step_valid
        end function

        integer(c_int) function pcl_reset_cfl(ctx) bind(C)
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
        end function

        integer(c_int) function pcl_advance_snapshot_index(ctx) bind(C)
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
        end function

        integer(c_int) function pcl_set_dt(ctx, dt) bind(C)
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            real(c_double), value :: dt
        end function

        integer(c_int) function pcl_get_time(ctx, time) bind(C)
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            real(c_double), intent(out) :: time
        end function

        integer(c_int) function pcl_get_dt(ctx, dt) bind(C)
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            real(c_double), intent(out) :: dt
        end function

        integer(c_int) function pcl_get_previous_dt(ctx, dt) bind(C)
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            real(c_double), intent(out) :: dt
        end function

        integer(c_int) function pcl_get_cfl(ctx, cfl) bind(C)
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            real(c_double), intent(out) :: cfl
        end function

        integer(c_int) function pcl_get_snapshot_index(ctx, idx) bind(C)
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
            integer(c_int), intent(out) :: idx
        end function

        integer(c_int) function pcl_get_snapshot_time(ctx, idx, t) bind(C)
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            integer(c_int), value :: idx
            real(c_double), intent(out) :: t
        end function

        integer(c_int) function pcl_advance(ctx, max_attempts, stats) bind(C)
            import :: c_int, c_ptr, c_long_long, pcl_run_stats
            type(c_ptr), value :: ctx
            integer(c_long_long), value :: max_attempts
            type(pcl_run_stats), intent(out) :: stats
        end function

        integer(c_int) function pcl_advance_to_snapshot(ctx, stats) bind(C)
            import :: c_int, c_ptr, pcl_run_stats
            type(c_ptr), value :: ctx
            type(pcl_run_stats), intent(out) :: stats
        end function

        integer(c_int) function pcl_get_stats(ctx, stats) bind(C)
            import :: c_int, c_ptr, pcl_run_stats
            type(c_ptr), value :: ctx
            type(pcl_run_stats), intent(out) :: stats
        end function

        integer(c_int) function pcl_reset_time_control(ctx) bind(C)
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
        end function

        integer(c_int) function pcl_write_snapshot(ctx, output_dir, wait) bind(C)
            import :: c_int, c_ptr, c_char
            type(c_ptr), value :: ctx
            character(kind=c_char), dimension(*), intent(in) :: output_dir
            integer(c_int), value :: wait
        end function

        integer(c_int) function pcl_snapshot_wait(ctx) bind(C)
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
        end function

        integer(c_int) function pcl_synchronize(ctx) bind(C)
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
        end function

        integer(c_long_long) function pcl_state_doubles(ctx) bind(C)
            import :: c_long_long, c_ptr
            type(c_ptr), value :: ctx
        end function

        type(c_ptr) function pcl_status_string(status) bind(C)
            import :: c_int, c_ptr
            integer(c_int), value :: status
        end function
    end interface

    ! the context of this process's grid (one rank, one GPU)
    type(c_ptr), save :: pcl_context = c_null_ptr

contains

    ! Stop the run the way the reference's abort_program does when a call fails.
    subroutine pcl_check(rc, where)
        integer(c_int), intent(in) :: rc
        character(len=*), intent(in) :: where
        if (rc < 0) then
            write(*, '(a, a, i0)') where, ': paraclaws_b200 status ', rc
            error stop "paraclaws_b200 call failed"
        end if
    end subroutine

end module MOD_paraclaws_b200
