! MOD_solve.f90 -- USER_DIR override of the reference's module MOD_solve (solver/MOD_solve.f90):
! the same public procedures with the same dummy arguments, running the step on the GPU through
! the paraclaws_b200 C ABI (MOD_paraclaws_b200.f90).  Not compiled here: no Fortran compiler in
! this image (tests/test_fortran_binding.py checks the calls against include/paraclaws_b200.h).
!
! The reference's time loop (main.f90:193-283) and its time control stay on the host and keep
! deciding: each attempt runs with the host's dt, the device's CFL starts from zero as the host's
! does after reset_CFL, and the attempt's CFL goes back into t_ctrl through update_max_CFL.  The
! device keeps the solution; a rejected attempt leaves it as it was (main.f90:221 then restores
! the host copy, which nothing reads), and execute_post, which main.f90 calls right before every
! writeData (:166, :257), first copies the device solution into solution%vars.
module MOD_solve
    implicit none

    public :: solve_dimensional_split, integrate_source_term, execute_post

contains

    ! solve_dimensional_split (solver/MOD_solve.f90:23-175): one attempted step, ierr = 1 accepted,
    ! -1 rejected
    subroutine solve_dimensional_split(decomposition, t_ctrl, work, mesh, solution, ierr)
        use iso_c_binding
        use MOD_paraclaws_b200
        use MOD_time_control, only: time_control
        use mpidcl, only: decomp_info
        use MOD_domain, only: solution_fields, mesh_fields
        use MOD_work_arrays, only: work_arrays

        type(decomp_info), intent(in) :: decomposition
        type(time_control), intent(inout) :: t_ctrl
        type(work_arrays), intent(inout) :: work        ! unused: the device keeps no work arrays
        type(mesh_fields) :: mesh
        type(solution_fields) :: solution
        integer, intent(inout) :: ierr

        integer(c_int) :: attempt
        real(c_double) :: cfl

        call pcl_check(pcl_set_dt(pcl_context, t_ctrl%get_dt()), 'pcl_set_dt')
        call pcl_check(pcl_reset_cfl(pcl_context), 'pcl_reset_cfl')
        call pcl_check(pcl_solve_dimensional_split(pcl_context, attempt), 'pcl_solve_dimensional_split')
        call pcl_check(pcl_get_cfl(pcl_context, cfl), 'pcl_get_cfl')
        call t_ctrl%update_max_CFL(cfl)
        ierr = attempt
    end subroutine

    ! integrate_source_term (solver/MOD_solve.f90:295-336): phi = 0 for the dam break, a no-op;
    ! a non-zero source runs as a device hook installed with pcl_set_source_hook
    subroutine integrate_source_term(decomposition, t_ctrl, mesh, solution)
        use iso_c_binding
        use MOD_paraclaws_b200
        use MOD_time_control, only: time_control
        use mpidcl, only: decomp_info
        use MOD_domain, only: mesh_fields, solution_fields

        type(decomp_info), intent(in) :: decomposition
        type(time_control), intent(in) :: t_ctrl
        type(mesh_fields), intent(in) :: mesh
        type(solution_fields), intent(inout) :: solution

        call pcl_check(pcl_integrate_source_term(pcl_context), 'pcl_integrate_source_term')
    end subroutine

    ! execute_post (solver/MOD_solve.f90:338-365): bring the device solution to the host, then the
    ! user's post-processing on every cell of the block, as the reference does
    subroutine execute_post(decomposition, mesh, solution)
        use iso_c_binding
        use MOD_paraclaws_b200
        use mpidcl, only: decomp_info
        use MOD_user_subroutines, only: user_post
        use MOD_domain

        type(decomp_info), intent(in) :: decomposition
        type(mesh_fields), intent(in) :: mesh
        type(solution_fields), intent(inout) :: solution

        integer :: ilo, ihi, jlo, jhi, i, j

        call pcl_check(pcl_download_state(pcl_context, solution%vars), 'pcl_download_state')
        call decomposition%get_local_block_bounds(ilo, ihi, jlo, jhi)
        do j = jlo, jhi
            do i = ilo, ihi
                call user_post(i, j, mesh, solution, decomposition)
            end do
        end do
    end subroutine

end module MOD_solve
