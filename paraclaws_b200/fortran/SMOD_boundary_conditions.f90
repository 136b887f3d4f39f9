! SMOD_boundary_conditions.f90 -- USER_DIR override of the reference's submodule
! SMOD_boundary_conditions of MOD_domain (user_subroutines/SMOD_boundary_conditions.f90): the
! ghost fill of update_rank_boundaries (interface MOD_domain.f90:191-201) on the GPU.  Not
! compiled here: no Fortran compiler in this image.
!
! main.f90 first calls update_rank_boundaries right after set_initial_conditions (:157-161), so
! that first call also creates the context: it reads control.in and custom.in as
! read_solver_control does, allocates the grid on the GPU, hands over the mesh metrics that
! finalize_mesh computed (any coordinate mapping; :151) and uploads the initial solution.  One
! rank holds the whole grid, so there is no halo exchange.
submodule(MOD_domain) SMOD_boundary_conditions
    implicit none

contains

    module subroutine update_rank_boundaries(decomposition, mesh, solution)
        use iso_c_binding
        use MOD_paraclaws_b200

        type(decomp_info), intent(in) :: decomposition
        type(mesh_fields), intent(in) :: mesh
        type(solution_fields), intent(inout) :: solution

        type(pcl_solver_control) :: ctl

        if (.not. c_associated(pcl_context)) then
            call pcl_check(pcl_read_solver_control('control.in'//c_null_char, 'custom.in'//c_null_char, ctl), &
                           'pcl_read_solver_control')
            call pcl_check(pcl_create(ctl, 0_c_int, pcl_context), 'pcl_create')
            ! the length ratios carry a leading component index: their first component is passed
            ! (the compiler copies the array section into contiguous storage)
            call pcl_check(pcl_set_mesh_metrics(pcl_context, mesh%quadrilateral_mapping%capacity, &
                                                mesh%quadrilateral_mapping%length_ratio_xi(1, :, :), &
                                                mesh%quadrilateral_mapping%length_ratio_eta(1, :, :)), &
                           'pcl_set_mesh_metrics')
            call pcl_check(pcl_upload_state(pcl_context, solution%vars), 'pcl_upload_state')
        end if
        call pcl_check(pcl_update_rank_boundaries(pcl_context), 'pcl_update_rank_boundaries')
    end subroutine

end submodule SMOD_boundary_conditions
