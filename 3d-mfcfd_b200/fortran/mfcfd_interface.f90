! mfcfd_interface.f90 - ISO_C_BINDING interface to the B200 q-LSKUM library
! (include/mfcfd.h).  A Fortran host that owns the reference's module
! globals (type(points) :: point, data_structure.f90:7-59) hands them to
! mfcfd_create once and then replaces every `call fpi_solver(t)`
! (q_lskum.f90:29) by mfcfd_fpi_step.  Arrays are passed in their Fortran
! layout; conn stays 1-based.
module mfcfd_interface
    use iso_c_binding
    implicit none

    integer(c_int32_t), parameter :: MFCFD_OK = 0
    integer(c_int32_t), parameter :: MFCFD_FIELD_PRIM = 0, MFCFD_FIELD_U = 1, MFCFD_FIELD_Q = 2, &
        MFCFD_FIELD_QM = 3, MFCFD_FIELD_DQ = 4, MFCFD_FIELD_DELT = 5, MFCFD_FIELD_FLUX_RES = 6, &
        MFCFD_FIELD_DELUP = 7, MFCFD_FIELD_DELUN = 8, MFCFD_FIELD_DINV = 9
    integer(c_int32_t), parameter :: MFCFD_SWEEP_DATAFLOW = 0, MFCFD_SWEEP_LEVELS = 1, &
        MFCFD_SWEEP_CHAINS = 2
    integer(c_int32_t), parameter :: MFCFD_PRECISION_FP64 = 0, MFCFD_PRECISION_MIXED = 1, &
        MFCFD_PRECISION_MIXED_DC = 2
    integer(c_int32_t), parameter :: MFCFD_UPDATE_IMPLICIT = 0, MFCFD_UPDATE_EXPLICIT = 1
    integer(c_int32_t), parameter :: MFCFD_SWEEPS_ALIAS = 0, MFCFD_SWEEPS_BACKUP = 1
    integer(c_int32_t), parameter :: MFCFD_ORDER_INDEX = 0, MFCFD_ORDER_MORTON = 1

    ! mirror of struct mfcfd_params
    type, bind(C) :: mfcfd_params
        real(c_double) :: power, vl_const, cfl
        real(c_double) :: rho_inf, u1_inf, u2_inf, u3_inf, pr_inf
        integer(c_int32_t) :: inner_iterations, split_capacity, precision, device, sweep_mode
        integer(c_int32_t) :: update_variant, sweep_variant, chain_warps, gpu_setup, graphs
        integer(c_int32_t) :: chain_spread, storage_order, flux_blocks_per_sm
    end type mfcfd_params

    interface
        subroutine mfcfd_params_init(p, mach, aoa_deg) bind(C, name="mfcfd_params_init")
            import :: mfcfd_params, c_double
            type(mfcfd_params), intent(out) :: p
            real(c_double), value :: mach, aoa_deg
        end subroutine mfcfd_params_init

        function mfcfd_create(params, n, status, x, y, z, tan1, tan2, nor, nbhs, conn, &
                              min_dist, h) result(rc) bind(C, name="mfcfd_create")
            import :: mfcfd_params, c_int, c_int32_t, c_double, c_ptr
            type(mfcfd_params), intent(in) :: params
            integer(c_int32_t), value :: n
            integer(c_int32_t), intent(in) :: status(*), nbhs(*), conn(*)
            real(c_double), intent(in) :: x(*), y(*), z(*), tan1(*), tan2(*), nor(*), min_dist(*)
            type(c_ptr), intent(out) :: h
            integer(c_int) :: rc
        end function mfcfd_create

        function mfcfd_set_prim(h, prim) result(rc) bind(C, name="mfcfd_set_prim")
            import :: c_ptr, c_double, c_int
            type(c_ptr), value :: h
            real(c_double), intent(in) :: prim(*)
            integer(c_int) :: rc
        end function mfcfd_set_prim

        function mfcfd_fpi_step(h, t, res_new, residue) result(rc) bind(C, name="mfcfd_fpi_step")
            import :: c_ptr, c_int32_t, c_double, c_int
            type(c_ptr), value :: h
            integer(c_int32_t), value :: t
            real(c_double), intent(out) :: res_new, residue
            integer(c_int) :: rc
        end function mfcfd_fpi_step

        function mfcfd_run(h, t0, iters, res_hist) result(rc) bind(C, name="mfcfd_run")
            import :: c_ptr, c_int32_t, c_double, c_int
            type(c_ptr), value :: h
            integer(c_int32_t), value :: t0, iters
            real(c_double), intent(out) :: res_hist(*)
            integer(c_int) :: rc
        end function mfcfd_run

        function mfcfd_get(h, field, out) result(rc) bind(C, name="mfcfd_get")
            import :: c_ptr, c_int32_t, c_double, c_int
            type(c_ptr), value :: h
            integer(c_int32_t), value :: field
            real(c_double), intent(out) :: out(*)
            integer(c_int) :: rc
        end function mfcfd_get

        function mfcfd_get_state(h, prim, delu, res_old) result(rc) bind(C, name="mfcfd_get_state")
            import :: c_ptr, c_double, c_int
            type(c_ptr), value :: h
            real(c_double), intent(out) :: prim(*), delu(*)
            real(c_double), intent(out) :: res_old
            integer(c_int) :: rc
        end function mfcfd_get_state

        function mfcfd_set_state(h, prim, delu, res_old) result(rc) bind(C, name="mfcfd_set_state")
            import :: c_ptr, c_double, c_int
            type(c_ptr), value :: h
            real(c_double), intent(in) :: prim(*), delu(*)
            real(c_double), value :: res_old
            integer(c_int) :: rc
        end function mfcfd_set_state

        function mfcfd_get_alias(h, alias, point_with_alias) result(rc) bind(C, name="mfcfd_get_alias")
            import :: c_ptr, c_int32_t, c_int
            type(c_ptr), value :: h
            integer(c_int32_t), intent(out) :: alias(*), point_with_alias(*)
            integer(c_int) :: rc
        end function mfcfd_get_alias

        function mfcfd_residual_noalloc(h, res_new) result(rc) bind(C, name="mfcfd_residual_noalloc")
            import :: c_ptr, c_double, c_int
            type(c_ptr), value :: h
            real(c_double), intent(out) :: res_new
            integer(c_int) :: rc
        end function mfcfd_residual_noalloc

        function mfcfd_set_precision(h, precision) result(rc) bind(C, name="mfcfd_set_precision")
            import :: c_ptr, c_int32_t, c_int
            type(c_ptr), value :: h
            integer(c_int32_t), value :: precision
            integer(c_int) :: rc
        end function mfcfd_set_precision

        ! the connectivity of a cloud given only its points: conn(27,N) of
        ! the k nearest neighbours, on GPU `device` (>= 0) or the host
        function mfcfd_knn(device, n, x, y, z, k, nbhs, conn, min_dist) result(rc) bind(C, name="mfcfd_knn")
            import :: c_int32_t, c_double, c_int
            integer(c_int32_t), value :: device, n, k
            real(c_double), intent(in) :: x(*), y(*), z(*)
            integer(c_int32_t), intent(out) :: nbhs(*), conn(27, *)
            real(c_double), intent(out) :: min_dist(*)
            integer(c_int) :: rc
        end function mfcfd_knn

        function mfcfd_set_fault_hook(h, point, wait_limit) result(rc) bind(C, name="mfcfd_set_fault_hook")
            import :: c_ptr, c_int32_t, c_int
            type(c_ptr), value :: h
            integer(c_int32_t), value :: point, wait_limit
            integer(c_int) :: rc
        end function mfcfd_set_fault_hook

        ! the reference program's files (meshfree_solver.f90:20-37)
        function mfcfd_count_input_points(path, n) result(rc) bind(C, name="mfcfd_count_input_points")
            import :: c_char, c_int32_t, c_int
            character(kind=c_char), dimension(*), intent(in) :: path
            integer(c_int32_t), intent(out) :: n
            integer(c_int) :: rc
        end function mfcfd_count_input_points

        function mfcfd_read_input_point_data(path, n, status, x, y, z, tan1, tan2, nor, nbhs, conn, &
                                             min_dist) result(rc) bind(C, name="mfcfd_read_input_point_data")
            import :: c_char, c_int32_t, c_double, c_int
            character(kind=c_char), dimension(*), intent(in) :: path
            integer(c_int32_t), value :: n
            integer(c_int32_t), intent(out) :: status(*), nbhs(*), conn(27, *)
            real(c_double), intent(out) :: x(*), y(*), z(*), tan1(3, *), tan2(3, *), nor(3, *), min_dist(*)
            integer(c_int) :: rc
        end function mfcfd_read_input_point_data

        function mfcfd_read_stored_solution(path, n, prim) result(rc) bind(C, name="mfcfd_read_stored_solution")
            import :: c_char, c_int32_t, c_double, c_int
            character(kind=c_char), dimension(*), intent(in) :: path
            integer(c_int32_t), value :: n
            real(c_double), intent(out) :: prim(5, *)
            integer(c_int) :: rc
        end function mfcfd_read_stored_solution

        function mfcfd_print_primal_output(h, dir) result(rc) bind(C, name="mfcfd_print_primal_output")
            import :: c_ptr, c_char, c_int
            type(c_ptr), value :: h
            character(kind=c_char), dimension(*), intent(in) :: dir
            integer(c_int) :: rc
        end function mfcfd_print_primal_output

        function mfcfd_write_residue(path, t0, iters, res_hist, append) result(rc) bind(C, name="mfcfd_write_residue")
            import :: c_char, c_int32_t, c_double, c_int
            character(kind=c_char), dimension(*), intent(in) :: path
            integer(c_int32_t), value :: t0, iters, append
            real(c_double), intent(in) :: res_hist(2, *)
            integer(c_int) :: rc
        end function mfcfd_write_residue

        ! CL/CD of the current state (no counterpart in the reference)
        function mfcfd_forces(h, wall_area, ref_area, cl, cd, force) result(rc) bind(C, name="mfcfd_forces")
            import :: c_ptr, c_double, c_int
            type(c_ptr), value :: h
            real(c_double), value :: wall_area, ref_area
            real(c_double), intent(out) :: cl, cd, force(3)
            integer(c_int) :: rc
        end function mfcfd_forces

        ! several clouds at once: hs(count) handles, t0(count), res_hist(2, iters, count)
        function mfcfd_run_batch(hs, count, t0, iters, res_hist, status) result(rc) bind(C, name="mfcfd_run_batch")
            import :: c_ptr, c_int32_t, c_double, c_int
            type(c_ptr), intent(in) :: hs(*)
            integer(c_int32_t), value :: count, iters
            integer(c_int32_t), intent(in) :: t0(*)
            real(c_double), intent(out) :: res_hist(*)
            integer(c_int32_t), intent(out) :: status(*)
            integer(c_int) :: rc
        end function mfcfd_run_batch

        ! the same in lockstep, each sweep of all count (<= 32) handles in one launch
        function mfcfd_run_group(hs, count, t0, iters, res_hist, status) result(rc) bind(C, name="mfcfd_run_group")
            import :: c_ptr, c_int32_t, c_double, c_int
            type(c_ptr), intent(in) :: hs(*)
            integer(c_int32_t), value :: count, iters
            integer(c_int32_t), intent(in) :: t0(*)
            real(c_double), intent(out) :: res_hist(*)
            integer(c_int32_t), intent(out) :: status(*)
            integer(c_int) :: rc
        end function mfcfd_run_group

        function mfcfd_tune_chain(h, candidates, count, iters, chosen, ms) result(rc) bind(C, name="mfcfd_tune_chain")
            import :: c_ptr, c_int32_t, c_int
            type(c_ptr), value :: h, candidates, ms
            integer(c_int32_t), value :: count, iters
            integer(c_int32_t), intent(out) :: chosen
            integer(c_int) :: rc
        end function mfcfd_tune_chain

        function mfcfd_launch(h, t0, iters) result(rc) bind(C, name="mfcfd_launch")
            import :: c_ptr, c_int32_t, c_int
            type(c_ptr), value :: h
            integer(c_int32_t), value :: t0, iters
            integer(c_int) :: rc
        end function mfcfd_launch

        function mfcfd_complete(h, wait, res_hist, done) result(rc) bind(C, name="mfcfd_complete")
            import :: c_ptr, c_int32_t, c_double, c_int
            type(c_ptr), value :: h
            integer(c_int32_t), value :: wait
            real(c_double), intent(out) :: res_hist(*)
            integer(c_int32_t), intent(out) :: done
            integer(c_int) :: rc
        end function mfcfd_complete

        function mfcfd_destroy(h) result(rc) bind(C, name="mfcfd_destroy")
            import :: c_ptr, c_int
            type(c_ptr), value :: h
            integer(c_int) :: rc
        end function mfcfd_destroy

        function mfcfd_last_error(h) result(msg) bind(C, name="mfcfd_last_error")
            import :: c_ptr
            type(c_ptr), value :: h
            type(c_ptr) :: msg
        end function mfcfd_last_error
    end interface
end module mfcfd_interface
