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

    ! mirror of struct mfcfd_params
    type, bind(C) :: mfcfd_params
        real(c_double) :: power, vl_const, cfl
        real(c_double) :: rho_inf, u1_inf, u2_inf, u3_inf, pr_inf
        integer(c_int32_t) :: inner_iterations, split_capacity, precision, device, sweep_mode
        integer(c_int32_t) :: reserved(7)
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
