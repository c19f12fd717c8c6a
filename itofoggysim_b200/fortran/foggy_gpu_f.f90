! foggy_gpu_f -- iso_c_binding module over the C ABI of libfoggy_b200 (include/foggy_gpu.h).
!
! It lets the FoggySim driver call the B200 solver in place of the Fortran solve path:
!   lib_mie_ms_constructor / lib_mie_ms_solver_constructor
!       (FoggySim/src/lib/mie_theory/lib_mie_multi_sphere.f90:111-150,
!        lib_mie_ms_solver_interface.f90:91-129)            -> foggy_ms_constructor
!   lib_mie_ms_solver_run (lib_mie_ms_solver_interface.f90:143-154)
!                                                           -> foggy_ms_solver_run
!   lib_mie_ms_solver_calculate_vector_b (:739-783)         -> foggy_ms_calculate_vector_b
!   lib_mie_ms_solver_get_backward_error (:203-209)         -> foggy_ms_get_backward_error
! Vectors keep the reference's flat layout (double complex, per sphere [a_nm | b_nm]), so the
! solution can be handed to lib_mie_ms_solver_set_sphere_parameter_ab_nm_all unchanged.
!
! No Fortran compiler exists on the machines this project is built on, so this file has not
! been compiled; its interfaces are checked by hand against include/foggy_gpu.h.
module foggy_gpu_f
    use iso_c_binding
    implicit none
    private

    integer(c_int32_t), parameter, public :: FOGGY_OK = 0
    integer(c_int32_t), parameter, public :: FOGGY_MEM_HOST = 0
    integer(c_int32_t), parameter, public :: FOGGY_MATVEC_DIRECT = 0
    integer(c_int32_t), parameter, public :: FOGGY_MATVEC_MLFMM = 1

    type, bind(c), public :: foggy_params
        real(c_double) :: lambda_0
        real(c_double) :: n_medium
        integer(c_int32_t) :: n_range(2)
        integer(c_int32_t) :: z_coupling
        integer(c_int32_t) :: reference_row_rule
        integer(c_int32_t) :: matvec_mode
        integer(c_int32_t) :: use_initial_guess
        integer(c_int32_t) :: gmres_restart
        integer(c_int32_t) :: gmres_max_iterations
        real(c_double) :: gmres_tolerance
        integer(c_int32_t) :: tree_l_max
        integer(c_int32_t) :: tree_s_opt
        real(c_double) :: fmm_digits
        integer(c_int64_t) :: device_memory_budget
        integer(c_int32_t) :: pair_tables
        integer(c_int32_t) :: fmm_convention
        integer(c_int32_t) :: z_translation_gt_r
        integer(c_int32_t) :: precision
    end type foggy_params

    type, bind(c), public :: foggy_stats
        integer(c_int32_t) :: iterations
        integer(c_int32_t) :: restarts
        integer(c_int32_t) :: matvecs
        integer(c_int32_t) :: status
        real(c_double) :: backward_error
        real(c_double) :: ms_total
        real(c_double) :: ms_matvec
        real(c_double) :: ms_setup
        integer(c_int64_t) :: kernel_launches
    end type foggy_stats

    ! one solve request of the server (foggy_request): every pointer is c_loc of a contiguous array
    type, bind(c), public :: foggy_request
        type(c_ptr) :: params
        integer(c_int32_t) :: n_spheres
        type(c_ptr) :: centres, param_index
        integer(c_int32_t) :: n_param
        type(c_ptr) :: refractive_index, radius, n_range
        integer(c_int32_t) :: nw
        type(c_ptr) :: theta, phi, jones, g, phase, d_0_i
        integer(c_int32_t) :: rhs_per_wave
    end type foggy_request

    type, bind(c), public :: foggy_request_info
        integer(c_int32_t) :: state, status, nrhs, reserved
        integer(c_int64_t) :: x_len, footprint
        real(c_double) :: ms_queued, ms_solve, ms_latency
        type(foggy_stats) :: stats
        character(kind=c_char) :: error(256)
    end type foggy_request_info

    interface
        subroutine foggy_default_params(p) bind(c, name="foggy_default_params")
            import :: foggy_params
            type(foggy_params), intent(out) :: p
        end subroutine
        function foggy_create(p, device, h) result(rc) bind(c, name="foggy_create")
            import :: foggy_params, c_int32_t, c_ptr
            type(foggy_params), intent(in) :: p
            integer(c_int32_t), value :: device
            type(c_ptr), intent(out) :: h
            integer(c_int32_t) :: rc
        end function
        function foggy_destroy(h) result(rc) bind(c, name="foggy_destroy")
            import :: c_ptr, c_int32_t
            type(c_ptr), value :: h
            integer(c_int32_t) :: rc
        end function
        function foggy_set_spheres(h, n, centres, param_index, n_param, refractive_index, radius, n_range) &
                result(rc) bind(c, name="foggy_set_spheres")
            import :: c_ptr, c_int32_t, c_double, c_double_complex
            type(c_ptr), value :: h
            integer(c_int32_t), value :: n, n_param
            real(c_double), intent(in) :: centres(3, *)
            integer(c_int32_t), intent(in) :: param_index(*)
            complex(c_double_complex), intent(in) :: refractive_index(*)
            real(c_double), intent(in) :: radius(*)
            integer(c_int32_t), intent(in) :: n_range(2, *)
            integer(c_int32_t) :: rc
        end function
        function foggy_set_plane_waves(h, nw, theta, phi, jones, g, phase, d_0_i) &
                result(rc) bind(c, name="foggy_set_plane_waves")
            import :: c_ptr, c_int32_t, c_double, c_double_complex
            type(c_ptr), value :: h
            integer(c_int32_t), value :: nw
            real(c_double), intent(in) :: theta(*), phi(*), g(*), phase(*), d_0_i(3, *)
            complex(c_double_complex), intent(in) :: jones(2, *)
            integer(c_int32_t) :: rc
        end function
        function foggy_vector_length(h) result(n) bind(c, name="foggy_vector_length")
            import :: c_ptr, c_int64_t
            type(c_ptr), value :: h
            integer(c_int64_t) :: n
        end function
        function foggy_matvec(h, x, y, mem) result(rc) bind(c, name="foggy_matvec")
            import :: c_ptr, c_int32_t
            type(c_ptr), value :: h, x, y
            integer(c_int32_t), value :: mem
            integer(c_int32_t) :: rc
        end function
        function foggy_solve(h, x0, x, mem, stats) result(rc) bind(c, name="foggy_solve")
            import :: c_ptr, c_int32_t, foggy_stats
            type(c_ptr), value :: h, x0, x
            integer(c_int32_t), value :: mem
            type(foggy_stats), intent(out) :: stats
            integer(c_int32_t) :: rc
        end function
        function foggy_get_backward_error(h) result(e) bind(c, name="foggy_get_backward_error")
            import :: c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double) :: e
        end function
        function foggy_cross_sections(h, x, mem, c_out) result(rc) bind(c, name="foggy_cross_sections")
            import :: c_ptr, c_int32_t, c_double
            type(c_ptr), value :: h, x
            integer(c_int32_t), value :: mem
            real(c_double), intent(out) :: c_out(3)
            integer(c_int32_t) :: rc
        end function
        function foggy_translation_coefficients(x, theta, phi, n_range, nu_range, z_selector, a, b) &
                result(rc) bind(c, name="foggy_translation_coefficients")
            import :: c_double, c_int32_t, c_double_complex
            real(c_double), value :: x, theta, phi
            integer(c_int32_t), intent(in) :: n_range(2), nu_range(2)
            integer(c_int32_t), value :: z_selector
            complex(c_double_complex), intent(out) :: a(*), b(*)
            integer(c_int32_t) :: rc
        end function
        function foggy_wigner_3j(j1, j2, j3, m1, m2, m3) result(w) bind(c, name="foggy_wigner_3j")
            import :: c_int32_t, c_double
            integer(c_int32_t), value :: j1, j2, j3, m1, m2, m3
            real(c_double) :: w
        end function
        function foggy_last_error(h) result(msg) bind(c, name="foggy_last_error")
            import :: c_ptr
            type(c_ptr), value :: h
            type(c_ptr) :: msg                ! NUL-terminated C string owned by the library
        end function
        function foggy_set_params(h, p) result(rc) bind(c, name="foggy_set_params")
            import :: c_ptr, c_int32_t, foggy_params
            type(c_ptr), value :: h
            type(foggy_params), intent(in) :: p
            integer(c_int32_t) :: rc
        end function
        function foggy_get_mie_coefficients(h, ip, a, b) result(rc) bind(c, name="foggy_get_mie_coefficients")
            import :: c_ptr, c_int32_t, c_double_complex
            type(c_ptr), value :: h
            integer(c_int32_t), value :: ip
            complex(c_double_complex), intent(out) :: a(*), b(*)
            integer(c_int32_t) :: rc
        end function
        function foggy_get_vector_b(h, b, mem) result(rc) bind(c, name="foggy_get_vector_b")
            import :: c_ptr, c_int32_t
            type(c_ptr), value :: h, b
            integer(c_int32_t), value :: mem
            integer(c_int32_t) :: rc
        end function
        function foggy_build_tree(h, uindex, order, l_min, l_max) result(rc) bind(c, name="foggy_build_tree")
            import :: c_ptr, c_int32_t, c_int64_t
            type(c_ptr), value :: h
            integer(c_int64_t), intent(out) :: uindex(*)
            integer(c_int32_t), intent(out) :: order(*), l_min, l_max
            integer(c_int32_t) :: rc
        end function
        function foggy_universal_index(n, points, l, out) result(rc) bind(c, name="foggy_universal_index")
            import :: c_int32_t, c_int64_t, c_double
            integer(c_int32_t), value :: n, l
            real(c_double), intent(in) :: points(3, *)
            integer(c_int64_t), intent(out) :: out(*)
            integer(c_int32_t) :: rc
        end function
        function foggy_estimate_solve_bytes(p, n_spheres, param_index, n_param, n_range, solve_bytes, &
                                            table_bytes) result(rc) bind(c, name="foggy_estimate_solve_bytes")
            import :: c_int32_t, c_int64_t, foggy_params
            type(foggy_params), intent(in) :: p
            integer(c_int32_t), value :: n_spheres, n_param
            integer(c_int32_t), intent(in) :: param_index(*), n_range(2, *)
            integer(c_int64_t), intent(out) :: solve_bytes, table_bytes
            integer(c_int32_t) :: rc
        end function
        function foggy_tree_parent(n, l, step, parent) result(rc) bind(c, name="foggy_tree_parent")
            import :: c_int32_t, c_int64_t
            integer(c_int64_t), value :: n
            integer(c_int32_t), value :: l, step
            integer(c_int64_t), intent(out) :: parent
            integer(c_int32_t) :: rc
        end function
        function foggy_tree_children(n, l, children) result(rc) bind(c, name="foggy_tree_children")
            import :: c_int32_t, c_int64_t
            integer(c_int64_t), value :: n
            integer(c_int32_t), value :: l
            integer(c_int64_t), intent(out) :: children(8)
            integer(c_int32_t) :: rc
        end function
        function foggy_tree_centre_of_box(n, l, centre) result(rc) bind(c, name="foggy_tree_centre_of_box")
            import :: c_int32_t, c_int64_t, c_double
            integer(c_int64_t), value :: n
            integer(c_int32_t), value :: l
            real(c_double), intent(out) :: centre(3)
            integer(c_int32_t) :: rc
        end function
        function foggy_tree_neighbours(n, l, out, count) result(rc) bind(c, name="foggy_tree_neighbours")
            import :: c_int32_t, c_int64_t
            integer(c_int64_t), value :: n
            integer(c_int32_t), value :: l
            integer(c_int64_t), intent(out) :: out(26)
            integer(c_int32_t), intent(out) :: count
            integer(c_int32_t) :: rc
        end function
        function foggy_tree_boxes(h, l, boxes, count) result(rc) bind(c, name="foggy_tree_boxes")
            import :: c_ptr, c_int32_t, c_int64_t
            type(c_ptr), value :: h
            integer(c_int32_t), value :: l
            type(c_ptr), value :: boxes         ! c_loc(boxes(1)), or c_null_ptr to query count
            integer(c_int32_t), intent(inout) :: count
            integer(c_int32_t) :: rc
        end function
        function foggy_tree_domain(h, l, n, kind, out, count) result(rc) bind(c, name="foggy_tree_domain")
            import :: c_ptr, c_int32_t, c_int64_t
            type(c_ptr), value :: h
            integer(c_int32_t), value :: l, kind
            integer(c_int64_t), value :: n
            type(c_ptr), value :: out           ! c_loc(out(1)), or c_null_ptr to query count
            integer(c_int32_t), intent(inout) :: count
            integer(c_int32_t) :: rc
        end function
        function foggy_get_field(h, x, mem, npoints, points, e_field_0, e_out, h_out) result(rc) &
                bind(c, name="foggy_get_field")
            import :: c_ptr, c_int32_t, c_double
            type(c_ptr), value :: h, x, points, e_out, h_out
            integer(c_int32_t), value :: mem, npoints
            real(c_double), value :: e_field_0
            integer(c_int32_t) :: rc
        end function
        function foggy_set_gaussian_beams(h, nb, waist, tem, theta, phi, jones, g, phase, d_0_i, convention) &
                result(rc) bind(c, name="foggy_set_gaussian_beams")
            import :: c_ptr, c_int32_t, c_double, c_double_complex
            type(c_ptr), value :: h
            integer(c_int32_t), value :: nb
            real(c_double), intent(in) :: waist(2, *), theta(*), phi(*), g(*)
            integer(c_int32_t), intent(in) :: tem(2, *)
            complex(c_double_complex), intent(in) :: jones(2, *)
            type(c_ptr), value :: phase, d_0_i, convention   ! c_loc(...) or c_null_ptr for defaults
            integer(c_int32_t) :: rc
        end function
        function foggy_solve_rhs(h, nrhs, x0, x, mem, stats, cross_sections) result(rc) bind(c, name="foggy_solve_rhs")
            import :: c_ptr, c_int32_t, foggy_stats
            type(c_ptr), value :: h, x0, x, cross_sections
            integer(c_int32_t), value :: nrhs, mem
            type(foggy_stats), intent(out) :: stats
            integer(c_int32_t) :: rc
        end function
        function foggy_matvec_rhs(h, nrhs, x, y, mem) result(rc) bind(c, name="foggy_matvec_rhs")
            import :: c_ptr, c_int32_t
            type(c_ptr), value :: h, x, y
            integer(c_int32_t), value :: nrhs, mem
            integer(c_int32_t) :: rc
        end function
        function foggy_server_start(device, max_concurrent, memory_budget, s) result(rc) &
                bind(c, name="foggy_server_start")
            import :: c_ptr, c_int32_t, c_int64_t
            integer(c_int32_t), value :: device, max_concurrent
            integer(c_int64_t), value :: memory_budget
            type(c_ptr), intent(out) :: s
            integer(c_int32_t) :: rc
        end function
        function foggy_server_submit(s, request, id) result(rc) bind(c, name="foggy_server_submit")
            import :: c_ptr, c_int32_t, c_int64_t, foggy_request
            type(c_ptr), value :: s
            type(foggy_request), intent(in) :: request
            integer(c_int64_t), intent(out) :: id
            integer(c_int32_t) :: rc
        end function
        function foggy_server_poll(s, id, wait_ms, info, x, x_len, cross_sections) result(rc) &
                bind(c, name="foggy_server_poll")
            import :: c_ptr, c_int32_t, c_int64_t, foggy_request_info
            type(c_ptr), value :: s, x, cross_sections
            integer(c_int64_t), value :: id, x_len
            integer(c_int32_t), value :: wait_ms
            type(foggy_request_info), intent(out) :: info
            integer(c_int32_t) :: rc
        end function
        function foggy_server_cancel(s, id) result(rc) bind(c, name="foggy_server_cancel")
            import :: c_ptr, c_int32_t, c_int64_t
            type(c_ptr), value :: s
            integer(c_int64_t), value :: id
            integer(c_int32_t) :: rc
        end function
        function foggy_server_release(s, id) result(rc) bind(c, name="foggy_server_release")
            import :: c_ptr, c_int32_t, c_int64_t
            type(c_ptr), value :: s
            integer(c_int64_t), value :: id
            integer(c_int32_t) :: rc
        end function
        function foggy_server_stop(s) result(rc) bind(c, name="foggy_server_stop")
            import :: c_ptr, c_int32_t
            type(c_ptr), value :: s
            integer(c_int32_t) :: rc
        end function
        function foggy_matvec_static(h, x, y) result(rc) bind(c, name="foggy_matvec_static")
            import :: c_ptr, c_int32_t
            type(c_ptr), value :: h, x, y       ! device pointers
            integer(c_int32_t) :: rc
        end function
        function foggy_solve_block(h, nrhs, x0, x, mem, stats, cross_sections, iterations, backward_errors) &
                result(rc) bind(c, name="foggy_solve_block")
            import :: c_ptr, c_int32_t, foggy_stats
            type(c_ptr), value :: h, x0, x, cross_sections, iterations, backward_errors
            integer(c_int32_t), value :: nrhs, mem
            type(foggy_stats), intent(out) :: stats
            integer(c_int32_t) :: rc
        end function
        function foggy_matvec_block(h, nrhs, precision, x, y, mem) result(rc) bind(c, name="foggy_matvec_block")
            import :: c_ptr, c_int32_t
            type(c_ptr), value :: h, x, y
            integer(c_int32_t), value :: nrhs, precision, mem
            integer(c_int32_t) :: rc
        end function
        function foggy_fmm_lists(h, part, out, count) result(rc) bind(c, name="foggy_fmm_lists")
            import :: c_ptr, c_int32_t
            type(c_ptr), value :: h, out
            integer(c_int32_t), value :: part
            integer(c_int32_t), intent(out) :: count
            integer(c_int32_t) :: rc
        end function
        function foggy_block_tiles(h, precision, nrhs, out, count) result(rc) bind(c, name="foggy_block_tiles")
            import :: c_ptr, c_int32_t
            type(c_ptr), value :: h, out
            integer(c_int32_t), value :: precision, nrhs
            integer(c_int32_t), intent(out) :: count
            integer(c_int32_t) :: rc
        end function
    end interface

    public :: foggy_default_params, foggy_create, foggy_destroy, foggy_set_spheres
    public :: foggy_set_plane_waves, foggy_vector_length, foggy_matvec, foggy_solve
    public :: foggy_get_backward_error, foggy_cross_sections, foggy_translation_coefficients
    public :: foggy_wigner_3j, foggy_last_error, foggy_set_params, foggy_get_mie_coefficients
    public :: foggy_get_vector_b, foggy_build_tree, foggy_universal_index, foggy_tree_boxes
    public :: foggy_tree_domain, foggy_get_field, foggy_matvec_static, foggy_set_gaussian_beams
    public :: foggy_solve_rhs, foggy_server_start, foggy_server_submit, foggy_server_poll
    public :: foggy_server_cancel, foggy_server_release, foggy_server_stop, foggy_matvec_rhs
    public :: foggy_tree_parent, foggy_tree_children, foggy_tree_centre_of_box, foggy_tree_neighbours
    public :: foggy_estimate_solve_bytes, foggy_solve_block, foggy_matvec_block, foggy_block_tiles
    public :: foggy_fmm_lists
    public :: foggy_ms_constructor, foggy_ms_solver_run, foggy_ms_solver_run_block, foggy_ms_calculate_vector_b
    public :: foggy_ms_get_backward_error, foggy_ms_destructor, foggy_ms_vector_length

    type(c_ptr), save :: m_handle = c_null_ptr

    contains

        ! Mirrors lib_mie_ms_constructor(n_range, use_ml_fmm, init_with_single_sphere) with the
        ! scene passed explicitly instead of through simulation_data.
        subroutine foggy_ms_constructor(p, centres, param_index, refractive_index, radius, n_range_param, &
                                        theta, phi, jones, g, phase, d_0_i, rc)
            type(foggy_params), intent(in) :: p
            real(c_double), intent(in) :: centres(:, :)
            integer(c_int32_t), intent(in) :: param_index(:)          ! 0-based
            complex(c_double_complex), intent(in) :: refractive_index(:)
            real(c_double), intent(in) :: radius(:)
            integer(c_int32_t), intent(in) :: n_range_param(:, :)
            real(c_double), intent(in) :: theta(:), phi(:), g(:), phase(:), d_0_i(:, :)
            complex(c_double_complex), intent(in) :: jones(:, :)
            integer(c_int32_t), intent(out) :: rc
            rc = foggy_create(p, 0_c_int32_t, m_handle)
            if (rc /= FOGGY_OK) return
            rc = foggy_set_spheres(m_handle, int(size(centres, 2), c_int32_t), centres, param_index, &
                                   int(size(radius), c_int32_t), refractive_index, radius, n_range_param)
            if (rc /= FOGGY_OK) return
            rc = foggy_set_plane_waves(m_handle, int(size(theta), c_int32_t), theta, phi, jones, g, phase, d_0_i)
        end subroutine

        ! Mirrors lib_mie_ms_solver_run: x receives the solution in the reference layout.
        subroutine foggy_ms_solver_run(x, stats, rc)
            complex(c_double_complex), intent(inout), target, contiguous :: x(:)
            type(foggy_stats), intent(out) :: stats
            integer(c_int32_t), intent(out) :: rc
            rc = foggy_solve(m_handle, c_null_ptr, c_loc(x), FOGGY_MEM_HOST, stats)
        end subroutine

        ! lib_mie_ms_solver_run once per plane wave of the constructor, all in one block: x(:, i) receives
        ! the solution of wave i alone, iterations(i) its Arnoldi steps (foggy_solve_block).
        subroutine foggy_ms_solver_run_block(x, iterations, stats, rc)
            complex(c_double_complex), intent(inout), target, contiguous :: x(:, :)
            integer(c_int32_t), intent(out), target, contiguous :: iterations(:)
            type(foggy_stats), intent(out) :: stats
            integer(c_int32_t), intent(out) :: rc
            rc = foggy_solve_block(m_handle, int(size(x, 2), c_int32_t), c_null_ptr, c_loc(x), FOGGY_MEM_HOST, &
                                   stats, c_null_ptr, c_loc(iterations), c_null_ptr)
        end subroutine

        ! Mirrors lib_mie_ms_solver_calculate_vector_b(vector_x, vector_b).
        subroutine foggy_ms_calculate_vector_b(vector_x, vector_b, rc)
            complex(c_double_complex), intent(in), target, contiguous :: vector_x(:)
            complex(c_double_complex), intent(inout), target, contiguous :: vector_b(:)
            integer(c_int32_t), intent(out) :: rc
            rc = foggy_matvec(m_handle, c_loc(vector_x), c_loc(vector_b), FOGGY_MEM_HOST)
        end subroutine

        function foggy_ms_get_backward_error() result(e)
            real(c_double) :: e
            e = foggy_get_backward_error(m_handle)
        end function

        ! entries of a solution vector of the current scene, in the reference's flat layout
        function foggy_ms_vector_length() result(n)
            integer(c_int64_t) :: n
            n = foggy_vector_length(m_handle)
        end function

        subroutine foggy_ms_destructor()
            integer(c_int32_t) :: rc
            if (c_associated(m_handle)) rc = foggy_destroy(m_handle)
            m_handle = c_null_ptr
        end subroutine

end module foggy_gpu_f
