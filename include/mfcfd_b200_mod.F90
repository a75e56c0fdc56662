! Fortran binding of the mfcfd_b200 C ABI (include/mfcfd_b200.h).
!
! A maintainer of the Fortran solver adds this module and replaces the call
! of q_lskum() in meshfree_solver.F90 by q_lskum_b200(), which runs the same
! pseudo-time loop (q_lskum.F90:16-79) on the GPU and writes the same
! residue and cp files.  The point arrays of module data_structure_mod are
! passed as they are (column-major conn(N,20), prim(4,N)).
!
! Build: compile with the solver and link -L<repo>/mfcfd_b200 -lmfcfd_b200.
! (No Fortran compiler exists on the machines this library was built on; the
! module is checked only by reading.)
module mfcfd_b200
    use iso_c_binding
    implicit none

    integer(c_int), parameter :: MFCFD_OK = 0, MFCFD_ERR_NONFINITE = -3
    integer(c_int), parameter :: MFCFD_FP64 = 0, MFCFD_FP32_MIXED = 1

    type, bind(C) :: mfcfd_grid
        integer(c_int) :: n
        type(c_ptr) :: x, y, nx, ny, min_dist
        type(c_ptr) :: flag_1, flag_2, left, right, nbhs, conn
        integer(c_int) :: ld_conn
        integer(c_int) :: shapes
    end type

    type, bind(C) :: mfcfd_params
        real(c_double) :: cfl, power, vl_const, mach, aoa
        integer(c_int) :: rks
        real(c_double) :: euler
        integer(c_int) :: inner_iterations, interior_points_normal_flag, format, restart
        real(c_double) :: res_old
        integer(c_int) :: precision, ordering
    end type

    interface
        integer(c_int) function mfcfd_create(grid, params, h) bind(C, name="mfcfd_create")
            import :: c_int, c_ptr, mfcfd_grid, mfcfd_params
            type(mfcfd_grid), intent(in) :: grid
            type(mfcfd_params), intent(in) :: params
            type(c_ptr), intent(out) :: h
        end function
        integer(c_int) function mfcfd_destroy(h) bind(C, name="mfcfd_destroy")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
        end function
        integer(c_int) function mfcfd_set_state(h, prim) bind(C, name="mfcfd_set_state")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(in) :: prim(*)
        end function
        integer(c_int) function mfcfd_get_state(h, prim) bind(C, name="mfcfd_get_state")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(out) :: prim(*)
        end function
        integer(c_int) function mfcfd_run(h, it_first, n_iters, residue, n_done) &
                bind(C, name="mfcfd_run")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            integer(c_int), value :: it_first, n_iters
            real(c_double), intent(out) :: residue(*)
            integer(c_int), intent(out) :: n_done
        end function
        integer(c_int) function mfcfd_forces(h, cl, cd, cm, cp) bind(C, name="mfcfd_forces")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(out) :: cl(*), cd(*), cm(*), cp(*)
        end function
        type(c_ptr) function mfcfd_strerror(status) bind(C, name="mfcfd_strerror")
            import :: c_int, c_ptr
            integer(c_int), value :: status
        end function
    end interface

contains

    ! Drop-in for q_lskum (q_lskum.F90:16-79) on a single rank.
    subroutine q_lskum_b200()
        use data_structure_mod
        use parameter_mod
        implicit none
        type(mfcfd_grid), target :: g
        type(mfcfd_params) :: p
        type(c_ptr) :: h
        integer(c_int) :: st, done
        real(c_double), allocatable, target :: res(:), cp(:)
        integer, allocatable, target :: conn_c(:,:)
        integer :: i, j

        allocate(conn_c(max_points, 20))
        conn_c = point%conn
        g%n = max_points
        g%x = c_loc(point%x); g%y = c_loc(point%y)
        g%nx = c_loc(point%nx); g%ny = c_loc(point%ny)
        g%min_dist = c_loc(point%min_dist)
        g%flag_1 = c_loc(point%flag_1); g%flag_2 = c_loc(point%flag_2)
        g%left = c_loc(point%left); g%right = c_loc(point%right)
        g%nbhs = c_loc(point%nbhs); g%conn = c_loc(conn_c)
        g%ld_conn = max_points
        g%shapes = shapes
        p%cfl = cfl; p%power = power; p%vl_const = vl_const
        p%mach = Mach; p%aoa = aoa
        p%rks = rks; p%euler = euler
        p%inner_iterations = inner_iterations
        p%interior_points_normal_flag = interior_points_normal_flag
        p%format = format; p%restart = restart; p%res_old = res_old
        p%precision = MFCFD_FP64; p%ordering = 0

        st = mfcfd_create(g, p, h)
        if (st /= MFCFD_OK) stop "mfcfd_create failed"
        st = mfcfd_set_state(h, point%prim)
        if (restart == 0) itr = 0
        allocate(res(max_iters), cp(shape_points))
        OPEN(UNIT=301, FILE="residue", FORM="FORMATTED", STATUS="REPLACE", ACTION="WRITE")
        st = mfcfd_run(h, itr + 1, max_iters, res, done)
        do i = 1, done
            it = itr + i
            write(*,'(a12,i8,a15,e30.20)') 'iterations:', it, 'residue:', res(i)
            write(301, *) it, res(i)
        end do
        CLOSE(UNIT=301)
        st = mfcfd_get_state(h, point%prim)
        st = mfcfd_forces(h, Cl, Cd, Cm, cp)
        vector_cost_func = Cd
        OPEN(UNIT=201, FILE='cp/cp-file', FORM="FORMATTED", STATUS="REPLACE", ACTION="WRITE")
        do j = 1, shape_points
            write(201, *) point%flag_2(shape_points_index(j)), point%x(shape_points_index(j)), cp(j)
        end do
        CLOSE(UNIT=201)
        write(*,*) "Vector function is ", vector_cost_func
        st = mfcfd_destroy(h)
    end subroutine

end module mfcfd_b200
