!> ISO_C_BINDING interface to libweno_sb.so (include/weno_sb.h).
!!
!! Drop-in for the device loops of the WENO harness
!! (wilfonba/WenoStandalone inputs/weno_standalone.f90): each wrapper keeps
!! the reference routine's name and replaces its `!$omp target` region with
!! one library call on the handle created by weno_sb_init.  Arrays are passed
!! by base address (c_loc of the first element) in the reference's own
!! column-major layouts.
!!
!! Build (with any Fortran 2008 compiler):
!!   gfortran -c m_weno_sb.f90
!!   gfortran my_driver.f90 m_weno_sb.o -L<dir> -lweno_sb -Wl,-rpath,<dir>
module m_weno_sb

    use, intrinsic :: iso_c_binding
    implicit none

    integer(c_int), parameter :: WENO_SB_JS = 0, WENO_SB_MAPPED = 1, WENO_SB_Z = 2
    integer(c_int), parameter :: WENO_SB_TENO = 3, WENO_SB_NONE = 4
    integer(c_int), parameter :: WENO_SB_FP64 = 0, WENO_SB_FP32 = 1
    integer(c_int), parameter :: WENO_SB_F_SPLIT = 1, WENO_SB_F_SPECIALIZED = 2
    integer(c_int), parameter :: WENO_SB_F_MP = 4, WENO_SB_F_FOLDED = 8
    integer(c_int), parameter :: WENO_SB_A_V_VF = 0

    !> struct weno_sb_grid (the &grid_params namelist, f90:117-118)
    type, bind(C) :: weno_sb_grid
        integer(c_int32_t) :: m_cells, n_cells, p_cells
        integer(c_int32_t) :: v_size, buff_size, scheme
        real(c_double) :: weno_eps, teno_CT
    end type weno_sb_grid

    interface
        integer(c_int) function weno_sb_init(g, precision, handle) bind(C, name='weno_sb_init')
            import :: c_int, weno_sb_grid
            type(weno_sb_grid), intent(in) :: g
            integer(c_int), value :: precision
            integer(c_int), intent(out) :: handle
        end function weno_sb_init

        integer(c_int) function weno_sb_finalize(handle) bind(C, name='weno_sb_finalize')
            import :: c_int
            integer(c_int), value :: handle
        end function weno_sb_finalize

        integer(c_int) function weno_sb_upload(handle, which, host) bind(C, name='weno_sb_upload')
            import :: c_int, c_ptr
            integer(c_int), value :: handle, which
            type(c_ptr), value :: host
        end function weno_sb_upload

        integer(c_int) function weno_sb_download(handle, which, host) bind(C, name='weno_sb_download')
            import :: c_int, c_ptr
            integer(c_int), value :: handle, which
            type(c_ptr), value :: host
        end function weno_sb_download

        integer(c_int) function weno_sb_initialize_weno(handle, dir) bind(C, name='weno_sb_initialize_weno')
            import :: c_int
            integer(c_int), value :: handle, dir
        end function weno_sb_initialize_weno

        integer(c_int) function weno_sb_weno(handle, dir, order, flags) bind(C, name='weno_sb_weno')
            import :: c_int
            integer(c_int), value :: handle, dir, order, flags
        end function weno_sb_weno

        integer(c_int) function weno_sb_preserve_monotonicity(handle, dir) &
            bind(C, name='weno_sb_preserve_monotonicity')
            import :: c_int
            integer(c_int), value :: handle, dir
        end function weno_sb_preserve_monotonicity

        integer(c_int) function weno_sb_checksum(handle, which, result) bind(C, name='weno_sb_checksum')
            import :: c_int, c_double
            integer(c_int), value :: handle, which
            real(c_double), intent(out) :: result
        end function weno_sb_checksum

        integer(c_int) function weno_sb_sync(handle) bind(C, name='weno_sb_sync')
            import :: c_int
            integer(c_int), value :: handle
        end function weno_sb_sync

        type(c_ptr) function weno_sb_last_error_string() bind(C, name='weno_sb_last_error_string')
            import :: c_ptr
        end function weno_sb_last_error_string
    end interface

    integer(c_int), save :: weno_sb_handle = 0

contains

    !> Array id helpers (WENO_SB_A_* in weno_sb.h); dir is 0, 1 or 2.
    integer(c_int) function weno_sb_a_rs(dir)
        integer, intent(in) :: dir
        weno_sb_a_rs = int(1 + dir, c_int)
    end function weno_sb_a_rs

    integer(c_int) function weno_sb_a_vl(dir)
        integer, intent(in) :: dir
        weno_sb_a_vl = int(4 + dir, c_int)
    end function weno_sb_a_vl

    integer(c_int) function weno_sb_a_vr(dir)
        integer, intent(in) :: dir
        weno_sb_a_vr = int(7 + dir, c_int)
    end function weno_sb_a_vr

    !> Stop with the library's message when a call fails (the reference
    !! aborts through OMP_TARGET_OFFLOAD=MANDATORY instead).
    subroutine s_weno_sb_check(rc, what)
        integer(c_int), intent(in) :: rc
        character(len=*), intent(in) :: what
        character(kind=c_char), pointer :: msg(:)
        integer :: n
        if (rc == 0) return
        call c_f_pointer(weno_sb_last_error_string(), msg, [512])
        n = 0
        do while (n < 512)
            if (msg(n + 1) == c_null_char) exit
            n = n + 1
        end do
        write(*, '(a,a,a,i0,a,512a)') '  ERROR in ', what, ' (status ', rc, '): ', msg(1:n)
        error stop 2
    end subroutine s_weno_sb_check

    ! ---- the reference routines, one library call each ----

    subroutine s_initialize_weno_x()    ! f90:281-296
        call s_weno_sb_check(weno_sb_initialize_weno(weno_sb_handle, 0_c_int), 's_initialize_weno_x')
    end subroutine s_initialize_weno_x

    subroutine s_initialize_weno_y()    ! f90:298-313
        call s_weno_sb_check(weno_sb_initialize_weno(weno_sb_handle, 1_c_int), 's_initialize_weno_y')
    end subroutine s_initialize_weno_y

    subroutine s_initialize_weno_z()    ! f90:315-330
        call s_weno_sb_check(weno_sb_initialize_weno(weno_sb_handle, 2_c_int), 's_initialize_weno_z')
    end subroutine s_initialize_weno_z

    !> s_order1_copy_{x,y,z} (f90:332-390); dir = 0, 1, 2
    subroutine s_order1_copy(dir)
        integer, intent(in) :: dir
        call s_weno_sb_check(weno_sb_weno(weno_sb_handle, int(dir, c_int), 1_c_int, 0_c_int), 's_order1_copy')
    end subroutine s_order1_copy

    !> s_weno3_kernel (f90:392-475)
    subroutine s_weno3_kernel(dir)
        integer, intent(in) :: dir
        call s_weno_sb_check(weno_sb_weno(weno_sb_handle, int(dir, c_int), 3_c_int, 0_c_int), 's_weno3_kernel')
    end subroutine s_weno3_kernel

    !> s_weno5_kernel_dispatch (f90:1399-1417): split or combined
    subroutine s_weno5_kernel_dispatch(dir, split)
        integer, intent(in) :: dir
        logical, intent(in) :: split
        integer(c_int) :: fl
        fl = 0_c_int
        if (split) fl = WENO_SB_F_SPLIT
        call s_weno_sb_check(weno_sb_weno(weno_sb_handle, int(dir, c_int), 5_c_int, fl), 's_weno5_kernel_dispatch')
    end subroutine s_weno5_kernel_dispatch

    !> s_weno5_kernel_{x,y,z} (f90:671-1143)
    subroutine s_weno5_kernel_specialized(dir)
        integer, intent(in) :: dir
        call s_weno_sb_check(weno_sb_weno(weno_sb_handle, int(dir, c_int), 5_c_int, WENO_SB_F_SPECIALIZED), &
                             's_weno5_kernel_specialized')
    end subroutine s_weno5_kernel_specialized

    !> s_weno7_kernel (f90:1419-1542)
    subroutine s_weno7_kernel(dir)
        integer, intent(in) :: dir
        call s_weno_sb_check(weno_sb_weno(weno_sb_handle, int(dir, c_int), 7_c_int, 0_c_int), 's_weno7_kernel')
    end subroutine s_weno7_kernel

    !> s_preserve_monotonicity (f90:1544-1615)
    subroutine s_preserve_monotonicity(dir)
        integer, intent(in) :: dir
        call s_weno_sb_check(weno_sb_preserve_monotonicity(weno_sb_handle, int(dir, c_int)), &
                             's_preserve_monotonicity')
    end subroutine s_preserve_monotonicity

end module m_weno_sb
