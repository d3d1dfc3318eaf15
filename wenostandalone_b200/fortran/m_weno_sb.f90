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
    integer(c_int), parameter :: WENO_SB_F_ACCUMULATE = 16
    integer(c_int), parameter :: WENO_SB_A_V_VF = 0
    integer(c_int), parameter :: WENO_SB_ERR_ARG = 1001, WENO_SB_ERR_HANDLE = 1002
    integer(c_int), parameter :: WENO_SB_ERR_UNSUPPORTED = 1003, WENO_SB_ERR_TIMEOUT = 1005

    !> struct weno_sb_grid (the &grid_params namelist, f90:117-118)
    type, bind(C) :: weno_sb_grid
        integer(c_int32_t) :: m_cells, n_cells, p_cells
        integer(c_int32_t) :: v_size, buff_size, scheme
        real(c_double) :: weno_eps, teno_CT
    end type weno_sb_grid

    !> struct weno_sb_coefs: device addresses of one direction's coefficient
    !! arrays (polyL/R (NC,5,3), d (5,NC), beta_coef (NC,5,6); f90:171-187)
    type, bind(C) :: weno_sb_coefs
        type(c_ptr) :: polyL, polyR, dL, dR, beta_coef
    end type weno_sb_coefs

    !> struct weno_sb_face_coefs: one face's coefficients on the host, for
    !! face-independent coefficients; polyL(r+1, s+1) = polyL(j, r, s),
    !! dL(r+1) = d_cbL(r, j), beta_coef(r+1, s+1) = beta_coef(j, r, s)
    type, bind(C) :: weno_sb_face_coefs
        real(c_double) :: polyL(5, 3), polyR(5, 3)
        real(c_double) :: dL(5), dR(5)
        real(c_double) :: beta_coef(5, 6)
    end type weno_sb_face_coefs

    !> struct weno_sb_block: one entry of a batch of uneven blocks
    type, bind(C) :: weno_sb_block
        type(weno_sb_grid) :: grid
        integer(c_int32_t) :: dir, order
        integer(c_int32_t) :: flags       ! unsigned in C; the same bits
        integer(c_int32_t) :: dtype
        type(c_ptr) :: v_in
        type(weno_sb_coefs) :: coefs
        type(c_ptr) :: vL, vR
    end type weno_sb_block

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

        !> v_vf without waiting: the folded sweeps overlap the copy; keep the
        !! (page-locked) host buffer unchanged until weno_sb_sync
        integer(c_int) function weno_sb_upload_async(handle, which, host) bind(C, name='weno_sb_upload_async')
            import :: c_int, c_ptr
            integer(c_int), value :: handle, which
            type(c_ptr), value :: host
        end function weno_sb_upload_async

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

        integer(c_int) function weno_sb_version() bind(C, name='weno_sb_version')
            import :: c_int
        end function weno_sb_version

        integer(c_int) function weno_sb_extents(g, dir, ns, c1, c2) bind(C, name='weno_sb_extents')
            import :: c_int, c_int64_t, weno_sb_grid
            type(weno_sb_grid), intent(in) :: g
            integer(c_int), value :: dir
            integer(c_int64_t), intent(out) :: ns, c1, c2
        end function weno_sb_extents

        integer(c_int) function weno_sb_array_info(handle, which, dev_ptr, n_elem, dtype) &
            bind(C, name='weno_sb_array_info')
            import :: c_int, c_int64_t, c_ptr
            integer(c_int), value :: handle, which
            type(c_ptr), intent(out) :: dev_ptr
            integer(c_int64_t), intent(out) :: n_elem
            integer(c_int), intent(out) :: dtype
        end function weno_sb_array_info

        integer(c_int) function weno_sb_stream(handle, stream) bind(C, name='weno_sb_stream')
            import :: c_int, c_ptr
            integer(c_int), value :: handle
            type(c_ptr), intent(out) :: stream
        end function weno_sb_stream

        integer(c_int) function weno_sb_check_device(stream) bind(C, name='weno_sb_check_device')
            import :: c_int, c_ptr
            type(c_ptr), value :: stream
        end function weno_sb_check_device

        !> adjoint on the handle's arrays; gL, gR, gv are device addresses
        integer(c_int) function weno_sb_vjp(handle, dir, order, flags, gL, gR, gv) bind(C, name='weno_sb_vjp')
            import :: c_int, c_ptr
            integer(c_int), value :: handle, dir, order, flags
            type(c_ptr), value :: gL, gR, gv
        end function weno_sb_vjp

        ! ---- device-pointer API (caller-owned device arrays, e.g. from
        ! ---- `!$omp target data use_device_ptr` or `!$acc host_data`)

        integer(c_int) function weno_sb_reshape_dev(g, dir, dtype, v_vf, v_rs_ws, stream) &
            bind(C, name='weno_sb_reshape_dev')
            import :: c_int, c_ptr, weno_sb_grid
            type(weno_sb_grid), intent(in) :: g
            integer(c_int), value :: dir, dtype
            type(c_ptr), value :: v_vf, v_rs_ws, stream
        end function weno_sb_reshape_dev

        integer(c_int) function weno_sb_order1_dev(g, dir, dtype, v_vf, vL, vR, stream) &
            bind(C, name='weno_sb_order1_dev')
            import :: c_int, c_ptr, weno_sb_grid
            type(weno_sb_grid), intent(in) :: g
            integer(c_int), value :: dir, dtype
            type(c_ptr), value :: v_vf, vL, vR, stream
        end function weno_sb_order1_dev

        integer(c_int) function weno_sb_weno_dev(g, dir, order, flags, dtype, v_in, coefs, vL, vR, stream) &
            bind(C, name='weno_sb_weno_dev')
            import :: c_int, c_ptr, weno_sb_grid, weno_sb_coefs
            type(weno_sb_grid), intent(in) :: g
            integer(c_int), value :: dir, order, flags, dtype
            type(c_ptr), value :: v_in
            type(weno_sb_coefs), intent(in) :: coefs
            type(c_ptr), value :: vL, vR, stream
        end function weno_sb_weno_dev

        integer(c_int) function weno_sb_weno_uniform_dev(g, dir, order, flags, dtype, v_in, face, vL, vR, stream) &
            bind(C, name='weno_sb_weno_uniform_dev')
            import :: c_int, c_ptr, weno_sb_grid, weno_sb_face_coefs
            type(weno_sb_grid), intent(in) :: g
            integer(c_int), value :: dir, order, flags, dtype
            type(c_ptr), value :: v_in
            type(weno_sb_face_coefs), intent(in) :: face
            type(c_ptr), value :: vL, vR, stream
        end function weno_sb_weno_uniform_dev

        !> coefs (c_loc of a weno_sb_coefs) or face (c_loc of a
        !! weno_sb_face_coefs): pass exactly one, the other c_null_ptr
        integer(c_int) function weno_sb_vjp_dev(g, dir, order, flags, v_in, coefs, face, gL, gR, gv, stream) &
            bind(C, name='weno_sb_vjp_dev')
            import :: c_int, c_ptr, weno_sb_grid
            type(weno_sb_grid), intent(in) :: g
            integer(c_int), value :: dir, order, flags
            type(c_ptr), value :: v_in, coefs, face, gL, gR, gv, stream
        end function weno_sb_vjp_dev

        integer(c_int) function weno_sb_preserve_monotonicity_dev(g, dir, dtype, v_rs_ws, vL, vR, stream) &
            bind(C, name='weno_sb_preserve_monotonicity_dev')
            import :: c_int, c_ptr, weno_sb_grid
            type(weno_sb_grid), intent(in) :: g
            integer(c_int), value :: dir, dtype
            type(c_ptr), value :: v_rs_ws, vL, vR, stream
        end function weno_sb_preserve_monotonicity_dev

        integer(c_size_t) function weno_sb_checksum_scratch_bytes(n) bind(C, name='weno_sb_checksum_scratch_bytes')
            import :: c_size_t, c_int64_t
            integer(c_int64_t), value :: n
        end function weno_sb_checksum_scratch_bytes

        integer(c_int) function weno_sb_checksum_dev(dtype, arr, n, scratch, d_result, stream) &
            bind(C, name='weno_sb_checksum_dev')
            import :: c_int, c_int64_t, c_ptr
            integer(c_int), value :: dtype
            type(c_ptr), value :: arr
            integer(c_int64_t), value :: n
            type(c_ptr), value :: scratch, d_result, stream
        end function weno_sb_checksum_dev

        !> f_checksum of up to 16 device arrays without any allocation:
        !! for drivers whose device heap belongs to the offload runtime
        integer(c_int) function weno_sb_checksum_noalloc(dtype, arrays, n, count, d_results, stream) &
            bind(C, name='weno_sb_checksum_noalloc')
            import :: c_int, c_int64_t, c_ptr
            integer(c_int), value :: dtype
            type(c_ptr), intent(in) :: arrays(*)
            integer(c_int64_t), intent(in) :: n(*)
            integer(c_int), value :: count
            type(c_ptr), value :: d_results, stream
        end function weno_sb_checksum_noalloc

        !> WENO-JS coefficients of order 3/5/7 for any cell widths (MFC's
        !! s_compute_weno_coefficients): x_cb(1:ns+1) the cell boundaries
        !! along the sweep; host arrays in the harness layouts, NC = ns - 6
        integer(c_int) function weno_sb_coefficients(order, ns, x_cb, polyL, polyR, dL, dR, beta_coef) &
            bind(C, name='weno_sb_coefficients')
            import :: c_int, c_int64_t, c_double
            integer(c_int), value :: order
            integer(c_int64_t), value :: ns
            real(c_double), intent(in) :: x_cb(*)
            real(c_double), intent(out) :: polyL(*), polyR(*), dL(*), dR(*), beta_coef(*)
        end function weno_sb_coefficients

        ! ---- batches of uneven blocks (one CUDA graph launch of all the blocks' sweeps;
        !      configure mode 0 persistent kernel, 1 graph of per-block sweeps,
        !      2 grouped marching sweeps with cols_per_item = faces per work item)

        integer(c_int) function weno_sb_batch_create(blocks, n, batch) bind(C, name='weno_sb_batch_create')
            import :: c_int, weno_sb_block
            type(weno_sb_block), intent(in) :: blocks(*)
            integer(c_int), value :: n
            integer(c_int), intent(out) :: batch
        end function weno_sb_batch_create

        integer(c_int) function weno_sb_batch_autotune(batch, stream, threads, cols_per_item, best_ms) &
            bind(C, name='weno_sb_batch_autotune')
            import :: c_int, c_ptr, c_double
            integer(c_int), value :: batch
            type(c_ptr), value :: stream
            integer(c_int), intent(out) :: threads, cols_per_item
            real(c_double), intent(out) :: best_ms
        end function weno_sb_batch_autotune

        integer(c_int) function weno_sb_batch_launch(batch, stream) bind(C, name='weno_sb_batch_launch')
            import :: c_int, c_ptr
            integer(c_int), value :: batch
            type(c_ptr), value :: stream
        end function weno_sb_batch_launch

        integer(c_int) function weno_sb_batch_configure(batch, mode, threads, cols_per_item, branches) &
            bind(C, name='weno_sb_batch_configure')
            import :: c_int
            integer(c_int), value :: batch, mode, threads, cols_per_item, branches
        end function weno_sb_batch_configure

        integer(c_int) function weno_sb_batch_query(batch, mode, threads, cols_per_item, branches) &
            bind(C, name='weno_sb_batch_query')
            import :: c_int
            integer(c_int), value :: batch
            integer(c_int), intent(out) :: mode, threads, cols_per_item, branches
        end function weno_sb_batch_query

        integer(c_int) function weno_sb_batch_destroy(batch) bind(C, name='weno_sb_batch_destroy')
            import :: c_int
            integer(c_int), value :: batch
        end function weno_sb_batch_destroy
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

    !> Adjoint of one sweep (no reference counterpart): gv = (dF/dv)^T (gL, gR)
    !! for the reconstruction of `order` (+ MP when mp), reading v_rs_ws_dir;
    !! gL, gR, gv are device addresses (c_loc under use_device_ptr).  With
    !! accumulate, gv is added to instead of overwritten.
    subroutine s_weno_vjp(dir, order, mp, accumulate, gL, gR, gv)
        integer, intent(in) :: dir, order
        logical, intent(in) :: mp, accumulate
        type(c_ptr), intent(in) :: gL, gR, gv
        integer(c_int) :: fl
        fl = 0_c_int
        if (mp) fl = ior(fl, WENO_SB_F_MP)
        if (accumulate) fl = ior(fl, WENO_SB_F_ACCUMULATE)
        call s_weno_sb_check(weno_sb_vjp(weno_sb_handle, int(dir, c_int), int(order, c_int), fl, gL, gR, gv), &
                             's_weno_vjp')
    end subroutine s_weno_vjp

end module m_weno_sb
