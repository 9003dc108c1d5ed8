!+---------------------------------------------------------------------+
!| ISO_C_BINDING interface to libastr_b200.so (include/astr_b200.h),    |
!| so that ASTR's Fortran solver and its miniapps call the B200 path in |
!| place of fd_scheme_initiate / fds%central / compact_filter /         |
!| rhscal / rk3.                                                        |
!+---------------------------------------------------------------------+
module astr_b200
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: ASTR_OK = 0, ASTR_HOST = 0, ASTR_DEVICE = 1

  type, bind(C) :: astr_params
    integer(c_int) :: im, jm, km
    real(c_double) :: mach, reynolds, prandtl, gamma, ref_tem, sutherland
    real(c_double) :: alfa_filter, beta_halo, beta_bound
    integer(c_int) :: filter_on
  end type astr_params

  interface
    integer(c_int) function astr_init(device, ctx) bind(C, name="astr_init")
      import :: c_int, c_ptr
      integer(c_int), value :: device
      type(c_ptr) :: ctx
    end function
    integer(c_int) function astr_destroy(ctx) bind(C, name="astr_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    type(c_ptr) function astr_last_error(ctx) bind(C, name="astr_last_error")
      import :: c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function astr_fd_scheme_create(ctx, scheme, ntype, dim, s) bind(C, name="astr_fd_scheme_create")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: ctx
      character(kind=c_char) :: scheme(4)
      integer(c_int), value :: ntype, dim
      type(c_ptr) :: s
    end function
    integer(c_int) function astr_filter_create(ctx, ntype, dim, alpha_f, beta_halo, beta_bound, no_filter, s) &
        bind(C, name="astr_filter_create")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: ntype, dim, no_filter
      real(c_double), value :: alpha_f, beta_halo, beta_bound
      type(c_ptr) :: s
    end function
    integer(c_int) function astr_deriv_lines(ctx, s, dir, f, fshape, flb, df, dshape, dlb, nfields, scale, where) &
        bind(C, name="astr_deriv_lines")
      import :: c_int, c_ptr, c_double, c_int64_t
      type(c_ptr), value :: ctx, s, f, df
      integer(c_int), value :: dir, nfields, where
      integer(c_int64_t) :: fshape(3), flb(3), dshape(3), dlb(3)
      real(c_double), value :: scale
    end function
    integer(c_int) function astr_filter_lines(ctx, s, dir, f, fshape, flb, ff, oshape, olb, nfields, where) &
        bind(C, name="astr_filter_lines")
      import :: c_int, c_ptr, c_int64_t
      type(c_ptr), value :: ctx, s, f, ff
      integer(c_int), value :: dir, nfields, where
      integer(c_int64_t) :: fshape(3), flb(3), oshape(3), olb(3)
    end function
    integer(c_int) function astr_state_create(ctx, p, st) bind(C, name="astr_state_create")
      import :: c_int, c_ptr, astr_params
      type(c_ptr), value :: ctx
      type(astr_params) :: p
      type(c_ptr) :: st
    end function
    integer(c_int) function astr_state_upload(st, q, shape, lb, where) bind(C, name="astr_state_upload")
      import :: c_int, c_ptr, c_int64_t
      type(c_ptr), value :: st, q
      integer(c_int64_t) :: shape(3), lb(3)
      integer(c_int), value :: where
    end function
    integer(c_int) function astr_state_download(st, q, shape, lb, where) bind(C, name="astr_state_download")
      import :: c_int, c_ptr, c_int64_t
      type(c_ptr), value :: st, q
      integer(c_int64_t) :: shape(3), lb(3)
      integer(c_int), value :: where
    end function
    integer(c_int) function astr_rhs(st, qrhs, shape, lb, where) bind(C, name="astr_rhs")
      import :: c_int, c_ptr, c_int64_t
      type(c_ptr), value :: st, qrhs
      integer(c_int64_t) :: shape(3), lb(3)
      integer(c_int), value :: where
    end function
    integer(c_int) function astr_rk3_step(st, dt, nsteps) bind(C, name="astr_rk3_step")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: st
      real(c_double), value :: dt
      integer(c_int), value :: nsteps
    end function
    integer(c_int) function astr_history(st, rows, maxrows, nrows) bind(C, name="astr_history")
      import :: c_int, c_ptr
      type(c_ptr), value :: st, rows
      integer(c_int), value :: maxrows
      integer(c_int) :: nrows
    end function
  end interface

contains

  ! df(0:dim) = fds%central(asolver, f, dim) for every line of f(-hm:,..,..) along dir (1..3):
  ! the drop-in for the line loops of gradcal/convection/diffusion.
  subroutine astr_central3d(ctx, scheme, dir, f, df, scale)
    type(c_ptr), intent(in) :: ctx, scheme
    integer, intent(in) :: dir
    real(8), intent(in), target, contiguous :: f(:,:,:)
    real(8), intent(inout), target, contiguous :: df(:,:,:)
    real(8), intent(in) :: scale
    integer(c_int64_t) :: fs(3), fl(3), ds(3), dl(3)
    integer(c_int) :: rc
    fs = shape(f, kind=c_int64_t); ds = shape(df, kind=c_int64_t)
    fl = 0; dl = 0
    fl(dir) = -5                         ! f(-hm:dim+hm) along the line, hm = 5
    rc = astr_deriv_lines(ctx, scheme, dir - 1, c_loc(f), fs, fl, c_loc(df), ds, dl, 1_c_int, scale, ASTR_HOST)
    if (rc /= ASTR_OK) stop ' !! astr_deriv_lines failed'
  end subroutine astr_central3d

end module astr_b200
