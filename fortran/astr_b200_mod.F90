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
    integer(c_int) :: ntype(3)
    real(c_double) :: twall
    integer(c_int) :: conschm
    real(c_double) :: bfacmpld
    integer(c_int) :: lchardecomp
    real(c_double) :: shkcrt
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
    integer(c_int) function astr_flux_create(ctx, scheme, ntype, dim, wind, bfac, s) bind(C, name="astr_flux_create")
      import :: c_int, c_ptr, c_char, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: scheme, ntype, dim
      character(kind=c_char), value :: wind
      real(c_double), value :: bfac
      type(c_ptr) :: s
    end function
    integer(c_int) function astr_flux_lines(ctx, s, dir, f, fshape, flb, fh, oshape, olb, nfields, where) &
        bind(C, name="astr_flux_lines")
      import :: c_int, c_ptr, c_int64_t
      type(c_ptr), value :: ctx, s, f, fh
      integer(c_int), value :: dir, nfields, where
      integer(c_int64_t) :: fshape(3), flb(3), oshape(3), olb(3)
    end function
    integer(c_int) function astr_flux_diff_lines(ctx, s, dir, f, fshape, flb, df, oshape, olb, nfields, scale, &
        accumulate, where) bind(C, name="astr_flux_diff_lines")
      import :: c_int, c_ptr, c_double, c_int64_t
      type(c_ptr), value :: ctx, s, f, df
      integer(c_int), value :: dir, nfields, accumulate, where
      integer(c_int64_t) :: fshape(3), flb(3), oshape(3), olb(3)
      real(c_double), value :: scale
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
    integer(c_int) function astr_set_stream(ctx, stream) bind(C, name="astr_set_stream")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, stream
    end function
    integer(c_int) function astr_synchronize(ctx) bind(C, name="astr_synchronize")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function astr_scheme_destroy(s) bind(C, name="astr_scheme_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: s
    end function
    integer(c_int) function astr_scheme_ac(s, ac, first_node, last_node) bind(C, name="astr_scheme_ac")
      import :: c_int, c_ptr
      type(c_ptr), value :: s, ac
      integer(c_int) :: first_node, last_node
    end function
    integer(c_int) function astr_state_destroy(st) bind(C, name="astr_state_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: st
    end function
    integer(c_int) function astr_state_init_tgv(st) bind(C, name="astr_state_init_tgv")
      import :: c_int, c_ptr
      type(c_ptr), value :: st
    end function
    integer(c_int) function astr_cfl_dt(st, cfl, dt) bind(C, name="astr_cfl_dt")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: st
      real(c_double), value :: cfl
      real(c_double) :: dt
    end function
    integer(c_int) function astr_rk3_step_host(st, q, shape, lb, dt, nsteps, diag_out) bind(C, name="astr_rk3_step_host")
      import :: c_int, c_ptr, c_double, c_int64_t
      type(c_ptr), value :: st, q
      integer(c_int64_t) :: shape(3), lb(3)
      real(c_double), value :: dt
      integer(c_int), value :: nsteps
      real(c_double) :: diag_out(3)
    end function
    integer(c_int) function astr_diagnostics(st, out) bind(C, name="astr_diagnostics")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: st
      real(c_double) :: out(3)
    end function
    integer(c_int) function astr_state_use_graph(st, on) bind(C, name="astr_state_use_graph")
      import :: c_int, c_ptr
      type(c_ptr), value :: st
      integer(c_int), value :: on
    end function
    integer(c_int) function astr_state_split_filter(st, on) bind(C, name="astr_state_split_filter")
      import :: c_int, c_ptr
      type(c_ptr), value :: st
      integer(c_int), value :: on
    end function
    integer(c_int) function astr_state_autotune(st, on) bind(C, name="astr_state_autotune")
      import :: c_int, c_ptr
      type(c_ptr), value :: st
      integer(c_int), value :: on
    end function
    integer(c_int) function astr_state_launch_shapes(st, shapes) bind(C, name="astr_state_launch_shapes")
      import :: c_int, c_ptr
      type(c_ptr), value :: st
      integer(c_int) :: shapes(42)
    end function
    integer(c_int) function astr_state_set_launch_shape(st, pass, s, wpl, ti, lpw, fps) &
        bind(C, name="astr_state_set_launch_shape")
      import :: c_int, c_ptr
      type(c_ptr), value :: st
      integer(c_int), value :: pass, s, wpl, ti, lpw, fps
    end function
    integer(c_int) function astr_pass_timings(st, dt, nsteps, ms) bind(C, name="astr_pass_timings")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: st
      real(c_double), value :: dt
      integer(c_int), value :: nsteps
      real(c_double) :: ms(8)
    end function
    integer(c_int) function astr_ensemble_create(ctx, boxes, nbox, e) bind(C, name="astr_ensemble_create")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      type(c_ptr) :: boxes(*)
      integer(c_int), value :: nbox
      type(c_ptr) :: e
    end function
    integer(c_int) function astr_ensemble_destroy(e) bind(C, name="astr_ensemble_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: e
    end function
    integer(c_int) function astr_ensemble_step(e, dt, nsteps) bind(C, name="astr_ensemble_step")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: e
      real(c_double) :: dt(*)
      integer(c_int), value :: nsteps
    end function
    integer(c_int) function astr_adjoint_create(st, checkpoint_every, adj) bind(C, name="astr_adjoint_create")
      import :: c_int, c_ptr
      type(c_ptr), value :: st
      integer(c_int), value :: checkpoint_every
      type(c_ptr) :: adj
    end function
    integer(c_int) function astr_adjoint_destroy(adj) bind(C, name="astr_adjoint_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: adj
    end function
    integer(c_int) function astr_adjoint_forward(adj, dt, nsteps, j) bind(C, name="astr_adjoint_forward")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: adj
      real(c_double), value :: dt
      integer(c_int), value :: nsteps
      real(c_double) :: j
    end function
    integer(c_int) function astr_adjoint_backward(adj, grad, shape, lb, where) bind(C, name="astr_adjoint_backward")
      import :: c_int, c_ptr, c_int64_t
      type(c_ptr), value :: adj, grad
      integer(c_int64_t) :: shape(3), lb(3)
      integer(c_int), value :: where
    end function
    integer(c_int) function astr_step_vjp(adj, dt, lam_in, lam_out, shape, lb, where) bind(C, name="astr_step_vjp")
      import :: c_int, c_ptr, c_double, c_int64_t
      type(c_ptr), value :: adj, lam_in, lam_out
      real(c_double), value :: dt
      integer(c_int64_t) :: shape(3), lb(3)
      integer(c_int), value :: where
    end function
    integer(c_int) function astr_scheme_apply_transpose(ctx, s, dir, g, dims, out, nfields, scale) &
        bind(C, name="astr_scheme_apply_transpose")
      import :: c_int, c_ptr, c_double, c_int64_t
      type(c_ptr), value :: ctx, s, g, out
      integer(c_int), value :: dir, nfields
      integer(c_int64_t) :: dims(3)
      real(c_double), value :: scale
    end function
    integer(c_int) function astr_cfl_dt_noalloc(ctx, q, shape, lb, im, jm, km, mach, gamma, cfl, dt) &
        bind(C, name="astr_cfl_dt_noalloc")
      import :: c_int, c_ptr, c_double, c_int64_t
      type(c_ptr), value :: ctx, q
      integer(c_int64_t) :: shape(3), lb(3)
      integer(c_int), value :: im, jm, km
      real(c_double), value :: mach, gamma, cfl
      real(c_double) :: dt
    end function
    integer(c_int) function astr_full_create(ctx, p, fs) bind(C, name="astr_full_create")
      import :: c_int, c_ptr, astr_params
      type(c_ptr), value :: ctx
      type(astr_params) :: p
      type(c_ptr) :: fs
    end function
    integer(c_int) function astr_full_destroy(fs) bind(C, name="astr_full_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: fs
    end function
    integer(c_int) function astr_full_upload(fs, q, shape, lb, where) bind(C, name="astr_full_upload")
      import :: c_int, c_ptr, c_int64_t
      type(c_ptr), value :: fs, q
      integer(c_int64_t) :: shape(3), lb(3)
      integer(c_int), value :: where
    end function
    integer(c_int) function astr_full_download(fs, q, shape, lb, where) bind(C, name="astr_full_download")
      import :: c_int, c_ptr, c_int64_t
      type(c_ptr), value :: fs, q
      integer(c_int64_t) :: shape(3), lb(3)
      integer(c_int), value :: where
    end function
    integer(c_int) function astr_full_step(fs, dt, nsteps) bind(C, name="astr_full_step")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: fs
      real(c_double), value :: dt
      integer(c_int), value :: nsteps
    end function
    integer(c_int) function astr_full_rhs(fs, qrhs, shape, lb, where) bind(C, name="astr_full_rhs")
      import :: c_int, c_ptr, c_int64_t
      type(c_ptr), value :: fs, qrhs
      integer(c_int64_t) :: shape(3), lb(3)
      integer(c_int), value :: where
    end function
    integer(c_int) function astr_full_history(fs, rows, maxrows, nrows) bind(C, name="astr_full_history")
      import :: c_int, c_ptr
      type(c_ptr), value :: fs, rows
      integer(c_int), value :: maxrows
      integer(c_int) :: nrows
    end function

    ! ---- checkpoint files: h5io_init / h5write / h5read / h5io_end (src/hdf5io.F90) without the
    ! HDF5 library; strings are NUL-terminated (trim(name)//c_null_char)
    integer(c_int) function astr_h5io_init(filename, mode, h) bind(C, name="astr_h5io_init")
      import :: c_int, c_ptr, c_char
      character(kind=c_char) :: filename(*), mode(*)
      type(c_ptr) :: h
    end function
    integer(c_int) function astr_h5io_end(h) bind(C, name="astr_h5io_end")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    type(c_ptr) function astr_h5_last_error(h) bind(C, name="astr_h5_last_error")
      import :: c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function astr_h5write_r8(h, varname, rank, dims, var) bind(C, name="astr_h5write_r8")
      import :: c_int, c_ptr, c_char, c_int64_t
      type(c_ptr), value :: h, var
      character(kind=c_char) :: varname(*)
      integer(c_int), value :: rank
      integer(c_int64_t) :: dims(*)
    end function
    integer(c_int) function astr_h5write_i4(h, varname, rank, dims, var) bind(C, name="astr_h5write_i4")
      import :: c_int, c_ptr, c_char, c_int64_t
      type(c_ptr), value :: h, var
      character(kind=c_char) :: varname(*)
      integer(c_int), value :: rank
      integer(c_int64_t) :: dims(*)
    end function
    integer(c_int) function astr_h5read_r8(h, varname, rank, dims, offset, mode, var) bind(C, name="astr_h5read_r8")
      import :: c_int, c_ptr, c_char, c_int64_t
      type(c_ptr), value :: h, offset, var
      character(kind=c_char) :: varname(*)
      integer(c_int), value :: rank
      integer(c_int64_t) :: dims(*)
      character(kind=c_char), value :: mode
    end function
    integer(c_int) function astr_h5read_i4(h, varname, rank, dims, offset, mode, var) bind(C, name="astr_h5read_i4")
      import :: c_int, c_ptr, c_char, c_int64_t
      type(c_ptr), value :: h, offset, var
      character(kind=c_char) :: varname(*)
      integer(c_int), value :: rank
      integer(c_int64_t) :: dims(*)
      character(kind=c_char), value :: mode
    end function
    integer(c_int) function astr_h5_dataset_info(h, varname, rank, dims, type_class, type_size) &
        bind(C, name="astr_h5_dataset_info")
      import :: c_int, c_ptr, c_char, c_int64_t
      type(c_ptr), value :: h
      character(kind=c_char) :: varname(*)
      integer(c_int) :: rank, type_class, type_size
      integer(c_int64_t) :: dims(*)
    end function
    integer(c_int) function astr_h5_count(h, n) bind(C, name="astr_h5_count")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
      integer(c_int) :: n
    end function
    integer(c_int) function astr_h5_name(h, i, name, len) bind(C, name="astr_h5_name")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: h
      integer(c_int), value :: i, len
      character(kind=c_char) :: name(*)
    end function
    ! writeflfed's flow field / readcheckpoint + updateq (src/readwrite.F90:1378-1528, 1720-1979)
    integer(c_int) function astr_state_write_flowfield(st, filename) bind(C, name="astr_state_write_flowfield")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: st
      character(kind=c_char) :: filename(*)
    end function
    integer(c_int) function astr_full_write_flowfield(fs, filename) bind(C, name="astr_full_write_flowfield")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: fs
      character(kind=c_char) :: filename(*)
    end function
    integer(c_int) function astr_state_read_flowfield(st, filename, mode, nstep, time) &
        bind(C, name="astr_state_read_flowfield")
      import :: c_int, c_ptr, c_char, c_double
      type(c_ptr), value :: st
      character(kind=c_char) :: filename(*)
      character(kind=c_char), value :: mode
      integer(c_int) :: nstep
      real(c_double) :: time
    end function
    integer(c_int) function astr_full_read_flowfield(fs, filename, mode, nstep, time) &
        bind(C, name="astr_full_read_flowfield")
      import :: c_int, c_ptr, c_char, c_double
      type(c_ptr), value :: fs
      character(kind=c_char) :: filename(*)
      character(kind=c_char), value :: mode
      integer(c_int) :: nstep
      real(c_double) :: time
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
