! lica_gpu.f90 -- Fortran 2003 ISO_C_BINDING interface to include/lica_gpu.h, written by
! include/make_fortran_module.py from the header (do not edit by hand).  A Fortran solver
! calls the library with `use lica_gpu`; opaque handles are type(c_ptr), device arrays
! are passed as type(c_ptr) device addresses, host arrays by reference.
module lica_gpu
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: LICA_OK = 0
  integer(c_int), parameter :: LICA_NOT_CONVERGED = 1
  integer(c_int), parameter :: LICA_BAND_OVERFLOW = 2
  integer(c_int), parameter :: LICA_NAN = 3
  integer(c_int), parameter :: LICA_BAD_ARG = 4
  integer(c_int), parameter :: LICA_ERR_CUDA = 5
  integer(c_int), parameter :: LICA_ERR_NOMEM = 6
  integer(c_int), parameter :: LICA_ERR_IO = 7
  integer(c_int), parameter :: LICA_STALLED = 8
  integer(c_int), parameter :: LICA_MG_DOWN0 = 0
  integer(c_int), parameter :: LICA_MG_DOWN = 1
  integer(c_int), parameter :: LICA_MG_UP0 = 2
  integer(c_int), parameter :: LICA_MG_UP = 3
  integer(c_int), parameter :: LICA_MG_CTA = 4
  integer(c_int), parameter :: LICA_MG_PUPDATE = 5
  integer(c_int), parameter :: LICA_MG_XUPDATE = 6
  integer(c_int), parameter :: LICA_MG_SETUP = 7
  integer(c_int), parameter :: LICA_MG_NCLASS = 8

  type, bind(c) :: lica_mg_options
    integer(c_int32_t) :: nlevels
    integer(c_int32_t) :: nu1
    integer(c_int32_t) :: nu2
    integer(c_int32_t) :: ncoarse
    integer(c_int32_t) :: precision
    integer(c_int32_t) :: use_graph
    integer(c_int32_t) :: smoother
  end type lica_mg_options

  type, bind(c) :: lica_mg_result
    integer(c_int32_t) :: iterations
    integer(c_int32_t) :: status
    real(c_double) :: rel_residual
  end type lica_mg_result

  type, bind(c) :: lica_lvs_params
    integer(c_int32_t) :: iphs
    integer(c_int32_t) :: first
    integer(c_int32_t) :: m_step
    integer(c_int32_t) :: mglobal
    real(c_double) :: denr
    real(c_double) :: dtconst
  end type lica_lvs_params

  type, bind(c) :: lica_col_props
    real(c_double) :: re
    real(c_double) :: visr
    real(c_double) :: denr
    real(c_double) :: weber
    real(c_double) :: fr
    real(c_double) :: prm
    real(c_double) :: scr
    real(c_double) :: tcr
    real(c_double) :: t_sat
    real(c_double) :: jakob
    real(c_double) :: cflmax
    real(c_double) :: dt0
    integer(c_int32_t) :: iphs
    integer(c_int32_t) :: mglobal
  end type lica_col_props

  type, bind(c) :: lica_col_state
    type(c_ptr) :: w
    type(c_ptr) :: p
    type(c_ptr) :: t
    type(c_ptr) :: psi_cn
    type(c_ptr) :: psi_zn
    type(c_ptr) :: phi
    type(c_ptr) :: layer
    type(c_ptr) :: psif
    type(c_ptr) :: wo
    type(c_ptr) :: mflvs
    type(c_ptr) :: sfgas
    type(c_ptr) :: sfgas2
    type(c_ptr) :: imask
    type(c_ptr) :: scal
    type(c_ptr) :: stats
  end type lica_col_state

  type, bind(c) :: lica_fld_info
    integer(c_int64_t) :: ihist
    integer(c_int64_t) :: m
    real(c_double) :: time
    real(c_double) :: dt
    real(c_double) :: qvol_ori
    integer(c_int32_t) :: ips
    integer(c_int32_t) :: ipx
    integer(c_int32_t) :: ipy
    integer(c_int32_t) :: ipz
    real(c_double) :: pra
    real(c_double) :: denr
    real(c_double) :: visr
    real(c_double) :: fr
    real(c_double) :: surf_j
    real(c_double) :: fk
    real(c_double) :: re_air
    real(c_double) :: prm
    real(c_double) :: scr
    real(c_double) :: tcr
    integer(c_int32_t) :: n_max
    integer(c_int32_t) :: contact
    integer(c_int32_t) :: contact_old
    integer(c_int32_t) :: lvson
    real(c_double) :: vol_tot_ori
    real(c_double) :: contact_start
    real(c_double) :: contact_time
    real(c_double) :: t_con
  end type lica_fld_info

  type, bind(c) :: lica_fld_options
    integer(c_int32_t) :: ireset
    integer(c_int32_t) :: idtold
    integer(c_int32_t) :: ipzero
  end type lica_fld_options

  type, bind(c) :: lica_col_geometry
    type(c_ptr) :: z
    type(c_ptr) :: zp
    type(c_ptr) :: sdz
    type(c_ptr) :: vdz
    type(c_ptr) :: ssdz
    type(c_ptr) :: vvdz
    type(c_ptr) :: kcou1
    type(c_ptr) :: kcou2
    type(c_ptr) :: kcoump1
    type(c_ptr) :: kcoump2
    type(c_ptr) :: kcou_vel
    type(c_ptr) :: kcoump_vel
  end type lica_col_geometry

  type, bind(c) :: lica_film2d_props
    real(c_double) :: re
    real(c_double) :: visr
    real(c_double) :: denr
    real(c_double) :: prm
    real(c_double) :: scr
    real(c_double) :: tcr
    real(c_double) :: jakob
    real(c_double) :: fr
    real(c_double) :: we
    real(c_double) :: rtol
    integer(c_int32_t) :: max_iters
    integer(c_int32_t) :: nreinit
  end type lica_film2d_props

  type, bind(c) :: lica_film2d_stats
    integer(c_int32_t) :: iterations(3)
    integer(c_int32_t) :: status(3)
    real(c_double) :: rel_residual(3)
    real(c_double) :: guess_rel(3)
  end type lica_film2d_stats

  type, bind(c) :: lica_bub_grid
    integer(c_int32_t) :: n1m
    integer(c_int32_t) :: n2m
    integer(c_int32_t) :: n3m
    integer(c_int32_t) :: ipx
    integer(c_int32_t) :: ipy
    integer(c_int32_t) :: ipz
    real(c_double) :: zl
    type(c_ptr) :: sdx
    type(c_ptr) :: sdy
    type(c_ptr) :: sdz
    type(c_ptr) :: xp
    type(c_ptr) :: yp
    type(c_ptr) :: zp
  end type lica_bub_grid

  type, bind(c) :: lica_bub_record
    real(c_double) :: time
    integer(c_int64_t) :: llvs
    real(c_double) :: col(9)
    real(c_double) :: vel(3)
    real(c_double) :: vol
    real(c_double) :: ami(3)
    integer(c_int64_t) :: iz_periodic
  end type lica_bub_record

  interface
    type(c_ptr) function lica_last_error() bind(c, name="lica_last_error")
      import
    end function lica_last_error

    integer(c_int64_t) function lica_kernel_launch_count() &
        bind(c, name="lica_kernel_launch_count")
      import
    end function lica_kernel_launch_count

    integer(c_int) function lica_debug_poison_shared(value, stream) &
        bind(c, name="lica_debug_poison_shared")
      import
      real(c_double), value :: value
      type(c_ptr), value :: stream
    end function lica_debug_poison_shared

    integer(c_int) function lica_gpu_trdiag3(A, B, C, R, UU, l1, l2, ll1, ll2, ld) &
        bind(c, name="lica_gpu_trdiag3")
      import
      real(c_double), intent(in) :: A(*)
      real(c_double), intent(in) :: B(*)
      real(c_double), intent(in) :: C(*)
      real(c_double), intent(inout) :: R(*)
      real(c_double), intent(inout) :: UU(*)
      integer(c_int64_t), value :: l1
      integer(c_int64_t), value :: l2
      integer(c_int64_t), value :: ll1
      integer(c_int64_t), value :: ll2
      integer(c_int64_t), value :: ld
    end function lica_gpu_trdiag3

    integer(c_int) function lica_gpu_trdiag3p(A, B, C, F, j1, j2, l1, l2, ld) &
        bind(c, name="lica_gpu_trdiag3p")
      import
      real(c_double), intent(in) :: A(*)
      real(c_double), intent(in) :: B(*)
      real(c_double), intent(in) :: C(*)
      real(c_double), intent(inout) :: F(*)
      integer(c_int64_t), value :: j1
      integer(c_int64_t), value :: j2
      integer(c_int64_t), value :: l1
      integer(c_int64_t), value :: l2
      integer(c_int64_t), value :: ld
    end function lica_gpu_trdiag3p

    integer(c_int) function lica_gpu_trdiag3_device(A, B, C, R, UU, l1, l2, ll1, ll2, ld, &
        stream) bind(c, name="lica_gpu_trdiag3_device")
      import
      type(c_ptr), value :: A
      type(c_ptr), value :: B
      type(c_ptr), value :: C
      type(c_ptr), value :: R
      type(c_ptr), value :: UU
      integer(c_int64_t), value :: l1
      integer(c_int64_t), value :: l2
      integer(c_int64_t), value :: ll1
      integer(c_int64_t), value :: ll2
      integer(c_int64_t), value :: ld
      type(c_ptr), value :: stream
    end function lica_gpu_trdiag3_device

    integer(c_int) function lica_gpu_trdiag3p_device(A, B, C, F, j1, j2, l1, l2, ld, stream) &
        bind(c, name="lica_gpu_trdiag3p_device")
      import
      type(c_ptr), value :: A
      type(c_ptr), value :: B
      type(c_ptr), value :: C
      type(c_ptr), value :: F
      integer(c_int64_t), value :: j1
      integer(c_int64_t), value :: j2
      integer(c_int64_t), value :: l1
      integer(c_int64_t), value :: l2
      integer(c_int64_t), value :: ld
      type(c_ptr), value :: stream
    end function lica_gpu_trdiag3p_device

    integer(c_int) function lica_gpu_trdiag3_noalloc_device(A, B, C, R, UU, l1, l2, ll1, ll2, &
        ld, stream) bind(c, name="lica_gpu_trdiag3_noalloc_device")
      import
      type(c_ptr), value :: A
      type(c_ptr), value :: B
      type(c_ptr), value :: C
      type(c_ptr), value :: R
      type(c_ptr), value :: UU
      integer(c_int64_t), value :: l1
      integer(c_int64_t), value :: l2
      integer(c_int64_t), value :: ll1
      integer(c_int64_t), value :: ll2
      integer(c_int64_t), value :: ld
      type(c_ptr), value :: stream
    end function lica_gpu_trdiag3_noalloc_device

    integer(c_int) function lica_gpu_poisson(m1, m2, m3, n1m, n2m, n3m, vvdz, ssdz, fixkl, kpv, &
        p, divgsum, denf_zi) bind(c, name="lica_gpu_poisson")
      import
      integer(c_int64_t), value :: m1
      integer(c_int64_t), value :: m2
      integer(c_int64_t), value :: m3
      integer(c_int64_t), value :: n1m
      integer(c_int64_t), value :: n2m
      integer(c_int64_t), value :: n3m
      real(c_double), intent(in) :: vvdz(*)
      real(c_double), intent(in) :: ssdz(*)
      real(c_double), intent(in) :: fixkl(*)
      integer(c_int64_t), intent(in) :: kpv(*)
      real(c_double), intent(inout) :: p(*)
      real(c_double), intent(in) :: divgsum(*)
      real(c_double), intent(in) :: denf_zi(*)
    end function lica_gpu_poisson

    integer(c_int) function lica_mg_create(out, nx, ny, hx, hy, opt) &
        bind(c, name="lica_mg_create")
      import
      type(c_ptr), intent(out) :: out
      integer(c_int32_t), value :: nx
      integer(c_int32_t), value :: ny
      real(c_double), value :: hx
      real(c_double), value :: hy
      type(lica_mg_options), intent(in) :: opt
    end function lica_mg_create

    integer(c_int) function lica_mg_destroy(mg) bind(c, name="lica_mg_destroy")
      import
      type(c_ptr), value :: mg
    end function lica_mg_destroy

    integer(c_int) function lica_mg_solve_device(mg, p, f, bx, by, rtol, max_iters, res, stream) &
        bind(c, name="lica_mg_solve_device")
      import
      type(c_ptr), value :: mg
      type(c_ptr), value :: p
      type(c_ptr), value :: f
      type(c_ptr), value :: bx
      type(c_ptr), value :: by
      real(c_double), value :: rtol
      integer(c_int32_t), value :: max_iters
      type(lica_mg_result), intent(inout) :: res
      type(c_ptr), value :: stream
    end function lica_mg_solve_device

    integer(c_int) function lica_mg_solve_host(mg, p, f, bx, by, rtol, max_iters, res, stream) &
        bind(c, name="lica_mg_solve_host")
      import
      type(c_ptr), value :: mg
      real(c_double), intent(inout) :: p(*)
      real(c_double), intent(in) :: f(*)
      real(c_double), intent(in) :: bx(*)
      real(c_double), intent(in) :: by(*)
      real(c_double), value :: rtol
      integer(c_int32_t), value :: max_iters
      type(lica_mg_result), intent(inout) :: res
      type(c_ptr), value :: stream
    end function lica_mg_solve_host

    integer(c_int) function lica_mg_solve_host_batch(mg, count, p, f, bx, by, rtol, max_iters, &
        res) bind(c, name="lica_mg_solve_host_batch")
      import
      type(c_ptr), value :: mg
      integer(c_int32_t), value :: count
      type(c_ptr), intent(in) :: p(*)
      type(c_ptr), intent(in) :: f(*)
      type(c_ptr), intent(in) :: bx(*)
      type(c_ptr), intent(in) :: by(*)
      real(c_double), value :: rtol
      integer(c_int32_t), value :: max_iters
      type(lica_mg_result), intent(inout) :: res(*)
    end function lica_mg_solve_host_batch

    integer(c_int) function lica_mg_precond_device(mg, z, r, bx, by, stream) &
        bind(c, name="lica_mg_precond_device")
      import
      type(c_ptr), value :: mg
      type(c_ptr), value :: z
      type(c_ptr), value :: r
      type(c_ptr), value :: bx
      type(c_ptr), value :: by
      type(c_ptr), value :: stream
    end function lica_mg_precond_device

    integer(c_int) function lica_mg_apply_device(mg, out, u, bx, by, stream) &
        bind(c, name="lica_mg_apply_device")
      import
      type(c_ptr), value :: mg
      type(c_ptr), value :: out
      type(c_ptr), value :: u
      type(c_ptr), value :: bx
      type(c_ptr), value :: by
      type(c_ptr), value :: stream
    end function lica_mg_apply_device

    integer(c_int) function lica_mg_profile(mg, enable) bind(c, name="lica_mg_profile")
      import
      type(c_ptr), value :: mg
      integer(c_int32_t), value :: enable
    end function lica_mg_profile

    integer(c_int) function lica_mg_profile_read(mg, kernel_class, total_ms, launches) &
        bind(c, name="lica_mg_profile_read")
      import
      type(c_ptr), value :: mg
      integer(c_int32_t), value :: kernel_class
      real(c_double), intent(out) :: total_ms
      integer(c_int64_t), intent(out) :: launches
    end function lica_mg_profile_read

    integer(c_int) function lica_gpu_lvs_transport(ncol, n, length, phi, layer, psif, wo, w, &
        mflvs, vol_tot_ori, vol_tot_iphs, psi_cn, psi_zn, status, stats, prm) &
        bind(c, name="lica_gpu_lvs_transport")
      import
      integer(c_int32_t), value :: ncol
      integer(c_int32_t), value :: n
      real(c_double), value :: length
      real(c_double), intent(inout) :: phi(*)
      integer(c_int32_t), intent(inout) :: layer(*)
      real(c_double), intent(inout) :: psif(*)
      real(c_double), intent(inout) :: wo(*)
      real(c_double), intent(in) :: w(*)
      real(c_double), intent(in) :: mflvs(*)
      real(c_double), intent(inout) :: vol_tot_ori(*)
      real(c_double), intent(in) :: vol_tot_iphs(*)
      real(c_double), intent(inout) :: psi_cn(*)
      real(c_double), intent(inout) :: psi_zn(*)
      integer(c_int32_t), intent(inout) :: status(*)
      real(c_double), intent(inout) :: stats(*)
      type(lica_lvs_params), intent(in) :: prm
    end function lica_gpu_lvs_transport

    integer(c_int) function lica_gpu_column_init(n, length, z0, props, st) &
        bind(c, name="lica_gpu_column_init")
      import
      integer(c_int32_t), value :: n
      real(c_double), value :: length
      real(c_double), value :: z0
      type(lica_col_props), intent(in) :: props
      type(lica_col_state), intent(inout) :: st
    end function lica_gpu_column_init

    integer(c_int) function lica_grid_section(iopt, xyzi, xyzf, ngi, ngf, fac1, fac2, xyz) &
        bind(c, name="lica_grid_section")
      import
      integer(c_int32_t), value :: iopt
      real(c_double), value :: xyzi
      real(c_double), value :: xyzf
      integer(c_int32_t), value :: ngi
      integer(c_int32_t), value :: ngf
      real(c_double), value :: fac1
      real(c_double), value :: fac2
      real(c_double), intent(inout) :: xyz(*)
    end function lica_grid_section

    integer(c_int) function lica_grid_metrics(n, z, sdz, vdz, ssdz, vvdz, zp) &
        bind(c, name="lica_grid_metrics")
      import
      integer(c_int32_t), value :: n
      real(c_double), intent(in) :: z(*)
      real(c_double), intent(inout) :: sdz(*)
      real(c_double), intent(inout) :: vdz(*)
      real(c_double), intent(inout) :: ssdz(*)
      real(c_double), intent(inout) :: vvdz(*)
      real(c_double), intent(inout) :: zp(*)
    end function lica_grid_metrics

    integer(c_int) function lica_grid_coupling_z(n3, z, n3f, zf, kcou1, kcou2, kcoump1, &
        kcoump2, kcou_vel, kcoump_vel) bind(c, name="lica_grid_coupling_z")
      import
      integer(c_int32_t), value :: n3
      real(c_double), intent(in) :: z(*)
      integer(c_int32_t), value :: n3f
      real(c_double), intent(in) :: zf(*)
      integer(c_int32_t), intent(inout) :: kcou1(*)
      integer(c_int32_t), intent(inout) :: kcou2(*)
      integer(c_int32_t), intent(inout) :: kcoump1(*)
      integer(c_int32_t), intent(inout) :: kcoump2(*)
      integer(c_int32_t), intent(inout) :: kcou_vel(*)
      integer(c_int32_t), intent(inout) :: kcoump_vel(*)
    end function lica_grid_coupling_z

    integer(c_int) function lica_mg_stretched_system(nx, ny, yface, bx, by, f, bx_out, by_out, &
        f_out) bind(c, name="lica_mg_stretched_system")
      import
      integer(c_int32_t), value :: nx
      integer(c_int32_t), value :: ny
      real(c_double), intent(in) :: yface(*)
      real(c_double), intent(in) :: bx(*)
      real(c_double), intent(in) :: by(*)
      real(c_double), intent(in) :: f(*)
      real(c_double), intent(inout) :: bx_out(*)
      real(c_double), intent(inout) :: by_out(*)
      real(c_double), intent(inout) :: f_out(*)
    end function lica_mg_stretched_system

    integer(c_int) function lica_fld_name(ihist, out, cap) bind(c, name="lica_fld_name")
      import
      integer(c_int64_t), value :: ihist
      character(kind=c_char), intent(inout) :: out(*)
      integer(c_int32_t), value :: cap
    end function lica_fld_name

    integer(c_int) function lica_col_fld_write(path, n, props, st, info) &
        bind(c, name="lica_col_fld_write")
      import
      character(kind=c_char), intent(in) :: path(*)
      integer(c_int32_t), value :: n
      type(lica_col_props), intent(in) :: props
      type(lica_col_state), intent(in) :: st
      type(lica_fld_info), intent(in) :: info
    end function lica_col_fld_write

    integer(c_int) function lica_col_fld_dims(path, n) bind(c, name="lica_col_fld_dims")
      import
      character(kind=c_char), intent(in) :: path(*)
      integer(c_int32_t), intent(out) :: n
    end function lica_col_fld_dims

    integer(c_int) function lica_col_fld_read(path, n, length, props, opt, st, info) &
        bind(c, name="lica_col_fld_read")
      import
      character(kind=c_char), intent(in) :: path(*)
      integer(c_int32_t), value :: n
      real(c_double), value :: length
      type(lica_col_props), intent(in) :: props
      type(lica_fld_options), intent(in) :: opt
      type(lica_col_state), intent(inout) :: st
      type(lica_fld_info), intent(inout) :: info
    end function lica_col_fld_read

    integer(c_size_t) function lica_gpu_column_scratch_bytes(ncol, n) &
        bind(c, name="lica_gpu_column_scratch_bytes")
      import
      integer(c_int32_t), value :: ncol
      integer(c_int32_t), value :: n
    end function lica_gpu_column_scratch_bytes

    integer(c_int) function lica_gpu_column_steps_device(ncol, n, length, props, st, nsteps, &
        threads, scratch, status, stream) bind(c, name="lica_gpu_column_steps_device")
      import
      integer(c_int32_t), value :: ncol
      integer(c_int32_t), value :: n
      real(c_double), value :: length
      type(lica_col_props), intent(in) :: props
      type(lica_col_state), intent(in) :: st
      integer(c_int32_t), value :: nsteps
      integer(c_int32_t), value :: threads
      type(c_ptr), value :: scratch
      type(c_ptr), value :: status
      type(c_ptr), value :: stream
    end function lica_gpu_column_steps_device

    integer(c_int) function lica_gpu_column_profile_device(prof) &
        bind(c, name="lica_gpu_column_profile_device")
      import
      type(c_ptr), value :: prof
    end function lica_gpu_column_profile_device

    integer(c_int) function lica_gpu_column_history_device(hist, capacity) &
        bind(c, name="lica_gpu_column_history_device")
      import
      type(c_ptr), value :: hist
      integer(c_int32_t), value :: capacity
    end function lica_gpu_column_history_device

    integer(c_int) function lica_gpu_column_batch_create(out, ncol, n, length, props) &
        bind(c, name="lica_gpu_column_batch_create")
      import
      type(c_ptr), intent(out) :: out
      integer(c_int32_t), value :: ncol
      integer(c_int32_t), intent(in) :: n(*)
      real(c_double), intent(in) :: length(*)
      type(lica_col_props), intent(in) :: props(*)
    end function lica_gpu_column_batch_create

    integer(c_int) function lica_gpu_column_batch_destroy(batch) &
        bind(c, name="lica_gpu_column_batch_destroy")
      import
      type(c_ptr), value :: batch
    end function lica_gpu_column_batch_destroy

    integer(c_int) function lica_gpu_column_batch_layout(batch, offsets, totals) &
        bind(c, name="lica_gpu_column_batch_layout")
      import
      type(c_ptr), value :: batch
      integer(c_int64_t), intent(inout) :: offsets(*)
      integer(c_int64_t), intent(inout) :: totals(*)
    end function lica_gpu_column_batch_layout

    integer(c_int) function lica_gpu_column_batch_steps_device(batch, st, nsteps, threads, &
        scratch, status, stream) bind(c, name="lica_gpu_column_batch_steps_device")
      import
      type(c_ptr), value :: batch
      type(lica_col_state), intent(in) :: st
      integer(c_int32_t), value :: nsteps
      integer(c_int32_t), value :: threads
      type(c_ptr), value :: scratch
      type(c_ptr), value :: status
      type(c_ptr), value :: stream
    end function lica_gpu_column_batch_steps_device

    integer(c_int) function lica_gpu_column_batch_steps_ex_device(batch, st, nsteps, threads, &
        tri_cap, scratch, status, stream) bind(c, name="lica_gpu_column_batch_steps_ex_device")
      import
      type(c_ptr), value :: batch
      type(lica_col_state), intent(in) :: st
      integer(c_int32_t), value :: nsteps
      integer(c_int32_t), value :: threads
      integer(c_int32_t), value :: tri_cap
      type(c_ptr), value :: scratch
      type(c_ptr), value :: status
      type(c_ptr), value :: stream
    end function lica_gpu_column_batch_steps_ex_device

    integer(c_int) function lica_gpu_column_steps(ncol, n, length, props, st, nsteps, status) &
        bind(c, name="lica_gpu_column_steps")
      import
      integer(c_int32_t), value :: ncol
      integer(c_int32_t), value :: n
      real(c_double), value :: length
      type(lica_col_props), intent(in) :: props
      type(lica_col_state), intent(inout) :: st
      integer(c_int32_t), value :: nsteps
      integer(c_int32_t), intent(inout) :: status(*)
    end function lica_gpu_column_steps

    integer(c_int) function lica_gpu_column_init_geometry(n, length, z0, props, geo, st) &
        bind(c, name="lica_gpu_column_init_geometry")
      import
      integer(c_int32_t), value :: n
      real(c_double), value :: length
      real(c_double), value :: z0
      type(lica_col_props), intent(in) :: props
      type(lica_col_geometry), intent(in) :: geo
      type(lica_col_state), intent(inout) :: st
    end function lica_gpu_column_init_geometry

    integer(c_int) function lica_gpu_column_geometry_create(out, n, length, geo) &
        bind(c, name="lica_gpu_column_geometry_create")
      import
      type(c_ptr), intent(out) :: out
      integer(c_int32_t), value :: n
      real(c_double), value :: length
      type(lica_col_geometry), intent(in) :: geo
    end function lica_gpu_column_geometry_create

    integer(c_int) function lica_gpu_column_geometry_destroy(geo) &
        bind(c, name="lica_gpu_column_geometry_destroy")
      import
      type(c_ptr), value :: geo
    end function lica_gpu_column_geometry_destroy

    integer(c_int) function lica_gpu_column_steps_geometry_device(geo, ncol, props, st, nsteps, &
        threads, scratch, status, stream) bind(c, name="lica_gpu_column_steps_geometry_device")
      import
      type(c_ptr), value :: geo
      integer(c_int32_t), value :: ncol
      type(lica_col_props), intent(in) :: props
      type(lica_col_state), intent(in) :: st
      integer(c_int32_t), value :: nsteps
      integer(c_int32_t), value :: threads
      type(c_ptr), value :: scratch
      type(c_ptr), value :: status
      type(c_ptr), value :: stream
    end function lica_gpu_column_steps_geometry_device

    integer(c_int) function lica_gpu_column_steps_geometry(geo, ncol, props, st, nsteps, status) &
        bind(c, name="lica_gpu_column_steps_geometry")
      import
      type(c_ptr), value :: geo
      integer(c_int32_t), value :: ncol
      type(lica_col_props), intent(in) :: props
      type(lica_col_state), intent(inout) :: st
      integer(c_int32_t), value :: nsteps
      integer(c_int32_t), intent(inout) :: status(*)
    end function lica_gpu_column_steps_geometry

    integer(c_int) function lica_gpu_lvs_transport_geometry_device(geo, ncol, phi, layer, psif, &
        wo, w, mflvs, vol_tot_ori, vol_tot_iphs, psi_cn, psi_zn, status, stats, prm, stream) &
        bind(c, name="lica_gpu_lvs_transport_geometry_device")
      import
      type(c_ptr), value :: geo
      integer(c_int32_t), value :: ncol
      type(c_ptr), value :: phi
      type(c_ptr), value :: layer
      type(c_ptr), value :: psif
      type(c_ptr), value :: wo
      type(c_ptr), value :: w
      type(c_ptr), value :: mflvs
      type(c_ptr), value :: vol_tot_ori
      type(c_ptr), value :: vol_tot_iphs
      type(c_ptr), value :: psi_cn
      type(c_ptr), value :: psi_zn
      type(c_ptr), value :: status
      type(c_ptr), value :: stats
      type(lica_lvs_params), intent(in) :: prm
      type(c_ptr), value :: stream
    end function lica_gpu_lvs_transport_geometry_device

    integer(c_int) function lica_gpu_lvs_transport_geometry(geo, ncol, phi, layer, psif, wo, w, &
        mflvs, vol_tot_ori, vol_tot_iphs, psi_cn, psi_zn, status, stats, prm) &
        bind(c, name="lica_gpu_lvs_transport_geometry")
      import
      type(c_ptr), value :: geo
      integer(c_int32_t), value :: ncol
      real(c_double), intent(inout) :: phi(*)
      integer(c_int32_t), intent(inout) :: layer(*)
      real(c_double), intent(inout) :: psif(*)
      real(c_double), intent(inout) :: wo(*)
      real(c_double), intent(in) :: w(*)
      real(c_double), intent(in) :: mflvs(*)
      real(c_double), intent(inout) :: vol_tot_ori(*)
      real(c_double), intent(in) :: vol_tot_iphs(*)
      real(c_double), intent(inout) :: psi_cn(*)
      real(c_double), intent(inout) :: psi_zn(*)
      integer(c_int32_t), intent(inout) :: status(*)
      real(c_double), intent(inout) :: stats(*)
      type(lica_lvs_params), intent(in) :: prm
    end function lica_gpu_lvs_transport_geometry

    integer(c_int) function lica_gpu_lvs_transport_device(ncol, n, length, phi, layer, psif, &
        wo, w, mflvs, vol_tot_ori, vol_tot_iphs, psi_cn, psi_zn, status, stats, prm, stream) &
        bind(c, name="lica_gpu_lvs_transport_device")
      import
      integer(c_int32_t), value :: ncol
      integer(c_int32_t), value :: n
      real(c_double), value :: length
      type(c_ptr), value :: phi
      type(c_ptr), value :: layer
      type(c_ptr), value :: psif
      type(c_ptr), value :: wo
      type(c_ptr), value :: w
      type(c_ptr), value :: mflvs
      type(c_ptr), value :: vol_tot_ori
      type(c_ptr), value :: vol_tot_iphs
      type(c_ptr), value :: psi_cn
      type(c_ptr), value :: psi_zn
      type(c_ptr), value :: status
      type(c_ptr), value :: stats
      type(lica_lvs_params), intent(in) :: prm
      type(c_ptr), value :: stream
    end function lica_gpu_lvs_transport_device

    integer(c_int) function lica_gpu_reinitialization(ncol, n, length, phi, layer, ilimit, &
        status) bind(c, name="lica_gpu_reinitialization")
      import
      integer(c_int32_t), value :: ncol
      integer(c_int32_t), value :: n
      real(c_double), value :: length
      real(c_double), intent(inout) :: phi(*)
      integer(c_int32_t), intent(in) :: layer(*)
      integer(c_int32_t), value :: ilimit
      integer(c_int32_t), intent(inout) :: status(*)
    end function lica_gpu_reinitialization

    integer(c_int) function lica_gpu_reinitialization_device(ncol, n, length, phi, layer, &
        ilimit, status, stream) bind(c, name="lica_gpu_reinitialization_device")
      import
      integer(c_int32_t), value :: ncol
      integer(c_int32_t), value :: n
      real(c_double), value :: length
      type(c_ptr), value :: phi
      type(c_ptr), value :: layer
      integer(c_int32_t), value :: ilimit
      type(c_ptr), value :: status
      type(c_ptr), value :: stream
    end function lica_gpu_reinitialization_device

    integer(c_int) function lica_gpu_grid_coupling(ncol, n, length, ini_psi, psif, layer, &
        psi_cn, psi_zn) bind(c, name="lica_gpu_grid_coupling")
      import
      integer(c_int32_t), value :: ncol
      integer(c_int32_t), value :: n
      real(c_double), value :: length
      integer(c_int32_t), value :: ini_psi
      real(c_double), intent(in) :: psif(*)
      integer(c_int32_t), intent(in) :: layer(*)
      real(c_double), intent(inout) :: psi_cn(*)
      real(c_double), intent(inout) :: psi_zn(*)
    end function lica_gpu_grid_coupling

    integer(c_int) function lica_gpu_grid_coupling_device(ncol, n, length, ini_psi, psif, &
        layer, psi_cn, psi_zn, stream) bind(c, name="lica_gpu_grid_coupling_device")
      import
      integer(c_int32_t), value :: ncol
      integer(c_int32_t), value :: n
      real(c_double), value :: length
      integer(c_int32_t), value :: ini_psi
      type(c_ptr), value :: psif
      type(c_ptr), value :: layer
      type(c_ptr), value :: psi_cn
      type(c_ptr), value :: psi_zn
      type(c_ptr), value :: stream
    end function lica_gpu_grid_coupling_device

    integer(c_int) function lica_gpu_temp_grad(ncol, n, length, props, dtconst, t, psi_cn, phi, &
        layer, mflvs, sfgas, sfgas2, imask, vol_tot_iphs, iterations, status) &
        bind(c, name="lica_gpu_temp_grad")
      import
      integer(c_int32_t), value :: ncol
      integer(c_int32_t), value :: n
      real(c_double), value :: length
      type(lica_col_props), intent(in) :: props
      real(c_double), value :: dtconst
      real(c_double), intent(in) :: t(*)
      real(c_double), intent(in) :: psi_cn(*)
      real(c_double), intent(in) :: phi(*)
      integer(c_int32_t), intent(in) :: layer(*)
      real(c_double), intent(inout) :: mflvs(*)
      real(c_double), intent(inout) :: sfgas(*)
      real(c_double), intent(inout) :: sfgas2(*)
      integer(c_int32_t), intent(inout) :: imask(*)
      real(c_double), intent(inout) :: vol_tot_iphs(*)
      integer(c_int32_t), intent(inout) :: iterations(*)
      integer(c_int32_t), intent(inout) :: status(*)
    end function lica_gpu_temp_grad

    integer(c_int) function lica_gpu_temp_grad_device(ncol, n, length, props, dtconst, t, &
        psi_cn, phi, layer, mflvs, sfgas, sfgas2, imask, vol_tot_iphs, iterations, status, &
        scratch, stream) bind(c, name="lica_gpu_temp_grad_device")
      import
      integer(c_int32_t), value :: ncol
      integer(c_int32_t), value :: n
      real(c_double), value :: length
      type(lica_col_props), intent(in) :: props
      real(c_double), value :: dtconst
      type(c_ptr), value :: t
      type(c_ptr), value :: psi_cn
      type(c_ptr), value :: phi
      type(c_ptr), value :: layer
      type(c_ptr), value :: mflvs
      type(c_ptr), value :: sfgas
      type(c_ptr), value :: sfgas2
      type(c_ptr), value :: imask
      type(c_ptr), value :: vol_tot_iphs
      type(c_ptr), value :: iterations
      type(c_ptr), value :: status
      type(c_ptr), value :: scratch
      type(c_ptr), value :: stream
    end function lica_gpu_temp_grad_device

    integer(c_int) function lica_gpu_pressure_correction(ncol, n, length, props, dtconst, w, p, &
        denf_zi, sfgas) bind(c, name="lica_gpu_pressure_correction")
      import
      integer(c_int32_t), value :: ncol
      integer(c_int32_t), value :: n
      real(c_double), value :: length
      type(lica_col_props), intent(in) :: props
      real(c_double), value :: dtconst
      real(c_double), intent(inout) :: w(*)
      real(c_double), intent(inout) :: p(*)
      real(c_double), intent(in) :: denf_zi(*)
      real(c_double), intent(in) :: sfgas(*)
    end function lica_gpu_pressure_correction

    integer(c_int) function lica_gpu_pressure_correction_device(ncol, n, length, props, &
        dtconst, w, p, denf_zi, sfgas, status, scratch, stream) &
        bind(c, name="lica_gpu_pressure_correction_device")
      import
      integer(c_int32_t), value :: ncol
      integer(c_int32_t), value :: n
      real(c_double), value :: length
      type(lica_col_props), intent(in) :: props
      real(c_double), value :: dtconst
      type(c_ptr), value :: w
      type(c_ptr), value :: p
      type(c_ptr), value :: denf_zi
      type(c_ptr), value :: sfgas
      type(c_ptr), value :: status
      type(c_ptr), value :: scratch
      type(c_ptr), value :: stream
    end function lica_gpu_pressure_correction_device

    integer(c_int) function lica_unet_conv3x3_device(x0, c0, x1, c1, w, bias, n, h, wd, cout, &
        relu, out, out32, out_c, out_c0, err, stream) bind(c, name="lica_unet_conv3x3_device")
      import
      type(c_ptr), value :: x0
      integer(c_int32_t), value :: c0
      type(c_ptr), value :: x1
      integer(c_int32_t), value :: c1
      type(c_ptr), value :: w
      type(c_ptr), value :: bias
      integer(c_int32_t), value :: n
      integer(c_int32_t), value :: h
      integer(c_int32_t), value :: wd
      integer(c_int32_t), value :: cout
      integer(c_int32_t), value :: relu
      type(c_ptr), value :: out
      type(c_ptr), value :: out32
      integer(c_int32_t), value :: out_c
      integer(c_int32_t), value :: out_c0
      type(c_ptr), value :: err
      type(c_ptr), value :: stream
    end function lica_unet_conv3x3_device

    integer(c_int) function lica_unet_create(out, n, h, w, seed) &
        bind(c, name="lica_unet_create")
      import
      type(c_ptr), intent(out) :: out
      integer(c_int32_t), value :: n
      integer(c_int32_t), value :: h
      integer(c_int32_t), value :: w
      integer(c_int64_t), value :: seed
    end function lica_unet_create

    integer(c_int) function lica_unet_destroy(net) bind(c, name="lica_unet_destroy")
      import
      type(c_ptr), value :: net
    end function lica_unet_destroy

    integer(c_int64_t) function lica_unet_param_count(net) bind(c, name="lica_unet_param_count")
      import
      type(c_ptr), value :: net
    end function lica_unet_param_count

    integer(c_int) function lica_unet_get_params(net, host, count) &
        bind(c, name="lica_unet_get_params")
      import
      type(c_ptr), value :: net
      real(c_float), intent(inout) :: host(*)
      integer(c_int64_t), value :: count
    end function lica_unet_get_params

    integer(c_int) function lica_unet_set_params(net, host, count) &
        bind(c, name="lica_unet_set_params")
      import
      type(c_ptr), value :: net
      real(c_float), intent(in) :: host(*)
      integer(c_int64_t), value :: count
    end function lica_unet_set_params

    integer(c_int) function lica_unet_guess_device(net, rho, f, hsq, x0, stream) &
        bind(c, name="lica_unet_guess_device")
      import
      type(c_ptr), value :: net
      type(c_ptr), value :: rho
      type(c_ptr), value :: f
      real(c_double), value :: hsq
      type(c_ptr), value :: x0
      type(c_ptr), value :: stream
    end function lica_unet_guess_device

    integer(c_int) function lica_unet_guess_checked_device(net, rho, f, bx, by, hx, hy, x0, &
        rel0, stream) bind(c, name="lica_unet_guess_checked_device")
      import
      type(c_ptr), value :: net
      type(c_ptr), value :: rho
      type(c_ptr), value :: f
      type(c_ptr), value :: bx
      type(c_ptr), value :: by
      real(c_double), value :: hx
      real(c_double), value :: hy
      type(c_ptr), value :: x0
      type(c_ptr), value :: rel0
      type(c_ptr), value :: stream
    end function lica_unet_guess_checked_device

    integer(c_int) function lica_unet_grad_device(net, rho, f, hsq, gx0, grad_host, count, &
        stream) bind(c, name="lica_unet_grad_device")
      import
      type(c_ptr), value :: net
      type(c_ptr), value :: rho
      type(c_ptr), value :: f
      real(c_double), value :: hsq
      type(c_ptr), value :: gx0
      type(c_ptr), value :: grad_host
      integer(c_int64_t), value :: count
      type(c_ptr), value :: stream
    end function lica_unet_grad_device

    integer(c_int) function lica_unet_train_step_device(net, rho, f, bx, by, p_star, hx, hy, &
        lr, loss, stream) bind(c, name="lica_unet_train_step_device")
      import
      type(c_ptr), value :: net
      type(c_ptr), value :: rho
      type(c_ptr), value :: f
      type(c_ptr), value :: bx
      type(c_ptr), value :: by
      type(c_ptr), value :: p_star
      real(c_double), value :: hx
      real(c_double), value :: hy
      real(c_float), value :: lr
      type(c_ptr), value :: loss
      type(c_ptr), value :: stream
    end function lica_unet_train_step_device

    integer(c_int) function lica_film2d_create(out, nx, ny, props, nlevels, precision) &
        bind(c, name="lica_film2d_create")
      import
      type(c_ptr), intent(out) :: out
      integer(c_int32_t), value :: nx
      integer(c_int32_t), value :: ny
      type(lica_film2d_props), intent(in) :: props
      integer(c_int32_t), value :: nlevels
      integer(c_int32_t), value :: precision
    end function lica_film2d_create

    integer(c_int) function lica_film2d_destroy(film) bind(c, name="lica_film2d_destroy")
      import
      type(c_ptr), value :: film
    end function lica_film2d_destroy

    integer(c_int) function lica_film2d_step_device(film, u, v, p, th, phi, dt, stats, stream) &
        bind(c, name="lica_film2d_step_device")
      import
      type(c_ptr), value :: film
      type(c_ptr), value :: u
      type(c_ptr), value :: v
      type(c_ptr), value :: p
      type(c_ptr), value :: th
      type(c_ptr), value :: phi
      real(c_double), value :: dt
      type(lica_film2d_stats), intent(inout) :: stats
      type(c_ptr), value :: stream
    end function lica_film2d_step_device

    integer(c_int) function lica_film2d_mdot_device(film, out, stream) &
        bind(c, name="lica_film2d_mdot_device")
      import
      type(c_ptr), value :: film
      type(c_ptr), value :: out
      type(c_ptr), value :: stream
    end function lica_film2d_mdot_device

    integer(c_int) function lica_film2d_set_guess(film, net) &
        bind(c, name="lica_film2d_set_guess")
      import
      type(c_ptr), value :: film
      type(c_ptr), value :: net
    end function lica_film2d_set_guess

    integer(c_int) function lica_film2d_set_warm_start(film, on) &
        bind(c, name="lica_film2d_set_warm_start")
      import
      type(c_ptr), value :: film
      integer(c_int32_t), value :: on
    end function lica_film2d_set_warm_start

    integer(c_int) function lica_film2d_capture_device(film, systems) &
        bind(c, name="lica_film2d_capture_device")
      import
      type(c_ptr), value :: film
      type(c_ptr), value :: systems
    end function lica_film2d_capture_device

    integer(c_int) function lica_gpu_bubble_grid_create(out, grid, max_lvs) &
        bind(c, name="lica_gpu_bubble_grid_create")
      import
      type(c_ptr), intent(out) :: out
      type(lica_bub_grid), intent(in) :: grid
      integer(c_int32_t), value :: max_lvs
    end function lica_gpu_bubble_grid_create

    integer(c_int) function lica_gpu_bubble_grid_destroy(geo) &
        bind(c, name="lica_gpu_bubble_grid_destroy")
      import
      type(c_ptr), value :: geo
    end function lica_gpu_bubble_grid_destroy

    integer(c_int) function lica_gpu_bubble_tracking_device(geo, nlvs, llvs0, psi_tmp, u, v, w, &
        time, icacy, out, stream) bind(c, name="lica_gpu_bubble_tracking_device")
      import
      type(c_ptr), value :: geo
      integer(c_int32_t), value :: nlvs
      integer(c_int32_t), value :: llvs0
      type(c_ptr), value :: psi_tmp
      type(c_ptr), value :: u
      type(c_ptr), value :: v
      type(c_ptr), value :: w
      real(c_double), value :: time
      integer(c_int32_t), value :: icacy
      type(c_ptr), value :: out
      type(c_ptr), value :: stream
    end function lica_gpu_bubble_tracking_device

    integer(c_int) function lica_gpu_bubble_tracking(grid, nlvs, llvs0, psi_tmp, u, v, w, time, &
        icacy, out) bind(c, name="lica_gpu_bubble_tracking")
      import
      type(lica_bub_grid), intent(in) :: grid
      integer(c_int32_t), value :: nlvs
      integer(c_int32_t), value :: llvs0
      real(c_double), intent(in) :: psi_tmp(*)
      real(c_double), intent(in) :: u(*)
      real(c_double), intent(in) :: v(*)
      real(c_double), intent(in) :: w(*)
      real(c_double), value :: time
      integer(c_int32_t), value :: icacy
      type(lica_bub_record), intent(inout) :: out(*)
    end function lica_gpu_bubble_tracking
  end interface
end module lica_gpu
