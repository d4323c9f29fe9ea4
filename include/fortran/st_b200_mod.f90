! st_b200_mod.f90 - Fortran 2003 (ISO_C_BINDING) interfaces to the C ABI of
! libst_b200 (include/st_b200.h), for the reference-named wrappers in
! st_stubs_mf.f and st_stubs_periodic.f.
!
! Every entry point returns an integer status (0 = ok, negative = error);
! st_check turns a failure into the reference's error behaviour, STOP.
! Arrays are passed by address as assumed-size REAL*8 arrays in the
! reference layout F(My,Mz,Mx[,n]); scalars the C side takes by value carry
! the VALUE attribute.  The module holds the one solver context that plays
! the role of the reference's COMMON blocks.
module st_b200
  use iso_c_binding
  implicit none
  private
  public :: st_params_t, st_ctx, st_check, st_error_message
  public :: st_create, st_destroy, st_last_error, st_default_params
  public :: st_set_state, st_get_state, st_set_tstep, st_get_tstep
  public :: st_get_common, st_set_common
  public :: st_tridiagonal, st_pentadiagonal
  public :: st_dfdx_sym, st_dfdy_sym, st_dfdz_sym, st_dfdx_asym, st_dfdy_asym, st_dfdz_asym
  public :: st_d2fdx2_sym, st_d2fdy2_sym, st_d2fdz2_sym
  public :: st_d2fdx2_asym, st_d2fdy2_asym, st_d2fdz2_asym
  public :: st_dfdx, st_dfdy, st_dfdz, st_d2fdx2, st_d2fdy2, st_d2fdz2
  public :: st_compact_filter
  public :: st_compact_filter_x_sym, st_compact_filter_y_sym, st_compact_filter_z_sym
  public :: st_compact_filter_x_asym, st_compact_filter_y_asym, st_compact_filter_z_asym
  public :: st_compact_filter_x, st_compact_filter_y, st_compact_filter_z
  public :: st_gaussian_filter, st_gaussian_filter_x, st_gaussian_filter_y, st_gaussian_filter_z
  public :: st_compute_gamma, st_rhs, st_compute_hyper, st_hyper_rhs, st_species_rhs
  public :: st_bc_rhs, st_sponge_forcing, st_fix_pressure
  public :: st_compute_cfl, st_compute_tstep, st_lddrk4, st_step, st_get_monitors, st_sync
  public :: st_compute_grad, st_shell_count, st_compute_srm_stats, st_generate_shock_surface
  public :: st_make_padded_arrays, st_write_visual

  ! st_params of include/st_b200.h, field for field
  type, bind(c) :: st_params_t
     integer(c_int) :: nx, ny, nz
     real(c_double) :: x_leng, y_leng, z_leng
     real(c_double) :: x_start, y_start, z_start
     real(c_double) :: re
     real(c_double) :: re1, re2, pr, sc
     real(c_double) :: gamma1, gamma2, epsilon, vis_exp, bulk_ratio, t_ratio
     integer(c_int) :: hyper_param
     integer(c_int) :: rk_mode
     real(c_double) :: cfl_cal
     real(c_double) :: c_beta_scale
     integer(c_int) :: device
     integer(c_int) :: family
     integer(c_int) :: precision
  end type st_params_t

  ! the context created by st_b200_init (st_stubs_*.f)
  type(c_ptr), save :: st_ctx = c_null_ptr

  interface
     ! ---- context ----------------------------------------------------------
     integer(c_int) function st_create(p, ctx) bind(c, name='st_create')
       import :: c_int, c_ptr, st_params_t
       type(st_params_t), intent(in) :: p
       type(c_ptr), intent(out) :: ctx
     end function
     integer(c_int) function st_destroy(ctx) bind(c, name='st_destroy')
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
     end function
     type(c_ptr) function st_last_error(ctx) bind(c, name='st_last_error')
       import :: c_ptr
       type(c_ptr), value :: ctx
     end function
     subroutine st_default_params(p, nx, ny, nz) bind(c, name='st_default_params')
       import :: c_int, st_params_t
       type(st_params_t), intent(out) :: p
       integer(c_int), value :: nx, ny, nz
     end subroutine
     ! Y: c_loc of the mass fraction, or c_null_ptr in the periodic family
     integer(c_int) function st_set_state(ctx, Q, Y) bind(c, name='st_set_state')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: Q(*)
       type(c_ptr), value :: Y
     end function
     integer(c_int) function st_get_state(ctx, Q, Y) bind(c, name='st_get_state')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(out) :: Q(*)
       type(c_ptr), value :: Y
     end function
     integer(c_int) function st_set_tstep(ctx, tstep) bind(c, name='st_set_tstep')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), value :: tstep
     end function
     integer(c_int) function st_get_tstep(ctx, tstep) bind(c, name='st_get_tstep')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(out) :: tstep
     end function
     integer(c_int) function st_get_common(ctx, name, out) bind(c, name='st_get_common')
       import :: c_int, c_ptr, c_char, c_double
       type(c_ptr), value :: ctx
       character(kind=c_char), intent(in) :: name(*)
       real(c_double), intent(out) :: out(*)
     end function
     integer(c_int) function st_set_common(ctx, name, in) bind(c, name='st_set_common')
       import :: c_int, c_ptr, c_char, c_double
       type(c_ptr), value :: ctx
       character(kind=c_char), intent(in) :: name(*)
       real(c_double), intent(in) :: in(*)
     end function

     ! ---- line solvers -------------------------------------------------------
     integer(c_int) function st_tridiagonal(ctx, A, B, C, R, n, lot, nper) bind(c, name='st_tridiagonal')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: A(*), B(*), C(*)
       real(c_double), intent(inout) :: R(*)
       integer(c_int), value :: n, lot, nper
     end function
     integer(c_int) function st_pentadiagonal(ctx, A, B, C, D, E, R, n, lot, nper) &
          bind(c, name='st_pentadiagonal')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: A(*), B(*), C(*), D(*), E(*)
       real(c_double), intent(inout) :: R(*)
       integer(c_int), value :: n, lot, nper
     end function

     ! ---- compact derivatives ------------------------------------------------
     integer(c_int) function st_dfdx_sym(ctx, F, dF, iadd, cadd) bind(c, name='st_dfdx_sym')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: dF(*)
       integer(c_int), value :: iadd
       real(c_double), value :: cadd
     end function
     integer(c_int) function st_dfdy_sym(ctx, F, dF, iadd, cadd) bind(c, name='st_dfdy_sym')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: dF(*)
       integer(c_int), value :: iadd
       real(c_double), value :: cadd
     end function
     integer(c_int) function st_dfdz_sym(ctx, F, dF, iadd, cadd) bind(c, name='st_dfdz_sym')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: dF(*)
       integer(c_int), value :: iadd
       real(c_double), value :: cadd
     end function
     integer(c_int) function st_dfdx_asym(ctx, F, dF, iadd, cadd) bind(c, name='st_dfdx_asym')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: dF(*)
       integer(c_int), value :: iadd
       real(c_double), value :: cadd
     end function
     integer(c_int) function st_dfdy_asym(ctx, F, dF, iadd, cadd) bind(c, name='st_dfdy_asym')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: dF(*)
       integer(c_int), value :: iadd
       real(c_double), value :: cadd
     end function
     integer(c_int) function st_dfdz_asym(ctx, F, dF, iadd, cadd) bind(c, name='st_dfdz_asym')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: dF(*)
       integer(c_int), value :: iadd
       real(c_double), value :: cadd
     end function
     integer(c_int) function st_d2fdx2_sym(ctx, F, dF, d2F, iadd) bind(c, name='st_d2fdx2_sym')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: dF(*), d2F(*)
       integer(c_int), value :: iadd
     end function
     integer(c_int) function st_d2fdy2_sym(ctx, F, dF, d2F, iadd) bind(c, name='st_d2fdy2_sym')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: dF(*), d2F(*)
       integer(c_int), value :: iadd
     end function
     integer(c_int) function st_d2fdz2_sym(ctx, F, dF, d2F, iadd) bind(c, name='st_d2fdz2_sym')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: dF(*), d2F(*)
       integer(c_int), value :: iadd
     end function
     integer(c_int) function st_d2fdx2_asym(ctx, F, dF, d2F, iadd) bind(c, name='st_d2fdx2_asym')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: dF(*), d2F(*)
       integer(c_int), value :: iadd
     end function
     integer(c_int) function st_d2fdy2_asym(ctx, F, dF, d2F, iadd) bind(c, name='st_d2fdy2_asym')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: dF(*), d2F(*)
       integer(c_int), value :: iadd
     end function
     integer(c_int) function st_d2fdz2_asym(ctx, F, dF, d2F, iadd) bind(c, name='st_d2fdz2_asym')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: dF(*), d2F(*)
       integer(c_int), value :: iadd
     end function
     ! periodic family
     integer(c_int) function st_dfdx(ctx, F, dF, iadd, cadd) bind(c, name='st_dfdx')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: dF(*)
       integer(c_int), value :: iadd
       real(c_double), value :: cadd
     end function
     integer(c_int) function st_dfdy(ctx, F, dF, iadd, cadd) bind(c, name='st_dfdy')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: dF(*)
       integer(c_int), value :: iadd
       real(c_double), value :: cadd
     end function
     integer(c_int) function st_dfdz(ctx, F, dF, iadd, cadd) bind(c, name='st_dfdz')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: dF(*)
       integer(c_int), value :: iadd
       real(c_double), value :: cadd
     end function
     integer(c_int) function st_d2fdx2(ctx, F, dF, d2F, iadd) bind(c, name='st_d2fdx2')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: dF(*), d2F(*)
       integer(c_int), value :: iadd
     end function
     integer(c_int) function st_d2fdy2(ctx, F, dF, d2F, iadd) bind(c, name='st_d2fdy2')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: dF(*), d2F(*)
       integer(c_int), value :: iadd
     end function
     integer(c_int) function st_d2fdz2(ctx, F, dF, d2F, iadd) bind(c, name='st_d2fdz2')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: dF(*), d2F(*)
       integer(c_int), value :: iadd
     end function

     ! ---- filters ------------------------------------------------------------
     integer(c_int) function st_compact_filter(ctx, F, F0, nvar) bind(c, name='st_compact_filter')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: F0(*)
       integer(c_int), value :: nvar
     end function
     integer(c_int) function st_compact_filter_x_sym(ctx, F, F0) bind(c, name='st_compact_filter_x_sym')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: F0(*)
     end function
     integer(c_int) function st_compact_filter_y_sym(ctx, F, F0) bind(c, name='st_compact_filter_y_sym')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: F0(*)
     end function
     integer(c_int) function st_compact_filter_z_sym(ctx, F, F0) bind(c, name='st_compact_filter_z_sym')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: F0(*)
     end function
     integer(c_int) function st_compact_filter_x_asym(ctx, F, F0) bind(c, name='st_compact_filter_x_asym')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: F0(*)
     end function
     integer(c_int) function st_compact_filter_y_asym(ctx, F, F0) bind(c, name='st_compact_filter_y_asym')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: F0(*)
     end function
     integer(c_int) function st_compact_filter_z_asym(ctx, F, F0) bind(c, name='st_compact_filter_z_asym')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: F0(*)
     end function
     integer(c_int) function st_compact_filter_x(ctx, F, F0) bind(c, name='st_compact_filter_x')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: F0(*)
     end function
     integer(c_int) function st_compact_filter_y(ctx, F, F0) bind(c, name='st_compact_filter_y')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: F0(*)
     end function
     integer(c_int) function st_compact_filter_z(ctx, F, F0) bind(c, name='st_compact_filter_z')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(inout) :: F0(*)
     end function
     integer(c_int) function st_gaussian_filter(ctx, F, Fg, nvar) bind(c, name='st_gaussian_filter')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(out) :: Fg(*)
       integer(c_int), value :: nvar
     end function
     integer(c_int) function st_gaussian_filter_x(ctx, F, Fg) bind(c, name='st_gaussian_filter_x')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(out) :: Fg(*)
     end function
     integer(c_int) function st_gaussian_filter_y(ctx, F, Fg) bind(c, name='st_gaussian_filter_y')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(out) :: Fg(*)
     end function
     integer(c_int) function st_gaussian_filter_z(ctx, F, Fg) bind(c, name='st_gaussian_filter_z')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: F(*)
       real(c_double), intent(out) :: Fg(*)
     end function

     ! ---- physics operators --------------------------------------------------
     integer(c_int) function st_compute_gamma(ctx, Y) bind(c, name='st_compute_gamma')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: Y(*)
     end function
     ! Y: c_loc of the mass fraction (_mf family), c_null_ptr (periodic family)
     integer(c_int) function st_rhs(ctx, Q, Qrhs, Y) bind(c, name='st_rhs')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(inout) :: Q(*)
       real(c_double), intent(out) :: Qrhs(*)
       type(c_ptr), value :: Y
     end function
     integer(c_int) function st_compute_hyper(ctx, Q, Y) bind(c, name='st_compute_hyper')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: Q(*)
       type(c_ptr), value :: Y
     end function
     integer(c_int) function st_hyper_rhs(ctx, Q, Qrhs, Y) bind(c, name='st_hyper_rhs')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: Q(*)
       real(c_double), intent(inout) :: Qrhs(*)
       type(c_ptr), value :: Y
     end function
     integer(c_int) function st_species_rhs(ctx, Q, Qrhs, Y, Yrhs) bind(c, name='st_species_rhs')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: Q(*), Y(*)
       real(c_double), intent(inout) :: Qrhs(*), Yrhs(*)
     end function
     integer(c_int) function st_bc_rhs(ctx, Q, Qrhs, Y, Yrhs, time) bind(c, name='st_bc_rhs')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(inout) :: Q(*), Qrhs(*), Yrhs(*)
       real(c_double), intent(in) :: Y(*)
       real(c_double), value :: time
     end function
     integer(c_int) function st_sponge_forcing(ctx, Q, Qrhs, Y, Yrhs) bind(c, name='st_sponge_forcing')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: Q(*), Y(*)
       real(c_double), intent(inout) :: Qrhs(*), Yrhs(*)
     end function
     integer(c_int) function st_fix_pressure(ctx, Q, Y) bind(c, name='st_fix_pressure')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(inout) :: Q(*)
       type(c_ptr), value :: Y
     end function
     integer(c_int) function st_compute_cfl(ctx, Q, cfl_stab, cfl_resv) bind(c, name='st_compute_cfl')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: Q(*)
       real(c_double), intent(out) :: cfl_stab, cfl_resv
     end function
     integer(c_int) function st_compute_tstep(ctx, Q, Y, cfl_resv, step, tstep) &
          bind(c, name='st_compute_tstep')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: Q(*)
       type(c_ptr), value :: Y
       real(c_double), value :: cfl_resv
       integer(c_int), value :: step
       real(c_double), intent(out) :: tstep
     end function

     ! ---- time integration on the resident state -----------------------------
     integer(c_int) function st_lddrk4(ctx, time, step) bind(c, name='st_lddrk4')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(inout) :: time
       integer(c_int), intent(inout) :: step
     end function
     integer(c_int) function st_step(ctx, time, step) bind(c, name='st_step')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(inout) :: time
       integer(c_int), intent(inout) :: step
     end function
     integer(c_int) function st_get_monitors(ctx, out) bind(c, name='st_get_monitors')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(out) :: out(10)
     end function
     integer(c_int) function st_sync(ctx) bind(c, name='st_sync')
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
     end function

     ! ---- Output-side diagnostics ---------------------------------------------
     integer(c_int) function st_compute_grad(ctx, Grad, maxdil, enstrophy) bind(c, name='st_compute_grad')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(out) :: Grad(*)
       real(c_double), intent(out) :: maxdil, enstrophy
     end function
     integer(c_int) function st_shell_count(ctx, n_avg) bind(c, name='st_shell_count')
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int), intent(out) :: n_avg
     end function
     integer(c_int) function st_compute_srm_stats(ctx, hmix, tke_total, ur_avg, y_avg) &
          bind(c, name='st_compute_srm_stats')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(out) :: hmix, tke_total
       real(c_double), intent(out) :: ur_avg(*), y_avg(*)
     end function
     integer(c_int) function st_generate_shock_surface(ctx, rad_avg, rad_skew_rms) &
          bind(c, name='st_generate_shock_surface')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(out) :: rad_avg, rad_skew_rms
     end function
     ! Grad: c_loc of the 4 Compute_Grad fields, or c_null_ptr
     integer(c_int) function st_make_padded_arrays(ctx, Grad, W, xx, yy, zz) &
          bind(c, name='st_make_padded_arrays')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       type(c_ptr), value :: Grad
       real(c_double), intent(out) :: W(*), xx(*), yy(*), zz(*)
     end function
     integer(c_int) function st_write_visual(ctx, Grad, vis_path, prefix, cue_vis, time, step) &
          bind(c, name='st_write_visual')
       import :: c_int, c_ptr, c_char, c_double
       type(c_ptr), value :: ctx
       type(c_ptr), value :: Grad
       character(kind=c_char), intent(in) :: vis_path(*), prefix(*)
       integer(c_int), value :: cue_vis
       real(c_double), value :: time
       integer(c_int), value :: step
     end function

     ! C library strlen, for the error message of st_last_error
     integer(c_size_t) function c_strlen(s) bind(c, name='strlen')
       import :: c_size_t, c_ptr
       type(c_ptr), value :: s
     end function
  end interface

contains

  ! The library's message for the last failure on the context.
  function st_error_message() result(msg)
    character(len=:), allocatable :: msg
    type(c_ptr) :: p
    character(kind=c_char), pointer :: chars(:)
    integer :: i, n
    msg = ''
    if (.not. c_associated(st_ctx)) return
    p = st_last_error(st_ctx)
    if (.not. c_associated(p)) return
    n = int(c_strlen(p))
    call c_f_pointer(p, chars, [n])
    allocate(character(len=n) :: msg)
    do i = 1, n
       msg(i:i) = chars(i)
    end do
  end function st_error_message

  ! A nonzero status ends the run with STOP, the reference's error handling
  ! (e.g. src/tridiagonal.f90:52).
  subroutine st_check(ierr, what)
    integer(c_int), intent(in) :: ierr
    character(len=*), intent(in) :: what
    if (ierr /= 0) then
       write(*, '(a, a, a, i0, a, a)') 'libst_b200: ', what, ' failed, status ', ierr, ': ', &
            st_error_message()
       stop 'libst_b200 error'
    end if
  end subroutine st_check

end module st_b200
