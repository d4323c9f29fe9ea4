************************************************************************
*  st_stubs_mf.f - reference-named wrappers over libst_b200 for the
*  two-species symmetric-octant build (src/makefile_mf).
*
*  Link this file, st_b200_mod.f90 and libst_b200.so in place of the
*  objects whose routines are listed below.  Every wrapper keeps the
*  reference's name and argument list, so src/main_mf.f and the routines
*  that stay in Fortran call them unchanged.  Fixed form, compiled with
*  the reference's 'header' (grid PARAMETERs and COMMON scalars).
*
*  One solver context (module st_b200) plays the role of the COMMON
*  blocks /RKWORK/, /SPECIES/, /THERMO/, /GRAD/ and /HYPER/: every
*  wrapped routine reads and writes the context's device copies.  The
*  host COMMON copies are refreshed where the reference program reads
*  them outside the wrapped routines:
*   - LDDRK4 copies /RKWORK/ Q and /SPECIES/ Y in and out, sets /TRACK/;
*   - Compute_gamma refreshes /THERMO/, Compute_hyper /HYPER/;
*   - Compute_Tstep sets Tstep in /TIME_RK/;
*   - st_b200_pull_commons copies /THERMO/, /GRAD/ and /HYPER/ back,
*     for a routine that stays in Fortran and reads them (a visualisation
*     writer, for instance).
*  A nonzero status from the library stops the run (st_check), as the
*  reference's own errors do.
*
*  The grid must sit on one GPU: Px = Py = Pz = 1 in 'header' (the
*  reference's MPI pencils are replaced by the whole grid in HBM), so
*  that Mx = Nx, My = Ny, Mz = Nz.
************************************************************************

*  Creates the context once, from the grid and flow parameters that
*  Define_Param and Setup_Grid have set (src/define_nonperiodic_mf.f,
*  src/grid.f:15-112).  Replaces the set-up of the constant LU factors.
      Subroutine st_b200_init

      Use iso_c_binding, only: c_associated
      Use st_b200

      Include 'header'

      Type(st_params_t) p

      If (c_associated(st_ctx)) Return
      If (Px*Py*Pz .NE. 1) Stop 'libst_b200: needs Px = Py = Pz = 1'

      Call st_default_params(p, Nx, Ny, Nz)
      p%x_leng = x_leng
      p%y_leng = y_leng
      p%z_leng = z_leng
      p%x_start = x_start
      p%y_start = y_start
      p%z_start = z_start
      p%re = Re
      p%re1 = Re1
      p%re2 = Re2
      p%pr = Pr
      p%sc = Sc
      p%gamma1 = gamma1
      p%gamma2 = gamma2
      p%epsilon = epsilon
      p%vis_exp = vis_exp
      p%bulk_ratio = bulk_ratio
      p%t_ratio = T_ratio
      p%hyper_param = hyper_param
*  rk_mode 0: the second LDDRK4 loop with the reference build's
*  unassigned (zero) alpha2/beta2
      p%rk_mode = 0
      p%cfl_cal = cfl_cal
      p%c_beta_scale = 1.0D0
      p%device = 0
      p%family = 0
      p%precision = 0
      Call st_check(st_create(p, st_ctx), 'st_create')

      Return

      End

*  Copies the context's /THERMO/, /GRAD/ and /HYPER/ into the host
*  COMMON blocks.
      Subroutine st_b200_pull_commons

      Use iso_c_binding, only: c_null_char
      Use st_b200

      Include 'header'

      Real*8  gamma_eff(My,Mz,Mx)
      Real*8  G(My,Mz,Mx,12)
      Real*8  H(My,Mz,Mx,4)

      Common /THERMO/ gamma_eff
      Common /GRAD/ G
      Common /HYPER/ H

      Character*10 gname(12), hname(4)
      Integer I

      Data gname /'dux_dx', 'duy_dx', 'duz_dx', 'dux_dy', 'duy_dy',
     .            'duz_dy', 'dux_dz', 'duy_dz', 'duz_dz', 'dTdx',
     .            'dTdy', 'dTdz'/
      Data hname /'beta_hyper', 'visc_hyper', 'k_hyper', 'D_hyper'/

      Call st_check(st_get_common(st_ctx, 'gamma_eff'//c_null_char,
     .              gamma_eff), 'st_b200_pull_commons')
      Do I = 1, 12
        Call st_check(st_get_common(st_ctx,
     .       trim(gname(I))//c_null_char, G(1,1,1,I)),
     .       'st_b200_pull_commons')
      End Do
      Do I = 1, 4
        Call st_check(st_get_common(st_ctx,
     .       trim(hname(I))//c_null_char, H(1,1,1,I)),
     .       'st_b200_pull_commons')
      End Do

      Return

      End

*  /TRACK/ monitors of (Q, /SPECIES/ Y) as the context computes them:
*  mon = KE, MomX, MomY, MomZ, Mass, Energy, Entropy, Entropy2
      Subroutine st_b200_monitors(Q, mon)

      Use iso_c_binding, only: c_loc
      Use st_b200

      Include 'header'

      Real*8  Q(My,Mz,Mx,5), mon(10)
      Real*8, Target :: Y(My,Mz,Mx,1)
      Real*8  drYi(My,Mz,Mx,1), rYW(My,Mz,Mx,1)

      Common /SPECIES/ Y, drYi, rYW

      Call st_b200_init
      Call st_check(st_set_state(st_ctx, Q, c_loc(Y)), 'monitors')
      Call st_check(st_get_monitors(st_ctx, mon), 'monitors')

      Return

      End

************************************************************************
*  Set-up: Setup_Derivatives_Sym src/derivCDopt6_sym_tri.f:9,
*  Setup_Derivatives_Asym src/derivCDopt6_asym_tri.f:9,
*  Init_Filters_sym src/filters_sym.f:9, Init_Filters_asym
*  src/filters_asym.f:9.  The context holds every LU factor.
************************************************************************
      Subroutine Setup_Derivatives_Sym
      Call st_b200_init
      Return
      End

      Subroutine Setup_Derivatives_Asym
      Call st_b200_init
      Return
      End

      Subroutine Init_Filters_sym
      Call st_b200_init
      Return
      End

      Subroutine Init_Filters_asym
      Call st_b200_init
      Return
      End

************************************************************************
*  Compact derivatives: src/derivCDopt6_sym_tri.f:409,538,672,801,932,
*  1062 and src/derivCDopt6_asym_tri.f:412,540,670,798,930,1061.
************************************************************************
      Subroutine DFDX_sym(F, dF, iadd, cadd)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), dF(My,Mz,Mx), cadd
      Integer iadd
      Call st_check(st_dfdx_sym(st_ctx, F, dF, iadd, cadd), 'DFDX_sym')
      Return
      End

      Subroutine DFDY_sym(F, dF, iadd, cadd)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), dF(My,Mz,Mx), cadd
      Integer iadd
      Call st_check(st_dfdy_sym(st_ctx, F, dF, iadd, cadd), 'DFDY_sym')
      Return
      End

      Subroutine DFDZ_sym(F, dF, iadd, cadd)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), dF(My,Mz,Mx), cadd
      Integer iadd
      Call st_check(st_dfdz_sym(st_ctx, F, dF, iadd, cadd), 'DFDZ_sym')
      Return
      End

      Subroutine DFDX_asym(F, dF, iadd, cadd)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), dF(My,Mz,Mx), cadd
      Integer iadd
      Call st_check(st_dfdx_asym(st_ctx, F, dF, iadd, cadd),
     .              'DFDX_asym')
      Return
      End

      Subroutine DFDY_asym(F, dF, iadd, cadd)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), dF(My,Mz,Mx), cadd
      Integer iadd
      Call st_check(st_dfdy_asym(st_ctx, F, dF, iadd, cadd),
     .              'DFDY_asym')
      Return
      End

      Subroutine DFDZ_asym(F, dF, iadd, cadd)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), dF(My,Mz,Mx), cadd
      Integer iadd
      Call st_check(st_dfdz_asym(st_ctx, F, dF, iadd, cadd),
     .              'DFDZ_asym')
      Return
      End

      Subroutine D2FDX2_sym(F, dF, d2F, iadd)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), dF(My,Mz,Mx), d2F(My,Mz,Mx)
      Integer iadd
      Call st_check(st_d2fdx2_sym(st_ctx, F, dF, d2F, iadd),
     .              'D2FDX2_sym')
      Return
      End

      Subroutine D2FDY2_sym(F, dF, d2F, iadd)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), dF(My,Mz,Mx), d2F(My,Mz,Mx)
      Integer iadd
      Call st_check(st_d2fdy2_sym(st_ctx, F, dF, d2F, iadd),
     .              'D2FDY2_sym')
      Return
      End

      Subroutine D2FDZ2_sym(F, dF, d2F, iadd)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), dF(My,Mz,Mx), d2F(My,Mz,Mx)
      Integer iadd
      Call st_check(st_d2fdz2_sym(st_ctx, F, dF, d2F, iadd),
     .              'D2FDZ2_sym')
      Return
      End

      Subroutine D2FDX2_asym(F, dF, d2F, iadd)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), dF(My,Mz,Mx), d2F(My,Mz,Mx)
      Integer iadd
      Call st_check(st_d2fdx2_asym(st_ctx, F, dF, d2F, iadd),
     .              'D2FDX2_asym')
      Return
      End

      Subroutine D2FDY2_asym(F, dF, d2F, iadd)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), dF(My,Mz,Mx), d2F(My,Mz,Mx)
      Integer iadd
      Call st_check(st_d2fdy2_asym(st_ctx, F, dF, d2F, iadd),
     .              'D2FDY2_asym')
      Return
      End

      Subroutine D2FDZ2_asym(F, dF, d2F, iadd)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), dF(My,Mz,Mx), d2F(My,Mz,Mx)
      Integer iadd
      Call st_check(st_d2fdz2_asym(st_ctx, F, dF, d2F, iadd),
     .              'D2FDZ2_asym')
      Return
      End

************************************************************************
*  Line solvers: tridiagonal src/tridiagonal.f90:1, pentadiagonal
*  src/pentadiagonal.f90:1.  Arrays (lot,n); R is overwritten.  ncom,
*  the communicator of the line direction, has one rank here.
************************************************************************
      Subroutine tridiagonal(A1, B1, C1, R, n, lot, nper, ncom)
      Use st_b200
      Integer n, lot, nper, ncom
      Real*8  A1(lot,n), B1(lot,n), C1(lot,n), R(lot,n)
      Call st_b200_init
      Call st_check(st_tridiagonal(st_ctx, A1, B1, C1, R, n, lot,
     .              nper), 'tridiagonal')
      Return
      End

      Subroutine pentadiagonal(A1, B1, C1, D1, E1, R, n, lot, nper,
     .                         ncom)
      Use st_b200
      Integer n, lot, nper, ncom
      Real*8  A1(lot,n), B1(lot,n), C1(lot,n), D1(lot,n), E1(lot,n)
      Real*8  R(lot,n)
      Call st_b200_init
      Call st_check(st_pentadiagonal(st_ctx, A1, B1, C1, D1, E1, R,
     .              n, lot, nper), 'pentadiagonal')
      Return
      End

************************************************************************
*  Filters: Compact_Filter src/filters_sym.f:398, Compact_Filter_X/Y/Z
*  _sym :436,637,838, _asym src/filters_asym.f:388,586,783,
*  Gaussian_Filter src/filters_sym.f:1046, Gaussian_Filter_X/Y/Z
*  :1072,1234,1396.  F0 may be F itself.
************************************************************************
      Subroutine Compact_Filter(F, F0, N)
      Use st_b200
      Include 'header'
      Integer N
      Real*8  F(My,Mz,Mx,N), F0(My,Mz,Mx,N)
      Call st_check(st_compact_filter(st_ctx, F, F0, N),
     .              'Compact_Filter')
      Return
      End

      Subroutine Compact_Filter_X_sym(F, F0)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), F0(My,Mz,Mx)
      Call st_check(st_compact_filter_x_sym(st_ctx, F, F0),
     .              'Compact_Filter_X_sym')
      Return
      End

      Subroutine Compact_Filter_Y_sym(F, F0)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), F0(My,Mz,Mx)
      Call st_check(st_compact_filter_y_sym(st_ctx, F, F0),
     .              'Compact_Filter_Y_sym')
      Return
      End

      Subroutine Compact_Filter_Z_sym(F, F0)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), F0(My,Mz,Mx)
      Call st_check(st_compact_filter_z_sym(st_ctx, F, F0),
     .              'Compact_Filter_Z_sym')
      Return
      End

      Subroutine Compact_Filter_X_asym(F, F0)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), F0(My,Mz,Mx)
      Call st_check(st_compact_filter_x_asym(st_ctx, F, F0),
     .              'Compact_Filter_X_asym')
      Return
      End

      Subroutine Compact_Filter_Y_asym(F, F0)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), F0(My,Mz,Mx)
      Call st_check(st_compact_filter_y_asym(st_ctx, F, F0),
     .              'Compact_Filter_Y_asym')
      Return
      End

      Subroutine Compact_Filter_Z_asym(F, F0)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), F0(My,Mz,Mx)
      Call st_check(st_compact_filter_z_asym(st_ctx, F, F0),
     .              'Compact_Filter_Z_asym')
      Return
      End

      Subroutine Gaussian_Filter(F, Fg, N)
      Use st_b200
      Include 'header'
      Integer N
      Real*8  F(My,Mz,Mx,N), Fg(My,Mz,Mx,N)
      Call st_check(st_gaussian_filter(st_ctx, F, Fg, N),
     .              'Gaussian_Filter')
      Return
      End

      Subroutine Gaussian_Filter_X(F, Fg)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), Fg(My,Mz,Mx)
      Call st_check(st_gaussian_filter_x(st_ctx, F, Fg),
     .              'Gaussian_Filter_X')
      Return
      End

      Subroutine Gaussian_Filter_Y(F, Fg)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), Fg(My,Mz,Mx)
      Call st_check(st_gaussian_filter_y(st_ctx, F, Fg),
     .              'Gaussian_Filter_Y')
      Return
      End

      Subroutine Gaussian_Filter_Z(F, Fg)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), Fg(My,Mz,Mx)
      Call st_check(st_gaussian_filter_z(st_ctx, F, Fg),
     .              'Gaussian_Filter_Z')
      Return
      End

************************************************************************
*  Physics: Compute_gamma src/lddrk4_nonperiodic_mf.f:342, RHS
*  src/rhsv_sym_mf.f:9, Compute_hyper src/hyper_dynamic_sym_mf.f:166,
*  Hyper_RHS src/hyper_rhs_sym_mf.f:12, Species_RHS
*  src/species_rhs_sym.f:9, bc_RHS src/bc_mf.f:11, Sponge_Forcing
*  src/sponge_mf.f:7, Fix_Pressure pproc/pproc_mf.f:190.
************************************************************************
      Subroutine Compute_gamma(Y)
      Use iso_c_binding, only: c_null_char
      Use st_b200
      Include 'header'
      Real*8  Y(My,Mz,Mx,1)
      Real*8  gamma_eff(My,Mz,Mx)
      Common /THERMO/ gamma_eff
      Call st_b200_init
      Call st_check(st_compute_gamma(st_ctx, Y), 'Compute_gamma')
      Call st_check(st_get_common(st_ctx, 'gamma_eff'//c_null_char,
     .              gamma_eff), 'Compute_gamma')
      Return
      End

      Subroutine RHS(Q, Qrhs, Y)
      Use iso_c_binding, only: c_loc
      Use st_b200
      Include 'header'
      Real*8  Q(My,Mz,Mx,5), Qrhs(My,Mz,Mx,5)
      Real*8, Target :: Y(My,Mz,Mx,1)
      Call st_check(st_rhs(st_ctx, Q, Qrhs, c_loc(Y)), 'RHS')
      Return
      End

      Subroutine Compute_hyper(Q, Y)
      Use iso_c_binding, only: c_loc, c_null_char
      Use st_b200
      Include 'header'
      Real*8  Q(My,Mz,Mx,5)
      Real*8, Target :: Y(My,Mz,Mx,1)
      Real*8  H(My,Mz,Mx,4)
      Common /HYPER/ H
      Call st_b200_init
      Call st_check(st_compute_hyper(st_ctx, Q, c_loc(Y)),
     .              'Compute_hyper')
      Call st_check(st_get_common(st_ctx, 'beta_hyper'//c_null_char,
     .              H(1,1,1,1)), 'Compute_hyper')
      Call st_check(st_get_common(st_ctx, 'visc_hyper'//c_null_char,
     .              H(1,1,1,2)), 'Compute_hyper')
      Call st_check(st_get_common(st_ctx, 'k_hyper'//c_null_char,
     .              H(1,1,1,3)), 'Compute_hyper')
      Call st_check(st_get_common(st_ctx, 'D_hyper'//c_null_char,
     .              H(1,1,1,4)), 'Compute_hyper')
      Return
      End

      Subroutine Hyper_RHS(Q, Qrhs, Y)
      Use iso_c_binding, only: c_loc
      Use st_b200
      Include 'header'
      Real*8  Q(My,Mz,Mx,5), Qrhs(My,Mz,Mx,5)
      Real*8, Target :: Y(My,Mz,Mx,1)
      Call st_check(st_hyper_rhs(st_ctx, Q, Qrhs, c_loc(Y)),
     .              'Hyper_RHS')
      Return
      End

      Subroutine Species_RHS(Q, Qrhs, Y, Yrhs)
      Use st_b200
      Include 'header'
      Real*8  Q(My,Mz,Mx,5), Qrhs(My,Mz,Mx,5)
      Real*8  Y(My,Mz,Mx,1), Yrhs(My,Mz,Mx,1)
      Call st_check(st_species_rhs(st_ctx, Q, Qrhs, Y, Yrhs),
     .              'Species_RHS')
      Return
      End

      Subroutine bc_RHS(Q, Qrhs, Y, Yrhs, time)
      Use st_b200
      Include 'header'
      Real*8  Q(My,Mz,Mx,5), Qrhs(My,Mz,Mx,5)
      Real*8  Y(My,Mz,Mx,1), Yrhs(My,Mz,Mx,1), time
      Call st_check(st_bc_rhs(st_ctx, Q, Qrhs, Y, Yrhs, time),
     .              'bc_RHS')
      Return
      End

      Subroutine Sponge_Forcing(Q, Qrhs, Y, Yrhs)
      Use st_b200
      Include 'header'
      Real*8  Q(My,Mz,Mx,5), Qrhs(My,Mz,Mx,5)
      Real*8  Y(My,Mz,Mx,1), Yrhs(My,Mz,Mx,1)
      Call st_check(st_sponge_forcing(st_ctx, Q, Qrhs, Y, Yrhs),
     .              'Sponge_Forcing')
      Return
      End

      Subroutine Fix_Pressure(Q, Y)
      Use iso_c_binding, only: c_loc
      Use st_b200
      Include 'header'
      Real*8  Q(My,Mz,Mx,5)
      Real*8, Target :: Y(My,Mz,Mx,1)
      Call st_check(st_fix_pressure(st_ctx, Q, c_loc(Y)),
     .              'Fix_Pressure')
      Return
      End

************************************************************************
*  Time step and integration: Compute_CFL and Compute_Tstep
*  src/lddrk4_nonperiodic_mf.f:7,75, LDDRK4 :428, and the monitors
*  Compute_KE/Mom/Mass/Energy/Entropy :168,216,243,267,288.
************************************************************************
      Subroutine Compute_CFL(Q, cfl_stab_all, cfl_resv_all, step)
      Use st_b200
      Include 'header'
      Real*8  Q(My,Mz,Mx,5), cfl_stab_all, cfl_resv_all
      Integer step
      Call st_b200_init
      Call st_check(st_compute_cfl(st_ctx, Q, cfl_stab_all,
     .              cfl_resv_all), 'Compute_CFL')
      Return
      End

*  Sets Tstep of /TIME_RK/.  The artificial-viscosity limits use the
*  context's /HYPER/, which Compute_hyper and LDDRK4 keep current.
      Subroutine Compute_Tstep(Q, Y, cfl_resv, step)
      Use iso_c_binding, only: c_loc
      Use st_b200
      Include 'header'
      Real*8  Q(My,Mz,Mx,5), cfl_resv
      Real*8, Target :: Y(My,Mz,Mx,1)
      Integer step
      Call st_b200_init
      Call st_check(st_compute_tstep(st_ctx, Q, c_loc(Y), cfl_resv,
     .              step, Tstep), 'Compute_Tstep')
      Return
      End

*  One LDDRK4 call on /RKWORK/ Q and /SPECIES/ Y with the Tstep of
*  /TIME_RK/: ten stages on the GPU, then Q, Y and the /TRACK/ monitors
*  come back.  Advances time by 2*Tstep and step by one, as the
*  reference does.  QW and rYW start at zero in both, dQ and drYi are
*  overwritten before they are read, so they need no copying.
      Subroutine LDDRK4(time, step)
      Use iso_c_binding, only: c_int, c_loc
      Use st_b200
      Include 'header'
      Integer step
      Real*8  time
      Real*8  Q(My,Mz,Mx,5), dQ(My,Mz,Mx,5), QW(My,Mz,Mx,5)
      Real*8, Target :: Y(My,Mz,Mx,1)
      Real*8  drYi(My,Mz,Mx,1), rYW(My,Mz,Mx,1)
      Common /RKWORK/ Q, dQ, QW
      Common /SPECIES/ Y, drYi, rYW
      Real*8  mon(10)
      Integer(c_int) istep
      Call st_b200_init
      Call st_check(st_set_state(st_ctx, Q, c_loc(Y)), 'LDDRK4')
      Call st_check(st_set_tstep(st_ctx, Tstep), 'LDDRK4')
      istep = step
      Call st_check(st_lddrk4(st_ctx, time, istep), 'LDDRK4')
      step = istep
      Call st_check(st_get_state(st_ctx, Q, c_loc(Y)), 'LDDRK4')
      Call st_check(st_get_monitors(st_ctx, mon), 'LDDRK4')
      KE = mon(1)
      MomX = mon(2)
      MomY = mon(3)
      MomZ = mon(4)
      Mass_t = mon(5)
      e_t = mon(6)
      Entropy = mon(7)
      Entropy2 = mon(8)
      Return
      End

      Subroutine Compute_KE(Q)
      Include 'header'
      Real*8  Q(My,Mz,Mx,5), mon(10)
      Call st_b200_monitors(Q, mon)
      KE = mon(1)
      Return
      End

      Subroutine Compute_Mom(Q)
      Include 'header'
      Real*8  Q(My,Mz,Mx,5), mon(10)
      Call st_b200_monitors(Q, mon)
      MomX = mon(2)
      MomY = mon(3)
      MomZ = mon(4)
      Return
      End

      Subroutine Compute_Mass(Q, Y)
      Include 'header'
      Real*8  Q(My,Mz,Mx,5), Y(My,Mz,Mx,1), mon(10)
      Call st_b200_monitors(Q, mon)
      Mass_t = mon(5)
      Return
      End

      Subroutine Compute_Energy(Q)
      Include 'header'
      Real*8  Q(My,Mz,Mx,5), mon(10)
      Call st_b200_monitors(Q, mon)
      e_t = mon(6)
      Return
      End

      Subroutine Compute_Entropy(Q, Y)
      Include 'header'
      Real*8  Q(My,Mz,Mx,5), Y(My,Mz,Mx,1), mon(10)
      Call st_b200_monitors(Q, mon)
      Entropy = mon(7)
      Entropy2 = mon(8)
      Return
      End

************************************************************************
*  Output-side diagnostics on /RKWORK/ Q and /SPECIES/ Y:
*  Compute_Grad src/grad_sym.f:13, Compute_SRM_Stats pproc/pproc_mf.f:4,
*  Generate_Shock_Surface src/shock.f:163.  The first two upload the
*  state first, so they also serve the initial Output before any LDDRK4
*  call; the two statistics routines append the reference's records.
************************************************************************
      Subroutine Compute_Grad
      Use iso_c_binding, only: c_loc
      Use st_b200
      Include 'header'
      Real*8  Q(My,Mz,Mx,5), Grad(My,Mz,Mx,4)
      Common /RKWORK/ Q, Grad
      Real*8, Target :: Y(My,Mz,Mx,1)
      Real*8  drYi(My,Mz,Mx,1), rYW(My,Mz,Mx,1)
      Common /SPECIES/ Y, drYi, rYW
      Call st_b200_init
      Call st_check(st_set_state(st_ctx, Q, c_loc(Y)), 'Compute_Grad')
      Call st_check(st_compute_grad(st_ctx, Grad, MaxDil, Enstrophy),
     .              'Compute_Grad')
      Return
      End

      Subroutine Compute_SRM_Stats(step)
      Use iso_c_binding, only: c_int, c_loc
      Use st_b200
      Include 'header'
      Integer step
      Real*8  Q(My,Mz,Mx,5)
      Common /RKWORK/ Q
      Real*8, Target :: Y(My,Mz,Mx,1)
      Common /SPECIES/ Y
      Real*8  hmix, tke_total
      Real*8  Ur_shell_avg(N_avg), Y_shell_avg(N_avg)
      Integer(c_int) navg
      Call st_b200_init
      Call st_check(st_shell_count(st_ctx, navg), 'Compute_SRM_Stats')
      If (navg .NE. N_avg) Stop 'libst_b200: N_avg differs'
      Call st_check(st_set_state(st_ctx, Q, c_loc(Y)),
     .              'Compute_SRM_Stats')
      Call st_check(st_compute_srm_stats(st_ctx, hmix, tke_total,
     .              Ur_shell_avg, Y_shell_avg), 'Compute_SRM_Stats')
      OPEN(UNIT=7,FILE="mix_stats",FORM="FORMATTED",
     .     STATUS="UNKNOWN", POSITION="APPEND")
      WRITE(7,7) hmix, tke_total
      CLOSE(7)
 7    Format(1x, 2(ES13.5))
      Return
      End

*  (reads the context's /HYPER/ beta_hyper, as the reference reads its
*  COMMON copy)
      Subroutine Generate_Shock_Surface
      Use st_b200
      Include 'header'
      Real*8  rad_avg, rad_skew_rms
      Call st_b200_init
      Call st_check(st_generate_shock_surface(st_ctx, rad_avg,
     .              rad_skew_rms), 'Generate_Shock_Surface')
      OPEN(UNIT=7,FILE="shock_stats",FORM="FORMATTED",
     .     STATUS="UNKNOWN", POSITION="APPEND")
      WRITE(7,*) rad_avg, rad_skew_rms
      CLOSE(7)
      Return
      End

************************************************************************
*  MakePaddedArrays src/vis_silo_mf.f:440 (nfields = 11) and
*  Write_Visual_Silo src/vis_silo_mf.f:7 on /RKWORK/ Q and Grad (filled
*  by Compute_Grad), the context's gamma_eff and /SPECIES/ Y.  The
*  visual file is a binary legacy VTK rectilinear grid with the Silo
*  file's mesh, variables, cycle and time (no Silo library in this
*  build), written to vis_path/ddd/prefix.000.vtk, ddd the three digits
*  of cue_vis; Output advances cue_vis as before.
************************************************************************
      Subroutine MakePaddedArrays(W, xx, yy, zz, nfields)
      Use iso_c_binding, only: c_loc
      Use st_b200
      Include 'header'
      Integer nfields
      Real*8  W(My+1,Mz+1,Mx+1,nfields)
      Real*8  xx(Mx+1), yy(My+1), zz(Mz+1)
      Real*8  Q(My,Mz,Mx,5)
      Real*8, Target :: Grad(My,Mz,Mx,4)
      Common /RKWORK/ Q, Grad
      Real*8, Target :: Y(My,Mz,Mx,1)
      Real*8  drYi(My,Mz,Mx,1), rYW(My,Mz,Mx,1)
      Common /SPECIES/ Y, drYi, rYW
      If (nfields .NE. 11) Stop 'libst_b200: nfields is not 11'
      Call st_b200_init
      Call st_check(st_set_state(st_ctx, Q, c_loc(Y)),
     .              'MakePaddedArrays')
      Call st_check(st_make_padded_arrays(st_ctx, c_loc(Grad), W,
     .              xx, yy, zz), 'MakePaddedArrays')
      Return
      End

      Subroutine Write_Visual_Silo(time, step)
      Use iso_c_binding, only: c_loc, c_null_char
      Use st_b200
      Include 'header'
      Real*8  time
      Integer step
      Real*8  Q(My,Mz,Mx,5)
      Real*8, Target :: Grad(My,Mz,Mx,4)
      Common /RKWORK/ Q, Grad
      Real*8, Target :: Y(My,Mz,Mx,1)
      Real*8  drYi(My,Mz,Mx,1), rYW(My,Mz,Mx,1)
      Common /SPECIES/ Y, drYi, rYW
      Call st_b200_init
      Call st_check(st_set_state(st_ctx, Q, c_loc(Y)),
     .              'Write_Visual_Silo')
      Call st_check(st_write_visual(st_ctx, c_loc(Grad),
     .              trim(vis_path)//c_null_char,
     .              trim(prefix)//c_null_char, cue_vis, time, step),
     .              'Write_Visual_Silo')
      Return
      End
