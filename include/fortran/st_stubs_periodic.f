************************************************************************
*  st_stubs_periodic.f - reference-named wrappers over libst_b200 for
*  the single-fluid triply periodic build (src/makefile_periodic:
*  src/main.f with derivCDopt6_periodic.f, filters_periodic.f,
*  rhsv_periodic_sf.f, hyper_dynamic.f, hyper_rhs.f, lddrk4_periodic_sf.f).
*
*  Same rules as st_stubs_mf.f: reference names and argument lists, one
*  context (family ST_FAMILY_PERIODIC) for the COMMON blocks, a nonzero
*  status stops the run, Px = Py = Pz = 1.  The family has no species:
*  the library's Y arguments get c_null_ptr.
************************************************************************

*  Creates the context once, from Define_Param (src/define_periodic_sf.f)
*  and Setup_Grid (src/grid.f:15-112): gamma is the fluid's ratio of
*  specific heats, Re its Reynolds number.
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
      p%re1 = Re
      p%pr = Pr
      p%gamma1 = gamma
      p%vis_exp = vis_exp
      p%bulk_ratio = bulk_ratio
      p%hyper_param = hyper_param
*  rk_mode 0: the second LDDRK4 loop with the reference build's
*  unassigned (zero) alpha2/beta2
      p%rk_mode = 0
      p%cfl_cal = cfl_cal
      p%c_beta_scale = 1.0D0
      p%device = 0
      p%family = 1
      p%precision = 0
      Call st_check(st_create(p, st_ctx), 'st_create')

      Return

      End

*  /TRACK/ monitors of Q as the context computes them:
*  mon = KE, MomX, MomY, MomZ, Mass, Energy, Entropy
      Subroutine st_b200_monitors(Q, mon)

      Use iso_c_binding, only: c_null_ptr
      Use st_b200

      Include 'header'

      Real*8  Q(My,Mz,Mx,5), mon(10)

      Call st_b200_init
      Call st_check(st_set_state(st_ctx, Q, c_null_ptr), 'monitors')
      Call st_check(st_get_monitors(st_ctx, mon), 'monitors')

      Return

      End

************************************************************************
*  Set-up: Setup_Derivatives src/derivCDopt6_periodic.f:9, Init_Filters
*  src/filters_periodic.f:9.
************************************************************************
      Subroutine Setup_Derivatives
      Call st_b200_init
      Return
      End

      Subroutine Init_Filters
      Call st_b200_init
      Return
      End

************************************************************************
*  Cyclic compact derivatives: DFDX, D2FDX2, DFDY, D2FDY2, DFDZ, D2FDZ2
*  src/derivCDopt6_periodic.f:164,281,400,515,631,747.
************************************************************************
      Subroutine DFDX(F, dF, iadd, cadd)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), dF(My,Mz,Mx), cadd
      Integer iadd
      Call st_check(st_dfdx(st_ctx, F, dF, iadd, cadd), 'DFDX')
      Return
      End

      Subroutine DFDY(F, dF, iadd, cadd)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), dF(My,Mz,Mx), cadd
      Integer iadd
      Call st_check(st_dfdy(st_ctx, F, dF, iadd, cadd), 'DFDY')
      Return
      End

      Subroutine DFDZ(F, dF, iadd, cadd)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), dF(My,Mz,Mx), cadd
      Integer iadd
      Call st_check(st_dfdz(st_ctx, F, dF, iadd, cadd), 'DFDZ')
      Return
      End

      Subroutine D2FDX2(F, dF, d2F, iadd)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), dF(My,Mz,Mx), d2F(My,Mz,Mx)
      Integer iadd
      Call st_check(st_d2fdx2(st_ctx, F, dF, d2F, iadd), 'D2FDX2')
      Return
      End

      Subroutine D2FDY2(F, dF, d2F, iadd)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), dF(My,Mz,Mx), d2F(My,Mz,Mx)
      Integer iadd
      Call st_check(st_d2fdy2(st_ctx, F, dF, d2F, iadd), 'D2FDY2')
      Return
      End

      Subroutine D2FDZ2(F, dF, d2F, iadd)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), dF(My,Mz,Mx), d2F(My,Mz,Mx)
      Integer iadd
      Call st_check(st_d2fdz2(st_ctx, F, dF, d2F, iadd), 'D2FDZ2')
      Return
      End

************************************************************************
*  Line solvers, as in st_stubs_mf.f.
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
*  Filters: Compact_Filter src/filters_periodic.f:90, Compact_Filter_X/
*  Y/Z :115,254,393, Gaussian_Filter :540, Gaussian_Filter_X/Y/Z
*  :565,680,793.
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

      Subroutine Compact_Filter_X(F, F0)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), F0(My,Mz,Mx)
      Call st_check(st_compact_filter_x(st_ctx, F, F0),
     .              'Compact_Filter_X')
      Return
      End

      Subroutine Compact_Filter_Y(F, F0)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), F0(My,Mz,Mx)
      Call st_check(st_compact_filter_y(st_ctx, F, F0),
     .              'Compact_Filter_Y')
      Return
      End

      Subroutine Compact_Filter_Z(F, F0)
      Use st_b200
      Include 'header'
      Real*8  F(My,Mz,Mx), F0(My,Mz,Mx)
      Call st_check(st_compact_filter_z(st_ctx, F, F0),
     .              'Compact_Filter_Z')
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
*  Physics: RHS src/rhsv_periodic_sf.f:9, Compute_hyper
*  src/hyper_dynamic.f:173, Hyper_RHS src/hyper_rhs.f:12, Fix_Pressure
*  src/lddrk4_periodic_sf.f:436.
************************************************************************
      Subroutine RHS(Q, Qrhs)
      Use iso_c_binding, only: c_null_ptr
      Use st_b200
      Include 'header'
      Real*8  Q(My,Mz,Mx,5), Qrhs(My,Mz,Mx,5)
      Call st_check(st_rhs(st_ctx, Q, Qrhs, c_null_ptr), 'RHS')
      Return
      End

*  Also refreshes beta_hyper, visc_hyper and k_hyper, the first three
*  arrays of the reference's /HYPER/.
      Subroutine Compute_hyper(Q)
      Use iso_c_binding, only: c_null_ptr, c_null_char
      Use st_b200
      Include 'header'
      Real*8  Q(My,Mz,Mx,5)
      Real*8  H(My,Mz,Mx,3)
      Common /HYPER/ H
      Call st_b200_init
      Call st_check(st_compute_hyper(st_ctx, Q, c_null_ptr),
     .              'Compute_hyper')
      Call st_check(st_get_common(st_ctx, 'beta_hyper'//c_null_char,
     .              H(1,1,1,1)), 'Compute_hyper')
      Call st_check(st_get_common(st_ctx, 'visc_hyper'//c_null_char,
     .              H(1,1,1,2)), 'Compute_hyper')
      Call st_check(st_get_common(st_ctx, 'k_hyper'//c_null_char,
     .              H(1,1,1,3)), 'Compute_hyper')
      Return
      End

      Subroutine Hyper_RHS(Q, Qrhs)
      Use iso_c_binding, only: c_null_ptr
      Use st_b200
      Include 'header'
      Real*8  Q(My,Mz,Mx,5), Qrhs(My,Mz,Mx,5)
      Call st_check(st_hyper_rhs(st_ctx, Q, Qrhs, c_null_ptr),
     .              'Hyper_RHS')
      Return
      End

      Subroutine Fix_Pressure(Q)
      Use iso_c_binding, only: c_null_ptr
      Use st_b200
      Include 'header'
      Real*8  Q(My,Mz,Mx,5)
      Call st_check(st_fix_pressure(st_ctx, Q, c_null_ptr),
     .              'Fix_Pressure')
      Return
      End

************************************************************************
*  Time step and integration: Compute_CFL, Compute_Tstep, LDDRK4
*  src/lddrk4_periodic_sf.f:7,74,311 and the monitors
*  Compute_KE/Mom/Mass/Energy/Entropy :153,201,228,247,268.
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

      Subroutine Compute_Tstep(Q, cfl_resv, step)
      Use iso_c_binding, only: c_null_ptr
      Use st_b200
      Include 'header'
      Real*8  Q(My,Mz,Mx,5), cfl_resv
      Integer step
      Call st_b200_init
      Call st_check(st_compute_tstep(st_ctx, Q, c_null_ptr, cfl_resv,
     .              step, Tstep), 'Compute_Tstep')
      Return
      End

*  One LDDRK4 call (5 + 6 stages) on /RKWORK/ Q with the Tstep of
*  /TIME_RK/; Q and the /TRACK/ monitors come back.
      Subroutine LDDRK4(time, step)
      Use iso_c_binding, only: c_int, c_null_ptr
      Use st_b200
      Include 'header'
      Integer step
      Real*8  time
      Real*8  Q(My,Mz,Mx,5), dQ(My,Mz,Mx,5), QW(My,Mz,Mx,5)
      Common /RKWORK/ Q, dQ, QW
      Real*8  mon(10)
      Integer(c_int) istep
      Call st_b200_init
      Call st_check(st_set_state(st_ctx, Q, c_null_ptr), 'LDDRK4')
      Call st_check(st_set_tstep(st_ctx, Tstep), 'LDDRK4')
      istep = step
      Call st_check(st_lddrk4(st_ctx, time, istep), 'LDDRK4')
      step = istep
      Call st_check(st_get_state(st_ctx, Q, c_null_ptr), 'LDDRK4')
      Call st_check(st_get_monitors(st_ctx, mon), 'LDDRK4')
      KE = mon(1)
      MomX = mon(2)
      MomY = mon(3)
      MomZ = mon(4)
      Mass_t = mon(5)
      e_t = mon(6)
      Entropy = mon(7)
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

      Subroutine Compute_Mass(Q)
      Include 'header'
      Real*8  Q(My,Mz,Mx,5), mon(10)
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

      Subroutine Compute_Entropy(Q)
      Include 'header'
      Real*8  Q(My,Mz,Mx,5), mon(10)
      Call st_b200_monitors(Q, mon)
      Entropy = mon(7)
      Return
      End
