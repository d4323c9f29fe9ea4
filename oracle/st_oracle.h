/*
 * st_oracle.h - CPU oracle for the per-stage RHS / LDDRK4 path.
 *
 * TEST INFRASTRUCTURE ONLY: the GPU results are checked against this plain-C restatement of
 * the reference Fortran (two-species "_mf" family) used by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg.  Nothing in
 * the product path links or calls it.
 *
 * Parity status: unpinned by the reference's own tests.  The reference ships
 * no test suite, no golden vectors and no fixtures, and it is Fortran+MPI
 * with no Fortran compiler in this image, so it cannot be built and run
 * here.  The restatement is pinned instead by analytic known-answer tests
 * (polynomial exactness of the compact schemes, filter transfer function,
 * dense-LU checks of the line solvers) and by the committed fixtures that it
 * generates for the GPU tests.
 *
 * Every function names the reference routine (file:line) it restates.
 * Arrays use the reference layout F(My,Mz,Mx[,n]) with y fastest.
 */
#ifndef ST_ORACLE_H
#define ST_ORACLE_H
#include "../include/st_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc orc;

orc *orc_create(const st_params *p);
void orc_destroy(orc *c);
void orc_set_threads(int n);

/* state and COMMON access (names as in st_get_common) */
void orc_set_state(orc *c, const double *Q, const double *Y);
void orc_get_state(orc *c, double *Q, double *Y);
void orc_set_tstep(orc *c, double t);
double orc_get_tstep(orc *c);
int  orc_get_common(orc *c, const char *name, double *out);
int  orc_set_common(orc *c, const char *name, const double *in);

/* line solvers with general (lot,n) coefficients */
void orc_tridiagonal(const double *A, const double *B, const double *C, double *R,
                     int n, int lot, int nper);
void orc_pentadiagonal(const double *A, const double *B, const double *C,
                       const double *D, const double *E, double *R,
                       int n, int lot, int nper);

/* dir: 0=x 1=y 2=z ; asym: 0 sym, 1 asym */
void orc_dfd(orc *c, int dir, int asym, const double *F, double *dF, int iadd, double cadd);
void orc_d2fd2(orc *c, int dir, int asym, const double *F, double *dF, double *d2F, int iadd);
void orc_filter(orc *c, int dir, int asym, const double *F, double *F0);
void orc_compact_filter(orc *c, const double *F, double *F0, int nvar);
void orc_gauss(orc *c, int dir, const double *F, double *Fg);
void orc_gaussian_filter(orc *c, const double *F, double *Fg, int nvar);

void orc_compute_gamma(orc *c, const double *Y);
void orc_rhs(orc *c, double *Q, double *Qrhs, const double *Y);
void orc_compute_hyper(orc *c, const double *Q, const double *Y);
void orc_hyper_rhs(orc *c, const double *Q, double *Qrhs, const double *Y);
void orc_species_rhs(orc *c, const double *Q, double *Qrhs, const double *Y, double *Yrhs);
void orc_bc_rhs(orc *c, double *Q, double *Qrhs, const double *Y, double *Yrhs, double time);
void orc_sponge_forcing(orc *c, const double *Q, double *Qrhs, const double *Y, double *Yrhs);
void orc_fix_pressure(orc *c, double *Q, const double *Y);
void orc_compute_cfl(orc *c, const double *Q, double *cfl_stab, double *cfl_resv);
double orc_compute_tstep(orc *c, const double *Q, const double *Y, double cfl_resv, int step);
void orc_lddrk4(orc *c, double *time, int *step);
void orc_step(orc *c, double *time, int *step);
void orc_get_monitors(orc *c, double out[10]);
/* Output-side diagnostics: Compute_Grad, Compute_SRM_Stats, Generate_Shock_Surface */
void orc_compute_grad(orc *c, double *Grad, double *maxdil, double *enstrophy);
int  orc_shell_count(const orc *c);
void orc_compute_srm_stats(orc *c, double *hmix, double *tke_total, double *ur_avg, double *y_avg);
void orc_shock_surface(orc *c, double *rad_avg, double *rad_skew_rms);
void orc_graph_bytes_reset(void);
double orc_graph_bytes(void);
void orc_make_padded_arrays(orc *c, const double *Grad, double *W, double *xx, double *yy, double *zz);

/* 1-D spherical-radial family (st_oracle_radial.c).  Q = (u_r, rho, s)
 * with s = P/rho^gamma, n points each; hyp = (beta_hyper, visc_hyper). */
void orc_rad_radius(int n, double x_leng, double *rad);
void orc_rad_dfdx(int n, double x_leng, const double *F, double *dF, int iadd, double cadd);
void orc_rad_d2fdx2(int n, double x_leng, const double *F, double *dF, double *d2F, int iadd);
void orc_rad_filter(int n, const double *F, double *F0);
void orc_rad_gauss(int n, const double *F, double *Fg);
void orc_rad_rhs(const st_radial_params *p, int n, double x_leng, const double *Q, double *Qrhs);
void orc_rad_compute_hyper(const st_radial_params *p, int n, double x_leng, const double *Q, double *hyp);
void orc_rad_hyper_rhs(const st_radial_params *p, int n, double x_leng, const double *Q, double *Qrhs,
                       double *hyp);
double orc_rad_tstep(const st_radial_params *p, int n, double x_leng, const double *Q, const double *hyp,
                     double *cfl_stab, double *cfl_resv);
void orc_rad_lddrk4(const st_radial_params *p, int n, double x_leng, double *Q, double *hyp, double dt,
                    double *time, int *step);
double orc_rad_step(const st_radial_params *p, int n, double x_leng, double *Q, double *hyp, double *time,
                    int *step);
void orc_rad_batch(const st_radial_params *p, int nprob, const int *n, const long long *off,
                   const double *x_leng, double *Q, double *hyp, double *time, int *step, int nsteps);

#ifdef __cplusplus
}
#endif
#endif
