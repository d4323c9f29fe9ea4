/*
 * st_b200.h - C ABI of the B200 (sm_100a) implementation of the per-stage
 * right-hand side and LDDRK4 stage update of the compact-difference
 * compressible Navier-Stokes shock-turbulence solver (two-species "_mf"
 * family: symmetry planes at x=y=z=0, one-sided closures, non-reflecting
 * outflow and sponge at the far faces).
 *
 * Conventions shared by every entry point
 *  - Arrays use the reference layout: Fortran F(My,Mz,Mx[,nvar]), i.e. y is
 *    the unit-stride index, then z, then x, then the variable index.  The
 *    conserved variables are ordered [rho*u, rho*v, rho*w, rho, rho*E].
 *  - Every array argument may be a host pointer or a device pointer; the
 *    library inspects each pointer (cudaPointerGetAttributes) and copies
 *    host data through device staging buffers.  Device pointers must belong
 *    to the context's device.
 *  - Every function returns 0 on success or a negative ST_E* code; nothing
 *    aborts the process.  st_last_error() gives a message for the last
 *    failure on a context.
 *  - The hidden state that the reference keeps in COMMON blocks
 *    (/RKWORK/ Q,dQ,QW; /SPECIES/ Y,drYi,rYW; /THERMO/ gamma_eff; /GRAD/;
 *    /HYPER/; /TIME_RK/ Tstep) lives on the device inside the context.
 *  - A context is not thread-safe; it owns one CUDA stream.
 *
 * Reference citations are path:line within the reference project.
 */
#ifndef ST_B200_H
#define ST_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define ST_OK            0
#define ST_E_ARG        -1  /* bad argument (null pointer, bad size, ...)  */
#define ST_E_NOMEM      -2  /* device or host allocation failed            */
#define ST_E_CUDA       -3  /* a CUDA runtime call failed                  */
#define ST_E_UNSUPPORTED -4 /* grid size or mode not supported             */
#define ST_E_NONFINITE  -5  /* non-finite value detected in the state      */
#define ST_E_NODEVICE   -6  /* no CUDA device / extension not usable       */

/* ---- run-time parameters --------------------------------------------- */
/* Carries what the reference fixes at compile time in src/header:5-10
 * (grid) and reads from srm.input.1 in src/define_nonperiodic_mf.f:17-84. */
typedef struct st_params {
    int    nx, ny, nz;          /* grid points (Mx=Nx, My=Ny, Mz=Nz: one GPU) */
    double x_leng, y_leng, z_leng;   /* domain lengths (period_x, ...)       */
    double x_start, y_start, z_start;
    double re;                  /* COMMON Re.  The _mf build never assigns it,
                                   so the molecular viscous/conductive term is
                                   computed but not added (src/rhsv_sym_mf.f:
                                   1420-1424).  re > 0 adds it.               */
    double re1, re2, pr, sc;
    double gamma1, gamma2, epsilon, vis_exp, bulk_ratio, t_ratio;
    int    hyper_param;         /* 1: artificial viscosity/diffusivity on     */
    int    rk_mode;             /* 0: second LDDRK4 loop with the unassigned
                                      (zero) alpha2/beta2 of the reference build
                                      (src/header:247-296);
                                   1: second loop reuses alpha1/beta1          */
    double cfl_cal;             /* target CFL (Compute_Tstep)                 */
    double c_beta_scale;        /* multiplies the dynamic bulk-viscosity
                                   coefficient; 1 reproduces the reference
                                   (src/hyper_dynamic_sym_mf.f:145-147)       */
    int    device;              /* CUDA device ordinal                        */
    int    family;              /* ST_FAMILY_MF: two-species symmetric octant
                                   (src/main_mf.f and the *_sym_mf, *_tri,
                                   filters_sym/asym routines);
                                   ST_FAMILY_PERIODIC: single-fluid triply
                                   periodic box (src/main.f with
                                   derivCDopt6_periodic.f, filters_periodic.f,
                                   rhsv_periodic_sf.f, hyper_dynamic.f,
                                   hyper_rhs.f, lddrk4_periodic_sf.f).  In the
                                   periodic family gamma1 is the fluid's gamma,
                                   re its Reynolds number (re1 is ignored), and
                                   x_leng = period_x*(nx-1)/nx as Define_Param
                                   sets it (src/define_periodic_sf.f:42).      */
    int    precision;           /* ST_PRECISION_FP64: every array in double
                                   (the reference's REAL*8 build);
                                   ST_PRECISION_FP32: the derivative, filter,
                                   artificial-viscosity and RHS intermediates
                                   (/GRAD/, /HYPER/, dQ, drYi and the scratch
                                   fields) are stored in float, while the state
                                   Q, Y, the LDDRK4 accumulators QW, rYW, the
                                   compact filter of the state and the pressure
                                   recovery (Fix_Pressure) stay double.  No
                                   counterpart in the reference.               */
} st_params;

#define ST_FAMILY_MF        0
#define ST_FAMILY_PERIODIC  1
#define ST_PRECISION_FP64   0
#define ST_PRECISION_FP32   1

typedef struct st_ctx st_ctx;

/* Parameters of the 1-D spherical-radial single-fluid family (the program
 * built by src/makefile_radial: rhsv_radial.f, derivCDopt6_radial.f,
 * filters_nonperiodic.f, hyper_radial.f, lddrk4_nonperiodic_sf.f).  Each
 * problem is one run of that program on a line of n points spanning -R..R. */
typedef struct st_radial_params {
    double gamma;               /* ratio of specific heats                    */
    double cfl_cal;             /* target CFL (Compute_Tstep)                 */
    int    hyper_param;         /* 1: artificial viscosity on                 */
    int    rk_mode;             /* 0: zero alpha2/beta2 (reference build);
                                   1: HHM 4-6 second-loop values               */
    int    device;              /* CUDA device ordinal                        */
} st_radial_params;

/* ---- context --------------------------------------------------------- */
/* Replaces Setup_Grid (src/grid.f:15-112), Setup_Derivatives_Sym/_Asym
 * (src/derivCDopt6_sym_tri.f:9-373, src/derivCDopt6_asym_tri.f:9-375) and
 * Init_Filters_sym/_asym (src/filters_sym.f:9-383, src/filters_asym.f:9-385):
 * builds the constant LU factors once per direction and allocates the
 * device mirrors of the COMMON blocks. */
int  st_create(const st_params *p, st_ctx **out);
int  st_destroy(st_ctx *c);
const char *st_last_error(const st_ctx *c);
const char *st_status_string(int status);
/* Fills p with the reference input values (init/srm.input.1:19-34) on an
 * n^3 unit-spacing grid. */
void st_default_params(st_params *p, int nx, int ny, int nz);

/* Resident state: /RKWORK/ Q(My,Mz,Mx,5) and /SPECIES/ Y(My,Mz,Mx).
 * st_set_state also clears QW, rYW, dQ, drYi (the reference zeroes QW and
 * rYW at the start of each LDDRK4 loop; dQ/drYi start as zero COMMON). */
int  st_set_state(st_ctx *c, const double *Q, const double *Y);
int  st_get_state(st_ctx *c, double *Q, double *Y);
int  st_set_tstep(st_ctx *c, double tstep);
int  st_get_tstep(st_ctx *c, double *tstep);
/* Copies a named COMMON array out of the context: "gamma_eff", "dux_dx",
 * "duy_dx", "duz_dx", "dux_dy", "duy_dy", "duz_dy", "dux_dz", "duy_dz",
 * "duz_dz", "dTdx", "dTdy", "dTdz", "beta_hyper", "visc_hyper", "k_hyper",
 * "D_hyper", "dQ" (5 fields), "QW" (5), "drYi", "rYW". */
int  st_get_common(st_ctx *c, const char *name, double *out);
int  st_set_common(st_ctx *c, const char *name, const double *in);

/* ---- line solvers ------------------------------------------------------ */
/* tridiagonal(A1,B1,C1,R,n,lot,nper,ncom), src/tridiagonal.f90:1-49; serial
 * paths :197-287.  Arrays (lot,n), lot fastest; R is overwritten.  nper=1
 * selects the periodic (bordered) solve.  General (per-line) coefficients. */
int  st_tridiagonal(st_ctx *c, const double *A, const double *B, const double *C,
                    double *R, int n, int lot, int nper);
/* pentadiagonal(A1..E1,R,n,lot,nper,ncom), src/pentadiagonal.f90:1-52;
 * serial paths :319-504. */
int  st_pentadiagonal(st_ctx *c, const double *A, const double *B, const double *C,
                      const double *D, const double *E, double *R,
                      int n, int lot, int nper);
/* No counterpart in the reference.  st_tridiagonal for callers that must not
 * allocate device memory (a host program that owns the device's memory through
 * its own pool, or a time-critical loop where a cudaMalloc may block on the
 * driver): the working copies of A and B live in a fixed static device array
 * instead of cudaMalloc'd buffers.
 * n*lot <= 262144 (ST_E_ARG beyond); A, B, C, R must be device arrays of the
 * context's device (ST_E_ARG for host arrays).  The first call on a device
 * looks the array up (cudaGetSymbolAddress) and should come before any stream
 * capture.  The array is shared per device: calls whose GPU work overlaps race
 * on it.  Returns once R is written. */
int  st_tridiagonal_noalloc(st_ctx *c, const double *A, const double *B, const double *C,
                            double *R, int n, int lot, int nper);

/* ---- compact derivatives ------------------------------------------------ */
/* DFDX_sym(F,dF,iadd,cadd) src/derivCDopt6_sym_tri.f:409-535, DFDY_sym :672,
 * DFDZ_sym :932; _asym variants src/derivCDopt6_asym_tri.f:412,670,930.
 * iadd=0: dF = cadd*dF/dx ; iadd=1: dF += cadd*dF/dx. */
int  st_dfdx_sym (st_ctx *c, const double *F, double *dF, int iadd, double cadd);
int  st_dfdy_sym (st_ctx *c, const double *F, double *dF, int iadd, double cadd);
int  st_dfdz_sym (st_ctx *c, const double *F, double *dF, int iadd, double cadd);
int  st_dfdx_asym(st_ctx *c, const double *F, double *dF, int iadd, double cadd);
int  st_dfdy_asym(st_ctx *c, const double *F, double *dF, int iadd, double cadd);
int  st_dfdz_asym(st_ctx *c, const double *F, double *dF, int iadd, double cadd);
/* D2FDX2_sym(F,dF,d2F,iadd) src/derivCDopt6_sym_tri.f:538-669, D2FDY2_sym
 * :801, D2FDZ2_sym :1062; _asym src/derivCDopt6_asym_tri.f:540,798,1061.
 * d2F = d2F/dx2; if iadd=1 also dF = dF/dx (overwritten). */
int  st_d2fdx2_sym (st_ctx *c, const double *F, double *dF, double *d2F, int iadd);
int  st_d2fdy2_sym (st_ctx *c, const double *F, double *dF, double *d2F, int iadd);
int  st_d2fdz2_sym (st_ctx *c, const double *F, double *dF, double *d2F, int iadd);
int  st_d2fdx2_asym(st_ctx *c, const double *F, double *dF, double *d2F, int iadd);
int  st_d2fdy2_asym(st_ctx *c, const double *F, double *dF, double *d2F, int iadd);
int  st_d2fdz2_asym(st_ctx *c, const double *F, double *dF, double *d2F, int iadd);
/* Periodic family (ST_FAMILY_PERIODIC contexts only): DFDX(F,dF,iadd,cadd)
 * src/derivCDopt6_periodic.f:164-278, DFDY :400, DFDZ :631 and
 * D2FDX2(F,dF,d2F,iadd) :281-397, D2FDY2 :515, D2FDZ2 :747.  Cyclic
 * sixth-order compact schemes with the FDL3DI constants. */
int  st_dfdx(st_ctx *c, const double *F, double *dF, int iadd, double cadd);
int  st_dfdy(st_ctx *c, const double *F, double *dF, int iadd, double cadd);
int  st_dfdz(st_ctx *c, const double *F, double *dF, int iadd, double cadd);
int  st_d2fdx2(st_ctx *c, const double *F, double *dF, double *d2F, int iadd);
int  st_d2fdy2(st_ctx *c, const double *F, double *dF, double *d2F, int iadd);
int  st_d2fdz2(st_ctx *c, const double *F, double *dF, double *d2F, int iadd);

/* ---- filters -------------------------------------------------------------- */
/* Compact_Filter(F,F0,N) src/filters_sym.f:398-432 (variable 1 filtered with
 * the x asym filter, 2 with y asym, 3 with z asym, all others sym; X then Y
 * then Z).  F0 may alias F. */
int  st_compact_filter(st_ctx *c, const double *F, double *F0, int nvar);
/* Compact_Filter_{X,Y,Z}_sym src/filters_sym.f:436-634,637-835,838-1034 and
 * _asym src/filters_asym.f:388-583,586-782,783-975.  F0 may alias F. */
int  st_compact_filter_x_sym (st_ctx *c, const double *F, double *F0);
int  st_compact_filter_y_sym (st_ctx *c, const double *F, double *F0);
int  st_compact_filter_z_sym (st_ctx *c, const double *F, double *F0);
int  st_compact_filter_x_asym(st_ctx *c, const double *F, double *F0);
int  st_compact_filter_y_asym(st_ctx *c, const double *F, double *F0);
int  st_compact_filter_z_asym(st_ctx *c, const double *F, double *F0);
/* Periodic family: Compact_Filter_{X,Y,Z} src/filters_periodic.f:115-250,
 * 254-389, 393-528 (cyclic eighth-order filter).  st_compact_filter and
 * st_gaussian_filter* serve both families. */
int  st_compact_filter_x(st_ctx *c, const double *F, double *F0);
int  st_compact_filter_y(st_ctx *c, const double *F, double *F0);
int  st_compact_filter_z(st_ctx *c, const double *F, double *F0);
/* Gaussian_Filter(F,Fg,N) src/filters_sym.f:1046-1071 and its X/Y/Z passes
 * :1076-1554 (coefficients rounded to float32, src/LES_header:153-157). */
int  st_gaussian_filter  (st_ctx *c, const double *F, double *Fg, int nvar);
int  st_gaussian_filter_x(st_ctx *c, const double *F, double *Fg);
int  st_gaussian_filter_y(st_ctx *c, const double *F, double *Fg);
int  st_gaussian_filter_z(st_ctx *c, const double *F, double *Fg);

/* ---- physics operators ------------------------------------------------------ */
/* Compute_gamma(Y) src/lddrk4_nonperiodic_mf.f:342-372 -> /THERMO/. */
int  st_compute_gamma(st_ctx *c, const double *Y);
/* RHS(Q,Qrhs,Y) src/rhsv_sym_mf.f:9-26 (RHS_x :37-481, RHS_yz :492-1428).
 * Overwrites Qrhs, writes /GRAD/, and (like the reference) rewrites the
 * momenta of Q as (m/rho)*rho. */
int  st_rhs(st_ctx *c, double *Q, double *Qrhs, const double *Y);
/* Compute_hyper(Q,Y) src/hyper_dynamic_sym_mf.f:166-334 -> /HYPER/. */
int  st_compute_hyper(st_ctx *c, const double *Q, const double *Y);
/* Hyper_RHS(Q,Qrhs,Y) src/hyper_rhs_sym_mf.f:12-500: Qrhs += artificial
 * stress/heat-flux divergence (calls Compute_hyper). */
int  st_hyper_rhs(st_ctx *c, const double *Q, double *Qrhs, const double *Y);
/* Species_RHS(Q,Qrhs,Y,Yrhs) src/species_rhs_sym.f:9-207. */
int  st_species_rhs(st_ctx *c, const double *Q, double *Qrhs, const double *Y,
                    double *Yrhs);
/* bc_RHS(Q,Qrhs,Y,Yrhs,time) src/bc_mf.f:11-463 (zeroes the normal momentum
 * of Q on the symmetry planes, overwrites the far-face rows). */
int  st_bc_rhs(st_ctx *c, double *Q, double *Qrhs, const double *Y, double *Yrhs,
               double time);
/* Sponge_Forcing(Q,Qrhs,Y,Yrhs) src/sponge_mf.f:7-127. */
int  st_sponge_forcing(st_ctx *c, const double *Q, double *Qrhs, const double *Y,
                       double *Yrhs);
/* Fix_Pressure(Q,Y) pproc/pproc_mf.f:190-233 (uses /THERMO/). */
int  st_fix_pressure(st_ctx *c, double *Q, const double *Y);
/* Compute_CFL(Q,cfl_stab,cfl_resv,step) src/lddrk4_nonperiodic_mf.f:7-66. */
int  st_compute_cfl(st_ctx *c, const double *Q, double *cfl_stab, double *cfl_resv);
/* Compute_Tstep(Q,Y,cfl_resv,step) src/lddrk4_nonperiodic_mf.f:75-160:
 * sets the context's Tstep and returns it in *tstep (may be NULL). */
int  st_compute_tstep(st_ctx *c, const double *Q, const double *Y, double cfl_resv,
                      int step, double *tstep);

/* ---- time integration on the resident state ------------------------------ */
/* LDDRK4(time,step) src/lddrk4_nonperiodic_mf.f:428-541 on /RKWORK/ and
 * /SPECIES/ held by the context (st_set_state), using the context Tstep.
 * Advances *time by 2*Tstep and *step by 1; the monitoring scalars
 * (KE, Mom, Mass, Energy, Entropy) are recomputed and can be read with
 * st_get_monitors. */
int  st_lddrk4(st_ctx *c, double *time, int *step);
/* One iteration of the main loop body of src/main_mf.f:137-145 (march_mode
 * 1): Compute_CFL, Compute_Tstep, LDDRK4.  dt stays on the device. */
int  st_step(st_ctx *c, double *time, int *step);
/* Compute_Mom/KE/Mass/Energy/Entropy src/lddrk4_nonperiodic_mf.f:168-327 on
 * the resident state: out[0..9] = KE, MomX, MomY, MomZ, Mass, Energy,
 * Entropy, Entropy2, cfl_resv of the last st_step, Tstep. */
int  st_get_monitors(st_ctx *c, double out[10]);
/* Synchronises the context stream. */
int  st_sync(st_ctx *c);
/* No reference counterpart: the main-loop step of st_step enqueued on the
 * context stream without waiting (time advances in device memory; st_set_time
 * sets it, st_get_time waits and reads it).  step is the caller's step
 * counter (Compute_Tstep uses it); from step 2 on the step replays a CUDA
 * graph captured on the first such call, so it costs one launch.  st_query
 * returns 1 when the context's work has finished, 0 while it runs. */
int  st_step_async(st_ctx *c, int step);
int  st_get_time(st_ctx *c, double *time);
int  st_set_time(st_ctx *c, double time);
int  st_query(st_ctx *c);
/* No reference counterpart: device bytes the context holds (COMMON mirrors,
 * scratch pool, tables); the pool grows during the first steps. */
int  st_memory(st_ctx *c, long long *bytes);

/* ---- Output-side diagnostics (_mf family) ----------------------------------
 * The per-step calls of Output (src/out_mf.f:671-705) on the context's state.
 * Compute_Grad src/grad_sym.f:13-120: Grad (4 fields w_x, w_y, w_z,
 * dilatation, or NULL), MaxDil = max|dilatation| and Enstrophy =
 * 0.5*sum(|w|^2)/(Nx*Ny*Nz) of /TRACK/; the nine velocity derivatives are
 * left in /GRAD/ as the reference leaves them (FP64 mode). */
int  st_compute_grad(st_ctx *c, double *Grad, double *maxdil, double *enstrophy);
/* Compute_SRM_Stats pproc/pproc_mf.f:4-186 (with Compute_shell_avg
 * src/auxiliary_mf.f:266-332): the mix_stats record (mixing width hmix,
 * mean turbulent kinetic energy tke_total) and, when not NULL, the N_avg
 * shell averages of the radial velocity and of Y (N_avg from
 * st_shell_count, src/header:14).  Cells beyond the last tke bin, which the
 * reference leaves unassigned, contribute 0. */
int  st_shell_count(st_ctx *c, int *n_avg);
int  st_compute_srm_stats(st_ctx *c, double *hmix, double *tke_total, double *ur_avg, double *y_avg);
/* Generate_Shock_Surface src/shock.f:163-260: the shock_stats record
 * (mean distance of the cells with beta_hyper > 0.1*max from their centroid,
 * and sqrt(sum of squared deviations)/(n*mean)). */
int  st_generate_shock_surface(st_ctx *c, double *rad_avg, double *rad_skew_rms);
/* MakePaddedArrays src/vis_silo_mf.f:440-689 (one rank): W =
 * W(My+1,Mz+1,Mx+1,11), the fields u, v, w, rho, P (:494-510), the four
 * Grad fields, gamma_eff and Y at the nodes of the grid padded by one node
 * per direction (each padding node a copy of the last node of its
 * direction, :640-686); xx/yy/zz (Mx+1, My+1, Mz+1, each may be NULL) the
 * node coordinates plus one spacing (:486-491).  Grad: the 4 fields of
 * st_compute_grad (/RKWORK/ Grad), or NULL to compute them first. */
int  st_make_padded_arrays(st_ctx *c, const double *Grad, double *W, double *xx, double *yy, double *zz);
/* Write_Visual_Silo src/vis_silo_mf.f:7-277 (one rank).  The same mesh
 * (collinear, axes y, z, x of sizes My+1, Mz+1, Mx+1), the eleven
 * node-centred variables rho, U, V, W, P, omx, omy, omz, dil, gamma, Y of
 * st_make_padded_arrays, the cycle (step) and the time, written as one
 * binary legacy VTK rectilinear-grid file (the Silo library is not part of
 * this build) to <vis_path>/<ddd>/<prefix>.000.vtk, ddd the three digits of
 * cue_vis (0..999); the directory is created as make_dir_ (src/dirs.c)
 * creates it.  Grad as for st_make_padded_arrays. */
int  st_write_visual(st_ctx *c, const double *Grad, const char *vis_path, const char *prefix, int cue_vis,
                     double time, int step);

/* ---- 1-D spherical-radial family, batched ---------------------------------
 * Many independent problems, each one run of the reference's radial program
 * (src/makefile_radial) on a line of n[k] points, 16 <= n[k] <= 4096, of
 * length x_leng[k] spanning -x_leng/2..x_leng/2.  Packed arrays: problem k's
 * state block Q of 3*n[k] values (u_r, rho, s = P/rho^gamma; the reference's
 * Q(:,1), Q(:,4), Q(:,5)) starts at 3*sum(n[j], j<k); single fields of the
 * line operators start at sum(n[j], j<k).  Host or device arrays. */
typedef struct st_radial st_radial;
int  st_radial_create(const st_radial_params *p, int nprob, const int *n, const double *x_leng,
                      st_radial **out);
int  st_radial_destroy(st_radial *h);
const char *st_radial_last_error(const st_radial *h);
int  st_radial_num_points(const st_radial *h, long long *npts);
/* Sets every problem's state (time and step counters restart at zero). */
int  st_radial_set_state(st_radial *h, const double *Q);
int  st_radial_get_state(st_radial *h, double *Q);
/* /HYPER/ of every problem: 2*n[k] values (beta_hyper, visc_hyper). */
int  st_radial_get_hyper(st_radial *h, double *hyp);
int  st_radial_get_time(st_radial *h, double *time, int *step);
/* nsteps iterations of the main loop (src/main.f:129-136: Compute_CFL,
 * Compute_Tstep, LDDRK4 src/lddrk4_nonperiodic_sf.f:376-468) of every
 * problem, each with its own time step, in one persistent launch per problem
 * class; a problem at step 0 first gets Compute_hyper (src/main.f:100).
 * st_radial_step waits for completion, st_radial_step_async does not. */
int  st_radial_step(st_radial *h, int nsteps);
int  st_radial_step_async(st_radial *h, int nsteps);
int  st_radial_set_stream(st_radial *h, void *stream);
/* Kernel configuration per problem class (n <= 1024, n > 1024): index 0..2
 * into (64,16)/(128,8)/(256,4) and (256,16)/(512,8)/(1024,4) threads x rows
 * per thread.  st_radial_tune times every candidate for one step of the
 * current state (which it leaves unchanged) and keeps the fastest; ms[0]
 * and ms[1] get the best times (ms) of the long and the short class.  No
 * reference counterpart. */
int  st_radial_config(st_radial *h, int *cfg_short, int *cfg_long, int set);
int  st_radial_tune(st_radial *h, double ms[2]);
/* Line operators of every problem: DFDX src/derivCDopt6_radial.f:637-791,
 * D2FDX2 :794-953, Compact_Filter_X src/filters_nonperiodic.f:418-619,
 * Gaussian_Filter_X :1055-1224, RHS (RHS_r src/rhsv_radial.f:30-157) and
 * RHS + Hyper_RHS (src/hyper_radial.f:75-187; refreshes /HYPER/). */
int  st_radial_dfdx(st_radial *h, const double *F, double *dF, int iadd, double cadd);
int  st_radial_d2fdx2(st_radial *h, const double *F, double *dF, double *d2F, int iadd);
int  st_radial_compact_filter_x(st_radial *h, const double *F, double *F0);
int  st_radial_gaussian_filter_x(st_radial *h, const double *F, double *Fg);
int  st_radial_rhs(st_radial *h, const double *Q, double *Qrhs);
int  st_radial_rhs_hyper(st_radial *h, const double *Q, double *Qrhs);
int  st_radial_launch_count(const st_radial *h, long long *count);

/* ---- batches of same-size cases (no reference counterpart) ----------------
 * A batch context holds ncase independent cases of one grid and one set of
 * parameters (serving: same-size requests stepped together).  On the device
 * every field holds ncase consecutive blocks of Nx*Ny*Nz cells, so each line
 * and pointwise kernel of a step is one launch over all active cases, not
 * one per case.  Cases 0 .. nactive-1 are stepped; each keeps its own time
 * step, time and step count, so cases that started at different times
 * advance together and each gives the same results as alone.  The
 * single-grid entry points above return ST_E_UNSUPPORTED on a batch
 * context.
 * st_case_start uploads case k's state (host or device arrays in the
 * reference layout), sets its time and step count 0 and runs its set-up
 * (Compute_gamma and Compute_hyper, src/main_mf.f:100-101).  st_case_get
 * reads a case's state, time and step count.  st_case_move copies case src
 * over case dst (to keep the active cases in front when one finishes).
 * st_batch_step_async enqueues one main-loop step (Compute_CFL,
 * Compute_Tstep, LDDRK4) of every active case: a CUDA graph per active
 * count, captured on its first use. */
int  st_create_batch(const st_params *p, int ncase, st_ctx **out);
int  st_batch_info(st_ctx *c, int *ncase, int *nactive);
int  st_set_active(st_ctx *c, int nactive);
int  st_case_start(st_ctx *c, int k, const double *Q, const double *Y, double time);
int  st_case_get(st_ctx *c, int k, double *Q, double *Y, double *time, int *step);
int  st_case_move(st_ctx *c, int src, int dst);
int  st_batch_step_async(st_ctx *c);

/* ---- streams, instrumentation (no reference counterpart) ------------------ */
/* Runs the context's work on a caller-owned cudaStream_t (NULL restores the
 * context's own stream), so callers can order and time it with their own
 * events; st_get_stream returns the stream in use. */
int  st_set_stream(st_ctx *c, void *stream);
int  st_get_stream(st_ctx *c, void **stream);
/* Per-kernel CUDA-event timing of every launch on the context stream while
 * enabled; st_profile_report writes a JSON object
 * {"kernel": {"launches": n, "ms": total, "bytes": algorithmic bytes}} and
 * clears the records.  st_launch_count returns the number of kernels the
 * context has launched since creation. */
int  st_profile(st_ctx *c, int enable);
int  st_profile_report(st_ctx *c, char *buf, int buflen);
int  st_launch_count(st_ctx *c, long long *count);

#ifdef __cplusplus
}
#endif
#endif /* ST_B200_H */
