/*
 * st_oracle.c - CPU oracle (TEST INFRASTRUCTURE, GPU results are checked against it; see
 * st_oracle.h).  Plain-C restatement of the reference's two-species "_mf"
 * right-hand side and LDDRK4 path, keeping the reference's expression
 * evaluation order (Fortran left-to-right) so that it reproduces the
 * reference's rounding, including the float32-typed quantities:
 *   - Gaussian filter coefficients are implicit REAL PARAMETERs
 *     (src/LES_header:153-157),
 *   - the sponge ramp ratio is a REAL/REAL quotient (src/sponge_mf.f:85-105),
 *   - fac1 in Compute_Tstep is implicit REAL (src/lddrk4_nonperiodic_mf.f:118).
 * Build with -ffp-contract=off so that no multiply-add is fused.
 *
 * Parity unpinned (no reference tests, golden vectors or Fortran compiler);
 * pinned by analytic known-answer tests in tests/.
 */
#include "st_oracle.h"
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define TINY ((double)FLT_MIN) /* tiny(1.0): single-precision tiny, src/tridiagonal.f90:275 */

/* ---- scheme constants (src/header:173-204, src/LES_header:107-157) ---- */
static const double a1_p6 = 14.0 / 18.0, b1_p6 = 1.0 / 36.0, alpha1_p6 = 1.0 / 3.0;
static const double a2_p6 = 12.0 / 11.0, b2_p6 = 3.0 / 44.0, alpha2_p6 = 2.0 / 11.0;
#define C2_P6 (2.0 * (a2_p6 + b2_p6))
static const double closure1 = 5.0 / 9.0, closure2 = 1.0 / 18.0;

static const double alpha_f4 = 6.6624e-01, beta_f4 = 1.6688e-01;
static const double a0_f4 = 9.9965e-01, a1_f4 = 0.66652, a2_f4 = 0.16674,
                    a3_f4 = 4.0e-05, a4_f4 = -5.0e-06;
static const double bndy_alpha = 0.45;

/* RK coefficients, src/header:284-296 */
static const double alpha1_rk[5] = {0.0, -4.801594388477952e-01, -1.404247195200064e+00,
                                    -2.016477077503357e+00, -1.056444269767207e+00};
static const double beta1_rk[5] = {1.028639988104959e-01, 7.408540575766301e-01,
                                   7.426530946683799e-01, 4.694937902357905e-01,
                                   1.881733382887932e-01};
static const double c1_rk[5] = {0.0, 1.028639988104959e-01, 4.879899878330192e-01,
                                6.885177231562036e-01, 9.023816453077341e-01};

/* CFL constants src/header:237-240 */
static const double k_max = 2.478, k_hug = 2.199;

struct bndyc {
    double c1[6], c2[6], c3[3], c4[4]; /* closure1 a1..a5, closure2 a0..a5, closure3 a0..a2, closure4 a0..a3 */
};

typedef struct { double *a, *b, *c; } tri_lhs;            /* 1-D rows, length n */
typedef struct { double *cst, *bp, *up; } tri_fac;         /* factorisation + upper diagonal */
typedef struct { double *A, *B, *C, *D, *E; } pen_lhs;
typedef struct { double *k1, *k2, k3, *Cp, *Dp, *E; } pen_fac;

struct orc {
    st_params p;
    int M[3];          /* Mx, My, Mz */
    size_t n3;
    double s1[3], s2[3];
    double DX, DY, DZ;
    double Re1_inv, Re2_inv, Pr_inv, Sc_inv;
    double Tstep;
    tri_fac d1[3][2], d2[3][2];   /* [dir][asym] */
    pen_fac fl[3][2];
    struct bndyc bc;
    float ag[5];                  /* Gaussian coefficients (REAL*4) */
    /* COMMON blocks */
    double *Q, *dQ, *QW, *Y, *drYi, *rYW, *gamma_eff;
    double *grad[12];
    double *hyp[4];               /* beta, visc, k, D */
    double *dYd[3];
    double mon[10];
    double last_cfl_resv;
};

enum { G_DUX_DX, G_DUY_DX, G_DUZ_DX, G_DUX_DY, G_DUY_DY, G_DUZ_DY,
       G_DUX_DZ, G_DUY_DZ, G_DUZ_DZ, G_DTDX, G_DTDY, G_DTDZ };
enum { H_BETA, H_VISC, H_K, H_D };

static double *dalloc(size_t n) {
    double *p = (double *)calloc(n ? n : 1, sizeof(double));
    if (!p) { fprintf(stderr, "oracle: out of memory\n"); abort(); }
    return p;
}
#define NEWF(c) dalloc((c)->n3)
#define IX(c, j, k, i) ((size_t)(j) + (size_t)(c)->M[1] * ((size_t)(k) + (size_t)(c)->M[2] * (size_t)(i)))

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ---- line geometry ------------------------------------------------------ */
static void line_geom(const orc *c, int d, int *n, size_t *st, size_t *lot) {
    int My = c->M[1], Mz = c->M[2], Mx = c->M[0];
    if (d == 0) { *n = Mx; *st = (size_t)My * Mz; *lot = (size_t)My * Mz; }
    else if (d == 1) { *n = My; *st = 1; *lot = (size_t)Mz * Mx; }
    else { *n = Mz; *st = (size_t)My; *lot = (size_t)Mx * My; }
}
static size_t line_base(const orc *c, int d, size_t L) {
    size_t My = c->M[1], Mz = c->M[2];
    if (d == 0) return L;                              /* L = j + My*k */
    if (d == 1) return My * L;                         /* L = k + Mz*i */
    return (L % My) + My * Mz * (L / My);              /* L = j + My*i */
}

/* ---- factorisations (same operation order as the serial solvers) ------- */
/* tridiagonal_serial, src/tridiagonal.f90:264-287 */
static tri_fac tri_factor(const double *a, const double *b, const double *c, int n) {
    tri_fac f;
    f.cst = dalloc(n); f.bp = dalloc(n); f.up = dalloc(n);
    memcpy(f.up, c, n * sizeof(double));
    f.bp[0] = b[0];
    for (int i = 1; i < n; i++) {
        f.cst[i] = a[i] / (f.bp[i - 1] + TINY);
        f.bp[i] = b[i] - c[i - 1] * f.cst[i];
    }
    return f;
}
/* per-line part of tridiagonal_serial on W(lot,n) (lot fastest) */
static void tri_apply(const tri_fac *f, double *W, int n, size_t lot) {
    const double *c = f->up;
    const size_t CH = 256;
#pragma omp parallel for schedule(static)
    for (size_t L0 = 0; L0 < lot; L0 += CH) {
        size_t L1 = L0 + CH < lot ? L0 + CH : lot;
        for (int i = 1; i < n; i++) {
            double cs = f->cst[i];
            double *r = W + (size_t)i * lot, *rm = W + (size_t)(i - 1) * lot;
            for (size_t L = L0; L < L1; L++) r[L] = r[L] - rm[L] * cs;
        }
        {
            double *r = W + (size_t)(n - 1) * lot, bn = f->bp[n - 1];
            for (size_t L = L0; L < L1; L++) r[L] = r[L] / bn;
        }
        for (int i = n - 2; i >= 0; i--) {
            double ci = c[i], den = f->bp[i] + TINY;
            double *r = W + (size_t)i * lot, *rp = W + (size_t)(i + 1) * lot;
            for (size_t L = L0; L < L1; L++) r[L] = (r[L] - ci * rp[L]) / den;
        }
    }
}
/* pentadiagonal_serial, src/pentadiagonal.f90:319-374 (n >= 3 path) */
static pen_fac pen_factor(const pen_lhs *m, int n) {
    pen_fac f;
    double *B = dalloc(n), *C = dalloc(n), *D = dalloc(n);
    memcpy(B, m->B, n * sizeof(double)); memcpy(C, m->C, n * sizeof(double));
    memcpy(D, m->D, n * sizeof(double));
    f.k1 = dalloc(n); f.k2 = dalloc(n); f.E = dalloc(n);
    memcpy(f.E, m->E, n * sizeof(double));
    for (int i = 0; i <= n - 3; i++) {
        double k1 = B[i + 1] / (C[i] + TINY);
        C[i + 1] = C[i + 1] - D[i] * k1;
        D[i + 1] = D[i + 1] - m->E[i] * k1;
        double k2 = m->A[i + 2] / (C[i] + TINY);
        B[i + 2] = B[i + 2] - D[i] * k2;
        C[i + 2] = C[i + 2] - m->E[i] * k2;
        f.k1[i] = k1; f.k2[i] = k2;
    }
    f.k3 = B[n - 1] / (C[n - 2] + TINY);
    C[n - 1] = C[n - 1] - D[n - 2] * f.k3;
    f.Cp = C; f.Dp = D;
    free(B);
    return f;
}
static void pen_apply(const pen_fac *f, double *W, int n, size_t lot) {
    const size_t CH = 256;
#pragma omp parallel for schedule(static)
    for (size_t L0 = 0; L0 < lot; L0 += CH) {
        size_t L1 = L0 + CH < lot ? L0 + CH : lot;
        for (int i = 0; i <= n - 3; i++) {
            double k1 = f->k1[i], k2 = f->k2[i];
            double *r0 = W + (size_t)i * lot, *r1 = W + (size_t)(i + 1) * lot,
                   *r2 = W + (size_t)(i + 2) * lot;
            for (size_t L = L0; L < L1; L++) {
                r1[L] = r1[L] - r0[L] * k1;
                r2[L] = r2[L] - r0[L] * k2;
            }
        }
        {
            double *r = W + (size_t)(n - 1) * lot, *rm = W + (size_t)(n - 2) * lot;
            for (size_t L = L0; L < L1; L++) r[L] = r[L] - rm[L] * f->k3;
        }
        {
            double *r = W + (size_t)(n - 1) * lot, den = f->Cp[n - 1] + TINY;
            for (size_t L = L0; L < L1; L++) r[L] = r[L] / den;
        }
        {
            double *r = W + (size_t)(n - 2) * lot, *rp = W + (size_t)(n - 1) * lot;
            double dd = f->Dp[n - 2], den = f->Cp[n - 2] + TINY;
            for (size_t L = L0; L < L1; L++) r[L] = (r[L] - dd * rp[L]) / den;
        }
        for (int i = n - 3; i >= 0; i--) {
            double *r = W + (size_t)i * lot, *r1 = W + (size_t)(i + 1) * lot,
                   *r2 = W + (size_t)(i + 2) * lot;
            double dd = f->Dp[i], ee = f->E[i], den = f->Cp[i] + TINY;
            for (size_t L = L0; L < L1; L++) r[L] = (r[L] - dd * r1[L] - ee * r2[L]) / den;
        }
    }
}

/* ---- LHS construction --------------------------------------------------- */
/* Setup_Derivatives_Sym src/derivCDopt6_sym_tri.f:41-372 and _Asym
 * src/derivCDopt6_asym_tri.f:41-374 (one-rank case: both boundary branches) */
static void build_deriv_lhs(tri_lhs *L1, tri_lhs *L2, int n, int asym) {
    L1->a = dalloc(n); L1->b = dalloc(n); L1->c = dalloc(n);
    L2->a = dalloc(n); L2->b = dalloc(n); L2->c = dalloc(n);
    for (int i = 0; i < n; i++) {
        L1->a[i] = alpha1_p6; L1->b[i] = 1.0; L1->c[i] = alpha1_p6;
        L2->a[i] = alpha2_p6; L2->b[i] = 1.0; L2->c[i] = alpha2_p6;
    }
    /* first node / last node */
    L1->a[0] = 0.0; L1->b[0] = 1.0; L1->c[0] = asym ? 2.0 * alpha1_p6 : 0.0;
    L1->a[n - 1] = 2.0; L1->b[n - 1] = 1.0; L1->c[n - 1] = 0.0;
    L1->a[1] = alpha1_p6; L1->b[1] = 1.0; L1->c[1] = alpha1_p6;
    L1->a[n - 2] = 1.0 / 2.0; L1->b[n - 2] = 1.0; L1->c[n - 2] = 1.0 / 6.0;
    L2->a[0] = 0.0; L2->b[0] = 1.0; L2->c[0] = asym ? 0.0 : 2.0 * alpha2_p6;
    L2->a[n - 1] = 1.1e1; L2->b[n - 1] = 1.0; L2->c[n - 1] = 0.0;
    L2->a[1] = alpha2_p6; L2->b[1] = 1.0; L2->c[1] = alpha2_p6;
    L2->a[n - 2] = -7.0 / 2.0e1; L2->b[n - 2] = 1.0; L2->c[n - 2] = 1.0e-1;
}
/* Init_Filters_sym src/filters_sym.f:44-382, Init_Filters_asym
 * src/filters_asym.f:44-384 */
static void build_filter_lhs(pen_lhs *m, int n, int asym) {
    m->A = dalloc(n); m->B = dalloc(n); m->C = dalloc(n); m->D = dalloc(n); m->E = dalloc(n);
    for (int i = 0; i < n; i++) {
        m->A[i] = beta_f4; m->B[i] = alpha_f4; m->C[i] = 1.0; m->D[i] = alpha_f4; m->E[i] = beta_f4;
    }
#define ROW(r, a, b, cc, d, e) do { m->A[r] = a; m->B[r] = b; m->C[r] = cc; m->D[r] = d; m->E[r] = e; } while (0)
    if (asym) ROW(0, 0.0, 0.0, 1.0, 0.0, 0.0);
    else ROW(0, 0.0, 0.0, 1.0, 2.0 * alpha_f4, 2.0 * beta_f4);
    ROW(n - 1, 0.0, 0.0, 1.0, 0.0, 0.0);
    if (asym) ROW(1, 0.0, alpha_f4, 1.0 - beta_f4, alpha_f4, beta_f4);
    else ROW(1, 0.0, alpha_f4, 1.0 + beta_f4, alpha_f4, beta_f4);
    ROW(n - 2, 0.0, bndy_alpha, 1.0, bndy_alpha, 0.0);
    ROW(2, beta_f4, alpha_f4, 1.0, alpha_f4, beta_f4);
    ROW(n - 3, 0.0, bndy_alpha, 1.0, bndy_alpha, 0.0);
    ROW(3, beta_f4, alpha_f4, 1.0, alpha_f4, beta_f4);
    ROW(n - 4, beta_f4, alpha_f4, 1.0, alpha_f4, beta_f4);
#undef ROW
}

orc *orc_create(const st_params *p) {
    orc *c = (orc *)calloc(1, sizeof(orc));
    c->p = *p;
    c->M[0] = p->nx; c->M[1] = p->ny; c->M[2] = p->nz;
    c->n3 = (size_t)p->nx * p->ny * p->nz;
    /* Setup_Grid src/grid.f:15-112, Uniform_X :116-128 */
    double leng[3] = {p->x_leng, p->y_leng, p->z_leng};
    double start[3] = {p->x_start, p->y_start, p->z_start};
    double D[3];
    for (int d = 0; d < 3; d++) {
        c->s1[d] = 1.0 / leng[d];
        c->s2[d] = c->s1[d] * c->s1[d];
        int n = c->M[d];
        double g1 = start[d] + leng[d] * (double)(0) / (double)(n - 1);
        double g2 = start[d] + leng[d] * (double)(1) / (double)(n - 1);
        D[d] = g2 - g1;
    }
    c->DX = D[0]; c->DY = D[1]; c->DZ = D[2];
    /* Define_Param src/define_nonperiodic_mf.f:182-204 */
    c->Re1_inv = p->re1 > 0.0 ? 1.0 / p->re1 : 0.0;
    c->Re2_inv = p->re2 > 0.0 ? 1.0 / p->re2 : 0.0;
    c->Pr_inv = p->pr > 0.0 ? 1.0 / p->pr : 0.0;
    c->Sc_inv = p->sc > 0.0 ? 1.0 / p->sc : 0.0;
    for (int d = 0; d < 3; d++) {
        for (int a = 0; a < 2; a++) {
            tri_lhs L1, L2; pen_lhs F;
            build_deriv_lhs(&L1, &L2, c->M[d], a);
            c->d1[d][a] = tri_factor(L1.a, L1.b, L1.c, c->M[d]);
            c->d2[d][a] = tri_factor(L2.a, L2.b, L2.c, c->M[d]);
            free(L1.a); free(L1.b); free(L1.c); free(L2.a); free(L2.b); free(L2.c);
            build_filter_lhs(&F, c->M[d], a);
            c->fl[d][a] = pen_factor(&F, c->M[d]);
            free(F.A); free(F.B); free(F.C); free(F.D); free(F.E);
        }
    }
    /* Visbal-Gaitonde closures, src/LES_header:118-146 */
    double ab = bndy_alpha, af = alpha_f4, bf = beta_f4;
    c->bc.c1[1] = 15.0 / 16.0; c->bc.c1[2] = 1.0 / 4.0; c->bc.c1[3] = -3.0 / 8.0;
    c->bc.c1[4] = 1.0 / 4.0; c->bc.c1[5] = -1.0 / 16.0;
    c->bc.c2[0] = (1.0 / 2.0 + ab);
    c->bc.c2[1] = (1.0 / 16.0 + (7.0 / 8.0) * ab);
    c->bc.c2[2] = (3.0 / 4.0 + (1.0 / 2.0) * ab);
    c->bc.c2[3] = (3.0 / 8.0 + (1.0 / 4.0) * ab);
    c->bc.c2[4] = (-1.0 / 4.0 + (1.0 / 2.0) * ab);
    c->bc.c2[5] = (1.0 / 16.0 - (1.0 / 8.0) * ab);
    c->bc.c3[0] = (5.0 / 8.0 + (3.0 / 4.0) * ab);
    c->bc.c3[1] = (1.0 / 2.0 + ab) / 2.0;
    c->bc.c3[2] = (-1.0 / 8.0 + ab / 4.0) / 2.0;
    c->bc.c4[0] = (11.0 / 16.0 + (5.0 / 8.0) * af - (5.0 / 8.0) * bf);
    c->bc.c4[1] = (15.0 / 32.0 + (17.0 / 16.0) * af + (15.0 / 16.0) * bf) / 2.0;
    c->bc.c4[2] = (-3.0 / 16.0 + (3.0 / 8.0) * af + (13.0 / 8.0) * bf) / 2.0;
    c->bc.c4[3] = (1.0 / 32.0 - af / 16.0 + bf / 16.0) / 2.0;
    /* implicit REAL PARAMETERs, src/LES_header:153-157 */
    c->ag[0] = (float)(3565.0 / 10368.0);
    c->ag[1] = (float)(3091.0 / 12960.0);
    c->ag[2] = (float)(1997.0 / 25920.0);
    c->ag[3] = (float)(149.0 / 12960.0);
    c->ag[4] = (float)(107.0 / 103680.0);
    c->Q = dalloc(5 * c->n3); c->dQ = dalloc(5 * c->n3); c->QW = dalloc(5 * c->n3);
    c->Y = NEWF(c); c->drYi = NEWF(c); c->rYW = NEWF(c); c->gamma_eff = NEWF(c);
    for (int g = 0; g < 12; g++) c->grad[g] = NEWF(c);
    for (int h = 0; h < 4; h++) c->hyp[h] = NEWF(c);
    for (int h = 0; h < 3; h++) c->dYd[h] = NEWF(c);
    if (c->p.family == ST_FAMILY_PERIODIC) {
        /* single fluid (src/define_periodic_sf.f:178-189): Re_inv = 1/Re, gamma
         * everywhere, mass fraction one, so the mixture formulas of the shared
         * RHS code reduce exactly to the single-fluid ones */
        c->Re1_inv = p->re > 0.0 ? 1.0 / p->re : 0.0;
        c->Re2_inv = 0.0;
        for (size_t q = 0; q < c->n3; q++) { c->gamma_eff[q] = p->gamma1; c->Y[q] = 1.0; }
    }
    return c;
}

void orc_destroy(orc *c) {
    if (!c) return;
    for (int d = 0; d < 3; d++)
        for (int a = 0; a < 2; a++) {
            free(c->d1[d][a].cst); free(c->d1[d][a].bp); free(c->d1[d][a].up);
            free(c->d2[d][a].cst); free(c->d2[d][a].bp); free(c->d2[d][a].up);
            free(c->fl[d][a].k1); free(c->fl[d][a].k2); free(c->fl[d][a].Cp);
            free(c->fl[d][a].Dp); free(c->fl[d][a].E);
        }
    free(c->Q); free(c->dQ); free(c->QW); free(c->Y); free(c->drYi); free(c->rYW);
    free(c->gamma_eff);
    for (int g = 0; g < 12; g++) free(c->grad[g]);
    for (int h = 0; h < 4; h++) free(c->hyp[h]);
    for (int h = 0; h < 3; h++) free(c->dYd[h]);
    free(c);
}

/* ---- periodic single-fluid family (ST_FAMILY_PERIODIC) --------------------
 * Operators of src/derivCDopt6_periodic.f and src/filters_periodic.f on one
 * rank: the MPI halo planes FP/FN are the line's own far rows, so every row
 * uses the interior formula with indices taken modulo n, and the system is
 * solved by pentadiagonal_periodic_serial (src/pentadiagonal.f90:381-504).
 *
 * Constant set (the periodic routines were written for a pentadiagonal
 * scheme with an f(i+-3) term, while src/header:191-204 activates the
 * FDL3DI tridiagonal set): the FDL3DI values are mapped onto the periodic
 * formulas as the tridiagonal scheme they denote -- first derivative
 * c1 = 0, beta1 = 0; second derivative with zero weight on f(i+-3) and
 * centre weight 2(a2+b2), beta2 = 0.  The shipped header's literal
 * substitution (c2_pade6 = 2(a2+b2) on f(i+-3), d2_pade6 = 0 at the centre,
 * src/derivCDopt6_periodic.f:326-329) is not a consistent second derivative
 * and is not reproduced. */
static const double per_c1 = 0.0;             /* f(i+-3) weight, first derivative  */
static const double per_c2 = 0.0;             /* f(i+-3) weight, second derivative */
#define PER_D2 C2_P6                          /* centre weight, second derivative   */

static int is_per(const orc *c) { return c->p.family == ST_FAMILY_PERIODIC; }

/* pentadiagonal_periodic_serial for one contiguous line with constant rows
 * (bt, al, 1, al, bt); wk holds 7n doubles.  src/pentadiagonal.f90:381-504 */
static void per_pen_line(double bt, double al, double *R, int n, double *wk) {
    if (n < 5) {
        double *A = wk, *B = wk + n, *C = wk + 2 * n, *D = wk + 3 * n, *E = wk + 4 * n;
        for (int i = 0; i < n; i++) { A[i] = bt; B[i] = al; C[i] = 1.0; D[i] = al; E[i] = bt; }
        orc_pentadiagonal(A, B, C, D, E, R, n, 1, 1);
        return;
    }
    double *A = wk, *B = wk + n, *C = wk + 2 * n, *D = wk + 3 * n, *E = wk + 4 * n;
    double *s1 = wk + 5 * n, *s2 = wk + 6 * n;
    for (int i = 0; i < n; i++) {
        A[i] = bt; B[i] = al; C[i] = 1.0; D[i] = al; E[i] = bt; s1[i] = 0.0; s2[i] = 0.0;
    }
    s1[0] = A[0];
    s1[n - 4] = s1[n - 4] + E[n - 4];
    s1[n - 3] = D[n - 3];
    s1[n - 2] = C[n - 2];
    s1[n - 1] = B[n - 1];
    s2[0] = B[0];
    s2[1] = A[1];
    s2[n - 3] = s2[n - 3] + E[n - 3];
    s2[n - 2] = D[n - 2];
    s2[n - 1] = C[n - 1];
    for (int i = 0; i <= n - 3; i++) {
        double cs = B[i + 1] / C[i];
        C[i + 1] = C[i + 1] - D[i] * cs;
        D[i + 1] = D[i + 1] - E[i] * cs;
        R[i + 1] = R[i + 1] - R[i] * cs;
        s1[i + 1] = s1[i + 1] - s1[i] * cs;
        s2[i + 1] = s2[i + 1] - s2[i] * cs;
        cs = A[i + 2] / C[i];
        B[i + 2] = B[i + 2] - D[i] * cs;
        C[i + 2] = C[i + 2] - E[i] * cs;
        R[i + 2] = R[i + 2] - R[i] * cs;
        s1[i + 2] = s1[i + 2] - s1[i] * cs;
        s2[i + 2] = s2[i + 2] - s2[i] * cs;
    }
    for (int i = n - 3; i >= 2; i--) {
        double cs = D[i - 1] / C[i];
        R[i - 1] = R[i - 1] - R[i] * cs;
        s1[i - 1] = s1[i - 1] - s1[i] * cs;
        s2[i - 1] = s2[i - 1] - s2[i] * cs;
        cs = E[i - 2] / C[i];
        R[i - 2] = R[i - 2] - R[i] * cs;
        s1[i - 2] = s1[i - 2] - s1[i] * cs;
        s2[i - 2] = s2[i - 2] - s2[i] * cs;
    }
    {
        double cs = D[0] / C[1];
        R[0] = R[0] - R[1] * cs;
        s1[0] = s1[0] - s1[1] * cs;
        s2[0] = s2[0] - s2[1] * cs;
    }
    double cs = E[n - 2] / C[0];
    R[n - 2] = R[n - 2] - R[0] * cs;
    s1[n - 2] = s1[n - 2] - s1[0] * cs;
    s2[n - 2] = s2[n - 2] - s2[0] * cs;
    cs = D[n - 1] / C[0];
    R[n - 1] = R[n - 1] - R[0] * cs;
    s1[n - 1] = s1[n - 1] - s1[0] * cs;
    s2[n - 1] = s2[n - 1] - s2[0] * cs;
    cs = E[n - 1] / C[1];
    R[n - 1] = R[n - 1] - R[1] * cs;
    s1[n - 1] = s1[n - 1] - s1[1] * cs;
    s2[n - 1] = s2[n - 1] - s2[1] * cs;
    cs = s1[n - 1] / s1[n - 2];
    R[n - 1] = R[n - 1] - R[n - 2] * cs;
    s2[n - 1] = s2[n - 1] - s2[n - 2] * cs;
    R[n - 1] = R[n - 1] / s2[n - 1];
    R[n - 2] = (R[n - 2] - s2[n - 2] * R[n - 1]) / s1[n - 2];
    for (int i = n - 3; i >= 0; i--) R[i] = (R[i] - s1[i] * R[n - 2] - s2[i] * R[n - 1]) / C[i];
}

enum { PER_D1, PER_D2OP, PER_FILT, PER_GAUSS };

/* One periodic line operator over all lines of direction d.
 * DFDX src/derivCDopt6_periodic.f:164-278 (RHS :205-248, solve :251),
 * D2FDX2 :281-397, Compact_Filter_X src/filters_periodic.f:115-250,
 * Gaussian_Filter_X :565-676, and the y/z twins of each. */
static void per_line_op(orc *c, int d, int kind, const double *F, double *O, int iadd, double cadd) {
    int n; size_t st, lot;
    line_geom(c, d, &n, &st, &lot);
    double fac = 0.0;
    if (kind == PER_D1) fac = cadd * c->s1[d] * (double)(n - 1);
    if (kind == PER_D2OP) fac = ((double)((n - 1) * (n - 1))) * c->s2[d];
    const double g0 = c->ag[0], g1 = c->ag[1], g2 = c->ag[2], g3 = c->ag[3], g4 = c->ag[4];
#pragma omp parallel
    {
        double *wk = dalloc(8 * (size_t)n);
        double *R = wk + 7 * (size_t)n;
#pragma omp for schedule(static)
        for (size_t L = 0; L < lot; L++) {
            const double *f = F + line_base(c, d, L);
#define FW_(i) f[(size_t)((((i) % n) + n) % n) * st]
            for (int i = 0; i < n; i++) {
                if (kind == PER_D1)
                    R[i] = fac * (per_c1 * (FW_(i + 3) - FW_(i - 3)) + b1_p6 * (FW_(i + 2) - FW_(i - 2))
                                  + a1_p6 * (FW_(i + 1) - FW_(i - 1)));
                else if (kind == PER_D2OP)
                    R[i] = fac * (per_c2 * (FW_(i + 3) + FW_(i - 3)) + b2_p6 * (FW_(i + 2) + FW_(i - 2))
                                  + a2_p6 * (FW_(i + 1) + FW_(i - 1)) - PER_D2 * FW_(i));
                else if (kind == PER_FILT)
                    R[i] = a4_f4 * (FW_(i + 4) + FW_(i - 4)) + a3_f4 * (FW_(i + 3) + FW_(i - 3))
                           + a2_f4 * (FW_(i + 2) + FW_(i - 2)) + a1_f4 * (FW_(i + 1) + FW_(i - 1))
                           + a0_f4 * FW_(i);
                else
                    R[i] = g4 * (FW_(i + 4) + FW_(i - 4)) + g3 * (FW_(i + 3) + FW_(i - 3))
                           + g2 * (FW_(i + 2) + FW_(i - 2)) + g1 * (FW_(i + 1) + FW_(i - 1)) + g0 * FW_(i);
            }
#undef FW_
            if (kind == PER_D1) per_pen_line(0.0, alpha1_p6, R, n, wk);
            else if (kind == PER_D2OP) per_pen_line(0.0, alpha2_p6, R, n, wk);
            else if (kind == PER_FILT) per_pen_line(beta_f4, alpha_f4, R, n, wk);
            double *o = O + line_base(c, d, L);
            for (int i = 0; i < n; i++) {
                if (iadd == 1) o[(size_t)i * st] = o[(size_t)i * st] + R[i];
                else o[(size_t)i * st] = R[i];
            }
        }
        free(wk);
    }
}

/* ---- operator-graph byte count ------------------------------------------- */
/* Interface bytes of the reference's operator graph, counted as its operator
 * calls happen (test infrastructure: the per-cell figure a GPU step is
 * compared with).  Per call and cell: DF* 16 B (read F, write dF), 24 B with
 * iadd (dF read too); D2F*2 16 B, 24 B with iadd (dF written as well, the
 * nested DF* call not counted again); one compact or Gaussian filter pass
 * 16 B; the LDDRK4 stage update 40 B per variable (read Q, QW, dQ; write Q,
 * QW).  Pointwise passes are not part of the graph. */
static double g_graph_bytes = 0.0;
static int g_graph_nested = 0;
void orc_graph_bytes_reset(void) { g_graph_bytes = 0.0; }
double orc_graph_bytes(void) { return g_graph_bytes; }
static void graph_count(const orc *c, double per_cell) {
    if (!g_graph_nested) g_graph_bytes += per_cell * (double)c->n3;
}

/* ---- derivatives ---------------------------------------------------------- */
/* DFDX_sym src/derivCDopt6_sym_tri.f:409-535 / DFDX_asym
 * src/derivCDopt6_asym_tri.f:412-537 and their y/z twins (the one-rank
 * branches xrank==0 and xrank==Px-1 both apply). */
void orc_dfd(orc *c, int d, int asym, const double *F, double *dF, int iadd, double cadd) {
    graph_count(c, iadd ? 24.0 : 16.0);
    if (is_per(c)) { per_line_op(c, d, PER_D1, F, dF, iadd, cadd); return; }
    int n; size_t st, lot;
    line_geom(c, d, &n, &st, &lot);
    double fac = cadd * c->s1[d] * (double)(n - 1);
    double *W = dalloc((size_t)n * lot);
#pragma omp parallel for schedule(static)
    for (size_t L = 0; L < lot; L++) {
        const double *f = F + line_base(c, d, L);
#define FF_(i) f[(size_t)(i) * st]
        for (int i = 2; i <= n - 3; i++)
            W[(size_t)i * lot + L] = fac * (b1_p6 * (FF_(i + 2) - FF_(i - 2)) + a1_p6 * (FF_(i + 1) - FF_(i - 1)));
        if (!asym) {
            W[L] = 0.0;
            W[lot + L] = fac * (b1_p6 * (FF_(3) - FF_(1)) + a1_p6 * (FF_(2) - FF_(0)));
        } else {
            W[L] = fac * (b1_p6 * (FF_(2) + FF_(2)) + a1_p6 * (FF_(1) + FF_(1)));
            W[lot + L] = fac * (b1_p6 * (FF_(3) + FF_(1)) + a1_p6 * (FF_(2) - FF_(0)));
        }
        W[(size_t)(n - 2) * lot + L] = fac * (closure1 * FF_(n - 1) + 5.0e-1 * FF_(n - 2)
                                              - FF_(n - 3) - closure2 * FF_(n - 4));
        W[(size_t)(n - 1) * lot + L] = fac * (2.5 * FF_(n - 1) - 2.0 * FF_(n - 2) - 5.0e-1 * FF_(n - 3));
#undef FF_
    }
    tri_apply(&c->d1[d][asym], W, n, lot);
#pragma omp parallel for schedule(static)
    for (size_t L = 0; L < lot; L++) {
        double *o = dF + line_base(c, d, L);
        for (int i = 0; i < n; i++) {
            double v = W[(size_t)i * lot + L];
            if (iadd == 0) o[(size_t)i * st] = v;
            else o[(size_t)i * st] = o[(size_t)i * st] + v;
        }
    }
    free(W);
}

/* D2FDX2_sym src/derivCDopt6_sym_tri.f:538-669 / D2FDX2_asym
 * src/derivCDopt6_asym_tri.f:540-667 and y/z twins */
static void orc_d2fd2_body(orc *c, int d, int asym, const double *F, double *dF, double *d2F, int iadd);
void orc_d2fd2(orc *c, int d, int asym, const double *F, double *dF, double *d2F, int iadd) {
    graph_count(c, iadd == 1 ? 24.0 : 16.0);
    g_graph_nested++;
    orc_d2fd2_body(c, d, asym, F, dF, d2F, iadd);
    g_graph_nested--;
}

static void orc_d2fd2_body(orc *c, int d, int asym, const double *F, double *dF, double *d2F, int iadd) {
    if (is_per(c)) {
        /* D2FDX2 src/derivCDopt6_periodic.f:270-392: dF by DFDX when iadd = 1 */
        if (iadd == 1) per_line_op(c, d, PER_D1, F, dF, 0, 1.0);
        per_line_op(c, d, PER_D2OP, F, d2F, 0, 1.0);
        return;
    }
    int n; size_t st, lot;
    line_geom(c, d, &n, &st, &lot);
    double fac = ((double)((n - 1) * (n - 1))) * c->s2[d];
    double c2 = C2_P6;
    double *W = dalloc((size_t)n * lot);
#pragma omp parallel for schedule(static)
    for (size_t L = 0; L < lot; L++) {
        const double *f = F + line_base(c, d, L);
#define FF_(i) f[(size_t)(i) * st]
        for (int i = 2; i <= n - 3; i++)
            W[(size_t)i * lot + L] = fac * (b2_p6 * (FF_(i + 2) + FF_(i - 2)) + a2_p6 * (FF_(i + 1) + FF_(i - 1))
                                            - c2 * FF_(i));
        if (!asym) {
            W[L] = fac * (b2_p6 * 2.0 * (FF_(2) - FF_(0)) + a2_p6 * 2.0 * (FF_(1) - FF_(0)));
            W[lot + L] = fac * (b2_p6 * (FF_(3) - 2.0 * FF_(1) + FF_(1)) + a2_p6 * (FF_(2) - 2.0 * FF_(1) + FF_(0)));
        } else {
            W[L] = 0.0;
            W[lot + L] = fac * (b2_p6 * (FF_(3) - 3.0 * FF_(1)) + a2_p6 * (FF_(2) - 2.0 * FF_(1)));
        }
        W[(size_t)(n - 2) * lot + L] = fac * (1.2375 * FF_(n - 1) - 3.0 * FF_(n - 2) + 2.325 * FF_(n - 3)
                                              - 6.0e-1 * FF_(n - 4) + 3.75e-2 * FF_(n - 5));
        W[(size_t)(n - 1) * lot + L] = fac * (1.3e1 * FF_(n - 1) - 2.7e1 * FF_(n - 2) + 1.5e1 * FF_(n - 3)
                                              - FF_(n - 4));
#undef FF_
    }
    if (iadd == 1) orc_dfd(c, d, asym, F, dF, 0, 1.0);
    tri_apply(&c->d2[d][asym], W, n, lot);
#pragma omp parallel for schedule(static)
    for (size_t L = 0; L < lot; L++) {
        double *o = d2F + line_base(c, d, L);
        for (int i = 0; i < n; i++) o[(size_t)i * st] = W[(size_t)i * lot + L];
    }
    free(W);
}

/* ---- filters -------------------------------------------------------------- */
/* Compact_Filter_X_sym src/filters_sym.f:436-634 / Compact_Filter_X_asym
 * src/filters_asym.f:388-583 and y/z twins */
void orc_filter(orc *c, int d, int asym, const double *F, double *F0) {
    graph_count(c, 16.0);
    if (is_per(c)) { per_line_op(c, d, PER_FILT, F, F0, 0, 1.0); return; }
    int n; size_t st, lot;
    line_geom(c, d, &n, &st, &lot);
    const struct bndyc *b = &c->bc;
    double *W = dalloc((size_t)n * lot);
#pragma omp parallel for schedule(static)
    for (size_t L = 0; L < lot; L++) {
        const double *f = F + line_base(c, d, L);
#define FF_(i) f[(size_t)(i) * st]
        for (int i = 4; i <= n - 5; i++)
            W[(size_t)i * lot + L] = a4_f4 * (FF_(i + 4) + FF_(i - 4)) + a3_f4 * (FF_(i + 3) + FF_(i - 3))
                                     + a2_f4 * (FF_(i + 2) + FF_(i - 2)) + a1_f4 * (FF_(i + 1) + FF_(i - 1))
                                     + a0_f4 * FF_(i);
        if (!asym) {
            W[L] = a4_f4 * (2.0 * FF_(4)) + a3_f4 * (2.0 * FF_(3)) + a2_f4 * (2.0 * FF_(2))
                   + a1_f4 * (2.0 * FF_(1)) + a0_f4 * FF_(0);
            W[lot + L] = a4_f4 * (FF_(3) + FF_(5)) + a3_f4 * (FF_(2) + FF_(4)) + a2_f4 * (FF_(1) + FF_(3))
                         + a1_f4 * (FF_(0) + FF_(2)) + a0_f4 * FF_(1);
            W[2 * lot + L] = a4_f4 * (FF_(2) + FF_(6)) + a3_f4 * (FF_(1) + FF_(5)) + a2_f4 * (FF_(0) + FF_(4))
                             + a1_f4 * (FF_(1) + FF_(3)) + a0_f4 * FF_(2);
            W[3 * lot + L] = a4_f4 * (FF_(1) + FF_(7)) + a3_f4 * (FF_(0) + FF_(6)) + a2_f4 * (FF_(1) + FF_(5))
                             + a1_f4 * (FF_(2) + FF_(4)) + a0_f4 * FF_(3);
        } else {
            W[L] = 0.0;
            W[lot + L] = a4_f4 * (FF_(5) - FF_(3)) + a3_f4 * (FF_(4) - FF_(2)) + a2_f4 * (FF_(3) - FF_(1))
                         + a1_f4 * (FF_(0) + FF_(2)) + a0_f4 * FF_(1);
            W[2 * lot + L] = a4_f4 * (FF_(6) - FF_(2)) + a3_f4 * (FF_(5) - FF_(1)) + a2_f4 * (FF_(0) + FF_(4))
                             + a1_f4 * (FF_(1) + FF_(3)) + a0_f4 * FF_(2);
            W[3 * lot + L] = a4_f4 * (FF_(7) - FF_(1)) + a3_f4 * (FF_(0) + FF_(6)) + a2_f4 * (FF_(1) + FF_(5))
                             + a1_f4 * (FF_(2) + FF_(4)) + a0_f4 * FF_(3);
        }
        W[(size_t)(n - 1) * lot + L] = b->c1[1] * FF_(n - 1) + b->c1[2] * FF_(n - 2) + b->c1[3] * FF_(n - 3)
                                       + b->c1[4] * FF_(n - 4) + b->c1[5] * FF_(n - 5);
        W[(size_t)(n - 2) * lot + L] = b->c2[1] * FF_(n - 1) + b->c2[2] * FF_(n - 2) + b->c2[3] * FF_(n - 3)
                                       + b->c2[4] * FF_(n - 4) + b->c2[5] * FF_(n - 5);
        W[(size_t)(n - 3) * lot + L] = b->c3[2] * FF_(n - 5) + b->c3[1] * FF_(n - 4) + b->c3[0] * FF_(n - 3)
                                       + b->c3[1] * FF_(n - 2) + b->c3[2] * FF_(n - 1);
        W[(size_t)(n - 4) * lot + L] = b->c4[3] * FF_(n - 7) + b->c4[2] * FF_(n - 6) + b->c4[1] * FF_(n - 5)
                                       + b->c4[0] * FF_(n - 4) + b->c4[1] * FF_(n - 3) + b->c4[2] * FF_(n - 2)
                                       + b->c4[3] * FF_(n - 1);
#undef FF_
    }
    pen_apply(&c->fl[d][asym], W, n, lot);
#pragma omp parallel for schedule(static)
    for (size_t L = 0; L < lot; L++) {
        double *o = F0 + line_base(c, d, L);
        for (int i = 0; i < n; i++) o[(size_t)i * st] = W[(size_t)i * lot + L];
    }
    free(W);
}

/* Compact_Filter src/filters_sym.f:398-432 */
void orc_compact_filter(orc *c, const double *F, double *F0, int nvar) {
    for (int l = 0; l < nvar; l++) {
        const double *f = F + (size_t)l * c->n3;
        double *g = F0 + (size_t)l * c->n3;
        orc_filter(c, 0, l == 0, f, g);
        orc_filter(c, 1, l == 1, g, g);
        orc_filter(c, 2, l == 2, g, g);
    }
}

/* Gaussian_Filter_X src/filters_sym.f:1076-1219 and Y/Z :1222-1554 */
void orc_gauss(orc *c, int d, const double *F, double *Fg) {
    graph_count(c, 16.0);
    if (is_per(c)) { per_line_op(c, d, PER_GAUSS, F, Fg, 0, 1.0); return; }
    int n; size_t st, lot;
    line_geom(c, d, &n, &st, &lot);
    double a0 = c->ag[0], a1 = c->ag[1], a2 = c->ag[2], a3 = c->ag[3], a4 = c->ag[4];
#pragma omp parallel for schedule(static)
    for (size_t L = 0; L < lot; L++) {
        const double *f = F + line_base(c, d, L);
        double *g = Fg + line_base(c, d, L);
#define FF_(i) f[(size_t)(i) * st]
#define GG_(i) g[(size_t)(i) * st]
        for (int i = 4; i <= n - 5; i++)
            GG_(i) = a4 * (FF_(i + 4) + FF_(i - 4)) + a3 * (FF_(i + 3) + FF_(i - 3))
                     + a2 * (FF_(i + 2) + FF_(i - 2)) + a1 * (FF_(i + 1) + FF_(i - 1)) + a0 * FF_(i);
        GG_(0) = a4 * (2.0 * FF_(4)) + a3 * (2.0 * FF_(3)) + a2 * (2.0 * FF_(2)) + a1 * (2.0 * FF_(1))
                 + a0 * FF_(0);
        GG_(1) = a4 * (FF_(3) + FF_(5)) + a3 * (FF_(2) + FF_(4)) + a2 * (FF_(1) + FF_(3))
                 + a1 * (FF_(0) + FF_(2)) + a0 * FF_(1);
        GG_(2) = a4 * (FF_(2) + FF_(6)) + a3 * (FF_(1) + FF_(5)) + a2 * (FF_(0) + FF_(4))
                 + a1 * (FF_(1) + FF_(3)) + a0 * FF_(2);
        GG_(3) = a4 * (FF_(1) + FF_(7)) + a3 * (FF_(0) + FF_(6)) + a2 * (FF_(1) + FF_(5))
                 + a1 * (FF_(2) + FF_(4)) + a0 * FF_(3);
        for (int i = 1; i <= 4; i++) GG_(n - i) = FF_(n - i);
#undef FF_
#undef GG_
    }
}

/* Gaussian_Filter src/filters_sym.f:1046-1071 */
void orc_gaussian_filter(orc *c, const double *F, double *Fg, int nvar) {
    double *tmp = NEWF(c);
    for (int l = 0; l < nvar; l++) {
        const double *f = F + (size_t)l * c->n3;
        double *g = Fg + (size_t)l * c->n3;
        orc_gauss(c, 0, f, g);
        orc_gauss(c, 1, g, tmp);
        orc_gauss(c, 2, tmp, g);
    }
    free(tmp);
}

/* ---- general line solvers ----------------------------------------------- */
/* tridiagonal (serial branch) src/tridiagonal.f90:1-49, 197-287 */
void orc_tridiagonal(const double *A1, const double *B1, const double *C1, double *R,
                     int n, int lot, int nper) {
    size_t N = (size_t)n * lot;
    double *a = dalloc(N), *b = dalloc(N), *cc = dalloc(N);
    memcpy(a, A1, N * sizeof(double)); memcpy(b, B1, N * sizeof(double));
    memcpy(cc, C1, N * sizeof(double));
#define A_(L, i) a[(size_t)(i) * lot + (L)]
#define B_(L, i) b[(size_t)(i) * lot + (L)]
#define C_(L, i) cc[(size_t)(i) * lot + (L)]
#define R_(L, i) R[(size_t)(i) * lot + (L)]
    for (int L = 0; L < lot; L++) {
        if (nper == 0) {
            for (int i = 1; i < n; i++) {
                double cs = A_(L, i) / (B_(L, i - 1) + TINY);
                B_(L, i) = B_(L, i) - C_(L, i - 1) * cs;
                R_(L, i) = R_(L, i) - R_(L, i - 1) * cs;
            }
            R_(L, n - 1) = R_(L, n - 1) / B_(L, n - 1);
            for (int i = n - 2; i >= 0; i--)
                R_(L, i) = (R_(L, i) - C_(L, i) * R_(L, i + 1)) / (B_(L, i) + TINY);
        } else {
            /* tridiagonal_periodic_serial src/tridiagonal.f90:197-258 */
            if (n == 1) { R_(L, 0) = R_(L, 0) / (A_(L, 0) + B_(L, 0) + C_(L, 0)); continue; }
            if (n == 2) {
                C_(L, 0) = C_(L, 0) + A_(L, 0);
                A_(L, 1) = A_(L, 1) + C_(L, 1);
                double cs = A_(L, 1) / B_(L, 0);
                B_(L, 1) = B_(L, 1) - C_(L, 0) * cs;
                R_(L, 1) = R_(L, 1) - R_(L, 0) * cs;
                R_(L, 1) = R_(L, 1) / B_(L, 1);
                R_(L, 0) = (R_(L, 0) - C_(L, 0) * R_(L, 1)) / B_(L, 0);
                continue;
            }
            for (int i = 1; i <= n - 3; i++) {
                double cs = A_(L, i) / B_(L, i - 1);
                B_(L, i) = B_(L, i) - C_(L, i - 1) * cs;
                R_(L, i) = R_(L, i) - R_(L, i - 1) * cs;
                A_(L, i) = -A_(L, i - 1) * cs;
            }
            int i = n - 2;
            double cs = A_(L, i) / B_(L, i - 1);
            B_(L, i) = B_(L, i) - C_(L, i - 1) * cs;
            R_(L, i) = R_(L, i) - R_(L, i - 1) * cs;
            A_(L, i) = C_(L, i) - A_(L, i - 1) * cs;
            i = n - 1;
            cs = A_(L, i) / B_(L, i - 1);
            R_(L, i) = R_(L, i) - R_(L, i - 1) * cs;
            A_(L, i) = B_(L, i) - A_(L, i - 1) * cs;
            for (i = n - 3; i >= 0; i--) {
                cs = C_(L, i) / B_(L, i + 1);
                R_(L, i) = R_(L, i) - R_(L, i + 1) * cs;
                A_(L, i) = A_(L, i) - A_(L, i + 1) * cs;
            }
            cs = C_(L, n - 1) / B_(L, 0);
            R_(L, n - 1) = R_(L, n - 1) - R_(L, 0) * cs;
            A_(L, n - 1) = A_(L, n - 1) - A_(L, 0) * cs;
            R_(L, n - 1) = R_(L, n - 1) / A_(L, n - 1);
            for (i = n - 2; i >= 0; i--) R_(L, i) = (R_(L, i) - A_(L, i) * R_(L, n - 1)) / B_(L, i);
        }
    }
#undef A_
#undef B_
#undef C_
#undef R_
    free(a); free(b); free(cc);
}

/* pentadiagonal (serial branch) src/pentadiagonal.f90:1-52, 319-504 */
void orc_pentadiagonal(const double *A1, const double *B1, const double *C1, const double *D1,
                       const double *E1, double *R, int n, int lot, int nper) {
    size_t N = (size_t)n * lot;
    double *A = dalloc(N), *B = dalloc(N), *C = dalloc(N), *D = dalloc(N), *E = dalloc(N);
    memcpy(A, A1, N * 8); memcpy(B, B1, N * 8); memcpy(C, C1, N * 8); memcpy(D, D1, N * 8);
    memcpy(E, E1, N * 8);
#define X_(arr, L, i) arr[(size_t)(i) * lot + (L)]
    for (int L = 0; L < lot; L++) {
        if (nper == 0) {
            if (n == 1) { X_(R, L, 0) = X_(R, L, 0) / X_(C, L, 0); continue; }
            if (n == 2) {
                double cs = X_(B, L, 1) / X_(C, L, 0);
                X_(C, L, 1) = X_(C, L, 1) - X_(D, L, 0) * cs;
                X_(R, L, 1) = X_(R, L, 1) - X_(R, L, 0) * cs;
                X_(R, L, 1) = X_(R, L, 1) / X_(C, L, 1);
                X_(R, L, 0) = (X_(R, L, 0) - X_(D, L, 0) * X_(R, L, 1)) / X_(C, L, 0);
                continue;
            }
            for (int i = 0; i <= n - 3; i++) {
                double cs = X_(B, L, i + 1) / (X_(C, L, i) + TINY);
                X_(C, L, i + 1) = X_(C, L, i + 1) - X_(D, L, i) * cs;
                X_(D, L, i + 1) = X_(D, L, i + 1) - X_(E, L, i) * cs;
                X_(R, L, i + 1) = X_(R, L, i + 1) - X_(R, L, i) * cs;
                cs = X_(A, L, i + 2) / (X_(C, L, i) + TINY);
                X_(B, L, i + 2) = X_(B, L, i + 2) - X_(D, L, i) * cs;
                X_(C, L, i + 2) = X_(C, L, i + 2) - X_(E, L, i) * cs;
                X_(R, L, i + 2) = X_(R, L, i + 2) - X_(R, L, i) * cs;
            }
            double cs = X_(B, L, n - 1) / (X_(C, L, n - 2) + TINY);
            X_(C, L, n - 1) = X_(C, L, n - 1) - X_(D, L, n - 2) * cs;
            X_(R, L, n - 1) = X_(R, L, n - 1) - X_(R, L, n - 2) * cs;
            X_(R, L, n - 1) = X_(R, L, n - 1) / (X_(C, L, n - 1) + TINY);
            X_(R, L, n - 2) = (X_(R, L, n - 2) - X_(D, L, n - 2) * X_(R, L, n - 1)) / (X_(C, L, n - 2) + TINY);
            for (int i = n - 3; i >= 0; i--)
                X_(R, L, i) = (X_(R, L, i) - X_(D, L, i) * X_(R, L, i + 1) - X_(E, L, i) * X_(R, L, i + 2))
                              / (X_(C, L, i) + TINY);
        } else {
            /* pentadiagonal_periodic_serial src/pentadiagonal.f90:381-504 */
            double *s1 = dalloc(n), *s2 = dalloc(n);
            if (n == 1) {
                X_(R, L, 0) = X_(R, L, 0) / (X_(A, L, 0) + X_(B, L, 0) + X_(C, L, 0) + X_(D, L, 0) + X_(E, L, 0));
                free(s1); free(s2); continue;
            }
            if (n == 2) {
                for (int i = 0; i < 2; i++) X_(C, L, i) = X_(C, L, i) + X_(A, L, i) + X_(E, L, i);
                X_(D, L, 0) = X_(D, L, 0) + X_(B, L, 0);
                X_(B, L, 1) = X_(B, L, 1) + X_(D, L, 1);
                double cs = X_(B, L, 1) / X_(C, L, 0);
                X_(C, L, 1) = X_(C, L, 1) - X_(D, L, 0) * cs;
                X_(R, L, 1) = X_(R, L, 1) - X_(R, L, 0) * cs;
                X_(R, L, 1) = X_(R, L, 1) / X_(C, L, 1);
                X_(R, L, 0) = (X_(R, L, 0) - X_(D, L, 0) * X_(R, L, 1)) / X_(C, L, 0);
                free(s1); free(s2); continue;
            }
            if (n == 3) {
                /* B+E, D+A then the periodic tridiagonal solve of this line */
                double tb[3], tc[3], td[3], tr[3];
                for (int i = 0; i < 3; i++) {
                    tb[i] = X_(B, L, i) + X_(E, L, i);
                    td[i] = X_(D, L, i) + X_(A, L, i);
                    tc[i] = X_(C, L, i);
                    tr[i] = X_(R, L, i);
                }
                orc_tridiagonal(tb, tc, td, tr, 3, 1, 1);
                for (int i = 0; i < 3; i++) X_(R, L, i) = tr[i];
                free(s1); free(s2); continue;
            }
            if (n == 4) {
                for (int i = 0; i < 4; i++) { X_(A, L, i) = X_(A, L, i) + X_(E, L, i); X_(E, L, i) = 0.0; }
            }
            s1[0] = X_(A, L, 0);
            s1[n - 4] = s1[n - 4] + X_(E, L, n - 4);
            s1[n - 3] = X_(D, L, n - 3);
            s1[n - 2] = X_(C, L, n - 2);
            s1[n - 1] = X_(B, L, n - 1);
            s2[0] = X_(B, L, 0);
            s2[1] = X_(A, L, 1);
            s2[n - 3] = s2[n - 3] + X_(E, L, n - 3);
            s2[n - 2] = X_(D, L, n - 2);
            s2[n - 1] = X_(C, L, n - 1);
            for (int i = 0; i <= n - 3; i++) {
                double cs = X_(B, L, i + 1) / X_(C, L, i);
                X_(C, L, i + 1) = X_(C, L, i + 1) - X_(D, L, i) * cs;
                X_(D, L, i + 1) = X_(D, L, i + 1) - X_(E, L, i) * cs;
                X_(R, L, i + 1) = X_(R, L, i + 1) - X_(R, L, i) * cs;
                s1[i + 1] = s1[i + 1] - s1[i] * cs;
                s2[i + 1] = s2[i + 1] - s2[i] * cs;
                cs = X_(A, L, i + 2) / X_(C, L, i);
                X_(B, L, i + 2) = X_(B, L, i + 2) - X_(D, L, i) * cs;
                X_(C, L, i + 2) = X_(C, L, i + 2) - X_(E, L, i) * cs;
                X_(R, L, i + 2) = X_(R, L, i + 2) - X_(R, L, i) * cs;
                s1[i + 2] = s1[i + 2] - s1[i] * cs;
                s2[i + 2] = s2[i + 2] - s2[i] * cs;
            }
            for (int i = n - 3; i >= 2; i--) {
                double cs = X_(D, L, i - 1) / X_(C, L, i);
                X_(R, L, i - 1) = X_(R, L, i - 1) - X_(R, L, i) * cs;
                s1[i - 1] = s1[i - 1] - s1[i] * cs;
                s2[i - 1] = s2[i - 1] - s2[i] * cs;
                cs = X_(E, L, i - 2) / X_(C, L, i);
                X_(R, L, i - 2) = X_(R, L, i - 2) - X_(R, L, i) * cs;
                s1[i - 2] = s1[i - 2] - s1[i] * cs;
                s2[i - 2] = s2[i - 2] - s2[i] * cs;
            }
            {
                int i = 1;
                double cs = X_(D, L, i - 1) / X_(C, L, i);
                X_(R, L, i - 1) = X_(R, L, i - 1) - X_(R, L, i) * cs;
                s1[i - 1] = s1[i - 1] - s1[i] * cs;
                s2[i - 1] = s2[i - 1] - s2[i] * cs;
            }
            double cs = X_(E, L, n - 2) / X_(C, L, 0);
            X_(R, L, n - 2) = X_(R, L, n - 2) - X_(R, L, 0) * cs;
            s1[n - 2] = s1[n - 2] - s1[0] * cs;
            s2[n - 2] = s2[n - 2] - s2[0] * cs;
            cs = X_(D, L, n - 1) / X_(C, L, 0);
            X_(R, L, n - 1) = X_(R, L, n - 1) - X_(R, L, 0) * cs;
            s1[n - 1] = s1[n - 1] - s1[0] * cs;
            s2[n - 1] = s2[n - 1] - s2[0] * cs;
            cs = X_(E, L, n - 1) / X_(C, L, 1);
            X_(R, L, n - 1) = X_(R, L, n - 1) - X_(R, L, 1) * cs;
            s1[n - 1] = s1[n - 1] - s1[1] * cs;
            s2[n - 1] = s2[n - 1] - s2[1] * cs;
            cs = s1[n - 1] / s1[n - 2];
            X_(R, L, n - 1) = X_(R, L, n - 1) - X_(R, L, n - 2) * cs;
            s2[n - 1] = s2[n - 1] - s2[n - 2] * cs;
            X_(R, L, n - 1) = X_(R, L, n - 1) / s2[n - 1];
            X_(R, L, n - 2) = (X_(R, L, n - 2) - s2[n - 2] * X_(R, L, n - 1)) / s1[n - 2];
            for (int i = n - 3; i >= 0; i--)
                X_(R, L, i) = (X_(R, L, i) - s1[i] * X_(R, L, n - 2) - s2[i] * X_(R, L, n - 1)) / X_(C, L, i);
            free(s1); free(s2);
        }
    }
#undef X_
    free(A); free(B); free(C); free(D); free(E);
}

/* ---- thermodynamics helpers -------------------------------------------- */
/* the P/T block repeated in RHS_x, RHS_yz, Hyper_RHS, Species_RHS, bc_RHS,
 * Fix_Pressure (e.g. src/rhsv_sym_mf.f:99-115) */
static inline void thermo(const orc *c, double g, double Y, double q1, double q2, double q3,
                          double q4, double q5, double *Vs, double *P, double *T) {
    double fac1 = g - 1.0;
    double fac3 = c->p.gamma1 / (c->p.gamma1 - 1.0);
    fac3 = fac3 * 1.0 / (Y + c->p.epsilon * (1.0 - Y));
    double vs = 1.0 / q4;
    double p = fac1 * (q5 - 5.0e-1 * vs * (q1 * q1 + q2 * q2 + q3 * q3));
    *Vs = vs; *P = p;
    *T = fac3 * vs * p;
}

/* Compute_gamma src/lddrk4_nonperiodic_mf.f:342-372 */
void orc_compute_gamma(orc *c, const double *Y) {
    double g1 = c->p.gamma1, g2 = c->p.gamma2, eps = c->p.epsilon;
#pragma omp parallel for schedule(static)
    for (size_t p = 0; p < c->n3; p++) {
        double fac1 = g1 - 1.0, fac2 = g2 - 1.0;
        double num = (Y[p] * g1 / fac1) + (eps * (1.0 - Y[p]) * g2 / fac2);
        double den = (Y[p] / fac1) + (eps * (1.0 - Y[p]) / fac2);
        c->gamma_eff[p] = num / den;
    }
}

/* viscosity law, src/rhsv_sym_mf.f:253-263 */
static inline void viscosity(const orc *c, double T, double Y, double *mu, double *dmu) {
    double fac1 = c->p.gamma1 - 1.0;
    double fac2 = c->p.vis_exp - 1.0;
    double se = sqrt(c->p.epsilon);
    double num = c->Re1_inv * Y + c->Re2_inv * se * (1.0 - Y);
    double den = Y + se * (1.0 - Y);
    *mu = pow(fac1 * T, c->p.vis_exp) * num / den;
    *dmu = pow(fac1 * T, fac2) * num / den * c->p.vis_exp * fac1;
}

#define PAR _Pragma("omp parallel for schedule(static)")
#define FOR_P for (size_t p = 0; p < n3; p++)

/* ---- RHS -------------------------------------------------------------------- */
/* RHS_x src/rhsv_sym_mf.f:37-481.  Q here is the copy Ux. */
static void rhs_x(orc *c, double *Q, double *Qrhs, const double *Y, double *Qcx, double *Qcy,
                  double *Qcz, double *Qv) {
    size_t n3 = c->n3;
    double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    double *P = NEWF(c), *Vs = NEWF(c), *T = NEWF(c), *FF = NEWF(c), *Flux = NEWF(c), *dF = NEWF(c);
    memset(Qrhs, 0, 5 * n3 * 8); memset(Qcx, 0, 5 * n3 * 8); memset(Qcy, 0, 5 * n3 * 8);
    memset(Qcz, 0, 5 * n3 * 8); memset(Qv, 0, 5 * n3 * 8);
    const double *g = c->gamma_eff;
    PAR FOR_P {
        thermo(c, g[p], Y[p], Q1[p], Q2[p], Q3[p], Q4[p], Q5[p], &Vs[p], &P[p], &T[p]);
        dF[p] = Q1[p] * Vs[p];
    }
    PAR FOR_P FF[p] = dF[p];
    PAR FOR_P Flux[p] = Q4[p] * FF[p];
    orc_dfd(c, 0, 1, Flux, Qcx + 3 * n3, 1, -1.0);
    PAR FOR_P Flux[p] = (Q5[p] + P[p]) * FF[p];
    orc_dfd(c, 0, 1, Flux, Qcx + 4 * n3, 1, -1.0);
    PAR FOR_P FF[p] = dF[p];
    PAR FOR_P Flux[p] = Q1[p] * FF[p];
    orc_dfd(c, 0, 0, Flux, Qcx, 1, -5.0e-1);
    orc_dfd(c, 0, 0, P, Qcx, 1, -1.0);
    PAR FOR_P Flux[p] = Q2[p] * FF[p];
    orc_dfd(c, 0, 1, Flux, Qcx + n3, 1, -5.0e-1);
    PAR FOR_P Flux[p] = Q3[p] * FF[p];
    orc_dfd(c, 0, 1, Flux, Qcx + 2 * n3, 1, -5.0e-1);
    orc_dfd(c, 0, 1, Q1, FF, 0, 1.0);
    PAR FOR_P {
        double mu, dmu;
        Q1[p] = dF[p];
        Q2[p] = Q2[p] * Vs[p];
        Q3[p] = Q3[p] * Vs[p];
        viscosity(c, T[p], Y[p], &mu, &dmu);
        Q5[p] = mu;
        Flux[p] = dmu;
    }
    PAR FOR_P {
        double fac2 = -5.0e-1 * FF[p];
        Qcx[p] = Qcx[p] + fac2 * Q1[p];
        Qcx[n3 + p] = Qcx[n3 + p] + fac2 * Q2[p];
        Qcx[2 * n3 + p] = Qcx[2 * n3 + p] + fac2 * Q3[p];
    }
    orc_d2fd2(c, 0, 0, T, FF, dF, 1);
    memcpy(c->grad[G_DTDX], FF, n3 * 8);
    {
        double fac1 = c->Pr_inv;
        PAR FOR_P Qv[4 * n3 + p] = Qv[4 * n3 + p] + fac1 * (Q5[p] * dF[p] + Flux[p] * FF[p] * FF[p]);
    }
    orc_d2fd2(c, 0, 1, Q1, Flux, dF, 1);
    memcpy(c->grad[G_DUX_DX], Flux, n3 * 8);
    {
        double fac1 = 4.0 / 3.0 + c->p.bulk_ratio;
        PAR FOR_P {
            double fac2 = fac1 * Q5[p] * dF[p];
            Qv[p] = Qv[p] + fac2;
            Qv[4 * n3 + p] = Qv[4 * n3 + p] + Q1[p] * fac2;
        }
    }
    orc_d2fd2(c, 0, 0, Q2, T, dF, 1);
    memcpy(c->grad[G_DUY_DX], T, n3 * 8);
    PAR FOR_P {
        double fac2 = Q5[p] * dF[p];
        Qv[n3 + p] = Qv[n3 + p] + fac2;
        Qv[4 * n3 + p] = Qv[4 * n3 + p] + Q2[p] * fac2;
        Q2[p] = T[p];
    }
    orc_d2fd2(c, 0, 0, Q3, Vs, dF, 1);
    memcpy(c->grad[G_DUZ_DX], Vs, n3 * 8);
    PAR FOR_P {
        double fac2 = Q5[p] * dF[p];
        Qv[2 * n3 + p] = Qv[2 * n3 + p] + fac2;
        Qv[4 * n3 + p] = Qv[4 * n3 + p] + Q3[p] * fac2;
        Q3[p] = Vs[p];
    }
    PAR FOR_P {
        double fac2 = -5.0e-1 * Q4[p] * Q1[p];
        Q1[p] = Flux[p];
        Q4[p] = FF[p];
        Qcx[p] = Qcx[p] + fac2 * Q1[p];
        Qcx[n3 + p] = Qcx[n3 + p] + fac2 * Q2[p];
        Qcx[2 * n3 + p] = Qcx[2 * n3 + p] + fac2 * Q3[p];
    }
    free(P); free(Vs); free(T); free(FF); free(Flux); free(dF);
}

/* RHS_yz src/rhsv_sym_mf.f:492-1428 */
static void rhs_yz(orc *c, double *Q, double *Ux, double *Qrhs, const double *Y, double *Qcx,
                   double *Qcy, double *Qcz, double *Qv) {
    size_t n3 = c->n3;
    double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    double *U1 = Ux, *U2 = Ux + n3, *U3 = Ux + 2 * n3, *U4 = Ux + 3 * n3, *U5 = Ux + 4 * n3;
    double *P = NEWF(c), *Vs = NEWF(c), *T = NEWF(c), *vis = NEWF(c), *dF = NEWF(c), *Flux = NEWF(c);
    double *Tdy = NEWF(c), *Tdz = NEWF(c), *Udz = NEWF(c), *dFz = NEWF(c), *Udx = NEWF(c), *Udy = NEWF(c);
    const double *g = c->gamma_eff;
    PAR FOR_P {
        thermo(c, g[p], Y[p], Q1[p], Q2[p], Q3[p], Q4[p], Q5[p], &Vs[p], &P[p], &T[p]);
        U5[p] = Q2[p] * Vs[p];
        Flux[p] = Q1[p] * U5[p];
    }
    orc_dfd(c, 1, 1, Q2, dF, 0, 1.0);
    PAR FOR_P Qcy[3 * n3 + p] = Qcy[3 * n3 + p] - dF[p];
    orc_dfd(c, 1, 1, Flux, Qcy, 1, -5.0e-1);
    PAR FOR_P Flux[p] = Q2[p] * U5[p];
    orc_dfd(c, 1, 0, Flux, Qcy + n3, 1, -5.0e-1);
    orc_dfd(c, 1, 0, P, Qcy + n3, 1, -1.0);
    PAR FOR_P Flux[p] = Q3[p] * U5[p];
    orc_dfd(c, 1, 1, Flux, Qcy + 2 * n3, 1, -5.0e-1);
    PAR FOR_P Flux[p] = (Q5[p] + P[p]) * U5[p];
    orc_dfd(c, 1, 1, Flux, Qcy + 4 * n3, 1, -1.0);
    orc_dfd(c, 2, 1, Q3, dFz, 0, 1.0);
    PAR FOR_P Qcz[3 * n3 + p] = Qcz[3 * n3 + p] - dFz[p];
    PAR FOR_P U5[p] = Q3[p] * Vs[p];
    PAR FOR_P Flux[p] = Q1[p] * U5[p];
    orc_dfd(c, 2, 1, Flux, Qcz, 1, -5.0e-1);
    PAR FOR_P Flux[p] = Q2[p] * U5[p];
    orc_dfd(c, 2, 1, Flux, Qcz + n3, 1, -5.0e-1);
    PAR FOR_P Flux[p] = Q3[p] * U5[p];
    orc_dfd(c, 2, 0, Flux, Qcz + 2 * n3, 1, -5.0e-1);
    orc_dfd(c, 2, 0, P, Qcz + 2 * n3, 1, -1.0);
    PAR FOR_P Flux[p] = (Q5[p] + P[p]) * U5[p];
    orc_dfd(c, 2, 1, Flux, Qcz + 4 * n3, 1, -1.0);
    PAR FOR_P {
        Q1[p] = Q1[p] * Vs[p];
        Q2[p] = Q2[p] * Vs[p];
        Q3[p] = Q3[p] * Vs[p];
    }
    PAR FOR_P {
        double fac2 = -5.0e-1 * dF[p];
        Qcy[p] = Qcy[p] + fac2 * Q1[p];
        Qcy[n3 + p] = Qcy[n3 + p] + fac2 * Q2[p];
        Qcy[2 * n3 + p] = Qcy[2 * n3 + p] + fac2 * Q3[p];
    }
    PAR FOR_P {
        double fac2 = -5.0e-1 * dFz[p];
        Qcz[p] = Qcz[p] + fac2 * Q1[p];
        Qcz[n3 + p] = Qcz[n3 + p] + fac2 * Q2[p];
        Qcz[2 * n3 + p] = Qcz[2 * n3 + p] + fac2 * Q3[p];
    }
    orc_d2fd2(c, 1, 0, T, Tdy, U5, 1);
    memcpy(c->grad[G_DTDY], Tdy, n3 * 8);
    orc_d2fd2(c, 2, 0, T, Tdz, Flux, 1);
    memcpy(c->grad[G_DTDZ], Tdz, n3 * 8);
    PAR FOR_P viscosity(c, T[p], Y[p], &vis[p], &Udz[p]);
    {
        double fac2 = c->Pr_inv;
        PAR FOR_P Qv[4 * n3 + p] = Qv[4 * n3 + p] + fac2 * (vis[p] * (U5[p] + Flux[p])
                                   + Udz[p] * (Tdy[p] * Tdy[p] + Tdz[p] * Tdz[p]));
    }
    PAR FOR_P {
        U4[p] = Udz[p] * U4[p];
        Tdy[p] = Udz[p] * Tdy[p];
        Tdz[p] = Udz[p] * Tdz[p];
    }
    orc_dfd(c, 1, 0, Q4, Udz, 0, 1.0);
    orc_d2fd2(c, 1, 0, Q1, P, U5, 1);
    memcpy(c->grad[G_DUX_DY], P, n3 * 8);
    orc_d2fd2(c, 1, 1, Q2, Flux, dF, 1);
    memcpy(c->grad[G_DUY_DY], Flux, n3 * 8);
    orc_d2fd2(c, 1, 0, Q3, Udz, T, 1);
    memcpy(c->grad[G_DUZ_DY], Udz, n3 * 8);
    orc_dfd(c, 2, 0, Q1, Udx, 0, 1.0);
    memcpy(c->grad[G_DUX_DZ], Udx, n3 * 8);
    orc_dfd(c, 2, 0, Q2, Udy, 0, 1.0);
    memcpy(c->grad[G_DUY_DZ], Udy, n3 * 8);
    orc_dfd(c, 2, 1, Q3, dFz, 0, 1.0);
    memcpy(c->grad[G_DUZ_DZ], dFz, n3 * 8);
    PAR FOR_P {
        double fac2 = -5.0e-1 * Q4[p] * Q2[p];
        Qcy[p] = Qcy[p] + fac2 * P[p];
        Qcy[n3 + p] = Qcy[n3 + p] + fac2 * Flux[p];
        Qcy[2 * n3 + p] = Qcy[2 * n3 + p] + fac2 * Udz[p];
    }
    PAR FOR_P {
        double fac2 = -5.0e-1 * Q4[p] * Q3[p];
        Qcz[p] = Qcz[p] + fac2 * Udx[p];
        Qcz[n3 + p] = Qcz[n3 + p] + fac2 * Udy[p];
        Qcz[2 * n3 + p] = Qcz[2 * n3 + p] + fac2 * dFz[p];
    }
    {
        double fac1 = c->p.bulk_ratio + 4.0 / 3.0;
        PAR FOR_P {
            double fac_X = vis[p] * U5[p];
            double fac_Y = fac1 * vis[p] * dF[p];
            double fac_Z = vis[p] * T[p];
            Qv[p] = Qv[p] + fac_X;
            Qv[n3 + p] = Qv[n3 + p] + fac_Y;
            Qv[2 * n3 + p] = Qv[2 * n3 + p] + fac_Z;
            Qv[4 * n3 + p] = Qv[4 * n3 + p] + Q1[p] * fac_X + Q2[p] * fac_Y + Q3[p] * fac_Z;
        }
    }
    orc_d2fd2(c, 2, 1, Q3, dF, T, 0);
    memcpy(dF, c->grad[G_DUZ_DZ], n3 * 8);
    orc_dfd(c, 1, 0, dF, U5, 0, 1.0);
    {
        double fac1 = c->p.bulk_ratio - 2.0 / 3.0;
        double fac2 = c->p.bulk_ratio + 4.0 / 3.0;
        double fac3 = c->p.bulk_ratio + 1.0 / 3.0;
        PAR FOR_P {
            double tmp1 = U1[p];
            double dil = tmp1 + Flux[p] + dF[p];
            double fac_X = U4[p] * (2.0 * tmp1 + fac1 * dil);
            double fac_Y = Tdy[p] * (2.0 * Flux[p] + fac1 * dil) + fac3 * vis[p] * U5[p];
            double fac_Z = Tdz[p] * (2.0 * dF[p] + fac1 * dil) + fac2 * vis[p] * T[p];
            Qv[p] = Qv[p] + fac_X;
            Qv[n3 + p] = Qv[n3 + p] + fac_Y;
            Qv[2 * n3 + p] = Qv[2 * n3 + p] + fac_Z;
            Qv[4 * n3 + p] = Qv[4 * n3 + p] + Q1[p] * fac_X + Q2[p] * fac_Y + Q3[p] * fac_Z
                             + vis[p] * (2.0 * (tmp1 * tmp1 + Flux[p] * Flux[p] + dF[p] * dF[p])
                                         + fac1 * dil * dil);
        }
        orc_d2fd2(c, 2, 0, Q1, T, dF, 0);
        memcpy(T, c->grad[G_DUX_DZ], n3 * 8);
        orc_d2fd2(c, 2, 0, Q2, Flux, U5, 0);
        memcpy(Flux, c->grad[G_DUY_DZ], n3 * 8);
        PAR FOR_P {
            double tmp1 = U2[p] + P[p];
            double tmp2 = U3[p] + T[p];
            double tmp3 = Udz[p] + Flux[p];
            double fac_X = Tdy[p] * tmp1 + Tdz[p] * tmp2 + vis[p] * dF[p];
            double fac_Y = U4[p] * tmp1 + Tdz[p] * tmp3 + vis[p] * U5[p];
            double fac_Z = U4[p] * tmp2 + Tdy[p] * tmp3;
            Qv[p] = Qv[p] + fac_X;
            Qv[n3 + p] = Qv[n3 + p] + fac_Y;
            Qv[2 * n3 + p] = Qv[2 * n3 + p] + fac_Z;
            Qv[4 * n3 + p] = Qv[4 * n3 + p] + Q1[p] * fac_X + Q2[p] * fac_Y + Q3[p] * fac_Z
                             + vis[p] * (tmp1 * tmp1 + tmp2 * tmp2 + tmp3 * tmp3);
        }
        orc_dfd(c, 1, 0, U1, U4, 0, 1.0);
        orc_dfd(c, 2, 0, U1, U5, 0, 1.0);
        orc_dfd(c, 1, 1, U2, Tdy, 0, 1.0);
        orc_dfd(c, 2, 1, U3, Tdz, 0, 1.0);
        orc_dfd(c, 1, 1, Flux, T, 0, 1.0);
        PAR FOR_P {
            double fac_X = fac3 * vis[p] * (Tdy[p] + Tdz[p]);
            double fac_Y = fac3 * vis[p] * U4[p];
            double fac_Z = fac3 * vis[p] * (U5[p] + T[p]);
            Qv[p] = Qv[p] + fac_X;
            Qv[n3 + p] = Qv[n3 + p] + fac_Y;
            Qv[2 * n3 + p] = Qv[2 * n3 + p] + fac_Z;
            Qv[4 * n3 + p] = Qv[4 * n3 + p] + Q1[p] * fac_X + Q2[p] * fac_Y + Q3[p] * fac_Z;
        }
    }
    PAR FOR_P {
        Q1[p] = Q1[p] * Q4[p];
        Q2[p] = Q2[p] * Q4[p];
        Q3[p] = Q3[p] * Q4[p];
    }
    /* src/rhsv_sym_mf.f:1420-1424 adds Qvisc only when Re > 0;
     * src/rhsv_periodic_sf.f:1381 always adds it */
    if (c->p.re > 0.0 || c->p.family == ST_FAMILY_PERIODIC) {
        PAR FOR_P for (int l = 0; l < 5; l++) {
            size_t q = l * n3 + p;
            Qrhs[q] = Qrhs[q] + Qcx[q] + Qcy[q] + Qcz[q] + Qv[q];
        }
    } else {
        PAR FOR_P for (int l = 0; l < 5; l++) {
            size_t q = l * n3 + p;
            Qrhs[q] = Qrhs[q] + Qcx[q] + Qcy[q] + Qcz[q];
        }
    }
    free(P); free(Vs); free(T); free(vis); free(dF); free(Flux);
    free(Tdy); free(Tdz); free(Udz); free(dFz); free(Udx); free(Udy);
}

/* RHS src/rhsv_sym_mf.f:9-26 */
void orc_rhs(orc *c, double *Q, double *Qrhs, const double *Y) {
    if (!Y) Y = c->Y;   /* the periodic single-fluid routines take no Y */
    size_t n3 = c->n3;
    double *Ux = dalloc(5 * n3), *Qcx = dalloc(5 * n3), *Qcy = dalloc(5 * n3), *Qcz = dalloc(5 * n3),
           *Qv = dalloc(5 * n3);
    memcpy(Ux, Q, 5 * n3 * 8);
    rhs_x(c, Ux, Qrhs, Y, Qcx, Qcy, Qcz, Qv);
    rhs_yz(c, Q, Ux, Qrhs, Y, Qcx, Qcy, Qcz, Qv);
    free(Ux); free(Qcx); free(Qcy); free(Qcz); free(Qv);
}

/* ---- artificial viscosity ------------------------------------------------ */
/* Compute_Laplacian src/hyper_dynamic_sym_mf.f:41-65 */
static void laplacian(orc *c, const double *S, double *d2S) {
    size_t n3 = c->n3;
    double *dS = NEWF(c), *t1 = NEWF(c), *t2 = NEWF(c);
    if (is_per(c)) {
        /* Compute_Laplacian src/hyper_dynamic.f:41-58 */
        orc_d2fd2(c, 0, 0, S, dS, t1, 0);
        orc_d2fd2(c, 1, 0, S, dS, t2, 0);
        orc_d2fd2(c, 2, 0, S, dS, d2S, 0);
        PAR FOR_P d2S[p] = d2S[p] + t1[p] + t2[p];
        free(dS); free(t1); free(t2);
        return;
    }
    orc_dfd(c, 0, 0, S, dS, 0, 1.0);
    orc_dfd(c, 0, 1, dS, t1, 0, 1.0);
    orc_dfd(c, 1, 0, S, dS, 0, 1.0);
    orc_dfd(c, 1, 1, dS, t2, 0, 1.0);
    orc_dfd(c, 2, 0, S, dS, 0, 1.0);
    orc_dfd(c, 2, 1, dS, d2S, 0, 1.0);
    PAR FOR_P d2S[p] = d2S[p] + t1[p] + t2[p];
    free(dS); free(t1); free(t2);
}

/* Compute_hyper of the periodic single-fluid family, src/hyper_dynamic.f:
 * Compute_coeff1 :72-165 (vorticity and dilatation from periodic first
 * derivatives of u), Compute_hyper :173-321 (Laplacians by D2FD*2 :41-58,
 * three Gaussian-filtered fields, coefficients applied after the filter). */
static void compute_hyper_sf(orc *c, const double *Q) {
    size_t n3 = c->n3;
    const double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    double **G = c->grad;
    const double gam = c->p.gamma1;
    double *U = dalloc(3 * n3), *Gr = dalloc(4 * n3), *tmp = NEWF(c), *Cbeta = NEWF(c);
    /* Compute_coeff1 */
    PAR FOR_P {
        double t = 1.0 / Q4[p];
        U[p] = Q1[p] * t; U[n3 + p] = Q2[p] * t; U[2 * n3 + p] = Q3[p] * t;
    }
    orc_dfd(c, 1, 0, U + 2 * n3, Gr, 0, 1.0);
    orc_dfd(c, 2, 0, U + n3, Gr, 1, -1.0);
    orc_dfd(c, 0, 0, U + 2 * n3, Gr + n3, 0, -1.0);
    orc_dfd(c, 2, 0, U, Gr + n3, 1, 1.0);
    orc_dfd(c, 0, 0, U + n3, Gr + 2 * n3, 0, 1.0);
    orc_dfd(c, 1, 0, U, Gr + 2 * n3, 1, -1.0);
    orc_dfd(c, 0, 0, U, Gr + 3 * n3, 0, 1.0);
    orc_dfd(c, 1, 0, U + n3, tmp, 0, 1.0);
    PAR FOR_P Gr[3 * n3 + p] = Gr[3 * n3 + p] + tmp[p];
    orc_dfd(c, 2, 0, U + 2 * n3, tmp, 0, 1.0);
    PAR FOR_P Gr[3 * n3 + p] = Gr[3 * n3 + p] + tmp[p];
    double scale = c->p.c_beta_scale;
    PAR FOR_P {
        double eps = 1.0e-7, fac2 = 10.0;
        double G1 = Gr[p], G2 = Gr[n3 + p], G3 = Gr[2 * n3 + p], G4 = Gr[3 * n3 + p];
        double fac = 5.0e-1 * (1.0 - tanh(2.5 + fac2 * G4));
        double om2 = G1 * G1 + G2 * G2 + G3 * G3;
        Cbeta[p] = (fac * G4 * G4 / (G4 * G4 + om2 + eps) + 1.0e-20) * scale;
    }
    const double C_mu = 2.0e-3, C_k = 1.0e-2;
    /* strain magnitude, P, T, e */
    double *S = NEWF(c), *e = NEWF(c), *P = NEWF(c), *T = NEWF(c), *Vs = NEWF(c);
    double *d2 = NEWF(c), *d4S = NEWF(c), *d4e = NEWF(c);
    double fac1 = gam - 1.0, fac2 = gam / fac1;
    PAR FOR_P {
        double s1 = G[G_DUX_DX][p], s5 = G[G_DUY_DY][p], s9 = G[G_DUZ_DZ][p];
        double s2 = 5.0e-1 * (G[G_DUX_DY][p] + G[G_DUY_DX][p]);
        double s3 = 5.0e-1 * (G[G_DUX_DZ][p] + G[G_DUZ_DX][p]);
        double s6 = 5.0e-1 * (G[G_DUY_DZ][p] + G[G_DUZ_DY][p]);
        double s4 = s2, s7 = s3, s8 = s6;
        Vs[p] = 1.0 / Q4[p];
        P[p] = fac1 * (Q5[p] - 5.0e-1 * Vs[p] * (Q1[p] * Q1[p] + Q2[p] * Q2[p] + Q3[p] * Q3[p]));
        T[p] = fac2 * Vs[p] * P[p];
        e[p] = Vs[p] * (Q5[p] - 5.0e-1 * Vs[p] * (Q1[p] * Q1[p] + Q2[p] * Q2[p] + Q3[p] * Q3[p]));
        S[p] = sqrt(5.0e-1 * (s1 * s1 + s5 * s5 + s9 * s9 + 2.0 * (s2 * s4 + s3 * s7 + s6 * s8)));
    }
    laplacian(c, S, d2);
    laplacian(c, d2, d4S);
    laplacian(c, e, d2);
    laplacian(c, d2, d4e);
    PAR FOR_P { d4S[p] = fabs(d4S[p]); d4e[p] = fabs(d4e[p]); }
    double *eta = dalloc(3 * n3), *etag = dalloc(3 * n3);
    PAR FOR_P {
        double fac3 = (Q4[p] / T[p]) * sqrt(gam * P[p] * Vs[p]);
        eta[p] = Q4[p] * d4S[p];
        eta[2 * n3 + p] = Q4[p] * d4S[p];
        eta[n3 + p] = fac3 * d4e[p];
    }
    orc_gaussian_filter(c, eta, etag, 3);
    double DX6 = pow(c->DX, 6.0), DX5 = pow(c->DX, 5.0);
    PAR FOR_P {
        c->hyp[H_BETA][p] = Cbeta[p] * etag[2 * n3 + p] * DX6;
        c->hyp[H_VISC][p] = C_mu * etag[p] * DX6;
        c->hyp[H_K][p] = C_k * etag[n3 + p] * DX5;
    }
    free(U); free(Gr); free(tmp); free(Cbeta); free(S); free(e); free(P); free(T); free(Vs);
    free(d2); free(d4S); free(d4e); free(eta); free(etag);
}

/* Compute_hyper src/hyper_dynamic_sym_mf.f:166-334 with Compute_coeff1
 * :79-158 and Compute_Contraction :12-33 */
void orc_compute_hyper(orc *c, const double *Q, const double *Y) {
    if (!Y) Y = c->Y;   /* the periodic single-fluid routines take no Y */
    if (is_per(c)) { compute_hyper_sf(c, Q); return; }
    size_t n3 = c->n3;
    const double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    double **G = c->grad;
    double *Cbeta = NEWF(c), *S = NEWF(c), *e = NEWF(c), *P = NEWF(c), *T = NEWF(c), *Vs = NEWF(c);
    double *d2 = NEWF(c), *d4S = NEWF(c), *d4e = NEWF(c), *d4Y = NEWF(c);
    double *eta = dalloc(5 * n3), *etag = dalloc(5 * n3);
    const double *g = c->gamma_eff;
    const double C_mu = 2.0e-3, C_k = 1.0e-2, C_D = 1.0e-4, C_Y = 100.0;
    double scale = c->p.c_beta_scale;
    PAR FOR_P {
        double G1 = G[G_DUZ_DY][p] - G[G_DUY_DZ][p];
        double G2 = G[G_DUX_DZ][p] - G[G_DUZ_DX][p];
        double G3 = G[G_DUY_DX][p] - G[G_DUX_DY][p];
        double G4 = 0.0;
        G4 = G[G_DUX_DX][p] + G[G_DUY_DY][p] + G[G_DUZ_DZ][p];
        double eps = 1.0e-7, fac2 = 0.2;
        double fac = 5.0e-1 * (1.0 - tanh(2.5 + fac2 * G4));
        double om2 = G1 * G1 + G2 * G2 + G3 * G3;
        Cbeta[p] = (fac * G4 * G4 / (G4 * G4 + om2 + eps)) * scale;
    }
    PAR FOR_P {
        double s1 = G[G_DUX_DX][p], s5 = G[G_DUY_DY][p], s9 = G[G_DUZ_DZ][p];
        double s2 = 5.0e-1 * (G[G_DUX_DY][p] + G[G_DUY_DX][p]);
        double s3 = 5.0e-1 * (G[G_DUX_DZ][p] + G[G_DUZ_DX][p]);
        double s6 = 5.0e-1 * (G[G_DUY_DZ][p] + G[G_DUZ_DY][p]);
        double s4 = s2, s7 = s3, s8 = s6;
        double fac1 = g[p] - 1.0;
        double fac3 = c->p.gamma1 / (c->p.gamma1 - 1.0);
        fac3 = fac3 * 1.0 / (Y[p] + c->p.epsilon * (1.0 - Y[p]));
        Vs[p] = 1.0 / Q4[p];
        P[p] = fac1 * (Q5[p] - 5.0e-1 * Vs[p] * (Q1[p] * Q1[p] + Q2[p] * Q2[p] + Q3[p] * Q3[p]));
        T[p] = fac3 * Vs[p] * P[p];
        e[p] = Vs[p] * (Q5[p] - 5.0e-1 * Vs[p] * (Q1[p] * Q1[p] + Q2[p] * Q2[p] + Q3[p] * Q3[p]));
        S[p] = sqrt(5.0e-1 * (s1 * s1 + s5 * s5 + s9 * s9 + 2.0 * (s2 * s4 + s3 * s7 + s6 * s8)));
    }
    laplacian(c, S, d2);
    laplacian(c, d2, d4S);
    laplacian(c, e, d2);
    laplacian(c, d2, d4e);
    laplacian(c, Y, d2);
    laplacian(c, d2, d4Y);
    PAR FOR_P {
        d4S[p] = fabs(d4S[p]); d4e[p] = fabs(d4e[p]); d4Y[p] = fabs(d4Y[p]);
    }
    PAR FOR_P {
        double cs = sqrt(g[p] * P[p] * Vs[p]);
        double fac3 = (Q4[p] / T[p]) * sqrt(g[p] * P[p] * Vs[p]);
        eta[p] = C_mu * Q4[p] * d4S[p];
        eta[2 * n3 + p] = Cbeta[p] * Q4[p] * d4S[p];
        eta[n3 + p] = C_k * fac3 * d4e[p];
        eta[4 * n3 + p] = cs * d4Y[p];
        double tmp1 = (Y[p] < 1.0) ? 0.0 : 1.0;
        double tmp2 = (Y[p] < 0.0) ? 0.0 : 1.0;
        eta[3 * n3 + p] = cs * ((Y[p] - 1.0) * tmp1 - Y[p] * (1.0 - tmp2));
    }
    orc_gaussian_filter(c, eta, etag, 5);
    double DX6 = pow(c->DX, 6.0), DX5 = pow(c->DX, 5.0), DX = c->DX;
    PAR FOR_P {
        c->hyp[H_BETA][p] = etag[2 * n3 + p] * DX6;
        c->hyp[H_VISC][p] = etag[p] * DX6;
        c->hyp[H_K][p] = etag[n3 + p] * DX5;
        c->hyp[H_D][p] = C_D * etag[4 * n3 + p] * DX5 + C_Y * etag[3 * n3 + p] * DX;
    }
    free(Cbeta); free(S); free(e); free(P); free(T); free(Vs); free(d2); free(d4S); free(d4e);
    free(d4Y); free(eta); free(etag);
}

/* Hyper_RHS src/hyper_rhs_sym_mf.f:12-500 */
void orc_hyper_rhs(orc *c, const double *Q, double *Qrhs, const double *Y) {
    if (!Y) Y = c->Y;   /* the periodic single-fluid routines take no Y */
    if (c->p.hyper_param == 0) return;
    size_t n3 = c->n3;
    const double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    double **G = c->grad;
    double *Qh = dalloc(5 * n3);
    orc_compute_hyper(c, Q, Y);
    double *U = dalloc(3 * n3), *dila = NEWF(c), *S = dalloc(3 * n3), *Flux = NEWF(c), *FF = NEWF(c);
    double *dFx = NEWF(c), *dFy = NEWF(c), *dFz = NEWF(c), *dEx = NEWF(c), *dEy = NEWF(c), *dEz = NEWF(c);
    double *Vs = NEWF(c), *P = NEWF(c), *T = NEWF(c);
    const double *vh = c->hyp[H_VISC], *bh = c->hyp[H_BETA], *kh = c->hyp[H_K];
    PAR FOR_P {
        U[p] = Q1[p] / Q4[p];
        U[n3 + p] = Q2[p] / Q4[p];
        U[2 * n3 + p] = Q3[p] / Q4[p];
    }
    PAR FOR_P dila[p] = G[G_DUX_DX][p] + G[G_DUY_DY][p] + G[G_DUZ_DZ][p];
    PAR FOR_P S[p] = G[G_DUX_DY][p] + G[G_DUY_DX][p];
    PAR FOR_P S[n3 + p] = G[G_DUX_DZ][p] + G[G_DUZ_DX][p];
    PAR FOR_P S[2 * n3 + p] = G[G_DUY_DZ][p] + G[G_DUZ_DY][p];
    PAR FOR_P thermo(c, c->gamma_eff[p], Y[p], Q1[p], Q2[p], Q3[p], Q4[p], Q5[p], &Vs[p], &P[p], &T[p]);
#define SUM3(dst, a, b, cc) PAR FOR_P dst[p] = dst[p] + a[p] + b[p] + cc[p]
    /* x momentum */
    PAR FOR_P {
        Flux[p] = 2.0 * vh[p] * G[G_DUX_DX][p] + (bh[p] - (2.0 / 3.0) * vh[p]) * dila[p];
        FF[p] = U[p] * Flux[p];
    }
    orc_dfd(c, 0, 0, Flux, dFx, 0, 1.0);
    orc_dfd(c, 0, 1, FF, dEx, 0, 1.0);
    PAR FOR_P { Flux[p] = vh[p] * S[p]; FF[p] = U[p] * Flux[p]; }
    orc_dfd(c, 1, 1, Flux, dFy, 0, 1.0);
    orc_dfd(c, 1, 1, FF, dEy, 0, 1.0);
    PAR FOR_P { Flux[p] = vh[p] * S[n3 + p]; FF[p] = U[p] * Flux[p]; }
    orc_dfd(c, 2, 1, Flux, dFz, 0, 1.0);
    orc_dfd(c, 2, 1, FF, dEz, 0, 1.0);
    { double *h1 = Qh, *h5 = Qh + 4 * n3; SUM3(h1, dFx, dFy, dFz); SUM3(h5, dEx, dEy, dEz); }
    /* y momentum */
    PAR FOR_P {
        Flux[p] = 2.0 * vh[p] * G[G_DUY_DY][p] + (bh[p] - (2.0 / 3.0) * vh[p]) * dila[p];
        FF[p] = U[n3 + p] * Flux[p];
    }
    orc_dfd(c, 1, 0, Flux, dFy, 0, 1.0);
    orc_dfd(c, 1, 1, FF, dEy, 0, 1.0);
    PAR FOR_P { Flux[p] = vh[p] * S[p]; FF[p] = U[n3 + p] * Flux[p]; }
    orc_dfd(c, 0, 1, Flux, dFx, 0, 1.0);
    orc_dfd(c, 0, 1, FF, dEx, 0, 1.0);
    PAR FOR_P { Flux[p] = vh[p] * S[2 * n3 + p]; FF[p] = U[n3 + p] * Flux[p]; }
    orc_dfd(c, 2, 1, Flux, dFz, 0, 1.0);
    orc_dfd(c, 2, 1, FF, dEz, 0, 1.0);
    { double *h2 = Qh + n3, *h5 = Qh + 4 * n3; SUM3(h2, dFx, dFy, dFz); SUM3(h5, dEx, dEy, dEz); }
    /* z momentum */
    PAR FOR_P {
        Flux[p] = 2.0 * vh[p] * G[G_DUZ_DZ][p] + (bh[p] - (2.0 / 3.0) * vh[p]) * dila[p];
        FF[p] = U[2 * n3 + p] * Flux[p];
    }
    orc_dfd(c, 2, 0, Flux, dFz, 0, 1.0);
    orc_dfd(c, 2, 1, FF, dEz, 0, 1.0);
    PAR FOR_P { Flux[p] = vh[p] * S[n3 + p]; FF[p] = U[2 * n3 + p] * Flux[p]; }
    orc_dfd(c, 0, 1, Flux, dFx, 0, 1.0);
    orc_dfd(c, 0, 1, FF, dEx, 0, 1.0);
    PAR FOR_P { Flux[p] = vh[p] * S[2 * n3 + p]; FF[p] = U[2 * n3 + p] * Flux[p]; }
    orc_dfd(c, 1, 1, Flux, dFy, 0, 1.0);
    orc_dfd(c, 1, 1, FF, dEy, 0, 1.0);
    { double *h3 = Qh + 2 * n3, *h5 = Qh + 4 * n3; SUM3(h3, dFx, dFy, dFz); SUM3(h5, dEx, dEy, dEz); }
    /* heat flux */
    PAR FOR_P Flux[p] = kh[p] * G[G_DTDX][p];
    orc_dfd(c, 0, 0, Flux, dFx, 0, 1.0);
    PAR FOR_P Flux[p] = kh[p] * G[G_DTDY][p];
    orc_dfd(c, 1, 0, Flux, dFy, 0, 1.0);
    PAR FOR_P Flux[p] = kh[p] * G[G_DTDZ][p];
    orc_dfd(c, 2, 0, Flux, dFz, 0, 1.0);
    { double *h5 = Qh + 4 * n3; SUM3(h5, dFx, dFy, dFz); }
#undef SUM3
    PAR for (size_t q = 0; q < 5 * n3; q++) Qrhs[q] = Qrhs[q] + Qh[q];
    free(Qh); free(U); free(dila); free(S); free(Flux); free(FF); free(dFx); free(dFy); free(dFz);
    free(dEx); free(dEy); free(dEz); free(Vs); free(P); free(T);
}

/* Species_RHS src/species_rhs_sym.f:9-207 */
void orc_species_rhs(orc *c, const double *Q, double *Qrhs, const double *Y, double *Yrhs) {
    if (c->p.hyper_param == 0) return;
    size_t n3 = c->n3;
    const double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    double *Ycx = NEWF(c), *Ycy = NEWF(c), *Ycz = NEWF(c), *Yd = NEWF(c);
    double *Flux = NEWF(c), *FF = NEWF(c), *Vs = NEWF(c), *P = NEWF(c), *T = NEWF(c);
    const double *Dh = c->hyp[H_D];
    memset(Yrhs, 0, n3 * 8);
    PAR FOR_P thermo(c, c->gamma_eff[p], Y[p], Q1[p], Q2[p], Q3[p], Q4[p], Q5[p], &Vs[p], &P[p], &T[p]);
    orc_dfd(c, 0, 0, Y, c->dYd[0], 0, 1.0);
    orc_dfd(c, 1, 0, Y, c->dYd[1], 0, 1.0);
    orc_dfd(c, 2, 0, Y, c->dYd[2], 0, 1.0);
    PAR FOR_P Flux[p] = Q1[p] * Y[p];
    orc_dfd(c, 0, 1, Flux, Ycx, 1, -1.0);
    PAR FOR_P Flux[p] = Q2[p] * Y[p];
    orc_dfd(c, 1, 1, Flux, Ycy, 1, -1.0);
    PAR FOR_P Flux[p] = Q3[p] * Y[p];
    orc_dfd(c, 2, 1, Flux, Ycz, 1, -1.0);
    double g1 = c->p.gamma1, g2 = c->p.gamma2, eps = c->p.epsilon;
    double Re1i = c->Re1_inv, Sci = c->Sc_inv;
    for (int d = 0; d < 3; d++) {
        const double *dY = c->dYd[d];
        PAR FOR_P {
            Flux[p] = Q4[p] * Dh[p] * dY[p] + Q4[p] * dY[p] * Re1i * Sci;
            FF[p] = (1.0 - eps * g2 * (g1 - 1.0) / (g1 * (g2 - 1.0))) * T[p] * Flux[p];
        }
        orc_dfd(c, d, 1, Flux, Yd, 1, 1.0);
        orc_dfd(c, d, 1, FF, Qrhs + 4 * n3, 1, 1.0);
    }
    PAR FOR_P Yrhs[p] = Ycx[p] + Ycy[p] + Ycz[p] + Yd[p];
    free(Ycx); free(Ycy); free(Ycz); free(Yd); free(Flux); free(FF); free(Vs); free(P); free(T);
}

/* bc_RHS src/bc_mf.f:11-463 (the active face blocks; edges/corners are
 * commented out in the reference) */
void orc_bc_rhs(orc *c, double *Q, double *Qrhs, const double *Y, double *Yrhs, double time) {
    (void)time;
    size_t n3 = c->n3;
    int Mx = c->M[0], My = c->M[1], Mz = c->M[2];
    double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    double **G = c->grad;
    const double *g = c->gamma_eff;
    for (int j = 0; j < My; j++) for (int k = 0; k < Mz; k++) Q1[IX(c, j, k, 0)] = 0.0;
    for (int i = 0; i < Mx; i++) for (int j = 0; j < My; j++) Q3[IX(c, j, 0, i)] = 0.0;
    for (int i = 0; i < Mx; i++) for (int k = 0; k < Mz; k++) Q2[IX(c, 0, k, i)] = 0.0;
    double *Vs = NEWF(c), *P = NEWF(c), *T = NEWF(c), *U = dalloc(3 * n3), *Ur = NEWF(c);
    double *dF = dalloc(3 * n3);
    PAR FOR_P {
        thermo(c, g[p], Y[p], Q1[p], Q2[p], Q3[p], Q4[p], Q5[p], &Vs[p], &P[p], &T[p]);
        U[p] = Q1[p] * Vs[p];
        U[n3 + p] = Q2[p] * Vs[p];
        U[2 * n3 + p] = Q3[p] * Vs[p];
        Ur[p] = sqrt(U[p] * U[p] + U[n3 + p] * U[n3 + p] + U[2 * n3 + p] * U[2 * n3 + p]);
    }
    orc_dfd(c, 0, 0, P, dF, 0, 1.0);
    orc_dfd(c, 1, 0, P, dF + n3, 0, 1.0);
    orc_dfd(c, 2, 0, P, dF + 2 * n3, 0, 1.0);
    /* x face: i = Mx */
    for (int j = 0; j < My; j++) for (int k = 0; k < Mz; k++) {
        size_t p = IX(c, j, k, Mx - 1);
        double tmp2 = sqrt(g[p] * Vs[p] * P[p]);
        double L1 = 0.0, L2 = 0.0, L3 = 0.0, L4 = 0.0, L6 = 0.0;
        double L5 = (U[p] + tmp2) * (dF[p] + tmp2 * Q4[p] * G[G_DUX_DX][p]);
        double d1 = (1.0 / (tmp2 * tmp2)) * (L2 + 5.0e-1 * (L1 + L5));
        double d2 = 5.0e-1 * (L5 + L1);
        double d3 = (5.0e-1 / (Q4[p] * tmp2)) * (L5 - L1);
        double d4 = L3, d5 = L4, d6 = L6;
        Qrhs[3 * n3 + p] = -d1;
        Qrhs[4 * n3 + p] = -5.0e-1 * Ur[p] * Ur[p] * d1 - d2 / (g[p] - 1.0) - Q1[p] * d3 - Q2[p] * d4
                           - Q3[p] * d5;
        Qrhs[p] = -U[p] * d1 - Q4[p] * d3;
        Qrhs[n3 + p] = -U[n3 + p] * d1 - Q4[p] * d4;
        Qrhs[2 * n3 + p] = -U[2 * n3 + p] * d1 - Q4[p] * d5;
        Yrhs[p] = -Q4[p] * d6;
    }
    /* y face: j = My */
    for (int i = 0; i < Mx; i++) for (int k = 0; k < Mz; k++) {
        size_t p = IX(c, My - 1, k, i);
        double tmp2 = sqrt(g[p] * Vs[p] * P[p]);
        double M1 = 0.0, M2 = 0.0, M3 = 0.0, M4 = 0.0, M6 = 0.0;
        double M5 = (U[n3 + p] + tmp2) * (dF[n3 + p] + tmp2 * Q4[p] * G[G_DUY_DY][p]);
        double e1 = (1.0 / (tmp2 * tmp2)) * (M2 + 5.0e-1 * (M1 + M5));
        double e2 = 5.0e-1 * (M5 + M1);
        double e3 = (5.0e-1 / (Q4[p] * tmp2)) * (M5 - M1);
        double e4 = M3, e5 = M4, e6 = M6;
        Qrhs[3 * n3 + p] = -e1;
        Qrhs[4 * n3 + p] = -5.0e-1 * Ur[p] * Ur[p] * e1 - e2 / (g[p] - 1.0) - Q2[p] * e3 - Q1[p] * e4
                           - Q3[p] * e5;
        Qrhs[n3 + p] = -U[n3 + p] * e1 - Q4[p] * e3;
        Qrhs[p] = -U[p] * e1 - Q4[p] * e4;
        Qrhs[2 * n3 + p] = -U[2 * n3 + p] * e1 - Q4[p] * e5;
        Yrhs[p] = -Q4[p] * e6;
    }
    /* z face: k = Mz */
    for (int i = 0; i < Mx; i++) for (int j = 0; j < My; j++) {
        size_t p = IX(c, j, Mz - 1, i);
        double tmp2 = sqrt(g[p] * Vs[p] * P[p]);
        double N1 = 0.0, N2 = 0.0, N3 = 0.0, N4 = 0.0, N6 = 0.0;
        double N5 = (U[2 * n3 + p] + tmp2) * (dF[2 * n3 + p] + tmp2 * Q4[p] * G[G_DUZ_DZ][p]);
        double f1 = (1.0 / (tmp2 * tmp2)) * (N2 + 5.0e-1 * (N1 + N5));
        double f2 = 5.0e-1 * (N5 + N1);
        double f3 = (5.0e-1 / (Q4[p] * tmp2)) * (N5 - N1);
        double f4 = N3, f5 = N4, f6 = N6;
        Qrhs[3 * n3 + p] = -f1;
        Qrhs[4 * n3 + p] = -5.0e-1 * Ur[p] * Ur[p] * f1 - f2 / (g[p] - 1.0) - Q3[p] * f3 - Q1[p] * f4
                           - Q2[p] * f5;
        Qrhs[2 * n3 + p] = -U[2 * n3 + p] * f1 - Q4[p] * f3;
        Qrhs[p] = -U[p] * f1 - Q4[p] * f4;
        Qrhs[n3 + p] = -U[n3 + p] * f1 - Q4[p] * f5;
        Yrhs[p] = -Q4[p] * f6;
    }
    free(Vs); free(P); free(T); free(U); free(Ur); free(dF);
}

/* Sponge_Forcing src/sponge_mf.f:7-127 */
void orc_sponge_forcing(orc *c, const double *Q, double *Qrhs, const double *Y, double *Yrhs) {
    size_t n3 = c->n3;
    int Mx = c->M[0], My = c->M[1], Mz = c->M[2];
    double g1 = c->p.gamma1;
    double base_pressure = 0.71429, Ms = 1.8, A_sponge = 4.0, s_exp = 3.0;
    double frac = 0.1;
    double vel_ref = 0.0;
    double rho_ref = (g1 + 1.0) * Ms * Ms / ((g1 - 1.0) * Ms * Ms + 2.0);
    double P_ref = ((2.0 * g1 / (g1 + 1.0)) * (Ms * Ms - 1.0) + 1.0) * base_pressure;
    double Y_ref = 1.0;
    double Qref[5] = {vel_ref, vel_ref, vel_ref, rho_ref, P_ref / (g1 - 1.0)};
    int Ns[3] = {Mx, My, Mz};
    int start[3], len[3];
    for (int d = 0; d < 3; d++) {
        start[d] = Ns[d] - (int)ceil(frac * Ns[d]);
        len[d] = Ns[d] - start[d];
    }
    double *sig[3];
    for (int d = 0; d < 3; d++) {
        sig[d] = dalloc(Ns[d]);
        for (int q = 0; q < Ns[d]; q++) {
            int gI = q + 1;
            if (gI >= start[d]) {
                float r = (float)(gI - start[d]) / (float)len[d];
                sig[d][q] = A_sponge * pow((double)r, s_exp);
            } else sig[d][q] = 0.0;
        }
    }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < Mx; i++)
        for (int k = 0; k < Mz; k++)
            for (int j = 0; j < My; j++) {
                size_t p = IX(c, j, k, i);
                double s = sig[0][i] + sig[1][j] + sig[2][k];
                for (int l = 0; l < 5; l++)
                    Qrhs[l * n3 + p] = Qrhs[l * n3 + p] - s * (Q[l * n3 + p] - Qref[l]);
                Yrhs[p] = Yrhs[p] - s * (Q[3 * n3 + p] * Y[p] - Q[3 * n3 + p] * Y_ref);
            }
    for (int d = 0; d < 3; d++) free(sig[d]);
}

/* Fix_Pressure pproc/pproc_mf.f:190-233 */
void orc_fix_pressure(orc *c, double *Q, const double *Y) {
    if (!Y) Y = c->Y;   /* the periodic single-fluid routines take no Y */
    (void)Y;
    size_t n3 = c->n3;
    double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    const double *g = c->gamma_eff;
    /* Fix_Pressure of the periodic family, src/lddrk4_periodic_sf.f:436-473 */
    double base_pressure = is_per(c) ? 0.71463 : 0.71429;
    PAR FOR_P {
        double fac1 = g[p] - 1.0;
        double Vs = 1.0 / Q4[p];
        double P = fac1 * (Q5[p] - 5.0e-1 * Vs * (Q1[p] * Q1[p] + Q2[p] * Q2[p] + Q3[p] * Q3[p]));
        if (P < 0.0) P = base_pressure;
        Q5[p] = (1.0 / fac1) * P + 5.0e-1 * Vs * (Q1[p] * Q1[p] + Q2[p] * Q2[p] + Q3[p] * Q3[p]);
    }
}

/* Compute_CFL src/lddrk4_nonperiodic_mf.f:7-66 */
void orc_compute_cfl(orc *c, const double *Q, double *cfl_stab, double *cfl_resv) {
    size_t n3 = c->n3;
    const double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    const double *g = c->gamma_eff;
    double DX = c->DX, DY = c->DY, DZ = c->DZ;
    double m1 = -INFINITY, m2 = -INFINITY;
#pragma omp parallel for schedule(static) reduction(max : m1, m2)
    for (size_t p = 0; p < n3; p++) {
        double fac = g[p] * (g[p] - 1.0);
        double tmp1 = 1.0 / Q4[p];
        double tmp2 = sqrt(fac * tmp1 * (Q5[p] - 5.0e-1 * tmp1 * (Q1[p] * Q1[p] + Q2[p] * Q2[p] + Q3[p] * Q3[p])));
        double ux = fabs(Q1[p] * tmp1), uy = fabs(Q2[p] * tmp1), uz = fabs(Q3[p] * tmp1);
        double w1 = ((tmp2 + ux) * k_max / DX + (tmp2 + uy) * k_max / DY + (tmp2 + uz) * k_max / DZ);
        double w2 = ((tmp2 + ux) * k_hug / DX + (tmp2 + uy) * k_hug / DY + (tmp2 + uz) * k_hug / DZ);
        if (w1 > m1) m1 = w1;
        if (w2 > m2) m2 = w2;
    }
    *cfl_stab = m1; *cfl_resv = m2;
}

/* Compute_Tstep src/lddrk4_nonperiodic_mf.f:75-160 */
/* Compute_Tstep of the periodic family, src/lddrk4_periodic_sf.f:74-145:
 * hyperviscous limits from step 2 on, single-fluid temperature, and the
 * factor 0.2 written as a default-REAL literal (float32). */
static double compute_tstep_sf(orc *c, const double *Q, double cfl_resv, int step) {
    size_t n3 = c->n3;
    const double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    double Tstep = c->p.cfl_cal / cfl_resv;
    double del = c->DX, gam = c->p.gamma1;
    double fac = gam * (gam - 1.0);
    if (c->p.hyper_param == 1 && step > 1) {
        double m3 = INFINITY, m4 = INFINITY, m5 = INFINITY;
        const double *vh = c->hyp[H_VISC], *bh = c->hyp[H_BETA], *kh = c->hyp[H_K];
#pragma omp parallel for schedule(static) reduction(min : m3, m4, m5)
        for (size_t p = 0; p < n3; p++) {
            double tmp1 = 1.0 / Q4[p];
            double tmp2 = sqrt(fac * tmp1 * (Q5[p] - 5.0e-1 * tmp1 * (Q1[p] * Q1[p] + Q2[p] * Q2[p] + Q3[p] * Q3[p])));
            double T = gam * tmp1 * (Q5[p] - 5.0e-1 * tmp1 * (Q1[p] * Q1[p] + Q2[p] * Q2[p] + Q3[p] * Q3[p]));
            double w3 = Q4[p] * pow(del, 2.0) / vh[p];
            double w4 = Q4[p] * pow(del, 2.0) / bh[p];
            double w5 = Q4[p] * pow(del * tmp2, 2.0) / ((kh[p]) * T);
            if (w3 < m3) m3 = w3;
            if (w4 < m4) m4 = w4;
            if (w5 < m5) m5 = w5;
        }
        const double f02 = (double)0.2f;
        double t = c->p.cfl_cal / cfl_resv;
        double cand[3] = {f02 * m3, f02 * m4, f02 * m5};
        for (int q = 0; q < 3; q++) if (cand[q] < t) t = cand[q];
        Tstep = t;
    }
    c->Tstep = Tstep;
    return Tstep;
}

double orc_compute_tstep(orc *c, const double *Q, const double *Y, double cfl_resv, int step) {
    if (!Y) Y = c->Y;   /* the periodic single-fluid routines take no Y */
    if (is_per(c)) return compute_tstep_sf(c, Q, cfl_resv, step);
    size_t n3 = c->n3;
    const double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    const double *g = c->gamma_eff;
    double Tstep = c->p.cfl_cal / cfl_resv;
    double del = c->DX;
    if (c->p.hyper_param == 1 && step > 0) {
        double g1 = c->p.gamma1, g2 = c->p.gamma2, eps = c->p.epsilon;
        double m3 = INFINITY, m4 = INFINITY, m5 = INFINITY, m6 = INFINITY;
        const double *vh = c->hyp[H_VISC], *bh = c->hyp[H_BETA], *kh = c->hyp[H_K], *Dh = c->hyp[H_D];
#pragma omp parallel for schedule(static) reduction(min : m3, m4, m5, m6)
        for (size_t p = 0; p < n3; p++) {
            double fac = g[p] * (g[p] - 1.0);
            float fac1 = (float)(Y[p] + (eps * (g1 - 1.0) / (g2 - 1.0)) * (1.0 - Y[p]));
            double tmp1 = 1.0 / Q4[p];
            double ke = 5.0e-1 * tmp1 * (Q1[p] * Q1[p] + Q2[p] * Q2[p] + Q3[p] * Q3[p]);
            double tmp2 = sqrt(fac * tmp1 * (Q5[p] - ke));
            double T = g1 * tmp1 * (Q5[p] - 5.0e-1 * tmp1 * (Q1[p] * Q1[p] + Q2[p] * Q2[p] + Q3[p] * Q3[p]));
            T = T / (double)fac1;
            double w3 = Q4[p] * pow(del, 2.0) / vh[p];
            double w4 = Q4[p] * pow(del, 2.0) / bh[p];
            double w5 = Q4[p] * pow(del * tmp2, 2.0) / (kh[p] * T);
            double w6 = pow(del, 2.0) / Dh[p];
            if (w3 < m3) m3 = w3;
            if (w4 < m4) m4 = w4;
            if (w5 < m5) m5 = w5;
            if (w6 < m6) m6 = w6;
        }
        double t = c->p.cfl_cal / cfl_resv;
        double cand[4] = {0.2 * m3, 0.2 * m4, 0.2 * m5, 0.2 * m6};
        for (int q = 0; q < 4; q++) if (cand[q] < t) t = cand[q];
        Tstep = t;
    }
    c->Tstep = Tstep;
    return Tstep;
}

/* ---- monitoring (Compute_Sum order: I, J, K with K innermost) ----------- */
static double csum(const orc *c, const double *F) {
    double s = 0.0;
    for (int i = 0; i < c->M[0]; i++)
        for (int j = 0; j < c->M[1]; j++)
            for (int k = 0; k < c->M[2]; k++) s = s + F[IX(c, j, k, i)];
    return s;
}
static void monitors(orc *c) {
    size_t n3 = c->n3;
    double *Q = c->Q, *Y = c->Y, *tmp = NEWF(c), *tmp2 = NEWF(c);
    double N = (double)(c->M[0] * c->M[1] * c->M[2]);
    /* Compute_Mom :209-231 */
    c->mon[1] = csum(c, Q) / N;
    c->mon[2] = csum(c, Q + n3) / N;
    c->mon[3] = csum(c, Q + 2 * n3) / N;
    /* Compute_KE :168-201 */
    PAR FOR_P {
        double t = 1.0 / Q[3 * n3 + p];
        double acc = 0.0;
        for (int l = 0; l < 3; l++) {
            double u = Q[l * n3 + p] * t;
            acc = acc + Q[3 * n3 + p] * u * u;
        }
        tmp[p] = acc;
    }
    c->mon[0] = 0.5 * csum(c, tmp) / N;
    /* Compute_Mass :240-258 */
    c->mon[4] = csum(c, Q + 3 * n3) / N;
    /* Compute_Energy :265-278 */
    c->mon[5] = csum(c, Q + 4 * n3) / N;
    if (is_per(c)) {
        /* Compute_Entropy src/lddrk4_periodic_sf.f:268-300: fac1 is an
         * undeclared (default REAL, float32) local; Entropy2 is not computed */
        float fac1 = (float)(c->p.gamma1 - 1.0);
        double gam = c->p.gamma1;
        PAR FOR_P {
            double Vs = 1.0 / Q[3 * n3 + p];
            double q1 = Q[p], q2 = Q[n3 + p], q3 = Q[2 * n3 + p];
            double P = (double)fac1 * (Q[4 * n3 + p] - 5.0e-1 * Vs * (q1 * q1 + q2 * q2 + q3 * q3));
            tmp[p] = Q[3 * n3 + p] * log(P * pow(Vs, gam));
        }
        c->mon[6] = csum(c, tmp) / N;
        c->mon[7] = 0.0;
        free(tmp); free(tmp2);
        return;
    }
    /* Compute_Entropy :287-327 */
    PAR FOR_P {
        double fac1 = c->gamma_eff[p] - 1.0;
        double Vs = 1.0 / Q[3 * n3 + p];
        double q1 = Q[p], q2 = Q[n3 + p], q3 = Q[2 * n3 + p];
        double P = fac1 * (Q[4 * n3 + p] - 5.0e-1 * Vs * (q1 * q1 + q2 * q2 + q3 * q3));
        tmp[p] = Q[3 * n3 + p] * log(P * pow(Vs, c->gamma_eff[p]));
        tmp2[p] = Q[3 * n3 + p] * tmp[p] * tmp[p];
    }
    c->mon[6] = csum(c, tmp) / N;
    c->mon[7] = csum(c, tmp2) / N;
    (void)Y;
    free(tmp); free(tmp2);
}

/* Second-loop coefficients of the commented-out HHM 4-6 scheme,
 * src/header:267-276 (used by rk_mode 1 of the periodic family). */
static const double alpha2_hhm[6] = {0.0, -4.4127377153877382565e-1, -1.073982008079781868e0,
                                     -1.7063570791256758809e0, -2.7979293162682443056e0,
                                     -4.0913537120919160454e0};
static const double beta2_hhm[6] = {1.1584888181285561688e-1, 3.7287699051652864918e-1,
                                    7.3795368921435295698e-1, 5.7981109366311039538e-1,
                                    1.031284991300145194e0, 1.5e-1};

/* LDDRK4 of the periodic family, src/lddrk4_periodic_sf.f:311-430:
 * 5 stages with alpha1/beta1, then 6 stages with alpha2/beta2 (never
 * assigned in the reference build: zero, rk_mode 0). */
static void lddrk4_sf(orc *c, double *time, int *step) {
    size_t n3 = c->n3;
    double *Q = c->Q, *dQ = c->dQ, *QW = c->QW;
    double *Qf = dalloc(5 * n3);
    double dt = c->Tstep;
    for (int loop = 0; loop < 2; loop++) {
        memset(QW, 0, 5 * n3 * 8);
        int ns = loop == 0 ? 5 : 6;
        for (int K = 0; K < ns; K++) {
            double al, be;
            if (loop == 0) { al = alpha1_rk[K]; be = beta1_rk[K]; }
            else if (c->p.rk_mode == 1) { al = alpha2_hhm[K]; be = beta2_hhm[K]; }
            else { al = 0.0; be = 0.0; }
            orc_rhs(c, Q, dQ, c->Y);
            orc_hyper_rhs(c, Q, dQ, c->Y);
            graph_count(c, 5 * 40.0);
            PAR for (size_t q = 0; q < 5 * n3; q++) QW[q] = al * QW[q] + dt * dQ[q];
            PAR for (size_t q = 0; q < 5 * n3; q++) Q[q] = Q[q] + be * QW[q];
            orc_compact_filter(c, Q, Qf, 5);
            memcpy(Q, Qf, 5 * n3 * 8);
            orc_fix_pressure(c, Q, c->Y);
        }
        *time = *time + dt;
    }
    *step = *step + 1;
    monitors(c);
    free(Qf);
}

/* LDDRK4 src/lddrk4_nonperiodic_mf.f:428-541 */
void orc_lddrk4(orc *c, double *time, int *step) {
    if (is_per(c)) { lddrk4_sf(c, time, step); return; }
    size_t n3 = c->n3;
    double *Q = c->Q, *dQ = c->dQ, *QW = c->QW, *Y = c->Y, *drYi = c->drYi, *rYW = c->rYW;
    double *rY = NEWF(c), *Qf = dalloc(5 * n3);
    double dt = c->Tstep;
    for (int loop = 0; loop < 2; loop++) {
        memset(QW, 0, 5 * n3 * 8);
        memset(rYW, 0, n3 * 8);
        for (int K = 0; K < 5; K++) {
            double al, be;
            if (loop == 0 || c->p.rk_mode == 1) { al = alpha1_rk[K]; be = beta1_rk[K]; }
            else { al = 0.0; be = 0.0; }
            double tstage = *time + (loop == 0 || c->p.rk_mode == 1 ? c1_rk[K] : 0.0) * dt;
            orc_compute_gamma(c, Y);
            orc_rhs(c, Q, dQ, Y);
            orc_hyper_rhs(c, Q, dQ, Y);
            orc_species_rhs(c, Q, dQ, Y, drYi);
            orc_bc_rhs(c, Q, dQ, Y, drYi, tstage);
            orc_sponge_forcing(c, Q, dQ, Y, drYi);
            PAR FOR_P rY[p] = Q[3 * n3 + p] * Y[p];
            graph_count(c, 6 * 40.0);       /* Q (5 fields) and rY */
            PAR for (size_t q = 0; q < 5 * n3; q++) QW[q] = al * QW[q] + dt * dQ[q];
            PAR for (size_t q = 0; q < 5 * n3; q++) Q[q] = Q[q] + be * QW[q];
            PAR FOR_P rYW[p] = al * rYW[p] + dt * drYi[p];
            PAR FOR_P rY[p] = rY[p] + be * rYW[p];
            orc_compact_filter(c, Q, Qf, 5);
            orc_filter(c, 0, 0, rY, rY);
            orc_filter(c, 1, 0, rY, rY);
            orc_filter(c, 2, 0, rY, rY);
            memcpy(Q, Qf, 5 * n3 * 8);
            PAR FOR_P Y[p] = rY[p] / Q[3 * n3 + p];
            orc_fix_pressure(c, Q, Y);
        }
        *time = *time + dt;
    }
    *step = *step + 1;
    monitors(c);
    free(rY); free(Qf);
}

/* main loop body src/main_mf.f:137-143 (march_mode 1) */
void orc_step(orc *c, double *time, int *step) {
    double cs, cr;
    orc_compute_cfl(c, c->Q, &cs, &cr);
    c->last_cfl_resv = cr;
    orc_compute_tstep(c, c->Q, c->Y, cr, *step);
    orc_lddrk4(c, time, step);
}

void orc_get_monitors(orc *c, double out[10]) {
    memcpy(out, c->mon, 8 * sizeof(double));
    out[8] = c->last_cfl_resv;
    out[9] = c->Tstep;
}

/* ---- state / COMMON access -------------------------------------------------- */
void orc_set_state(orc *c, const double *Q, const double *Y) {
    memcpy(c->Q, Q, 5 * c->n3 * 8);
    if (Y && !is_per(c)) memcpy(c->Y, Y, c->n3 * 8);
    memset(c->QW, 0, 5 * c->n3 * 8); memset(c->dQ, 0, 5 * c->n3 * 8);
    memset(c->rYW, 0, c->n3 * 8); memset(c->drYi, 0, c->n3 * 8);
}
void orc_get_state(orc *c, double *Q, double *Y) {
    if (Q) memcpy(Q, c->Q, 5 * c->n3 * 8);
    if (Y) memcpy(Y, c->Y, c->n3 * 8);
}
void orc_set_tstep(orc *c, double t) { c->Tstep = t; }
double orc_get_tstep(orc *c) { return c->Tstep; }

static double *common_ptr(orc *c, const char *name, size_t *nf) {
    static const char *gn[12] = {"dux_dx", "duy_dx", "duz_dx", "dux_dy", "duy_dy", "duz_dy",
                                 "dux_dz", "duy_dz", "duz_dz", "dTdx", "dTdy", "dTdz"};
    static const char *hn[4] = {"beta_hyper", "visc_hyper", "k_hyper", "D_hyper"};
    *nf = 1;
    for (int q = 0; q < 12; q++) if (!strcmp(name, gn[q])) return c->grad[q];
    for (int q = 0; q < 4; q++) if (!strcmp(name, hn[q])) return c->hyp[q];
    if (!strcmp(name, "gamma_eff")) return c->gamma_eff;
    if (!strcmp(name, "drYi")) return c->drYi;
    if (!strcmp(name, "rYW")) return c->rYW;
    *nf = 5;
    if (!strcmp(name, "dQ")) return c->dQ;
    if (!strcmp(name, "QW")) return c->QW;
    return NULL;
}
int orc_get_common(orc *c, const char *name, double *out) {
    size_t nf; double *p = common_ptr(c, name, &nf);
    if (!p) return -1;
    memcpy(out, p, nf * c->n3 * 8);
    return 0;
}
int orc_set_common(orc *c, const char *name, const double *in) {
    size_t nf; double *p = common_ptr(c, name, &nf);
    if (!p) return -1;
    memcpy(p, in, nf * c->n3 * 8);
    return 0;
}

/* ---- Output-side diagnostics ------------------------------------------------ */
/* grid coordinate xcor(I) of Uniform_X, src/grid.f:116-128 (i 0-based) */
static double gcor(const orc *c, int d, int i) {
    const double leng[3] = {c->p.x_leng, c->p.y_leng, c->p.z_leng};
    const double start[3] = {c->p.x_start, c->p.y_start, c->p.z_start};
    return start[d] + leng[d] * (double)(i) / (double)(c->M[d] - 1);
}

/* Compute_Grad src/grad_sym.f:13-120: Grad = (w_x, w_y, w_z, dilatation) of
 * the state in /RKWORK/, the nine velocity derivatives left in /GRAD/ as the
 * reference leaves them, MaxDil = max|Dil| (Compute_Max), Enstrophy =
 * 0.5*sum(w.w)/(Nx*Ny*Nz) with Compute_Sum's loop order (src/auxiliary_mf.f:
 * 187-213: I outer, K inner). */
void orc_compute_grad(orc *c, double *Grad, double *maxdil, double *enstrophy) {
    const size_t n3 = c->n3;
    double *U = dalloc(3 * n3);
    const double *Q = c->Q;
    for (size_t p = 0; p < n3; p++) {
        double tmp = 1.0 / Q[3 * n3 + p];
        U[p] = Q[p] * tmp;
        U[n3 + p] = Q[n3 + p] * tmp;
        U[2 * n3 + p] = Q[2 * n3 + p] * tmp;
    }
    double **G = c->grad;
    orc_dfd(c, 1, 0, U + 2 * n3, G[G_DUZ_DY], 0, 1.0);
    orc_dfd(c, 2, 0, U + n3, G[G_DUY_DZ], 0, 1.0);
    for (size_t p = 0; p < n3; p++) Grad[p] = G[G_DUZ_DY][p] - G[G_DUY_DZ][p];
    orc_dfd(c, 0, 0, U + 2 * n3, G[G_DUZ_DX], 0, 1.0);
    orc_dfd(c, 2, 0, U, G[G_DUX_DZ], 0, 1.0);
    for (size_t p = 0; p < n3; p++) Grad[n3 + p] = G[G_DUX_DZ][p] - G[G_DUZ_DX][p];
    orc_dfd(c, 0, 0, U + n3, G[G_DUY_DX], 0, 1.0);
    orc_dfd(c, 1, 0, U, G[G_DUX_DY], 0, 1.0);
    for (size_t p = 0; p < n3; p++) Grad[2 * n3 + p] = G[G_DUY_DX][p] - G[G_DUX_DY][p];
    orc_dfd(c, 0, 1, U, G[G_DUX_DX], 0, 1.0);
    orc_dfd(c, 1, 1, U + n3, G[G_DUY_DY], 0, 1.0);
    orc_dfd(c, 2, 1, U + 2 * n3, G[G_DUZ_DZ], 0, 1.0);
    for (size_t p = 0; p < n3; p++) Grad[3 * n3 + p] = G[G_DUX_DX][p] + G[G_DUY_DY][p] + G[G_DUZ_DZ][p];
    double mx = 0.0, sum = 0.0;
    for (size_t p = 0; p < n3; p++) if (fabs(Grad[3 * n3 + p]) > mx) mx = fabs(Grad[3 * n3 + p]);
    for (int i = 0; i < c->M[0]; i++)
        for (int j = 0; j < c->M[1]; j++)
            for (int k = 0; k < c->M[2]; k++) {
                size_t p = IX(c, j, k, i);
                double w1 = Grad[p], w2 = Grad[n3 + p], w3 = Grad[2 * n3 + p];
                sum = sum + (w1 * w1 + w2 * w2 + w3 * w3);
            }
    *maxdil = mx;
    *enstrophy = 0.5 * sum / (double)(c->M[0] * c->M[1] * c->M[2]);
    free(U);
}

/* N_avg src/header:14 (symmetry boundaries) */
int orc_shell_count(const orc *c) { return c->M[0] / 2 + 10 * (c->M[0] / 128); }

/* radius of cell (i,j,k) from the origin, IX = DBLE(II-1)
 * (src/auxiliary_mf.f:289-300, pproc/pproc_mf.f:102-110) */
static double cell_rad(const orc *c, int i, int j, int k) {
    double IXd = (double)(i + 1) - 1.0, IYd = (double)(j + 1) - 1.0, IZd = (double)(k + 1) - 1.0;
    return sqrt((IXd * c->DX) * (IXd * c->DX) + (IYd * c->DY) * (IYd * c->DY) + (IZd * c->DZ) * (IZd * c->DZ));
}

/* Compute_shell_avg src/auxiliary_mf.f:266-332: N_avg bins, the first three
 * 2*DX*sqrt(3) wide and the rest DX*sqrt(3); empty bins divide 0 by 0 */
static void shell_avg(const orc *c, const double *F, double *avg) {
    const int na = orc_shell_count(c);
    double *r = dalloc(na + 1), *s = dalloc(na);
    long *cnt = (long *)calloc(na, sizeof(long));
    r[0] = 0.0;
    for (int M = 2; M <= na + 1; M++)
        r[M - 1] = r[M - 2] + (M <= 4 ? c->DX * 2.0 * sqrt(3.0) : c->DX * sqrt(3.0));
    for (int i = 0; i < c->M[0]; i++)
        for (int j = 0; j < c->M[1]; j++)
            for (int k = 0; k < c->M[2]; k++) {
                double rad = cell_rad(c, i, j, k);
                for (int M = 0; M < na; M++)
                    if (rad >= r[M] && rad < r[M + 1]) { s[M] = s[M] + F[IX(c, j, k, i)]; cnt[M]++; }
            }
    for (int M = 0; M < na; M++) avg[M] = s[M] / (double)cnt[M];
    free(r); free(s); free(cnt);
}

/* Compute_SRM_Stats pproc/pproc_mf.f:4-186: radial velocity Ur, its shell
 * average and that of Y, tke = |u_t|^2 + (Ur - <Ur>)^2 summed over the cells
 * that fall in one of its (uniform, DX*sqrt(3)) bins, and the mixing width
 * hmix = sum 8<Y>(1-<Y>)DX*sqrt(3) over bins with 0 < <Y> < 1.  Cells beyond
 * the last bin leave tke unassigned in the reference (a local array); here
 * they contribute 0. */
void orc_compute_srm_stats(orc *c, double *hmix, double *tke_total, double *ur_avg, double *y_avg) {
    const size_t n3 = c->n3;
    const int na = orc_shell_count(c);
    const double *Q = c->Q;
    double *U = dalloc(3 * n3), *Ur = dalloc(n3), *rad = dalloc(n3);
    for (int i = 0; i < c->M[0]; i++)
        for (int j = 0; j < c->M[1]; j++)
            for (int k = 0; k < c->M[2]; k++) {
                size_t p = IX(c, j, k, i);
                double tmp = 1.0 / Q[3 * n3 + p];
                U[p] = Q[p] * tmp; U[n3 + p] = Q[n3 + p] * tmp; U[2 * n3 + p] = Q[2 * n3 + p] * tmp;
                rad[p] = cell_rad(c, i, j, k);
                if (i == 0 && j == 0 && k == 0) Ur[p] = 0.0;
                else Ur[p] = (gcor(c, 0, i) / rad[p]) * U[p] + (gcor(c, 1, j) / rad[p]) * U[n3 + p] +
                             (gcor(c, 2, k) / rad[p]) * U[2 * n3 + p];
            }
    double *ura = dalloc(na), *ya = dalloc(na), *r = dalloc(na + 1);
    shell_avg(c, Ur, ura);
    shell_avg(c, c->Y, ya);
    r[0] = 0.0;
    for (int M = 2; M <= na + 1; M++) r[M - 1] = r[M - 2] + c->DX * sqrt(3.0);
    double tke = 0.0;
    for (int i = 0; i < c->M[0]; i++)
        for (int j = 0; j < c->M[1]; j++)
            for (int k = 0; k < c->M[2]; k++) {
                size_t p = IX(c, j, k, i);
                double t = 0.0;
                for (int M = 0; M < na; M++)
                    if (rad[p] >= r[M] && rad[p] < r[M + 1]) {
                        double d = Ur[p] - ura[M];
                        double urp2 = d * d, t1 = 0.0, t2 = 0.0, t3 = 0.0;
                        if (i > 0 && j > 0 && k > 0) {
                            double IXd = (double)(i + 1) - 1.0, IYd = (double)(j + 1) - 1.0, IZd = (double)(k + 1) - 1.0;
                            t1 = U[p] - Ur[p] * (IXd * c->DX / rad[p]);
                            t2 = U[n3 + p] - Ur[p] * (IYd * c->DY / rad[p]);
                            t3 = U[2 * n3 + p] - Ur[p] * (IZd * c->DZ / rad[p]);
                        }
                        double utp2 = t1 * t1 + t2 * t2 + t3 * t3;
                        t = utp2 + urp2;
                    }
                tke = tke + t;
            }
    *tke_total = tke / (double)(c->M[0] * c->M[1] * c->M[2]);
    double h = 0.0;
    for (int M = 0; M < na; M++)
        if (ya[M] > 0.0 && ya[M] < 1.0) h = h + 8.0 * ya[M] * (1.0 - ya[M]) * c->DX * sqrt(3.0);
    *hmix = h;
    if (ur_avg) memcpy(ur_avg, ura, na * sizeof(double));
    if (y_avg) memcpy(y_avg, ya, na * sizeof(double));
    free(U); free(Ur); free(rad); free(ura); free(ya); free(r);
}

/* Generate_Shock_Surface src/shock.f:163-260: cells with beta_hyper above
 * 0.1*max(beta_hyper) form the shock; their centroid, mean distance from it
 * and sqrt(sum (rad - rad_avg)^2)/(n*rad_avg) */
void orc_shock_surface(orc *c, double *rad_avg, double *rad_skew_rms) {
    const double *b = c->hyp[H_BETA];
    double bmax = -INFINITY;
    for (size_t p = 0; p < c->n3; p++) if (b[p] > bmax) bmax = b[p];
    const double thr = 0.1 * bmax;
    double xc = 0.0, yc = 0.0, zc = 0.0, n = 0.0;
    for (int i = 0; i < c->M[0]; i++)
        for (int j = 0; j < c->M[1]; j++)
            for (int k = 0; k < c->M[2]; k++)
                if (b[IX(c, j, k, i)] > thr) {
                    xc = xc + gcor(c, 0, i); yc = yc + gcor(c, 1, j); zc = zc + gcor(c, 2, k); n = n + 1.0;
                }
    xc = xc / n; yc = yc / n; zc = zc / n;
    double rs = 0.0;
    for (int i = 0; i < c->M[0]; i++)
        for (int j = 0; j < c->M[1]; j++)
            for (int k = 0; k < c->M[2]; k++)
                if (b[IX(c, j, k, i)] > thr) {
                    double dx = gcor(c, 0, i) - xc, dy = gcor(c, 1, j) - yc, dz = gcor(c, 2, k) - zc;
                    rs = rs + sqrt(dx * dx + dy * dy + dz * dz);
                }
    const double ra = rs / n;
    double sk = 0.0;
    for (int i = 0; i < c->M[0]; i++)
        for (int j = 0; j < c->M[1]; j++)
            for (int k = 0; k < c->M[2]; k++)
                if (b[IX(c, j, k, i)] > thr) {
                    double dx = gcor(c, 0, i) - xc, dy = gcor(c, 1, j) - yc, dz = gcor(c, 2, k) - zc;
                    double d = sqrt(dx * dx + dy * dy + dz * dz) - ra;
                    sk = sk + d * d;
                }
    *rad_avg = ra;
    *rad_skew_rms = sqrt(sk) / (n * ra);
}

/* MakePaddedArrays, src/vis_silo_mf.f:440-689, on one rank (Px = Py = Pz = 1).
 * W(My+1, Mz+1, Mx+1, 11): the primitive variables of :494-510 (u, v, w =
 * Q1..Q3 / Q4, rho = Q4, P = fac1 (Q5 - 0.5 Vs (Q1^2 + Q2^2 + Q3^2)) with
 * fac1 = gamma_eff - 1, Vs = 1/Q4), the four Grad fields (w_x, w_y, w_z,
 * dilatation), gamma_eff and Y.  Without neighbour ranks every padding node
 * copies the last node of its direction: faces :640-666, edges :668-684,
 * corner :686.  xx/yy/zz (Mx+1, My+1, Mz+1): the coordinates of Setup_Grid
 * (src/grid.f:28-40, Uniform_X :116-128), the extra node one spacing
 * (gxcor(2) - gxcor(1)) beyond the last (:486-491). */
void orc_make_padded_arrays(orc *c, const double *Grad, double *W, double *xx, double *yy, double *zz) {
    const int Mx = c->M[0], My = c->M[1], Mz = c->M[2];
    const size_t n3 = c->n3, Pj = (size_t)My + 1, Pk = (size_t)Mz + 1;
    const size_t np = Pj * Pk * ((size_t)Mx + 1);
    const double *Q = c->Q;
    for (int i = 0; i <= Mx; i++)
        for (int k = 0; k <= Mz; k++)
            for (int j = 0; j <= My; j++) {
                const size_t p = (size_t)j + Pj * ((size_t)k + Pk * (size_t)i);
                const size_t q = IX(c, j < My ? j : My - 1, k < Mz ? k : Mz - 1, i < Mx ? i : Mx - 1);
                const double q1 = Q[q], q2 = Q[n3 + q], q3 = Q[2 * n3 + q], q4 = Q[3 * n3 + q], q5 = Q[4 * n3 + q];
                const double fac1 = c->gamma_eff[q] - 1.0;
                const double vs = 1.0 / q4;
                W[p] = q1 / q4;
                W[np + p] = q2 / q4;
                W[2 * np + p] = q3 / q4;
                W[3 * np + p] = q4;
                W[4 * np + p] = fac1 * (q5 - 5.0e-1 * vs * (q1 * q1 + q2 * q2 + q3 * q3));
                for (int f = 0; f < 4; f++) W[(5 + f) * np + p] = Grad[f * n3 + q];
                W[9 * np + p] = c->gamma_eff[q];
                W[10 * np + p] = c->Y[q];
            }
    const st_params *pp = &c->p;
    const double st[3] = {pp->x_start, pp->y_start, pp->z_start}, ln[3] = {pp->x_leng, pp->y_leng, pp->z_leng};
    double *cor[3] = {xx, yy, zz};
    for (int d = 0; d < 3; d++) {
        const int n = c->M[d];
        for (int i = 0; i < n; i++) cor[d][i] = st[d] + ln[d] * (double)i / (double)(n - 1);
        cor[d][n] = cor[d][n - 1] + (cor[d][1] - cor[d][0]);
    }
}
