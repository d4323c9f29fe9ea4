/*
 * st_oracle_radial.c - CPU oracle (TEST INFRASTRUCTURE: GPU results are checked against it) for the
 * 1-D spherical-radial single-fluid family: src/rhsv_radial.f,
 * src/derivCDopt6_radial.f, src/filters_nonperiodic.f (x passes),
 * src/hyper_radial.f and src/lddrk4_nonperiodic_sf.f, one problem being one
 * run of that program with Nx = n, one rank.
 *
 * A problem is a line of n points spanning -R..R; its state is
 * (u_r, rho, s = P/rho^gamma) (the reference's Q(:,1), Q(:,4), Q(:,5);
 * Q(:,2) and Q(:,3) are identically zero and are not stored).
 *
 * Where the shipped reference does not define the radial program's
 * behaviour, this restatement fixes it as follows:
 *  - Fix_Pressure and Debug, called by the radial LDDRK4
 *    (src/lddrk4_nonperiodic_sf.f:403,437), come from pproc_radial.o, whose
 *    source is not part of the reference: no pressure clip is applied.
 *  - the y and z filter passes and the y/z CFL terms act on directions of one
 *    point (My = Mz = 1), for which the reference's stencils and DY, DZ are
 *    undefined: the filters are the x passes, the CFL sum is its x term.
 *  - the second derivative uses the FDL3DI constants as the tridiagonal
 *    scheme they define (zero weight on f(i+-3), centre weight 2(a2+b2)),
 *    as in the periodic family.
 *
 * Parity unpinned: the reference ships no radial test vectors and cannot be
 * compiled here; pinned by the analytic tests in tests/.
 * Build with -ffp-contract=off.
 */
#include "st_oracle.h"
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>

static const double a1_p6 = 14.0 / 18.0, b1_p6 = 1.0 / 36.0, c1_p6 = 0.0;
static const double a2_p6 = 12.0 / 11.0, b2_p6 = 3.0 / 44.0, c2_rad = 0.0;
#define D2_RAD (2.0 * (a2_p6 + b2_p6))
static const double closure1 = 5.0 / 9.0, closure2 = 1.0 / 1.8e1;
static const double closure3 = 1.0 / 3.6e1, closure4 = 7.0 / 9.0;
static const double closure5 = 3.0 / 4.4e1, closure6 = 1.2e1 / 1.1e1;
static const double alpha_f4 = 6.6624e-01, beta_f4 = 1.6688e-01;
static const double a0_f4 = 9.9965e-01, a1_f4 = 0.66652, a2_f4 = 0.16674, a3_f4 = 4.0e-05, a4_f4 = -5.0e-06;
static const double bndy_alpha = 0.45;

static const double alpha1_rk[5] = {0.0, -4.801594388477952e-01, -1.404247195200064e+00,
                                    -2.016477077503357e+00, -1.056444269767207e+00};
static const double beta1_rk[5] = {1.028639988104959e-01, 7.408540575766301e-01, 7.426530946683799e-01,
                                   4.694937902357905e-01, 1.881733382887932e-01};
static const double alpha2_hhm[6] = {0.0, -4.4127377153877382565e-1, -1.073982008079781868e0,
                                     -1.7063570791256758809e0, -2.7979293162682443056e0,
                                     -4.0913537120919160454e0};
static const double beta2_hhm[6] = {1.1584888181285561688e-1, 3.7287699051652864918e-1,
                                    7.3795368921435295698e-1, 5.7981109366311039538e-1,
                                    1.031284991300145194e0, 1.5e-1};

static double *ralloc(size_t n) {
    double *p = (double *)calloc(n ? n : 1, sizeof(double));
    if (!p) { fprintf(stderr, "oracle: out of memory\n"); abort(); }
    return p;
}

/* Setup_Grid src/grid.f:15-45 (x_start = 0): DX = gxcor(2) - gxcor(1) */
static double rad_dx(int n, double x_leng) {
    double g1 = x_leng * (double)(0) / (double)(n - 1), g2 = x_leng * (double)(1) / (double)(n - 1);
    return g2 - g1;
}

/* rad(I) = |(REAL(I - Nx/2) - 0.5) DX|, src/rhsv_radial.f:55-59 */
void orc_rad_radius(int n, double x_leng, double *rad) {
    double DX = rad_dx(n, x_leng);
    for (int i = 0; i < n; i++) {
        int II = i + 1;
        double IX = (double)(float)(II - n / 2) - 0.5;
        rad[i] = fabs(IX * DX);
    }
}

/* pentadiagonal_serial (src/pentadiagonal.f90:319-374) of one line */
static void pen_line(double *A, double *B, double *C, double *D, double *E, double *R, int n) {
    orc_pentadiagonal(A, B, C, D, E, R, n, 1, 0);
}

/* Setup_Derivatives src/derivCDopt6_radial.f:9-600 (x, one rank): order 1 or 2 */
static void rad_deriv_lhs(int n, int order, double *A, double *B, double *C, double *D, double *E) {
    double al = order == 1 ? 1.0 / 3.0 : 2.0 / 11.0;
    for (int i = 0; i < n; i++) { A[i] = 0.0; B[i] = al; C[i] = 1.0; D[i] = al; E[i] = 0.0; }
    if (order == 1) {
        B[0] = 0.0; D[0] = 2.0;
        B[n - 1] = 2.0; D[n - 1] = 0.0;
        B[1] = 1.0 / 6.0; D[1] = 1.0 / 2.0;
        B[n - 2] = 1.0 / 2.0; D[n - 2] = 1.0 / 6.0;
        B[2] = 1.0 / 3.0; D[2] = 1.0 / 3.0;
        B[n - 3] = 1.0 / 3.0; D[n - 3] = 1.0 / 3.0;
    } else {
        B[0] = 0.0; D[0] = 1.1e1;
        B[n - 1] = 1.1e1; D[n - 1] = 0.0;
        B[1] = 1.0e-1; D[1] = -7.0 / 2.0e1;
        B[n - 2] = -7.0 / 2.0e1; D[n - 2] = 1.0e-1;
        B[2] = 2.0 / 1.1e1; D[2] = 2.0 / 1.1e1;
        B[n - 3] = 2.0 / 1.1e1; D[n - 3] = 2.0 / 1.1e1;
    }
}

/* DFDX src/derivCDopt6_radial.f:637-791 (xrank = 0 = Px-1): one-sided rows
 * at both ends, and dF/dr = -dF/dx on the left half (II <= Nx/2). */
void orc_rad_dfdx(int n, double x_leng, const double *F, double *dF, int iadd, double cadd) {
    double sx = 1.0 / x_leng;
    double fac = cadd * sx * (double)(n - 1);
    double *W = ralloc((size_t)n * 6), *A = W + n, *B = W + 2 * n, *C = W + 3 * n, *D = W + 4 * n, *E = W + 5 * n;
    for (int i = 3; i <= n - 4; i++)
        W[i] = fac * (c1_p6 * (F[i + 3] - F[i - 3]) + b1_p6 * (F[i + 2] - F[i - 2]) + a1_p6 * (F[i + 1] - F[i - 1]));
    W[2] = fac * (closure3 * (F[4] - F[0]) + closure4 * (F[3] - F[1]));
    W[1] = fac * (-closure1 * F[0] - 5.0e-1 * F[1] + F[2] + closure2 * F[3]);
    W[0] = fac * (-2.5 * F[0] + 2.0 * F[1] + 5.0e-1 * F[2]);
    W[n - 3] = fac * (closure3 * (F[n - 1] - F[n - 5]) + closure4 * (F[n - 2] - F[n - 4]));
    W[n - 2] = fac * (closure1 * F[n - 1] + 5.0e-1 * F[n - 2] - F[n - 3] - closure2 * F[n - 4]);
    W[n - 1] = fac * (2.5 * F[n - 1] - 2.0 * F[n - 2] - 5.0e-1 * F[n - 3]);
    rad_deriv_lhs(n, 1, A, B, C, D, E);
    pen_line(A, B, C, D, E, W, n);
    for (int i = 0; i < n; i++) {
        double w = (i + 1 <= n / 2) ? -W[i] : W[i];
        dF[i] = iadd == 1 ? dF[i] + w : w;
    }
    free(W);
}

/* D2FDX2 src/derivCDopt6_radial.f:794-953 */
void orc_rad_d2fdx2(int n, double x_leng, const double *F, double *dF, double *d2F, int iadd) {
    double sx = 1.0 / x_leng, sx2 = sx * sx;
    double fac = ((double)((n - 1) * (n - 1))) * sx2;
    double *W = ralloc((size_t)n * 6), *A = W + n, *B = W + 2 * n, *C = W + 3 * n, *D = W + 4 * n, *E = W + 5 * n;
    for (int i = 3; i <= n - 4; i++)
        W[i] = fac * (c2_rad * (F[i + 3] + F[i - 3]) + b2_p6 * (F[i + 2] + F[i - 2]) + a2_p6 * (F[i + 1] + F[i - 1])
                      - D2_RAD * F[i]);
    W[2] = fac * (closure5 * (F[0] - 2.0 * F[2] + F[4]) + closure6 * (F[1] - 2.0 * F[2] + F[3]));
    W[1] = fac * (1.2375 * F[0] - 3.0 * F[1] + 2.325 * F[2] - 6.0e-1 * F[3] + 3.75e-2 * F[4]);
    W[0] = fac * (1.3e1 * F[0] - 2.7e1 * F[1] + 1.5e1 * F[2] - F[3]);
    W[n - 3] = fac * (closure5 * (F[n - 1] - 2.0 * F[n - 3] + F[n - 5]) + closure6 * (F[n - 2] - 2.0 * F[n - 3] + F[n - 4]));
    W[n - 2] = fac * (1.2375 * F[n - 1] - 3.0 * F[n - 2] + 2.325 * F[n - 3] - 6.0e-1 * F[n - 4] + 3.75e-2 * F[n - 5]);
    W[n - 1] = fac * (1.3e1 * F[n - 1] - 2.7e1 * F[n - 2] + 1.5e1 * F[n - 3] - F[n - 4]);
    if (iadd == 1) orc_rad_dfdx(n, x_leng, F, dF, 0, 1.0);
    rad_deriv_lhs(n, 2, A, B, C, D, E);
    pen_line(A, B, C, D, E, W, n);
    memcpy(d2F, W, (size_t)n * 8);
    free(W);
}

/* Visbal-Gaitonde closure coefficients, src/LES_header:118-146 */
static void rad_bndy(double c1[6], double c2[6], double c3[3], double c4[4]) {
    double ab = bndy_alpha, af = alpha_f4, bf = beta_f4;
    c1[0] = 0.0;
    c1[1] = 15.0 / 16.0; c1[2] = 1.0 / 4.0; c1[3] = -3.0 / 8.0; c1[4] = 1.0 / 4.0; c1[5] = -1.0 / 16.0;
    c2[0] = (1.0 / 2.0 + ab);
    c2[1] = (1.0 / 16.0 + (7.0 / 8.0) * ab);
    c2[2] = (3.0 / 4.0 + (1.0 / 2.0) * ab);
    c2[3] = (3.0 / 8.0 + (1.0 / 4.0) * ab);
    c2[4] = (-1.0 / 4.0 + (1.0 / 2.0) * ab);
    c2[5] = (1.0 / 16.0 - (1.0 / 8.0) * ab);
    c3[0] = (5.0 / 8.0 + (3.0 / 4.0) * ab);
    c3[1] = (1.0 / 2.0 + ab) / 2.0;
    c3[2] = (-1.0 / 8.0 + ab / 4.0) / 2.0;
    c4[0] = (11.0 / 16.0 + (5.0 / 8.0) * af - (5.0 / 8.0) * bf);
    c4[1] = (15.0 / 32.0 + (17.0 / 16.0) * af + (15.0 / 16.0) * bf) / 2.0;
    c4[2] = (-3.0 / 16.0 + (3.0 / 8.0) * af + (13.0 / 8.0) * bf) / 2.0;
    c4[3] = (1.0 / 32.0 - af / 16.0 + bf / 16.0) / 2.0;
}

/* Compact_Filter_X src/filters_nonperiodic.f:418-619 with the LHS of
 * Init_Filters :9-390: explicit end points, one-sided closures at both ends */
void orc_rad_filter(int n, const double *F, double *F0) {
    double c1[6], c2[6], c3[3], c4[4];
    rad_bndy(c1, c2, c3, c4);
    double *W = ralloc((size_t)n * 6), *A = W + n, *B = W + 2 * n, *C = W + 3 * n, *D = W + 4 * n, *E = W + 5 * n;
    for (int i = 4; i <= n - 5; i++)
        W[i] = a4_f4 * (F[i + 4] + F[i - 4]) + a3_f4 * (F[i + 3] + F[i - 3]) + a2_f4 * (F[i + 2] + F[i - 2])
               + a1_f4 * (F[i + 1] + F[i - 1]) + a0_f4 * F[i];
    W[0] = c1[1] * F[0] + c1[2] * F[1] + c1[3] * F[2] + c1[4] * F[3] + c1[5] * F[4];
    W[1] = c2[1] * F[0] + c2[2] * F[1] + c2[3] * F[2] + c2[4] * F[3] + c2[5] * F[4];
    W[2] = c3[2] * F[4] + c3[1] * F[3] + c3[0] * F[2] + c3[1] * F[1] + c3[2] * F[0];
    W[3] = c4[3] * F[6] + c4[2] * F[5] + c4[1] * F[4] + c4[0] * F[3] + c4[1] * F[2] + c4[2] * F[1] + c4[3] * F[0];
    W[n - 1] = c1[1] * F[n - 1] + c1[2] * F[n - 2] + c1[3] * F[n - 3] + c1[4] * F[n - 4] + c1[5] * F[n - 5];
    W[n - 2] = c2[1] * F[n - 1] + c2[2] * F[n - 2] + c2[3] * F[n - 3] + c2[4] * F[n - 4] + c2[5] * F[n - 5];
    W[n - 3] = c3[2] * F[n - 5] + c3[1] * F[n - 4] + c3[0] * F[n - 3] + c3[1] * F[n - 2] + c3[2] * F[n - 1];
    W[n - 4] = c4[3] * F[n - 7] + c4[2] * F[n - 6] + c4[1] * F[n - 5] + c4[0] * F[n - 4] + c4[1] * F[n - 3]
               + c4[2] * F[n - 2] + c4[3] * F[n - 1];
    for (int i = 0; i < n; i++) { A[i] = beta_f4; B[i] = alpha_f4; C[i] = 1.0; D[i] = alpha_f4; E[i] = beta_f4; }
    A[0] = B[0] = D[0] = E[0] = 0.0;
    A[n - 1] = B[n - 1] = D[n - 1] = E[n - 1] = 0.0;
    A[1] = 0.0; B[1] = bndy_alpha; D[1] = bndy_alpha; E[1] = 0.0;
    A[n - 2] = 0.0; B[n - 2] = bndy_alpha; D[n - 2] = bndy_alpha; E[n - 2] = 0.0;
    A[2] = 0.0; B[2] = bndy_alpha; D[2] = bndy_alpha; E[2] = 0.0;
    A[n - 3] = 0.0; B[n - 3] = bndy_alpha; D[n - 3] = bndy_alpha; E[n - 3] = 0.0;
    pen_line(A, B, C, D, E, W, n);
    memcpy(F0, W, (size_t)n * 8);
    free(W);
}

/* Gaussian_Filter_X src/filters_nonperiodic.f:1055-1224: symmetric reflection
 * at both ends; coefficients are default-REAL (float32) PARAMETERs */
void orc_rad_gauss(int n, const double *F, double *Fg) {
    const double g0 = (float)(3565.0 / 10368.0), g1 = (float)(3091.0 / 12960.0), g2 = (float)(1997.0 / 25920.0),
                 g3 = (float)(149.0 / 12960.0), g4 = (float)(107.0 / 103680.0);
    for (int i = 4; i <= n - 5; i++)
        Fg[i] = g4 * (F[i + 4] + F[i - 4]) + g3 * (F[i + 3] + F[i - 3]) + g2 * (F[i + 2] + F[i - 2])
                + g1 * (F[i + 1] + F[i - 1]) + g0 * F[i];
    Fg[0] = g4 * (2.0 * F[4]) + g3 * (2.0 * F[3]) + g2 * (2.0 * F[2]) + g1 * (2.0 * F[1]) + g0 * F[0];
    Fg[1] = g4 * (F[3] + F[5]) + g3 * (F[2] + F[4]) + g2 * (F[1] + F[3]) + g1 * (F[0] + F[2]) + g0 * F[1];
    Fg[2] = g4 * (F[2] + F[6]) + g3 * (F[1] + F[5]) + g2 * (F[0] + F[4]) + g1 * (F[1] + F[3]) + g0 * F[2];
    Fg[3] = g4 * (F[1] + F[7]) + g3 * (F[0] + F[6]) + g2 * (F[1] + F[5]) + g1 * (F[2] + F[4]) + g0 * F[3];
    int m = n - 1;
    Fg[m] = g4 * (2.0 * F[m - 4]) + g3 * (2.0 * F[m - 3]) + g2 * (2.0 * F[m - 2]) + g1 * (2.0 * F[m - 1]) + g0 * F[m];
    Fg[m - 1] = g4 * (F[m - 3] + F[m - 5]) + g3 * (F[m - 2] + F[m - 4]) + g2 * (F[m - 1] + F[m - 3])
                + g1 * (F[m] + F[m - 2]) + g0 * F[m - 1];
    Fg[m - 2] = g4 * (F[m - 2] + F[m - 6]) + g3 * (F[m - 1] + F[m - 5]) + g2 * (F[m] + F[m - 4])
                + g1 * (F[m - 1] + F[m - 3]) + g0 * F[m - 2];
    Fg[m - 3] = g4 * (F[m - 1] + F[m - 7]) + g3 * (F[m] + F[m - 6]) + g2 * (F[m - 1] + F[m - 5])
                + g1 * (F[m - 2] + F[m - 4]) + g0 * F[m - 3];
}

/* RHS_r src/rhsv_radial.f:30-157.  Q = (u, rho, s), Qrhs likewise. */
void orc_rad_rhs(const st_radial_params *p, int n, double x_leng, const double *Q, double *Qrhs) {
    const double *u = Q, *rho = Q + n, *s = Q + 2 * n;
    double *Ru = Qrhs, *Rr = Qrhs + n, *Rs = Qrhs + 2 * n;
    double *rad = ralloc((size_t)n * 4), *FF = rad + n, *Flux = rad + 2 * n, *P = rad + 3 * n;
    orc_rad_radius(n, x_leng, rad);
    memset(Qrhs, 0, 3 * (size_t)n * 8);
    orc_rad_dfdx(n, x_leng, rho, Rr, 1, -1.0);
    for (int i = 0; i < n; i++) Rr[i] = Rr[i] * u[i];
    for (int i = 0; i < n; i++) FF[i] = u[i] * rad[i] * rad[i];
    orc_rad_dfdx(n, x_leng, FF, Flux, 0, 1.0);
    for (int i = 0; i < n; i++) Rr[i] = Rr[i] - Flux[i] * (rho[i] / (rad[i] * rad[i]));
    orc_rad_dfdx(n, x_leng, u, Ru, 1, -1.0);
    for (int i = 0; i < n; i++) Ru[i] = u[i] * Ru[i];
    for (int i = 0; i < n; i++) P[i] = s[i] * pow(rho[i], p->gamma);
    orc_rad_dfdx(n, x_leng, P, FF, 0, 1.0);
    for (int i = 0; i < n; i++) Ru[i] = Ru[i] - (FF[i] / rho[i]);
    orc_rad_dfdx(n, x_leng, s, Rs, 1, -1.0);
    for (int i = 0; i < n; i++) Rs[i] = Rs[i] * u[i];
    free(rad);
}

/* Compute_hyper src/hyper_radial.f:9-62: hyp = (beta, visc) */
void orc_rad_compute_hyper(const st_radial_params *p, int n, double x_leng, const double *Q, double *hyp) {
    (void)p;
    double *S = ralloc((size_t)n * 4), *d2S = S + n, *d4S = S + 2 * n, *etag = S + 3 * n;
    orc_rad_d2fdx2(n, x_leng, Q, S, d2S, 0);
    orc_rad_d2fdx2(n, x_leng, d2S, S, d4S, 0);
    for (int i = 0; i < n; i++) d4S[i] = fabs(d4S[i]);
    orc_rad_gauss(n, d4S, etag);
    const double C_mu4 = 2.0e-3, C_beta4 = 1.0;
    double DX5 = pow(rad_dx(n, x_leng), 5.0);
    for (int i = 0; i < n; i++) {
        hyp[i] = C_beta4 * etag[i] * DX5;
        hyp[n + i] = C_mu4 * etag[i] * DX5;
    }
    free(S);
}

/* Hyper_RHS src/hyper_radial.f:75-187: Qrhs(:,1) += Qh(:,1) */
void orc_rad_hyper_rhs(const st_radial_params *p, int n, double x_leng, const double *Q, double *Qrhs,
                       double *hyp) {
    if (p->hyper_param == 0) return;
    const double *u = Q;
    orc_rad_compute_hyper(p, n, x_leng, Q, hyp);
    const double *bh = hyp, *vh = hyp + n;
    double *rad = ralloc((size_t)n * 5), *dur = rad + n, *FF = rad + 2 * n, *Flux = rad + 3 * n, *Qh = rad + 4 * n;
    orc_rad_radius(n, x_leng, rad);
    orc_rad_dfdx(n, x_leng, u, dur, 0, 1.0);
    for (int i = 0; i < n; i++) FF[i] = rad[i] * rad[i] * 2.0 * vh[i] * dur[i];
    orc_rad_dfdx(n, x_leng, FF, Flux, 0, 1.0);
    for (int i = 0; i < n; i++) Qh[i] = (1.0 / (rad[i] * rad[i])) * Flux[i];
    for (int i = 0; i < n; i++)
        FF[i] = rad[i] * rad[i] * (bh[i] - (2.0 / 3.0) * vh[i]) * (dur[i] + 2.0 * u[i] / rad[i]);
    orc_rad_dfdx(n, x_leng, FF, Flux, 0, 1.0);
    for (int i = 0; i < n; i++) Qh[i] = Qh[i] + (1.0 / (rad[i] * rad[i])) * Flux[i];
    for (int i = 0; i < n; i++) Qrhs[i] = Qrhs[i] + Qh[i];
    free(rad);
}

/* Compute_CFL src/lddrk4_nonperiodic_sf.f:7-66 (x term) and Compute_Tstep
 * :74-146 (k_hyper is never assigned by the radial Compute_hyper, so its
 * limit is +inf; 0.2 is a default-REAL literal).  Returns dt. */
double orc_rad_tstep(const st_radial_params *p, int n, double x_leng, const double *Q, const double *hyp,
                     double *cfl_stab, double *cfl_resv) {
    const double *u = Q, *rho = Q + n, *s = Q + 2 * n;
    const double *bh = hyp, *vh = hyp + n;
    const double g = p->gamma, fac = g * (g - 1.0);
    const double kmax = 2.478, khug = 2.199;
    double DX = rad_dx(n, x_leng), del = DX;
    double m1 = -INFINITY, m2 = -INFINITY;
    for (int i = 0; i < n; i++) {
        double tmp1 = 1.0 / rho[i];
        double tmp2 = sqrt(fac * tmp1 * (s[i] - 5.0e-1 * tmp1 * (u[i] * u[i] + 0.0 + 0.0)));
        double ux = fabs(u[i] * tmp1);
        double w1 = (tmp2 + ux) * kmax / DX, w2 = (tmp2 + ux) * khug / DX;
        if (w1 > m1) m1 = w1;
        if (w2 > m2) m2 = w2;
    }
    *cfl_stab = m1; *cfl_resv = m2;
    double dt = p->cfl_cal / m2;
    if (p->hyper_param == 1) {
        double m3 = INFINITY, m4 = INFINITY;
        for (int i = 0; i < n; i++) {
            double w3 = rho[i] * pow(del, 2.0) / vh[i];
            double w4 = rho[i] * pow(del, 2.0) / bh[i];
            if (w3 < m3) m3 = w3;
            if (w4 < m4) m4 = w4;
        }
        const double f02 = (double)0.2f;
        double cand[2] = {f02 * m3, f02 * m4};
        for (int q = 0; q < 2; q++) if (cand[q] < dt) dt = cand[q];
    }
    return dt;
}

/* LDDRK4 src/lddrk4_nonperiodic_sf.f:376-468 (5 + 6 stages; rk_mode as in
 * the periodic family) for one problem, state Q = (u, rho, s), hyp =
 * (beta, visc) (/HYPER/, refreshed by every Hyper_RHS). */
void orc_rad_lddrk4(const st_radial_params *p, int n, double x_leng, double *Q, double *hyp, double dt,
                    double *time, int *step) {
    double *QW = ralloc(3 * (size_t)n), *dQ = ralloc(3 * (size_t)n);
    for (int loop = 0; loop < 2; loop++) {
        memset(QW, 0, 3 * (size_t)n * 8);
        int ns = loop == 0 ? 5 : 6;
        for (int K = 0; K < ns; K++) {
            double al, be;
            if (loop == 0) { al = alpha1_rk[K]; be = beta1_rk[K]; }
            else if (p->rk_mode == 1) { al = alpha2_hhm[K]; be = beta2_hhm[K]; }
            else { al = 0.0; be = 0.0; }
            orc_rad_rhs(p, n, x_leng, Q, dQ);
            orc_rad_hyper_rhs(p, n, x_leng, Q, dQ, hyp);
            for (int q = 0; q < 3 * n; q++) QW[q] = al * QW[q] + dt * dQ[q];
            for (int q = 0; q < 3 * n; q++) Q[q] = Q[q] + be * QW[q];
            for (int f = 0; f < 3; f++) orc_rad_filter(n, Q + (size_t)f * n, Q + (size_t)f * n);
        }
        *time = *time + dt;
    }
    *step = *step + 1;
    free(QW); free(dQ);
}

/* One iteration of the main loop (src/main.f:129-136): Compute_CFL,
 * Compute_Tstep (from the /HYPER/ of the previous Hyper_RHS), LDDRK4. */
double orc_rad_step(const st_radial_params *p, int n, double x_leng, double *Q, double *hyp, double *time,
                    int *step) {
    double cs, cr;
    double dt = orc_rad_tstep(p, n, x_leng, Q, hyp, &cs, &cr);
    orc_rad_lddrk4(p, n, x_leng, Q, hyp, dt, time, step);
    return dt;
}

/* Independent problems (packed: problem k's Q block of 3 n_k doubles starts
 * at 3*off[k], its hyp block at 2*off[k]), nsteps steps each; OpenMP over
 * problems.  Compute_hyper runs first where *step == 0 (src/main.f:100). */
void orc_rad_batch(const st_radial_params *p, int nprob, const int *n, const long long *off,
                   const double *x_leng, double *Q, double *hyp, double *time, int *step, int nsteps) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 0; k < nprob; k++) {
        double *q = Q + 3 * off[k], *h = hyp + 2 * off[k];
        if (step[k] == 0) orc_rad_compute_hyper(p, n[k], x_leng[k], q, h);
        for (int it = 0; it < nsteps; it++) orc_rad_step(p, n[k], x_leng[k], q, h, &time[k], &step[k]);
    }
}
