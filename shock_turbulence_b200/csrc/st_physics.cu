// st_physics.cu - right-hand side, artificial viscosity, species, boundary
// conditions, sponge, time step and LDDRK4 stage update on device arrays.
//
// Each routine keeps the operand order of the reference expression it
// implements (the library is compiled with --fmad=false, so products and sums
// round exactly as written); explicit fma() appears only in the line solvers.
#include <cfloat>
#include <cmath>
#include "st_internal.h"

namespace st {

// ---- launch helpers ----------------------------------------------------------
// Four 256-thread CTAs per SM (at most 64 registers a thread): the two
// largest passes (the fused RHS flux passes, 80 registers uncapped) spill
// about 100 bytes but gain the occupancy; measured 10 % faster on the FP32
// mode's pointwise family and 2 % on the FP64 one.
template <class Fn>
__global__ void __launch_bounds__(256, 4) k_pfor(size_t n, Fn fn) {
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
        fn(p);
}
// site: "k_pointwise@<source line>" for the per-launch timing report
// bpe: algorithmic bytes per element (every array element the launch reads
// or writes, once; an element both read and written counts twice)
template <class Fn>
static int pfor(st_ctx *c, size_t n, const char *site, double bpe, Fn fn) {
    size_t blocks = (n + 255) / 256;    // one element per thread
    if (blocks == 0) return ST_OK;
    int pi = prof_start(c, site, bpe * (double)n);
    k_pfor<<<(unsigned)blocks, 256, 0, c->stream>>>(n, fn);
    prof_stop(c, pi);
    ST_CUDA(c, cudaGetLastError());
    return ST_OK;
}
#define ST_STR2(x) #x
#define ST_STR(x) ST_STR2(x)
#define PFOR(c, n, bpe, ...) \
    ST_TRY(pfor((c), (n), "k_pointwise@" ST_STR(__LINE__), (bpe), [=] __device__(size_t p) __VA_ARGS__))
// bytes of one element of each listed array (its element type's size), for
// the algorithmic byte count of a pointwise launch
template <class... P>
static constexpr double io(const P *...) { return (0.0 + ... + (double)sizeof(P)); }

// producer expressions evaluated by the derivative kernels while loading
template <class R>
static ProdT<R> pr_one(const R *a) { ProdT<R> p{}; p.op = PR_A; p.a = a; return p; }
template <class R>
static ProdT<R> pr_mul(const R *a, const R *b) { ProdT<R> p{}; p.op = PR_MUL; p.a = a; p.b = b; return p; }
template <class R>
static ProdT<R> pr_addmul(const R *a, const R *b, const R *c) {
    ProdT<R> p{}; p.op = PR_ADDMUL; p.a = a; p.b = b; p.c = c; return p;
}
template <class R>
static ProdT<R> pr_mulmul(const R *a, const R *b, const R *c) {
    ProdT<R> p{}; p.op = PR_MULMUL; p.a = a; p.b = b; p.c = c; return p;
}

// Line operators by field type: double arrays, or float arrays in the FP32
// mode (the kernels compute in double either way; only storage differs).
static int dfd(st_ctx *c, int dir, int asym, const double *F, double *dF, int iadd, double cadd) {
    return dev_dfd(c, dir, asym, F, dF, iadd, cadd);
}
static int dfd(st_ctx *c, int dir, int asym, const float *F, float *dF, int iadd, double cadd) {
    return dev_dfd_f(c, dir, asym, F, dF, iadd, cadd);
}
static int dfd(st_ctx *c, int dir, int asym, const Prod &F, double *dF, int iadd, double cadd) {
    return dev_dfd_prod(c, dir, asym, F, dF, iadd, cadd);
}
static int dfd(st_ctx *c, int dir, int asym, const ProdF &F, float *dF, int iadd, double cadd) {
    return dev_dfd_prod_f(c, dir, asym, F, dF, iadd, cadd);
}
static int d2fd2(st_ctx *c, int dir, int asym, const double *F, double *dF, double *d2F, int iadd) {
    return dev_d2fd2(c, dir, asym, F, dF, d2F, iadd);
}
static int d2fd2(st_ctx *c, int dir, int asym, const float *F, float *dF, float *d2F, int iadd) {
    return dev_d2fd2_f(c, dir, asym, F, dF, d2F, iadd);
}
static int dfd_sum(st_ctx *c, int dir, int asym, const double *F, double *dF, const double *E1,
                   const double *E2) {
    return dev_dfd_sum(c, dir, asym, F, dF, E1, E2);
}
static int dfd_sum(st_ctx *c, int dir, int asym, const float *F, float *dF, const float *E1, const float *E2) {
    return dev_dfd_sum_f(c, dir, asym, F, dF, E1, E2);
}
static int d2fd2_sum(st_ctx *c, int dir, int asym, const double *F, double *d2F, const double *E1,
                     const double *E2) {
    return dev_d2fd2_sum(c, dir, asym, F, d2F, E1, E2);
}
static int d2fd2_sum(st_ctx *c, int dir, int asym, const float *F, float *d2F, const float *E1,
                     const float *E2) {
    return dev_d2fd2_sum_f(c, dir, asym, F, d2F, E1, E2);
}
// two first derivatives of one direction in order (producer, output, asym,
// iadd[, cadd] of each; cadd 1 where not given), one launch where they share
// fields
template <class R>
static int dfd_pair(st_ctx *c, int dir, ProdT<R> F0, R *O0, int asym0, int iadd0, double cadd0, ProdT<R> F1, R *O1,
                    int asym1, int iadd1, double cadd1) {
    const D1SpecT<R> ops[2] = {{F0, O0, asym0, iadd0, cadd0}, {F1, O1, asym1, iadd1, cadd1}};
    if constexpr (sizeof(R) == 8) return dev_dfd_pair(c, dir, ops);
    else return dev_dfd_pair_f(c, dir, ops);
}
template <class R>
static int dfd_pair(st_ctx *c, int dir, ProdT<R> F0, R *O0, int asym0, int iadd0, ProdT<R> F1, R *O1, int asym1,
                    int iadd1) {
    return dfd_pair<R>(c, dir, F0, O0, asym0, iadd0, 1.0, F1, O1, asym1, iadd1, 1.0);
}
static int gauss(st_ctx *c, int dir, const double *F, double *Fg) { return dev_gauss(c, dir, F, Fg); }
static int gauss(st_ctx *c, int dir, const float *F, float *Fg) { return dev_gauss_f(c, dir, F, Fg); }

// COMMON arrays of the intermediate type R
template <class R> struct Store;
template <> struct Store<double> {
    static double **grad(st_ctx *c) { return c->grad; }
    static double **hyp(st_ctx *c) { return c->hyp; }
    static double **dYd(st_ctx *c) { return c->dYd; }
    static double *dQ(st_ctx *c) { return c->dQ; }
    static double *drYi(st_ctx *c) { return c->drYi; }
};
template <> struct Store<float> {
    static float **grad(st_ctx *c) { return c->gradf; }
    static float **hyp(st_ctx *c) { return c->hypf; }
    static float **dYd(st_ctx *c) { return c->dYdf; }
    static float *dQ(st_ctx *c) { return c->dQf; }
    static float *drYi(st_ctx *c) { return c->drYif; }
};
template <class R> constexpr bool is_fp64() { return sizeof(R) == sizeof(double); }

struct Phys {
    double g1, g2, eps, vis_exp, Re1_inv, Re2_inv, Pr_inv, Sc_inv, bulk;
};
static Phys phys(const st_ctx *c) {
    Phys f;
    f.g1 = c->p.gamma1; f.g2 = c->p.gamma2; f.eps = c->p.epsilon; f.vis_exp = c->p.vis_exp;
    f.Re1_inv = c->Re1_inv; f.Re2_inv = c->Re2_inv; f.Pr_inv = c->Pr_inv; f.Sc_inv = c->Sc_inv;
    f.bulk = c->p.bulk_ratio;
    return f;
}

// P and T block (e.g. src/rhsv_sym_mf.f:99-115)
__device__ __forceinline__ void thermo(const Phys &f, double g, double Y, double q1, double q2, double q3,
                                       double q4, double q5, double &Vs, double &P, double &T) {
    double fac1 = g - 1.0;
    double fac3 = f.g1 / (f.g1 - 1.0);
    fac3 = fac3 * 1.0 / (Y + f.eps * (1.0 - Y));
    Vs = 1.0 / q4;
    P = fac1 * (q5 - 5.0e-1 * Vs * (q1 * q1 + q2 * q2 + q3 * q3));
    T = fac3 * Vs * P;
}
// viscosity law, src/rhsv_sym_mf.f:253-263
__device__ __forceinline__ void viscosity(const Phys &f, double T, double Y, double &mu, double &dmu) {
    double fac1 = f.g1 - 1.0;
    double fac2 = f.vis_exp - 1.0;
    double se = sqrt(f.eps);
    double num = f.Re1_inv * Y + f.Re2_inv * se * (1.0 - Y);
    double den = Y + se * (1.0 - Y);
    mu = pow(fac1 * T, f.vis_exp) * num / den;
    dmu = pow(fac1 * T, fac2) * num / den * f.vis_exp * fac1;
}

// n separate scratch fields
template <class R>
struct ScratchNT {
    st_ctx *c; std::vector<R *> f;
    ScratchNT(st_ctx *cc, int n) : c(cc) { for (int i = 0; i < n; i++) f.push_back(scratch_t<R>(cc, 1)); }
    ~ScratchNT() { for (R *p : f) release(c, p); }
    R *operator[](int i) const { return f[i]; }
};

int dev_fill(st_ctx *c, double *x, size_t n, double v) {
    PFOR(c, n, io(x), { x[p] = v; });
    return ST_OK;
}
int dev_to_float(st_ctx *c, const double *x, float *y, size_t n) {
    PFOR(c, n, io(x, y), { y[p] = (float)x[p]; });
    return ST_OK;
}
int dev_to_double(st_ctx *c, const float *x, double *y, size_t n) {
    PFOR(c, n, io(x, y), { y[p] = (double)x[p]; });
    return ST_OK;
}

int dev_compute_gamma(st_ctx *c, const double *Y) {
    Phys f = phys(c);
    double *ge = c->gamma_eff;
    PFOR(c, c->ncell(), io(Y, ge), {
        double fac1 = f.g1 - 1.0, fac2 = f.g2 - 1.0;
        double num = (Y[p] * f.g1 / fac1) + (f.eps * (1.0 - Y[p]) * f.g2 / fac2);
        double den = (Y[p] / fac1) + (f.eps * (1.0 - Y[p]) / fac2);
        ge[p] = num / den;
    });
    return ST_OK;
}

// ---- RHS (src/rhsv_sym_mf.f:9-1428) ------------------------------------------
// The reference runs RHS_x on a copy Ux of Q and hands Ux to RHS_yz holding
// du/dx, dv/dx, dw/dx, dT/dx and mu.  Here those quantities live in the
// /GRAD/ arrays and in named scratch fields, with these exact rewrites:
//  - accumulators (Qrhs, Qconvx/y/z, Qvisc) are assigned by their first
//    contribution instead of being zeroed first (0 + x == x);
//  - the /GRAD/ copies are written in place by the derivative kernels;
//  - quantities RHS_yz recomputes with the same expression from the same
//    inputs (Vs, P, T, u, v, w, mu, dmu/dT) are computed once;
//  - d(rho)/dy (src/rhsv_sym_mf.f:953), which the reference overwrites before
//    any use, is not computed;
//  - when the molecular viscous term is not added (Re <= 0, the reference
//    build, src/rhsv_sym_mf.f:1420-1424) the Qvisc work, whose only consumer
//    is that sum, is skipped; the /GRAD/ first derivatives are still formed.
//
// R is the storage type of every field except the state: double, or float in
// the FP32 mode.  Qr is the state in that type (Q itself in FP64); the
// derivative operands come from Qr, the pointwise thermodynamics from Q.
template <class R>
static int rhs_t(st_ctx *c, double *Q, const R *Qr, R *Qrhs, const double *Y) {
    const size_t n3 = c->fs, nc = c->ncell();   // field stride; cells processed
    const Phys f = phys(c);
    // src/rhsv_periodic_sf.f:1381 adds Qvisc unconditionally
    const bool visc = c->p.re > 0.0 || c->p.family == ST_FAMILY_PERIODIC;
    double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    const R *q1r = Qr, *q2r = Qr + n3, *q3r = Qr + 2 * n3, *q4r = Qr + 3 * n3, *q5r = Qr + 4 * n3;
    R **G = Store<R>::grad(c);
    R *Gxx = G[G_DUX_DX], *Gyx = G[G_DUY_DX], *Gzx = G[G_DUZ_DX];
    R *Gxy = G[G_DUX_DY], *Gyy = G[G_DUY_DY], *Gzy = G[G_DUZ_DY];
    R *Gxz = G[G_DUX_DZ], *Gyz = G[G_DUY_DZ], *Gzz = G[G_DUZ_DZ];
    R *GTx = G[G_DTDX], *GTy = G[G_DTDY], *GTz = G[G_DTDZ];
    ScratchT<R> sQcx(c, 5), sQcy(c, 5), sQcz(c, 5), sQv(c, 5);
    R *Qcx = sQcx, *Qcy = sQcy, *Qcz = sQcz, *Qv = sQv;   // Qv(:,:,:,4) is never formed
    ScratchNT<R> s(c, 8);
    R *P = s[0], *T = s[1], *u = s[2], *v = s[3], *w = s[4], *mu = s[5], *dmu = s[6], *FF = s[7];
    // second derivatives and derivatives of /GRAD/ consumed by the two
    // pointwise passes below (one field each, so that all of them can be
    // formed before the pass that uses them)
    ScratchNT<R> dd(c, 14);
    const double *g = c->gamma_eff;

    // ---- RHS_x (src/rhsv_sym_mf.f:37-481)
    // P, T, u, and (the same expressions the reference evaluates later from
    // the same inputs) v, w, mu, dmu/dT
    PFOR(c, nc, io(g, Y, Q1, Q2, Q3, Q4, Q5, P, T, u, v, w, mu, dmu), {
        double vs, pp, tt, m, dm;
        thermo(f, g[p], Y[p], Q1[p], Q2[p], Q3[p], Q4[p], Q5[p], vs, pp, tt);
        P[p] = pp; T[p] = tt;
        u[p] = Q1[p] * vs;
        v[p] = Q2[p] * vs;
        w[p] = Q3[p] * vs;
        viscosity(f, (R)tt, Y[p], m, dm);
        mu[p] = m;
        dmu[p] = dm;
    });
    // adjacent fluxes sharing u (or the second adding dP/dx to what the first
    // wrote) run as pairs, in the reference's order
    const R *cu = u, *cv = v, *cw = w, *cP = P;
    ST_TRY(dfd_pair<R>(c, 0, pr_mul(q4r, cu), Qcx + 3 * n3, 1, 0, -1.0, pr_addmul(q5r, cP, cu), Qcx + 4 * n3, 1, 0,
                       -1.0));
    ST_TRY(dfd_pair<R>(c, 0, pr_mul(q1r, cu), Qcx, 0, 0, -5.0e-1, pr_one(cP), Qcx, 0, 1, -1.0));
    ST_TRY(dfd_pair<R>(c, 0, pr_mul(q2r, cu), Qcx + n3, 1, 0, -5.0e-1, pr_mul(q3r, cu), Qcx + 2 * n3, 1, 0,
                       -5.0e-1));
    ST_TRY(dfd(c, 0, 1, q1r, FF, 0, 1.0));
    R *dTx = dd[0], *duxx = dd[1], *dvxx = dd[2], *dwxx = dd[3];
    if (visc) {
        ST_TRY(d2fd2(c, 0, 0, (const R *)T, GTx, dTx, 1));
        ST_TRY(d2fd2(c, 0, 1, (const R *)u, Gxx, duxx, 1));
        ST_TRY(d2fd2(c, 0, 0, (const R *)v, Gyx, dvxx, 1));
        ST_TRY(d2fd2(c, 0, 0, (const R *)w, Gzx, dwxx, 1));
    } else {
        ST_TRY(dfd(c, 0, 0, (const R *)T, GTx, 0, 1.0));
        ST_TRY(dfd(c, 0, 1, (const R *)u, Gxx, 0, 1.0));
        ST_TRY(dfd(c, 0, 0, (const R *)v, Gyx, 0, 1.0));
        ST_TRY(dfd(c, 0, 0, (const R *)w, Gzx, 0, 1.0));
    }
    // convective terms -0.5*d(rho u)/dx*(u,v,w) and -0.5*rho*u*d(u,v,w)/dx,
    // and the x part of Qvisc, in the reference's order of accumulation
    {
        const double Pri = f.Pr_inv, fac1 = 4.0 / 3.0 + f.bulk;
        PFOR(c, nc, io(FF, u, v, w, Q4, Gxx, Gyx, Gzx) + 6 * io(Qcx) + (visc ? io(mu, dTx, dmu, GTx, duxx, dvxx, dwxx) + 4 * io(Qv) : 0.0), {
            double fac2 = -5.0e-1 * FF[p];
            double c1 = Qcx[p] + fac2 * u[p];
            double c2 = Qcx[n3 + p] + fac2 * v[p];
            double c3 = Qcx[2 * n3 + p] + fac2 * w[p];
            if (visc) {
                double q5 = Pri * (mu[p] * dTx[p] + dmu[p] * GTx[p] * GTx[p]);
                double fx = fac1 * mu[p] * duxx[p];
                q5 = q5 + u[p] * fx;
                double fy = mu[p] * dvxx[p];
                q5 = q5 + v[p] * fy;
                double fz = mu[p] * dwxx[p];
                q5 = q5 + w[p] * fz;
                Qv[p] = fx;
                Qv[n3 + p] = fy;
                Qv[2 * n3 + p] = fz;
                Qv[4 * n3 + p] = q5;
            }
            fac2 = -5.0e-1 * Q4[p] * u[p];
            Qcx[p] = c1 + fac2 * Gxx[p];
            Qcx[n3 + p] = c2 + fac2 * Gyx[p];
            Qcx[2 * n3 + p] = c3 + fac2 * Gzx[p];
        });
    }

    // ---- RHS_yz (src/rhsv_sym_mf.f:492-1428)
    // d(rho v)/dy and d(rho w)/dz with iadd=0, cadd=-1: Qconv(4) = 0 - d(.) exactly
    ST_TRY(dfd(c, 1, 1, q2r, Qcy + 3 * n3, 0, -1.0));
    ST_TRY(dfd(c, 1, 1, pr_mul(q1r, v), Qcy, 0, -5.0e-1));
    ST_TRY(dfd_pair<R>(c, 1, pr_mul(q2r, cv), Qcy + n3, 0, 0, -5.0e-1, pr_one(cP), Qcy + n3, 0, 1, -1.0));
    ST_TRY(dfd_pair<R>(c, 1, pr_mul(q3r, cv), Qcy + 2 * n3, 1, 0, -5.0e-1, pr_addmul(q5r, cP, cv), Qcy + 4 * n3, 1,
                       0, -1.0));
    ST_TRY(dfd(c, 2, 1, q3r, Qcz + 3 * n3, 0, -1.0));
    ST_TRY(dfd_pair<R>(c, 2, pr_mul(q1r, cw), Qcz, 1, 0, -5.0e-1, pr_mul(q2r, cw), Qcz + n3, 1, 0, -5.0e-1));
    ST_TRY(dfd_pair<R>(c, 2, pr_mul(q3r, cw), Qcz + 2 * n3, 0, 0, -5.0e-1, pr_one(cP), Qcz + 2 * n3, 0, 1, -1.0));
    ST_TRY(dfd(c, 2, 1, pr_addmul(q5r, P, w), Qcz + 4 * n3, 0, -1.0));
    R *d2Ty = dd[0], *d2Tz = dd[1], *d2uy = dd[2], *d2vy = dd[3], *d2wy = dd[4], *d2wz = dd[5];
    R *dGzz_y = dd[6], *d2uz = dd[7], *d2vz = dd[8], *dGxx_y = dd[9], *dGxx_z = dd[10], *dGyx_y = dd[11];
    R *dGzx_z = dd[12], *dGyz_y = dd[13];
    if (visc) {
        ST_TRY(d2fd2(c, 1, 0, (const R *)T, GTy, d2Ty, 1));
        ST_TRY(d2fd2(c, 2, 0, (const R *)T, GTz, d2Tz, 1));
        ST_TRY(d2fd2(c, 1, 0, (const R *)u, Gxy, d2uy, 1));
        ST_TRY(d2fd2(c, 1, 1, (const R *)v, Gyy, d2vy, 1));
        ST_TRY(d2fd2(c, 1, 0, (const R *)w, Gzy, d2wy, 1));
    } else {
        ST_TRY(dfd(c, 1, 0, (const R *)T, GTy, 0, 1.0));
        ST_TRY(dfd(c, 2, 0, (const R *)T, GTz, 0, 1.0));
        ST_TRY(dfd(c, 1, 0, (const R *)u, Gxy, 0, 1.0));
        ST_TRY(dfd(c, 1, 1, (const R *)v, Gyy, 0, 1.0));
        ST_TRY(dfd(c, 1, 0, (const R *)w, Gzy, 0, 1.0));
    }
    ST_TRY(dfd(c, 2, 0, (const R *)u, Gxz, 0, 1.0));
    ST_TRY(dfd(c, 2, 0, (const R *)v, Gyz, 0, 1.0));
    ST_TRY(dfd(c, 2, 1, (const R *)w, Gzz, 0, 1.0));
    if (visc) {
        ST_TRY(d2fd2(c, 2, 1, (const R *)w, (R *)nullptr, d2wz, 0));
        ST_TRY(dfd(c, 1, 0, (const R *)Gzz, dGzz_y, 0, 1.0));
        ST_TRY(d2fd2(c, 2, 0, (const R *)u, (R *)nullptr, d2uz, 0));
        ST_TRY(d2fd2(c, 2, 0, (const R *)v, (R *)nullptr, d2vz, 0));
        ST_TRY(dfd(c, 1, 0, (const R *)Gxx, dGxx_y, 0, 1.0));
        ST_TRY(dfd(c, 2, 0, (const R *)Gxx, dGxx_z, 0, 1.0));
        ST_TRY(dfd(c, 1, 1, (const R *)Gyx, dGyx_y, 0, 1.0));
        ST_TRY(dfd(c, 2, 1, (const R *)Gzx, dGzx_z, 0, 1.0));
        ST_TRY(dfd(c, 1, 1, (const R *)Gyz, dGyz_y, 0, 1.0));
    }
    // One pass for the rest of RHS_yz and the sum Qrhs = Qconvx + Qconvy +
    // Qconvz + Qvisc: each accumulator receives its terms in the order the
    // reference adds them (src/rhsv_sym_mf.f:992-1424), in registers.
    {
        const double Pri = f.Pr_inv;
        const double fb43 = f.bulk + 4.0 / 3.0, fb23 = f.bulk - 2.0 / 3.0, fb13 = f.bulk + 1.0 / 3.0;
        const bool fp64 = is_fp64<R>();
        PFOR(c, nc, io(u, v, w, Q4, Gxx, Gyx, Gzx, Gxy, Gyy, Gzy, Gxz, Gyz, Gzz) + 5 * io(Qcx, Qcy, Qcz, Qrhs) + (fp64 ? io(Q1, Q2, Q3) : 0.0) + (visc ? io(mu, dmu, d2Ty, d2Tz, GTy, GTz, GTx, d2uy, d2vy, d2wy, dGzz_y, d2wz, d2uz, d2vz, dGyx_y, dGzx_z, dGxx_y, dGxx_z, dGyz_y) + 4 * io(Qv) : 0.0), {
            const double uu = u[p], vv = v[p], ww = w[p], q4 = Q4[p];
            // -0.5*d(rho v)/dy = 0.5*Qconvy(4) exactly (cadd flips only the sign)
            double fac2 = -5.0e-1 * (-(double)Qcy[3 * n3 + p]);
            double cy1 = Qcy[p] + fac2 * uu, cy2 = Qcy[n3 + p] + fac2 * vv, cy3 = Qcy[2 * n3 + p] + fac2 * ww;
            fac2 = -5.0e-1 * (-(double)Qcz[3 * n3 + p]);
            double cz1 = Qcz[p] + fac2 * uu, cz2 = Qcz[n3 + p] + fac2 * vv, cz3 = Qcz[2 * n3 + p] + fac2 * ww;
            double v1 = 0.0, v2 = 0.0, v3 = 0.0, v5 = 0.0, U4 = 0.0, Tdy = 0.0, Tdz = 0.0, m = 0.0;
            if (visc) {
                m = mu[p];
                const double dm = dmu[p];
                v5 = Qv[4 * n3 + p] + Pri * (m * (d2Ty[p] + d2Tz[p]) +
                                             dm * (GTy[p] * GTy[p] + GTz[p] * GTz[p]));
                U4 = dm * GTx[p];
                Tdy = dm * GTy[p];
                Tdz = dm * GTz[p];
            }
            const double gxx = Gxx[p], gyx = Gyx[p], gzx = Gzx[p], gxy = Gxy[p], gyy = Gyy[p], gzy = Gzy[p];
            const double gxz = Gxz[p], gyz = Gyz[p], gzz = Gzz[p];
            fac2 = -5.0e-1 * q4 * vv;
            cy1 = cy1 + fac2 * gxy;
            cy2 = cy2 + fac2 * gyy;
            cy3 = cy3 + fac2 * gzy;
            fac2 = -5.0e-1 * q4 * ww;
            cz1 = cz1 + fac2 * gxz;
            cz2 = cz2 + fac2 * gyz;
            cz3 = cz3 + fac2 * gzz;
            if (visc) {
                // mu * d2(u,v,w)/dy2 terms
                double fX = m * d2uy[p];
                double fY = fb43 * m * d2vy[p];
                double fZ = m * d2wy[p];
                v1 = Qv[p] + fX;
                v2 = Qv[n3 + p] + fY;
                v3 = Qv[2 * n3 + p] + fZ;
                v5 = v5 + uu * fX + vv * fY + ww * fZ;
                // dilatation terms
                double tmp1 = gxx;
                double dil = tmp1 + gyy + gzz;
                fX = U4 * (2.0 * tmp1 + fb23 * dil);
                fY = Tdy * (2.0 * gyy + fb23 * dil) + fb13 * m * dGzz_y[p];
                fZ = Tdz * (2.0 * gzz + fb23 * dil) + fb43 * m * d2wz[p];
                v1 = v1 + fX;
                v2 = v2 + fY;
                v3 = v3 + fZ;
                v5 = v5 + uu * fX + vv * fY + ww * fZ +
                     m * (2.0 * (tmp1 * tmp1 + gyy * gyy + gzz * gzz) + fb23 * dil * dil);
                // shear terms
                double t1 = gyx + gxy, t2 = gzx + gxz, t3 = gzy + gyz;
                fX = Tdy * t1 + Tdz * t2 + m * d2uz[p];
                fY = U4 * t1 + Tdz * t3 + m * d2vz[p];
                fZ = U4 * t2 + Tdy * t3;
                v1 = v1 + fX;
                v2 = v2 + fY;
                v3 = v3 + fZ;
                v5 = v5 + uu * fX + vv * fY + ww * fZ + m * (t1 * t1 + t2 * t2 + t3 * t3);
                // cross derivatives of the velocity gradient
                fX = fb13 * m * (dGyx_y[p] + dGzx_z[p]);
                fY = fb13 * m * dGxx_y[p];
                fZ = fb13 * m * (dGxx_z[p] + dGyz_y[p]);
                v1 = v1 + fX;
                v2 = v2 + fY;
                v3 = v3 + fZ;
                v5 = v5 + uu * fX + vv * fY + ww * fZ;
            }
            // velocities back to momenta, (m/rho)*rho as the reference does;
            // the FP32 mode keeps the double momenta instead of rounding them
            // through the float velocities
            if (fp64) {
                Q1[p] = uu * q4;
                Q2[p] = vv * q4;
                Q3[p] = ww * q4;
            }
            const double cy[5] = {cy1, cy2, cy3, Qcy[3 * n3 + p], Qcy[4 * n3 + p]};
            const double cz[5] = {cz1, cz2, cz3, Qcz[3 * n3 + p], Qcz[4 * n3 + p]};
            const double vq[5] = {v1, v2, v3, 0.0, v5};
            for (int l = 0; l < 5; l++) {
                size_t q = l * n3 + p;
                double r = Qcx[q] + cy[l] + cz[l];
                if (visc && l != 3) r = r + vq[l];   // Qvisc(:,:,:,4) stays zero
                Qrhs[q] = r;
            }
        });
    }
    return ST_OK;
}

// Gaussian_Filter src/filters_sym.f:1046-1071
template <class R>
static int gaussian_filter_t(st_ctx *c, const R *F, R *Fg, int nvar) {
    const size_t n3 = c->fs, nc = c->ncell();   // field stride; cells processed
    ScratchT<R> tmp(c);
    R *t = tmp;
    for (int l = 0; l < nvar; l++) {
        ST_TRY(gauss(c, 0, F + l * n3, Fg + l * n3));
        ST_TRY(gauss(c, 1, Fg + l * n3, t));
        ST_TRY(gauss(c, 2, t, Fg + l * n3));
    }
    return ST_OK;
}

// ---- artificial viscosity -----------------------------------------------------
// Compute_Laplacian src/hyper_dynamic_sym_mf.f:41-65
template <class R>
static int laplacian(st_ctx *c, const R *S, R *d2S) {
    ScratchT<R> dS(c), t1(c), t2(c);
    R *pt1 = t1, *pt2 = t2;
    if (c->p.family == ST_FAMILY_PERIODIC) {
        // Compute_Laplacian src/hyper_dynamic.f:41-58 (second derivatives)
        ST_TRY(d2fd2(c, 0, 0, S, (R *)nullptr, (R *)t1, 0));
        ST_TRY(d2fd2(c, 1, 0, S, (R *)nullptr, (R *)t2, 0));
        // d2S = d2S + t1 + t2 in the z pass's store
        return d2fd2_sum(c, 2, 0, S, d2S, (const R *)pt1, (const R *)pt2);
    }
    ST_TRY(dfd(c, 0, 0, S, (R *)dS, 0, 1.0));
    ST_TRY(dfd(c, 0, 1, (const R *)dS, (R *)t1, 0, 1.0));
    ST_TRY(dfd(c, 1, 0, S, (R *)dS, 0, 1.0));
    ST_TRY(dfd(c, 1, 1, (const R *)dS, (R *)t2, 0, 1.0));
    ST_TRY(dfd(c, 2, 0, S, (R *)dS, 0, 1.0));
    // d2S = d2S + temp1 + temp2 (src/hyper_dynamic_sym_mf.f:61) in the z pass's store
    return dfd_sum(c, 2, 1, (const R *)dS, d2S, (const R *)pt1, (const R *)pt2);
}

// Compute_hyper src/hyper_dynamic_sym_mf.f:166-334 (+ Compute_coeff1 :79-158,
// Compute_Contraction :12-33)
// Compute_hyper of the periodic single-fluid family, src/hyper_dynamic.f:
// Compute_coeff1 :72-165 forms vorticity and dilatation from periodic first
// derivatives of u (the dilatation sums Grad4 + temp are the iadd
// accumulations of the derivative kernels), Compute_hyper :173-321 filters
// eta = (rho|d4S|, fac3|d4e|, rho|d4S|) and applies the coefficients after the
// filter.  The third field equals the first, so its filtered value is the
// first one's (same input, same arithmetic) and is filtered once.
template <class R>
static int compute_hyper_sf(st_ctx *c, const double *Q) {
    const size_t n3 = c->fs, nc = c->ncell();   // field stride; cells processed
    const double gam = c->p.gamma1;
    const double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    ScratchNT<R> s(c, 14);
    R *U1 = s[0], *U2 = s[1], *U3 = s[2], *W1 = s[3], *W2 = s[4], *W3 = s[5], *Dl = s[6];
    R *Cbeta = s[7], *S = s[8], *e = s[9], *T = s[10], *d2 = s[11], *d4S = s[12], *d4e = s[13];
    PFOR(c, nc, io(Q1, Q2, Q3, Q4, U1, U2, U3), {
        double t = 1.0 / Q4[p];
        U1[p] = Q1[p] * t; U2[p] = Q2[p] * t; U3[p] = Q3[p] * t;
    });
    ST_TRY(dfd(c, 1, 0, U3, W1, 0, 1.0));
    ST_TRY(dfd(c, 2, 0, U2, W1, 1, -1.0));
    ST_TRY(dfd(c, 0, 0, U3, W2, 0, -1.0));
    ST_TRY(dfd(c, 2, 0, U1, W2, 1, 1.0));
    ST_TRY(dfd(c, 0, 0, U2, W3, 0, 1.0));
    ST_TRY(dfd(c, 1, 0, U1, W3, 1, -1.0));
    ST_TRY(dfd(c, 0, 0, U1, Dl, 0, 1.0));
    ST_TRY(dfd(c, 1, 0, U2, Dl, 1, 1.0));
    ST_TRY(dfd(c, 2, 0, U3, Dl, 1, 1.0));
    R *const *Gr = Store<R>::grad(c);
    const R *G0 = Gr[0], *G1 = Gr[1], *G2 = Gr[2], *G3 = Gr[3], *G4 = Gr[4], *G5 = Gr[5], *G6 = Gr[6],
            *G7 = Gr[7], *G8 = Gr[8];
    const double scale = c->p.c_beta_scale;
    R *P = U1, *Vs = U2;   // the velocities are dead from here on
    PFOR(c, nc, io(Dl, W1, W2, W3, G0, G1, G2, G3, G4, G5, G6, G7, G8, Q1, Q2, Q3, Q4, Q5, Cbeta, Vs, P, T, e, S), {
        double eps = 1.0e-7, fac2 = 10.0;
        double dil = Dl[p];
        double fac = 5.0e-1 * (1.0 - tanh(2.5 + fac2 * dil));
        double om2 = W1[p] * W1[p] + W2[p] * W2[p] + W3[p] * W3[p];
        Cbeta[p] = (fac * dil * dil / (dil * dil + om2 + eps) + 1.0e-20) * scale;
        double s1 = G0[p], s5 = G4[p], s9 = G8[p];
        double s2 = 5.0e-1 * (G3[p] + G1[p]);
        double s3 = 5.0e-1 * (G6[p] + G2[p]);
        double s6 = 5.0e-1 * (G7[p] + G5[p]);
        double s4 = s2, s7 = s3, s8 = s6;
        double fac1 = gam - 1.0, fac2t = gam / fac1;
        double vs = 1.0 / Q4[p];
        double pp = fac1 * (Q5[p] - 5.0e-1 * vs * (Q1[p] * Q1[p] + Q2[p] * Q2[p] + Q3[p] * Q3[p]));
        Vs[p] = vs;
        P[p] = pp;
        T[p] = fac2t * vs * pp;
        e[p] = vs * (Q5[p] - 5.0e-1 * vs * (Q1[p] * Q1[p] + Q2[p] * Q2[p] + Q3[p] * Q3[p]));
        S[p] = sqrt(5.0e-1 * (s1 * s1 + s5 * s5 + s9 * s9 + 2.0 * (s2 * s4 + s3 * s7 + s6 * s8)));
    });
    ST_TRY(laplacian(c, S, d2));
    ST_TRY(laplacian(c, d2, d4S));
    ST_TRY(laplacian(c, e, d2));
    ST_TRY(laplacian(c, d2, d4e));
    ScratchT<R> etas(c, 4);
    R *eta = etas, *etag = eta + 2 * n3;   // [rho|d4S|, fac3|d4e|] and their filtered values
    PFOR(c, nc, io(Q4, T, P, Vs, d4S, d4e) + 2 * io(eta), {
        double fac3 = (Q4[p] / T[p]) * sqrt(gam * P[p] * Vs[p]);
        eta[p] = Q4[p] * fabs(d4S[p]);
        eta[n3 + p] = fac3 * fabs(d4e[p]);
    });
    ST_TRY(gaussian_filter_t<R>(c, eta, etag, 2));
    const double DX6 = pow(c->DX, 6.0), DX5 = pow(c->DX, 5.0);
    const double C_mu = 2.0e-3, C_k = 1.0e-2;
    R **H = Store<R>::hyp(c);
    R *hb = H[H_BETA], *hv = H[H_VISC], *hk = H[H_K];
    PFOR(c, nc, io(Cbeta, hb, hv, hk) + 2 * io(etag), {
        hb[p] = Cbeta[p] * etag[p] * DX6;
        hv[p] = C_mu * etag[p] * DX6;
        hk[p] = C_k * etag[n3 + p] * DX5;
    });
    return ST_OK;
}

// Yr: the mass fraction in the type R (Y itself in FP64)
template <class R>
static int compute_hyper_t(st_ctx *c, const double *Q, const double *Y, const R *Yr) {
    if (c->p.family == ST_FAMILY_PERIODIC) return compute_hyper_sf<R>(c, Q);
    const size_t n3 = c->fs, nc = c->ncell();   // field stride; cells processed
    Phys f = phys(c);
    const double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    ScratchNT<R> s(c, 10);
    R *Cbeta = s[0], *S = s[1], *e = s[2], *P = s[3], *T = s[4], *Vs = s[5], *d2 = s[6];
    R *d4S = s[7], *d4e = s[8], *d4Y = s[9];
    ScratchT<R> etas(c, 10);
    R *eta = etas, *etag = eta + 5 * n3;
    const double *g = c->gamma_eff;
    R *const *Gr = Store<R>::grad(c);
    const R *G0 = Gr[0], *G1 = Gr[1], *G2 = Gr[2], *G3 = Gr[3], *G4 = Gr[4], *G5 = Gr[5], *G6 = Gr[6],
            *G7 = Gr[7], *G8 = Gr[8];
    const double scale = c->p.c_beta_scale;
    {
        PFOR(c, nc, io(G0, G1, G2, G3, G4, G5, G6, G7, G8, g, Y, Q1, Q2, Q3, Q4, Q5, Cbeta, Vs, P, T, e, S), {
            // G0..G8 = dux_dx, duy_dx, duz_dx, dux_dy, duy_dy, duz_dy, dux_dz, duy_dz, duz_dz
            double w1 = G5[p] - G7[p];
            double w2 = G6[p] - G2[p];
            double w3 = G1[p] - G3[p];
            double dil = G0[p] + G4[p] + G8[p];
            double eps = 1.0e-7, fac2 = 0.2;
            double fac = 5.0e-1 * (1.0 - tanh(2.5 + fac2 * dil));
            double om2 = w1 * w1 + w2 * w2 + w3 * w3;
            Cbeta[p] = (fac * dil * dil / (dil * dil + om2 + eps)) * scale;
            double s1 = G0[p], s5 = G4[p], s9 = G8[p];
            double s2 = 5.0e-1 * (G3[p] + G1[p]);
            double s3 = 5.0e-1 * (G6[p] + G2[p]);
            double s6 = 5.0e-1 * (G7[p] + G5[p]);
            double s4 = s2, s7 = s3, s8 = s6;
            double fac1 = g[p] - 1.0;
            double fac3 = f.g1 / (f.g1 - 1.0);
            fac3 = fac3 * 1.0 / (Y[p] + f.eps * (1.0 - Y[p]));
            double vs = 1.0 / Q4[p];
            double pp = fac1 * (Q5[p] - 5.0e-1 * vs * (Q1[p] * Q1[p] + Q2[p] * Q2[p] + Q3[p] * Q3[p]));
            Vs[p] = vs;
            P[p] = pp;
            T[p] = fac3 * vs * pp;
            e[p] = vs * (Q5[p] - 5.0e-1 * vs * (Q1[p] * Q1[p] + Q2[p] * Q2[p] + Q3[p] * Q3[p]));
            S[p] = sqrt(5.0e-1 * (s1 * s1 + s5 * s5 + s9 * s9 + 2.0 * (s2 * s4 + s3 * s7 + s6 * s8)));
        });
        ST_TRY(laplacian(c, S, d2));
        ST_TRY(laplacian(c, d2, d4S));
        ST_TRY(laplacian(c, e, d2));
        ST_TRY(laplacian(c, d2, d4e));
        ST_TRY(laplacian(c, Yr, d2));
        ST_TRY(laplacian(c, d2, d4Y));
        const double C_mu = 2.0e-3, C_k = 1.0e-2;
        PFOR(c, nc, io(d4S, d4e, d4Y, g, P, Vs, Q4, T, Cbeta, Y) + 5 * io(eta), {
            double a4S = fabs(d4S[p]), a4e = fabs(d4e[p]), a4Y = fabs(d4Y[p]);
            double cs = sqrt(g[p] * P[p] * Vs[p]);
            double fac3 = (Q4[p] / T[p]) * sqrt(g[p] * P[p] * Vs[p]);
            eta[p] = C_mu * Q4[p] * a4S;
            eta[2 * n3 + p] = Cbeta[p] * Q4[p] * a4S;
            eta[n3 + p] = C_k * fac3 * a4e;
            eta[4 * n3 + p] = cs * a4Y;
            double tmp1 = (Y[p] < 1.0) ? 0.0 : 1.0;
            double tmp2 = (Y[p] < 0.0) ? 0.0 : 1.0;
            eta[3 * n3 + p] = cs * ((Y[p] - 1.0) * tmp1 - Y[p] * (1.0 - tmp2));
        });
        ST_TRY(gaussian_filter_t<R>(c, eta, etag, 5));
        const double DX6 = pow(c->DX, 6.0), DX5 = pow(c->DX, 5.0), DX = c->DX;
        const double C_D = 1.0e-4, C_Y = 100.0;
        R **H = Store<R>::hyp(c);
        R *hb = H[H_BETA], *hv = H[H_VISC], *hk = H[H_K], *hd = H[H_D];
        PFOR(c, nc, 5 * io(etag) + io(hb, hv, hk, hd), {
            hb[p] = etag[2 * n3 + p] * DX6;
            hv[p] = etag[p] * DX6;
            hk[p] = etag[n3 + p] * DX5;
            hd[p] = C_D * etag[4 * n3 + p] * DX5 + C_Y * etag[3 * n3 + p] * DX;
        });
    }
    return ST_OK;
}

// Hyper_RHS src/hyper_rhs_sym_mf.f:12-500.  Each sum Qh = Qh + dFx + dFy + dFz
// is accumulated by the derivative kernels themselves in the reference's
// x, y, z order (iadd), so dF*/dE* are never stored; fluxes that are products
// of stored fields are formed by the derivative kernels while loading.
template <class R>
static int hyper_rhs_t(st_ctx *c, const double *Q, R *Qrhs, const double *Y, const R *Yr) {
    if (c->p.hyper_param == 0) return ST_OK;
    const size_t n3 = c->fs, nc = c->ncell();   // field stride; cells processed
    ST_TRY(compute_hyper_t<R>(c, Q, Y, Yr));
    const double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3;
    ScratchNT<R> s(c, 9);
    R *U1 = s[0], *U2 = s[1], *U3 = s[2], *dila = s[3], *S1 = s[4], *S2 = s[5], *S3 = s[6];
    R *Flux = s[7], *Flux2 = s[8];
    ScratchT<R> Qhs(c, 5);
    R *Qh = Qhs;   // Qh(:,:,:,4) stays zero and is never added
    R *h1 = Qh, *h2 = Qh + n3, *h3 = Qh + 2 * n3, *h5 = Qh + 4 * n3;
    R *const *Gr = Store<R>::grad(c);
    const R *G0 = Gr[0], *G1 = Gr[1], *G2 = Gr[2], *G3 = Gr[3], *G4 = Gr[4], *G5 = Gr[5], *G6 = Gr[6],
            *G7 = Gr[7], *G8 = Gr[8];
    const R *GTx = Gr[G_DTDX], *GTy = Gr[G_DTDY], *GTz = Gr[G_DTDZ];
    R *const *H = Store<R>::hyp(c);
    const R *vh = H[H_VISC], *bh = H[H_BETA], *kh = H[H_K];
    PFOR(c, nc, io(Q1, Q2, Q3, Q4, G0, G1, G2, G3, G4, G5, G6, G7, G8, vh, bh, U1, U2, U3, dila, S1, S2, S3, Flux, Flux2), {
        U1[p] = Q1[p] / Q4[p];
        U2[p] = Q2[p] / Q4[p];
        U3[p] = Q3[p] / Q4[p];
        dila[p] = G0[p] + G4[p] + G8[p];
        S1[p] = G3[p] + G1[p];
        S2[p] = G6[p] + G2[p];
        S3[p] = G7[p] + G5[p];
        Flux[p] = 2.0 * vh[p] * G0[p] + (bh[p] - (2.0 / 3.0) * vh[p]) * dila[p];
        Flux2[p] = 2.0 * vh[p] * G4[p] + (bh[p] - (2.0 / 3.0) * vh[p]) * dila[p];
    });
    // x momentum: Qh1 = dFx + dFy + dFz, Qh5 = dEx + dEy + dEz
    // (each line pair: a flux and its product with a velocity component, the
    // second reading what the first reads; one launch per pair)
    const R *cF = Flux, *cF2 = Flux2;
    ST_TRY(dfd_pair<R>(c, 0, pr_one(cF), h1, 0, 0, pr_mul(U1, cF), h5, 1, 0));
    ST_TRY(dfd_pair<R>(c, 1, pr_mul(vh, S1), h1, 1, 1, pr_mulmul(vh, S1, U1), h5, 1, 1));
    ST_TRY(dfd_pair<R>(c, 2, pr_mul(vh, S2), h1, 1, 1, pr_mulmul(vh, S2, U1), h5, 1, 1));
    // y momentum (x, y, z accumulation order)
    ST_TRY(dfd_pair<R>(c, 0, pr_mul(vh, S1), h2, 1, 0, pr_mulmul(vh, S1, U2), h5, 1, 1));
    ST_TRY(dfd_pair<R>(c, 1, pr_one(cF2), h2, 0, 1, pr_mul(U2, cF2), h5, 1, 1));
    ST_TRY(dfd_pair<R>(c, 2, pr_mul(vh, S3), h2, 1, 1, pr_mulmul(vh, S3, U2), h5, 1, 1));
    // z momentum
    PFOR(c, nc, io(vh, G8, bh, dila, Flux), { Flux[p] = 2.0 * vh[p] * G8[p] + (bh[p] - (2.0 / 3.0) * vh[p]) * dila[p]; });
    ST_TRY(dfd_pair<R>(c, 0, pr_mul(vh, S2), h3, 1, 0, pr_mulmul(vh, S2, U3), h5, 1, 1));
    ST_TRY(dfd_pair<R>(c, 1, pr_mul(vh, S3), h3, 1, 1, pr_mulmul(vh, S3, U3), h5, 1, 1));
    ST_TRY(dfd_pair<R>(c, 2, pr_one(cF), h3, 0, 1, pr_mul(U3, cF), h5, 1, 1));
    // artificial heat flux
    ST_TRY(dfd(c, 0, 0, pr_mul(kh, GTx), h5, 1, 1.0));
    ST_TRY(dfd(c, 1, 0, pr_mul(kh, GTy), h5, 1, 1.0));
    ST_TRY(dfd(c, 2, 0, pr_mul(kh, GTz), h5, 1, 1.0));
    PFOR(c, nc, 4 * io(Qrhs, Qrhs, Qh), {
        for (int l = 0; l < 5; l++)
            if (l != 3) Qrhs[l * n3 + p] = Qrhs[l * n3 + p] + Qh[l * n3 + p];
    });
    return ST_OK;
}

// Species_RHS src/species_rhs_sym.f:9-207.  Yrhs accumulates the three
// convective derivatives in x, y, z order, then adds Ydiff, as
// Yrhs = Yconvx + Yconvy + Yconvz + Ydiff does.
template <class R>
static int species_rhs_t(st_ctx *c, const double *Q, const R *Qr, R *Qrhs, const double *Y, const R *Yr,
                         R *Yrhs) {
    if (c->p.hyper_param == 0) return ST_OK;
    const size_t n3 = c->fs, nc = c->ncell();   // field stride; cells processed
    Phys f = phys(c);
    const double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    const R *q1r = Qr, *q2r = Qr + n3, *q3r = Qr + 2 * n3, *q4r = Qr + 3 * n3;
    ScratchNT<R> s(c, 2);
    R *Yd = s[0], *T = s[1];
    R *const *dYd = Store<R>::dYd(c);
    const R *Dh = Store<R>::hyp(c)[H_D];
    const double *g = c->gamma_eff;
    PFOR(c, nc, io(g, Y, Q1, Q2, Q3, Q4, Q5, T), {
        double Vs, P, Tt;
        thermo(f, g[p], Y[p], Q1[p], Q2[p], Q3[p], Q4[p], Q5[p], Vs, P, Tt);
        T[p] = Tt;
    });
    // dY/dx_i and d(rho u_i Y)/dx_i per direction, one launch each (the
    // gradient and the flux are independent; the flux keeps its x, y, z order)
    const R *qr[3] = {q1r, q2r, q3r};
    for (int d = 0; d < 3; d++) {
        const D1SpecT<R> ops[2] = {{pr_one(Yr), dYd[d], 0, 0, 1.0},
                                   {pr_mul(qr[d], Yr), Yrhs, 1, d == 0 ? 0 : 1, -1.0}};
        if constexpr (sizeof(R) == 8) ST_TRY(dev_dfd_pair(c, d, ops));
        else ST_TRY(dev_dfd_pair_f(c, d, ops));
    }
    const double cst = 1.0 - f.eps * f.g2 * (f.g1 - 1.0) / (f.g1 * (f.g2 - 1.0));
    for (int d = 0; d < 3; d++) {
        ProdT<R> fl{};
        fl.op = PR_SPEC; fl.a = q4r; fl.b = Dh; fl.c = dYd[d]; fl.k0 = f.Re1_inv; fl.k1 = f.Sc_inv;
        ProdT<R> ft = fl;
        ft.op = PR_SPECT; ft.d = T; ft.k2 = cst;
        ST_TRY(dfd_pair<R>(c, d, fl, Yd, 1, d == 0 ? 0 : 1, ft, Qrhs + 4 * n3, 1, 1));
    }
    PFOR(c, nc, io(Yrhs, Yrhs, Yd), { Yrhs[p] = Yrhs[p] + Yd[p]; });
    return ST_OK;
}

// bc_RHS src/bc_mf.f:11-463 (active face blocks)
template <class R>
static int bc_rhs_t(st_ctx *c, double *Q, R *Qrhs, const double *Y, R *Yrhs) {
    const size_t n3 = c->fs, nc = c->ncell();   // field stride; cells processed
    const int Mx = c->dm.n[0], My = c->dm.n[1], Mz = c->dm.n[2];
    Phys f = phys(c);
    double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    const double *g = c->gamma_eff;
    // symmetry planes: x=0 (rho u), z=0 (rho w), y=0 (rho v); one launch per
    // plane over its cells only
    // (each plane of every processed case: case k's cells start at k*n3c)
    const size_t n3c = c->dm.n3, na = (size_t)c->na;
    {
        const size_t MyMz = (size_t)My * Mz, MyMx = (size_t)My * Mx, MzMx = (size_t)Mz * Mx;
        PFOR(c, na * MyMz, io(Q1), {                                          // i = 0: p = j + My*k
            size_t k = p / MyMz;
            Q1[k * n3c + (p - k * MyMz)] = 0.0;
        });
        PFOR(c, na * MyMx, io(Q3), {                                          // k = 0: p = j + My*i
            size_t k = p / MyMx, q = p - k * MyMx;
            Q3[k * n3c + (q % My) + MyMz * (q / My)] = 0.0;
        });
        PFOR(c, na * MzMx, io(Q2), {                                          // j = 0: p = k + Mz*i
            size_t k = p / MzMx;
            Q2[k * n3c + (size_t)My * (p - k * MzMx)] = 0.0;
        });
    }
    ScratchNT<R> s(c, 4);
    R *P = s[0], *dPx = s[1], *dPy = s[2], *dPz = s[3];
    PFOR(c, nc, io(g, Y, Q1, Q2, Q3, Q4, Q5, P), {
        double Vs, Pp, T;
        thermo(f, g[p], Y[p], Q1[p], Q2[p], Q3[p], Q4[p], Q5[p], Vs, Pp, T);
        P[p] = Pp;
    });
    ST_TRY(dfd(c, 0, 0, P, dPx, 0, 1.0));
    ST_TRY(dfd(c, 1, 0, P, dPy, 0, 1.0));
    ST_TRY(dfd(c, 2, 0, P, dPz, 0, 1.0));
    R *const *Gr = Store<R>::grad(c);
    const R *Gxx = Gr[G_DUX_DX], *Gyy = Gr[G_DUY_DY], *Gzz = Gr[G_DUZ_DZ];
    // faces in the reference order x, y, z (later faces overwrite edges)
    for (int face = 0; face < 3; face++) {
        size_t nf = face == 0 ? (size_t)My * Mz : face == 1 ? (size_t)Mx * Mz : (size_t)Mx * My;
        PFOR(c, na * nf, io(Q1, Q2, Q3, Q4, P, g, dPx, Gxx, Yrhs) + 5 * io(Qrhs), {
            const size_t k = p / nf, pl = p - k * nf;
            size_t q;
            if (face == 0) q = pl + (size_t)My * Mz * (Mx - 1);                    // pl = j + My*k
            else if (face == 1) q = (My - 1) + (size_t)My * pl;                    // pl = k + Mz*i
            else q = (pl % My) + (size_t)My * (Mz - 1) + (size_t)My * Mz * (pl / My);  // pl = j + My*i
            q += k * n3c;
            double Vs = 1.0 / Q4[q];
            double Pq = P[q];
            double U[3] = {Q1[q] * Vs, Q2[q] * Vs, Q3[q] * Vs};
            double Ur = sqrt(U[0] * U[0] + U[1] * U[1] + U[2] * U[2]);
            double tmp2 = sqrt(g[q] * Vs * Pq);
            double dPn = face == 0 ? dPx[q] : face == 1 ? dPy[q] : dPz[q];
            double dun = face == 0 ? Gxx[q] : face == 1 ? Gyy[q] : Gzz[q];
            double un = U[face];
            double L1 = 0.0, L2 = 0.0, L3 = 0.0, L4 = 0.0, L6 = 0.0;
            double L5 = (un + tmp2) * (dPn + tmp2 * Q4[q] * dun);
            double d1 = (1.0 / (tmp2 * tmp2)) * (L2 + 5.0e-1 * (L1 + L5));
            double d2 = 5.0e-1 * (L5 + L1);
            double d3 = (5.0e-1 / (Q4[q] * tmp2)) * (L5 - L1);
            double d4 = L3, d5 = L4, d6 = L6;
            double Qm[3] = {Q1[q], Q2[q], Q3[q]};
            // normal momentum component gets d3; the two tangential get d4, d5
            int t1 = face == 0 ? 1 : 0, t2 = face == 2 ? 1 : 2;
            Qrhs[3 * n3 + q] = -d1;
            Qrhs[4 * n3 + q] = -5.0e-1 * Ur * Ur * d1 - d2 / (g[q] - 1.0) - Qm[face] * d3 - Qm[t1] * d4 -
                               Qm[t2] * d5;
            Qrhs[face * n3 + q] = -U[face] * d1 - Q4[q] * d3;
            Qrhs[t1 * n3 + q] = -U[t1] * d1 - Q4[q] * d4;
            Qrhs[t2 * n3 + q] = -U[t2] * d1 - Q4[q] * d5;
            Yrhs[q] = -Q4[q] * d6;
        });
    }
    return ST_OK;
}

// Sponge_Forcing src/sponge_mf.f:7-127
template <class R>
static int sponge_t(st_ctx *c, const double *Q, R *Qrhs, const double *Y, R *Yrhs) {
    const size_t n3 = c->fs, nc = c->ncell();   // field stride; cells processed
    const int Mx = c->dm.n[0], My = c->dm.n[1], Mz = c->dm.n[2];
    const double g1 = c->p.gamma1;
    const double base_pressure = 0.71429, Ms = 1.8;
    const double rho_ref = (g1 + 1.0) * Ms * Ms / ((g1 - 1.0) * Ms * Ms + 2.0);
    const double P_ref = ((2.0 * g1 / (g1 + 1.0)) * (Ms * Ms - 1.0) + 1.0) * base_pressure;
    const double E_ref = P_ref / (g1 - 1.0), Y_ref = 1.0;
    int start[3], len[3];
    const int Ns[3] = {Mx, My, Mz};
    for (int d = 0; d < 3; d++) {
        start[d] = Ns[d] - (int)ceil(0.1 * Ns[d]);
        len[d] = Ns[d] - start[d];
    }
    const int sx = start[0], sy = start[1], sz = start[2], lx = len[0], ly = len[1], lz = len[2];
    const size_t n3c = c->dm.n3;
    const bool idx32 = nc <= 0xffffffffull;   // 32-bit index arithmetic when it suffices
    const bool one = c->na == 1;
    // fraction of the cells in the sponge shell (the only ones touched)
    const double shell = (double)(n3c - (size_t)sx * sy * sz) / (double)n3c;
    PFOR(c, nc, shell * (10 * io(Qrhs) + 5 * io(Q) + io(Y) + 2 * io(Yrhs)), {
        int j, k, i;
        if (idx32) {
            unsigned q = (unsigned)p;
            if (!one) q -= (q / (unsigned)n3c) * (unsigned)n3c;   // position within the case
            unsigned r = q / (unsigned)My;
            j = (int)(q - r * (unsigned)My); k = (int)(r % (unsigned)Mz); i = (int)(r / (unsigned)Mz);
        } else {
            size_t q = one ? p : p - (p / n3c) * n3c;
            size_t r = q / My;
            j = (int)(q - r * My); k = (int)(r % Mz); i = (int)(r / Mz);
        }
        auto sig = [](int gI, int st, int ln) -> double {
            if (gI >= st) {
                float r = (float)(gI - st) / (float)ln;   // REAL/REAL, src/sponge_mf.f:87-89
                return 4.0 * pow((double)r, 3.0);
            }
            return 0.0;
        };
        double s = sig(i + 1, sx, lx) + sig(j + 1, sy, ly) + sig(k + 1, sz, lz);
        // outside the sponge shell the forcing is 0*(...): the right-hand
        // sides keep their values (up to the sign of a zero), so those cells
        // are not touched
        if (s == 0.0) return;
        double Qref[5] = {0.0, 0.0, 0.0, rho_ref, E_ref};
        for (int l = 0; l < 5; l++) Qrhs[l * n3 + p] = Qrhs[l * n3 + p] - s * (Q[l * n3 + p] - Qref[l]);
        Yrhs[p] = Yrhs[p] - s * (Q[3 * n3 + p] * Y[p] - Q[3 * n3 + p] * Y_ref);
    });
    return ST_OK;
}

// ---- entry points on double arrays -----------------------------------------------
// In the FP32 mode the caller's double arrays are rounded to float copies,
// the float form runs, and accumulated outputs are widened back.
int dev_rhs(st_ctx *c, double *Q, double *Qrhs, const double *Y) {
    if (!fp32_mode(c)) return rhs_t<double>(c, Q, Q, Qrhs, Y);
    const size_t n3 = c->fs, nc = c->ncell();   // field stride; cells processed
    ScratchT<float> Qs(c, 5), Rs(c, 5);
    ST_TRY(dev_to_float(c, Q, Qs, 5 * n3));
    ST_TRY(rhs_t<float>(c, Q, Qs, Rs, Y));
    return dev_to_double(c, Rs, Qrhs, 5 * n3);
}

int dev_compute_hyper(st_ctx *c, const double *Q, const double *Y) {
    if (!fp32_mode(c)) return compute_hyper_t<double>(c, Q, Y, Y);
    ScratchT<float> Ys(c, 1);
    ST_TRY(dev_to_float(c, Y, Ys, c->ncell()));
    return compute_hyper_t<float>(c, Q, Y, Ys);
}

int dev_hyper_rhs(st_ctx *c, const double *Q, double *Qrhs, const double *Y) {
    if (!fp32_mode(c)) return hyper_rhs_t<double>(c, Q, Qrhs, Y, Y);
    const size_t n3 = c->fs, nc = c->ncell();   // field stride; cells processed
    ScratchT<float> Ys(c, 1), Rs(c, 5);
    ST_TRY(dev_to_float(c, Y, Ys, n3));
    ST_TRY(dev_to_float(c, Qrhs, Rs, 5 * n3));
    ST_TRY(hyper_rhs_t<float>(c, Q, Rs, Y, Ys));
    return dev_to_double(c, Rs, Qrhs, 5 * n3);
}

int dev_species_rhs(st_ctx *c, const double *Q, double *Qrhs, const double *Y, double *Yrhs) {
    if (!fp32_mode(c)) return species_rhs_t<double>(c, Q, Q, Qrhs, Y, Y, Yrhs);
    const size_t n3 = c->fs, nc = c->ncell();   // field stride; cells processed
    ScratchT<float> Qs(c, 5), Ys(c, 1), Rs(c, 5), YRs(c, 1);
    ST_TRY(dev_to_float(c, Q, Qs, 5 * n3));
    ST_TRY(dev_to_float(c, Y, Ys, n3));
    ST_TRY(dev_to_float(c, Qrhs, Rs, 5 * n3));
    ST_TRY(species_rhs_t<float>(c, Q, Qs, Rs, Y, Ys, YRs));
    ST_TRY(dev_to_double(c, Rs, Qrhs, 5 * n3));
    return dev_to_double(c, YRs, Yrhs, n3);
}

int dev_bc_rhs(st_ctx *c, double *Q, double *Qrhs, const double *Y, double *Yrhs) {
    if (!fp32_mode(c)) return bc_rhs_t<double>(c, Q, Qrhs, Y, Yrhs);
    const size_t n3 = c->fs, nc = c->ncell();   // field stride; cells processed
    ScratchT<float> Rs(c, 5), YRs(c, 1);
    ST_TRY(dev_to_float(c, Qrhs, Rs, 5 * n3));
    ST_TRY(dev_to_float(c, Yrhs, YRs, n3));
    ST_TRY(bc_rhs_t<float>(c, Q, Rs, Y, YRs));
    ST_TRY(dev_to_double(c, Rs, Qrhs, 5 * n3));
    return dev_to_double(c, YRs, Yrhs, n3);
}

int dev_sponge(st_ctx *c, const double *Q, double *Qrhs, const double *Y, double *Yrhs) {
    if (!fp32_mode(c)) return sponge_t<double>(c, Q, Qrhs, Y, Yrhs);
    const size_t n3 = c->fs, nc = c->ncell();   // field stride; cells processed
    ScratchT<float> Rs(c, 5), YRs(c, 1);
    ST_TRY(dev_to_float(c, Qrhs, Rs, 5 * n3));
    ST_TRY(dev_to_float(c, Yrhs, YRs, n3));
    ST_TRY(sponge_t<float>(c, Q, Rs, Y, YRs));
    ST_TRY(dev_to_double(c, Rs, Qrhs, 5 * n3));
    return dev_to_double(c, YRs, Yrhs, n3);
}

// Fix_Pressure pproc/pproc_mf.f:190-233; periodic family
// src/lddrk4_periodic_sf.f:436-473 (base pressure 0.71463, gamma_eff = gamma)
int dev_fix_pressure(st_ctx *c, double *Q) {
    const size_t n3 = c->fs, nc = c->ncell();   // field stride; cells processed
    double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    const double *g = c->gamma_eff;
    const double base = c->p.family == ST_FAMILY_PERIODIC ? 0.71463 : 0.71429;
    PFOR(c, nc, io(g, Q1, Q2, Q3, Q4, Q5, Q5), {
        double fac1 = g[p] - 1.0;
        double Vs = 1.0 / Q4[p];
        double P = fac1 * (Q5[p] - 5.0e-1 * Vs * (Q1[p] * Q1[p] + Q2[p] * Q2[p] + Q3[p] * Q3[p]));
        if (P < 0.0) P = base;
        Q5[p] = (1.0 / fac1) * P + 5.0e-1 * Vs * (Q1[p] * Q1[p] + Q2[p] * Q2[p] + Q3[p] * Q3[p]);
    });
    return ST_OK;
}

// Fix_Pressure of the FP32 mode's stages: as above, and the float copy of
// the state for the next stage
static int fix_pressure_copy(st_ctx *c, double *Q, float *qs) {
    const size_t n3 = c->fs, nc = c->ncell();   // field stride; cells processed
    double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    const double *g = c->gamma_eff;
    const double base = c->p.family == ST_FAMILY_PERIODIC ? 0.71463 : 0.71429;
    PFOR(c, nc, io(g, Q1, Q2, Q3, Q4, Q5, Q5) + 5 * io(qs), {
        double fac1 = g[p] - 1.0;
        double Vs = 1.0 / Q4[p];
        double P = fac1 * (Q5[p] - 5.0e-1 * Vs * (Q1[p] * Q1[p] + Q2[p] * Q2[p] + Q3[p] * Q3[p]));
        if (P < 0.0) P = base;
        double q5 = (1.0 / fac1) * P + 5.0e-1 * Vs * (Q1[p] * Q1[p] + Q2[p] * Q2[p] + Q3[p] * Q3[p]);
        Q5[p] = q5;
        qs[p] = (float)Q1[p]; qs[n3 + p] = (float)Q2[p]; qs[2 * n3 + p] = (float)Q3[p];
        qs[3 * n3 + p] = (float)Q4[p]; qs[4 * n3 + p] = (float)q5;
    });
    return ST_OK;
}

// Compact_Filter src/filters_sym.f:398-432
int dev_compact_filter(st_ctx *c, const double *F, double *F0, int nvar) {
    const size_t n3 = c->fs, nc = c->ncell();   // field stride; cells processed
    for (int l = 0; l < nvar; l++) {
        ST_TRY(dev_filter(c, 0, l == 0, F + l * n3, F0 + l * n3));
        ST_TRY(dev_filter(c, 1, l == 1, F0 + l * n3, F0 + l * n3));
        ST_TRY(dev_filter(c, 2, l == 2, F0 + l * n3, F0 + l * n3));
    }
    return ST_OK;
}

int dev_gaussian_filter(st_ctx *c, const double *F, double *Fg, int nvar) {
    return gaussian_filter_t<double>(c, F, Fg, nvar);
}

// ---- reductions ----------------------------------------------------------------
// max/min of non-negative doubles through their ordered bit patterns
__device__ __forceinline__ void atomic_max_pos(double *a, double v) {
    atomicMax((unsigned long long *)a, (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ void atomic_min_pos(double *a, double v) {
    atomicMin((unsigned long long *)a, (unsigned long long)__double_as_longlong(v));
}

// Compute_CFL src/lddrk4_nonperiodic_mf.f:7-66 -> dscal[0]=stab, dscal[1]=resv
// of each case (blockIdx.y: case; n3: cells of a case; fs: field stride)
__global__ void k_cfl(const double *Q, const double *g, size_t n3c, size_t fs, double DX, double DY, double DZ,
                      double *out) {
    const double kmax = 2.478, khug = 2.199;   // src/header:237-240
    const size_t n3 = fs, c0 = (size_t)blockIdx.y * n3c, end = c0 + n3c;
    out += (size_t)blockIdx.y * kScal;
    double m1 = 0.0, m2 = 0.0;
    for (size_t p = c0 + (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < end; p += (size_t)gridDim.x * blockDim.x) {
        double fac = g[p] * (g[p] - 1.0);
        double tmp1 = 1.0 / Q[3 * n3 + p];
        double q1 = Q[p], q2 = Q[n3 + p], q3 = Q[2 * n3 + p];
        double tmp2 = sqrt(fac * tmp1 * (Q[4 * n3 + p] - 5.0e-1 * tmp1 * (q1 * q1 + q2 * q2 + q3 * q3)));
        double ux = fabs(q1 * tmp1), uy = fabs(q2 * tmp1), uz = fabs(q3 * tmp1);
        double w1 = ((tmp2 + ux) * kmax / DX + (tmp2 + uy) * kmax / DY + (tmp2 + uz) * kmax / DZ);
        double w2 = ((tmp2 + ux) * khug / DX + (tmp2 + uy) * khug / DY + (tmp2 + uz) * khug / DZ);
        m1 = fmax(m1, w1);
        m2 = fmax(m2, w2);
    }
    for (int o = 16; o > 0; o >>= 1) {
        m1 = fmax(m1, __shfl_down_sync(0xffffffffu, m1, o));
        m2 = fmax(m2, __shfl_down_sync(0xffffffffu, m2, o));
    }
    if ((threadIdx.x & 31) == 0) { atomic_max_pos(out + 0, m1); atomic_max_pos(out + 1, m2); }
}

// Compute_Tstep hyperviscous limits src/lddrk4_nonperiodic_mf.f:100-145 -> out[2..5] minima
template <class R>
__global__ void k_tstep(const double *Q, const double *Y, const double *g, const R *vh, const R *bh,
                        const R *kh, const R *Dh, size_t n3c, size_t fs, double del, double g1, double g2,
                        double eps, double *out) {
    const size_t n3 = fs, c0 = (size_t)blockIdx.y * n3c, end = c0 + n3c;
    out += (size_t)blockIdx.y * kScal;
    double m3 = INFINITY, m4 = INFINITY, m5 = INFINITY, m6 = INFINITY;
    for (size_t p = c0 + (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < end; p += (size_t)gridDim.x * blockDim.x) {
        double fac = g[p] * (g[p] - 1.0);
        float fac1 = (float)(Y[p] + (eps * (g1 - 1.0) / (g2 - 1.0)) * (1.0 - Y[p]));   // implicit REAL
        double tmp1 = 1.0 / Q[3 * n3 + p];
        double q1 = Q[p], q2 = Q[n3 + p], q3 = Q[2 * n3 + p], q5 = Q[4 * n3 + p];
        double tmp2 = sqrt(fac * tmp1 * (q5 - 5.0e-1 * tmp1 * (q1 * q1 + q2 * q2 + q3 * q3)));
        double T = g1 * tmp1 * (q5 - 5.0e-1 * tmp1 * (q1 * q1 + q2 * q2 + q3 * q3));
        T = T / (double)fac1;
        double q4 = Q[3 * n3 + p];
        double w3 = q4 * pow(del, 2.0) / (double)vh[p];
        double w4 = q4 * pow(del, 2.0) / (double)bh[p];
        double w5 = q4 * pow(del * tmp2, 2.0) / ((double)kh[p] * T);
        double w6 = pow(del, 2.0) / (double)Dh[p];
        m3 = fmin(m3, w3); m4 = fmin(m4, w4); m5 = fmin(m5, w5); m6 = fmin(m6, w6);
    }
    for (int o = 16; o > 0; o >>= 1) {
        m3 = fmin(m3, __shfl_down_sync(0xffffffffu, m3, o));
        m4 = fmin(m4, __shfl_down_sync(0xffffffffu, m4, o));
        m5 = fmin(m5, __shfl_down_sync(0xffffffffu, m5, o));
        m6 = fmin(m6, __shfl_down_sync(0xffffffffu, m6, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomic_min_pos(out + 2, m3); atomic_min_pos(out + 3, m4);
        atomic_min_pos(out + 4, m5); atomic_min_pos(out + 5, m6);
    }
}

// Compute_Tstep of the periodic family, src/lddrk4_periodic_sf.f:105-135:
// single-fluid temperature, no diffusivity limit (out[5] stays +inf)
template <class R>
__global__ void k_tstep_sf(const double *Q, const R *vh, const R *bh, const R *kh, size_t n3c, size_t fs,
                           double del, double gam, double *out) {
    const size_t n3 = fs, c0 = (size_t)blockIdx.y * n3c, end = c0 + n3c;
    out += (size_t)blockIdx.y * kScal;
    double m3 = INFINITY, m4 = INFINITY, m5 = INFINITY;
    const double fac = gam * (gam - 1.0);
    for (size_t p = c0 + (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < end; p += (size_t)gridDim.x * blockDim.x) {
        double tmp1 = 1.0 / Q[3 * n3 + p];
        double q1 = Q[p], q2 = Q[n3 + p], q3 = Q[2 * n3 + p], q4 = Q[3 * n3 + p], q5 = Q[4 * n3 + p];
        double tmp2 = sqrt(fac * tmp1 * (q5 - 5.0e-1 * tmp1 * (q1 * q1 + q2 * q2 + q3 * q3)));
        double T = gam * tmp1 * (q5 - 5.0e-1 * tmp1 * (q1 * q1 + q2 * q2 + q3 * q3));
        double w3 = q4 * pow(del, 2.0) / (double)vh[p];
        double w4 = q4 * pow(del, 2.0) / (double)bh[p];
        double w5 = q4 * pow(del * tmp2, 2.0) / ((double)kh[p] * T);
        m3 = fmin(m3, w3); m4 = fmin(m4, w4); m5 = fmin(m5, w5);
    }
    for (int o = 16; o > 0; o >>= 1) {
        m3 = fmin(m3, __shfl_down_sync(0xffffffffu, m3, o));
        m4 = fmin(m4, __shfl_down_sync(0xffffffffu, m4, o));
        m5 = fmin(m5, __shfl_down_sync(0xffffffffu, m5, o));
    }
    if ((threadIdx.x & 31) == 0) { atomic_min_pos(out + 2, m3); atomic_min_pos(out + 3, m4); atomic_min_pos(out + 4, m5); }
}

// dt = min(cfl_cal/cfl_resv, f*minima) -> out[6]; resv taken from out[1].
// f is 0.2D0 in src/lddrk4_nonperiodic_mf.f:156-157 and the default-REAL
// literal 0.2 (float32) in src/lddrk4_periodic_sf.f:141-142; out[5] = +inf
// when a limit is absent.
// Thread k: case k.  use_hyper < 0: each case decides from its own step
// count (out[SC_STEP], advanced here), with the limits from step > hyper_from.
__global__ void k_tstep_final(double *out, int ncase, double cfl_cal, int use_hyper, int hyper_from, int resv_dev,
                              double resv_host, double f) {
    const int k = threadIdx.x;
    if (k >= ncase) return;
    out += (size_t)k * kScal;
    double resv = resv_dev ? out[1] : resv_host;
    double t = cfl_cal / resv;
    bool hyp = use_hyper > 0;
    if (use_hyper < 0) {
        hyp = out[SC_STEP] > (double)hyper_from;
        out[SC_STEP] = out[SC_STEP] + 1.0;
    }
    if (hyp) {
        double cand[4] = {f * out[2], f * out[3], f * out[4], f * out[5]};
        for (int q = 0; q < 4; q++) if (cand[q] < t) t = cand[q];
    }
    out[6] = t;
}

static int grid_blocks(size_t n) {
    size_t b = (n + 255) / 256;
    return (int)(b > 148 * 8 ? 148 * 8 : (b ? b : 1));
}

int dev_compute_cfl(st_ctx *c, const double *Q, bool to_host, double *stab, double *resv) {
    ST_CUDA(c, cudaMemset2DAsync(c->dscal, kScal * sizeof(double), 0, 2 * sizeof(double), c->na, c->stream));
    int pi = prof_start(c, "k_cfl", 48.0 * c->ncell());
    const dim3 grid(grid_blocks(c->dm.n3), c->na);
    k_cfl<<<grid, 256, 0, c->stream>>>(Q, c->gamma_eff, c->dm.n3, c->fs, c->DX, c->DY, c->DZ, c->dscal);
    prof_stop(c, pi);
    ST_CUDA(c, cudaGetLastError());
    if (to_host) {
        ST_CUDA(c, cudaMemcpyAsync(c->hpinned, c->dscal, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        ST_CUDA(c, cudaStreamSynchronize(c->stream));
        if (stab) *stab = c->hpinned[0];
        if (resv) *resv = c->hpinned[1];
        c->last_cfl_stab = c->hpinned[0];
        c->last_cfl_resv = c->hpinned[1];
    }
    return ST_OK;
}

// dt lands in dscal[6] (device); the context's host copy is refreshed only
// when the caller asks for it.
template <class R>
static int tstep_hyper(st_ctx *c, const double *Q, const double *Y, bool sf) {
    R *const *H = Store<R>::hyp(c);
    const dim3 grid(grid_blocks(c->dm.n3), c->na);
    if (sf) {
        int pi = prof_start(c, "k_tstep", (40.0 + 3 * sizeof(R)) * c->ncell());
        k_tstep_sf<R><<<grid, 256, 0, c->stream>>>(Q, H[H_VISC], H[H_BETA], H[H_K], c->dm.n3, c->fs, c->DX,
                                                   c->p.gamma1, c->dscal);
        prof_stop(c, pi);
    } else {
        int pi = prof_start(c, "k_tstep", (56.0 + 4 * sizeof(R)) * c->ncell());
        k_tstep<R><<<grid, 256, 0, c->stream>>>(Q, Y, c->gamma_eff, H[H_VISC], H[H_BETA], H[H_K], H[H_D],
                                                c->dm.n3, c->fs, c->DX, c->p.gamma1, c->p.gamma2, c->p.epsilon,
                                                c->dscal);
        prof_stop(c, pi);
    }
    ST_CUDA(c, cudaGetLastError());
    return ST_OK;
}

// step < 0: a batch step, in which each case takes its own step count from
// its scalars (the limits may apply to some cases and not others).
int dev_compute_tstep(st_ctx *c, const double *Q, const double *Y, int step, bool resv_on_device,
                      double cfl_resv_host) {
    const bool sf = c->p.family == ST_FAMILY_PERIODIC;
    // hyperviscous limits from the first step on (_mf) or the second (periodic)
    const int hyper_from = sf ? 1 : 0;
    const bool per_case = step < 0;
    const bool use_hyper = c->p.hyper_param == 1 && (per_case || step > hyper_from);
    if (use_hyper) {
        // minima start at +inf (a device fill, so that the step can be captured in a graph)
        double *d = c->dscal;
        PFOR(c, (size_t)c->na * 4, io(d), { d[(p >> 2) * kScal + 2 + (p & 3)] = INFINITY; });
        ST_TRY(fp32_mode(c) ? tstep_hyper<float>(c, Q, Y, sf) : tstep_hyper<double>(c, Q, Y, sf));
    }
    c->launches++;
    const double f = sf ? (double)0.2f : 0.2;
    const int mode = !use_hyper ? 0 : (per_case ? -1 : 1);
    k_tstep_final<<<1, ((c->na + 31) / 32) * 32, 0, c->stream>>>(c->dscal, c->na, c->p.cfl_cal, mode, hyper_from,
                                                                 resv_on_device ? 1 : 0, cfl_resv_host, f);
    ST_CUDA(c, cudaGetLastError());
    return ST_OK;
}

// ---- LDDRK4 (src/lddrk4_nonperiodic_mf.f:428-541) -------------------------------
// dt is read from dscal[6] on the device (set by dev_compute_tstep or
// st_set_tstep), so the whole step can run without a host round trip.
// The QW = 0 / rYW = 0 resets at the start of each loop are folded into the
// first stage, whose coefficient alpha(1) is 0 (0*0 + dt*dQ == dt*dQ); the
// last filter pass of each conserved variable writes Q itself (Q = Qf), and
// Compute_Y is fused with Fix_Pressure.
// LDDRK4 of the periodic family, src/lddrk4_periodic_sf.f:311-430: 5 stages
// with alpha1/beta1, then 6 with alpha2/beta2 (unassigned in the reference
// build, i.e. zero: rk_mode 0; rk_mode 1 takes the commented-out HHM 4-6
// values of src/header:267-276).  Each stage: RHS, Hyper_RHS, update,
// Compact_Filter (Q = Qf), Fix_Pressure.
// The state in the intermediate type R: the state arrays themselves in FP64;
// float copies, refreshed before each stage, in the FP32 mode.
template <class R> struct StateCopy;
template <> struct StateCopy<double> {
    StateCopy(st_ctx *) {}
    const double *q(const double *Q) const { return Q; }
    const double *y(const double *Y) const { return Y; }
};
template <> struct StateCopy<float> {
    ScratchT<float> qs, ys;
    explicit StateCopy(st_ctx *c) : qs(c, 5), ys(c, 1) {}
    const float *q(const double *) const { return qs; }
    const float *y(const double *) const { return ys; }
};
// (the Compute_Y/Fix_Pressure kernel at the end of a stage writes the copy
// for the next stage; a call's first stage makes it here)
template <class R>
static int refresh(st_ctx *c, StateCopy<R> &sc, const double *Q, const double *Y, bool with_y) {
    if constexpr (!is_fp64<R>()) {
        const size_t n3 = c->fs, nc = c->ncell();   // field stride; cells processed
        float *qs = sc.qs, *ys = sc.ys;
        PFOR(c, nc, 5 * io(Q, qs) + (with_y ? io(Y, ys) : 0.0), {
            for (int l = 0; l < 5; l++) qs[l * n3 + p] = (float)Q[l * n3 + p];
            if (with_y) ys[p] = (float)Y[p];
        });
    }
    return ST_OK;
}

template <class R>
static int lddrk4_sf(st_ctx *c) {
    static const double alpha1[5] = {0.0, -4.801594388477952e-01, -1.404247195200064e+00,
                                     -2.016477077503357e+00, -1.056444269767207e+00};
    static const double beta1[5] = {1.028639988104959e-01, 7.408540575766301e-01, 7.426530946683799e-01,
                                    4.694937902357905e-01, 1.881733382887932e-01};
    static const double alpha2[6] = {0.0, -4.4127377153877382565e-1, -1.073982008079781868e0,
                                     -1.7063570791256758809e0, -2.7979293162682443056e0,
                                     -4.0913537120919160454e0};
    static const double beta2[6] = {1.1584888181285561688e-1, 3.7287699051652864918e-1,
                                    7.3795368921435295698e-1, 5.7981109366311039538e-1,
                                    1.031284991300145194e0, 1.5e-1};
    const size_t n3 = c->fs, nc = c->ncell();   // field stride; cells processed
    Scratch Qfs(c, 5);
    double *Qf = Qfs;
    StateCopy<R> sc(c);
    bool fresh = false;   // the float state copy holds the current state
    const double *dtp = c->dscal + SC_DT;     // time step and time of case k at k*kScal
    double *timep = c->dscal + SC_TIME;
    const size_t n3c = c->dm.n3;
    const bool one = c->na == 1;
    for (int loop = 0; loop < 2; loop++) {
        const int ns = loop == 0 ? 5 : 6;
        for (int K = 0; K < ns; K++) {
            double al, be;
            if (loop == 0) { al = alpha1[K]; be = beta1[K]; }
            else if (c->p.rk_mode == 1) { al = alpha2[K]; be = beta2[K]; }
            else { al = 0.0; be = 0.0; }
            const bool first = K == 0;
            double *Q = c->Q, *QW = c->QW;
            R *dQ = Store<R>::dQ(c);
            if (!fresh) ST_TRY(refresh<R>(c, sc, Q, c->Y, false));
            ST_TRY(rhs_t<R>(c, Q, sc.q(Q), dQ, c->Y));
            ST_TRY(hyper_rhs_t<R>(c, Q, dQ, c->Y, sc.y(c->Y)));
            PFOR(c, nc, 5 * io(dQ, Q, Q, QW) + (first ? 0.0 : 5 * io(QW)), {
                double dt = dtp[(one ? 0 : p / n3c) * kScal];
                for (int l = 0; l < 5; l++) {
                    size_t q = l * n3 + p;
                    double qw = first ? dt * dQ[q] : al * QW[q] + dt * dQ[q];
                    QW[q] = qw;
                    Q[q] = Q[q] + be * qw;
                }
            });
            for (int l = 0; l < 5; l++) {
                ST_TRY(dev_filter(c, 0, 0, Q + l * n3, Qf + l * n3));
                ST_TRY(dev_filter(c, 1, 0, Qf + l * n3, Qf + l * n3));
                ST_TRY(dev_filter(c, 2, 0, Qf + l * n3, Q + l * n3));
            }
            if constexpr (is_fp64<R>()) {
                ST_TRY(dev_fix_pressure(c, Q));
            } else {
                ST_TRY(fix_pressure_copy(c, Q, sc.qs));
                fresh = true;
            }
        }
        PFOR(c, (size_t)c->na, io(timep, timep), { timep[p * kScal] = timep[p * kScal] + dtp[p * kScal]; });
    }
    return ST_OK;
}

template <class R>
static int lddrk4_mf(st_ctx *c) {
    static const double alpha1[5] = {0.0, -4.801594388477952e-01, -1.404247195200064e+00,
                                     -2.016477077503357e+00, -1.056444269767207e+00};
    static const double beta1[5] = {1.028639988104959e-01, 7.408540575766301e-01, 7.426530946683799e-01,
                                    4.694937902357905e-01, 1.881733382887932e-01};
    const size_t n3 = c->fs, nc = c->ncell();   // field stride; cells processed
    Scratch rYs(c), Qfs(c, 5);
    double *rY = rYs, *Qf = Qfs;
    StateCopy<R> sc(c);
    bool fresh = false;   // the float state copy holds the current state
    const double *dtp = c->dscal + SC_DT;     // time step and time of case k at k*kScal
    double *timep = c->dscal + SC_TIME;
    const size_t n3c = c->dm.n3;
    const bool one = c->na == 1;
    for (int loop = 0; loop < 2; loop++) {
        for (int K = 0; K < 5; K++) {
            const bool real = loop == 0 || c->p.rk_mode == 1;
            const double al = real ? alpha1[K] : 0.0, be = real ? beta1[K] : 0.0;
            const bool first = K == 0;
            double *Q = c->Q, *QW = c->QW, *Y = c->Y, *rYW = c->rYW;
            R *dQ = Store<R>::dQ(c), *drYi = Store<R>::drYi(c);
            if (!fresh) ST_TRY(refresh<R>(c, sc, Q, Y, true));
            ST_TRY(dev_compute_gamma(c, Y));
            ST_TRY(rhs_t<R>(c, Q, sc.q(Q), dQ, Y));
            ST_TRY(hyper_rhs_t<R>(c, Q, dQ, Y, sc.y(Y)));
            ST_TRY(species_rhs_t<R>(c, Q, sc.q(Q), dQ, Y, sc.y(Y), drYi));
            ST_TRY(bc_rhs_t<R>(c, Q, dQ, Y, drYi));
            ST_TRY(sponge_t<R>(c, Q, dQ, Y, drYi));
            PFOR(c, nc, 5 * io(dQ, Q, Q, QW) + (first ? 0.0 : 5 * io(QW)) + io(Y, drYi, rYW, rY) + (first ? 0.0 : io(rYW)), {
                double dt = dtp[(one ? 0 : p / n3c) * kScal];
                double ry = Q[3 * n3 + p] * Y[p];
                for (int l = 0; l < 5; l++) {
                    size_t q = l * n3 + p;
                    double qw = first ? dt * dQ[q] : al * QW[q] + dt * dQ[q];
                    QW[q] = qw;
                    Q[q] = Q[q] + be * qw;
                }
                double rw = first ? dt * drYi[p] : al * rYW[p] + dt * drYi[p];
                rYW[p] = rw;
                rY[p] = ry + be * rw;
            });
            // Compact_Filter(Q, Qf, 5) then Q = Qf (src/lddrk4_nonperiodic_mf.f:476-481)
            for (int l = 0; l < 5; l++) {
                ST_TRY(dev_filter(c, 0, l == 0, Q + l * n3, Qf + l * n3));
                ST_TRY(dev_filter(c, 1, l == 1, Qf + l * n3, Qf + l * n3));
                ST_TRY(dev_filter(c, 2, l == 2, Qf + l * n3, Q + l * n3));
            }
            ST_TRY(dev_filter(c, 0, 0, rY, rY));
            ST_TRY(dev_filter(c, 1, 0, rY, rY));
            ST_TRY(dev_filter(c, 2, 0, rY, rY));
            // Compute_Y + Fix_Pressure (pproc/pproc_mf.f:190-233); the FP32
            // mode also writes the next stage's float copy of the state
            const double *g = c->gamma_eff;
            float *qs = nullptr, *ys = nullptr;
            if constexpr (!is_fp64<R>()) { qs = sc.qs; ys = sc.ys; fresh = true; }
            PFOR(c, nc, 5 * io(Q) + io(rY, g, Y, Q) + (qs ? 5 * io(qs) + io(ys) : 0.0), {
                double q1 = Q[p], q2 = Q[n3 + p], q3 = Q[2 * n3 + p], q4 = Q[3 * n3 + p];
                double y = rY[p] / q4;
                Y[p] = y;
                double fac1 = g[p] - 1.0;
                double Vs = 1.0 / q4;
                double P = fac1 * (Q[4 * n3 + p] - 5.0e-1 * Vs * (q1 * q1 + q2 * q2 + q3 * q3));
                if (P < 0.0) P = 0.71429;
                double q5 = (1.0 / fac1) * P + 5.0e-1 * Vs * (q1 * q1 + q2 * q2 + q3 * q3);
                Q[4 * n3 + p] = q5;
                if (qs) {
                    qs[p] = (float)q1; qs[n3 + p] = (float)q2; qs[2 * n3 + p] = (float)q3;
                    qs[3 * n3 + p] = (float)q4; qs[4 * n3 + p] = (float)q5;
                    ys[p] = (float)y;
                }
            });
        }
        PFOR(c, (size_t)c->na, io(timep, timep), { timep[p * kScal] = timep[p * kScal] + dtp[p * kScal]; });
    }
    return ST_OK;
}

int dev_lddrk4(st_ctx *c, bool) {
    const bool f32 = fp32_mode(c);
    if (c->p.family == ST_FAMILY_PERIODIC) return f32 ? lddrk4_sf<float>(c) : lddrk4_sf<double>(c);
    return f32 ? lddrk4_mf<float>(c) : lddrk4_mf<double>(c);
}

// monitoring sums (Compute_Mom/KE/Mass/Energy/Entropy), two-pass block sums
// sf: periodic family, whose Compute_Entropy (src/lddrk4_periodic_sf.f:268-300)
// holds gamma - 1 in an undeclared (float32) local and skips Entropy2
__global__ void k_monitor_partial(const double *Q, const double *g, size_t n3c, size_t fs, double *part, int sf) {
    const size_t n3 = fs;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n3c; p += (size_t)gridDim.x * blockDim.x) {
        double q1 = Q[p], q2 = Q[n3 + p], q3 = Q[2 * n3 + p], q4 = Q[3 * n3 + p], q5 = Q[4 * n3 + p];
        double t = 1.0 / q4;
        double ke = 0.0;
        double u1 = q1 * t, u2 = q2 * t, u3 = q3 * t;
        ke = ke + q4 * u1 * u1;
        ke = ke + q4 * u2 * u2;
        ke = ke + q4 * u3 * u3;
        double fac1 = sf ? (double)(float)(g[p] - 1.0) : g[p] - 1.0;
        double Vs = 1.0 / q4;
        double P = fac1 * (q5 - 5.0e-1 * Vs * (q1 * q1 + q2 * q2 + q3 * q3));
        double s1 = q4 * log(P * pow(Vs, g[p]));
        double s2 = sf ? 0.0 : q4 * s1 * s1;
        acc[0] += ke; acc[1] += q1; acc[2] += q2; acc[3] += q3; acc[4] += q4; acc[5] += q5;
        acc[6] += s1; acc[7] += s2;
    }
    __shared__ double sh[8][256];
    for (int k = 0; k < 8; k++) sh[k][threadIdx.x] = acc[k];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            for (int k = 0; k < 8; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 8; k++) part[(size_t)k * gridDim.x + blockIdx.x] = sh[k][0];
}

int dev_monitors(st_ctx *c) {
    const int nb = 256;
    Scratch parts(c);   // >= 8*nb doubles for every supported grid (n3 >= 32^3)
    double *part = parts;
    c->launches++;
    k_monitor_partial<<<nb, 256, 0, c->stream>>>(c->Q, c->gamma_eff, c->dm.n3, c->fs, part,
                                                 c->p.family == ST_FAMILY_PERIODIC ? 1 : 0);
    ST_CUDA(c, cudaGetLastError());
    std::vector<double> h(8 * nb);
    ST_CUDA(c, cudaMemcpyAsync(h.data(), part, 8 * nb * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    ST_CUDA(c, cudaStreamSynchronize(c->stream));
    double s[8] = {0};
    for (int k = 0; k < 8; k++) for (int b = 0; b < nb; b++) s[k] += h[(size_t)k * nb + b];
    const double N = (double)(c->dm.n[0] * c->dm.n[1] * c->dm.n[2]);
    c->mon[0] = 0.5 * s[0] / N;
    for (int k = 1; k < 8; k++) c->mon[k] = s[k] / N;
    return ST_OK;
}

}  // namespace st
