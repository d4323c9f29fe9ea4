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
template <class Fn>
__global__ void k_pfor(size_t n, Fn fn) {
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
        fn(p);
}
template <class Fn>
static int pfor(st_ctx *c, size_t n, Fn fn) {
    size_t blocks = (n + 255) / 256;
    if (blocks > 148 * 32) blocks = 148 * 32;
    if (blocks == 0) return ST_OK;
    int pi = prof_start(c, "k_pointwise", 0.0);
    k_pfor<<<(unsigned)blocks, 256, 0, c->stream>>>(n, fn);
    prof_stop(c, pi);
    ST_CUDA(c, cudaGetLastError());
    return ST_OK;
}
#define PFOR(c, n, ...) ST_TRY(pfor((c), (n), [=] __device__(size_t p) __VA_ARGS__))

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

// contiguous multi-field scratch (n fields)
struct ScratchN {
    st_ctx *c; std::vector<double *> f;
    ScratchN(st_ctx *cc, int n) : c(cc) { for (int i = 0; i < n; i++) f.push_back(scratch(cc)); }
    ~ScratchN() { for (double *p : f) release(c, p); }
    double *operator[](int i) const { return f[i]; }
};

int dev_compute_gamma(st_ctx *c, const double *Y) {
    Phys f = phys(c);
    double *ge = c->gamma_eff;
    PFOR(c, c->dm.n3, {
        double fac1 = f.g1 - 1.0, fac2 = f.g2 - 1.0;
        double num = (Y[p] * f.g1 / fac1) + (f.eps * (1.0 - Y[p]) * f.g2 / fac2);
        double den = (Y[p] / fac1) + (f.eps * (1.0 - Y[p]) / fac2);
        ge[p] = num / den;
    });
    return ST_OK;
}

// ---- RHS_x (src/rhsv_sym_mf.f:37-481); Q is the copy Ux --------------------
static int rhs_x(st_ctx *c, double *Q, double *Qrhs, const double *Y, double *Qcx, double *Qcy, double *Qcz,
                 double *Qv) {
    const size_t n3 = c->dm.n3;
    Phys f = phys(c);
    double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    Scratch P(c), Vs(c), T(c), FF(c), Flux(c), dF(c);
    double *pP = P, *pVs = Vs, *pT = T, *pFF = FF, *pFl = Flux, *pdF = dF;
    ST_CUDA(c, cudaMemsetAsync(Qrhs, 0, 5 * n3 * 8, c->stream));
    ST_CUDA(c, cudaMemsetAsync(Qcx, 0, 5 * n3 * 8, c->stream));
    ST_CUDA(c, cudaMemsetAsync(Qcy, 0, 5 * n3 * 8, c->stream));
    ST_CUDA(c, cudaMemsetAsync(Qcz, 0, 5 * n3 * 8, c->stream));
    ST_CUDA(c, cudaMemsetAsync(Qv, 0, 5 * n3 * 8, c->stream));
    const double *g = c->gamma_eff;
    PFOR(c, n3, {
        thermo(f, g[p], Y[p], Q1[p], Q2[p], Q3[p], Q4[p], Q5[p], pVs[p], pP[p], pT[p]);
        pdF[p] = Q1[p] * pVs[p];
        pFF[p] = pdF[p];
        pFl[p] = Q4[p] * pFF[p];
    });
    ST_TRY(dev_dfd(c, 0, 1, pFl, Qcx + 3 * n3, 1, -1.0));
    PFOR(c, n3, { pFl[p] = (Q5[p] + pP[p]) * pFF[p]; });
    ST_TRY(dev_dfd(c, 0, 1, pFl, Qcx + 4 * n3, 1, -1.0));
    PFOR(c, n3, { pFF[p] = pdF[p]; pFl[p] = Q1[p] * pFF[p]; });
    ST_TRY(dev_dfd(c, 0, 0, pFl, Qcx, 1, -5.0e-1));
    ST_TRY(dev_dfd(c, 0, 0, pP, Qcx, 1, -1.0));
    PFOR(c, n3, { pFl[p] = Q2[p] * pFF[p]; });
    ST_TRY(dev_dfd(c, 0, 1, pFl, Qcx + n3, 1, -5.0e-1));
    PFOR(c, n3, { pFl[p] = Q3[p] * pFF[p]; });
    ST_TRY(dev_dfd(c, 0, 1, pFl, Qcx + 2 * n3, 1, -5.0e-1));
    ST_TRY(dev_dfd(c, 0, 1, Q1, pFF, 0, 1.0));
    PFOR(c, n3, {
        double mu, dmu;
        Q1[p] = pdF[p];
        Q2[p] = Q2[p] * pVs[p];
        Q3[p] = Q3[p] * pVs[p];
        viscosity(f, pT[p], Y[p], mu, dmu);
        Q5[p] = mu;
        pFl[p] = dmu;
        double fac2 = -5.0e-1 * pFF[p];
        Qcx[p] = Qcx[p] + fac2 * Q1[p];
        Qcx[n3 + p] = Qcx[n3 + p] + fac2 * Q2[p];
        Qcx[2 * n3 + p] = Qcx[2 * n3 + p] + fac2 * Q3[p];
    });
    ST_TRY(dev_d2fd2(c, 0, 0, pT, pFF, pdF, 1));
    ST_CUDA(c, cudaMemcpyAsync(c->grad[G_DTDX], pFF, n3 * 8, cudaMemcpyDeviceToDevice, c->stream));
    {
        double fac1 = f.Pr_inv;
        PFOR(c, n3, { Qv[4 * n3 + p] = Qv[4 * n3 + p] + fac1 * (Q5[p] * pdF[p] + pFl[p] * pFF[p] * pFF[p]); });
    }
    ST_TRY(dev_d2fd2(c, 0, 1, Q1, pFl, pdF, 1));
    ST_CUDA(c, cudaMemcpyAsync(c->grad[G_DUX_DX], pFl, n3 * 8, cudaMemcpyDeviceToDevice, c->stream));
    {
        double fac1 = 4.0 / 3.0 + f.bulk;
        PFOR(c, n3, {
            double fac2 = fac1 * Q5[p] * pdF[p];
            Qv[p] = Qv[p] + fac2;
            Qv[4 * n3 + p] = Qv[4 * n3 + p] + Q1[p] * fac2;
        });
    }
    ST_TRY(dev_d2fd2(c, 0, 0, Q2, pT, pdF, 1));
    ST_CUDA(c, cudaMemcpyAsync(c->grad[G_DUY_DX], pT, n3 * 8, cudaMemcpyDeviceToDevice, c->stream));
    PFOR(c, n3, {
        double fac2 = Q5[p] * pdF[p];
        Qv[n3 + p] = Qv[n3 + p] + fac2;
        Qv[4 * n3 + p] = Qv[4 * n3 + p] + Q2[p] * fac2;
        Q2[p] = pT[p];
    });
    ST_TRY(dev_d2fd2(c, 0, 0, Q3, pVs, pdF, 1));
    ST_CUDA(c, cudaMemcpyAsync(c->grad[G_DUZ_DX], pVs, n3 * 8, cudaMemcpyDeviceToDevice, c->stream));
    PFOR(c, n3, {
        double fac2 = Q5[p] * pdF[p];
        Qv[2 * n3 + p] = Qv[2 * n3 + p] + fac2;
        Qv[4 * n3 + p] = Qv[4 * n3 + p] + Q3[p] * fac2;
        Q3[p] = pVs[p];
    });
    PFOR(c, n3, {
        double fac2 = -5.0e-1 * Q4[p] * Q1[p];
        Q1[p] = pFl[p];
        Q4[p] = pFF[p];
        Qcx[p] = Qcx[p] + fac2 * Q1[p];
        Qcx[n3 + p] = Qcx[n3 + p] + fac2 * Q2[p];
        Qcx[2 * n3 + p] = Qcx[2 * n3 + p] + fac2 * Q3[p];
    });
    return ST_OK;
}

// ---- RHS_yz (src/rhsv_sym_mf.f:492-1428) ---------------------------------
static int rhs_yz(st_ctx *c, double *Q, double *Ux, double *Qrhs, const double *Y, double *Qcx, double *Qcy,
                  double *Qcz, double *Qv) {
    const size_t n3 = c->dm.n3;
    Phys f = phys(c);
    double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    double *U1 = Ux, *U2 = Ux + n3, *U3 = Ux + 2 * n3, *U4 = Ux + 3 * n3, *U5 = Ux + 4 * n3;
    ScratchN s(c, 12);
    double *P = s[0], *Vs = s[1], *T = s[2], *vis = s[3], *dF = s[4], *Flux = s[5];
    double *Tdy = s[6], *Tdz = s[7], *Udz = s[8], *dFz = s[9], *Udx = s[10], *Udy = s[11];
    const double *g = c->gamma_eff;
    double **G = c->grad;
    PFOR(c, n3, {
        thermo(f, g[p], Y[p], Q1[p], Q2[p], Q3[p], Q4[p], Q5[p], Vs[p], P[p], T[p]);
        U5[p] = Q2[p] * Vs[p];
        Flux[p] = Q1[p] * U5[p];
    });
    ST_TRY(dev_dfd(c, 1, 1, Q2, dF, 0, 1.0));
    PFOR(c, n3, { Qcy[3 * n3 + p] = Qcy[3 * n3 + p] - dF[p]; });
    ST_TRY(dev_dfd(c, 1, 1, Flux, Qcy, 1, -5.0e-1));
    PFOR(c, n3, { Flux[p] = Q2[p] * U5[p]; });
    ST_TRY(dev_dfd(c, 1, 0, Flux, Qcy + n3, 1, -5.0e-1));
    ST_TRY(dev_dfd(c, 1, 0, P, Qcy + n3, 1, -1.0));
    PFOR(c, n3, { Flux[p] = Q3[p] * U5[p]; });
    ST_TRY(dev_dfd(c, 1, 1, Flux, Qcy + 2 * n3, 1, -5.0e-1));
    PFOR(c, n3, { Flux[p] = (Q5[p] + P[p]) * U5[p]; });
    ST_TRY(dev_dfd(c, 1, 1, Flux, Qcy + 4 * n3, 1, -1.0));
    ST_TRY(dev_dfd(c, 2, 1, Q3, dFz, 0, 1.0));
    PFOR(c, n3, {
        Qcz[3 * n3 + p] = Qcz[3 * n3 + p] - dFz[p];
        U5[p] = Q3[p] * Vs[p];
        Flux[p] = Q1[p] * U5[p];
    });
    ST_TRY(dev_dfd(c, 2, 1, Flux, Qcz, 1, -5.0e-1));
    PFOR(c, n3, { Flux[p] = Q2[p] * U5[p]; });
    ST_TRY(dev_dfd(c, 2, 1, Flux, Qcz + n3, 1, -5.0e-1));
    PFOR(c, n3, { Flux[p] = Q3[p] * U5[p]; });
    ST_TRY(dev_dfd(c, 2, 0, Flux, Qcz + 2 * n3, 1, -5.0e-1));
    ST_TRY(dev_dfd(c, 2, 0, P, Qcz + 2 * n3, 1, -1.0));
    PFOR(c, n3, { Flux[p] = (Q5[p] + P[p]) * U5[p]; });
    ST_TRY(dev_dfd(c, 2, 1, Flux, Qcz + 4 * n3, 1, -1.0));
    PFOR(c, n3, {
        Q1[p] = Q1[p] * Vs[p];
        Q2[p] = Q2[p] * Vs[p];
        Q3[p] = Q3[p] * Vs[p];
        double fac2 = -5.0e-1 * dF[p];
        Qcy[p] = Qcy[p] + fac2 * Q1[p];
        Qcy[n3 + p] = Qcy[n3 + p] + fac2 * Q2[p];
        Qcy[2 * n3 + p] = Qcy[2 * n3 + p] + fac2 * Q3[p];
        fac2 = -5.0e-1 * dFz[p];
        Qcz[p] = Qcz[p] + fac2 * Q1[p];
        Qcz[n3 + p] = Qcz[n3 + p] + fac2 * Q2[p];
        Qcz[2 * n3 + p] = Qcz[2 * n3 + p] + fac2 * Q3[p];
    });
    ST_TRY(dev_d2fd2(c, 1, 0, T, Tdy, U5, 1));
    ST_CUDA(c, cudaMemcpyAsync(G[G_DTDY], Tdy, n3 * 8, cudaMemcpyDeviceToDevice, c->stream));
    ST_TRY(dev_d2fd2(c, 2, 0, T, Tdz, Flux, 1));
    ST_CUDA(c, cudaMemcpyAsync(G[G_DTDZ], Tdz, n3 * 8, cudaMemcpyDeviceToDevice, c->stream));
    {
        double fac2 = f.Pr_inv;
        PFOR(c, n3, {
            viscosity(f, T[p], Y[p], vis[p], Udz[p]);
            Qv[4 * n3 + p] = Qv[4 * n3 + p] + fac2 * (vis[p] * (U5[p] + Flux[p]) +
                                                      Udz[p] * (Tdy[p] * Tdy[p] + Tdz[p] * Tdz[p]));
            U4[p] = Udz[p] * U4[p];
            Tdy[p] = Udz[p] * Tdy[p];
            Tdz[p] = Udz[p] * Tdz[p];
        });
    }
    // d(rho)/dy into Udz: computed by the reference and overwritten before use
    ST_TRY(dev_dfd(c, 1, 0, Q4, Udz, 0, 1.0));
    ST_TRY(dev_d2fd2(c, 1, 0, Q1, P, U5, 1));
    ST_CUDA(c, cudaMemcpyAsync(G[G_DUX_DY], P, n3 * 8, cudaMemcpyDeviceToDevice, c->stream));
    ST_TRY(dev_d2fd2(c, 1, 1, Q2, Flux, dF, 1));
    ST_CUDA(c, cudaMemcpyAsync(G[G_DUY_DY], Flux, n3 * 8, cudaMemcpyDeviceToDevice, c->stream));
    ST_TRY(dev_d2fd2(c, 1, 0, Q3, Udz, T, 1));
    ST_CUDA(c, cudaMemcpyAsync(G[G_DUZ_DY], Udz, n3 * 8, cudaMemcpyDeviceToDevice, c->stream));
    ST_TRY(dev_dfd(c, 2, 0, Q1, Udx, 0, 1.0));
    ST_CUDA(c, cudaMemcpyAsync(G[G_DUX_DZ], Udx, n3 * 8, cudaMemcpyDeviceToDevice, c->stream));
    ST_TRY(dev_dfd(c, 2, 0, Q2, Udy, 0, 1.0));
    ST_CUDA(c, cudaMemcpyAsync(G[G_DUY_DZ], Udy, n3 * 8, cudaMemcpyDeviceToDevice, c->stream));
    ST_TRY(dev_dfd(c, 2, 1, Q3, dFz, 0, 1.0));
    ST_CUDA(c, cudaMemcpyAsync(G[G_DUZ_DZ], dFz, n3 * 8, cudaMemcpyDeviceToDevice, c->stream));
    {
        double fac1 = f.bulk + 4.0 / 3.0;
        PFOR(c, n3, {
            double fac2 = -5.0e-1 * Q4[p] * Q2[p];
            Qcy[p] = Qcy[p] + fac2 * P[p];
            Qcy[n3 + p] = Qcy[n3 + p] + fac2 * Flux[p];
            Qcy[2 * n3 + p] = Qcy[2 * n3 + p] + fac2 * Udz[p];
            fac2 = -5.0e-1 * Q4[p] * Q3[p];
            Qcz[p] = Qcz[p] + fac2 * Udx[p];
            Qcz[n3 + p] = Qcz[n3 + p] + fac2 * Udy[p];
            Qcz[2 * n3 + p] = Qcz[2 * n3 + p] + fac2 * dFz[p];
            double fac_X = vis[p] * U5[p];
            double fac_Y = fac1 * vis[p] * dF[p];
            double fac_Z = vis[p] * T[p];
            Qv[p] = Qv[p] + fac_X;
            Qv[n3 + p] = Qv[n3 + p] + fac_Y;
            Qv[2 * n3 + p] = Qv[2 * n3 + p] + fac_Z;
            Qv[4 * n3 + p] = Qv[4 * n3 + p] + Q1[p] * fac_X + Q2[p] * fac_Y + Q3[p] * fac_Z;
        });
    }
    ST_TRY(dev_d2fd2(c, 2, 1, Q3, dF, T, 0));
    ST_CUDA(c, cudaMemcpyAsync(dF, G[G_DUZ_DZ], n3 * 8, cudaMemcpyDeviceToDevice, c->stream));
    ST_TRY(dev_dfd(c, 1, 0, dF, U5, 0, 1.0));
    const double fac1 = f.bulk - 2.0 / 3.0, fac2 = f.bulk + 4.0 / 3.0, fac3 = f.bulk + 1.0 / 3.0;
    PFOR(c, n3, {
        double tmp1 = U1[p];
        double dil = tmp1 + Flux[p] + dF[p];
        double fac_X = U4[p] * (2.0 * tmp1 + fac1 * dil);
        double fac_Y = Tdy[p] * (2.0 * Flux[p] + fac1 * dil) + fac3 * vis[p] * U5[p];
        double fac_Z = Tdz[p] * (2.0 * dF[p] + fac1 * dil) + fac2 * vis[p] * T[p];
        Qv[p] = Qv[p] + fac_X;
        Qv[n3 + p] = Qv[n3 + p] + fac_Y;
        Qv[2 * n3 + p] = Qv[2 * n3 + p] + fac_Z;
        Qv[4 * n3 + p] = Qv[4 * n3 + p] + Q1[p] * fac_X + Q2[p] * fac_Y + Q3[p] * fac_Z +
                         vis[p] * (2.0 * (tmp1 * tmp1 + Flux[p] * Flux[p] + dF[p] * dF[p]) + fac1 * dil * dil);
    });
    ST_TRY(dev_d2fd2(c, 2, 0, Q1, T, dF, 0));
    ST_CUDA(c, cudaMemcpyAsync(T, G[G_DUX_DZ], n3 * 8, cudaMemcpyDeviceToDevice, c->stream));
    ST_TRY(dev_d2fd2(c, 2, 0, Q2, Flux, U5, 0));
    ST_CUDA(c, cudaMemcpyAsync(Flux, G[G_DUY_DZ], n3 * 8, cudaMemcpyDeviceToDevice, c->stream));
    PFOR(c, n3, {
        double tmp1 = U2[p] + P[p];
        double tmp2 = U3[p] + T[p];
        double tmp3 = Udz[p] + Flux[p];
        double fac_X = Tdy[p] * tmp1 + Tdz[p] * tmp2 + vis[p] * dF[p];
        double fac_Y = U4[p] * tmp1 + Tdz[p] * tmp3 + vis[p] * U5[p];
        double fac_Z = U4[p] * tmp2 + Tdy[p] * tmp3;
        Qv[p] = Qv[p] + fac_X;
        Qv[n3 + p] = Qv[n3 + p] + fac_Y;
        Qv[2 * n3 + p] = Qv[2 * n3 + p] + fac_Z;
        Qv[4 * n3 + p] = Qv[4 * n3 + p] + Q1[p] * fac_X + Q2[p] * fac_Y + Q3[p] * fac_Z +
                         vis[p] * (tmp1 * tmp1 + tmp2 * tmp2 + tmp3 * tmp3);
    });
    ST_TRY(dev_dfd(c, 1, 0, U1, U4, 0, 1.0));
    ST_TRY(dev_dfd(c, 2, 0, U1, U5, 0, 1.0));
    ST_TRY(dev_dfd(c, 1, 1, U2, Tdy, 0, 1.0));
    ST_TRY(dev_dfd(c, 2, 1, U3, Tdz, 0, 1.0));
    ST_TRY(dev_dfd(c, 1, 1, Flux, T, 0, 1.0));
    const bool add_visc = c->p.re > 0.0;
    PFOR(c, n3, {
        double fac_X = fac3 * vis[p] * (Tdy[p] + Tdz[p]);
        double fac_Y = fac3 * vis[p] * U4[p];
        double fac_Z = fac3 * vis[p] * (U5[p] + T[p]);
        Qv[p] = Qv[p] + fac_X;
        Qv[n3 + p] = Qv[n3 + p] + fac_Y;
        Qv[2 * n3 + p] = Qv[2 * n3 + p] + fac_Z;
        Qv[4 * n3 + p] = Qv[4 * n3 + p] + Q1[p] * fac_X + Q2[p] * fac_Y + Q3[p] * fac_Z;
        Q1[p] = Q1[p] * Q4[p];
        Q2[p] = Q2[p] * Q4[p];
        Q3[p] = Q3[p] * Q4[p];
        for (int l = 0; l < 5; l++) {
            size_t q = l * n3 + p;
            if (add_visc) Qrhs[q] = Qrhs[q] + Qcx[q] + Qcy[q] + Qcz[q] + Qv[q];
            else Qrhs[q] = Qrhs[q] + Qcx[q] + Qcy[q] + Qcz[q];
        }
    });
    return ST_OK;
}

int dev_rhs(st_ctx *c, double *Q, double *Qrhs, const double *Y) {
    const size_t n3 = c->dm.n3;
    Scratch Ux(c, 5), Qcx(c, 5), Qcy(c, 5), Qcz(c, 5), Qv(c, 5);
    ST_CUDA(c, cudaMemcpyAsync(Ux, Q, 5 * n3 * 8, cudaMemcpyDeviceToDevice, c->stream));
    ST_TRY(rhs_x(c, Ux, Qrhs, Y, Qcx, Qcy, Qcz, Qv));
    return rhs_yz(c, Q, Ux, Qrhs, Y, Qcx, Qcy, Qcz, Qv);
}

// ---- artificial viscosity -----------------------------------------------------
// Compute_Laplacian src/hyper_dynamic_sym_mf.f:41-65
static int laplacian(st_ctx *c, const double *S, double *d2S) {
    Scratch dS(c), t1(c), t2(c);
    double *pt1 = t1, *pt2 = t2;
    ST_TRY(dev_dfd(c, 0, 0, S, dS, 0, 1.0));
    ST_TRY(dev_dfd(c, 0, 1, dS, t1, 0, 1.0));
    ST_TRY(dev_dfd(c, 1, 0, S, dS, 0, 1.0));
    ST_TRY(dev_dfd(c, 1, 1, dS, t2, 0, 1.0));
    ST_TRY(dev_dfd(c, 2, 0, S, dS, 0, 1.0));
    ST_TRY(dev_dfd(c, 2, 1, dS, d2S, 0, 1.0));
    PFOR(c, c->dm.n3, { d2S[p] = d2S[p] + pt1[p] + pt2[p]; });
    return ST_OK;
}

// Compute_hyper src/hyper_dynamic_sym_mf.f:166-334 (+ Compute_coeff1 :79-158,
// Compute_Contraction :12-33)
int dev_compute_hyper(st_ctx *c, const double *Q, const double *Y) {
    const size_t n3 = c->dm.n3;
    Phys f = phys(c);
    const double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    ScratchN s(c, 10);
    double *Cbeta = s[0], *S = s[1], *e = s[2], *P = s[3], *T = s[4], *Vs = s[5], *d2 = s[6];
    double *d4S = s[7], *d4e = s[8], *d4Y = s[9];
    Scratch etas(c, 10);
    double *eta = etas, *etag = eta + 5 * n3;
    const double *g = c->gamma_eff;
    const double *G0 = c->grad[0], *G1 = c->grad[1], *G2 = c->grad[2], *G3 = c->grad[3], *G4 = c->grad[4],
                 *G5 = c->grad[5], *G6 = c->grad[6], *G7 = c->grad[7], *G8 = c->grad[8];
    const double scale = c->p.c_beta_scale;
    {
        PFOR(c, n3, {
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
            Vs[p] = 1.0 / Q4[p];
            P[p] = fac1 * (Q5[p] - 5.0e-1 * Vs[p] * (Q1[p] * Q1[p] + Q2[p] * Q2[p] + Q3[p] * Q3[p]));
            T[p] = fac3 * Vs[p] * P[p];
            e[p] = Vs[p] * (Q5[p] - 5.0e-1 * Vs[p] * (Q1[p] * Q1[p] + Q2[p] * Q2[p] + Q3[p] * Q3[p]));
            S[p] = sqrt(5.0e-1 * (s1 * s1 + s5 * s5 + s9 * s9 + 2.0 * (s2 * s4 + s3 * s7 + s6 * s8)));
        });
        ST_TRY(laplacian(c, S, d2));
        ST_TRY(laplacian(c, d2, d4S));
        ST_TRY(laplacian(c, e, d2));
        ST_TRY(laplacian(c, d2, d4e));
        ST_TRY(laplacian(c, Y, d2));
        ST_TRY(laplacian(c, d2, d4Y));
        const double C_mu = 2.0e-3, C_k = 1.0e-2;
        PFOR(c, n3, {
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
        ST_TRY(dev_gaussian_filter(c, eta, etag, 5));
        const double DX6 = pow(c->DX, 6.0), DX5 = pow(c->DX, 5.0), DX = c->DX;
        const double C_D = 1.0e-4, C_Y = 100.0;
        double *hb = c->hyp[H_BETA], *hv = c->hyp[H_VISC], *hk = c->hyp[H_K], *hd = c->hyp[H_D];
        PFOR(c, n3, {
            hb[p] = etag[2 * n3 + p] * DX6;
            hv[p] = etag[p] * DX6;
            hk[p] = etag[n3 + p] * DX5;
            hd[p] = C_D * etag[4 * n3 + p] * DX5 + C_Y * etag[3 * n3 + p] * DX;
        });
    }
    return ST_OK;
}

// Hyper_RHS src/hyper_rhs_sym_mf.f:12-500
int dev_hyper_rhs(st_ctx *c, const double *Q, double *Qrhs, const double *Y) {
    if (c->p.hyper_param == 0) return ST_OK;
    const size_t n3 = c->dm.n3;
    ST_TRY(dev_compute_hyper(c, Q, Y));
    const double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3;
    ScratchN s(c, 16);
    double *U1 = s[0], *U2 = s[1], *U3 = s[2], *dila = s[3], *S1 = s[4], *S2 = s[5], *S3 = s[6];
    double *Flux = s[7], *FF = s[8], *dFx = s[9], *dFy = s[10], *dFz = s[11], *dEx = s[12], *dEy = s[13],
           *dEz = s[14];
    Scratch Qhs(c, 5);
    double *Qh = Qhs;
    ST_CUDA(c, cudaMemsetAsync(Qh, 0, 5 * n3 * 8, c->stream));
    const double *G0 = c->grad[0], *G1 = c->grad[1], *G2 = c->grad[2], *G3 = c->grad[3], *G4 = c->grad[4],
                 *G5 = c->grad[5], *G6 = c->grad[6], *G7 = c->grad[7], *G8 = c->grad[8];
    const double *GTx = c->grad[G_DTDX], *GTy = c->grad[G_DTDY], *GTz = c->grad[G_DTDZ];
    const double *vh = c->hyp[H_VISC], *bh = c->hyp[H_BETA], *kh = c->hyp[H_K];
    {
        PFOR(c, n3, {
            U1[p] = Q1[p] / Q4[p];
            U2[p] = Q2[p] / Q4[p];
            U3[p] = Q3[p] / Q4[p];
            dila[p] = G0[p] + G4[p] + G8[p];
            S1[p] = G3[p] + G1[p];
            S2[p] = G6[p] + G2[p];
            S3[p] = G7[p] + G5[p];
        });
        double *h1 = Qh, *h2 = Qh + n3, *h3 = Qh + 2 * n3, *h5 = Qh + 4 * n3;
        // x momentum
        PFOR(c, n3, {
            Flux[p] = 2.0 * vh[p] * G0[p] + (bh[p] - (2.0 / 3.0) * vh[p]) * dila[p];
            FF[p] = U1[p] * Flux[p];
        });
        ST_TRY(dev_dfd(c, 0, 0, Flux, dFx, 0, 1.0));
        ST_TRY(dev_dfd(c, 0, 1, FF, dEx, 0, 1.0));
        PFOR(c, n3, { Flux[p] = vh[p] * S1[p]; FF[p] = U1[p] * Flux[p]; });
        ST_TRY(dev_dfd(c, 1, 1, Flux, dFy, 0, 1.0));
        ST_TRY(dev_dfd(c, 1, 1, FF, dEy, 0, 1.0));
        PFOR(c, n3, { Flux[p] = vh[p] * S2[p]; FF[p] = U1[p] * Flux[p]; });
        ST_TRY(dev_dfd(c, 2, 1, Flux, dFz, 0, 1.0));
        ST_TRY(dev_dfd(c, 2, 1, FF, dEz, 0, 1.0));
        PFOR(c, n3, {
            h1[p] = h1[p] + dFx[p] + dFy[p] + dFz[p];
            h5[p] = h5[p] + dEx[p] + dEy[p] + dEz[p];
        });
        // y momentum
        PFOR(c, n3, {
            Flux[p] = 2.0 * vh[p] * G4[p] + (bh[p] - (2.0 / 3.0) * vh[p]) * dila[p];
            FF[p] = U2[p] * Flux[p];
        });
        ST_TRY(dev_dfd(c, 1, 0, Flux, dFy, 0, 1.0));
        ST_TRY(dev_dfd(c, 1, 1, FF, dEy, 0, 1.0));
        PFOR(c, n3, { Flux[p] = vh[p] * S1[p]; FF[p] = U2[p] * Flux[p]; });
        ST_TRY(dev_dfd(c, 0, 1, Flux, dFx, 0, 1.0));
        ST_TRY(dev_dfd(c, 0, 1, FF, dEx, 0, 1.0));
        PFOR(c, n3, { Flux[p] = vh[p] * S3[p]; FF[p] = U2[p] * Flux[p]; });
        ST_TRY(dev_dfd(c, 2, 1, Flux, dFz, 0, 1.0));
        ST_TRY(dev_dfd(c, 2, 1, FF, dEz, 0, 1.0));
        PFOR(c, n3, {
            h2[p] = h2[p] + dFx[p] + dFy[p] + dFz[p];
            h5[p] = h5[p] + dEx[p] + dEy[p] + dEz[p];
        });
        // z momentum
        PFOR(c, n3, {
            Flux[p] = 2.0 * vh[p] * G8[p] + (bh[p] - (2.0 / 3.0) * vh[p]) * dila[p];
            FF[p] = U3[p] * Flux[p];
        });
        ST_TRY(dev_dfd(c, 2, 0, Flux, dFz, 0, 1.0));
        ST_TRY(dev_dfd(c, 2, 1, FF, dEz, 0, 1.0));
        PFOR(c, n3, { Flux[p] = vh[p] * S2[p]; FF[p] = U3[p] * Flux[p]; });
        ST_TRY(dev_dfd(c, 0, 1, Flux, dFx, 0, 1.0));
        ST_TRY(dev_dfd(c, 0, 1, FF, dEx, 0, 1.0));
        PFOR(c, n3, { Flux[p] = vh[p] * S3[p]; FF[p] = U3[p] * Flux[p]; });
        ST_TRY(dev_dfd(c, 1, 1, Flux, dFy, 0, 1.0));
        ST_TRY(dev_dfd(c, 1, 1, FF, dEy, 0, 1.0));
        PFOR(c, n3, {
            h3[p] = h3[p] + dFx[p] + dFy[p] + dFz[p];
            h5[p] = h5[p] + dEx[p] + dEy[p] + dEz[p];
        });
        // artificial heat flux
        PFOR(c, n3, { Flux[p] = kh[p] * GTx[p]; });
        ST_TRY(dev_dfd(c, 0, 0, Flux, dFx, 0, 1.0));
        PFOR(c, n3, { FF[p] = kh[p] * GTy[p]; });
        ST_TRY(dev_dfd(c, 1, 0, FF, dFy, 0, 1.0));
        PFOR(c, n3, { Flux[p] = kh[p] * GTz[p]; });
        ST_TRY(dev_dfd(c, 2, 0, Flux, dFz, 0, 1.0));
        PFOR(c, n3, {
            h5[p] = h5[p] + dFx[p] + dFy[p] + dFz[p];
            for (int l = 0; l < 5; l++) Qrhs[l * n3 + p] = Qrhs[l * n3 + p] + Qh[l * n3 + p];
        });
    }
    return ST_OK;
}

// Species_RHS src/species_rhs_sym.f:9-207
int dev_species_rhs(st_ctx *c, const double *Q, double *Qrhs, const double *Y, double *Yrhs) {
    if (c->p.hyper_param == 0) return ST_OK;
    const size_t n3 = c->dm.n3;
    Phys f = phys(c);
    const double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    ScratchN s(c, 7);
    double *Ycx = s[0], *Ycy = s[1], *Ycz = s[2], *Yd = s[3], *Flux = s[4], *FF = s[5], *T = s[6];
    const double *Dh = c->hyp[H_D];
    const double *g = c->gamma_eff;
    PFOR(c, n3, {
        double Vs, P, Tt;
        thermo(f, g[p], Y[p], Q1[p], Q2[p], Q3[p], Q4[p], Q5[p], Vs, P, Tt);
        T[p] = Tt;
        Yrhs[p] = 0.0; Ycx[p] = 0.0; Ycy[p] = 0.0; Ycz[p] = 0.0; Yd[p] = 0.0;
    });
    ST_TRY(dev_dfd(c, 0, 0, Y, c->dYd[0], 0, 1.0));
    ST_TRY(dev_dfd(c, 1, 0, Y, c->dYd[1], 0, 1.0));
    ST_TRY(dev_dfd(c, 2, 0, Y, c->dYd[2], 0, 1.0));
    PFOR(c, n3, { Flux[p] = Q1[p] * Y[p]; });
    ST_TRY(dev_dfd(c, 0, 1, Flux, Ycx, 1, -1.0));
    PFOR(c, n3, { Flux[p] = Q2[p] * Y[p]; });
    ST_TRY(dev_dfd(c, 1, 1, Flux, Ycy, 1, -1.0));
    PFOR(c, n3, { Flux[p] = Q3[p] * Y[p]; });
    ST_TRY(dev_dfd(c, 2, 1, Flux, Ycz, 1, -1.0));
    const double cst0 = f.eps * f.g2 * (f.g1 - 1.0) / (f.g1 * (f.g2 - 1.0));
    const double Re1i = f.Re1_inv, Sci = f.Sc_inv;
    for (int d = 0; d < 3; d++) {
        const double *dY = c->dYd[d];
        PFOR(c, n3, {
            Flux[p] = Q4[p] * Dh[p] * dY[p] + Q4[p] * dY[p] * Re1i * Sci;
            FF[p] = (1.0 - cst0) * T[p] * Flux[p];
        });
        ST_TRY(dev_dfd(c, d, 1, Flux, Yd, 1, 1.0));
        ST_TRY(dev_dfd(c, d, 1, FF, Qrhs + 4 * n3, 1, 1.0));
    }
    PFOR(c, n3, { Yrhs[p] = Ycx[p] + Ycy[p] + Ycz[p] + Yd[p]; });
    return ST_OK;
}

// bc_RHS src/bc_mf.f:11-463 (active face blocks)
int dev_bc_rhs(st_ctx *c, double *Q, double *Qrhs, const double *Y, double *Yrhs) {
    const size_t n3 = c->dm.n3;
    const int Mx = c->dm.n[0], My = c->dm.n[1], Mz = c->dm.n[2];
    Phys f = phys(c);
    double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    const double *g = c->gamma_eff;
    // symmetry planes: x=0 (rho u), z=0 (rho w), y=0 (rho v)
    PFOR(c, n3, {
        size_t j = p % My, k = (p / My) % Mz, i = p / ((size_t)My * Mz);
        if (i == 0) Q1[p] = 0.0;
        if (k == 0) Q3[p] = 0.0;
        if (j == 0) Q2[p] = 0.0;
    });
    ScratchN s(c, 4);
    double *P = s[0], *dPx = s[1], *dPy = s[2], *dPz = s[3];
    PFOR(c, n3, {
        double Vs, Pp, T;
        thermo(f, g[p], Y[p], Q1[p], Q2[p], Q3[p], Q4[p], Q5[p], Vs, Pp, T);
        P[p] = Pp;
    });
    ST_TRY(dev_dfd(c, 0, 0, P, dPx, 0, 1.0));
    ST_TRY(dev_dfd(c, 1, 0, P, dPy, 0, 1.0));
    ST_TRY(dev_dfd(c, 2, 0, P, dPz, 0, 1.0));
    const double *Gxx = c->grad[G_DUX_DX], *Gyy = c->grad[G_DUY_DY], *Gzz = c->grad[G_DUZ_DZ];
    // faces in the reference order x, y, z (later faces overwrite edges)
    for (int face = 0; face < 3; face++) {
        size_t nf = face == 0 ? (size_t)My * Mz : face == 1 ? (size_t)Mx * Mz : (size_t)Mx * My;
        PFOR(c, nf, {
            size_t q;
            if (face == 0) q = p + (size_t)My * Mz * (Mx - 1);                    // p = j + My*k
            else if (face == 1) q = (My - 1) + (size_t)My * p;                    // p = k + Mz*i
            else q = (p % My) + (size_t)My * (Mz - 1) + (size_t)My * Mz * (p / My);  // p = j + My*i
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
int dev_sponge(st_ctx *c, const double *Q, double *Qrhs, const double *Y, double *Yrhs) {
    const size_t n3 = c->dm.n3;
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
    PFOR(c, n3, {
        int j = (int)(p % My), k = (int)((p / My) % Mz), i = (int)(p / ((size_t)My * Mz));
        auto sig = [](int gI, int st, int ln) -> double {
            if (gI >= st) {
                float r = (float)(gI - st) / (float)ln;   // REAL/REAL, src/sponge_mf.f:87-89
                return 4.0 * pow((double)r, 3.0);
            }
            return 0.0;
        };
        double s = sig(i + 1, sx, lx) + sig(j + 1, sy, ly) + sig(k + 1, sz, lz);
        double Qref[5] = {0.0, 0.0, 0.0, rho_ref, E_ref};
        for (int l = 0; l < 5; l++) Qrhs[l * n3 + p] = Qrhs[l * n3 + p] - s * (Q[l * n3 + p] - Qref[l]);
        Yrhs[p] = Yrhs[p] - s * (Q[3 * n3 + p] * Y[p] - Q[3 * n3 + p] * Y_ref);
    });
    return ST_OK;
}

// Fix_Pressure pproc/pproc_mf.f:190-233
int dev_fix_pressure(st_ctx *c, double *Q) {
    const size_t n3 = c->dm.n3;
    double *Q1 = Q, *Q2 = Q + n3, *Q3 = Q + 2 * n3, *Q4 = Q + 3 * n3, *Q5 = Q + 4 * n3;
    const double *g = c->gamma_eff;
    PFOR(c, n3, {
        double fac1 = g[p] - 1.0;
        double Vs = 1.0 / Q4[p];
        double P = fac1 * (Q5[p] - 5.0e-1 * Vs * (Q1[p] * Q1[p] + Q2[p] * Q2[p] + Q3[p] * Q3[p]));
        if (P < 0.0) P = 0.71429;
        Q5[p] = (1.0 / fac1) * P + 5.0e-1 * Vs * (Q1[p] * Q1[p] + Q2[p] * Q2[p] + Q3[p] * Q3[p]);
    });
    return ST_OK;
}

// Compact_Filter src/filters_sym.f:398-432
int dev_compact_filter(st_ctx *c, const double *F, double *F0, int nvar) {
    const size_t n3 = c->dm.n3;
    for (int l = 0; l < nvar; l++) {
        ST_TRY(dev_filter(c, 0, l == 0, F + l * n3, F0 + l * n3));
        ST_TRY(dev_filter(c, 1, l == 1, F0 + l * n3, F0 + l * n3));
        ST_TRY(dev_filter(c, 2, l == 2, F0 + l * n3, F0 + l * n3));
    }
    return ST_OK;
}

// Gaussian_Filter src/filters_sym.f:1046-1071
int dev_gaussian_filter(st_ctx *c, const double *F, double *Fg, int nvar) {
    const size_t n3 = c->dm.n3;
    Scratch tmp(c);
    for (int l = 0; l < nvar; l++) {
        ST_TRY(dev_gauss(c, 0, F + l * n3, Fg + l * n3));
        ST_TRY(dev_gauss(c, 1, Fg + l * n3, tmp));
        ST_TRY(dev_gauss(c, 2, tmp, Fg + l * n3));
    }
    return ST_OK;
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
__global__ void k_cfl(const double *Q, const double *g, size_t n3, double DX, double DY, double DZ,
                      double *out) {
    const double kmax = 2.478, khug = 2.199;   // src/header:237-240
    double m1 = 0.0, m2 = 0.0;
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n3; p += (size_t)gridDim.x * blockDim.x) {
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
__global__ void k_tstep(const double *Q, const double *Y, const double *g, const double *vh, const double *bh,
                        const double *kh, const double *Dh, size_t n3, double del, double g1, double g2,
                        double eps, double *out) {
    double m3 = INFINITY, m4 = INFINITY, m5 = INFINITY, m6 = INFINITY;
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n3; p += (size_t)gridDim.x * blockDim.x) {
        double fac = g[p] * (g[p] - 1.0);
        float fac1 = (float)(Y[p] + (eps * (g1 - 1.0) / (g2 - 1.0)) * (1.0 - Y[p]));   // implicit REAL
        double tmp1 = 1.0 / Q[3 * n3 + p];
        double q1 = Q[p], q2 = Q[n3 + p], q3 = Q[2 * n3 + p], q5 = Q[4 * n3 + p];
        double tmp2 = sqrt(fac * tmp1 * (q5 - 5.0e-1 * tmp1 * (q1 * q1 + q2 * q2 + q3 * q3)));
        double T = g1 * tmp1 * (q5 - 5.0e-1 * tmp1 * (q1 * q1 + q2 * q2 + q3 * q3));
        T = T / (double)fac1;
        double q4 = Q[3 * n3 + p];
        double w3 = q4 * pow(del, 2.0) / vh[p];
        double w4 = q4 * pow(del, 2.0) / bh[p];
        double w5 = q4 * pow(del * tmp2, 2.0) / (kh[p] * T);
        double w6 = pow(del, 2.0) / Dh[p];
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

// dt = min(cfl_cal/cfl_resv, 0.2*minima) -> out[6]; resv taken from out[1]
__global__ void k_tstep_final(double *out, double cfl_cal, int use_hyper, int resv_dev, double resv_host) {
    double resv = resv_dev ? out[1] : resv_host;
    double t = cfl_cal / resv;
    if (use_hyper) {
        double cand[4] = {0.2 * out[2], 0.2 * out[3], 0.2 * out[4], 0.2 * out[5]};
        for (int q = 0; q < 4; q++) if (cand[q] < t) t = cand[q];
    }
    out[6] = t;
}

static int grid_blocks(size_t n) {
    size_t b = (n + 255) / 256;
    return (int)(b > 148 * 8 ? 148 * 8 : (b ? b : 1));
}

int dev_compute_cfl(st_ctx *c, const double *Q, bool to_host, double *stab, double *resv) {
    ST_CUDA(c, cudaMemsetAsync(c->dscal, 0, 2 * sizeof(double), c->stream));
    int pi = prof_start(c, "k_cfl", 48.0 * c->dm.n3);
    k_cfl<<<grid_blocks(c->dm.n3), 256, 0, c->stream>>>(Q, c->gamma_eff, c->dm.n3, c->DX, c->DY, c->DZ,
                                                       c->dscal);
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
int dev_compute_tstep(st_ctx *c, const double *Q, const double *Y, int step, bool resv_on_device,
                      double cfl_resv_host) {
    const bool use_hyper = c->p.hyper_param == 1 && step > 0;
    if (use_hyper) {
        const double inf = INFINITY;
        double init[4] = {inf, inf, inf, inf};
        ST_CUDA(c, cudaMemcpyAsync(c->dscal + 2, init, sizeof(init), cudaMemcpyHostToDevice, c->stream));
        int pi = prof_start(c, "k_tstep", 88.0 * c->dm.n3);
        k_tstep<<<grid_blocks(c->dm.n3), 256, 0, c->stream>>>(
            Q, Y, c->gamma_eff, c->hyp[H_VISC], c->hyp[H_BETA], c->hyp[H_K], c->hyp[H_D], c->dm.n3, c->DX,
            c->p.gamma1, c->p.gamma2, c->p.epsilon, c->dscal);
        prof_stop(c, pi);
        ST_CUDA(c, cudaGetLastError());
    }
    c->launches++;
    k_tstep_final<<<1, 1, 0, c->stream>>>(c->dscal, c->p.cfl_cal, use_hyper ? 1 : 0, resv_on_device ? 1 : 0,
                                          cfl_resv_host);
    ST_CUDA(c, cudaGetLastError());
    return ST_OK;
}

// ---- LDDRK4 (src/lddrk4_nonperiodic_mf.f:428-541) -------------------------------
// dt is read from dscal[6] on the device (set by dev_compute_tstep or
// st_set_tstep), so the whole step can run without a host round trip.
int dev_lddrk4(st_ctx *c, bool) {
    static const double alpha1[5] = {0.0, -4.801594388477952e-01, -1.404247195200064e+00,
                                     -2.016477077503357e+00, -1.056444269767207e+00};
    static const double beta1[5] = {1.028639988104959e-01, 7.408540575766301e-01, 7.426530946683799e-01,
                                    4.694937902357905e-01, 1.881733382887932e-01};
    const size_t n3 = c->dm.n3;
    Scratch rYs(c), Qfs(c, 5);
    double *rY = rYs, *Qf = Qfs;
    const double *dtp = c->dscal + 6;
    double *timep = c->dscal + 7;
    for (int loop = 0; loop < 2; loop++) {
        ST_CUDA(c, cudaMemsetAsync(c->QW, 0, 5 * n3 * 8, c->stream));
        ST_CUDA(c, cudaMemsetAsync(c->rYW, 0, n3 * 8, c->stream));
        for (int K = 0; K < 5; K++) {
            const bool real = loop == 0 || c->p.rk_mode == 1;
            const double al = real ? alpha1[K] : 0.0, be = real ? beta1[K] : 0.0;
            double *Q = c->Q, *dQ = c->dQ, *QW = c->QW, *Y = c->Y, *drYi = c->drYi, *rYW = c->rYW;
            ST_TRY(dev_compute_gamma(c, Y));
            ST_TRY(dev_rhs(c, Q, dQ, Y));
            ST_TRY(dev_hyper_rhs(c, Q, dQ, Y));
            ST_TRY(dev_species_rhs(c, Q, dQ, Y, drYi));
            ST_TRY(dev_bc_rhs(c, Q, dQ, Y, drYi));
            ST_TRY(dev_sponge(c, Q, dQ, Y, drYi));
            PFOR(c, n3, {
                double dt = *dtp;
                double ry = Q[3 * n3 + p] * Y[p];
                for (int l = 0; l < 5; l++) {
                    size_t q = l * n3 + p;
                    QW[q] = al * QW[q] + dt * dQ[q];
                    Q[q] = Q[q] + be * QW[q];
                }
                rYW[p] = al * rYW[p] + dt * drYi[p];
                rY[p] = ry + be * rYW[p];
            });
            ST_TRY(dev_compact_filter(c, Q, Qf, 5));
            ST_TRY(dev_filter(c, 0, 0, rY, rY));
            ST_TRY(dev_filter(c, 1, 0, rY, rY));
            ST_TRY(dev_filter(c, 2, 0, rY, rY));
            PFOR(c, n3, {
                for (int l = 0; l < 5; l++) Q[l * n3 + p] = Qf[l * n3 + p];
                Y[p] = rY[p] / Q[3 * n3 + p];
            });
            ST_TRY(dev_fix_pressure(c, Q));
        }
        PFOR(c, 1, { timep[0] = timep[0] + dtp[0]; });
    }
    return ST_OK;
}

// monitoring sums (Compute_Mom/KE/Mass/Energy/Entropy), two-pass block sums
__global__ void k_monitor_partial(const double *Q, const double *g, size_t n3, double *part) {
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n3; p += (size_t)gridDim.x * blockDim.x) {
        double q1 = Q[p], q2 = Q[n3 + p], q3 = Q[2 * n3 + p], q4 = Q[3 * n3 + p], q5 = Q[4 * n3 + p];
        double t = 1.0 / q4;
        double ke = 0.0;
        double u1 = q1 * t, u2 = q2 * t, u3 = q3 * t;
        ke = ke + q4 * u1 * u1;
        ke = ke + q4 * u2 * u2;
        ke = ke + q4 * u3 * u3;
        double fac1 = g[p] - 1.0;
        double Vs = 1.0 / q4;
        double P = fac1 * (q5 - 5.0e-1 * Vs * (q1 * q1 + q2 * q2 + q3 * q3));
        double s1 = q4 * log(P * pow(Vs, g[p]));
        double s2 = q4 * s1 * s1;
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
    k_monitor_partial<<<nb, 256, 0, c->stream>>>(c->Q, c->gamma_eff, c->dm.n3, part);
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
