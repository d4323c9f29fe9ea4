// st_diag.cu - the Output-side diagnostics of the main loop (src/out_mf.f:
// 671-705): Compute_Grad (vorticity, dilatation, MaxDil, Enstrophy),
// Compute_SRM_Stats (shell averages, turbulent kinetic energy, mixing width)
// and Generate_Shock_Surface (mean shock radius and its spread), on the
// device-resident state of a context.
//
// Every sum is a two-pass block reduction (per-block partials, summed on the
// host in block order) or a per-block shared-memory histogram added into
// global bins; the reference sums sequentially, so results agree to rounding.
#include <cfloat>
#include <cmath>
#include <vector>
#include "st_internal.h"

namespace st {

namespace {

constexpr int kRB = 256;         // threads per reduction block
constexpr int kRG = 148 * 4;     // reduction blocks

// grid coordinate xcor(I), Uniform_X src/grid.f:116-128 (i 0-based)
struct Grid {
    double start[3], leng[3];
    int n[3];
    double D[3];
    __device__ __forceinline__ double cor(int d, int i) const {
        return start[d] + leng[d] * (double)(i) / (double)(n[d] - 1);
    }
    // distance of cell (i,j,k) from the origin with IX = DBLE(II-1)
    // (src/auxiliary_mf.f:289-300, pproc/pproc_mf.f:102-110)
    __device__ __forceinline__ double rad(int i, int j, int k) const {
        double x = ((double)(i + 1) - 1.0) * D[0], y = ((double)(j + 1) - 1.0) * D[1],
               z = ((double)(k + 1) - 1.0) * D[2];
        return sqrt(x * x + y * y + z * z);
    }
};

Grid grid_of(const st_ctx *c) {
    Grid g;
    const st_params &p = c->p;
    g.start[0] = p.x_start; g.start[1] = p.y_start; g.start[2] = p.z_start;
    g.leng[0] = p.x_leng; g.leng[1] = p.y_leng; g.leng[2] = p.z_leng;
    for (int d = 0; d < 3; d++) g.n[d] = c->dm.n[d];
    g.D[0] = c->DX; g.D[1] = c->DY; g.D[2] = c->DZ;
    return g;
}

__device__ __forceinline__ void cell_ijk(size_t p, int My, int Mz, int &i, int &j, int &k) {
    size_t r = p / My;
    j = (int)(p - r * My);
    k = (int)(r % Mz);
    i = (int)(r / Mz);
}

// block sums of NV values per thread into part[v * gridDim.x + blockIdx.x]
template <int NV>
__device__ __forceinline__ void block_sums(double (&acc)[NV], double *part) {
    __shared__ double sh[NV][kRB];
    for (int v = 0; v < NV; v++) sh[v][threadIdx.x] = acc[v];
    __syncthreads();
    for (int s = kRB / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            for (int v = 0; v < NV; v++) sh[v][threadIdx.x] += sh[v][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int v = 0; v < NV; v++) part[(size_t)v * gridDim.x + blockIdx.x] = sh[v][0];
}

// ---- Compute_Grad -------------------------------------------------------------
__global__ void k_velocity(const double *Q, double *U, size_t n3) {
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n3; p += (size_t)gridDim.x * blockDim.x) {
        double tmp = 1.0 / Q[3 * n3 + p];
        U[p] = Q[p] * tmp;
        U[n3 + p] = Q[n3 + p] * tmp;
        U[2 * n3 + p] = Q[2 * n3 + p] * tmp;
    }
}

// Grad = (duz_dy - duy_dz, dux_dz - duz_dx, duy_dx - dux_dy, dux_dx + duy_dy +
// duz_dz); per-block partials of max|Dil| and of sum(w.w)
struct Grad9 { const double *g[9]; };   // the nine velocity derivatives, /GRAD/ order
__global__ void k_vort(Grad9 G, double *Grad, size_t n3, double *part) {
    double acc[2] = {0.0, 0.0};
    const double *gzy = G.g[G_DUZ_DY], *gyz = G.g[G_DUY_DZ], *gxz = G.g[G_DUX_DZ], *gzx = G.g[G_DUZ_DX];
    const double *gyx = G.g[G_DUY_DX], *gxy = G.g[G_DUX_DY], *gxx = G.g[G_DUX_DX], *gyy = G.g[G_DUY_DY],
                 *gzz = G.g[G_DUZ_DZ];
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n3; p += (size_t)gridDim.x * blockDim.x) {
        double w1 = gzy[p] - gyz[p], w2 = gxz[p] - gzx[p], w3 = gyx[p] - gxy[p];
        double dil = gxx[p] + gyy[p] + gzz[p];
        if (Grad) { Grad[p] = w1; Grad[n3 + p] = w2; Grad[2 * n3 + p] = w3; Grad[3 * n3 + p] = dil; }
        acc[0] = fmax(acc[0], fabs(dil));
        acc[1] += w1 * w1 + w2 * w2 + w3 * w3;
    }
    __shared__ double sh[2][kRB];
    sh[0][threadIdx.x] = acc[0];
    sh[1][threadIdx.x] = acc[1];
    __syncthreads();
    for (int s = kRB / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            sh[0][threadIdx.x] = fmax(sh[0][threadIdx.x], sh[0][threadIdx.x + s]);
            sh[1][threadIdx.x] += sh[1][threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) { part[blockIdx.x] = sh[0][0]; part[gridDim.x + blockIdx.x] = sh[1][0]; }
}

// ---- shell statistics ------------------------------------------------------------
// bin M with r[M] <= rad < r[M+1] over the ascending table r[0..na], or -1
__device__ __forceinline__ int find_bin(const double *r, int na, double rad) {
    if (!(rad >= r[0]) || !(rad < r[na])) return -1;
    int lo = 0, hi = na;   // r[lo] <= rad < r[hi]
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (rad >= r[mid]) lo = mid; else hi = mid;
    }
    return lo;
}

// Ur of every cell (pproc/pproc_mf.f:98-121) and the shell sums of Ur and Y
// over the bins of Compute_Shell_Avg (table rs): per-block shared histograms
__global__ void k_shell_sums(const double *Q, const double *Y, Grid g, int My, int Mz, size_t n3,
                             const double *rs, int na, double *U, double *Ur, double *bsum, unsigned long long *bcnt) {
    extern __shared__ double hs[];   // [2][na] sums, then [na] counts (as doubles)
    for (int q = threadIdx.x; q < 3 * na; q += blockDim.x) hs[q] = 0.0;
    __syncthreads();
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n3; p += (size_t)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_ijk(p, My, Mz, i, j, k);
        double tmp = 1.0 / Q[3 * n3 + p];
        double u1 = Q[p] * tmp, u2 = Q[n3 + p] * tmp, u3 = Q[2 * n3 + p] * tmp;
        U[p] = u1; U[n3 + p] = u2; U[2 * n3 + p] = u3;
        double rad = g.rad(i, j, k);
        double ur = (i == 0 && j == 0 && k == 0)
                        ? 0.0
                        : (g.cor(0, i) / rad) * u1 + (g.cor(1, j) / rad) * u2 + (g.cor(2, k) / rad) * u3;
        Ur[p] = ur;
        int M = find_bin(rs, na, rad);
        if (M >= 0) {
            atomicAdd(&hs[M], ur);
            atomicAdd(&hs[na + M], Y[p]);
            atomicAdd(&hs[2 * na + M], 1.0);
        }
    }
    __syncthreads();
    for (int q = threadIdx.x; q < na; q += blockDim.x) {
        if (hs[2 * na + q] != 0.0) {
            atomicAdd(&bsum[q], hs[q]);
            atomicAdd(&bsum[na + q], hs[na + q]);
            atomicAdd(&bcnt[q], (unsigned long long)hs[2 * na + q]);
        }
    }
}

// tke over the uniform bins ru of Compute_SRM_Stats (pproc/pproc_mf.f:131-164)
__global__ void k_tke(const double *U, const double *Ur, const double *ura, Grid g, int My, int Mz, size_t n3,
                      const double *ru, int na, double *part) {
    double acc[1] = {0.0};
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n3; p += (size_t)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_ijk(p, My, Mz, i, j, k);
        double rad = g.rad(i, j, k);
        int M = find_bin(ru, na, rad);
        if (M < 0) continue;   // unassigned in the reference: contributes 0
        double d = Ur[p] - ura[M];
        double urp2 = d * d, t1 = 0.0, t2 = 0.0, t3 = 0.0;
        if (i > 0 && j > 0 && k > 0) {
            double ix = (double)(i + 1) - 1.0, iy = (double)(j + 1) - 1.0, iz = (double)(k + 1) - 1.0;
            t1 = U[p] - Ur[p] * (ix * g.D[0] / rad);
            t2 = U[n3 + p] - Ur[p] * (iy * g.D[1] / rad);
            t3 = U[2 * n3 + p] - Ur[p] * (iz * g.D[2] / rad);
        }
        acc[0] += (t1 * t1 + t2 * t2 + t3 * t3) + urp2;
    }
    block_sums<1>(acc, part);
}

// ---- Generate_Shock_Surface -------------------------------------------------------
__global__ void k_max(const double *b, size_t n3, double *part) {
    double m = -INFINITY;
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n3; p += (size_t)gridDim.x * blockDim.x)
        m = fmax(m, b[p]);
    __shared__ double sh[kRB];
    sh[threadIdx.x] = m;
    __syncthreads();
    for (int s = kRB / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// pass 0: sums of xcor, ycor, zcor and the count over the shock cells;
// pass 1: sum of their distances from the centroid c; pass 2: sum of the
// squared deviations of those distances from ra
template <int PASS>
__global__ void k_shock(const double *b, double thr, Grid g, int My, int Mz, size_t n3, double cx, double cy,
                        double cz, double ra, double *part) {
    constexpr int NV = PASS == 0 ? 4 : 1;
    double acc[NV];
    for (int v = 0; v < NV; v++) acc[v] = 0.0;
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n3; p += (size_t)gridDim.x * blockDim.x) {
        if (!(b[p] > thr)) continue;
        int i, j, k;
        cell_ijk(p, My, Mz, i, j, k);
        if constexpr (PASS == 0) {
            acc[0] += g.cor(0, i);
            acc[NV > 1 ? 1 : 0] += g.cor(1, j);
            acc[NV > 2 ? 2 : 0] += g.cor(2, k);
            acc[NV > 3 ? 3 : 0] += 1.0;
        } else {
            double dx = g.cor(0, i) - cx, dy = g.cor(1, j) - cy, dz = g.cor(2, k) - cz;
            double r = sqrt(dx * dx + dy * dy + dz * dz);
            if constexpr (PASS == 1) acc[0] += r;
            else { double d = r - ra; acc[0] += d * d; }
        }
    }
    block_sums<NV>(acc, part);
}

// host sums of the per-block partials (block order)
int fetch_sums(st_ctx *c, const double *part, int nv, double *out) {
    std::vector<double> h((size_t)nv * kRG);
    ST_CUDA(c, cudaMemcpyAsync(h.data(), part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    ST_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int v = 0; v < nv; v++) {
        double s = 0.0;
        for (int b = 0; b < kRG; b++) s += h[(size_t)v * kRG + b];
        out[v] = s;
    }
    return ST_OK;
}
int fetch_max(st_ctx *c, const double *part, double *out) {
    std::vector<double> h(kRG);
    ST_CUDA(c, cudaMemcpyAsync(h.data(), part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    ST_CUDA(c, cudaStreamSynchronize(c->stream));
    double m = -INFINITY;
    for (double v : h) m = std::fmax(m, v);
    *out = m;
    return ST_OK;
}

}  // namespace

int shell_count(const st_ctx *c) { return c->dm.n[0] / 2 + 10 * (c->dm.n[0] / 128); }

// the per-block partials (up to 4 sums of kRG blocks) and the bin tables live
// in one scratch field
static int diag_size_ok(st_ctx *c) {
    const size_t need = 4 * (size_t)kRG + 6 * (size_t)shell_count(c) + 8;
    if (c->dm.n3 < need) return fail(c, ST_E_UNSUPPORTED, "grid too small for the diagnostics");
    return ST_OK;
}

// Compute_Grad src/grad_sym.f:13-120.  In the FP64 mode the nine velocity
// derivatives are left in /GRAD/ as the reference leaves them (the next RHS
// overwrites them before any use); the FP32 mode keeps them in scratch.
int dev_compute_grad(st_ctx *c, double *Grad, double *maxdil, double *enstrophy) {
    ST_TRY(diag_size_ok(c));
    const size_t n3 = c->dm.n3;
    Scratch Us(c, 3), parts(c, 1);
    ScratchT<double> gs(c, fp32_mode(c) ? 9 : 1);
    double *U = Us;
    double *G[12] = {nullptr};
    for (int q = 0; q < 9; q++) G[q] = fp32_mode(c) ? (double *)gs + (size_t)q * n3 : c->grad[q];
    c->launches++;
    k_velocity<<<kRG, kRB, 0, c->stream>>>(c->Q, U, n3);
    ST_CUDA(c, cudaGetLastError());
    ST_TRY(dev_dfd(c, 1, 0, U + 2 * n3, G[G_DUZ_DY], 0, 1.0));
    ST_TRY(dev_dfd(c, 2, 0, U + n3, G[G_DUY_DZ], 0, 1.0));
    ST_TRY(dev_dfd(c, 0, 0, U + 2 * n3, G[G_DUZ_DX], 0, 1.0));
    ST_TRY(dev_dfd(c, 2, 0, U, G[G_DUX_DZ], 0, 1.0));
    ST_TRY(dev_dfd(c, 0, 0, U + n3, G[G_DUY_DX], 0, 1.0));
    ST_TRY(dev_dfd(c, 1, 0, U, G[G_DUX_DY], 0, 1.0));
    ST_TRY(dev_dfd(c, 0, 1, U, G[G_DUX_DX], 0, 1.0));
    ST_TRY(dev_dfd(c, 1, 1, U + n3, G[G_DUY_DY], 0, 1.0));
    ST_TRY(dev_dfd(c, 2, 1, U + 2 * n3, G[G_DUZ_DZ], 0, 1.0));
    double *part = parts;
    Grad9 g9;
    for (int q = 0; q < 9; q++) g9.g[q] = G[q];
    c->launches++;
    k_vort<<<kRG, kRB, 0, c->stream>>>(g9, Grad, n3, part);
    ST_CUDA(c, cudaGetLastError());
    double s[2];
    ST_TRY(fetch_max(c, part, &s[0]));
    ST_TRY(fetch_sums(c, part + kRG, 1, &s[1]));
    *maxdil = s[0];
    *enstrophy = 0.5 * s[1] / (double)(c->dm.n[0] * c->dm.n[1] * c->dm.n[2]);
    return ST_OK;
}

// Compute_SRM_Stats pproc/pproc_mf.f:4-186 with Compute_shell_avg
// src/auxiliary_mf.f:266-332
int dev_compute_srm_stats(st_ctx *c, double *hmix, double *tke_total, double *ur_avg, double *y_avg) {
    ST_TRY(diag_size_ok(c));
    const size_t n3 = c->dm.n3;
    const int na = shell_count(c);
    const int My = c->dm.n[1], Mz = c->dm.n[2];
    Scratch Us(c, 3), Urs(c, 1), parts(c, 1);
    double *U = Us, *Ur = Urs, *part = parts;
    // bin tables, sums and counts in the parts buffer: rs[na+1], ru[na+1],
    // bsum[2na], bcnt[na], ura[na] after the kRG partials
    std::vector<double> rs(na + 1), ru(na + 1);
    rs[0] = 0.0; ru[0] = 0.0;
    for (int M = 2; M <= na + 1; M++) {
        rs[M - 1] = rs[M - 2] + (M <= 4 ? c->DX * 2.0 * std::sqrt(3.0) : c->DX * std::sqrt(3.0));
        ru[M - 1] = ru[M - 2] + c->DX * std::sqrt(3.0);
    }
    double *d_rs = part + kRG, *d_ru = d_rs + na + 1, *d_sum = d_ru + na + 1, *d_ura = d_sum + 2 * na;
    unsigned long long *d_cnt = reinterpret_cast<unsigned long long *>(d_ura + na);
    ST_CUDA(c, cudaMemcpyAsync(d_rs, rs.data(), (na + 1) * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    ST_CUDA(c, cudaMemcpyAsync(d_ru, ru.data(), (na + 1) * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    ST_CUDA(c, cudaMemsetAsync(d_sum, 0, 2 * na * sizeof(double), c->stream));
    ST_CUDA(c, cudaMemsetAsync(d_cnt, 0, na * sizeof(unsigned long long), c->stream));
    const Grid g = grid_of(c);
    c->launches++;
    k_shell_sums<<<kRG, kRB, 3 * na * sizeof(double), c->stream>>>(c->Q, c->Y, g, My, Mz, n3, d_rs, na, U, Ur, d_sum,
                                                                   d_cnt);
    ST_CUDA(c, cudaGetLastError());
    std::vector<double> hsum(2 * na);
    std::vector<unsigned long long> hcnt(na);
    ST_CUDA(c, cudaMemcpyAsync(hsum.data(), d_sum, 2 * na * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    ST_CUDA(c, cudaMemcpyAsync(hcnt.data(), d_cnt, na * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
    ST_CUDA(c, cudaStreamSynchronize(c->stream));
    std::vector<double> ura(na), ya(na);
    for (int M = 0; M < na; M++) {
        ura[M] = hsum[M] / (double)hcnt[M];
        ya[M] = hsum[na + M] / (double)hcnt[M];
    }
    ST_CUDA(c, cudaMemcpyAsync(d_ura, ura.data(), na * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    c->launches++;
    k_tke<<<kRG, kRB, 0, c->stream>>>(U, Ur, d_ura, g, My, Mz, n3, d_ru, na, part);
    ST_CUDA(c, cudaGetLastError());
    double tke;
    ST_TRY(fetch_sums(c, part, 1, &tke));
    *tke_total = tke / (double)(c->dm.n[0] * c->dm.n[1] * c->dm.n[2]);
    double h = 0.0;
    for (int M = 0; M < na; M++)
        if (ya[M] > 0.0 && ya[M] < 1.0) h = h + 8.0 * ya[M] * (1.0 - ya[M]) * c->DX * std::sqrt(3.0);
    *hmix = h;
    if (ur_avg) std::copy(ura.begin(), ura.end(), ur_avg);
    if (y_avg) std::copy(ya.begin(), ya.end(), y_avg);
    return ST_OK;
}

// Generate_Shock_Surface src/shock.f:163-260 on /HYPER/ beta_hyper
int dev_shock_surface(st_ctx *c, double *rad_avg, double *rad_skew_rms) {
    ST_TRY(diag_size_ok(c));
    const size_t n3 = c->dm.n3;
    const int My = c->dm.n[1], Mz = c->dm.n[2];
    Scratch parts(c, 1), bws(c, 1);
    double *part = parts;
    const double *b = c->hyp[H_BETA];
    if (fp32_mode(c)) {   // widen the float /HYPER/ beta
        ST_TRY(dev_to_double(c, c->hypf[H_BETA], bws, n3));
        b = bws;
    }
    const Grid g = grid_of(c);
    double bmax;
    c->launches++;
    k_max<<<kRG, kRB, 0, c->stream>>>(b, n3, part);
    ST_CUDA(c, cudaGetLastError());
    ST_TRY(fetch_max(c, part, &bmax));
    const double thr = 0.1 * bmax;
    double s0[4];
    c->launches++;
    k_shock<0><<<kRG, kRB, 0, c->stream>>>(b, thr, g, My, Mz, n3, 0.0, 0.0, 0.0, 0.0, part);
    ST_CUDA(c, cudaGetLastError());
    ST_TRY(fetch_sums(c, part, 4, s0));
    const double n = s0[3];
    const double xc = s0[0] / n, yc = s0[1] / n, zc = s0[2] / n;
    double rs;
    c->launches++;
    k_shock<1><<<kRG, kRB, 0, c->stream>>>(b, thr, g, My, Mz, n3, xc, yc, zc, 0.0, part);
    ST_CUDA(c, cudaGetLastError());
    ST_TRY(fetch_sums(c, part, 1, &rs));
    const double ra = rs / n;
    double sk;
    c->launches++;
    k_shock<2><<<kRG, kRB, 0, c->stream>>>(b, thr, g, My, Mz, n3, xc, yc, zc, ra, part);
    ST_CUDA(c, cudaGetLastError());
    ST_TRY(fetch_sums(c, part, 1, &sk));
    *rad_avg = ra;
    *rad_skew_rms = std::sqrt(sk) / (n * ra);
    return ST_OK;
}

// ---- MakePaddedArrays -----------------------------------------------------------
// src/vis_silo_mf.f:440-689 on one rank (Px = Py = Pz = 1): the eleven visual
// fields at the nodes of the grid padded by one node per direction,
// W(My+1, Mz+1, Mx+1, 11) = (u, v, w, rho, P, w_x, w_y, w_z, dilatation,
// gamma_eff, Y), with the primitive variables of :494-510 (u = Q1/Q4, ...,
// P = fac1 (Q5 - 0.5 Vs (Q1^2 + Q2^2 + Q3^2)), fac1 = gamma_eff - 1,
// Vs = 1/Q4).  With no neighbour rank each padding node copies the last node
// of its direction (faces :640-666, edges :668-684, corner :686), so the
// source cell is the node index clamped to the grid.  One thread per padded
// node: 11 fields read, 11 written.
__global__ void k_padded(const double *__restrict__ Q, const double *__restrict__ Grad,
                         const double *__restrict__ gam, const double *__restrict__ Y, double *__restrict__ W,
                         int My, int Mz, int Mx, size_t n3) {
    const size_t Pj = (size_t)My + 1, Pk = (size_t)Mz + 1, np = Pj * Pk * ((size_t)Mx + 1);
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < np; p += (size_t)gridDim.x * blockDim.x) {
        const size_t r = p / Pj, j = p - r * Pj, i = r / Pk, k = r - i * Pk;
        const size_t q = (j < (size_t)My ? j : My - 1) +
                         (size_t)My * ((k < (size_t)Mz ? k : Mz - 1) + (size_t)Mz * (i < (size_t)Mx ? i : Mx - 1));
        const double q1 = Q[q], q2 = Q[n3 + q], q3 = Q[2 * n3 + q], q4 = Q[3 * n3 + q], q5 = Q[4 * n3 + q];
        const double g = gam[q];
        const double fac1 = g - 1.0;
        const double vs = 1.0 / q4;
        W[p] = q1 / q4;
        W[np + p] = q2 / q4;
        W[2 * np + p] = q3 / q4;
        W[3 * np + p] = q4;
        W[4 * np + p] = fac1 * (q5 - 5.0e-1 * vs * (q1 * q1 + q2 * q2 + q3 * q3));
#pragma unroll
        for (int f = 0; f < 4; f++) W[(5 + f) * np + p] = Grad[f * n3 + q];
        W[9 * np + p] = g;
        W[10 * np + p] = Y[q];
    }
}

size_t padded_nodes(const st_ctx *c) {
    return ((size_t)c->dm.n[0] + 1) * ((size_t)c->dm.n[1] + 1) * ((size_t)c->dm.n[2] + 1);
}

// W (device, 11 padded fields) from the context's state; Grad (device, the
// 4 fields of Compute_Grad) or NULL: then Compute_Grad runs first, as Output
// calls it before the visual file is written (src/out_mf.f:681-698)
static int launch_padded(st_ctx *c, const double *Grad, double *W) {
    const size_t np = padded_nodes(c);
    const int blocks = (int)std::min<size_t>((np + kRB - 1) / kRB, (size_t)148 * 16);
    c->launches++;
    k_padded<<<blocks, kRB, 0, c->stream>>>(c->Q, Grad, c->gamma_eff, c->Y, W, c->dm.n[1], c->dm.n[2], c->dm.n[0],
                                            c->dm.n3);
    ST_CUDA(c, cudaGetLastError());
    return ST_OK;
}

int dev_make_padded_arrays(st_ctx *c, const double *Grad, double *W) {
    if (Grad) return launch_padded(c, Grad, W);
    Scratch gs(c, 4);
    double maxdil, enstrophy;
    ST_TRY(dev_compute_grad(c, gs, &maxdil, &enstrophy));
    return launch_padded(c, gs, W);
}

// the padded coordinates (src/vis_silo_mf.f:486-491): Setup_Grid's nodes
// (src/grid.f:28-40, Uniform_X :116-128) and one spacing beyond the last
void padded_coords(const st_ctx *c, double *cor[3]) {
    const Grid g = grid_of(c);
    for (int d = 0; d < 3; d++) {
        const int n = g.n[d];
        for (int i = 0; i < n; i++) cor[d][i] = g.start[d] + g.leng[d] * (double)i / (double)(n - 1);
        cor[d][n] = cor[d][n - 1] + (cor[d][1] - cor[d][0]);
    }
}

}  // namespace st
