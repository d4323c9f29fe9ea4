// st_radial.cu - batched 1-D spherical-radial single-fluid family: many
// independent problems (each one run of the reference's radial program,
// src/makefile_radial) of different lengths advanced together on one GPU.
//
// Work decomposition: one CTA owns one problem at a time.  A problem's line
// of n <= T*SMAX points is split into T contiguous segments of S = ceil(n/T)
// rows, one per thread, held in registers.  Every line operator
//   - stages its input line in shared memory (coalesced), so the explicit
//     stencils read any neighbour directly and the boundary rows are plain
//     index cases;
//   - solves its constant-coefficient banded system by local recurrences per
//     segment plus a block-wide scan of the segments' affine carry maps
//     (scalar maps for the tridiagonal derivative systems, 2-vector maps with
//     2x2 matrices for the pentadiagonal filter).  In exact arithmetic this is
//     the forward elimination / back substitution of pentadiagonal_serial
//     (src/pentadiagonal.f90:319-374); no per-length carry tables are needed.
// LU factors: the rows of every system are the same for all problems except
// the last few, so the factors of rows 0..n-5 are one universal table (the
// elimination of row i only involves rows <= i) and only rows n-4..n-1 come
// from a small per-length tail table.
//
// A persistent kernel pulls problems (longest first) from a queue and runs all
// the requested LDDRK4 steps of a problem before taking the next; problems
// are independent, so no grid-wide synchronisation exists.  Two kernel
// configurations (threads per CTA, rows per thread) serve short and long
// problems; st_radial_tune times the candidates and keeps the fastest.
#include <cfloat>
#include <cmath>
#include <algorithm>
#include <numeric>
#include <string>
#include <vector>
#include "st_internal.h"

namespace st {
namespace rad {

constexpr int kTail = 4;            // per-length tail rows n-4..n-1
constexpr int kMinN = 16;

// scheme constants (src/header:173-204, src/LES_header:107-157)
struct K {
    double a1, b1, a2, b2, d2, cl1, cl2, cl3, cl4, cl5, cl6;
    double fa0, fa1, fa2, fa3, fa4;
    double bc1[6], bc2[6], bc3[3], bc4[4];
    double g[5];
};

__constant__ K c_k;        // scheme constants, identical for every batch

struct Tabs {
    const double *L1, *I1, *U1;       // first-derivative system: multiplier, 1/pivot, upper
    const double *L2, *I2, *U2;       // second-derivative system
    const double *P1, *P2, *Q1, *Q2, *IF;   // filter system
    const double *T1, *T2;            // tails [(nmax+1)][kTail][3]
    const double *TF;                 // tail  [(nmax+1)][kTail][5]
};

struct Batch {
    const long long *off;             // point offset of each problem
    const int *n;
    const double *xl;                 // x_leng
    const int *order;                 // processing order (longest first)
    double *Q, *QW, *hyp;             // 3n, 3n, 2n per problem
    double *time;
    int *step;
    double gamma, cfl;
    int hyper, rk_mode;
};

// ---- factor access ------------------------------------------------------------
__device__ __forceinline__ double tri_f(const double *pre, const double *tail, int n, int i, int k) {
    return i >= n - kTail ? __ldg(tail + ((size_t)n * kTail + (i - (n - kTail))) * 3 + k) : __ldg(pre + i);
}
__device__ __forceinline__ double pen_f(const double *pre, const double *tail, int n, int i, int k) {
    return i >= n - kTail ? __ldg(tail + ((size_t)n * kTail + (i - (n - kTail))) * 5 + k) : __ldg(pre + i);
}

// ---- block scans of affine carry maps -----------------------------------------
// scalar map c -> A + G c; "a then b" composes to (Ab + Gb Aa, Gb Ga)
struct Map1 { double A, G; };
__device__ __forceinline__ Map1 comp1(const Map1 &first, const Map1 &then) {
    return {fma(then.G, first.A, then.A), then.G * first.G};
}
// 2-vector map c -> A + M c (M row-major)
struct Map2 { double A0, A1, M00, M01, M10, M11; };
__device__ __forceinline__ Map2 comp2(const Map2 &f, const Map2 &t) {
    Map2 r;
    r.A0 = fma(t.M00, f.A0, fma(t.M01, f.A1, t.A0));
    r.A1 = fma(t.M10, f.A0, fma(t.M11, f.A1, t.A1));
    r.M00 = t.M00 * f.M00 + t.M01 * f.M10;
    r.M01 = t.M00 * f.M01 + t.M01 * f.M11;
    r.M10 = t.M10 * f.M00 + t.M11 * f.M10;
    r.M11 = t.M10 * f.M01 + t.M11 * f.M11;
    return r;
}
__device__ __forceinline__ Map1 shfl_up(const Map1 &m, int d) {
    return {__shfl_up_sync(0xffffffffu, m.A, d), __shfl_up_sync(0xffffffffu, m.G, d)};
}
__device__ __forceinline__ Map1 shfl_down(const Map1 &m, int d) {
    return {__shfl_down_sync(0xffffffffu, m.A, d), __shfl_down_sync(0xffffffffu, m.G, d)};
}
__device__ __forceinline__ Map2 shfl_up(const Map2 &m, int d) {
    return {__shfl_up_sync(0xffffffffu, m.A0, d), __shfl_up_sync(0xffffffffu, m.A1, d),
            __shfl_up_sync(0xffffffffu, m.M00, d), __shfl_up_sync(0xffffffffu, m.M01, d),
            __shfl_up_sync(0xffffffffu, m.M10, d), __shfl_up_sync(0xffffffffu, m.M11, d)};
}
__device__ __forceinline__ Map2 shfl_down(const Map2 &m, int d) {
    return {__shfl_down_sync(0xffffffffu, m.A0, d), __shfl_down_sync(0xffffffffu, m.A1, d),
            __shfl_down_sync(0xffffffffu, m.M00, d), __shfl_down_sync(0xffffffffu, m.M01, d),
            __shfl_down_sync(0xffffffffu, m.M10, d), __shfl_down_sync(0xffffffffu, m.M11, d)};
}
__device__ __forceinline__ Map1 ident(Map1) { return {0.0, 1.0}; }
__device__ __forceinline__ Map2 ident(Map2) { return {0.0, 0.0, 1.0, 0.0, 0.0, 1.0}; }
__device__ __forceinline__ Map1 comp(const Map1 &f, const Map1 &t) { return comp1(f, t); }
__device__ __forceinline__ Map2 comp(const Map2 &f, const Map2 &t) { return comp2(f, t); }

// Exclusive scan over the threads of the CTA.  FWD: thread t receives the
// composition of the maps of threads 0..t-1 (applied in that order);
// otherwise of threads T-1..t+1 (applied from the last down).  sh holds
// >= 2*T/32 maps.  Ends with the CTA synchronised.
template <class M, bool FWD, int T>
__device__ __forceinline__ M block_scan_excl(M m, M *sh) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    constexpr int NW = T / 32;
    M inc = m;   // inclusive within the warp
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        M o = FWD ? shfl_up(inc, d) : shfl_down(inc, d);
        bool take = FWD ? lane >= d : lane + d < 32;
        if (take) inc = FWD ? comp(o, inc) : comp(o, inc);
    }
    M ex = FWD ? shfl_up(inc, 1) : shfl_down(inc, 1);
    if (FWD ? lane == 0 : lane == 31) ex = ident(m);
    if (FWD ? lane == 31 : lane == 0) sh[w] = inc;
    __syncthreads();
    if constexpr (NW > 8) {
        // warp 0 scans the warp totals; sh[NW + w] receives warp w's prefix
        if (w == 0) {
            M tot = lane < NW ? sh[lane] : ident(m);
            M iw = tot;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                M o = FWD ? shfl_up(iw, d) : shfl_down(iw, d);
                bool take = FWD ? lane >= d : lane + d < 32;
                if (take) iw = comp(o, iw);
            }
            M xw = FWD ? shfl_up(iw, 1) : shfl_down(iw, 1);
            if (FWD ? lane == 0 : lane == 31) xw = ident(m);
            if (lane < NW) sh[NW + lane] = xw;
        }
        __syncthreads();
        ex = comp(sh[NW + w], ex);
    } else if constexpr (NW > 1) {
        M pre = ident(m);
        if (FWD) { for (int v = 0; v < w; v++) pre = comp(pre, sh[v]); }
        else { for (int v = NW - 1; v > w; v--) pre = comp(pre, sh[v]); }
        ex = comp(pre, ex);
    }
    __syncthreads();
    return ex;
}

// ---- banded solves of one line (rows a..a+cnt-1 of this thread) ---------------
// Tridiagonal system with factors (l, 1/pivot, upper): forward
// r'_i = r_i - l_i r'_{i-1}, backward x_i = (r'_i - u_i x_{i+1}) / pivot_i.
template <int SMAX, int T>
__device__ __forceinline__ void tri_solve(double (&r)[SMAX], int a, int cnt, int n, const double *L,
                                          const double *I, const double *U, const double *tail, Map1 *sh) {
    double v = 0.0, g = 1.0;
#pragma unroll
    for (int q = 0; q < SMAX; q++)
        if (q < cnt) {
            int i = a + q;
            double l = i == 0 ? 0.0 : tri_f(L, tail, n, i, 0);
            v = fma(-l, v, r[q]);
            r[q] = v;
            g = -l * g;
        }
    Map1 m = cnt > 0 ? Map1{v, g} : Map1{0.0, 1.0};
    Map1 ex = block_scan_excl<Map1, true, T>(m, sh);
    const double cin = ex.A;
    g = 1.0;
#pragma unroll
    for (int q = 0; q < SMAX; q++)
        if (q < cnt) {
            int i = a + q;
            double l = i == 0 ? 0.0 : tri_f(L, tail, n, i, 0);
            g = -l * g;
            r[q] = fma(g, cin, r[q]);
        }
    double x = 0.0, h = 1.0;
#pragma unroll
    for (int q = SMAX - 1; q >= 0; q--)
        if (q < cnt) {
            int i = a + q;
            double u = i == n - 1 ? 0.0 : tri_f(U, tail, n, i, 2);
            double id = tri_f(I, tail, n, i, 1);
            x = fma(-u, x, r[q]) * id;
            r[q] = x;
            h = -u * id * h;
        }
    Map1 mb = cnt > 0 ? Map1{x, h} : Map1{0.0, 1.0};
    Map1 eb = block_scan_excl<Map1, false, T>(mb, sh);
    const double ein = eb.A;
    h = 1.0;
#pragma unroll
    for (int q = SMAX - 1; q >= 0; q--)
        if (q < cnt) {
            int i = a + q;
            double u = i == n - 1 ? 0.0 : tri_f(U, tail, n, i, 2);
            double id = tri_f(I, tail, n, i, 1);
            h = -u * id * h;
            r[q] = fma(h, ein, r[q]);
        }
}

// Pentadiagonal system with the elimination order of pentadiagonal_serial:
// r'_i = (r_i - p2_i r'_{i-2}) - p1_i r'_{i-1};
// x_i = ((r'_i - q1_i x_{i+1}) - q2_i x_{i+2}) * id_i.
template <int SMAX, int T>
__device__ __forceinline__ void pen_solve(double (&r)[SMAX], int a, int cnt, int n, const Tabs *__restrict__ tb, Map2 *sh) {
    // forward: state (r'_{i-1}, r'_{i-2}); local run plus the responses to
    // the incoming state's two components
    double s1 = 0.0, s2 = 0.0, e11 = 1.0, e12 = 0.0, e21 = 0.0, e22 = 1.0;   // e_k: response to unit c_k
#pragma unroll
    for (int q = 0; q < SMAX; q++)
        if (q < cnt) {
            int i = a + q;
            double p1 = i == 0 ? 0.0 : pen_f(tb->P1, tb->TF, n, i, 0);
            double p2 = i < 2 ? 0.0 : pen_f(tb->P2, tb->TF, n, i, 1);
            double v = fma(-p1, s1, fma(-p2, s2, r[q]));
            double w1 = fma(-p1, e11, -p2 * e21);   // response of row i to c1
            double w2 = fma(-p1, e12, -p2 * e22);   // to c2
            r[q] = v;
            s2 = s1; s1 = v;
            e21 = e11; e22 = e12; e11 = w1; e12 = w2;
        }
    // outgoing state (r'_{b-1}, r'_{b-2}) = A + M c
    Map2 m = cnt > 0 ? Map2{s1, s2, e11, e12, e21, e22} : Map2{0.0, 0.0, 1.0, 0.0, 0.0, 1.0};
    Map2 ex = block_scan_excl<Map2, true, T>(m, sh);
    const double c1 = ex.A0, c2 = ex.A1;
    e11 = 1.0; e12 = 0.0; e21 = 0.0; e22 = 1.0;
#pragma unroll
    for (int q = 0; q < SMAX; q++)
        if (q < cnt) {
            int i = a + q;
            double p1 = i == 0 ? 0.0 : pen_f(tb->P1, tb->TF, n, i, 0);
            double p2 = i < 2 ? 0.0 : pen_f(tb->P2, tb->TF, n, i, 1);
            double w1 = fma(-p1, e11, -p2 * e21);
            double w2 = fma(-p1, e12, -p2 * e22);
            e21 = e11; e22 = e12; e11 = w1; e12 = w2;
            r[q] = fma(w1, c1, fma(w2, c2, r[q]));
        }
    // backward: state (x_{i+1}, x_{i+2})
    double x1 = 0.0, x2 = 0.0;
    double f11 = 1.0, f12 = 0.0, f21 = 0.0, f22 = 1.0;
#pragma unroll
    for (int q = SMAX - 1; q >= 0; q--)
        if (q < cnt) {
            int i = a + q;
            double q1 = i >= n - 1 ? 0.0 : pen_f(tb->Q1, tb->TF, n, i, 2);
            double q2 = i >= n - 2 ? 0.0 : pen_f(tb->Q2, tb->TF, n, i, 3);
            double id = pen_f(tb->IF, tb->TF, n, i, 4);
            double v = fma(-q2, x2, fma(-q1, x1, r[q])) * id;
            double w1 = fma(-q2, f21, -q1 * f11) * id;
            double w2 = fma(-q2, f22, -q1 * f12) * id;
            r[q] = v;
            x2 = x1; x1 = v;
            f21 = f11; f22 = f12; f11 = w1; f12 = w2;
        }
    Map2 mb = cnt > 0 ? Map2{x1, x2, f11, f12, f21, f22} : Map2{0.0, 0.0, 1.0, 0.0, 0.0, 1.0};
    Map2 eb = block_scan_excl<Map2, false, T>(mb, sh);
    const double d1 = eb.A0, d2 = eb.A1;
    f11 = 1.0; f12 = 0.0; f21 = 0.0; f22 = 1.0;
#pragma unroll
    for (int q = SMAX - 1; q >= 0; q--)
        if (q < cnt) {
            int i = a + q;
            double q1 = i >= n - 1 ? 0.0 : pen_f(tb->Q1, tb->TF, n, i, 2);
            double q2 = i >= n - 2 ? 0.0 : pen_f(tb->Q2, tb->TF, n, i, 3);
            double id = pen_f(tb->IF, tb->TF, n, i, 4);
            double w1 = fma(-q2, f21, -q1 * f11) * id;
            double w2 = fma(-q2, f22, -q1 * f12) * id;
            f21 = f11; f22 = f12; f11 = w1; f12 = w2;
            r[q] = fma(w1, d1, fma(w2, d2, r[q]));
        }
}

// ---- explicit right-hand sides from the staged line X -------------------------
enum Op { OP_D1 = 0, OP_D2, OP_FILT, OP_GAUSS, OP_RHS, OP_HYPER };

// boundary rows (first and last four) of each operator:
// DFDX src/derivCDopt6_radial.f:703-760, D2FDX2 :862-918,
// Compact_Filter_X src/filters_nonperiodic.f:479-589 and
// Gaussian_Filter_X :1108-1221 (symmetric reflection at both ends)
__device__ __noinline__ double boundary_row(int op, int i, const double *X, int n, double fac) {
    if (op == OP_D1) {
        if (i >= 3 && i <= n - 4) return fac * (c_k.b1 * (X[i + 2] - X[i - 2]) + c_k.a1 * (X[i + 1] - X[i - 1]));
        if (i == 2) return fac * (c_k.cl3 * (X[4] - X[0]) + c_k.cl4 * (X[3] - X[1]));
        if (i == 1) return fac * (-c_k.cl1 * X[0] - 5.0e-1 * X[1] + X[2] + c_k.cl2 * X[3]);
        if (i == 0) return fac * (-2.5 * X[0] + 2.0 * X[1] + 5.0e-1 * X[2]);
        if (i == n - 3) return fac * (c_k.cl3 * (X[n - 1] - X[n - 5]) + c_k.cl4 * (X[n - 2] - X[n - 4]));
        if (i == n - 2) return fac * (c_k.cl1 * X[n - 1] + 5.0e-1 * X[n - 2] - X[n - 3] - c_k.cl2 * X[n - 4]);
        return fac * (2.5 * X[n - 1] - 2.0 * X[n - 2] - 5.0e-1 * X[n - 3]);
    }
    if (op == OP_D2) {
        if (i >= 3 && i <= n - 4)
            return fac * (c_k.b2 * (X[i + 2] + X[i - 2]) + c_k.a2 * (X[i + 1] + X[i - 1]) - c_k.d2 * X[i]);
        if (i == 2) return fac * (c_k.cl5 * (X[0] - 2.0 * X[2] + X[4]) + c_k.cl6 * (X[1] - 2.0 * X[2] + X[3]));
        if (i == 1) return fac * (1.2375 * X[0] - 3.0 * X[1] + 2.325 * X[2] - 6.0e-1 * X[3] + 3.75e-2 * X[4]);
        if (i == 0) return fac * (1.3e1 * X[0] - 2.7e1 * X[1] + 1.5e1 * X[2] - X[3]);
        if (i == n - 3)
            return fac * (c_k.cl5 * (X[n - 1] - 2.0 * X[n - 3] + X[n - 5]) +
                          c_k.cl6 * (X[n - 2] - 2.0 * X[n - 3] + X[n - 4]));
        if (i == n - 2)
            return fac * (1.2375 * X[n - 1] - 3.0 * X[n - 2] + 2.325 * X[n - 3] - 6.0e-1 * X[n - 4] +
                          3.75e-2 * X[n - 5]);
        return fac * (1.3e1 * X[n - 1] - 2.7e1 * X[n - 2] + 1.5e1 * X[n - 3] - X[n - 4]);
    }
    if (op == OP_FILT) {
        if (i == 0) return c_k.bc1[1] * X[0] + c_k.bc1[2] * X[1] + c_k.bc1[3] * X[2] + c_k.bc1[4] * X[3] + c_k.bc1[5] * X[4];
        if (i == 1) return c_k.bc2[1] * X[0] + c_k.bc2[2] * X[1] + c_k.bc2[3] * X[2] + c_k.bc2[4] * X[3] + c_k.bc2[5] * X[4];
        if (i == 2) return c_k.bc3[2] * X[4] + c_k.bc3[1] * X[3] + c_k.bc3[0] * X[2] + c_k.bc3[1] * X[1] + c_k.bc3[2] * X[0];
        if (i == 3)
            return c_k.bc4[3] * X[6] + c_k.bc4[2] * X[5] + c_k.bc4[1] * X[4] + c_k.bc4[0] * X[3] + c_k.bc4[1] * X[2] +
                   c_k.bc4[2] * X[1] + c_k.bc4[3] * X[0];
        if (i == n - 1)
            return c_k.bc1[1] * X[n - 1] + c_k.bc1[2] * X[n - 2] + c_k.bc1[3] * X[n - 3] + c_k.bc1[4] * X[n - 4] +
                   c_k.bc1[5] * X[n - 5];
        if (i == n - 2)
            return c_k.bc2[1] * X[n - 1] + c_k.bc2[2] * X[n - 2] + c_k.bc2[3] * X[n - 3] + c_k.bc2[4] * X[n - 4] +
                   c_k.bc2[5] * X[n - 5];
        if (i == n - 3)
            return c_k.bc3[2] * X[n - 5] + c_k.bc3[1] * X[n - 4] + c_k.bc3[0] * X[n - 3] + c_k.bc3[1] * X[n - 2] +
                   c_k.bc3[2] * X[n - 1];
        return c_k.bc4[3] * X[n - 7] + c_k.bc4[2] * X[n - 6] + c_k.bc4[1] * X[n - 5] + c_k.bc4[0] * X[n - 4] +
               c_k.bc4[1] * X[n - 3] + c_k.bc4[2] * X[n - 2] + c_k.bc4[3] * X[n - 1];
    }
    // Gaussian (a+b == b+a, so reflected pairs need no particular order)
    const double *g = c_k.g;
    if (i == 0) return g[4] * (2.0 * X[4]) + g[3] * (2.0 * X[3]) + g[2] * (2.0 * X[2]) + g[1] * (2.0 * X[1]) + g[0] * X[0];
    if (i == n - 1)
        return g[4] * (2.0 * X[n - 5]) + g[3] * (2.0 * X[n - 4]) + g[2] * (2.0 * X[n - 3]) + g[1] * (2.0 * X[n - 2]) +
               g[0] * X[n - 1];
    auto f = [&](int j) {
        j = j < 0 ? -j : j;
        j = j > n - 1 ? 2 * (n - 1) - j : j;
        return X[j];
    };
    return g[4] * (f(i + 4) + f(i - 4)) + g[3] * (f(i + 3) + f(i - 3)) + g[2] * (f(i + 2) + f(i - 2)) +
           g[1] * (f(i + 1) + f(i - 1)) + g[0] * X[i];
}

// explicit right-hand side of rows a..a+cnt-1 (interior rows inline)
template <int SMAX>
__device__ __forceinline__ void rhs_rows(double (&r)[SMAX], int op, const double *X, int a, int cnt, int n,
                                         double fac) {
#pragma unroll
    for (int q = 0; q < SMAX; q++)
        if (q < cnt) {
            const int i = a + q;
            double w;
            if (i >= 4 && i <= n - 5) {
                if (op == OP_D1) w = fac * (c_k.b1 * (X[i + 2] - X[i - 2]) + c_k.a1 * (X[i + 1] - X[i - 1]));
                else if (op == OP_D2)
                    w = fac * (c_k.b2 * (X[i + 2] + X[i - 2]) + c_k.a2 * (X[i + 1] + X[i - 1]) - c_k.d2 * X[i]);
                else if (op == OP_FILT)
                    w = c_k.fa4 * (X[i + 4] + X[i - 4]) + c_k.fa3 * (X[i + 3] + X[i - 3]) + c_k.fa2 * (X[i + 2] + X[i - 2]) +
                        c_k.fa1 * (X[i + 1] + X[i - 1]) + c_k.fa0 * X[i];
                else
                    w = c_k.g[4] * (X[i + 4] + X[i - 4]) + c_k.g[3] * (X[i + 3] + X[i - 3]) +
                        c_k.g[2] * (X[i + 2] + X[i - 2]) + c_k.g[1] * (X[i + 1] + X[i - 1]) + c_k.g[0] * X[i];
            } else {
                w = boundary_row(op, i, X, n, fac);
            }
            r[q] = w;
        }
}

// ---- per-problem geometry ---------------------------------------------------------
struct Geo {
    int n;
    double DX, fac1, fac2;            // DX; cadd = 1 factor of DFDX; factor of D2FDX2
};
__device__ __forceinline__ Geo geo(int n, double xl) {
    Geo g;
    g.n = n;
    g.DX = xl * (double)(1) / (double)(n - 1) - xl * (double)(0) / (double)(n - 1);   // src/grid.f:25-36
    const double sx = 1.0 / xl;
    g.fac1 = 1.0 * sx * (double)(n - 1);
    g.fac2 = ((double)((n - 1) * (n - 1))) * (sx * sx);
    return g;
}
// rad(I) = |(REAL(I - Nx/2) - 0.5) DX|, src/rhsv_radial.f:55-59
__device__ __forceinline__ double radius(int i, const Geo &g) {
    double IX = (double)(float)(i + 1 - g.n / 2) - 0.5;
    return fabs(IX * g.DX);
}

// shared-memory working set of one CTA
template <int T, int SMAX>
struct Smem {
    static constexpr int N = T * SMAX;
    double X[N];          // staged input line
    double Y[N];          // line-operator result
    double Ru[N], Rr[N], Rs[N];   // dQ of the stage (u, rho, s)
    double Du[N];         // -du/dr (DFDX(u, -1)), reused by Hyper_RHS
    Map2 sc[2 * (T / 32)];   // scan scratch (also holds Map1 values)
    double red[T / 32][4];
    int prob;
};

// One line operator on the staged line S.X; this thread's rows of the result
// go to S.Y (rows a..a+cnt-1, read back by the same thread).  DFDX flips the
// sign on the left half (dF/dr = -dF/dx for II <= Nx/2,
// src/derivCDopt6_radial.f:772-784).  fac: cadd*sx*(n-1) (DFDX) or
// (n-1)^2*sx^2 (D2FDX2).
template <int T, int SMAX>
__device__ __noinline__ void line_op(Smem<T, SMAX> &S, int op, int n, double fac, const Tabs *__restrict__ tb) {
    const int t = threadIdx.x, Sr = (n + T - 1) / T, a = t * Sr, cnt = max(0, min(Sr, n - a));
    double r[SMAX];
    rhs_rows<SMAX>(r, op, S.X, a, cnt, n, fac);
    if (op == OP_D1 || op == OP_D2) {
        const bool d1 = op == OP_D1;
        tri_solve<SMAX, T>(r, a, cnt, n, d1 ? tb->L1 : tb->L2, d1 ? tb->I1 : tb->I2, d1 ? tb->U1 : tb->U2,
                           d1 ? tb->T1 : tb->T2, reinterpret_cast<Map1 *>(S.sc));
    } else if (op == OP_FILT) {
        pen_solve<SMAX, T>(r, a, cnt, n, tb, S.sc);
    }
#pragma unroll
    for (int q = 0; q < SMAX; q++)
        if (q < cnt) S.Y[a + q] = (op == OP_D1 && a + q + 1 <= n / 2) ? -r[q] : r[q];
}

// stage a line into S.X: X[i] = f(i) for i < n, then synchronise.  The
// caller guarantees every earlier reader of X has passed a barrier.
template <int T, int SMAX, class F>
__device__ __forceinline__ void stage(Smem<T, SMAX> &S, int n, F f) {
    for (int i = threadIdx.x; i < n; i += T) S.X[i] = f(i);
    __syncthreads();
}

// this thread's rows a..a+cnt-1
#define RAD_ROWS(T_, n_)                                                                       \
    const int Sr_ = ((n_) + (T_) - 1) / (T_), a = (int)threadIdx.x * Sr_, cnt = max(0, min(Sr_, (n_) - a))

// Compute_hyper src/hyper_radial.f:9-62: d4 = D2(D2(u)), hyp = (1, 2e-3) *
// Gauss(|d4|) * DX^5
template <int T, int SMAX>
__device__ __noinline__ void problem_hyper_core(Smem<T, SMAX> &S, const Geo &G, const double *u, double *hyp,
                                                const Tabs *__restrict__ tb) {
    const int n = G.n;
    RAD_ROWS(T, n);
    stage(S, n, [&](int i) { return u[i]; });
    line_op<T, SMAX>(S, OP_D2, n, G.fac2, tb);
    __syncthreads();                                        // every read of X is done
    for (int q = 0; q < cnt; q++) S.X[a + q] = S.Y[a + q];
    __syncthreads();
    line_op<T, SMAX>(S, OP_D2, n, G.fac2, tb);
    __syncthreads();
    for (int q = 0; q < cnt; q++) S.X[a + q] = fabs(S.Y[a + q]);
    __syncthreads();
    line_op<T, SMAX>(S, OP_GAUSS, n, 0.0, tb);
    const double DX5 = pow(G.DX, 5.0);
    for (int q = 0; q < cnt; q++) {
        hyp[a + q] = 1.0 * S.Y[a + q] * DX5;
        hyp[n + a + q] = 2.0e-3 * S.Y[a + q] * DX5;
    }
    __syncthreads();
}

// RHS_r (src/rhsv_radial.f:30-157) and, when hyper, Hyper_RHS
// (src/hyper_radial.f:75-187) of one problem: leaves dQ in S.Ru/Rr/Rs and
// refreshes /HYPER/ (hyp).
template <int T, int SMAX>
__device__ __noinline__ void problem_rhs(Smem<T, SMAX> &S, const Geo &G, const double *u, const double *rho,
                                         const double *s, double *hyp, double gam, int hyper,
                                         const Tabs *__restrict__ tb) {
    const int n = G.n;
    RAD_ROWS(T, n);
    // d rho/dt = -u d rho/dr  (DFDX(rho, Qrhs4, 1, -1): 0 + W)
    stage(S, n, [&](int i) { return rho[i]; });
    line_op<T, SMAX>(S, OP_D1, n, -G.fac1, tb);
    for (int q = 0; q < cnt; q++) S.Rr[a + q] = S.Y[a + q] * u[a + q];
    __syncthreads();
    // - rho/r^2 d(u r^2)/dr
    stage(S, n, [&](int i) { double rd = radius(i, G); return u[i] * rd * rd; });
    line_op<T, SMAX>(S, OP_D1, n, G.fac1, tb);
    for (int q = 0; q < cnt; q++) {
        const int i = a + q;
        double rd = radius(i, G);
        S.Rr[i] = S.Rr[i] - S.Y[i] * (rho[i] / (rd * rd));
    }
    __syncthreads();
    // d u/dt = -u du/dr
    stage(S, n, [&](int i) { return u[i]; });
    line_op<T, SMAX>(S, OP_D1, n, -G.fac1, tb);
    for (int q = 0; q < cnt; q++) { S.Du[a + q] = S.Y[a + q]; S.Ru[a + q] = u[a + q] * S.Y[a + q]; }
    __syncthreads();
    // - (dP/dr)/rho,  P = s rho^gamma
    stage(S, n, [&](int i) { return s[i] * pow(rho[i], gam); });
    line_op<T, SMAX>(S, OP_D1, n, G.fac1, tb);
    for (int q = 0; q < cnt; q++) S.Ru[a + q] = S.Ru[a + q] - (S.Y[a + q] / rho[a + q]);
    __syncthreads();
    // d s/dt = -u ds/dr
    stage(S, n, [&](int i) { return s[i]; });
    line_op<T, SMAX>(S, OP_D1, n, -G.fac1, tb);
    for (int q = 0; q < cnt; q++) S.Rs[a + q] = S.Y[a + q] * u[a + q];
    __syncthreads();
    if (!hyper) return;
    problem_hyper_core<T, SMAX>(S, G, u, hyp, tb);
    const double *bh = hyp, *vh = hyp + n;
    // 1/r^2 d/dr(r^2 2 nu du/dr)   (du/dr = -Du exactly: DFDX is odd in cadd)
    stage(S, n, [&](int i) { double rd = radius(i, G); return rd * rd * 2.0 * vh[i] * (-S.Du[i]); });
    line_op<T, SMAX>(S, OP_D1, n, G.fac1, tb);
    double qh[SMAX];                          // first Hyper_RHS term of this thread's rows
#pragma unroll
    for (int q = 0; q < SMAX; q++)
        if (q < cnt) { double rd = radius(a + q, G); qh[q] = (1.0 / (rd * rd)) * S.Y[a + q]; }
    __syncthreads();
    // 1/r^2 d/dr(r^2 (beta - 2/3 nu)(du/dr + 2u/r))
    stage(S, n, [&](int i) {
        double rd = radius(i, G);
        return rd * rd * (bh[i] - (2.0 / 3.0) * vh[i]) * (-S.Du[i] + 2.0 * u[i] / rd);
    });
    line_op<T, SMAX>(S, OP_D1, n, G.fac1, tb);
#pragma unroll
    for (int q = 0; q < SMAX; q++)
        if (q < cnt) {
            double rd = radius(a + q, G);
            double h = qh[q] + (1.0 / (rd * rd)) * S.Y[a + q];
            S.Ru[a + q] = S.Ru[a + q] + h;
        }
    __syncthreads();
}

// block reductions (T/32 partials in S.red)
template <int T, int SMAX>
__device__ __forceinline__ double block_max(Smem<T, SMAX> &S, double v, int slot) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) S.red[threadIdx.x >> 5][slot] = v;
    __syncthreads();
    double m = S.red[0][slot];
    for (int w = 1; w < T / 32; w++) m = fmax(m, S.red[w][slot]);
    __syncthreads();
    return m;
}
template <int T, int SMAX>
__device__ __forceinline__ double block_min(Smem<T, SMAX> &S, double v, int slot) {
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) S.red[threadIdx.x >> 5][slot] = v;
    __syncthreads();
    double m = S.red[0][slot];
    for (int w = 1; w < T / 32; w++) m = fmin(m, S.red[w][slot]);
    __syncthreads();
    return m;
}

__constant__ double c_alpha1[5] = {0.0, -4.801594388477952e-01, -1.404247195200064e+00, -2.016477077503357e+00,
                                   -1.056444269767207e+00};
__constant__ double c_beta1[5] = {1.028639988104959e-01, 7.408540575766301e-01, 7.426530946683799e-01,
                                  4.694937902357905e-01, 1.881733382887932e-01};
__constant__ double c_alpha2[6] = {0.0, -4.4127377153877382565e-1, -1.073982008079781868e0,
                                   -1.7063570791256758809e0, -2.7979293162682443056e0, -4.0913537120919160454e0};
__constant__ double c_beta2[6] = {1.1584888181285561688e-1, 3.7287699051652864918e-1, 7.3795368921435295698e-1,
                                  5.7981109366311039538e-1, 1.031284991300145194e0, 1.5e-1};

// One main-loop iteration of one problem (src/main.f:129-136):
// Compute_CFL + Compute_Tstep (src/lddrk4_nonperiodic_sf.f:7-146, x term),
// then LDDRK4 (:376-468; no Fix_Pressure: its radial source is not shipped).
template <int T, int SMAX>
__device__ __noinline__ void problem_step(Smem<T, SMAX> &S, const Batch &B, int p, const Tabs *__restrict__ tb) {
    const int n = B.n[p];
    const Geo G = geo(n, B.xl[p]);
    const size_t o = (size_t)B.off[p];
    double *u = B.Q + 3 * o, *rho = u + n, *s = rho + n;
    double *wu = B.QW + 3 * o, *wr = wu + n, *ws = wr + n;
    double *hyp = B.hyp + 2 * o;
    const double gam = B.gamma, fac = gam * (gam - 1.0);
    const int t = threadIdx.x;
    RAD_ROWS(T, n);
    // CFL and hyperviscous limits
    double m2 = 0.0, m3 = INFINITY, m4 = INFINITY;
    const double khug = 2.199, del = G.DX;
    for (int i = t; i < n; i += T) {
        double tmp1 = 1.0 / rho[i];
        double tmp2 = sqrt(fac * tmp1 * (s[i] - 5.0e-1 * tmp1 * (u[i] * u[i] + 0.0 + 0.0)));
        double ux = fabs(u[i] * tmp1);
        m2 = fmax(m2, (tmp2 + ux) * khug / G.DX);
        if (B.hyper == 1) {
            m3 = fmin(m3, rho[i] * pow(del, 2.0) / hyp[n + i]);
            m4 = fmin(m4, rho[i] * pow(del, 2.0) / hyp[i]);
        }
    }
    const double resv = block_max(S, m2, 0);
    double dt = B.cfl / resv;
    if (B.hyper == 1) {
        const double f02 = (double)0.2f;
        double c3 = f02 * block_min(S, m3, 1), c4 = f02 * block_min(S, m4, 2);
        if (c3 < dt) dt = c3;
        if (c4 < dt) dt = c4;
    }
    double tm = B.time[p];
    for (int loop = 0; loop < 2; loop++) {
        const int ns = loop == 0 ? 5 : 6;
        for (int K = 0; K < ns; K++) {
            double al, be;
            if (loop == 0) { al = c_alpha1[K]; be = c_beta1[K]; }
            else if (B.rk_mode == 1) { al = c_alpha2[K]; be = c_beta2[K]; }
            else { al = 0.0; be = 0.0; }
            const bool first = K == 0;          // QW = 0 at the loop start and alpha(1) = 0
            problem_rhs<T, SMAX>(S, G, u, rho, s, hyp, gam, B.hyper, tb);
            // update, then filter u, rho, s in place (Compact_Filter x pass)
            for (int i = t; i < n; i += T) {
                const double d0 = S.Ru[i], d1 = S.Rr[i], d2 = S.Rs[i];
                double q0 = first ? dt * d0 : al * wu[i] + dt * d0;
                double q1 = first ? dt * d1 : al * wr[i] + dt * d1;
                double q2 = first ? dt * d2 : al * ws[i] + dt * d2;
                wu[i] = q0; wr[i] = q1; ws[i] = q2;
                u[i] = u[i] + be * q0;
                rho[i] = rho[i] + be * q1;
                s[i] = s[i] + be * q2;
            }
            __syncthreads();
            for (int f = 0; f < 3; f++) {
                double *F = f == 0 ? u : (f == 1 ? rho : s);
                stage(S, n, [&](int i) { return F[i]; });
                line_op<T, SMAX>(S, OP_FILT, n, 0.0, tb);
                for (int q = 0; q < cnt; q++) F[a + q] = S.Y[a + q];
                __syncthreads();
            }
        }
        tm = tm + dt;
    }
    if (t == 0) { B.time[p] = tm; B.step[p] = B.step[p] + 1; }
    __syncthreads();
}

// Persistent kernel: CTAs take problems (in B.order from index first..last-1)
// from the queue counter and run nsteps steps of each; a problem whose step
// counter is 0 first gets the set-up Compute_hyper (src/main.f:100).
template <int T, int SMAX>
__global__ void __launch_bounds__(T) k_rad_steps(Batch B, const Tabs *__restrict__ tb, int first, int last, int nsteps,
                                                   int *queue) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem<T, SMAX> &S = *reinterpret_cast<Smem<T, SMAX> *>(smem_raw);
    for (;;) {
        if (threadIdx.x == 0) S.prob = first + atomicAdd(queue, 1);
        __syncthreads();
        const int idx = S.prob;
        __syncthreads();
        if (idx >= last) return;
        const int p = B.order[idx];
        if (B.step[p] == 0) {
            const size_t o = (size_t)B.off[p];
            problem_hyper_core<T, SMAX>(S, geo(B.n[p], B.xl[p]), B.Q + 3 * o, B.hyp + 2 * o, tb);
        }
        for (int it = 0; it < nsteps; it++) problem_step<T, SMAX>(S, B, p, tb);
    }
}

// Per-operator kernel for the C ABI's line operators: one CTA per problem.
template <int T, int SMAX>
__global__ void __launch_bounds__(T) k_rad_op(Batch B, const Tabs *__restrict__ tb, int op, const double *F, double *O1,
                                                double *O2, int iadd, double cadd) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem<T, SMAX> &S = *reinterpret_cast<Smem<T, SMAX> *>(smem_raw);
    const int p = blockIdx.x;
    const int n = B.n[p];
    const Geo G = geo(n, B.xl[p]);
    const size_t o = (size_t)B.off[p];
    RAD_ROWS(T, n);
    if (op == OP_RHS || op == OP_HYPER) {
        const double *u = F + 3 * o, *rho = u + n, *s = rho + n;
        problem_rhs<T, SMAX>(S, G, u, rho, s, B.hyp + 2 * o, B.gamma, op == OP_HYPER ? B.hyper : 0, tb);
        double *R = O1 + 3 * o;
        for (int i = threadIdx.x; i < n; i += T) { R[i] = S.Ru[i]; R[n + i] = S.Rr[i]; R[2 * n + i] = S.Rs[i]; }
        return;
    }
    const double *f = F + o;
    stage(S, n, [&](int i) { return f[i]; });
    const double fac = op == OP_D1 ? cadd * (1.0 / B.xl[p]) * (double)(n - 1) : G.fac2;
    line_op<T, SMAX>(S, op, n, fac, tb);
    double *out = (op == OP_D2 ? O2 : O1) + o;
    for (int q = 0; q < cnt; q++) out[a + q] = (op == OP_D1 && iadd == 1) ? out[a + q] + S.Y[a + q] : S.Y[a + q];
    if (op == OP_D2 && iadd == 1) {
        __syncthreads();
        line_op<T, SMAX>(S, OP_D1, n, 1.0 * (1.0 / B.xl[p]) * (double)(n - 1), tb);
        for (int q = 0; q < cnt; q++) O1[o + a + q] = S.Y[a + q];
    }
}

// ---- host side: factor tables ---------------------------------------------------
static const double kTiny = (double)FLT_MIN;

// tridiagonal factors in pentadiagonal_serial's order with A = E = 0:
// l_i = B_i/(C'_{i-1}+tiny), C'_i = C_i - D_{i-1} l_i, id_i = 1/(C'_i+tiny)
static void tri_factor(const std::vector<double> &B, const std::vector<double> &C, const std::vector<double> &D,
                       std::vector<double> &l, std::vector<double> &id, std::vector<double> &up) {
    int n = (int)C.size();
    std::vector<double> Cp(C);
    l.assign(n, 0.0); id.assign(n, 0.0); up = D;
    for (int i = 1; i < n; i++) {
        l[i] = B[i] / (Cp[i - 1] + kTiny);
        Cp[i] = Cp[i] - D[i - 1] * l[i];
    }
    for (int i = 0; i < n; i++) id[i] = 1.0 / (Cp[i] + kTiny);
    up[n - 1] = 0.0;
}
// Setup_Derivatives src/derivCDopt6_radial.f:9-600 (order 1 or 2)
static void deriv_rows(int n, int order, std::vector<double> &B, std::vector<double> &C, std::vector<double> &D) {
    double al = order == 1 ? 1.0 / 3.0 : 2.0 / 11.0;
    B.assign(n, al); C.assign(n, 1.0); D.assign(n, al);
    if (order == 1) {
        B[0] = 0.0; D[0] = 2.0; B[n - 1] = 2.0; D[n - 1] = 0.0;
        B[1] = 1.0 / 6.0; D[1] = 1.0 / 2.0; B[n - 2] = 1.0 / 2.0; D[n - 2] = 1.0 / 6.0;
        B[2] = 1.0 / 3.0; D[2] = 1.0 / 3.0; B[n - 3] = 1.0 / 3.0; D[n - 3] = 1.0 / 3.0;
    } else {
        B[0] = 0.0; D[0] = 1.1e1; B[n - 1] = 1.1e1; D[n - 1] = 0.0;
        B[1] = 1.0e-1; D[1] = -7.0 / 2.0e1; B[n - 2] = -7.0 / 2.0e1; D[n - 2] = 1.0e-1;
        B[2] = 2.0 / 1.1e1; D[2] = 2.0 / 1.1e1; B[n - 3] = 2.0 / 1.1e1; D[n - 3] = 2.0 / 1.1e1;
    }
}
// Init_Filters src/filters_nonperiodic.f:9-390 and the pentadiagonal_serial
// factors (p1, p2 forward multipliers; q1, q2 upper entries; id)
static void filt_factor(int n, std::vector<double> f[5]) {
    const double af = 6.6624e-01, bf = 1.6688e-01, ab = 0.45;
    std::vector<double> A(n, bf), B(n, af), C(n, 1.0), D(n, af), E(n, bf);
    auto row = [&](int r, double a_, double b_, double c_, double d_, double e_) {
        A[r] = a_; B[r] = b_; C[r] = c_; D[r] = d_; E[r] = e_;
    };
    row(0, 0, 0, 1, 0, 0); row(n - 1, 0, 0, 1, 0, 0);
    row(1, 0, ab, 1, ab, 0); row(n - 2, 0, ab, 1, ab, 0);
    row(2, 0, ab, 1, ab, 0); row(n - 3, 0, ab, 1, ab, 0);
    std::vector<double> k1(n, 0.0), k2(n, 0.0);
    for (int i = 0; i <= n - 3; i++) {
        k1[i] = B[i + 1] / (C[i] + kTiny);
        C[i + 1] = C[i + 1] - D[i] * k1[i];
        D[i + 1] = D[i + 1] - E[i] * k1[i];
        k2[i] = A[i + 2] / (C[i] + kTiny);
        B[i + 2] = B[i + 2] - D[i] * k2[i];
        C[i + 2] = C[i + 2] - E[i] * k2[i];
    }
    double k3 = B[n - 1] / (C[n - 2] + kTiny);
    C[n - 1] = C[n - 1] - D[n - 2] * k3;
    for (int q = 0; q < 5; q++) f[q].assign(n, 0.0);
    f[0][1] = k1[0];
    for (int i = 2; i <= n - 2; i++) { f[0][i] = k1[i - 1]; f[1][i] = k2[i - 2]; }
    f[0][n - 1] = k3; f[1][n - 1] = k2[n - 3];
    for (int i = 0; i <= n - 2; i++) f[2][i] = D[i];
    for (int i = 0; i <= n - 3; i++) f[3][i] = E[i];
    for (int i = 0; i < n; i++) f[4][i] = 1.0 / (C[i] + kTiny);
}

static void fill_k(K &k) {
    k.a1 = 14.0 / 18.0; k.b1 = 1.0 / 36.0;
    k.a2 = 12.0 / 11.0; k.b2 = 3.0 / 44.0; k.d2 = 2.0 * (k.a2 + k.b2);
    k.cl1 = 5.0 / 9.0; k.cl2 = 1.0 / 1.8e1; k.cl3 = 1.0 / 3.6e1; k.cl4 = 7.0 / 9.0;
    k.cl5 = 3.0 / 4.4e1; k.cl6 = 1.2e1 / 1.1e1;
    k.fa0 = 9.9965e-01; k.fa1 = 0.66652; k.fa2 = 0.16674; k.fa3 = 4.0e-05; k.fa4 = -5.0e-06;
    const double ab = 0.45, af = 6.6624e-01, bf = 1.6688e-01;
    k.bc1[0] = 0.0; k.bc1[1] = 15.0 / 16.0; k.bc1[2] = 1.0 / 4.0; k.bc1[3] = -3.0 / 8.0;
    k.bc1[4] = 1.0 / 4.0; k.bc1[5] = -1.0 / 16.0;
    k.bc2[0] = (1.0 / 2.0 + ab); k.bc2[1] = (1.0 / 16.0 + (7.0 / 8.0) * ab);
    k.bc2[2] = (3.0 / 4.0 + (1.0 / 2.0) * ab); k.bc2[3] = (3.0 / 8.0 + (1.0 / 4.0) * ab);
    k.bc2[4] = (-1.0 / 4.0 + (1.0 / 2.0) * ab); k.bc2[5] = (1.0 / 16.0 - (1.0 / 8.0) * ab);
    k.bc3[0] = (5.0 / 8.0 + (3.0 / 4.0) * ab); k.bc3[1] = (1.0 / 2.0 + ab) / 2.0;
    k.bc3[2] = (-1.0 / 8.0 + ab / 4.0) / 2.0;
    k.bc4[0] = (11.0 / 16.0 + (5.0 / 8.0) * af - (5.0 / 8.0) * bf);
    k.bc4[1] = (15.0 / 32.0 + (17.0 / 16.0) * af + (15.0 / 16.0) * bf) / 2.0;
    k.bc4[2] = (-3.0 / 16.0 + (3.0 / 8.0) * af + (13.0 / 8.0) * bf) / 2.0;
    k.bc4[3] = (1.0 / 32.0 - af / 16.0 + bf / 16.0) / 2.0;
    k.g[0] = (double)(float)(3565.0 / 10368.0);
    k.g[1] = (double)(float)(3091.0 / 12960.0);
    k.g[2] = (double)(float)(1997.0 / 25920.0);
    k.g[3] = (double)(float)(149.0 / 12960.0);
    k.g[4] = (double)(float)(107.0 / 103680.0);
}

// kernel configurations (threads per CTA, rows per thread): the short-problem
// class (n <= 1024) picks one of (64,16), (128,8), (256,4), the long class
// (n <= 4096) one of (256,16), (512,8), (1024,4); see launch_class
constexpr int kShortMax = 1024, kLongMax = 4096;

template <int T, int SMAX>
static size_t smem_bytes() { return sizeof(Smem<T, SMAX>); }

}  // namespace rad
}  // namespace st

// ---- handle and C ABI -------------------------------------------------------------
using namespace st;
using namespace st::rad;

struct st_radial {
    st_radial_params p{};
    int dev = 0;
    cudaStream_t stream = nullptr, aux = nullptr, own = nullptr;   // stream in use, fork stream, own stream
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    std::string err;
    int nprob = 0, nmax = 0;
    long long npts = 0;
    std::vector<int> n_h;
    std::vector<long long> off_h;
    std::vector<int> order_h;
    int nshort = 0;                 // problems [0, nshort) of order_h are short (n <= kShortMax)
    int cfg_short = 1, cfg_long = 1;
    // device arrays
    long long *off = nullptr;
    int *n = nullptr, *order = nullptr, *step = nullptr, *queue = nullptr;
    double *xl = nullptr, *Q = nullptr, *QW = nullptr, *hyp = nullptr, *time = nullptr;
    double *tabs = nullptr;         // all factor tables in one allocation
    K k{};
    Tabs tb{};
    Tabs *dtb = nullptr;            // device copy of tb
    long long launches = 0;
};

static int rfail(st_radial *h, int code, const std::string &m) {
    if (h) h->err = m;
    return code;
}
#define RCUDA(h, call)                                                                                  \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) return rfail((h), ST_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

static Batch make_batch(st_radial *h) {
    Batch b;
    b.off = h->off; b.n = h->n; b.xl = h->xl; b.order = h->order;
    b.Q = h->Q; b.QW = h->QW; b.hyp = h->hyp; b.time = h->time; b.step = h->step;
    b.gamma = h->p.gamma; b.cfl = h->p.cfl_cal; b.hyper = h->p.hyper_param; b.rk_mode = h->p.rk_mode;
    return b;
}

template <int T, int SMAX>
static int launch_steps(st_radial *h, int first, int last, int nsteps, int *queue, cudaStream_t st) {
    if (last <= first) return ST_OK;
    const size_t sm = smem_bytes<T, SMAX>();
    RCUDA(h, cudaFuncSetAttribute(k_rad_steps<T, SMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int per_sm = 0;
    RCUDA(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rad_steps<T, SMAX>, T, sm));
    int nsm = 0;
    RCUDA(h, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->dev));
    int grid = std::max(1, std::min(per_sm * nsm, last - first));
    h->launches++;
    k_rad_steps<T, SMAX><<<grid, T, sm, st>>>(make_batch(h), h->dtb, first, last, nsteps, queue);
    RCUDA(h, cudaGetLastError());
    return ST_OK;
}
static int launch_class(st_radial *h, bool is_short, int cfg, int first, int last, int nsteps, int *queue,
                        cudaStream_t st) {
    if (is_short) {
        switch (cfg) {
            case 0: return launch_steps<64, 16>(h, first, last, nsteps, queue, st);
            case 1: return launch_steps<128, 8>(h, first, last, nsteps, queue, st);
            default: return launch_steps<256, 4>(h, first, last, nsteps, queue, st);
        }
    }
    switch (cfg) {
        case 0: return launch_steps<256, 16>(h, first, last, nsteps, queue, st);
        case 1: return launch_steps<512, 8>(h, first, last, nsteps, queue, st);
        default: return launch_steps<1024, 4>(h, first, last, nsteps, queue, st);
    }
}

// both classes, concurrently on two streams (long problems first in order_h)
static int run_steps(st_radial *h, int nsteps) {
    RCUDA(h, cudaMemsetAsync(h->queue, 0, 2 * sizeof(int), h->stream));
    RCUDA(h, cudaEventRecord(h->ev_fork, h->stream));
    RCUDA(h, cudaStreamWaitEvent(h->aux, h->ev_fork, 0));
    const int nlong = h->nprob - h->nshort;
    int rc = launch_class(h, false, h->cfg_long, 0, nlong, nsteps, h->queue, h->stream);
    if (rc != ST_OK) return rc;
    rc = launch_class(h, true, h->cfg_short, nlong, h->nprob, nsteps, h->queue + 1, h->aux);
    if (rc != ST_OK) return rc;
    RCUDA(h, cudaEventRecord(h->ev_join, h->aux));
    RCUDA(h, cudaStreamWaitEvent(h->stream, h->ev_join, 0));
    return ST_OK;
}

template <int T, int SMAX>
static int launch_op(st_radial *h, int op, const double *F, double *O1, double *O2, int iadd, double cadd) {
    const size_t sm = smem_bytes<T, SMAX>();
    RCUDA(h, cudaFuncSetAttribute(k_rad_op<T, SMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    h->launches++;
    k_rad_op<T, SMAX><<<h->nprob, T, sm, h->stream>>>(make_batch(h), h->dtb, op, F, O1, O2, iadd, cadd);
    RCUDA(h, cudaGetLastError());
    RCUDA(h, cudaStreamSynchronize(h->stream));
    return ST_OK;
}

extern "C" {

const char *st_radial_last_error(const st_radial *h) { return h ? h->err.c_str() : "null handle"; }

int st_radial_create(const st_radial_params *p, int nprob, const int *n, const double *x_leng, st_radial **out) {
    if (!p || !n || !x_leng || !out || nprob < 1) return ST_E_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return ST_E_NODEVICE; }
    if (p->device < 0 || p->device >= ndev || (p->rk_mode != 0 && p->rk_mode != 1)) return ST_E_ARG;
    for (int k = 0; k < nprob; k++)
        if (n[k] < kMinN || n[k] > kLongMax || !(x_leng[k] > 0.0)) return ST_E_UNSUPPORTED;
    st_radial *h = new (std::nothrow) st_radial();
    if (!h) return ST_E_NOMEM;
    auto bail = [&](int code, const std::string &m) { h->err = m; st_radial_destroy(h); return code; };
    h->p = *p;
    h->dev = p->device;
    h->nprob = nprob;
    h->n_h.assign(n, n + nprob);
    h->off_h.resize(nprob);
    long long acc = 0;
    for (int k = 0; k < nprob; k++) { h->off_h[k] = acc; acc += n[k]; h->nmax = std::max(h->nmax, n[k]); }
    h->npts = acc;
    // longest first (the queue then finishes with short problems), long class first
    h->order_h.resize(nprob);
    std::iota(h->order_h.begin(), h->order_h.end(), 0);
    std::stable_sort(h->order_h.begin(), h->order_h.end(), [&](int a, int b) { return n[a] > n[b]; });
    h->nshort = 0;
    for (int k = 0; k < nprob; k++) if (n[k] <= kShortMax) h->nshort++;
    if (cudaSetDevice(h->dev) != cudaSuccess) return bail(ST_E_CUDA, "cudaSetDevice");
    if (cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->aux, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming) != cudaSuccess)
        return bail(ST_E_CUDA, "stream/event creation");
    h->stream = h->own;
    fill_k(h->k);
    // factor tables: universal prefixes from the longest length, tails per length
    const int NM = std::max(h->nmax, kMinN);
    std::vector<double> B, C, D, l1, i1, u1, l2, i2, u2, F[5];
    deriv_rows(NM, 1, B, C, D); tri_factor(B, C, D, l1, i1, u1);
    deriv_rows(NM, 2, B, C, D); tri_factor(B, C, D, l2, i2, u2);
    filt_factor(NM, F);
    std::vector<double> t1((size_t)(NM + 1) * kTail * 3, 0.0), t2(t1.size(), 0.0), tf((size_t)(NM + 1) * kTail * 5, 0.0);
    std::vector<char> seen(NM + 1, 0);
    for (int k = 0; k < nprob; k++) seen[n[k]] = 1;
    for (int m = kMinN; m <= NM; m++) {
        if (!seen[m]) continue;
        std::vector<double> l, id, up, G[5];
        for (int order = 1; order <= 2; order++) {
            deriv_rows(m, order, B, C, D); tri_factor(B, C, D, l, id, up);
            std::vector<double> &T = order == 1 ? t1 : t2;
            const std::vector<double> &Lp = order == 1 ? l1 : l2, &Ip = order == 1 ? i1 : i2, &Up = order == 1 ? u1 : u2;
            for (int i = 0; i < m - kTail; i++)   // the prefix really is universal
                if (l[i] != Lp[i] || id[i] != Ip[i] || up[i] != Up[i])
                    return bail(ST_E_UNSUPPORTED, "radial derivative factors are not length-independent");
            for (int q = 0; q < kTail; q++) {
                int i = m - kTail + q;
                T[((size_t)m * kTail + q) * 3 + 0] = l[i];
                T[((size_t)m * kTail + q) * 3 + 1] = id[i];
                T[((size_t)m * kTail + q) * 3 + 2] = up[i];
            }
        }
        filt_factor(m, G);
        for (int i = 0; i < m - kTail; i++)
            for (int q = 0; q < 5; q++)
                if (G[q][i] != F[q][i]) return bail(ST_E_UNSUPPORTED, "radial filter factors are not length-independent");
        for (int q = 0; q < kTail; q++)
            for (int c = 0; c < 5; c++) tf[((size_t)m * kTail + q) * 5 + c] = G[c][m - kTail + q];
    }
    std::vector<double> all;
    auto put = [&](const std::vector<double> &v) { size_t o = all.size(); all.insert(all.end(), v.begin(), v.end()); return o; };
    size_t o_l1 = put(l1), o_i1 = put(i1), o_u1 = put(u1), o_l2 = put(l2), o_i2 = put(i2), o_u2 = put(u2);
    size_t o_f[5];
    for (int q = 0; q < 5; q++) o_f[q] = put(F[q]);
    size_t o_t1 = put(t1), o_t2 = put(t2), o_tf = put(tf);
    const size_t P = (size_t)h->npts;
    bool ok = cudaMalloc((void **)&h->tabs, all.size() * 8) == cudaSuccess &&
              cudaMalloc((void **)&h->off, nprob * sizeof(long long)) == cudaSuccess &&
              cudaMalloc((void **)&h->n, nprob * sizeof(int)) == cudaSuccess &&
              cudaMalloc((void **)&h->order, nprob * sizeof(int)) == cudaSuccess &&
              cudaMalloc((void **)&h->step, nprob * sizeof(int)) == cudaSuccess &&
              cudaMalloc((void **)&h->queue, 2 * sizeof(int)) == cudaSuccess &&
              cudaMalloc((void **)&h->xl, nprob * sizeof(double)) == cudaSuccess &&
              cudaMalloc((void **)&h->time, nprob * sizeof(double)) == cudaSuccess &&
              cudaMalloc((void **)&h->Q, 3 * P * 8) == cudaSuccess &&
              cudaMalloc((void **)&h->QW, 3 * P * 8) == cudaSuccess &&
              cudaMalloc((void **)&h->hyp, 2 * P * 8) == cudaSuccess;
    if (!ok) { cudaGetLastError(); return bail(ST_E_NOMEM, "device allocation of the radial batch failed"); }
    ok = cudaMemcpy(h->tabs, all.data(), all.size() * 8, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(h->off, h->off_h.data(), nprob * sizeof(long long), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(h->n, n, nprob * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(h->order, h->order_h.data(), nprob * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(h->xl, x_leng, nprob * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemset(h->step, 0, nprob * sizeof(int)) == cudaSuccess &&
         cudaMemset(h->time, 0, nprob * sizeof(double)) == cudaSuccess &&
         cudaMemset(h->Q, 0, 3 * P * 8) == cudaSuccess && cudaMemset(h->QW, 0, 3 * P * 8) == cudaSuccess &&
         cudaMemset(h->hyp, 0, 2 * P * 8) == cudaSuccess;
    if (!ok) { cudaGetLastError(); return bail(ST_E_CUDA, "uploading the radial batch tables"); }
    const double *T0 = h->tabs;
    h->tb.L1 = T0 + o_l1; h->tb.I1 = T0 + o_i1; h->tb.U1 = T0 + o_u1;
    h->tb.L2 = T0 + o_l2; h->tb.I2 = T0 + o_i2; h->tb.U2 = T0 + o_u2;
    h->tb.P1 = T0 + o_f[0]; h->tb.P2 = T0 + o_f[1]; h->tb.Q1 = T0 + o_f[2]; h->tb.Q2 = T0 + o_f[3]; h->tb.IF = T0 + o_f[4];
    h->tb.T1 = T0 + o_t1; h->tb.T2 = T0 + o_t2; h->tb.TF = T0 + o_tf;
    if (cudaMalloc((void **)&h->dtb, sizeof(Tabs)) != cudaSuccess ||
        cudaMemcpy(h->dtb, &h->tb, sizeof(Tabs), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpyToSymbol(c_k, &h->k, sizeof(K)) != cudaSuccess) {
        cudaGetLastError();
        return bail(ST_E_CUDA, "uploading the radial constants");
    }
    *out = h;
    return ST_OK;
}

int st_radial_destroy(st_radial *h) {
    if (!h) return ST_E_ARG;
    cudaSetDevice(h->dev);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->aux) cudaStreamSynchronize(h->aux);
    void *ptrs[] = {h->tabs, h->dtb, h->off, h->n, h->order, h->step, h->queue, h->xl, h->time, h->Q, h->QW, h->hyp};
    for (void *q : ptrs) if (q) cudaFree(q);
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_join) cudaEventDestroy(h->ev_join);
    if (h->own) cudaStreamDestroy(h->own);
    if (h->aux) cudaStreamDestroy(h->aux);
    delete h;
    return ST_OK;
}

int st_radial_num_points(const st_radial *h, long long *npts) {
    if (!h || !npts) return ST_E_ARG;
    *npts = h->npts;
    return ST_OK;
}

int st_radial_set_state(st_radial *h, const double *Q) {
    if (!h || !Q) return ST_E_ARG;
    if (cudaSetDevice(h->dev) != cudaSuccess) return rfail(h, ST_E_CUDA, "cudaSetDevice");
    const size_t P = (size_t)h->npts;
    RCUDA(h, cudaMemcpyAsync(h->Q, Q, 3 * P * 8, cudaMemcpyDefault, h->stream));
    RCUDA(h, cudaMemsetAsync(h->QW, 0, 3 * P * 8, h->stream));
    RCUDA(h, cudaMemsetAsync(h->hyp, 0, 2 * P * 8, h->stream));
    RCUDA(h, cudaMemsetAsync(h->step, 0, h->nprob * sizeof(int), h->stream));
    RCUDA(h, cudaMemsetAsync(h->time, 0, h->nprob * sizeof(double), h->stream));
    RCUDA(h, cudaStreamSynchronize(h->stream));
    return ST_OK;
}

int st_radial_get_state(st_radial *h, double *Q) {
    if (!h || !Q) return ST_E_ARG;
    if (cudaSetDevice(h->dev) != cudaSuccess) return rfail(h, ST_E_CUDA, "cudaSetDevice");
    RCUDA(h, cudaMemcpyAsync(Q, h->Q, 3 * (size_t)h->npts * 8, cudaMemcpyDefault, h->stream));
    RCUDA(h, cudaStreamSynchronize(h->stream));
    return ST_OK;
}

int st_radial_get_hyper(st_radial *h, double *hyp) {
    if (!h || !hyp) return ST_E_ARG;
    if (cudaSetDevice(h->dev) != cudaSuccess) return rfail(h, ST_E_CUDA, "cudaSetDevice");
    RCUDA(h, cudaMemcpyAsync(hyp, h->hyp, 2 * (size_t)h->npts * 8, cudaMemcpyDefault, h->stream));
    RCUDA(h, cudaStreamSynchronize(h->stream));
    return ST_OK;
}

int st_radial_get_time(st_radial *h, double *time, int *step) {
    if (!h || (!time && !step)) return ST_E_ARG;
    if (cudaSetDevice(h->dev) != cudaSuccess) return rfail(h, ST_E_CUDA, "cudaSetDevice");
    if (time) RCUDA(h, cudaMemcpyAsync(time, h->time, h->nprob * sizeof(double), cudaMemcpyDefault, h->stream));
    if (step) RCUDA(h, cudaMemcpyAsync(step, h->step, h->nprob * sizeof(int), cudaMemcpyDefault, h->stream));
    RCUDA(h, cudaStreamSynchronize(h->stream));
    return ST_OK;
}

int st_radial_step(st_radial *h, int nsteps) {
    if (!h || nsteps < 0) return ST_E_ARG;
    if (nsteps == 0) return ST_OK;
    if (cudaSetDevice(h->dev) != cudaSuccess) return rfail(h, ST_E_CUDA, "cudaSetDevice");
    int rc = run_steps(h, nsteps);
    if (rc != ST_OK) return rc;
    RCUDA(h, cudaStreamSynchronize(h->stream));
    return ST_OK;
}

int st_radial_set_stream(st_radial *h, void *stream) {
    if (!h) return ST_E_ARG;
    h->stream = stream ? (cudaStream_t)stream : h->own;
    return ST_OK;
}

int st_radial_step_async(st_radial *h, int nsteps) {
    if (!h || nsteps < 1) return ST_E_ARG;
    if (cudaSetDevice(h->dev) != cudaSuccess) return rfail(h, ST_E_CUDA, "cudaSetDevice");
    return run_steps(h, nsteps);
}

int st_radial_config(st_radial *h, int *cfg_short, int *cfg_long, int set) {
    if (!h || !cfg_short || !cfg_long) return ST_E_ARG;
    if (set) {
        if (*cfg_short < 0 || *cfg_short > 2 || *cfg_long < 0 || *cfg_long > 2) return ST_E_ARG;
        h->cfg_short = *cfg_short; h->cfg_long = *cfg_long;
    } else {
        *cfg_short = h->cfg_short; *cfg_long = h->cfg_long;
    }
    return ST_OK;
}

int st_radial_tune(st_radial *h, double *ms_out) {
    if (!h) return ST_E_ARG;
    if (cudaSetDevice(h->dev) != cudaSuccess) return rfail(h, ST_E_CUDA, "cudaSetDevice");
    const size_t P = (size_t)h->npts;
    // work on a copy of the state: the tuning steps must not advance the batch
    double *sQ = nullptr, *sW = nullptr, *sH = nullptr, *sT = nullptr;
    int *sS = nullptr;
    bool ok = cudaMalloc((void **)&sQ, 3 * P * 8) == cudaSuccess && cudaMalloc((void **)&sW, 3 * P * 8) == cudaSuccess &&
              cudaMalloc((void **)&sH, 2 * P * 8) == cudaSuccess &&
              cudaMalloc((void **)&sT, h->nprob * 8) == cudaSuccess && cudaMalloc((void **)&sS, h->nprob * 4) == cudaSuccess;
    auto release = [&]() { cudaFree(sQ); cudaFree(sW); cudaFree(sH); cudaFree(sT); cudaFree(sS); };
    if (!ok) { cudaGetLastError(); release(); return rfail(h, ST_E_NOMEM, "tuning copies"); }
    cudaMemcpyAsync(sQ, h->Q, 3 * P * 8, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(sW, h->QW, 3 * P * 8, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(sH, h->hyp, 2 * P * 8, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(sT, h->time, h->nprob * 8, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(sS, h->step, h->nprob * 4, cudaMemcpyDeviceToDevice, h->stream);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    const int nlong = h->nprob - h->nshort;
    int rc = ST_OK;
    for (int cls = 0; cls < 2 && rc == ST_OK; cls++) {
        const bool is_short = cls == 1;
        const int first = is_short ? nlong : 0, last = is_short ? h->nprob : nlong;
        if (last <= first) continue;
        float best = 1e30f;
        int best_c = is_short ? h->cfg_short : h->cfg_long;
        for (int c = 0; c < 3 && rc == ST_OK; c++) {
            float ms = 0.f;
            for (int rep = 0; rep < 2 && rc == ST_OK; rep++) {   // first run warms up
                cudaMemcpyAsync(h->Q, sQ, 3 * P * 8, cudaMemcpyDeviceToDevice, h->stream);
                cudaMemcpyAsync(h->QW, sW, 3 * P * 8, cudaMemcpyDeviceToDevice, h->stream);
                cudaMemcpyAsync(h->hyp, sH, 2 * P * 8, cudaMemcpyDeviceToDevice, h->stream);
                cudaMemcpyAsync(h->time, sT, h->nprob * 8, cudaMemcpyDeviceToDevice, h->stream);
                cudaMemcpyAsync(h->step, sS, h->nprob * 4, cudaMemcpyDeviceToDevice, h->stream);
                cudaMemsetAsync(h->queue, 0, 2 * sizeof(int), h->stream);
                cudaEventRecord(e0, h->stream);
                rc = launch_class(h, is_short, c, first, last, 1, h->queue + cls, h->stream);
                cudaEventRecord(e1, h->stream);
                cudaEventSynchronize(e1);
                cudaEventElapsedTime(&ms, e0, e1);
            }
            if (rc == ST_OK && ms < best) { best = ms; best_c = c; }
        }
        if (is_short) h->cfg_short = best_c; else h->cfg_long = best_c;
        if (ms_out) ms_out[cls] = best;
    }
    // restore the state
    cudaMemcpyAsync(h->Q, sQ, 3 * P * 8, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(h->QW, sW, 3 * P * 8, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(h->hyp, sH, 2 * P * 8, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(h->time, sT, h->nprob * 8, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(h->step, sS, h->nprob * 4, cudaMemcpyDeviceToDevice, h->stream);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    release();
    if (rc != ST_OK) return rc;
    if (e != cudaSuccess) return rfail(h, ST_E_CUDA, cudaGetErrorString(e));
    return ST_OK;
}

// line operators on packed arrays (device pointers of the handle's device,
// or host arrays staged here); one problem per CTA, longest class config
static int rad_op(st_radial *h, int op, const double *F, double *O1, double *O2, int iadd, double cadd, int nf_in,
                  int nf_out) {
    if (!h || !F || (!O1 && !O2)) return ST_E_ARG;
    if (cudaSetDevice(h->dev) != cudaSuccess) return rfail(h, ST_E_CUDA, "cudaSetDevice");
    const size_t P = (size_t)h->npts;
    double *buf = nullptr;
    RCUDA(h, cudaMalloc((void **)&buf, (nf_in + 2 * nf_out) * P * 8));
    double *dF = buf, *d1 = buf + nf_in * P, *d2 = d1 + nf_out * P;
    cudaMemcpyAsync(dF, F, nf_in * P * 8, cudaMemcpyDefault, h->stream);
    if (O1) cudaMemcpyAsync(d1, O1, nf_out * P * 8, cudaMemcpyDefault, h->stream);
    int rc = h->nmax <= kShortMax ? launch_op<128, 8>(h, op, dF, d1, d2, iadd, cadd)
                                  : launch_op<512, 8>(h, op, dF, d1, d2, iadd, cadd);
    if (rc == ST_OK) {
        if (O1) cudaMemcpyAsync(O1, d1, nf_out * P * 8, cudaMemcpyDefault, h->stream);
        if (O2) cudaMemcpyAsync(O2, d2, nf_out * P * 8, cudaMemcpyDefault, h->stream);
    }
    cudaError_t e = cudaStreamSynchronize(h->stream);
    cudaFree(buf);
    if (rc != ST_OK) return rc;
    if (e != cudaSuccess) return rfail(h, ST_E_CUDA, cudaGetErrorString(e));
    return ST_OK;
}

int st_radial_dfdx(st_radial *h, const double *F, double *dF, int iadd, double cadd) {
    if (iadd != 0 && iadd != 1) return ST_E_ARG;
    return rad_op(h, OP_D1, F, dF, nullptr, iadd, cadd, 1, 1);
}
int st_radial_d2fdx2(st_radial *h, const double *F, double *dF, double *d2F, int iadd) {
    if (!d2F || (iadd && !dF)) return ST_E_ARG;
    return rad_op(h, OP_D2, F, iadd ? dF : nullptr, d2F, iadd, 1.0, 1, 1);
}
int st_radial_compact_filter_x(st_radial *h, const double *F, double *F0) {
    return rad_op(h, OP_FILT, F, F0, nullptr, 0, 1.0, 1, 1);
}
int st_radial_gaussian_filter_x(st_radial *h, const double *F, double *Fg) {
    return rad_op(h, OP_GAUSS, F, Fg, nullptr, 0, 1.0, 1, 1);
}
int st_radial_rhs(st_radial *h, const double *Q, double *Qrhs) {
    return rad_op(h, OP_RHS, Q, Qrhs, nullptr, 0, 1.0, 3, 3);
}
int st_radial_rhs_hyper(st_radial *h, const double *Q, double *Qrhs) {
    return rad_op(h, OP_HYPER, Q, Qrhs, nullptr, 0, 1.0, 3, 3);
}
int st_radial_launch_count(const st_radial *h, long long *count) {
    if (!h || !count) return ST_E_ARG;
    *count = h->launches;
    return ST_OK;
}

}  // extern "C"
