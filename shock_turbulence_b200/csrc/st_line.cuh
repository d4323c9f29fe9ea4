// st_line.cuh - device building blocks of the line operators.
//
// Work decomposition ("columns"): a CTA owns 16 neighbouring lines of one
// direction; thread t works on line t%16 and on the rows [s*S, s*S+S) of
// segment s = t/16, held in registers (a warp holds two adjacent segments).
// Consequences:
//  - for x and z lines 16 threads touch 16 adjacent doubles of every row, so
//    every global access is a full 128-byte transaction;
//  - the 16 threads of a segment are on the same row, so the LU-table reads
//    are uniform per half-warp (two broadcasts per warp);
//  - boundary rows belong to the first and last segments only;
//  - 512-thread CTAs at 64 registers let two CTAs share an SM, so one CTA's
//    loads overlap the other's solve;
//  - segments exchange their end values through shared memory once per
//    recurrence direction; the carry into each segment is a fixed linear
//    combination of those values (tables wf/wb, mf/mb).
#pragma once
#include "st_internal.h"

namespace st {

// element (lane, row) of a CTA's 32 lines is base + lane*lstride + row*rstride
struct ColMap {
    size_t base, lstride, rstride;
};
struct LineGeo {
    int dir, n, My, Mz;
    __device__ __forceinline__ ColMap map(unsigned blk) const {
        ColMap m;
        const size_t sMy = My, sMz = Mz, jb = My / kLanes;
        if (dir == 0) {            // lines (j,k): 32 consecutive j at one k
            m.base = (blk % jb) * kLanes + sMy * (blk / jb); m.lstride = 1; m.rstride = sMy * sMz;
        } else if (dir == 1) {     // lines (k,i): 32 consecutive lines, each contiguous
            m.base = sMy * (size_t)blk * kLanes; m.lstride = sMy; m.rstride = 1;
        } else {                   // lines (j,i): 32 consecutive j at one i
            m.base = (blk % jb) * kLanes + sMy * sMz * (blk / jb); m.lstride = 1; m.rstride = sMy;
        }
        return m;
    }
};

// The producer's fields are double or float (FP32 mode); values are
// converted to double as they are loaded and every operation is in double.
template <class T>
__device__ __forceinline__ double ld(const T *p) { return (double)__ldg(p); }

template <int OP, class T>
__device__ __forceinline__ double prod_eval(const ProdT<T> &P, size_t i) {
    if constexpr (OP == PR_MUL) {
        return ld(P.a + i) * ld(P.b + i);
    } else if constexpr (OP == PR_ADDMUL) {
        return (ld(P.a + i) + ld(P.b + i)) * ld(P.c + i);
    } else if constexpr (OP == PR_MULMUL) {
        return ld(P.c + i) * (ld(P.a + i) * ld(P.b + i));
    } else if constexpr (OP == PR_SPEC) {
        double a = ld(P.a + i), b = ld(P.b + i), c = ld(P.c + i);
        return a * b * c + a * c * P.k0 * P.k1;
    } else if constexpr (OP == PR_SPECT) {
        double a = ld(P.a + i), b = ld(P.b + i), c = ld(P.c + i), d = ld(P.d + i);
        double fl = a * b * c + a * c * P.k0 * P.k1;
        return P.k2 * d * fl;
    } else {
        return ld(P.a + i);
    }
}

// row index of a halo row: wrapped around the line for periodic lines,
// otherwise clamped into the line (clamped values are never used by the
// stencils, whose boundary rows re-read what they need)
__device__ __forceinline__ int halo_row(int row, int n, int cyc) {
    return row < 0 ? (cyc ? row + n : 0) : (row > n - 1 ? (cyc ? row - n : n - 1) : row);
}

// rows a-H .. a+S+H-1 of this lane's line into v
template <int S, int H, int OP, class T>
__device__ __forceinline__ void load_rows(double (&v)[S + 2 * H], const ProdT<T> &F, const ColMap &m, int lane,
                                          int a, int n, int cyc) {
    const size_t p = m.base + (size_t)lane * m.lstride;
#pragma unroll
    for (int q = 0; q < S + 2 * H; q++) {
        int row = halo_row(a - H + q, n, cyc);
        v[q] = prod_eval<OP>(F, p + (size_t)row * m.rstride);
    }
}

template <int S, int N, class T>
__device__ __forceinline__ void store_rows(const double (&r)[N], T *__restrict__ O, const ColMap &m,
                                           int lane, int a, int add) {
    T *p = O + m.base + (size_t)lane * m.lstride + (size_t)a * m.rstride;
    if (add) {
        double prev[S];
#pragma unroll
        for (int t = 0; t < S; t++) prev[t] = (double)p[(size_t)t * m.rstride];
#pragma unroll
        for (int t = 0; t < S; t++) p[(size_t)t * m.rstride] = (T)(prev[t] + r[t]);
    } else {
#pragma unroll
        for (int t = 0; t < S; t++) p[(size_t)t * m.rstride] = (T)r[t];
    }
}

// shared buffers for the segment end values of one solve, and the corner
// values of a periodic line (rows 0, 1, n-2, n-1 of the banded solution)
struct CarryBuf {
    double a[kMaxSeg][kLanes][2];
    double b[kMaxSeg][kLanes][2];
    double cy[kLanes][4];
};

// ---- periodic lines: corner correction after the banded solve ------------
// x_i = y_i - sum_k K_ik y_{j_k} with the corner rows j = {0, n-1} (K = 2,
// tridiagonal) or {0, 1, n-2, n-1} (K = 4, pentadiagonal); the table holds
// -K row-major.  The first and last segments publish the corner values; the
// barrier also orders them after every read of the previous solve's cy.
template <int S, int N, int KC>
__device__ __forceinline__ void cyc_fix(double (&r)[N], const double *__restrict__ Kt, int s, int P, int lane,
                                        CarryBuf &cb) {
    if (KC == 2) {
        if (s == 0) cb.cy[lane][0] = r[0];
        if (s == P - 1) cb.cy[lane][1] = r[S - 1];
    } else {
        if (s == 0) { cb.cy[lane][0] = r[0]; cb.cy[lane][1] = r[1]; }
        if (s == P - 1) { cb.cy[lane][2] = r[S - 2]; cb.cy[lane][3] = r[S - 1]; }
    }
    __syncthreads();
    double y[KC];
#pragma unroll
    for (int k = 0; k < KC; k++) y[k] = cb.cy[lane][k];
    const double *kr = Kt + (size_t)s * S * KC;
#pragma unroll
    for (int t = 0; t < S; t++) {
        double v = r[t];
#pragma unroll
        for (int k = 0; k < KC; k++) v = fma(__ldg(kr + t * KC + k), y[k], v);
        r[t] = v;
    }
}

// ---- segmented constant-coefficient tridiagonal solve --------------------
// Forward elimination r'_i = r_i - l_i r'_{i-1} and back substitution
// x_i = (r'_i - c_i x_{i+1}) / (b'_i + tiny) of tridiagonal_serial
// (src/tridiagonal.f90:274-284) per segment with zero carries, then the
// carry corrections.  Caller guarantees cb is free (synchronised).
template <int S, int N>
__device__ __forceinline__ void tri_solve(double (&r)[N], const TriTab &T, int s, int P, int lane,
                                          CarryBuf &cb) {
    const int a = s * S;
#pragma unroll
    for (int t = 1; t < S; t++) r[t] = r[t] - r[t - 1] * __ldg(T.l + a + t);
    cb.a[s][lane][0] = r[S - 1];
    __syncthreads();
    double cin = 0.0;
    for (int sp = max(0, s - T.kf); sp < s; sp++) cin = fma(__ldg(T.wf + sp * P + s), cb.a[sp][lane][0], cin);
#pragma unroll
    for (int t = 0; t < S; t++) r[t] = fma(__ldg(T.g + a + t), cin, r[t]);
    r[S - 1] = r[S - 1] * __ldg(T.id + a + S - 1);
#pragma unroll
    for (int t = S - 2; t >= 0; t--) r[t] = (r[t] - __ldg(T.up + a + t) * r[t + 1]) * __ldg(T.id + a + t);
    cb.b[s][lane][0] = r[0];
    __syncthreads();
    double ein = 0.0;
    for (int sp = s + 1, se = min(P, s + 1 + T.kb); sp < se; sp++)
        ein = fma(__ldg(T.wb + sp * P + s), cb.b[sp][lane][0], ein);
#pragma unroll
    for (int t = 0; t < S; t++) r[t] = fma(__ldg(T.h + a + t), ein, r[t]);
}

// ---- segmented constant-coefficient pentadiagonal solve ------------------
// Elimination order of pentadiagonal_serial (src/pentadiagonal.f90:340-372):
// r'_i = (r_i - k2 r'_{i-2}) - k1 r'_{i-1};  x_i = ((r'_i - D'_i x_{i+1})
// - E_i x_{i+2}) / (C'_i + tiny).  Carries are 2-vectors.
template <int S, int N>
__device__ __forceinline__ void pen_solve(double (&r)[N], const PenTab &T, int s, int P, int lane,
                                          CarryBuf &cb) {
    const int a = s * S;
#pragma unroll
    for (int t = 1; t < S; t++) {
        double v = r[t];
        if (t >= 2) v = v - __ldg(T.p2 + a + t) * r[t >= 2 ? t - 2 : 0];
        v = v - __ldg(T.p1 + a + t) * r[t - 1];
        r[t] = v;
    }
    cb.a[s][lane][0] = r[S - 1];
    cb.a[s][lane][1] = (S >= 2) ? r[S >= 2 ? S - 2 : 0] : 0.0;
    __syncthreads();
    double c1 = 0.0, c2 = 0.0;
    for (int sp = max(0, s - T.kf); sp < s; sp++) {
        const double *m = T.mf + ((size_t)sp * P + s) * 4;
        double a1 = cb.a[sp][lane][0], a2 = cb.a[sp][lane][1];
        c1 = fma(__ldg(m + 0), a1, fma(__ldg(m + 1), a2, c1));
        c2 = fma(__ldg(m + 2), a1, fma(__ldg(m + 3), a2, c2));
    }
#pragma unroll
    for (int t = 0; t < S; t++) r[t] = fma(__ldg(T.g1 + a + t), c1, fma(__ldg(T.g2 + a + t), c2, r[t]));
#pragma unroll
    for (int t = S - 1; t >= 0; t--) {
        double v = r[t];
        if (t + 1 < S) v = v - __ldg(T.q1 + a + t) * r[t + 1 < S ? t + 1 : t];
        if (t + 2 < S) v = v - __ldg(T.q2 + a + t) * r[t + 2 < S ? t + 2 : t];
        r[t] = v * __ldg(T.id + a + t);
    }
    cb.b[s][lane][0] = r[0];
    cb.b[s][lane][1] = (S >= 2) ? r[S >= 2 ? 1 : 0] : 0.0;
    __syncthreads();
    double e1 = 0.0, e2 = 0.0;
    for (int sp = s + 1, se = min(P, s + 1 + T.kb); sp < se; sp++) {
        const double *m = T.mb + ((size_t)sp * P + s) * 4;
        double b1 = cb.b[sp][lane][0], b2 = cb.b[sp][lane][1];
        e1 = fma(__ldg(m + 0), b1, fma(__ldg(m + 1), b2, e1));
        e2 = fma(__ldg(m + 2), b1, fma(__ldg(m + 3), b2, e2));
    }
#pragma unroll
    for (int t = 0; t < S; t++) r[t] = fma(__ldg(T.h1 + a + t), e1, fma(__ldg(T.h2 + a + t), e2, r[t]));
}

// ---- explicit right-hand sides ------------------------------------------
// v holds rows a-H .. a+S+H-1 on entry; the RHS of row a+t is written into
// v[t] (in place, ascending t: row a+t only needs v[t..t+2H]).  Rows follow
// the reference formulas term by term (Fortran evaluates left to right).
// Boundary rows belong to the first/last segment only: those warps re-read
// the few rows they need from global memory (warp-uniform branch).
template <int OP, class T = double>
struct RowReader {
    const double *tile;       // shared tile row (y lines) or null
    const ProdT<T> *F;        // global producer (x, z lines)
    size_t base, rstride;
    __device__ __forceinline__ double operator()(int row) const {
        return tile ? tile[row] : prod_eval<OP>(*F, base + (size_t)row * rstride);
    }
};

// ---- y lines: staging through shared memory ------------------------------
// The 32 lines of a y CTA are one contiguous block of 32*n doubles.  They
// are copied with 16-byte coalesced accesses into a [32][n+1] tile (odd
// stride: lane l reading row r of line l hits bank (l*(n+1)+r) mod 32, all
// distinct), so that each thread reads its segment conflict-free.
template <int OP, class T>
__device__ __forceinline__ void ytile_load(double *tile, const ProdT<T> &F, size_t base, int n) {
    const int half = kLanes * n / 2;
    if (sizeof(T) == 8 && OP == PR_A && ((reinterpret_cast<uintptr_t>(F.a + base) & 15) == 0)) {
        if constexpr (sizeof(T) == 8) {
            const double2 *src = reinterpret_cast<const double2 *>(F.a + base);
            for (int q = threadIdx.x; q < half; q += blockDim.x) {
                double2 d = __ldg(src + q);
                int e = 2 * q, line = e / n, row = e - line * n;
                tile[line * (n + 1) + row] = d.x;
                tile[line * (n + 1) + row + 1] = d.y;
            }
        }
    } else {
        for (int q = threadIdx.x; q < 2 * half; q += blockDim.x) {
            int line = q / n, row = q - line * n;
            tile[line * (n + 1) + row] = prod_eval<OP>(F, base + q);
        }
    }
}
template <class T>
__device__ __forceinline__ void ytile_store(const double *tile, T *__restrict__ O, size_t base, int n,
                                            int add) {
    if (sizeof(T) != 8 || (reinterpret_cast<uintptr_t>(O + base) & 15)) {
        for (int q = threadIdx.x; q < kLanes * n; q += blockDim.x) {
            int line = q / n, row = q - line * n;
            double v = tile[line * (n + 1) + row];
            O[base + q] = (T)(add ? (double)O[base + q] + v : v);
        }
        return;
    }
    if constexpr (sizeof(T) == 8) {
        double2 *dst = reinterpret_cast<double2 *>(O + base);
        const int half = kLanes * n / 2;
        for (int q = threadIdx.x; q < half; q += blockDim.x) {
            int e = 2 * q, line = e / n, row = e - line * n;
            double2 d = make_double2(tile[line * (n + 1) + row], tile[line * (n + 1) + row + 1]);
            if (add) {
                double2 o = dst[q];
                d.x = o.x + d.x;
                d.y = o.y + d.y;
            }
            dst[q] = d;
        }
    }
}
template <int S, int H>
__device__ __forceinline__ void ytile_rows(double (&v)[S + 2 * H], const double *tile, int lane, int a, int n,
                                           int cyc) {
    const double *p = tile + lane * (n + 1);
#pragma unroll
    for (int q = 0; q < S + 2 * H; q++) v[q] = p[halo_row(a - H + q, n, cyc)];
}
template <int S, int N>
__device__ __forceinline__ void ytile_put(double *tile, const double (&r)[N], int lane, int a, int n) {
    double *p = tile + lane * (n + 1) + a;
#pragma unroll
    for (int t = 0; t < S; t++) p[t] = r[t];
}

// DFDX_sym/_asym RHS, src/derivCDopt6_sym_tri.f:458-514,
// src/derivCDopt6_asym_tri.f:461-516  (H = 2).  Periodic DFDX,
// src/derivCDopt6_periodic.f:205-248: the interior formula on every row with
// wrapped halos (its f(i+-3) weight c1 is zero for the FDL3DI set).
template <int S, int H, class RD>
__device__ __forceinline__ void rhs_d1(double (&v)[S + 2 * H], int a, int n, int asym, int cyc, double fac,
                                       const Consts &K, const RD &F) {
#pragma unroll
    for (int t = 0; t < S; t++) {
        auto f = [&](int k) { return v[t + k + H]; };
        v[t] = fac * (K.b1 * (f(2) - f(-2)) + K.a1 * (f(1) - f(-1)));
    }
    if (!cyc && (a < 2 || a + S > n - 2)) {
#pragma unroll
        for (int t = 0; t < S; t++) {
            const int i = a + t;
            auto f = [&](int k) { return F(i + k); };
            if (i == 0) v[t] = asym ? fac * (K.b1 * (f(2) + f(2)) + K.a1 * (f(1) + f(1))) : 0.0;
            else if (i == 1) v[t] = asym ? fac * (K.b1 * (f(2) + f(0)) + K.a1 * (f(1) - f(-1)))
                                         : fac * (K.b1 * (f(2) - f(0)) + K.a1 * (f(1) - f(-1)));
            else if (i == n - 2)
                v[t] = fac * (K.closure1 * f(1) + 5.0e-1 * f(0) - f(-1) - K.closure2 * f(-2));
            else if (i == n - 1) v[t] = fac * (2.5 * f(0) - 2.0 * f(-1) - 5.0e-1 * f(-2));
        }
    }
}

// D2FDX2_sym/_asym RHS, src/derivCDopt6_sym_tri.f:587-645,
// src/derivCDopt6_asym_tri.f:588-643  (H = 2).  Periodic D2FDX2,
// src/derivCDopt6_periodic.f:316-370, with zero f(i+-3) weight and centre
// weight 2(a2+b2).
template <int S, int H, class RD>
__device__ __forceinline__ void rhs_d2(double (&v)[S + 2 * H], int a, int n, int asym, int cyc, double fac,
                                       const Consts &K, const RD &F) {
#pragma unroll
    for (int t = 0; t < S; t++) {
        auto f = [&](int k) { return v[t + k + H]; };
        v[t] = fac * (K.b2 * (f(2) + f(-2)) + K.a2 * (f(1) + f(-1)) - K.c2 * f(0));
    }
    if (!cyc && (a < 2 || a + S > n - 2)) {
#pragma unroll
        for (int t = 0; t < S; t++) {
            const int i = a + t;
            auto f = [&](int k) { return F(i + k); };
            if (i == 0) v[t] = asym ? 0.0 : fac * (K.b2 * 2.0 * (f(2) - f(0)) + K.a2 * 2.0 * (f(1) - f(0)));
            else if (i == 1)
                v[t] = asym ? fac * (K.b2 * (f(2) - 3.0 * f(0)) + K.a2 * (f(1) - 2.0 * f(0)))
                            : fac * (K.b2 * (f(2) - 2.0 * f(0) + f(0)) + K.a2 * (f(1) - 2.0 * f(0) + f(-1)));
            else if (i == n - 2)
                v[t] = fac * (1.2375 * f(1) - 3.0 * f(0) + 2.325 * f(-1) - 6.0e-1 * f(-2) + 3.75e-2 * f(-3));
            else if (i == n - 1) v[t] = fac * (1.3e1 * f(0) - 2.7e1 * f(-1) + 1.5e1 * f(-2) - f(-3));
        }
    }
}

// Compact_Filter_X_sym/_asym RHS, src/filters_sym.f:483-616,
// src/filters_asym.f:435-565  (H = 4).  Periodic Compact_Filter_X,
// src/filters_periodic.f:155-229: interior formula, wrapped halos.
template <int S, int H, class RD>
__device__ __forceinline__ void rhs_filter(double (&v)[S + 2 * H], int a, int n, int asym, int cyc,
                                           const Consts &K, const RD &F) {
#pragma unroll
    for (int t = 0; t < S; t++) {
        auto f = [&](int k) { return v[t + k + H]; };
        v[t] = K.fa4 * (f(4) + f(-4)) + K.fa3 * (f(3) + f(-3)) + K.fa2 * (f(2) + f(-2)) +
               K.fa1 * (f(1) + f(-1)) + K.fa0 * f(0);
    }
    if (!cyc && (a < 4 || a + S > n - 4)) {
#pragma unroll
        for (int t = 0; t < S; t++) {
            const int i = a + t;
            auto f = [&](int k) { return F(i + k); };
            double w = v[t];
            if (!asym) {
                if (i == 0) w = K.fa4 * (2.0 * f(4)) + K.fa3 * (2.0 * f(3)) + K.fa2 * (2.0 * f(2)) +
                                K.fa1 * (2.0 * f(1)) + K.fa0 * f(0);
                else if (i == 1) w = K.fa4 * (f(2) + f(4)) + K.fa3 * (f(1) + f(3)) + K.fa2 * (f(0) + f(2)) +
                                     K.fa1 * (f(-1) + f(1)) + K.fa0 * f(0);
                else if (i == 2) w = K.fa4 * (f(0) + f(4)) + K.fa3 * (f(-1) + f(3)) + K.fa2 * (f(-2) + f(2)) +
                                     K.fa1 * (f(-1) + f(1)) + K.fa0 * f(0);
                else if (i == 3) w = K.fa4 * (f(-2) + f(4)) + K.fa3 * (f(-3) + f(3)) + K.fa2 * (f(-2) + f(2)) +
                                     K.fa1 * (f(-1) + f(1)) + K.fa0 * f(0);
            } else {
                if (i == 0) w = 0.0;
                else if (i == 1) w = K.fa4 * (f(4) - f(2)) + K.fa3 * (f(3) - f(1)) + K.fa2 * (f(2) - f(0)) +
                                     K.fa1 * (f(-1) + f(1)) + K.fa0 * f(0);
                else if (i == 2) w = K.fa4 * (f(4) - f(0)) + K.fa3 * (f(3) - f(-1)) + K.fa2 * (f(-2) + f(2)) +
                                     K.fa1 * (f(-1) + f(1)) + K.fa0 * f(0);
                else if (i == 3) w = K.fa4 * (f(4) - f(-2)) + K.fa3 * (f(-3) + f(3)) + K.fa2 * (f(-2) + f(2)) +
                                     K.fa1 * (f(-1) + f(1)) + K.fa0 * f(0);
            }
            if (i == n - 1) w = K.bc1[1] * f(0) + K.bc1[2] * f(-1) + K.bc1[3] * f(-2) + K.bc1[4] * f(-3) +
                                K.bc1[5] * f(-4);
            else if (i == n - 2) w = K.bc2[1] * f(1) + K.bc2[2] * f(0) + K.bc2[3] * f(-1) + K.bc2[4] * f(-2) +
                                     K.bc2[5] * f(-3);
            else if (i == n - 3) w = K.bc3[2] * f(-2) + K.bc3[1] * f(-1) + K.bc3[0] * f(0) + K.bc3[1] * f(1) +
                                     K.bc3[2] * f(2);
            else if (i == n - 4) w = K.bc4[3] * f(-3) + K.bc4[2] * f(-2) + K.bc4[1] * f(-1) + K.bc4[0] * f(0) +
                                     K.bc4[1] * f(1) + K.bc4[2] * f(2) + K.bc4[3] * f(3);
            v[t] = w;
        }
    }
}

// Gaussian_Filter_X, src/filters_sym.f:1119-1212: explicit, symmetric low end,
// last four points copied  (H = 4).  Periodic family,
// src/filters_periodic.f:601-675: interior formula, wrapped halos.
template <int S, int H, class RD>
__device__ __forceinline__ void rhs_gauss(double (&v)[S + 2 * H], int a, int n, int cyc, const Consts &K,
                                          const RD &F) {
    const double *g = K.ga;
#pragma unroll
    for (int t = 0; t < S; t++) {
        auto f = [&](int k) { return v[t + k + H]; };
        v[t] = g[4] * (f(4) + f(-4)) + g[3] * (f(3) + f(-3)) + g[2] * (f(2) + f(-2)) + g[1] * (f(1) + f(-1)) +
               g[0] * f(0);
    }
    if (!cyc && (a < 4 || a + S > n - 4)) {
#pragma unroll
        for (int t = 0; t < S; t++) {
            const int i = a + t;
            auto f = [&](int k) { return F(i + k); };
            if (i == 0) v[t] = g[4] * (2.0 * f(4)) + g[3] * (2.0 * f(3)) + g[2] * (2.0 * f(2)) +
                               g[1] * (2.0 * f(1)) + g[0] * f(0);
            else if (i == 1) v[t] = g[4] * (f(2) + f(4)) + g[3] * (f(1) + f(3)) + g[2] * (f(0) + f(2)) +
                                    g[1] * (f(-1) + f(1)) + g[0] * f(0);
            else if (i == 2) v[t] = g[4] * (f(0) + f(4)) + g[3] * (f(-1) + f(3)) + g[2] * (f(-2) + f(2)) +
                                    g[1] * (f(-1) + f(1)) + g[0] * f(0);
            else if (i == 3) v[t] = g[4] * (f(-2) + f(4)) + g[3] * (f(-3) + f(3)) + g[2] * (f(-2) + f(2)) +
                                    g[1] * (f(-1) + f(1)) + g[0] * f(0);
            if (i >= n - 4) v[t] = f(0);
        }
    }
}

}  // namespace st
