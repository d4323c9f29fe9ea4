// st_line.cuh - device building blocks of the line operators.
//
// Work decomposition: one warp owns one grid line of n = 32*S points; lane s
// owns the contiguous rows [s*S, s*S+S) in registers.  Lines are staged in
// shared memory with one padding double after every segment, so that the 32
// lanes reading "their" row t hit 32 different banks (row stride S+1).
#pragma once
#include "st_internal.h"

namespace st {

constexpr unsigned kFull = 0xffffffffu;

// shared-memory geometry of one staged line
template <int S>
struct LineGeom {
    static constexpr int kPadL = 8 * (S + 1);          // room for out-of-line stencil reads
    static constexpr int kBody = kSeg * (S + 1);
    static constexpr int kStride = kPadL + kBody + 8 * (S + 1) + 1;   // odd stride
    __device__ static int pos(int row) { return kPadL + (row / S) * (S + 1) + (row % S); }
};

// value of row (lane*S + u) of a staged line; u is a compile-time constant
// after unrolling, so the segment jump folds to a constant offset.
template <int S>
__device__ __forceinline__ double ldrow(const double *line, int lane, int u) {
    const int q = (u >= 0) ? u / S : -((-u + S - 1) / S);
    const int off = u - q * S;
    return line[LineGeom<S>::kPadL + (lane + q) * (S + 1) + off];
}

// ---- segmented constant-coefficient tridiagonal solve --------------------
// Forward elimination r'_i = r_i - l_i r'_{i-1} and back substitution
// x_i = (r'_i - c_i x_{i+1}) / (b'_i + tiny) of tridiagonal_serial
// (src/tridiagonal.f90:274-284), run per segment with zero carries, then
// corrected by the carries that a warp scan of the segment maps produces.
template <int S>
__device__ __forceinline__ void tri_solve(double (&r)[S], const TriTab &T, int lane) {
    const int a = lane * S;
#pragma unroll
    for (int t = 1; t < S; t++) r[t] = r[t] - r[t - 1] * __ldg(T.l + a + t);
    double A = r[S - 1];
#pragma unroll
    for (int k = 0; k < kScanSteps; k++) {
        const int off = 1 << k;
        double o = __shfl_up_sync(kFull, A, off);
        if (lane >= off) A = fma(__ldg(T.bk + lane * kScanSteps + k), o, A);
    }
    double cin = __shfl_up_sync(kFull, A, 1);
    if (lane == 0) cin = 0.0;
#pragma unroll
    for (int t = 0; t < S; t++) r[t] = fma(__ldg(T.g + a + t), cin, r[t]);
    r[S - 1] = r[S - 1] * __ldg(T.id + a + S - 1);
#pragma unroll
    for (int t = S - 2; t >= 0; t--) r[t] = (r[t] - __ldg(T.up + a + t) * r[t + 1]) * __ldg(T.id + a + t);
    double F = r[0];
#pragma unroll
    for (int k = 0; k < kScanSteps; k++) {
        const int off = 1 << k;
        double o = __shfl_down_sync(kFull, F, off);
        if (lane + off < kSeg) F = fma(__ldg(T.gk + lane * kScanSteps + k), o, F);
    }
    double ein = __shfl_down_sync(kFull, F, 1);
    if (lane == kSeg - 1) ein = 0.0;
#pragma unroll
    for (int t = 0; t < S; t++) r[t] = fma(__ldg(T.h + a + t), ein, r[t]);
}

// ---- segmented constant-coefficient pentadiagonal solve ------------------
// Elimination order of pentadiagonal_serial (src/pentadiagonal.f90:340-372):
// r'_i = (r_i - k2 r'_{i-2}) - k1 r'_{i-1};  x_i = ((r'_i - D'_i x_{i+1})
// - E_i x_{i+2}) / (C'_i + tiny).  Carries are 2-vectors.
template <int S>
__device__ __forceinline__ void pen_solve(double (&r)[S], const PenTab &T, int lane) {
    const int a = lane * S;
#pragma unroll
    for (int t = 1; t < S; t++) {
        double v = r[t];
        if (t >= 2) v = v - __ldg(T.p2 + a + t) * r[t - 2];
        v = v - __ldg(T.p1 + a + t) * r[t - 1];
        r[t] = v;
    }
    double A1 = r[S - 1], A2 = (S >= 2) ? r[S >= 2 ? S - 2 : 0] : 0.0;
#pragma unroll
    for (int k = 0; k < kScanSteps; k++) {
        const int off = 1 << k;
        double o1 = __shfl_up_sync(kFull, A1, off);
        double o2 = __shfl_up_sync(kFull, A2, off);
        if (lane >= off) {
            const double *m = T.mk + (lane * kScanSteps + k) * 4;
            double n1 = fma(__ldg(m + 0), o1, fma(__ldg(m + 1), o2, A1));
            double n2 = fma(__ldg(m + 2), o1, fma(__ldg(m + 3), o2, A2));
            A1 = n1; A2 = n2;
        }
    }
    double c1 = __shfl_up_sync(kFull, A1, 1), c2 = __shfl_up_sync(kFull, A2, 1);
    if (lane == 0) { c1 = 0.0; c2 = 0.0; }
#pragma unroll
    for (int t = 0; t < S; t++) r[t] = fma(__ldg(T.g1 + a + t), c1, fma(__ldg(T.g2 + a + t), c2, r[t]));
#pragma unroll
    for (int t = S - 1; t >= 0; t--) {
        double v = r[t];
        if (t + 1 < S) v = v - __ldg(T.q1 + a + t) * r[t + 1 < S ? t + 1 : t];
        if (t + 2 < S) v = v - __ldg(T.q2 + a + t) * r[t + 2 < S ? t + 2 : t];
        r[t] = v * __ldg(T.id + a + t);
    }
    double B1 = r[0], B2 = (S >= 2) ? r[S >= 2 ? 1 : 0] : 0.0;
#pragma unroll
    for (int k = 0; k < kScanSteps; k++) {
        const int off = 1 << k;
        double o1 = __shfl_down_sync(kFull, B1, off);
        double o2 = __shfl_down_sync(kFull, B2, off);
        if (lane + off < kSeg) {
            const double *m = T.nk + (lane * kScanSteps + k) * 4;
            double n1 = fma(__ldg(m + 0), o1, fma(__ldg(m + 1), o2, B1));
            double n2 = fma(__ldg(m + 2), o1, fma(__ldg(m + 3), o2, B2));
            B1 = n1; B2 = n2;
        }
    }
    double e1 = __shfl_down_sync(kFull, B1, 1), e2 = __shfl_down_sync(kFull, B2, 1);
    if (lane == kSeg - 1) { e1 = 0.0; e2 = 0.0; }
#pragma unroll
    for (int t = 0; t < S; t++) r[t] = fma(__ldg(T.h1 + a + t), e1, fma(__ldg(T.h2 + a + t), e2, r[t]));
}

// ---- explicit right-hand sides ------------------------------------------
// Rows follow the reference formulas term by term (Fortran evaluates
// left to right); f(k) is the value k rows away from row i.

// DFDX_sym/_asym RHS, src/derivCDopt6_sym_tri.f:458-514,
// src/derivCDopt6_asym_tri.f:461-516
template <int S>
__device__ __forceinline__ void rhs_d1(double (&r)[S], const double *line, int lane, int n, int asym,
                                       double fac, const Consts &K) {
#pragma unroll
    for (int t = 0; t < S; t++) {
        auto f = [&](int k) { return ldrow<S>(line, lane, t + k); };
        const int i = lane * S + t;
        double w = fac * (K.b1 * (f(2) - f(-2)) + K.a1 * (f(1) - f(-1)));
        if (i < 2 || i >= n - 2) {
            if (i == 0) w = asym ? fac * (K.b1 * (f(2) + f(2)) + K.a1 * (f(1) + f(1))) : 0.0;
            else if (i == 1) w = asym ? fac * (K.b1 * (f(2) + f(0)) + K.a1 * (f(1) - f(-1)))
                                      : fac * (K.b1 * (f(2) - f(0)) + K.a1 * (f(1) - f(-1)));
            else if (i == n - 2)
                w = fac * (K.closure1 * f(1) + 5.0e-1 * f(0) - f(-1) - K.closure2 * f(-2));
            else w = fac * (2.5 * f(0) - 2.0 * f(-1) - 5.0e-1 * f(-2));
        }
        r[t] = w;
    }
}

// D2FDX2_sym/_asym RHS, src/derivCDopt6_sym_tri.f:587-645,
// src/derivCDopt6_asym_tri.f:588-643
template <int S>
__device__ __forceinline__ void rhs_d2(double (&r)[S], const double *line, int lane, int n, int asym,
                                       double fac, const Consts &K) {
#pragma unroll
    for (int t = 0; t < S; t++) {
        auto f = [&](int k) { return ldrow<S>(line, lane, t + k); };
        const int i = lane * S + t;
        double w = fac * (K.b2 * (f(2) + f(-2)) + K.a2 * (f(1) + f(-1)) - K.c2 * f(0));
        if (i < 2 || i >= n - 2) {
            if (i == 0) w = asym ? 0.0 : fac * (K.b2 * 2.0 * (f(2) - f(0)) + K.a2 * 2.0 * (f(1) - f(0)));
            else if (i == 1)
                w = asym ? fac * (K.b2 * (f(2) - 3.0 * f(0)) + K.a2 * (f(1) - 2.0 * f(0)))
                         : fac * (K.b2 * (f(2) - 2.0 * f(0) + f(0)) + K.a2 * (f(1) - 2.0 * f(0) + f(-1)));
            else if (i == n - 2)
                w = fac * (1.2375 * f(1) - 3.0 * f(0) + 2.325 * f(-1) - 6.0e-1 * f(-2) + 3.75e-2 * f(-3));
            else w = fac * (1.3e1 * f(0) - 2.7e1 * f(-1) + 1.5e1 * f(-2) - f(-3));
        }
        r[t] = w;
    }
}

// Compact_Filter_X_sym/_asym RHS, src/filters_sym.f:483-616,
// src/filters_asym.f:435-565
template <int S>
__device__ __forceinline__ void rhs_filter(double (&r)[S], const double *line, int lane, int n, int asym,
                                           const Consts &K) {
#pragma unroll
    for (int t = 0; t < S; t++) {
        auto f = [&](int k) { return ldrow<S>(line, lane, t + k); };
        const int i = lane * S + t;
        double w = K.fa4 * (f(4) + f(-4)) + K.fa3 * (f(3) + f(-3)) + K.fa2 * (f(2) + f(-2)) +
                   K.fa1 * (f(1) + f(-1)) + K.fa0 * f(0);
        if (i < 4 || i >= n - 4) {
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
        }
        r[t] = w;
    }
}

// Gaussian_Filter_X, src/filters_sym.f:1119-1212: explicit, symmetric low end,
// last four points copied
template <int S>
__device__ __forceinline__ void rhs_gauss(double (&r)[S], const double *line, int lane, int n,
                                          const Consts &K) {
    const double *g = K.ga;
#pragma unroll
    for (int t = 0; t < S; t++) {
        auto f = [&](int k) { return ldrow<S>(line, lane, t + k); };
        const int i = lane * S + t;
        double w = g[4] * (f(4) + f(-4)) + g[3] * (f(3) + f(-3)) + g[2] * (f(2) + f(-2)) +
                   g[1] * (f(1) + f(-1)) + g[0] * f(0);
        if (i < 4 || i >= n - 4) {
            if (i == 0) w = g[4] * (2.0 * f(4)) + g[3] * (2.0 * f(3)) + g[2] * (2.0 * f(2)) +
                            g[1] * (2.0 * f(1)) + g[0] * f(0);
            else if (i == 1) w = g[4] * (f(2) + f(4)) + g[3] * (f(1) + f(3)) + g[2] * (f(0) + f(2)) +
                                 g[1] * (f(-1) + f(1)) + g[0] * f(0);
            else if (i == 2) w = g[4] * (f(0) + f(4)) + g[3] * (f(-1) + f(3)) + g[2] * (f(-2) + f(2)) +
                                 g[1] * (f(-1) + f(1)) + g[0] * f(0);
            else if (i == 3) w = g[4] * (f(-2) + f(4)) + g[3] * (f(-3) + f(3)) + g[2] * (f(-2) + f(2)) +
                                 g[1] * (f(-1) + f(1)) + g[0] * f(0);
            if (i >= n - 4) w = f(0);
        }
        r[t] = w;
    }
}

// ---- line tiles -----------------------------------------------------------
// A CTA of W warps stages W lines of direction d.  Lines are numbered so
// that W consecutive lines are W consecutive addresses (x, z) or W
// consecutive contiguous lines (y):
//   x: L = j + My*k,  element (L,i) at L + My*Mz*i
//   y: L = k + Mz*i,  element (L,j) at My*L + j
//   z: L = j + My*i,  element (L,k) at (L%My) + My*Mz*(L/My) + My*k
struct LineMap {
    int dir, n, My, Mz;
    __device__ __forceinline__ size_t addr(size_t L, int row) const {
        if (dir == 0) return L + (size_t)My * Mz * row;
        if (dir == 1) return (size_t)My * L + row;
        return (L % My) + (size_t)My * Mz * (L / My) + (size_t)My * row;
    }
};

// cooperative coalesced load of W lines into padded shared memory
template <int S, int W>
__device__ __forceinline__ void tile_load(double *sm, const double *__restrict__ F, const LineMap &m,
                                          size_t L0) {
    const int n = kSeg * S;
    for (int idx = threadIdx.x; idx < W * n; idx += blockDim.x) {
        int w, row;
        if (m.dir == 1) { w = idx / n; row = idx - w * n; }
        else { row = idx / W; w = idx - row * W; }
        sm[w * LineGeom<S>::kStride + LineGeom<S>::pos(row)] = __ldg(F + m.addr(L0 + w, row));
    }
}

// cooperative store (mode 0: out = v, 1: out += v)
template <int S, int W>
__device__ __forceinline__ void tile_store(const double *sm, double *__restrict__ O, const LineMap &m,
                                           size_t L0, int add) {
    const int n = kSeg * S;
    for (int idx = threadIdx.x; idx < W * n; idx += blockDim.x) {
        int w, row;
        if (m.dir == 1) { w = idx / n; row = idx - w * n; }
        else { row = idx / W; w = idx - row * W; }
        size_t g = m.addr(L0 + w, row);
        double v = sm[w * LineGeom<S>::kStride + LineGeom<S>::pos(row)];
        O[g] = add ? O[g] + v : v;
    }
}

// write a lane's segment back into its staged line
template <int S>
__device__ __forceinline__ void seg_to_line(double *line, int lane, const double (&r)[S]) {
#pragma unroll
    for (int t = 0; t < S; t++) line[LineGeom<S>::kPadL + lane * (S + 1) + t] = r[t];
}

}  // namespace st
