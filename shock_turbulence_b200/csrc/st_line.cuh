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
//
// FP32 mode: fields are float and the solves run in float, and a thread
// works on TWO neighbouring lines (lanes 2l, 2l+1 of a 32-line CTA) through a
// two-lane value type F2: one 8-byte access covers both lines' row, the LU
// table value of a row is loaded once for both, and the two recurrences give
// the dependent chains twice the independent work.
#pragma once
#include "st_internal.h"

namespace st {

// two float lines at one row
struct F2 {
    float x, y;
    F2() = default;
    __host__ __device__ constexpr F2(float a, float b) : x(a), y(b) {}
    __host__ __device__ F2(double v) : x((float)v), y((float)v) {}   // a constant on both lines
};
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return F2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return F2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ F2 operator-(F2 a) { return F2(-a.x, -a.y); }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return F2(a.x * b.x, a.y * b.y); }
__device__ __forceinline__ F2 operator*(float k, F2 a) { return F2(k * a.x, k * a.y); }
__device__ __forceinline__ F2 operator*(F2 a, float k) { return F2(a.x * k, a.y * k); }
__device__ __forceinline__ F2 operator*(double k, F2 a) { return (float)k * a; }
__device__ __forceinline__ F2 operator*(F2 a, double k) { return a * (float)k; }
// k*b + c with one rounding (the solves' explicit fma)
__device__ __forceinline__ double vfma(double k, double b, double c) { return fma(k, b, c); }
__device__ __forceinline__ F2 vfma(float k, F2 b, F2 c) { return F2(fmaf(k, b.x, c.x), fmaf(k, b.y, c.y)); }

// storage type T -> value type V of a thread's lines, its scalar A, lines per thread W
template <class T> struct Val;
template <> struct Val<double> { using V = double; using A = double; static constexpr int W = 1; };
template <> struct Val<float> { using V = F2; using A = float; static constexpr int W = 2; };

// element (lane, row) of a CTA's lines is base + lane*W*lstride + row*rstride
struct ColMap {
    size_t base, lstride, rstride;
};
struct LineGeo {
    int dir, n, My, Mz;
    // batches: blocks of CTAs per case (set by the launcher for its lines per
    // block) and the cells of a case; block blk works on case blk / cblk
    unsigned cblk;
    size_t cstride;
    // W lines per thread: a CTA owns kLanes*W lines
    template <int W>
    __device__ __forceinline__ ColMap map(unsigned blk) const {
        constexpr int NL = kLanes * W;
        ColMap m;
        const unsigned cs = blk / cblk;
        blk -= cs * cblk;
        const size_t sMy = My, sMz = Mz, jb = My / NL;
        if (dir == 0) {            // lines (j,k): NL consecutive j at one k
            m.base = (blk % jb) * NL + sMy * (blk / jb); m.lstride = 1; m.rstride = sMy * sMz;
        } else if (dir == 1) {     // lines (k,i): NL consecutive lines, each contiguous
            m.base = sMy * (size_t)blk * NL; m.lstride = sMy; m.rstride = 1;
        } else {                   // lines (j,i): NL consecutive j at one i
            m.base = (blk % jb) * NL + sMy * sMz * (blk / jb); m.lstride = 1; m.rstride = sMy;
        }
        m.base += (size_t)cs * cstride;
        return m;
    }
};

// Loads of one value: a double (a float field read in double), a float, or
// the two float lines at p and p+1 (8-byte aligned) as one F2.
template <class V, class T> struct Ld;
template <class T> struct Ld<double, T> {
    __device__ __forceinline__ static double get(const T *p) { return (double)__ldg(p); }
};
template <> struct Ld<float, float> {
    __device__ __forceinline__ static float get(const float *p) { return __ldg(p); }
};
template <> struct Ld<F2, float> {
    __device__ __forceinline__ static F2 get(const float *p) {
        float2 v = __ldg(reinterpret_cast<const float2 *>(p));
        return F2(v.x, v.y);
    }
};

template <int OP, class V = double, class T>
__device__ __forceinline__ V prod_eval(const ProdT<T> &P, size_t i) {
    using A = typename Val<T>::A;
    auto ld = [&](const T *p) { return Ld<V, T>::get(p); };
    if constexpr (OP == PR_MUL) {
        return ld(P.a + i) * ld(P.b + i);
    } else if constexpr (OP == PR_ADDMUL) {
        return (ld(P.a + i) + ld(P.b + i)) * ld(P.c + i);
    } else if constexpr (OP == PR_MULMUL) {
        return ld(P.c + i) * (ld(P.a + i) * ld(P.b + i));
    } else if constexpr (OP == PR_SPEC) {
        V a = ld(P.a + i), b = ld(P.b + i), c = ld(P.c + i);
        return a * b * c + a * c * (A)P.k0 * (A)P.k1;
    } else if constexpr (OP == PR_SPECT) {
        V a = ld(P.a + i), b = ld(P.b + i), c = ld(P.c + i), d = ld(P.d + i);
        V fl = a * b * c + a * c * (A)P.k0 * (A)P.k1;
        return (A)P.k2 * d * fl;
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

// rows a-H .. a+S+H-1 of this lane's line(s) into v (x and z lines: the W
// lines of a thread are neighbours in memory, lstride = 1)
template <int S, int H, int OP, class T, class V>
__device__ __forceinline__ void load_rows(V (&v)[S + 2 * H], const ProdT<T> &F, const ColMap &m, int lane,
                                          int a, int n, int cyc) {
    const size_t p = m.base + (size_t)lane * Val<T>::W * m.lstride;
#pragma unroll
    for (int q = 0; q < S + 2 * H; q++) {
        int row = halo_row(a - H + q, n, cyc);
        v[q] = prod_eval<OP, V>(F, p + (size_t)row * m.rstride);
    }
}

// plain (not read-only-path) load and store of one value
__device__ __forceinline__ double ldp(const double *p) { return *p; }
__device__ __forceinline__ F2 ldp2(const float *p) {
    float2 v = *reinterpret_cast<const float2 *>(p);
    return F2(v.x, v.y);
}
__device__ __forceinline__ void stv(double *p, double v) { *p = v; }
__device__ __forceinline__ void stv(float *p, double v) { *p = (float)v; }
__device__ __forceinline__ void stv(float *p, F2 v) { *reinterpret_cast<float2 *>(p) = make_float2(v.x, v.y); }

// add: O += r; otherwise O = r, or O = (r + E1) + E2 when E1 is given (the
// sum that follows the last derivative of a Laplacian, fused into its store)
template <int S, int N, class T, class V>
__device__ __forceinline__ void store_rows(const V (&r)[N], T *__restrict__ O, const ColMap &m,
                                           int lane, int a, int add, const T *E1 = nullptr,
                                           const T *E2 = nullptr) {
    const size_t off = m.base + (size_t)lane * Val<T>::W * m.lstride + (size_t)a * m.rstride;
    T *p = O + off;
    if (E1) {
        V e1[S], e2[S];
#pragma unroll
        for (int t = 0; t < S; t++) {
            e1[t] = Ld<V, T>::get(E1 + off + (size_t)t * m.rstride);
            e2[t] = Ld<V, T>::get(E2 + off + (size_t)t * m.rstride);
        }
#pragma unroll
        for (int t = 0; t < S; t++) stv(p + (size_t)t * m.rstride, (r[t] + e1[t]) + e2[t]);
        return;
    }
    if (add) {
        V prev[S];
#pragma unroll
        for (int t = 0; t < S; t++) {
            if constexpr (Val<T>::W == 2) prev[t] = ldp2(p + (size_t)t * m.rstride);
            else prev[t] = (double)p[(size_t)t * m.rstride];
        }
#pragma unroll
        for (int t = 0; t < S; t++) stv(p + (size_t)t * m.rstride, prev[t] + r[t]);
    } else {
#pragma unroll
        for (int t = 0; t < S; t++) stv(p + (size_t)t * m.rstride, r[t]);
    }
}

// shared buffers for the segment end values of one solve, and the corner
// values of a periodic line (rows 0, 1, n-2, n-1 of the banded solution)
template <class V>
struct CarryBufT {
    V a[kMaxSeg][kLanes][2];
    V b[kMaxSeg][kLanes][2];
    V cy[kLanes][4];
};
using CarryBuf = CarryBufT<double>;

// ---- periodic lines: corner correction after the banded solve ------------
// x_i = y_i - sum_k K_ik y_{j_k} with the corner rows j = {0, n-1} (K = 2,
// tridiagonal) or {0, 1, n-2, n-1} (K = 4, pentadiagonal); the table holds
// -K row-major.  The first and last segments publish the corner values; the
// barrier also orders them after every read of the previous solve's cy.
template <int S, int N, int KC, class V, class A>
__device__ __forceinline__ void cyc_fix(V (&r)[N], const A *__restrict__ Kt, int s, int P, int lane,
                                        CarryBufT<V> &cb) {
    if (KC == 2) {
        if (s == 0) cb.cy[lane][0] = r[0];
        if (s == P - 1) cb.cy[lane][1] = r[S - 1];
    } else {
        if (s == 0) { cb.cy[lane][0] = r[0]; cb.cy[lane][1] = r[1]; }
        if (s == P - 1) { cb.cy[lane][2] = r[S - 2]; cb.cy[lane][3] = r[S - 1]; }
    }
    __syncthreads();
    V y[KC];
#pragma unroll
    for (int k = 0; k < KC; k++) y[k] = cb.cy[lane][k];
    const A *kr = Kt + (size_t)s * S * KC;
#pragma unroll
    for (int t = 0; t < S; t++) {
        V v = r[t];
#pragma unroll
        for (int k = 0; k < KC; k++) v = vfma(__ldg(kr + t * KC + k), y[k], v);
        r[t] = v;
    }
}

// ---- scan of scalar carries over the segments, one warp per line ----------
// buf[ln*(kMaxSeg+1) + s] holds segment s's value of line ln on entry and the
// inclusive scan value on exit: f(s) = a(s) + t_k(s) f(s - 2^k) (FWD) or
// g(s) = b(s) + u_k(s) g(s + 2^k), k = 0, 1, ... while 2^k < P, with the
// products of 2^k consecutive transfer factors in [kScanSteps][kMaxSeg]
// tables.  Lane s of a warp takes segment s and reads the others by
// shuffles (no CTA barrier); the arithmetic and its order are those of a
// Hillis-Steele scan over shared memory.  The full warps take lines w,
// w + nwarps, ... (a CTA has 16 P threads: with P odd its last warp is a half
// warp, which takes none; every full warp has 32 >= P lanes).
__device__ __forceinline__ double shfl_seg(bool up, double v, int d) {
    return up ? __shfl_up_sync(0xffffffffu, v, d) : __shfl_down_sync(0xffffffffu, v, d);
}
__device__ __forceinline__ F2 shfl_seg(bool up, F2 v, int d) {
    return F2(up ? __shfl_up_sync(0xffffffffu, v.x, d) : __shfl_down_sync(0xffffffffu, v.x, d),
              up ? __shfl_up_sync(0xffffffffu, v.y, d) : __shfl_down_sync(0xffffffffu, v.y, d));
}
template <bool FWD, class V, class A>
__device__ __forceinline__ void seg_scan1_warp(V *buf, const A *__restrict__ tab, int P) {
    const int l = threadIdx.x & 31, nw = blockDim.x >> 5;
    if ((int)(threadIdx.x >> 5) >= nw) return;     // the half warp of an odd P takes no line
    for (int ln = threadIdx.x >> 5; ln < kLanes; ln += nw) {
        V *row = buf + ln * (kMaxSeg + 1);
        V f = l < P ? row[l] : V(0.0);
        for (int k = 0, d = 1; d < P; k++, d <<= 1) {
            const V o = shfl_seg(FWD, f, d);
            if (FWD ? (l >= d && l < P) : (l + d < P)) f = vfma(__ldg(tab + k * kMaxSeg + l), o, f);
        }
        if (l < P) row[l] = f;
    }
}

// ---- segmented constant-coefficient tridiagonal solve --------------------
// Forward elimination r'_i = r_i - l_i r'_{i-1} and back substitution
// x_i = (r'_i - c_i x_{i+1}) / (b'_i + tiny) of tridiagonal_serial
// (src/tridiagonal.f90:274-284) per segment with zero carries, then the
// carry corrections.  Caller guarantees cb is free (synchronised).
template <int S, int N, class V, class A>
__device__ __forceinline__ void tri_back(V (&r)[N], const TriTabT<A> &T, int a, bool flat) {
    if (flat) {
        const A up = T.cup, id = T.cid;
        r[S - 1] = r[S - 1] * id;
#pragma unroll
        for (int t = S - 2; t >= 0; t--) r[t] = (r[t] - up * r[t + 1]) * id;
    } else {
        r[S - 1] = r[S - 1] * __ldg(T.id + a + S - 1);
#pragma unroll
        for (int t = S - 2; t >= 0; t--) r[t] = (r[t] - __ldg(T.up + a + t) * r[t + 1]) * __ldg(T.id + a + t);
    }
}

template <int S, int N, class V, class A>
__device__ __forceinline__ void tri_solve(V (&r)[N], const TriTabT<A> &T, int s, int P, int lane,
                                          CarryBufT<V> &cb) {
    const int a = s * S;
    const bool flat = s >= T.slo && s < T.shi;   // interior: constant factors in registers
    if (flat) {
        const A l = T.cl;
#pragma unroll
        for (int t = 1; t < S; t++) r[t] = r[t] - r[t - 1] * l;
    } else {
#pragma unroll
        for (int t = 1; t < S; t++) r[t] = r[t] - r[t - 1] * __ldg(T.l + a + t);
    }
    // Carries reaching more than twice as many segments as a scan has steps
    // (short segments: small grids, n <= 128) come from a log2(P)-step warp
    // scan per direction, f(s) = a(s) + B_s f(s-1), carry into s = f(s-1);
    // otherwise from the sum over the kf segments before s (kb after s for
    // the right carry; measured faster for n >= 256).  The choice is uniform
    // over the CTA.
    const bool scan = T.kf > 2 * kScanSteps || T.kb > 2 * kScanSteps;
    if (scan) {
        constexpr int LS = kMaxSeg + 1;
        V cin = V(0.0);
        V *fa = &cb.a[0][0][0];          // [kLanes][kMaxSeg + 1]
        fa[lane * LS + s] = r[S - 1];
        __syncthreads();
        seg_scan1_warp<true>(fa, T.sf, P);
        __syncthreads();
        if (s > 0) cin = fa[lane * LS + s - 1];
#pragma unroll
        for (int t = 0; t < S; t++) r[t] = vfma(__ldg(T.g + a + t), cin, r[t]);
        tri_back<S>(r, T, a, flat);
        // the second buffer: the first is still read until the barrier below
        V ein = V(0.0);
        V *fb = &cb.b[0][0][0];
        fb[lane * LS + s] = r[0];
        __syncthreads();
        seg_scan1_warp<false>(fb, T.sb, P);
        __syncthreads();
        if (s + 1 < P) ein = fb[lane * LS + s + 1];
#pragma unroll
        for (int t = 0; t < S; t++) r[t] = vfma(__ldg(T.h + a + t), ein, r[t]);
    } else {
        V cin = V(0.0), ein = V(0.0);
        cb.a[s][lane][0] = r[S - 1];
        __syncthreads();
#pragma unroll 4
        for (int sp = max(0, s - T.kf); sp < s; sp++) cin = vfma(__ldg(T.wf + sp * P + s), cb.a[sp][lane][0], cin);
#pragma unroll
        for (int t = 0; t < S; t++) r[t] = vfma(__ldg(T.g + a + t), cin, r[t]);
        tri_back<S>(r, T, a, flat);
        cb.b[s][lane][0] = r[0];
        __syncthreads();
#pragma unroll 4
        for (int sp = s + 1, se = min(P, s + 1 + T.kb); sp < se; sp++)
            ein = vfma(__ldg(T.wb + sp * P + s), cb.b[sp][lane][0], ein);
#pragma unroll
        for (int t = 0; t < S; t++) r[t] = vfma(__ldg(T.h + a + t), ein, r[t]);
    }
}

// ---- segmented constant-coefficient pentadiagonal solve ------------------
// Elimination order of pentadiagonal_serial (src/pentadiagonal.f90:340-372):
// r'_i = (r_i - k2 r'_{i-2}) - k1 r'_{i-1};  x_i = ((r'_i - D'_i x_{i+1})
// - E_i x_{i+2}) / (C'_i + tiny).  Carries are 2-vectors.
template <int S, int N>
__device__ __forceinline__ void pen_solve(double (&r)[N], const PenTab &T, int s, int P, int lane,
                                          CarryBuf &cb) {
    const int a = s * S;
    const bool flat = s >= T.slo && s < T.shi;   // interior: constant factors in registers
    if (flat) {
        const double p1 = T.cp1, p2 = T.cp2;
#pragma unroll
        for (int t = 1; t < S; t++) {
            double v = r[t];
            if (t >= 2) v = v - p2 * r[t >= 2 ? t - 2 : 0];
            v = v - p1 * r[t - 1];
            r[t] = v;
        }
    } else {
#pragma unroll
        for (int t = 1; t < S; t++) {
            double v = r[t];
            if (t >= 2) v = v - __ldg(T.p2 + a + t) * r[t >= 2 ? t - 2 : 0];
            v = v - __ldg(T.p1 + a + t) * r[t - 1];
            r[t] = v;
        }
    }
    // carry into segment s: c(s) = f(s-1) of the inclusive scan
    // f(s) = a(s) + M_s f(s-1) over the segments' end values a(s), in
    // log2(P) steps over a double buffer (the reach of the carries, up to the
    // whole line for this nearly singular system, costs every segment the
    // same)
    double f1 = r[S - 1], f2 = (S >= 2) ? r[S >= 2 ? S - 2 : 0] : 0.0;
    double(*cur)[kLanes][2] = cb.a;
    double(*nxt)[kLanes][2] = cb.b;
    cur[s][lane][0] = f1;
    cur[s][lane][1] = f2;
    __syncthreads();
    for (int k = 0, d = 1; d < P; k++, d <<= 1) {
        if (s >= d) {
            const double *m = T.sf + ((size_t)k * kMaxSeg + s) * 4;
            const double o1 = cur[s - d][lane][0], o2 = cur[s - d][lane][1];
            f1 = fma(__ldg(m + 0), o1, fma(__ldg(m + 1), o2, f1));
            f2 = fma(__ldg(m + 2), o1, fma(__ldg(m + 3), o2, f2));
        }
        nxt[s][lane][0] = f1;
        nxt[s][lane][1] = f2;
        __syncthreads();
        double(*t)[kLanes][2] = cur; cur = nxt; nxt = t;
    }
    const double c1 = s > 0 ? cur[s - 1][lane][0] : 0.0, c2 = s > 0 ? cur[s - 1][lane][1] : 0.0;
#pragma unroll
    for (int t = 0; t < S; t++) r[t] = fma(__ldg(T.g1 + a + t), c1, fma(__ldg(T.g2 + a + t), c2, r[t]));
    if (flat) {
        const double q1 = T.cq1, q2 = T.cq2, id = T.cid;
#pragma unroll
        for (int t = S - 1; t >= 0; t--) {
            double v = r[t];
            if (t + 1 < S) v = v - q1 * r[t + 1 < S ? t + 1 : t];
            if (t + 2 < S) v = v - q2 * r[t + 2 < S ? t + 2 : t];
            r[t] = v * id;
        }
    } else {
#pragma unroll
        for (int t = S - 1; t >= 0; t--) {
            double v = r[t];
            if (t + 1 < S) v = v - __ldg(T.q1 + a + t) * r[t + 1 < S ? t + 1 : t];
            if (t + 2 < S) v = v - __ldg(T.q2 + a + t) * r[t + 2 < S ? t + 2 : t];
            r[t] = v * __ldg(T.id + a + t);
        }
    }
    // carry from the right: e(s) = g(s+1) of g(s) = b(s) + N_s g(s+1); the
    // first write goes to the buffer nobody reads after the forward scan
    double g1 = r[0], g2 = (S >= 2) ? r[S >= 2 ? 1 : 0] : 0.0;
    nxt[s][lane][0] = g1;
    nxt[s][lane][1] = g2;
    {
        double(*t)[kLanes][2] = cur; cur = nxt; nxt = t;
    }
    __syncthreads();
    for (int k = 0, d = 1; d < P; k++, d <<= 1) {
        if (s + d < P) {
            const double *m = T.sb + ((size_t)k * kMaxSeg + s) * 4;
            const double o1 = cur[s + d][lane][0], o2 = cur[s + d][lane][1];
            g1 = fma(__ldg(m + 0), o1, fma(__ldg(m + 1), o2, g1));
            g2 = fma(__ldg(m + 2), o1, fma(__ldg(m + 3), o2, g2));
        }
        nxt[s][lane][0] = g1;
        nxt[s][lane][1] = g2;
        __syncthreads();
        double(*t)[kLanes][2] = cur; cur = nxt; nxt = t;
    }
    const double e1 = s + 1 < P ? cur[s + 1][lane][0] : 0.0, e2 = s + 1 < P ? cur[s + 1][lane][1] : 0.0;
#pragma unroll
    for (int t = 0; t < S; t++) r[t] = fma(__ldg(T.h1 + a + t), e1, fma(__ldg(T.h2 + a + t), e2, r[t]));
}

// ---- explicit right-hand sides ------------------------------------------
// v holds rows a-H .. a+S+H-1 on entry; the RHS of row a+t is written into
// v[t] (in place, ascending t: row a+t only needs v[t..t+2H]).  Rows follow
// the reference formulas term by term (Fortran evaluates left to right).
// Boundary rows belong to the first/last segment only: those warps re-read
// the few rows they need from global memory (warp-uniform branch).
template <int OP, class T = double, class V = double>
struct RowReader {
    using A = typename Val<T>::A;
    const A *tile;            // shared tile row of the thread's (first) line (y lines) or null
    const ProdT<T> *F;        // global producer (x, z lines)
    size_t base, rstride;
    int tstride;              // tile distance between a thread's two lines (W = 2)
    __device__ __forceinline__ V operator()(int row) const {
        if constexpr (Val<T>::W == 2) {
            return tile ? V(tile[row], tile[row + tstride]) : prod_eval<OP, V>(*F, base + (size_t)row * rstride);
        } else {
            return tile ? tile[row] : prod_eval<OP, V>(*F, base + (size_t)row * rstride);
        }
    }
};

// ---- y lines: staging through shared memory ------------------------------
// The NL = kLanes*W lines of a y CTA are one contiguous block of NL*n values.
// They are copied with 16-byte coalesced accesses into an [NL][n+1] tile of
// the arithmetic type (odd stride: the lines of a half-warp start in distinct
// banks), so that each thread reads its segment conflict-free.
// Each thread keeps kTB loads in flight: a batch of loads is issued before
// any of them is stored into the tile (a load-then-store loop would wait for
// every load in turn).
constexpr int kTB = 4;

template <int OP, class T>
__device__ __forceinline__ void ytile_load(typename Val<T>::A *tile, const ProdT<T> &F, size_t base, int n) {
    constexpr int NL = kLanes * Val<T>::W;
    const int nt = blockDim.x;
    if constexpr (sizeof(T) == 8) {
        const int half = NL * n / 2;
        if (OP == PR_A && ((reinterpret_cast<uintptr_t>(F.a + base) & 15) == 0)) {
            const double2 *src = reinterpret_cast<const double2 *>(F.a + base);
            for (int q0 = threadIdx.x; q0 < half; q0 += kTB * nt) {
                double2 d[kTB];
#pragma unroll
                for (int u = 0; u < kTB; u++)
                    if (q0 + u * nt < half) d[u] = __ldg(src + q0 + u * nt);
#pragma unroll
                for (int u = 0; u < kTB; u++) {
                    const int q = q0 + u * nt;
                    if (q < half) {
                        int e = 2 * q, line = e / n, row = e - line * n;
                        tile[line * (n + 1) + row] = d[u].x;
                        tile[line * (n + 1) + row + 1] = d[u].y;
                    }
                }
            }
            return;
        }
    } else {
        const int quarter = NL * n / 4;
        if (OP == PR_A && ((reinterpret_cast<uintptr_t>(F.a + base) & 15) == 0)) {
            const float4 *src = reinterpret_cast<const float4 *>(F.a + base);
            for (int q0 = threadIdx.x; q0 < quarter; q0 += kTB * nt) {
                float4 d[kTB];
#pragma unroll
                for (int u = 0; u < kTB; u++)
                    if (q0 + u * nt < quarter) d[u] = __ldg(src + q0 + u * nt);
#pragma unroll
                for (int u = 0; u < kTB; u++) {
                    const int q = q0 + u * nt;
                    if (q < quarter) {
                        int e = 4 * q, line = e / n, row = e - line * n;   // n % 4 == 0: one line
                        float *t = tile + line * (n + 1) + row;
                        t[0] = d[u].x; t[1] = d[u].y; t[2] = d[u].z; t[3] = d[u].w;
                    }
                }
            }
            return;
        }
    }
    using A = typename Val<T>::A;
    const int tot = NL * n;
    for (int q0 = threadIdx.x; q0 < tot; q0 += kTB * nt) {
        A d[kTB];
#pragma unroll
        for (int u = 0; u < kTB; u++)
            if (q0 + u * nt < tot) d[u] = prod_eval<OP, A>(F, base + q0 + u * nt);
#pragma unroll
        for (int u = 0; u < kTB; u++) {
            const int q = q0 + u * nt;
            if (q < tot) {
                int line = q / n, row = q - line * n;
                tile[line * (n + 1) + row] = d[u];
            }
        }
    }
}
template <class T>
__device__ __forceinline__ void ytile_store(const typename Val<T>::A *tile, T *__restrict__ O, size_t base, int n,
                                            int add) {
    constexpr int NL = kLanes * Val<T>::W;
    const int nt = blockDim.x;
    if constexpr (sizeof(T) == 8) {
        if (!(reinterpret_cast<uintptr_t>(O + base) & 15)) {
            double2 *dst = reinterpret_cast<double2 *>(O + base);
            const int half = NL * n / 2;
            for (int q0 = threadIdx.x; q0 < half; q0 += kTB * nt) {
                double2 o[kTB];
                if (add) {
#pragma unroll
                    for (int u = 0; u < kTB; u++)
                        if (q0 + u * nt < half) o[u] = dst[q0 + u * nt];
                }
#pragma unroll
                for (int u = 0; u < kTB; u++) {
                    const int q = q0 + u * nt;
                    if (q < half) {
                        int e = 2 * q, line = e / n, row = e - line * n;
                        double2 d = make_double2(tile[line * (n + 1) + row], tile[line * (n + 1) + row + 1]);
                        if (add) {
                            d.x = o[u].x + d.x;
                            d.y = o[u].y + d.y;
                        }
                        dst[q] = d;
                    }
                }
            }
            return;
        }
    } else {
        if (!(reinterpret_cast<uintptr_t>(O + base) & 15)) {
            float4 *dst = reinterpret_cast<float4 *>(O + base);
            const int quarter = NL * n / 4;
            for (int q0 = threadIdx.x; q0 < quarter; q0 += kTB * nt) {
                float4 o[kTB];
                if (add) {
#pragma unroll
                    for (int u = 0; u < kTB; u++)
                        if (q0 + u * nt < quarter) o[u] = dst[q0 + u * nt];
                }
#pragma unroll
                for (int u = 0; u < kTB; u++) {
                    const int q = q0 + u * nt;
                    if (q < quarter) {
                        int e = 4 * q, line = e / n, row = e - line * n;
                        const float *t = tile + line * (n + 1) + row;
                        float4 d = make_float4(t[0], t[1], t[2], t[3]);
                        if (add) {
                            d.x = o[u].x + d.x; d.y = o[u].y + d.y; d.z = o[u].z + d.z; d.w = o[u].w + d.w;
                        }
                        dst[q] = d;
                    }
                }
            }
            return;
        }
    }
    for (int q = threadIdx.x; q < NL * n; q += nt) {
        int line = q / n, row = q - line * n;
        auto v = tile[line * (n + 1) + row];
        O[base + q] = (T)(add ? (T)O[base + q] + v : v);
    }
}
// rows of the thread's line(s) from the tile; W = 2: lines 2*lane and 2*lane+1
template <int S, int H, class V, class A>
__device__ __forceinline__ void ytile_rows(V (&v)[S + 2 * H], const A *tile, int lane, int a, int n, int cyc) {
    if constexpr (sizeof(V) == 2 * sizeof(A)) {
        const A *p = tile + 2 * lane * (n + 1);
#pragma unroll
        for (int q = 0; q < S + 2 * H; q++) {
            int row = halo_row(a - H + q, n, cyc);
            v[q] = V(p[row], p[row + n + 1]);
        }
    } else {
        const A *p = tile + lane * (n + 1);
#pragma unroll
        for (int q = 0; q < S + 2 * H; q++) v[q] = p[halo_row(a - H + q, n, cyc)];
    }
}
template <int S, int N, class V, class A>
__device__ __forceinline__ void ytile_put(A *tile, const V (&r)[N], int lane, int a, int n) {
    if constexpr (sizeof(V) == 2 * sizeof(A)) {
        A *p = tile + 2 * lane * (n + 1) + a;
#pragma unroll
        for (int t = 0; t < S; t++) { p[t] = r[t].x; p[t + n + 1] = r[t].y; }
    } else {
        A *p = tile + lane * (n + 1) + a;
#pragma unroll
        for (int t = 0; t < S; t++) p[t] = r[t];
    }
}

// DFDX_sym/_asym RHS, src/derivCDopt6_sym_tri.f:458-514,
// src/derivCDopt6_asym_tri.f:461-516  (H = 2).  Periodic DFDX,
// src/derivCDopt6_periodic.f:205-248: the interior formula on every row with
// wrapped halos (its f(i+-3) weight c1 is zero for the FDL3DI set).
template <int S, int H, class RD, class V>
__device__ __forceinline__ void rhs_d1(V (&v)[S + 2 * H], int a, int n, int asym, int cyc, double fac,
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
template <int S, int H, class RD, class V>
__device__ __forceinline__ void rhs_d2(V (&v)[S + 2 * H], int a, int n, int asym, int cyc, double fac,
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
template <int S, int H, class RD, class V>
__device__ __forceinline__ void rhs_gauss(V (&v)[S + 2 * H], int a, int n, int cyc, const Consts &K,
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
