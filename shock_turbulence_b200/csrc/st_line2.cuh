// st_line2.cuh - persistent line kernels with whole lines staged in shared
// memory (bounded-line family, lines of n = 32*S rows, n >= 64).
//
// Work decomposition ("tiles"): a tile is KW*LPW neighbouring lines of one
// direction, copied whole into shared memory with cp.async.  A CTA of KW
// warps owns one tile at a time and walks over tiles blockIdx.x,
// blockIdx.x + gridDim.x, ... (one CTA per SM); the copies of the next tiles
// are in flight while it solves the current one (NB-stage ring of tile
// buffers).  Within a tile, warp w solves its line (FP64) or its two
// neighbouring lines at once (FP32: value type F2, LPW = 2), lane s the
// line's segment of S rows (P = 32 segments):
//  - the global copies are the same coalesced rows as before (a row of the
//    tile's lines is one contiguous run of x and z lines, and the tile is one
//    contiguous block of y lines);
//  - each lane reads its rows (and the stencil halo) from the tile, whose
//    segments are padded to an odd stride, so the 32 lanes of a warp hit 32
//    different banks;
//  - a derivative of a product (the flux forms of RHS, Hyper_RHS and
//    Species_RHS) copies each factor's tile and forms the product as it
//    reads the window, in the operand order of the reference statement;
//  - the carries between segments are scans over the 32 lanes of one warp
//    (shuffles, no barriers); each segment first runs its recurrence with a
//    zero carry to get the end values the scan needs, then runs it again with
//    the true carry, so no per-row carry-response tables are read;
//  - the per-row LU factors live in shared memory, transposed ([row in
//    segment][segment]) so that a warp's 32 lanes read 32 consecutive
//    values; lanes whose segment lies in the factorisation's interior fixed
//    point use register constants instead and skip those loads;
//  - results go back into the tile (the warp's own line) and leave it with
//    the same coalesced rows, with the accumulate (iadd) and the fused
//    Laplacian sum applied on the way out.
// Three barriers per tile (copies landed, line solves done, tile stored)
// replace the dozen CTA-wide barriers of the segmented solves in st_line.cuh.
#pragma once
#include "st_line.cuh"

// LineArgsT (st_linekern.cuh) is declared before this header is included.

namespace st {
namespace lk2 {

constexpr unsigned kFull = 0xffffffffu;

// element type of a tile slot: one FP64 line, or two FP32 lines side by side
template <class T> struct Elt;
template <> struct Elt<double> {
    using E = double; using V = double; using A = double;
    static constexpr int LPW = 1;
    __device__ __forceinline__ static V get(const E &e) { return e; }
    __device__ __forceinline__ static void put(E &e, V v) { e = v; }
};
template <> struct Elt<float> {
    using E = float2; using V = F2; using A = float;
    static constexpr int LPW = 2;
    __device__ __forceinline__ static V get(const E &e) { return F2(e.x, e.y); }
    __device__ __forceinline__ static void put(E &e, V v) { e = make_float2(v.x, v.y); }
};

__device__ __forceinline__ double shfl_up(double v, int d) { return __shfl_up_sync(kFull, v, d); }
__device__ __forceinline__ double shfl_down(double v, int d) { return __shfl_down_sync(kFull, v, d); }
__device__ __forceinline__ F2 shfl_up(F2 v, int d) {
    return F2(__shfl_up_sync(kFull, v.x, d), __shfl_up_sync(kFull, v.y, d));
}
__device__ __forceinline__ F2 shfl_down(F2 v, int d) {
    return F2(__shfl_down_sync(kFull, v.x, d), __shfl_down_sync(kFull, v.y, d));
}

// odd segment stride (conflict-free lane reads) and odd line stride
// (conflict-free row writes of the copy-in), in 8-byte slots
template <int S, int KW>
struct Pad {
    static constexpr int SP = (S % 2 == 0) ? S + 1 : S + 2;
    static constexpr int LS = 32 * SP + 1;
    static constexpr int TB = KW * LS;          // slots of one tile buffer
};

template <int S>
__device__ __forceinline__ int pidx(int r) {
    constexpr int SP = (S % 2 == 0) ? S + 1 : S + 2;
    return (r / S) * SP + (r - (r / S) * S);
}

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// The tile of NL lines with index blk (LineGeo::map for NL lines per tile;
// g.cblk tiles per case of a batch): element (line l, row r) at
// base + l*lstride + r*rstride.
template <int NL>
__device__ __forceinline__ ColMap tile_map(const LineGeo &g, unsigned blk) {
    ColMap m;
    const unsigned cs = blk / g.cblk;      // case of a batch
    blk -= cs * g.cblk;
    const size_t sMy = g.My, sMz = g.Mz, jb = g.My / NL;
    if (g.dir == 0) { m.base = (blk % jb) * NL + sMy * (blk / jb); m.lstride = 1; m.rstride = sMy * sMz; }
    else if (g.dir == 1) { m.base = sMy * (size_t)blk * NL; m.lstride = sMy; m.rstride = 1; }
    else { m.base = (blk % jb) * NL + sMy * sMz * (blk / jb); m.lstride = 1; m.rstride = sMy; }
    m.base += (size_t)cs * g.cstride;
    return m;
}

// Slot e of a tile (0 <= e < KW n): warp-line w (lines LPW w ..) and row r.
// x and z lines: the tile's lines at one row are consecutive values
// (e = KW r + w); y lines: the tile is a block of whole lines (e = n w + r).
template <int S, int KW>
__device__ __forceinline__ void slot(int dir, int e, int &w, int &r) {
    constexpr int n = 32 * S;
    if (dir == 1) { w = e / n; r = e - w * n; }
    else { w = e % KW; r = e / KW; }
}
template <class T>
__device__ __forceinline__ size_t goff(const ColMap &m, int w, int r, int line_in_pair) {
    return (size_t)(Elt<T>::LPW * w + line_in_pair) * m.lstride + (size_t)r * m.rstride;
}

// issues the copies of one field's tile into buf (S slots per thread)
template <int S, int KW, class T>
__device__ __forceinline__ void issue_field(typename Elt<T>::E *buf, const T *F, const ColMap &m, int dir) {
    using E = typename Elt<T>::E;
    const T *src = F + m.base;
#pragma unroll
    for (int k = 0; k < S; k++) {
        int w, r;
        slot<S, KW>(dir, (int)threadIdx.x + KW * 32 * k, w, r);
        E *dst = buf + w * Pad<S, KW>::LS + pidx<S>(r);
        if (sizeof(T) == 8 || dir != 1) {
            cp_async8(dst, src + goff<T>(m, w, r, 0));       // FP32 x/z: the pair is adjacent
        } else {
            float *d = reinterpret_cast<float *>(dst);
            cp_async4(d, src + goff<T>(m, w, r, 0));
            cp_async4(d + 1, src + goff<T>(m, w, r, 1));
        }
    }
}

// fields a producer expression reads
template <int OP>
struct NIn { static constexpr int v = OP == PR_A ? 1 : OP == PR_MUL ? 2 : OP == PR_SPECT ? 4 : 3; };

// the producer expressions of prod_eval (st_line.cuh), from tile values
template <int OP, class V, class A, class T>
__device__ __forceinline__ V combine(const ProdT<T> &P, V a, V b, V c, V d) {
    if constexpr (OP == PR_MUL) {
        return a * b;
    } else if constexpr (OP == PR_ADDMUL) {
        return (a + b) * c;
    } else if constexpr (OP == PR_MULMUL) {
        return c * (a * b);
    } else if constexpr (OP == PR_SPEC) {
        return a * b * c + a * c * (A)P.k0 * (A)P.k1;
    } else if constexpr (OP == PR_SPECT) {
        V fl = a * b * c + a * c * (A)P.k0 * (A)P.k1;
        return (A)P.k2 * d * fl;
    } else {
        (void)P; (void)b; (void)c; (void)d;
        return a;
    }
}

// the tiles of the current ring slot (one per input field), at one
// warp-line, and the producer they feed
template <int OP, class T>
struct Slot {
    using E = typename Elt<T>::E;
    using V = typename Elt<T>::V;
    const E *f[4];
    const ProdT<T> *P;
    __device__ __forceinline__ V at(int q) const {
        using A = typename Elt<T>::A;
        constexpr int NI = NIn<OP>::v;
        V a = Elt<T>::get(f[0][q]);
        V b = NI > 1 ? Elt<T>::get(f[1][q]) : a;
        V c = NI > 2 ? Elt<T>::get(f[2][q]) : a;
        V d = NI > 3 ? Elt<T>::get(f[3][q]) : a;
        return combine<OP, V, A>(*P, a, b, c, d);
    }
};

// boundary rows of the stencils read any row of the warp's line from the tile
template <int S, int OP, class T>
struct TileRow {
    Slot<OP, T> sl;
    __device__ __forceinline__ typename Elt<T>::V operator()(int row) const { return sl.at(pidx<S>(row)); }
};

// rows a-H .. a+S+H-1 of the lane's segment (out-of-line halo rows clamped;
// the stencils never use them, their boundary rows re-read what they need)
template <int S, int H, int OP, class T, class V>
__device__ __forceinline__ void window(V (&v)[S + 2 * H], const Slot<OP, T> &sl, int s) {
    constexpr int n = 32 * S, SP = (S % 2 == 0) ? S + 1 : S + 2;
    const int a = s * S;
#pragma unroll
    for (int q = 0; q < H; q++) {
        int row = a - H + q;
        v[q] = sl.at(pidx<S>(row < 0 ? 0 : row));
        int rr = a + S + q;
        v[S + H + q] = sl.at(pidx<S>(rr > n - 1 ? n - 1 : rr));
    }
#pragma unroll
    for (int t = 0; t < S; t++) v[H + t] = sl.at(s * SP + t);
}

// Per-row LU factors in shared memory, transposed: entry (t, s) of a table
// is the factor of row s*S + t, at t*32 + s.
template <int S, class A>
__device__ __forceinline__ void stage_table(A *dst, const A *src) {
    constexpr int n = 32 * S;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        int s = i / S, t = i - s * S;
        dst[t * 32 + s] = src[i];
    }
}

// ---- segmented tridiagonal solve over the lanes of a warp ------------------
// Same factorisation and scan factors as tri_solve (st_line.cuh); ft holds
// l, up, id transposed (3 n values).
template <int S, class V, class A, int N>
__device__ __forceinline__ void tri_solve_w(V (&r)[N], const TriTabT<A> &T, const A *ft, int s) {
    constexpr int n = 32 * S;
    const bool flat = s >= T.slo && s < T.shi;
    const A *fl = ft + s, *fu = ft + n + s, *fi = ft + 2 * n + s;
    auto L = [&](int t) { return flat ? T.cl : fl[t * 32]; };
    auto U = [&](int t) { return flat ? T.cup : fu[t * 32]; };
    auto I = [&](int t) { return flat ? T.cid : fi[t * 32]; };
    // forward: r'_i = r_i - l_i r'_{i-1}; zero-carry end value, then the scan
    V x = V(0.0);
#pragma unroll
    for (int t = 0; t < S; t++) x = r[t] - x * L(t);
    V f = x;
#pragma unroll
    for (int k = 0, d = 1; k < kScanSteps; k++, d <<= 1) {
        const V o = shfl_up(f, d);
        if (s >= d) f = vfma(__ldg(T.sf + k * kMaxSeg + s), o, f);
    }
    x = shfl_up(f, 1);
    if (s == 0) x = V(0.0);
#pragma unroll
    for (int t = 0; t < S; t++) { x = r[t] - x * L(t); r[t] = x; }
    // backward: x_i = (r'_i - c_i x_{i+1}) / (b'_i + tiny)
    V y = V(0.0);
#pragma unroll
    for (int t = S - 1; t >= 0; t--) y = (r[t] - U(t) * y) * I(t);
    V g = y;
#pragma unroll
    for (int k = 0, d = 1; k < kScanSteps; k++, d <<= 1) {
        const V o = shfl_down(g, d);
        if (s + d < 32) g = vfma(__ldg(T.sb + k * kMaxSeg + s), o, g);
    }
    y = shfl_down(g, 1);
    if (s == 31) y = V(0.0);
#pragma unroll
    for (int t = S - 1; t >= 0; t--) { y = (r[t] - U(t) * y) * I(t); r[t] = y; }
}

// ---- segmented pentadiagonal solve over the lanes of a warp (FP64) ---------
// Same factorisation and scan factors as pen_solve (st_line.cuh); ft holds
// p1, p2, q1, q2, id transposed (5 n values).
template <int S, int N>
__device__ __forceinline__ void pen_solve_w(double (&r)[N], const PenTab &T, const double *ft, int s) {
    constexpr int n = 32 * S;
    const bool flat = s >= T.slo && s < T.shi;
    const double *f1p = ft + s, *f2p = ft + n + s, *q1p = ft + 2 * n + s, *q2p = ft + 3 * n + s,
                 *idp = ft + 4 * n + s;
    auto P1 = [&](int t) { return flat ? T.cp1 : f1p[t * 32]; };
    auto P2 = [&](int t) { return flat ? T.cp2 : f2p[t * 32]; };
    auto Q1 = [&](int t) { return flat ? T.cq1 : q1p[t * 32]; };
    auto Q2 = [&](int t) { return flat ? T.cq2 : q2p[t * 32]; };
    auto ID = [&](int t) { return flat ? T.cid : idp[t * 32]; };
    // forward: r'_i = (r_i - k2 r'_{i-2}) - k1 r'_{i-1}, carry (r'_{a-1}, r'_{a-2})
    double x1 = 0.0, x2 = 0.0;
#pragma unroll
    for (int t = 0; t < S; t++) {
        const double v = (r[t] - P2(t) * x2) - P1(t) * x1;
        x2 = x1; x1 = v;
    }
    double f1 = x1, f2 = x2;
#pragma unroll
    for (int k = 0, d = 1; k < kScanSteps; k++, d <<= 1) {
        const double o1 = shfl_up(f1, d), o2 = shfl_up(f2, d);
        if (s >= d) {
            const double *m = T.sf + ((size_t)k * kMaxSeg + s) * 4;
            f1 = fma(__ldg(m + 0), o1, fma(__ldg(m + 1), o2, f1));
            f2 = fma(__ldg(m + 2), o1, fma(__ldg(m + 3), o2, f2));
        }
    }
    x1 = shfl_up(f1, 1);
    x2 = shfl_up(f2, 1);
    if (s == 0) x1 = x2 = 0.0;
#pragma unroll
    for (int t = 0; t < S; t++) {
        const double v = (r[t] - P2(t) * x2) - P1(t) * x1;
        x2 = x1; x1 = v; r[t] = v;
    }
    // backward: x_i = ((r'_i - D'_i x_{i+1}) - E_i x_{i+2}) / (C'_i + tiny),
    // carry (x_{b+1}, x_{b+2})
    double y1 = 0.0, y2 = 0.0;
#pragma unroll
    for (int t = S - 1; t >= 0; t--) {
        const double v = ((r[t] - Q1(t) * y1) - Q2(t) * y2) * ID(t);
        y2 = y1; y1 = v;
    }
    double g1 = y1, g2 = y2;
#pragma unroll
    for (int k = 0, d = 1; k < kScanSteps; k++, d <<= 1) {
        const double o1 = shfl_down(g1, d), o2 = shfl_down(g2, d);
        if (s + d < 32) {
            const double *m = T.sb + ((size_t)k * kMaxSeg + s) * 4;
            g1 = fma(__ldg(m + 0), o1, fma(__ldg(m + 1), o2, g1));
            g2 = fma(__ldg(m + 2), o1, fma(__ldg(m + 3), o2, g2));
        }
    }
    y1 = shfl_down(g1, 1);
    y2 = shfl_down(g2, 1);
    if (s == 31) y1 = y2 = 0.0;
#pragma unroll
    for (int t = S - 1; t >= 0; t--) {
        const double v = ((r[t] - Q1(t) * y1) - Q2(t) * y2) * ID(t);
        y2 = y1; y1 = v; r[t] = v;
    }
}

// ---- kernels -------------------------------------------------------------------
enum Kind2 { K2_D1 = 0, K2_D2 = 1, K2_FILTER = 2 };

// Shared memory of a kernel: the factor tables, NB ring slots of NI tile
// buffers each, and a tile buffer of its own for the second derivative's
// first derivative (iadd).  Three slots when they fit, else two.
template <int S, int KIND, int OP, int KW, class T>
struct Ring {
    using A = typename Elt<T>::A;
    static constexpr int NI = NIn<OP>::v;
    static constexpr int NT = KIND == K2_FILTER ? 5 : (KIND == K2_D2 ? 6 : 3);   // factor tables
    static constexpr size_t kTab = ((size_t)NT * 32 * S * sizeof(A) + 15) / 16 * 16;
    static constexpr size_t kBuf = (size_t)Pad<S, KW>::TB * 8;
    static constexpr int kExtra = KIND == K2_D2 ? 1 : 0;
    static constexpr size_t kMax = 227 * 1024;
    static constexpr int NB = (kTab + (3 * NI + kExtra) * kBuf <= kMax) ? 3 : 2;
    static constexpr size_t kSmem = kTab + (NB * NI + kExtra) * kBuf;
    static constexpr bool kFits = kSmem <= kMax;
};

// stores a tile's results: O (=|+=) R, or O = (R + E1) + E2; R2 -> O2 when set
template <int S, int KW, class T>
__device__ __forceinline__ void store_tile(const typename Elt<T>::E *R, T *O, const typename Elt<T>::E *R2, T *O2,
                                           const ColMap &m, int dir, int add, const T *E1, const T *E2) {
    using V = typename Elt<T>::V;
    constexpr int LPW = Elt<T>::LPW;
#pragma unroll 4
    for (int k = 0; k < S; k++) {
        int w, r;
        slot<S, KW>(dir, (int)threadIdx.x + KW * 32 * k, w, r);
        const int q = w * Pad<S, KW>::LS + pidx<S>(r);
        if constexpr (LPW == 1) {
            const size_t o = m.base + goff<T>(m, w, r, 0);
            double v = R[q];
            if (E1) v = (v + __ldg(E1 + o)) + __ldg(E2 + o);
            else if (add) v = O[o] + v;
            O[o] = v;
            if (R2) O2[o] = R2[q];
        } else {
            V v = Elt<T>::get(R[q]);
            V v2 = R2 ? Elt<T>::get(R2[q]) : V(0.0);
            if (dir != 1) {            // the two lines are adjacent: one 8-byte access
                const size_t o = m.base + goff<T>(m, w, r, 0);
                if (E1) v = (v + Ld<F2, float>::get(E1 + o)) + Ld<F2, float>::get(E2 + o);
                else if (add) v = ldp2(O + o) + v;
                stv(O + o, v);
                if (R2) stv(O2 + o, v2);
            } else {
                const size_t o0 = m.base + goff<T>(m, w, r, 0), o1 = m.base + goff<T>(m, w, r, 1);
                if (E1) {
                    v = (v + F2(__ldg(E1 + o0), __ldg(E1 + o1))) + F2(__ldg(E2 + o0), __ldg(E2 + o1));
                } else if (add) {
                    v = F2(O[o0], O[o1]) + v;
                }
                O[o0] = v.x; O[o1] = v.y;
                if (R2) { O2[o0] = v2.x; O2[o1] = v2.y; }
            }
        }
    }
}

// One kernel for the three solve kinds: K2_D1 (DF*: O1 = fac1 * d/ds of the
// producer OP of the input fields, iadd accumulates, E1/E2 fused sum), K2_D2
// (D2F*2: O2 = second derivative, plus O1 = first derivative when iadd) and
// K2_FILTER (Compact_Filter_*, FP64: O1 = filtered F, O1 may alias F).
template <int S, int KIND, int OP, int KW, class T>
__global__ void __launch_bounds__(KW * 32, 1) k_line2(LineArgsT<T> a, unsigned ntiles) {
    using RG = Ring<S, KIND, OP, KW, T>;
    using E = typename Elt<T>::E;
    using V = typename Elt<T>::V;
    using A = typename Elt<T>::A;
    constexpr int n = 32 * S, TB = Pad<S, KW>::TB, NB = RG::NB, NI = RG::NI;
    constexpr int NL = KW * Elt<T>::LPW, SP = Pad<S, KW>::SP, LS = Pad<S, KW>::LS;
    extern __shared__ __align__(16) unsigned char sm2_raw[];
    A *tab = reinterpret_cast<A *>(sm2_raw);                             // factor tables
    E *ring = reinterpret_cast<E *>(sm2_raw + RG::kTab);                 // NB slots x NI tiles
    E *xout = ring + (size_t)NB * NI * TB;                               // K2_D2 with iadd
    if constexpr (KIND == K2_FILTER) {
        stage_table<S>(tab, a.p.p1); stage_table<S>(tab + n, a.p.p2); stage_table<S>(tab + 2 * n, a.p.q1);
        stage_table<S>(tab + 3 * n, a.p.q2); stage_table<S>(tab + 4 * n, a.p.id);
    } else {
        const TriTabT<A> &Tt = KIND == K2_D1 ? a.t1 : a.t2;
        stage_table<S>(tab, Tt.l); stage_table<S>(tab + n, Tt.up); stage_table<S>(tab + 2 * n, Tt.id);
        if (KIND == K2_D2 && a.iadd) {
            stage_table<S>(tab + 3 * n, a.t1.l); stage_table<S>(tab + 4 * n, a.t1.up);
            stage_table<S>(tab + 5 * n, a.t1.id);
        }
    }
    const T *fin[4] = {a.F.a, a.F.b, a.F.c, a.F.d};
    auto issue = [&](int sl, unsigned t) {
        const ColMap m = tile_map<NL>(a.geo, t);
#pragma unroll
        for (int i = 0; i < NI; i++) issue_field<S, KW, T>(ring + ((size_t)sl * NI + i) * TB, fin[i], m, a.geo.dir);
    };
    const unsigned step = gridDim.x;
#pragma unroll
    for (int q = 0; q < NB - 1; q++) {
        const unsigned t = blockIdx.x + q * step;
        if (t < ntiles) issue(q, t);
        cp_commit();
    }
    const int w = threadIdx.x >> 5, s = threadIdx.x & 31;
    int cur = 0;
    for (unsigned t = blockIdx.x; t < ntiles; t += step) {
        {   // copies of the tile NB-1 ahead, into the slot the previous tile freed
            const unsigned tn = t + (NB - 1) * step;
            int sn = cur + NB - 1;
            if (sn >= NB) sn -= NB;
            if (tn < ntiles) issue(sn, tn);
            cp_commit();
        }
        cp_wait<NB - 1>();
        __syncthreads();
        E *buf = ring + (size_t)cur * NI * TB;
        Slot<OP, T> sl;
#pragma unroll
        for (int i = 0; i < 4; i++) sl.f[i] = buf + (size_t)(i < NI ? i : 0) * TB + w * LS;
        sl.P = &a.F;
        const TileRow<S, OP, T> rd{sl};
        const int row0 = s * S;
        E *Ln = buf + w * LS;                       // results replace the first input's tile
        if constexpr (KIND == K2_FILTER) {
            double v[S + 8];
            window<S, 4>(v, sl, s);
            rhs_filter<S, 4>(v, row0, n, a.asym, 0, a.K, rd);
            pen_solve_w<S>(v, a.p, tab, s);
            __syncwarp();
#pragma unroll
            for (int q = 0; q < S; q++) Elt<T>::put(Ln[s * SP + q], v[q]);
        } else if constexpr (KIND == K2_D1) {
            V v[S + 4];
            window<S, 2>(v, sl, s);
            rhs_d1<S, 2>(v, row0, n, a.asym, 0, a.fac1, a.K, rd);
            tri_solve_w<S>(v, a.t1, tab, s);
            __syncwarp();
#pragma unroll
            for (int q = 0; q < S; q++) Elt<T>::put(Ln[s * SP + q], v[q]);
        } else {
            V v[S + 4], u[S + 4];
            window<S, 2>(v, sl, s);
            if (a.iadd) {
#pragma unroll
                for (int q = 0; q < S + 4; q++) u[q] = v[q];
            }
            rhs_d2<S, 2>(v, row0, n, a.asym, 0, a.fac2, a.K, rd);
            tri_solve_w<S>(v, a.t2, tab, s);
            if (a.iadd) {
                rhs_d1<S, 2>(u, row0, n, a.asym, 0, a.fac1, a.K, rd);
                tri_solve_w<S>(u, a.t1, tab + 3 * n, s);
                E *Lx = xout + w * LS;
#pragma unroll
                for (int q = 0; q < S; q++) Elt<T>::put(Lx[s * SP + q], u[q]);
            }
            __syncwarp();
#pragma unroll
            for (int q = 0; q < S; q++) Elt<T>::put(Ln[s * SP + q], v[q]);
        }
        __syncthreads();
        const ColMap m = tile_map<NL>(a.geo, t);
        if constexpr (KIND == K2_D2)
            store_tile<S, KW, T>(buf, a.O2, a.iadd ? xout : nullptr, a.O1, m, a.geo.dir, 0, a.E1, a.E2);
        else
            store_tile<S, KW, T>(buf, a.O1, nullptr, nullptr, m, a.geo.dir, KIND == K2_D1 ? a.iadd : 0, a.E1,
                                 a.E2);
        __syncthreads();
        cur = cur + 1 == NB ? 0 : cur + 1;
    }
    cp_wait<0>();
}

// CTAs of the persistent launch: one per SM (the ring fills most of the
// shared memory)
inline int persistent_ctas(int dev) {
    static int sms[64] = {0};
    if (dev < 0 || dev >= 64) return 148;
    if (!sms[dev]) {
        int v = 0;
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        sms[dev] = v > 0 ? v : 148;
    }
    return sms[dev];
}

}  // namespace lk2
}  // namespace st
