// st_linekern.cuh - the line-operator kernels (compact derivatives, compact
// filter, Gaussian filter) and their launch dispatch, templated on the family:
// CYC = false for the _mf family's bounded lines, CYC = true for periodic
// lines (wrapped halos and the corner correction after the banded solve).
// The two families are instantiated in separate translation units
// (st_kernels.cu, st_kernels_cyc.cu) so that the bounded-line kernels keep
// their register allocation.
#pragma once
#include <cfloat>
#include "st_line.cuh"

namespace st {

// T: element type of the fields read and written and of the arithmetic:
// double, or float in the FP32 mode, whose kernels give each thread two
// neighbouring lines (value type F2, 32 lines per CTA).
template <class T>
struct LineArgsT {
    ProdT<T> F;
    T *O1, *O2;
    LineGeo geo;
    int S, P;
    double fac1, fac2;
    int asym, iadd;
    const T *E1, *E2;   // x and z lines: O1 (k_dfd) / O2 (k_d2fd2) = (result + E1) + E2 when E1 is set
    int cyc;            // periodic family: wrapped halos, corner correction (selects the CYC kernels)
    TriTabT<T> t1, t2;
    PenTab p;
    Consts K;
};
using LineArgs = LineArgsT<double>;
using LineArgsF = LineArgsT<float>;

// Every line kernel is instantiated for x/z lines (YT = false: direct
// coalesced row accesses) and for y lines (YT = true: staged through a
// shared [32][n+1] tile).
#define LINE_PROLOGUE                                                                  \
    using V = typename Val<T>::V;                                                      \
    using A = typename Val<T>::A;                                                      \
    constexpr int W = Val<T>::W;                                                       \
    __shared__ CarryBufT<V> cb;                                                        \
    extern __shared__ __align__(16) unsigned char smem_raw[];                          \
    A *tile = reinterpret_cast<A *>(smem_raw);                                         \
    const int lane = threadIdx.x & (kLanes - 1), s = threadIdx.x / kLanes, n = a.geo.n, row0 = s * S; \
    const ColMap m = a.geo.template map<W>(blockIdx.x);                                \
    const RowReader<OP, T, V> rd = YT ? RowReader<OP, T, V>{tile + W * lane * (n + 1), nullptr, 0, 0, n + 1} \
                                      : RowReader<OP, T, V>{nullptr, &a.F, m.base + (size_t)lane * W * m.lstride, \
                                                            m.rstride, 0};

// L2 prefetch of the rows the block kAhead blocks later will load (about one
// wave of resident CTAs ahead: 2 per SM on 148 SMs), so that the next wave's
// loads find their lines in L2 while this wave solves.
constexpr unsigned kAhead = kLineCtasPerSm * 148;
__device__ __forceinline__ void pf_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

template <int S, bool YT, int OP, class T>
__device__ __forceinline__ void prefetch_next(const LineGeo &geo, const ProdT<T> &F, int lane, int row0) {
    const unsigned nb = blockIdx.x + kAhead;
    if (nb >= gridDim.x) return;
    constexpr int W = Val<T>::W;
    constexpr int NI = OP == PR_A ? 1 : OP == PR_MUL ? 2 : OP == PR_SPECT ? 4 : 3;   // fields the producer reads
    const ColMap m = geo.template map<W>(nb);
    const T *f[4] = {F.a, F.b, F.c, F.d};
    if (YT) {
        // the block's lines are one contiguous range: one 128-byte line per thread and pass
        const size_t bytes = (size_t)kLanes * W * geo.n * sizeof(T);
        for (size_t off = (size_t)threadIdx.x * 128; off < bytes; off += (size_t)blockDim.x * 128)
#pragma unroll
            for (int k = 0; k < NI; k++) pf_l2(reinterpret_cast<const char *>(f[k] + m.base) + off);
    } else {
        // a row of the block's lines is 128 contiguous bytes: lane 0 of each segment
        if (lane != 0) return;
#pragma unroll
        for (int t = 0; t < S; t++)
#pragma unroll
            for (int k = 0; k < NI; k++) pf_l2(f[k] + m.base + (size_t)(row0 + t) * m.rstride);
    }
}

template <int S, int H, bool YT, int OP, class T, class V, class A>
__device__ __forceinline__ void get_rows(V (&v)[S + 2 * H], const A *tile, const ProdT<T> &F,
                                         const ColMap &m, int lane, int a, int n, int cyc) {
    if (YT) ytile_rows<S, H>(v, tile, lane, a, n, cyc);
    else load_rows<S, H, OP>(v, F, m, lane, a, n, cyc);
}
// SYNCED: a barrier since the last read of the tile (the solves' exchange)
template <int S, bool YT, bool SYNCED, int N, class T, class V, class A>
__device__ __forceinline__ void put_rows(const V (&v)[N], A *tile, T *O, const ColMap &m,
                                         int lane, int a, int n, int add, const T *E1 = nullptr,
                                         const T *E2 = nullptr) {
    if (YT) {
        if (!SYNCED) __syncthreads();    // every thread has finished reading the tile
        ytile_put<S>(tile, v, lane, a, n);
        __syncthreads();
        ytile_store<T>(tile, O, m.base, n, add);
    } else {
        store_rows<S>(v, O, m, lane, a, add, E1, E2);
    }
}

// DF*_sym/_asym and the periodic DF*: O1 (=|+=) cadd * dF/ds
template <int S, bool YT, int OP, bool CYC, class T>
__global__ void __launch_bounds__(kLineThreads, kLineCtasPerSm) k_dfd(LineArgsT<T> a) {
    LINE_PROLOGUE
    if (YT) { ytile_load<OP>(tile, a.F, m.base, n); prefetch_next<S, YT, OP>(a.geo, a.F, lane, row0); __syncthreads(); }
    V v[S + 4];
    get_rows<S, 2, YT, OP>(v, tile, a.F, m, lane, row0, n, CYC);
    if (!YT) prefetch_next<S, YT, OP>(a.geo, a.F, lane, row0);
    rhs_d1<S, 2>(v, row0, n, a.asym, CYC, a.fac1, a.K, rd);
    tri_solve<S>(v, a.t1, s, a.P, lane, cb);
    if constexpr (CYC) cyc_fix<S, S + 4, 2>(v, a.t1.cyc, s, a.P, lane, cb);
    put_rows<S, YT, true>(v, tile, a.O1, m, lane, row0, n, a.iadd, a.E1, a.E2);
}

// D2F*2_sym/_asym and the periodic D2F*2: O2 = d2F/ds2; if iadd, O1 = dF/ds
// (cadd = 1).  The first
// derivative re-reads the rows (the CTA's lines are still in L2).
template <int S, bool YT, bool CYC, class T>
__global__ void __launch_bounds__(kLineThreads, kLineCtasPerSm) k_d2fd2(LineArgsT<T> a) {
    constexpr int OP = PR_A;
    LINE_PROLOGUE
    {
        if (YT) { ytile_load<OP>(tile, a.F, m.base, n); prefetch_next<S, YT, OP>(a.geo, a.F, lane, row0); __syncthreads(); }
        V v[S + 4];
        get_rows<S, 2, YT, OP>(v, tile, a.F, m, lane, row0, n, CYC);
        if (!YT) prefetch_next<S, YT, OP>(a.geo, a.F, lane, row0);
        rhs_d2<S, 2>(v, row0, n, a.asym, CYC, a.fac2, a.K, rd);
        tri_solve<S>(v, a.t2, s, a.P, lane, cb);
        if constexpr (CYC) cyc_fix<S, S + 4, 2>(v, a.t2.cyc, s, a.P, lane, cb);
        put_rows<S, YT, true>(v, tile, a.O2, m, lane, row0, n, 0, a.E1, a.E2);
    }
    if (a.iadd) {
        __syncthreads();   // carry buffers and tile are reused
        if (YT) { ytile_load<OP>(tile, a.F, m.base, n); __syncthreads(); }
        V v[S + 4];
        get_rows<S, 2, YT, OP>(v, tile, a.F, m, lane, row0, n, CYC);
        rhs_d1<S, 2>(v, row0, n, a.asym, CYC, a.fac1, a.K, rd);
        tri_solve<S>(v, a.t1, s, a.P, lane, cb);
        if constexpr (CYC) cyc_fix<S, S + 4, 2>(v, a.t1.cyc, s, a.P, lane, cb);
        put_rows<S, YT, true>(v, tile, a.O1, m, lane, row0, n, 0);
    }
}

// Compact_Filter_*_sym/_asym and the periodic Compact_Filter_*: O1 = filtered
// F.  O1 may alias F: every read of
// F (including the boundary re-reads) happens before the solve's first
// barrier and every write after its last one.
template <int S, bool YT, bool CYC, class T>
__global__ void __launch_bounds__(kLineThreads, kLineCtasPerSm) k_filter(LineArgsT<T> a) {
    constexpr int OP = PR_A;
    LINE_PROLOGUE
    if (YT) { ytile_load<OP>(tile, a.F, m.base, n); prefetch_next<S, YT, OP>(a.geo, a.F, lane, row0); __syncthreads(); }
    double v[S + 8];
    get_rows<S, 4, YT, OP>(v, tile, a.F, m, lane, row0, n, CYC);
    if (!YT) prefetch_next<S, YT, OP>(a.geo, a.F, lane, row0);
    rhs_filter<S, 4>(v, row0, n, a.asym, CYC, a.K, rd);
    pen_solve<S>(v, a.p, s, a.P, lane, cb);
    if constexpr (CYC) cyc_fix<S, S + 8, 4>(v, a.p.cyc, s, a.P, lane, cb);
    put_rows<S, YT, true>(v, tile, a.O1, m, lane, row0, n, 0);
}

// Gaussian_Filter_X/Y/Z (both families): O1 = explicit 9-point Gaussian of F
// (O1 != F)
template <int S, bool YT, bool CYC, class T>
__global__ void __launch_bounds__(kLineThreads, kLineCtasPerSm) k_gauss(LineArgsT<T> a) {
    constexpr int OP = PR_A;
    LINE_PROLOGUE
    (void)cb;
    if (YT) { ytile_load<OP>(tile, a.F, m.base, n); prefetch_next<S, YT, OP>(a.geo, a.F, lane, row0); __syncthreads(); }
    V v[S + 8];
    get_rows<S, 4, YT, OP>(v, tile, a.F, m, lane, row0, n, CYC);
    if (!YT) prefetch_next<S, YT, OP>(a.geo, a.F, lane, row0);
    rhs_gauss<S, 4>(v, row0, n, CYC, a.K, rd);
    put_rows<S, YT, false>(v, tile, a.O1, m, lane, row0, n, 0);
}

// ---- two first derivatives along one direction in one launch ------------
// Hyper_RHS (src/hyper_rhs_sym_mf.f) differentiates, in each direction, a
// viscous flux and then its product with a velocity component (v_h S_12 and
// then v_h S_12 u, or tau_xx and then u tau_xx); Species_RHS
// (src/species_rhs_sym.f) the diffusive flux of Y and then its energy
// counterpart, and Y and then rho u_i Y.  The second operand set contains
// the first, so one CTA runs both on its own lines: the second
// operation finds the shared rows in L2, as the first derivative of
// D2F*2 with iadd does.  (An accumulated output, the pressure-gradient case
// below, is re-read by the thread that wrote it, with plain loads, so it is
// coherent without a barrier.)  The convective fluxes of RHS pair up the same way
// where two adjacent ones share the velocity factor, or where the second
// adds the pressure gradient to what the first wrote.  Each operation is
// exactly the k_dfd of its arguments, so the results are bitwise those of
// two launches.
template <class T>
struct D1OpT {
    ProdT<T> F;
    T *O1;
    double fac1;
    int asym, iadd;
    TriTabT<T> t1;
};
template <class T>
struct D1PairT {
    LineArgsT<T> a;      // geometry, segmentation and scheme constants (its F, O1, t1 unused)
    D1OpT<T> op[2];
};

// block and thread index read so that the compiler keeps nothing derived
// from them live from the first operation to the second
__device__ __forceinline__ unsigned opaque_ctaid() {
    unsigned v;
    asm volatile("mov.u32 %0, %%ctaid.x;" : "=r"(v));
    return v;
}
__device__ __forceinline__ unsigned opaque_tid() {
    unsigned v;
    asm volatile("mov.u32 %0, %%tid.x;" : "=r"(v));
    return v;
}

// one operation; PF: the L2 prefetch of the next wave's rows of the first
// operation (OPF, producer FN), issued with the second operation
template <int S, bool YT, int OP, bool PF, int OPF, class T>
__device__ __forceinline__ void pair_d1(const LineArgsT<T> &a, const D1OpT<T> &o, const ProdT<T> &FN,
                                        CarryBufT<typename Val<T>::V> &cb, typename Val<T>::A *tile) {
    using V = typename Val<T>::V;
    constexpr int W = Val<T>::W;
    const unsigned tid = opaque_tid();
    const int lane = tid & (kLanes - 1), s = tid / kLanes, row0 = s * S, n = a.geo.n;
    const ColMap m = a.geo.template map<W>(opaque_ctaid());
    const RowReader<OP, T, V> rd = YT ? RowReader<OP, T, V>{tile + W * lane * (n + 1), nullptr, 0, 0, n + 1}
                                      : RowReader<OP, T, V>{nullptr, &o.F, m.base + (size_t)lane * W * m.lstride,
                                                            m.rstride, 0};
    if (YT) {
        ytile_load<OP>(tile, o.F, m.base, n);
        if (PF) prefetch_next<S, YT, OPF>(a.geo, FN, lane, row0);
        __syncthreads();
    }
    V v[S + 4];
    get_rows<S, 2, YT, OP>(v, tile, o.F, m, lane, row0, n, 0);
    if (!YT && PF) prefetch_next<S, YT, OPF>(a.geo, FN, lane, row0);
    rhs_d1<S, 2>(v, row0, n, o.asym, 0, o.fac1, a.K, rd);
    tri_solve<S>(v, o.t1, s, a.P, lane, cb);
    put_rows<S, YT, true>(v, tile, o.O1, m, lane, row0, n, o.iadd);
}

template <int S, bool YT, class T, int OP0, int OP1>
__global__ void __launch_bounds__(kLineThreads, kLineCtasPerSm) k_dfd_pair(D1PairT<T> g) {
    using V = typename Val<T>::V;
    using A = typename Val<T>::A;
    __shared__ CarryBufT<V> cb;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    A *tile = reinterpret_cast<A *>(smem_raw);
    pair_d1<S, YT, OP0, false, OP0>(g.a, g.op[0], g.op[0].F, cb, tile);
    __syncthreads();                     // tile and carry buffers are reused
    pair_d1<S, YT, OP1, true, OP0>(g.a, g.op[1], g.op[0].F, cb, tile);
}

enum OpKind { OP_D1, OP_D2, OP_FILTER, OP_GAUSS };

// opt in to the dynamic shared memory a kernel needs on top of its static
// carry buffers (the default cap is 48 KB in total); once per kernel and size
template <auto Kern>
static void set_smem(size_t bytes) {
    static size_t done = 0;   // one counter per kernel instantiation
    if (bytes > done) {
        cudaFuncSetAttribute(Kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        done = bytes;
    }
}

template <int S, bool YT, bool CYC, class T>
static void launch_SY(st_ctx *c, OpKind op, const LineArgsT<T> &a0, cudaStream_t st) {
    const size_t nlines = c->dm.n3 / (size_t)a0.geo.n;     // lines of one case
    constexpr int NL = kLanes * Val<T>::W;
    LineArgsT<T> a = a0;
    a.geo.cblk = (unsigned)(nlines / NL);                  // CTAs per case
    a.geo.cstride = c->dm.n3;
    dim3 grid(a.geo.cblk * (unsigned)c->na), block(kLanes * a.P);
    const size_t smem = YT ? (size_t)NL * (a.geo.n + 1) * sizeof(T) : 0;
    // algorithmic bytes: every input and output field touched once
    const double n3 = (double)c->ncell();
    // inputs: 1 field, or every field a producer expression reads
    static const int nin[6] = {1, 2, 3, 3, 3, 4};
    const double es = (double)sizeof(T);
    double b = es * nin[a.F.op] + es;              // + one output
    if (op == OP_D1 && a.iadd) b += es;            // read-modify-write
    if (op == OP_D2 && a.iadd) b += es;            // second output
    if (a.E1) b += 2 * es;                         // epilogue addends
    static const char *names[4] = {"k_dfd", "k_d2fd2", "k_filter", "k_gauss"};
    int pi = prof_start(c, names[op], b * n3);
    switch (op) {
        case OP_D1:
            switch (a.F.op) {
#define PCASE(o_) case o_: set_smem<k_dfd<S, YT, o_, CYC, T>>(smem); k_dfd<S, YT, o_, CYC, T><<<grid, block, smem, st>>>(a); break;
                PCASE(PR_A) PCASE(PR_MUL) PCASE(PR_ADDMUL) PCASE(PR_MULMUL) PCASE(PR_SPEC) PCASE(PR_SPECT)
#undef PCASE
            }
            break;
        case OP_D2: set_smem<k_d2fd2<S, YT, CYC, T>>(smem); k_d2fd2<S, YT, CYC, T><<<grid, block, smem, st>>>(a); break;
        case OP_FILTER:
            if constexpr (sizeof(T) == 8) {   // the compact filter acts on the FP64 state only
                set_smem<k_filter<S, YT, CYC, T>>(smem); k_filter<S, YT, CYC, T><<<grid, block, smem, st>>>(a);
            }
            break;
        case OP_GAUSS: set_smem<k_gauss<S, YT, CYC, T>>(smem); k_gauss<S, YT, CYC, T><<<grid, block, smem, st>>>(a); break;
    }
    prof_stop(c, pi);
}

template <int S, bool CYC, class T>
static void launch_S(st_ctx *c, OpKind op, const LineArgsT<T> &a, cudaStream_t st) {
    if (a.geo.dir == 1) launch_SY<S, true, CYC, T>(c, op, a, st);
    else launch_SY<S, false, CYC, T>(c, op, a, st);
}

// all line-operator launches of one family (CYC: periodic lines)
template <bool CYC, class T>
static int launch_line_t(st_ctx *c, OpKind op, const LineArgsT<T> &a) {
    switch (a.S) {
#define CASE(s_) case s_: launch_S<s_, CYC, T>(c, op, a, c->stream); break;
        CASE(2) CASE(3) CASE(4) CASE(6) CASE(8) CASE(12) CASE(16)
#undef CASE
        default: return fail(c, ST_E_UNSUPPORTED, "unsupported line segmentation");
    }
    ST_CUDA(c, cudaGetLastError());
    return ST_OK;
}


// one launch of a pair (bounded lines), producers as in kPairOps;
// bytes: algorithmic bytes per cell (every distinct field read or written once)
template <int S, bool YT, class T, int OP0, int OP1>
static void launch_pair_SY(st_ctx *c, const D1PairT<T> &g0, double bytes, cudaStream_t st) {
    const size_t nlines = c->dm.n3 / (size_t)g0.a.geo.n;   // lines of one case
    constexpr int NL = kLanes * Val<T>::W;
    D1PairT<T> g = g0;
    g.a.geo.cblk = (unsigned)(nlines / NL);                  // CTAs per case
    g.a.geo.cstride = c->dm.n3;
    dim3 grid(g.a.geo.cblk * (unsigned)c->na), block(kLanes * g.a.P);
    const size_t smem = YT ? (size_t)NL * (g.a.geo.n + 1) * sizeof(T) : 0;
    int pi = prof_start(c, "k_dfd_pair", bytes * (double)c->ncell());
    set_smem<k_dfd_pair<S, YT, T, OP0, OP1>>(smem);
    k_dfd_pair<S, YT, T, OP0, OP1><<<grid, block, smem, st>>>(g);
    prof_stop(c, pi);
}

// the producer pairs compiled (first, second); pair_kind gives the index
constexpr int kPairOps[][2] = {{PR_A, PR_MUL},   {PR_MUL, PR_MULMUL}, {PR_SPEC, PR_SPECT},
                               {PR_MUL, PR_ADDMUL}, {PR_MUL, PR_A},    {PR_MUL, PR_MUL}};
inline int pair_kind(int op0, int op1) {
    for (int k = 0; k < (int)(sizeof(kPairOps) / sizeof(kPairOps[0])); k++)
        if (kPairOps[k][0] == op0 && kPairOps[k][1] == op1) return k;
    return -1;
}

template <int S, bool YT, class T>
static void launch_pair_SYT(st_ctx *c, const D1PairT<T> &g, double bytes) {
    switch (pair_kind(g.op[0].F.op, g.op[1].F.op)) {
        case 0: launch_pair_SY<S, YT, T, PR_A, PR_MUL>(c, g, bytes, c->stream); break;
        case 1: launch_pair_SY<S, YT, T, PR_MUL, PR_MULMUL>(c, g, bytes, c->stream); break;
        case 2: launch_pair_SY<S, YT, T, PR_SPEC, PR_SPECT>(c, g, bytes, c->stream); break;
        case 3: launch_pair_SY<S, YT, T, PR_MUL, PR_ADDMUL>(c, g, bytes, c->stream); break;
        case 4: launch_pair_SY<S, YT, T, PR_MUL, PR_A>(c, g, bytes, c->stream); break;
        default: launch_pair_SY<S, YT, T, PR_MUL, PR_MUL>(c, g, bytes, c->stream); break;
    }
}

template <class T>
static int launch_pair_t(st_ctx *c, const D1PairT<T> &g, double bytes) {
    switch (g.a.S) {
#define CASE(s_)                                                       \
    case s_:                                                           \
        if (g.a.geo.dir == 1) launch_pair_SYT<s_, true, T>(c, g, bytes); \
        else launch_pair_SYT<s_, false, T>(c, g, bytes);                 \
        break;
        CASE(2) CASE(3) CASE(4) CASE(6) CASE(8) CASE(12) CASE(16)
#undef CASE
        default: return fail(c, ST_E_UNSUPPORTED, "unsupported line segmentation");
    }
    ST_CUDA(c, cudaGetLastError());
    return ST_OK;
}

// launches of the other instantiations, each in its own translation unit:
// periodic lines (st_kernels_cyc.cu), FP32 fields (st_kernels_f32.cu) and
// both (st_kernels_cyc_f32.cu)
int launch_line_cyc(st_ctx *c, OpKind op, const LineArgs &a);
int launch_line_f32(st_ctx *c, OpKind op, const LineArgsF &a);
int launch_line_cyc_f32(st_ctx *c, OpKind op, const LineArgsF &a);

}  // namespace st
