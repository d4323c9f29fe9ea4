// st_kernels.cu - compact derivative, compact filter and Gaussian filter line
// operators, and the general (per-line coefficient) tri/pentadiagonal solvers.
#include <cfloat>
#include "st_line.cuh"

namespace st {

struct LineArgs {
    Prod F;
    double *O1, *O2;
    LineGeo geo;
    int S, P;
    double fac1, fac2;
    int asym, iadd;
    TriTab t1, t2;
    PenTab p;
    Consts K;
};

// Every line kernel is instantiated for x/z lines (YT = false: direct
// coalesced row accesses) and for y lines (YT = true: staged through a
// shared [32][n+1] tile).
#define LINE_PROLOGUE                                                                  \
    __shared__ CarryBuf cb;                                                            \
    extern __shared__ double tile[];                                                   \
    const int lane = threadIdx.x & (kLanes - 1), s = threadIdx.x / kLanes, n = a.geo.n, row0 = s * S; \
    const ColMap m = a.geo.map(blockIdx.x);                                            \
    const RowReader<OP> rd = YT ? RowReader<OP>{tile + lane * (n + 1), nullptr, 0, 0}  \
                                : RowReader<OP>{nullptr, &a.F, m.base + (size_t)lane * m.lstride, m.rstride};

template <int S, int H, bool YT, int OP>
__device__ __forceinline__ void get_rows(double (&v)[S + 2 * H], const double *tile, const Prod &F,
                                         const ColMap &m, int lane, int a, int n) {
    if (YT) ytile_rows<S, H>(v, tile, lane, a, n);
    else load_rows<S, H, OP>(v, F, m, lane, a, n);
}
template <int S, bool YT, int N>
__device__ __forceinline__ void put_rows(const double (&v)[N], double *tile, double *O, const ColMap &m,
                                         int lane, int a, int n, int add) {
    if (YT) {
        __syncthreads();                 // every thread has finished reading the tile
        ytile_put<S>(tile, v, lane, a, n);
        __syncthreads();
        ytile_store(tile, O, m.base, n, add);
    } else {
        store_rows<S>(v, O, m, lane, a, add);
    }
}

// DF*_sym/_asym: O1 (=|+=) cadd * dF/ds
template <int S, bool YT, int OP>
__global__ void __launch_bounds__(512, 2) k_dfd(LineArgs a) {
    LINE_PROLOGUE
    if (YT) { ytile_load<OP>(tile, a.F, m.base, n); __syncthreads(); }
    double v[S + 4];
    get_rows<S, 2, YT, OP>(v, tile, a.F, m, lane, row0, n);
    rhs_d1<S, 2>(v, row0, n, a.asym, a.fac1, a.K, rd);
    tri_solve<S>(v, a.t1, s, a.P, lane, cb);
    put_rows<S, YT>(v, tile, a.O1, m, lane, row0, n, a.iadd);
}

// D2F*2_sym/_asym: O2 = d2F/ds2; if iadd, O1 = dF/ds (cadd = 1).  The first
// derivative re-reads the rows (the CTA's lines are still in L2).
template <int S, bool YT>
__global__ void __launch_bounds__(512, 2) k_d2fd2(LineArgs a) {
    constexpr int OP = PR_A;
    LINE_PROLOGUE
    {
        if (YT) { ytile_load<OP>(tile, a.F, m.base, n); __syncthreads(); }
        double v[S + 4];
        get_rows<S, 2, YT, OP>(v, tile, a.F, m, lane, row0, n);
        rhs_d2<S, 2>(v, row0, n, a.asym, a.fac2, a.K, rd);
        tri_solve<S>(v, a.t2, s, a.P, lane, cb);
        put_rows<S, YT>(v, tile, a.O2, m, lane, row0, n, 0);
    }
    if (a.iadd) {
        __syncthreads();   // carry buffers and tile are reused
        if (YT) { ytile_load<OP>(tile, a.F, m.base, n); __syncthreads(); }
        double v[S + 4];
        get_rows<S, 2, YT, OP>(v, tile, a.F, m, lane, row0, n);
        rhs_d1<S, 2>(v, row0, n, a.asym, a.fac1, a.K, rd);
        tri_solve<S>(v, a.t1, s, a.P, lane, cb);
        put_rows<S, YT>(v, tile, a.O1, m, lane, row0, n, 0);
    }
}

// Compact_Filter_*_sym/_asym: O1 = filtered F.  O1 may alias F: every read of
// F (including the boundary re-reads) happens before the solve's first
// barrier and every write after its last one.
template <int S, bool YT>
__global__ void __launch_bounds__(512, 2) k_filter(LineArgs a) {
    constexpr int OP = PR_A;
    LINE_PROLOGUE
    if (YT) { ytile_load<OP>(tile, a.F, m.base, n); __syncthreads(); }
    double v[S + 8];
    get_rows<S, 4, YT, OP>(v, tile, a.F, m, lane, row0, n);
    rhs_filter<S, 4>(v, row0, n, a.asym, a.K, rd);
    pen_solve<S>(v, a.p, s, a.P, lane, cb);
    put_rows<S, YT>(v, tile, a.O1, m, lane, row0, n, 0);
}

// Gaussian_Filter_X/Y/Z: O1 = explicit 9-point Gaussian of F (O1 != F)
template <int S, bool YT>
__global__ void __launch_bounds__(512, 2) k_gauss(LineArgs a) {
    constexpr int OP = PR_A;
    LINE_PROLOGUE
    (void)cb;
    if (YT) { ytile_load<OP>(tile, a.F, m.base, n); __syncthreads(); }
    double v[S + 8];
    get_rows<S, 4, YT, OP>(v, tile, a.F, m, lane, row0, n);
    rhs_gauss<S, 4>(v, row0, n, a.K, rd);
    put_rows<S, YT>(v, tile, a.O1, m, lane, row0, n, 0);
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

template <int S, bool YT>
static void launch_SY(st_ctx *c, OpKind op, const LineArgs &a, cudaStream_t st) {
    const size_t nlines = c->dm.n3 / (size_t)a.geo.n;
    dim3 grid((unsigned)(nlines / kLanes)), block(kLanes * a.P);
    const size_t smem = YT ? (size_t)kLanes * (a.geo.n + 1) * sizeof(double) : 0;
    // algorithmic bytes: every input and output field touched once
    const double n3 = (double)c->dm.n3;
    // inputs: 1 field, or every field a producer expression reads
    static const int nin[6] = {1, 2, 3, 3, 3, 4};
    double b = 8.0 * nin[a.F.op] + 8.0;          // + one output
    if (op == OP_D1 && a.iadd) b += 8.0;           // read-modify-write
    if (op == OP_D2 && a.iadd) b += 8.0;           // second output
    static const char *names[4] = {"k_dfd", "k_d2fd2", "k_filter", "k_gauss"};
    int pi = prof_start(c, names[op], b * n3);
    switch (op) {
        case OP_D1:
            switch (a.F.op) {
#define PCASE(o_) case o_: set_smem<k_dfd<S, YT, o_>>(smem); k_dfd<S, YT, o_><<<grid, block, smem, st>>>(a); break;
                PCASE(PR_A) PCASE(PR_MUL) PCASE(PR_ADDMUL) PCASE(PR_MULMUL) PCASE(PR_SPEC) PCASE(PR_SPECT)
#undef PCASE
            }
            break;
        case OP_D2: set_smem<k_d2fd2<S, YT>>(smem); k_d2fd2<S, YT><<<grid, block, smem, st>>>(a); break;
        case OP_FILTER: set_smem<k_filter<S, YT>>(smem); k_filter<S, YT><<<grid, block, smem, st>>>(a); break;
        case OP_GAUSS: set_smem<k_gauss<S, YT>>(smem); k_gauss<S, YT><<<grid, block, smem, st>>>(a); break;
    }
    prof_stop(c, pi);
}

template <int S>
static void launch_S(st_ctx *c, OpKind op, const LineArgs &a, cudaStream_t st) {
    if (a.geo.dir == 1) launch_SY<S, true>(c, op, a, st);
    else launch_SY<S, false>(c, op, a, st);
}

static int launch_line(st_ctx *c, OpKind op, const LineArgs &a) {
    switch (a.S) {
#define CASE(s_) case s_: launch_S<s_>(c, op, a, c->stream); break;
        CASE(2) CASE(3) CASE(4) CASE(6) CASE(8) CASE(12) CASE(16)
#undef CASE
        default: return fail(c, ST_E_UNSUPPORTED, "unsupported line segmentation");
    }
    ST_CUDA(c, cudaGetLastError());
    return ST_OK;
}

static LineArgs make_args(st_ctx *c, int dir) {
    LineArgs a{};
    a.geo.dir = dir;
    a.geo.n = c->dm.n[dir];
    a.geo.My = c->dm.n[1];
    a.geo.Mz = c->dm.n[2];
    a.S = c->seg[dir];
    a.P = a.geo.n / a.S;
    a.K = c->k;
    return a;
}

static Prod plain(const double *F) {
    Prod p{};
    p.op = PR_A;
    p.a = F;
    return p;
}

int dev_dfd(st_ctx *c, int dir, int asym, const double *F, double *dF, int iadd, double cadd) {
    return dev_dfd_prod(c, dir, asym, plain(F), dF, iadd, cadd);
}

int dev_dfd_prod(st_ctx *c, int dir, int asym, const Prod &F, double *dF, int iadd, double cadd) {
    LineArgs a = make_args(c, dir);
    a.F = F; a.O1 = dF; a.asym = asym; a.iadd = iadd;
    a.fac1 = cadd * c->s1[dir] * (double)(a.geo.n - 1);           // src/derivCDopt6_sym_tri.f:424
    a.t1 = c->tri[dir][asym ? K_D1A : K_D1S];
    return launch_line(c, OP_D1, a);
}

int dev_d2fd2(st_ctx *c, int dir, int asym, const double *F, double *dF, double *d2F, int iadd) {
    LineArgs a = make_args(c, dir);
    a.F = plain(F); a.O1 = dF; a.O2 = d2F; a.asym = asym; a.iadd = iadd;
    a.fac1 = 1.0 * c->s1[dir] * (double)(a.geo.n - 1);
    a.fac2 = ((double)((a.geo.n - 1) * (a.geo.n - 1))) * c->s2[dir];   // src/derivCDopt6_sym_tri.f:554
    a.t1 = c->tri[dir][asym ? K_D1A : K_D1S];
    a.t2 = c->tri[dir][asym ? K_D2A : K_D2S];
    return launch_line(c, OP_D2, a);
}

int dev_filter(st_ctx *c, int dir, int asym, const double *F, double *F0) {
    LineArgs a = make_args(c, dir);
    a.F = plain(F); a.O1 = F0; a.asym = asym;
    a.p = c->pen[dir][asym ? K_FA : K_FS];
    return launch_line(c, OP_FILTER, a);
}

int dev_gauss(st_ctx *c, int dir, const double *F, double *Fg) {
    LineArgs a = make_args(c, dir);
    a.F = plain(F); a.O1 = Fg;
    return launch_line(c, OP_GAUSS, a);
}

// ---- general solvers (per-line coefficients), thread per line ---------------
// tridiagonal_serial / tridiagonal_periodic_serial, src/tridiagonal.f90:197-287.
// Arrays (lot,n) with lot fastest; A,B,C are copied into scratch first (the
// reference's A=A1; B=B1; C=C1).
__global__ void k_tri_general(double *a, double *b, const double *cc, double *R, int n, int lot,
                              int nper) {
    int L = blockIdx.x * blockDim.x + threadIdx.x;
    if (L >= lot) return;
    const double tiny = (double)FLT_MIN;
#define A_(i) a[(size_t)(i) * lot + L]
#define B_(i) b[(size_t)(i) * lot + L]
#define C_(i) cc[(size_t)(i) * lot + L]
#define R_(i) R[(size_t)(i) * lot + L]
    if (nper == 0) {
        for (int i = 1; i < n; i++) {
            double cs = A_(i) / (B_(i - 1) + tiny);
            B_(i) = B_(i) - C_(i - 1) * cs;
            R_(i) = R_(i) - R_(i - 1) * cs;
        }
        R_(n - 1) = R_(n - 1) / B_(n - 1);
        for (int i = n - 2; i >= 0; i--) R_(i) = (R_(i) - C_(i) * R_(i + 1)) / (B_(i) + tiny);
        return;
    }
    double c0 = C_(0);
    if (n == 1) { R_(0) = R_(0) / (A_(0) + B_(0) + C_(0)); return; }
    if (n == 2) {
        c0 = C_(0) + A_(0);
        A_(1) = A_(1) + C_(1);
        double cs = A_(1) / B_(0);
        B_(1) = B_(1) - c0 * cs;
        R_(1) = R_(1) - R_(0) * cs;
        R_(1) = R_(1) / B_(1);
        R_(0) = (R_(0) - c0 * R_(1)) / B_(0);
        return;
    }
    for (int i = 1; i <= n - 3; i++) {
        double cs = A_(i) / B_(i - 1);
        B_(i) = B_(i) - C_(i - 1) * cs;
        R_(i) = R_(i) - R_(i - 1) * cs;
        A_(i) = -A_(i - 1) * cs;
    }
    int i = n - 2;
    double cs = A_(i) / B_(i - 1);
    B_(i) = B_(i) - C_(i - 1) * cs;
    R_(i) = R_(i) - R_(i - 1) * cs;
    A_(i) = C_(i) - A_(i - 1) * cs;
    i = n - 1;
    cs = A_(i) / B_(i - 1);
    R_(i) = R_(i) - R_(i - 1) * cs;
    A_(i) = B_(i) - A_(i - 1) * cs;
    for (i = n - 3; i >= 0; i--) {
        cs = C_(i) / B_(i + 1);
        R_(i) = R_(i) - R_(i + 1) * cs;
        A_(i) = A_(i) - A_(i + 1) * cs;
    }
    cs = C_(n - 1) / B_(0);
    R_(n - 1) = R_(n - 1) - R_(0) * cs;
    A_(n - 1) = A_(n - 1) - A_(0) * cs;
    R_(n - 1) = R_(n - 1) / A_(n - 1);
    for (i = n - 2; i >= 0; i--) R_(i) = (R_(i) - A_(i) * R_(n - 1)) / B_(i);
#undef A_
#undef B_
#undef C_
#undef R_
}

// pentadiagonal_serial / pentadiagonal_periodic_serial,
// src/pentadiagonal.f90:319-504 (n >= 5 for the periodic path)
__global__ void k_pen_general(double *A, double *B, double *C, double *D, double *E, double *R,
                              double *s1, double *s2, int n, int lot, int nper) {
    int L = blockIdx.x * blockDim.x + threadIdx.x;
    if (L >= lot) return;
    const double tiny = (double)FLT_MIN;
#define X_(arr, i) arr[(size_t)(i) * lot + L]
    if (nper == 0) {
        if (n == 1) { X_(R, 0) = X_(R, 0) / X_(C, 0); return; }
        if (n == 2) {
            double cs = X_(B, 1) / X_(C, 0);
            X_(C, 1) = X_(C, 1) - X_(D, 0) * cs;
            X_(R, 1) = X_(R, 1) - X_(R, 0) * cs;
            X_(R, 1) = X_(R, 1) / X_(C, 1);
            X_(R, 0) = (X_(R, 0) - X_(D, 0) * X_(R, 1)) / X_(C, 0);
            return;
        }
        for (int i = 0; i <= n - 3; i++) {
            double cs = X_(B, i + 1) / (X_(C, i) + tiny);
            X_(C, i + 1) = X_(C, i + 1) - X_(D, i) * cs;
            X_(D, i + 1) = X_(D, i + 1) - X_(E, i) * cs;
            X_(R, i + 1) = X_(R, i + 1) - X_(R, i) * cs;
            cs = X_(A, i + 2) / (X_(C, i) + tiny);
            X_(B, i + 2) = X_(B, i + 2) - X_(D, i) * cs;
            X_(C, i + 2) = X_(C, i + 2) - X_(E, i) * cs;
            X_(R, i + 2) = X_(R, i + 2) - X_(R, i) * cs;
        }
        double cs = X_(B, n - 1) / (X_(C, n - 2) + tiny);
        X_(C, n - 1) = X_(C, n - 1) - X_(D, n - 2) * cs;
        X_(R, n - 1) = X_(R, n - 1) - X_(R, n - 2) * cs;
        X_(R, n - 1) = X_(R, n - 1) / (X_(C, n - 1) + tiny);
        X_(R, n - 2) = (X_(R, n - 2) - X_(D, n - 2) * X_(R, n - 1)) / (X_(C, n - 2) + tiny);
        for (int i = n - 3; i >= 0; i--)
            X_(R, i) = (X_(R, i) - X_(D, i) * X_(R, i + 1) - X_(E, i) * X_(R, i + 2)) / (X_(C, i) + tiny);
        return;
    }
    for (int i = 0; i < n; i++) { X_(s1, i) = 0.0; X_(s2, i) = 0.0; }
    if (n == 4) for (int i = 0; i < 4; i++) { X_(A, i) = X_(A, i) + X_(E, i); X_(E, i) = 0.0; }
    X_(s1, 0) = X_(A, 0);
    X_(s1, n - 4) = X_(s1, n - 4) + X_(E, n - 4);
    X_(s1, n - 3) = X_(D, n - 3);
    X_(s1, n - 2) = X_(C, n - 2);
    X_(s1, n - 1) = X_(B, n - 1);
    X_(s2, 0) = X_(B, 0);
    X_(s2, 1) = X_(A, 1);
    X_(s2, n - 3) = X_(s2, n - 3) + X_(E, n - 3);
    X_(s2, n - 2) = X_(D, n - 2);
    X_(s2, n - 1) = X_(C, n - 1);
    for (int i = 0; i <= n - 3; i++) {
        double cs = X_(B, i + 1) / X_(C, i);
        X_(C, i + 1) = X_(C, i + 1) - X_(D, i) * cs;
        X_(D, i + 1) = X_(D, i + 1) - X_(E, i) * cs;
        X_(R, i + 1) = X_(R, i + 1) - X_(R, i) * cs;
        X_(s1, i + 1) = X_(s1, i + 1) - X_(s1, i) * cs;
        X_(s2, i + 1) = X_(s2, i + 1) - X_(s2, i) * cs;
        cs = X_(A, i + 2) / X_(C, i);
        X_(B, i + 2) = X_(B, i + 2) - X_(D, i) * cs;
        X_(C, i + 2) = X_(C, i + 2) - X_(E, i) * cs;
        X_(R, i + 2) = X_(R, i + 2) - X_(R, i) * cs;
        X_(s1, i + 2) = X_(s1, i + 2) - X_(s1, i) * cs;
        X_(s2, i + 2) = X_(s2, i + 2) - X_(s2, i) * cs;
    }
    for (int i = n - 3; i >= 2; i--) {
        double cs = X_(D, i - 1) / X_(C, i);
        X_(R, i - 1) = X_(R, i - 1) - X_(R, i) * cs;
        X_(s1, i - 1) = X_(s1, i - 1) - X_(s1, i) * cs;
        X_(s2, i - 1) = X_(s2, i - 1) - X_(s2, i) * cs;
        cs = X_(E, i - 2) / X_(C, i);
        X_(R, i - 2) = X_(R, i - 2) - X_(R, i) * cs;
        X_(s1, i - 2) = X_(s1, i - 2) - X_(s1, i) * cs;
        X_(s2, i - 2) = X_(s2, i - 2) - X_(s2, i) * cs;
    }
    {
        double cs = X_(D, 0) / X_(C, 1);
        X_(R, 0) = X_(R, 0) - X_(R, 1) * cs;
        X_(s1, 0) = X_(s1, 0) - X_(s1, 1) * cs;
        X_(s2, 0) = X_(s2, 0) - X_(s2, 1) * cs;
    }
    double cs = X_(E, n - 2) / X_(C, 0);
    X_(R, n - 2) = X_(R, n - 2) - X_(R, 0) * cs;
    X_(s1, n - 2) = X_(s1, n - 2) - X_(s1, 0) * cs;
    X_(s2, n - 2) = X_(s2, n - 2) - X_(s2, 0) * cs;
    cs = X_(D, n - 1) / X_(C, 0);
    X_(R, n - 1) = X_(R, n - 1) - X_(R, 0) * cs;
    X_(s1, n - 1) = X_(s1, n - 1) - X_(s1, 0) * cs;
    X_(s2, n - 1) = X_(s2, n - 1) - X_(s2, 0) * cs;
    cs = X_(E, n - 1) / X_(C, 1);
    X_(R, n - 1) = X_(R, n - 1) - X_(R, 1) * cs;
    X_(s1, n - 1) = X_(s1, n - 1) - X_(s1, 1) * cs;
    X_(s2, n - 1) = X_(s2, n - 1) - X_(s2, 1) * cs;
    cs = X_(s1, n - 1) / X_(s1, n - 2);
    X_(R, n - 1) = X_(R, n - 1) - X_(R, n - 2) * cs;
    X_(s2, n - 1) = X_(s2, n - 1) - X_(s2, n - 2) * cs;
    X_(R, n - 1) = X_(R, n - 1) / X_(s2, n - 1);
    X_(R, n - 2) = (X_(R, n - 2) - X_(s2, n - 2) * X_(R, n - 1)) / X_(s1, n - 2);
    for (int i = n - 3; i >= 0; i--)
        X_(R, i) = (X_(R, i) - X_(s1, i) * X_(R, n - 2) - X_(s2, i) * X_(R, n - 1)) / X_(C, i);
#undef X_
}

int dev_tridiagonal(st_ctx *c, const double *A, const double *B, const double *C, double *R, int n,
                    int lot, int nper) {
    size_t N = (size_t)n * lot;
    double *a = nullptr, *b = nullptr;
    ST_CUDA(c, cudaMallocAsync(&a, 2 * N * sizeof(double), c->stream));
    b = a + N;
    ST_CUDA(c, cudaMemcpyAsync(a, A, N * 8, cudaMemcpyDeviceToDevice, c->stream));
    ST_CUDA(c, cudaMemcpyAsync(b, B, N * 8, cudaMemcpyDeviceToDevice, c->stream));
    int pi = prof_start(c, "k_tri_general", 32.0 * N);
    k_tri_general<<<(lot + 127) / 128, 128, 0, c->stream>>>(a, b, C, R, n, lot, nper);
    prof_stop(c, pi);
    cudaError_t e = cudaGetLastError();
    cudaFreeAsync(a, c->stream);
    if (e != cudaSuccess) return fail(c, ST_E_CUDA, cudaGetErrorString(e));
    return ST_OK;
}

int dev_pentadiagonal(st_ctx *c, const double *A, const double *B, const double *C, const double *D,
                      const double *E, double *R, int n, int lot, int nper) {
    if (nper && n < 5) return fail(c, ST_E_UNSUPPORTED, "periodic pentadiagonal needs n >= 5");
    size_t N = (size_t)n * lot;
    double *buf = nullptr;
    ST_CUDA(c, cudaMallocAsync(&buf, 7 * N * sizeof(double), c->stream));
    double *a = buf, *b = buf + N, *cc = buf + 2 * N, *d = buf + 3 * N, *e = buf + 4 * N;
    double *s1 = buf + 5 * N, *s2 = buf + 6 * N;
    const double *src[5] = {A, B, C, D, E};
    double *dst[5] = {a, b, cc, d, e};
    for (int q = 0; q < 5; q++)
        ST_CUDA(c, cudaMemcpyAsync(dst[q], src[q], N * 8, cudaMemcpyDeviceToDevice, c->stream));
    int pi = prof_start(c, "k_pen_general", 48.0 * N);
    k_pen_general<<<(lot + 127) / 128, 128, 0, c->stream>>>(a, b, cc, d, e, R, s1, s2, n, lot, nper);
    prof_stop(c, pi);
    cudaError_t er = cudaGetLastError();
    cudaFreeAsync(buf, c->stream);
    if (er != cudaSuccess) return fail(c, ST_E_CUDA, cudaGetErrorString(er));
    return ST_OK;
}

}  // namespace st
