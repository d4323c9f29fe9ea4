// st_kernels.cu - compact derivative, compact filter and Gaussian filter line
// operators (bounded-line instantiations and the entry points of both
// families), and the general (per-line coefficient) tri/pentadiagonal solvers.
#include "st_linekern.cuh"

namespace st {

static int launch_line(st_ctx *c, OpKind op, const LineArgs &a) {
    return a.cyc ? launch_line_cyc(c, op, a) : launch_line_t<false, double>(c, op, a);
}
static int launch_line(st_ctx *c, OpKind op, const LineArgsF &a) {
    return a.cyc ? launch_line_cyc_f32(c, op, a) : launch_line_f32(c, op, a);
}

template <class T = double>
static LineArgsT<T> make_args(st_ctx *c, int dir) {
    LineArgsT<T> a{};
    a.geo.dir = dir;
    a.geo.n = c->dm.n[dir];
    a.geo.My = c->dm.n[1];
    a.geo.Mz = c->dm.n[2];
    a.S = c->seg[dir];
    a.P = a.geo.n / a.S;
    a.K = c->k;
    a.cyc = c->p.family == ST_FAMILY_PERIODIC;
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

// The last pass of a Laplacian with the sum of the three directions fused into
// its store: out = (d(F)/ds + E1) + E2 (first derivative, cadd = 1) or
// (d2(F)/ds2 + E1) + E2; x and z lines only.
int dev_dfd_sum(st_ctx *c, int dir, int asym, const double *F, double *dF, const double *E1, const double *E2) {
    if (dir == 1) return fail(c, ST_E_ARG, "fused sum: x or z lines only");
    LineArgs a = make_args(c, dir);
    a.F = plain(F); a.O1 = dF; a.asym = asym; a.iadd = 0; a.E1 = E1; a.E2 = E2;
    a.fac1 = 1.0 * c->s1[dir] * (double)(a.geo.n - 1);
    a.t1 = c->tri[dir][asym ? K_D1A : K_D1S];
    return launch_line(c, OP_D1, a);
}

int dev_d2fd2_sum(st_ctx *c, int dir, int asym, const double *F, double *d2F, const double *E1,
                  const double *E2) {
    if (dir == 1) return fail(c, ST_E_ARG, "fused sum: x or z lines only");
    LineArgs a = make_args(c, dir);
    a.F = plain(F); a.O2 = d2F; a.asym = asym; a.iadd = 0; a.E1 = E1; a.E2 = E2;
    a.fac2 = ((double)((a.geo.n - 1) * (a.geo.n - 1))) * c->s2[dir];
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

// ---- FP32 mode (float fields and arithmetic, two lines per thread) ----------
static ProdF plain_f(const float *F) {
    ProdF p{};
    p.op = PR_A;
    p.a = F;
    return p;
}

// the kernels access a thread's two lines with one 8-byte load or store
static int check_f2(st_ctx *c, const ProdF &F, const float *O1, const float *O2) {
    const void *ptrs[6] = {F.a, F.b, F.c, F.d, O1, O2};
    for (const void *p : ptrs)
        if (reinterpret_cast<uintptr_t>(p) & 7)
            return fail(c, ST_E_ARG, "FP32 line operators need 8-byte aligned fields");
    return ST_OK;
}

int dev_dfd_prod_f(st_ctx *c, int dir, int asym, const ProdF &F, float *dF, int iadd, double cadd) {
    ST_TRY(check_f2(c, F, dF, nullptr));
    LineArgsF a = make_args<float>(c, dir);
    a.F = F; a.O1 = dF; a.asym = asym; a.iadd = iadd;
    a.fac1 = cadd * c->s1[dir] * (double)(a.geo.n - 1);
    a.t1 = c->trif[dir][asym ? K_D1A : K_D1S];
    return launch_line(c, OP_D1, a);
}

int dev_dfd_f(st_ctx *c, int dir, int asym, const float *F, float *dF, int iadd, double cadd) {
    return dev_dfd_prod_f(c, dir, asym, plain_f(F), dF, iadd, cadd);
}

// ---- two first derivatives along one direction, one launch ---------------------
int launch_pair_f32(st_ctx *c, const D1PairT<float> &g, double bytes);

// Two first derivatives of the bounded lines whose producers form a compiled
// pair (kPairOps) run as one launch, in order; the periodic family and any
// other pair run as two launches, with the same results.  The callers pair
// operations that share fields (the second reads what the first reads, or
// adds to what it wrote), which is where one launch saves DRAM traffic.
template <class T>
static int dfd_pair_t(st_ctx *c, int dir, const D1SpecT<T> *ops) {
    const bool fuse = c->p.family != ST_FAMILY_PERIODIC && pair_kind(ops[0].F.op, ops[1].F.op) >= 0;
    if (!fuse) {
        for (int i = 0; i < 2; i++) {
            if constexpr (sizeof(T) == 8)
                ST_TRY(dev_dfd_prod(c, dir, ops[i].asym, ops[i].F, ops[i].dF, ops[i].iadd, ops[i].cadd));
            else
                ST_TRY(dev_dfd_prod_f(c, dir, ops[i].asym, ops[i].F, ops[i].dF, ops[i].iadd, ops[i].cadd));
        }
        return ST_OK;
    }
    D1PairT<T> g{};
    g.a = make_args<T>(c, dir);
    // algorithmic bytes per cell: each distinct field once (the producers'
    // operands and accumulated outputs read, the outputs written)
    const void *rd[10], *wr[2];
    int nr = 0, nw = 0;
    auto add_once = [](const void **v, int &n, const void *p) {
        for (int k = 0; k < n; k++) if (v[k] == p) return;
        v[n++] = p;
    };
    for (int i = 0; i < 2; i++) {
        const D1SpecT<T> &o = ops[i];
        if constexpr (sizeof(T) == 4) ST_TRY(check_f2(c, o.F, o.dF, nullptr));
        D1OpT<T> &d = g.op[i];
        d.F = o.F; d.O1 = o.dF; d.asym = o.asym; d.iadd = o.iadd;
        d.fac1 = o.cadd * c->s1[dir] * (double)(g.a.geo.n - 1);           // src/derivCDopt6_sym_tri.f:424
        if constexpr (sizeof(T) == 8) d.t1 = c->tri[dir][o.asym ? K_D1A : K_D1S];
        else d.t1 = c->trif[dir][o.asym ? K_D1A : K_D1S];
        const int op = o.F.op, ni = op == PR_A ? 1 : op == PR_MUL ? 2 : op == PR_SPECT ? 4 : 3;
        const T *in[4] = {o.F.a, o.F.b, o.F.c, o.F.d};
        for (int k = 0; k < ni; k++) add_once(rd, nr, in[k]);
        // an accumulated output is read, unless the first operation wrote it
        if (o.iadd && !(i == 1 && o.dF == ops[0].dF)) add_once(rd, nr, o.dF);
        add_once(wr, nw, o.dF);
    }
    const double bytes = (double)sizeof(T) * (double)(nr + nw);
    if constexpr (sizeof(T) == 8) return launch_pair_t<double>(c, g, bytes);
    else return launch_pair_f32(c, g, bytes);
}

int dev_dfd_pair(st_ctx *c, int dir, const D1SpecT<double> *ops) { return dfd_pair_t(c, dir, ops); }
int dev_dfd_pair_f(st_ctx *c, int dir, const D1SpecT<float> *ops) { return dfd_pair_t(c, dir, ops); }

int dev_d2fd2_f(st_ctx *c, int dir, int asym, const float *F, float *dF, float *d2F, int iadd) {
    LineArgsF a = make_args<float>(c, dir);
    a.F = plain_f(F); a.O1 = dF; a.O2 = d2F; a.asym = asym; a.iadd = iadd;
    ST_TRY(check_f2(c, a.F, dF, d2F));
    a.fac1 = 1.0 * c->s1[dir] * (double)(a.geo.n - 1);
    a.fac2 = ((double)((a.geo.n - 1) * (a.geo.n - 1))) * c->s2[dir];
    a.t1 = c->trif[dir][asym ? K_D1A : K_D1S];
    a.t2 = c->trif[dir][asym ? K_D2A : K_D2S];
    return launch_line(c, OP_D2, a);
}

int dev_dfd_sum_f(st_ctx *c, int dir, int asym, const float *F, float *dF, const float *E1, const float *E2) {
    if (dir == 1) return fail(c, ST_E_ARG, "fused sum: x or z lines only");
    ST_TRY(check_f2(c, plain_f(F), dF, E1) == ST_OK ? check_f2(c, plain_f(E2), nullptr, nullptr) : ST_E_ARG);
    LineArgsF a = make_args<float>(c, dir);
    a.F = plain_f(F); a.O1 = dF; a.asym = asym; a.iadd = 0; a.E1 = E1; a.E2 = E2;
    a.fac1 = 1.0 * c->s1[dir] * (double)(a.geo.n - 1);
    a.t1 = c->trif[dir][asym ? K_D1A : K_D1S];
    return launch_line(c, OP_D1, a);
}

int dev_d2fd2_sum_f(st_ctx *c, int dir, int asym, const float *F, float *d2F, const float *E1,
                    const float *E2) {
    if (dir == 1) return fail(c, ST_E_ARG, "fused sum: x or z lines only");
    ST_TRY(check_f2(c, plain_f(F), d2F, E1) == ST_OK ? check_f2(c, plain_f(E2), nullptr, nullptr) : ST_E_ARG);
    LineArgsF a = make_args<float>(c, dir);
    a.F = plain_f(F); a.O2 = d2F; a.asym = asym; a.iadd = 0; a.E1 = E1; a.E2 = E2;
    a.fac2 = ((double)((a.geo.n - 1) * (a.geo.n - 1))) * c->s2[dir];
    a.t2 = c->trif[dir][asym ? K_D2A : K_D2S];
    return launch_line(c, OP_D2, a);
}

int dev_gauss_f(st_ctx *c, int dir, const float *F, float *Fg) {
    ST_TRY(check_f2(c, plain_f(F), Fg, nullptr));
    LineArgsF a = make_args<float>(c, dir);
    a.F = plain_f(F); a.O1 = Fg;
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
