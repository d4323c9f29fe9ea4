// st_internal.h - private declarations of the B200 solver library.
//
// Device layout: every field is an N^3 double array in the reference layout
// F(My,Mz,Mx) (y fastest); multi-variable arrays are nvar consecutive fields.
// Lines along y are contiguous, lines along z have stride My and lines along
// x have stride My*Mz.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>
#include "../../include/st_b200.h"

namespace st {

constexpr int kMaxSeg = 32;       // max segments per line (warps per CTA)
constexpr int kLanes = 16;        // lines per CTA (half a warp; a warp holds two segments)
constexpr int kLineThreads = kLanes * kMaxSeg;     // threads of a line-kernel CTA at most
constexpr int kLineCtasPerSm = 32 / kLanes;        // resident CTAs per SM at 64 registers a thread
constexpr int kScanSteps = 5;     // log2(kMaxSeg): steps of a scan over the segments

// A line of n rows is split into P = n/S segments of S rows; thread t of a CTA
// works on line t%16 and segment t/16 of 16 neighbouring lines, so a warp
// holds two adjacent segments of the same 16 lines.  Supported S.
int choose_seg(int n);

// Row tables of a constant-coefficient tridiagonal system, factorised as the
// reference's tridiagonal_serial does (src/tridiagonal.f90:264-287), plus the
// carry tables of the segmented solve.
// A: arithmetic type of the solve (double; float for the FP32 mode's kernels).
template <class A>
struct TriTabT {
    const A *l;    // forward multiplier of row i (row 0: 0)
    const A *g;    // response of the forward value of row i to the carry-in
    const A *up;   // upper diagonal c_i
    const A *id;   // 1 / (b'_i + tiny)   (last row: 1 / b'_n)
    const A *h;    // response of x_i to the carry from the right
    const A *wf;   // [P][P]: carry into segment s = sum_{s'<s} wf[s'][s] * A_{s'}
    const A *wb;   // [P][P]: carry into segment s = sum_{s'>s} wb[s'][s] * B_{s'}
    int kf, kb;    // segments back/ahead whose carry weight can change a result of type A
    const A *cyc;  // periodic family: [n][2] corner correction (see st_tables.cpp), else null
    // Away from the line ends the factorisation reaches a fixed point: in
    // segments slo <= s < shi every row's l, up, id equal (bitwise) cl, cup,
    // cid, which the solve then keeps in registers instead of loading per row.
    int slo, shi;
    A cl, cup, cid;
    // scan factors [kScanSteps][kMaxSeg]: sf[k][s] = B_s B_{s-1} ... B_{s-2^k+1}
    // (B_s: response of segment s's last forward value to its carry-in) and
    // sb[k][s] = G_s ... G_{s+2^k-1} (G_s: of its first backward value)
    const A *sf, *sb;
};
using TriTab = TriTabT<double>;

// Same for the pentadiagonal systems of the compact filter
// (pentadiagonal_serial, src/pentadiagonal.f90:319-374); carries are
// 2-vectors, propagated across the segments by a scan with 2x2 factors.
struct PenTab {
    const double *p1, *p2;   // forward multipliers of r'_{i-1}, r'_{i-2}
    const double *g1, *g2;   // forward carry responses (carry = (r'_{a-1}, r'_{a-2}))
    const double *q1, *q2;   // back-substitution coefficients of x_{i+1}, x_{i+2}
    const double *id;        // 1 / (C'_i + tiny)
    const double *h1, *h2;   // backward carry responses (carry = (x_{b+1}, x_{b+2}))
    const double *cyc;       // periodic family: [n][4] corner correction, else null
    // segments slo <= s < shi: every row's p1, p2, q1, q2, id equal (bitwise)
    // the constants below (the factorisation's interior fixed point)
    int slo, shi;
    double cp1, cp2, cq1, cq2, cid;
    // Scan factors [kScanSteps][kMaxSeg][4]: products of 2^k consecutive
    // segment transfer matrices, sf[k][s] = M_s M_{s-1} ... M_{s-2^k+1}
    // (M_s: response of segment s's last two forward values to its carry-in)
    // and sb[k][s] = N_s ... N_{s+2^k-1} (N_s: of its first two backward values)
    const double *sf, *sb;
};

enum TriKind { K_D1S = 0, K_D1A = 1, K_D2S = 2, K_D2A = 3 };
enum PenKind { K_FS = 0, K_FA = 1 };

// Scheme constants (src/header:173-204, src/LES_header:107-157).
struct Consts {
    double a1, b1, a2, b2, c2, closure1, closure2;
    double fa0, fa1, fa2, fa3, fa4;        // compact filter RHS
    double bc1[6], bc2[6], bc3[3], bc4[4]; // Visbal-Gaitonde closures
    double ga[5];                          // Gaussian coefficients (float32 values)
};

// Pointwise expression that a line kernel evaluates while loading its rows
// (so that a flux need not be stored before it is differentiated).  The
// operand order of each form matches the reference statement it replaces.
enum ProdOp {
    PR_A = 0,        // a
    PR_MUL,          // a*b
    PR_ADDMUL,       // (a+b)*c
    PR_MULMUL,       // c*(a*b)
    PR_SPEC,         // a*b*c + a*c*k0*k1             (Species_RHS flux)
    PR_SPECT,        // (k0*d)*(a*b*c + a*c*k0b*k1)    (its energy counterpart)
};
template <class T>
struct ProdT {
    int op;
    const T *a, *b, *c, *d;     // fields (double, or float in the FP32 mode)
    double k0, k1, k2;
};
using Prod = ProdT<double>;
using ProdF = ProdT<float>;

enum { G_DUX_DX, G_DUY_DX, G_DUZ_DX, G_DUX_DY, G_DUY_DY, G_DUZ_DY,
       G_DUX_DZ, G_DUY_DZ, G_DUZ_DZ, G_DTDX, G_DTDY, G_DTDZ };
enum { H_BETA, H_VISC, H_K, H_D };

struct Dims {
    int n[3];          // Mx, My, Mz
    size_t n3;         // cells of one case
};

// Device scalars of one case: a block of kScal doubles (dscal + k*kScal)
constexpr int kScal = 16;
enum { SC_STAB = 0, SC_RESV = 1, SC_DT = 6, SC_TIME = 7, SC_STEP = 8 };

}  // namespace st

struct st_ctx {
    st_params p;
    st::Dims dm;
    // Batches of same-size cases: every field holds nb consecutive blocks of
    // dm.n3 cells (field f of case k at f*fs + k*dm.n3), so one launch of a
    // line or pointwise kernel covers every case.  Cases 0 .. na-1 are
    // processed.  A single-case context has nb = na = 1 and fs = dm.n3.
    int nb = 1, na = 1;
    size_t fs = 0;     // field stride: nb * dm.n3
    size_t ncell() const { return (size_t)na * dm.n3; }   // cells the kernels process
    int seg[3];        // rows per segment along x, y, z
    int dev = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    // derived scalars
    double s1[3], s2[3];
    double DX, DY, DZ;
    double Re1_inv, Re2_inv, Pr_inv, Sc_inv;
    double Tstep = 0.0;
    double last_cfl_resv = 0.0, last_cfl_stab = 0.0;
    double mon[10] = {0};
    st::Consts k;
    // tables [dir][kind]
    st::TriTab tri[3][4];
    st::TriTabT<float> trif[3][4];   // FP32 mode: the same factors rounded to float
    st::PenTab pen[3][2];
    std::vector<void *> table_allocs;
    size_t table_bytes = 0;
    // COMMON blocks
    double *Q = nullptr, *dQ = nullptr, *QW = nullptr;
    double *Y = nullptr, *drYi = nullptr, *rYW = nullptr, *gamma_eff = nullptr;
    double *grad[12] = {nullptr};
    double *hyp[4] = {nullptr};
    double *dYd[3] = {nullptr};
    // FP32 mode (precision ST_PRECISION_FP32): the same arrays in float; the
    // double ones above stay unallocated (the state Q, QW, Y, rYW and
    // gamma_eff are double in both modes)
    float *dQf = nullptr, *drYif = nullptr;
    float *gradf[12] = {nullptr};
    float *hypf[4] = {nullptr};
    float *dYdf[3] = {nullptr};
    // scratch field pool (entries of any byte size; float and double requests
    // of the same size share entries)
    struct PoolEntry { void *p; size_t bytes; bool used; };
    std::vector<PoolEntry> pool;
    bool pool_oom = false;
    // device scalars (reductions, dt)
    double *dscal = nullptr;     // [nb][kScal]
    double *hpinned = nullptr;   // pinned host mirror [nb][kScal]
    // host<->device staging for the per-operator entry points
    std::vector<double *> stage;
    cudaStream_t own_stream = nullptr;
    // instrumentation
    long long launches = 0;
    cudaGraphExec_t step_graph = nullptr;   // captured main-loop step (st_step_async)
    long long graph_kernels = 0;            // kernels in one replay of step_graph
    std::vector<cudaGraphExec_t> batch_graphs;   // batch step per active count (index na - 1)
    std::vector<long long> batch_graph_kernels;
    bool batch_warm = false;                     // a batch step has run eagerly (scratch pool sized)
    bool prof = false;
    struct ProfRec { const char *name; double bytes; cudaEvent_t a, b; };
    std::vector<ProfRec> prec;
    std::vector<cudaEvent_t> evpool;
};

namespace st {

// error helpers
int fail(st_ctx *c, int code, const std::string &msg);
#define ST_CUDA(c, call)                                                           \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess)                                                     \
            return ::st::fail((c), ST_E_CUDA, std::string(#call) + ": " +          \
                                                  cudaGetErrorString(e_));         \
    } while (0)
#define ST_TRY(expr)                 \
    do {                             \
        int r_ = (expr);             \
        if (r_ != ST_OK) return r_;  \
    } while (0)

// launch instrumentation: every kernel launch is bracketed by these
int prof_start(st_ctx *c, const char *name, double bytes);
void prof_stop(st_ctx *c, int idx);

// tables
int build_tables(st_ctx *c);
void free_tables(st_ctx *c);
void fill_consts(Consts &k);

// scratch pool
void *scratch_bytes(st_ctx *c, size_t bytes);
inline double *scratch(st_ctx *c, int nfields = 1) {   // nfields contiguous fields (of every case)
    return (double *)scratch_bytes(c, (size_t)nfields * c->fs * sizeof(double));
}
template <class R>
inline R *scratch_t(st_ctx *c, int nfields) { return (R *)scratch_bytes(c, (size_t)nfields * c->fs * sizeof(R)); }

// The context narrowed to case k of a batch while it lives: every per-case
// device pointer (state, COMMON mirrors, scalars) points at case k's block
// and one case is processed.  Scratch fields keep their stride.
struct CaseWindow {
    st_ctx *c;
    int k, na0;
    CaseWindow(st_ctx *cc, int kk);
    ~CaseWindow();
    CaseWindow(const CaseWindow &) = delete;
    CaseWindow &operator=(const CaseWindow &) = delete;
};
void release(st_ctx *c, const void *p);
template <class R>
struct ScratchT {                                // RAII helper
    st_ctx *c; R *p;
    explicit ScratchT(st_ctx *cc, int nf = 1) : c(cc), p(scratch_t<R>(cc, nf)) {}
    ~ScratchT() { release(c, p); }
    ScratchT(const ScratchT &) = delete;
    ScratchT &operator=(const ScratchT &) = delete;
    operator R *() const { return p; }
};
using Scratch = ScratchT<double>;
inline bool fp32_mode(const st_ctx *c) { return c->p.precision == ST_PRECISION_FP32; }

// line operators on device arrays (st_kernels.cu)
int dev_dfd(st_ctx *c, int dir, int asym, const double *F, double *dF, int iadd, double cadd);
int dev_dfd_prod(st_ctx *c, int dir, int asym, const Prod &F, double *dF, int iadd, double cadd);
// two first derivatives along one direction (DFD*_sym/_asym with iadd and
// cadd each), in order, one launch when the second operand set contains the
// first
template <class T>
struct D1SpecT {
    ProdT<T> F;
    T *dF;
    int asym, iadd;
    double cadd;
};
int dev_dfd_pair(st_ctx *c, int dir, const D1SpecT<double> *ops);
int dev_dfd_pair_f(st_ctx *c, int dir, const D1SpecT<float> *ops);
// FP32-field variants (FP32 mode): same operators, float inputs and outputs
int dev_dfd_f(st_ctx *c, int dir, int asym, const float *F, float *dF, int iadd, double cadd);
int dev_dfd_prod_f(st_ctx *c, int dir, int asym, const ProdF &F, float *dF, int iadd, double cadd);
int dev_d2fd2_f(st_ctx *c, int dir, int asym, const float *F, float *dF, float *d2F, int iadd);
int dev_gauss_f(st_ctx *c, int dir, const float *F, float *Fg);
// last pass of a Laplacian: out = (derivative + E1) + E2 (x and z lines)
int dev_dfd_sum(st_ctx *c, int dir, int asym, const double *F, double *dF, const double *E1, const double *E2);
int dev_d2fd2_sum(st_ctx *c, int dir, int asym, const double *F, double *d2F, const double *E1,
                  const double *E2);
int dev_dfd_sum_f(st_ctx *c, int dir, int asym, const float *F, float *dF, const float *E1, const float *E2);
int dev_d2fd2_sum_f(st_ctx *c, int dir, int asym, const float *F, float *d2F, const float *E1,
                    const float *E2);
int dev_d2fd2(st_ctx *c, int dir, int asym, const double *F, double *dF, double *d2F, int iadd);
int dev_filter(st_ctx *c, int dir, int asym, const double *F, double *F0);
int dev_gauss(st_ctx *c, int dir, const double *F, double *Fg);
int dev_fill(st_ctx *c, double *x, size_t n, double v);
int dev_to_float(st_ctx *c, const double *x, float *y, size_t n);
int dev_to_double(st_ctx *c, const float *x, double *y, size_t n);
int dev_tridiagonal(st_ctx *c, const double *A, const double *B, const double *C, double *R,
                    int n, int lot, int nper);
int dev_pentadiagonal(st_ctx *c, const double *A, const double *B, const double *C,
                      const double *D, const double *E, double *R, int n, int lot, int nper);

// physics on device arrays (st_physics.cu)
int dev_compute_gamma(st_ctx *c, const double *Y);
int dev_rhs(st_ctx *c, double *Q, double *Qrhs, const double *Y);
int dev_compute_hyper(st_ctx *c, const double *Q, const double *Y);
int dev_hyper_rhs(st_ctx *c, const double *Q, double *Qrhs, const double *Y);
int dev_species_rhs(st_ctx *c, const double *Q, double *Qrhs, const double *Y, double *Yrhs);
int dev_bc_rhs(st_ctx *c, double *Q, double *Qrhs, const double *Y, double *Yrhs);
int dev_sponge(st_ctx *c, const double *Q, double *Qrhs, const double *Y, double *Yrhs);
int dev_fix_pressure(st_ctx *c, double *Q);
int dev_compact_filter(st_ctx *c, const double *F, double *F0, int nvar);
int dev_gaussian_filter(st_ctx *c, const double *F, double *Fg, int nvar);
int dev_compute_cfl(st_ctx *c, const double *Q, bool to_host, double *stab, double *resv);
int dev_compute_tstep(st_ctx *c, const double *Q, const double *Y, int step, bool resv_on_device,
                      double cfl_resv_host);
int dev_lddrk4(st_ctx *c, bool dt_on_device);
int dev_monitors(st_ctx *c);

// Output-side diagnostics (st_diag.cu)
int shell_count(const st_ctx *c);
int dev_compute_grad(st_ctx *c, double *Grad, double *maxdil, double *enstrophy);
int dev_compute_srm_stats(st_ctx *c, double *hmix, double *tke_total, double *ur_avg, double *y_avg);
size_t padded_nodes(const st_ctx *c);
int dev_make_padded_arrays(st_ctx *c, const double *Grad, double *W);
void padded_coords(const st_ctx *c, double *cor[3]);
int dev_shock_surface(st_ctx *c, double *rad_avg, double *rad_skew_rms);

}  // namespace st
