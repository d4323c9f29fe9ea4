// st_api.cpp - C ABI (include/st_b200.h): context life cycle, COMMON-block
// mirrors, host/device argument staging and the reference-named entry points.
#include <sys/stat.h>
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <stdexcept>
#include "st_internal.h"

namespace st {

int fail(st_ctx *c, int code, const std::string &msg) {
    if (c) c->err = msg;
    return code;
}

struct OomError : std::runtime_error {
    OomError() : std::runtime_error("device scratch allocation failed") {}
};

void *scratch_bytes(st_ctx *c, size_t bytes) {
    for (auto &e : c->pool)
        if (!e.used && e.bytes == bytes) { e.used = true; return e.p; }
    void *p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        c->pool_oom = true;
        throw OomError();
    }
    c->pool.push_back({p, bytes, true});
    return p;
}

int prof_start(st_ctx *c, const char *name, double bytes) {
    c->launches++;
    if (!c->prof) return -1;
    cudaEvent_t ev[2];
    for (int q = 0; q < 2; q++) {
        if (!c->evpool.empty()) { ev[q] = c->evpool.back(); c->evpool.pop_back(); }
        else if (cudaEventCreate(&ev[q]) != cudaSuccess) { cudaGetLastError(); return -1; }
    }
    cudaEventRecord(ev[0], c->stream);
    c->prec.push_back({name, bytes, ev[0], ev[1]});
    return (int)c->prec.size() - 1;
}

void prof_stop(st_ctx *c, int idx) {
    if (idx >= 0) cudaEventRecord(c->prec[idx].b, c->stream);
}

void release(st_ctx *c, const void *p) {
    for (auto &e : c->pool)
        if (e.p == p) { e.used = false; return; }
}

// per-case device arrays of a context, offset together by CaseWindow
template <class F>
static void each_case_array(st_ctx *c, F f) {
    double **d[] = {&c->Q, &c->dQ, &c->QW, &c->Y, &c->drYi, &c->rYW, &c->gamma_eff};
    for (double **a : d) f(*a);
    for (double *&a : c->grad) f(a);
    for (double *&a : c->hyp) f(a);
    for (double *&a : c->dYd) f(a);
    float **fl[] = {&c->dQf, &c->drYif};
    for (float **a : fl) f(*a);
    for (float *&a : c->gradf) f(a);
    for (float *&a : c->hypf) f(a);
    for (float *&a : c->dYdf) f(a);
}

CaseWindow::CaseWindow(st_ctx *cc, int kk) : c(cc), k(kk), na0(cc->na) {
    const size_t off = (size_t)k * c->dm.n3;
    each_case_array(c, [&](auto *&a) { if (a) a += off; });
    c->dscal += (size_t)k * kScal;
    c->na = 1;
}
CaseWindow::~CaseWindow() {
    const size_t off = (size_t)k * c->dm.n3;
    each_case_array(c, [&](auto *&a) { if (a) a -= off; });
    c->dscal -= (size_t)k * kScal;
    c->na = na0;
}

// ---- argument staging ------------------------------------------------------
// Each array argument is either used in place (device memory of the context's
// device) or staged through a pooled device buffer (host memory).
class Args {
  public:
    explicit Args(st_ctx *c) : c_(c) {}
    ~Args() { for (auto &a : v_) if (a.staged) release(c_, a.dev); }
    // returns the device pointer to use for p (nf fields of N^3)
    double *map(const double *p, int nf, bool in, bool out) {
        for (auto &a : v_)
            if (a.host == p) { a.in |= in; a.out |= out; return a.dev; }
        Arg a{p, nullptr, nf, in, out, false};
        cudaPointerAttributes at{};
        bool dev = false;
        if (cudaPointerGetAttributes(&at, p) == cudaSuccess &&
            (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged))
            dev = at.device == c_->dev;
        cudaGetLastError();
        if (dev) {
            a.dev = const_cast<double *>(p);
        } else {
            a.dev = scratch(c_, nf);
            a.staged = true;
            if (in && cudaMemcpyAsync(a.dev, p, bytes(nf), cudaMemcpyHostToDevice, c_->stream) != cudaSuccess)
                err_ = true;
        }
        v_.push_back(a);
        return a.dev;
    }
    // late input flag: an argument that is both read and written
    int finish() {
        for (auto &a : v_)
            if (a.staged && a.out)
                if (cudaMemcpyAsync(const_cast<double *>(a.host), a.dev, bytes(a.nf), cudaMemcpyDeviceToHost,
                                    c_->stream) != cudaSuccess)
                    err_ = true;
        cudaError_t e = cudaStreamSynchronize(c_->stream);
        if (err_ || e != cudaSuccess)
            return fail(c_, ST_E_CUDA, std::string("argument transfer: ") + cudaGetErrorString(
                                                                                 e != cudaSuccess ? e : cudaErrorInvalidValue));
        return ST_OK;
    }

  private:
    struct Arg { const double *host; double *dev; int nf; bool in, out, staged; };
    size_t bytes(int nf) const { return (size_t)nf * c_->fs * sizeof(double); }
    st_ctx *c_;
    std::vector<Arg> v_;
    bool err_ = false;
};


// device memory of the context's device (used in place) or not (staged)
static bool on_device(const st_ctx *c, const void *p) {
    cudaPointerAttributes at{};
    bool dev = false;
    if (cudaPointerGetAttributes(&at, p) == cudaSuccess &&
        (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged))
        dev = at.device == c->dev;
    cudaGetLastError();
    return dev;
}

// ---- visual file: legacy VTK rectilinear grid ------------------------------
// The reference writes its visual fields with the LLNL Silo library
// (src/vis_silo_mf.f:7-277: a quad mesh with collinear coordinates "yc",
// "zc", "xc" of sizes My+1, Mz+1, Mx+1, eleven node-centred double
// variables, cycle and time options).  Silo is not available here; the same
// mesh, variables, names, centring, cycle and time go into one legacy VTK
// file (binary, big-endian), which VisIt and ParaView read: the VTK x axis is
// the reference's first mesh axis (y), then z, then x.
static const char *kVisNames[11] = {"rho", "U", "V", "W", "P", "omx", "omy", "omz", "dil", "gamma", "Y"};
static const int kVisField[11] = {3, 0, 1, 2, 4, 5, 6, 7, 8, 9, 10};   // W(..., f) of each name, 0-based

static bool put_be(FILE *f, const double *v, size_t n) {
    std::vector<uint64_t> b(std::min<size_t>(n, 1 << 20));
    for (size_t o = 0; o < n; o += b.size()) {
        const size_t m = std::min(b.size(), n - o);
        for (size_t q = 0; q < m; q++) {
            uint64_t u;
            std::memcpy(&u, v + o + q, 8);
            b[q] = __builtin_bswap64(u);
        }
        if (std::fwrite(b.data(), 8, m, f) != m) return false;
    }
    return std::fputc('\n', f) != EOF;
}

// <vis_path>/<ddd>/<prefix>.000.vtk, ddd the three digits of cue_vis (the
// directory make_dir_ creates, src/dirs.c, and the group file name of
// src/vis_silo_mf.f:97-106 for group 0)
static std::string visual_path(const char *vis_path, const char *prefix, int cue_vis, std::string *dir) {
    char d[16];
    std::snprintf(d, sizeof d, "/%d%d%d", (cue_vis / 100) % 10, (cue_vis % 100) / 10, cue_vis % 10);
    *dir = std::string(vis_path) + d;
    return *dir + "/" + prefix + ".000.vtk";
}

static int write_vtk(st_ctx *c, const std::string &path, const double *Wd, const double *cor[3], double time,
                     int step) {
    const int Mx = c->dm.n[0], My = c->dm.n[1], Mz = c->dm.n[2];
    const size_t np = padded_nodes(c);
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return fail(c, ST_E_ARG, "cannot create " + path + ": " + std::strerror(errno));
    bool ok = true;
    std::vector<double> h(np);
    ok = ok && std::fprintf(f, "# vtk DataFile Version 3.0\nshock-turbulence visual fields, time %.17g, step %d\n"
                                "BINARY\nDATASET RECTILINEAR_GRID\nFIELD FieldData 2\nTIME 1 1 double\n",
                            time, step) > 0;
    ok = ok && put_be(f, &time, 1);
    ok = ok && std::fprintf(f, "CYCLE 1 1 int\n") > 0;
    const uint32_t cyc = __builtin_bswap32((uint32_t)step);
    ok = ok && std::fwrite(&cyc, 4, 1, f) == 1 && std::fputc('\n', f) != EOF;
    ok = ok && std::fprintf(f, "DIMENSIONS %d %d %d\n", My + 1, Mz + 1, Mx + 1) > 0;
    const char *axis[3] = {"X", "Y", "Z"};
    const int order[3] = {1, 2, 0}, len[3] = {My + 1, Mz + 1, Mx + 1};
    for (int a = 0; a < 3 && ok; a++) {
        ok = std::fprintf(f, "%s_COORDINATES %d double\n", axis[a], len[a]) > 0;
        ok = ok && put_be(f, cor[order[a]], (size_t)len[a]);
    }
    ok = ok && std::fprintf(f, "POINT_DATA %zu\n", np) > 0;
    for (int v = 0; v < 11 && ok; v++) {
        if (cudaMemcpy(h.data(), Wd + (size_t)kVisField[v] * np, np * 8, cudaMemcpyDeviceToHost) != cudaSuccess) {
            std::fclose(f);
            return fail(c, ST_E_CUDA, "visual field copy");
        }
        ok = std::fprintf(f, "SCALARS %s double 1\nLOOKUP_TABLE default\n", kVisNames[v]) > 0;
        ok = ok && put_be(f, h.data(), np);
    }
    if (std::fclose(f) != 0) ok = false;
    if (!ok) return fail(c, ST_E_ARG, "write error on " + path);
    return ST_OK;
}

}  // namespace st

using namespace st;

#define API_BEGIN(c)                                                            \
    if (!(c)) return ST_E_ARG;                                                  \
    if (cudaSetDevice((c)->dev) != cudaSuccess) return fail(c, ST_E_CUDA, "cudaSetDevice"); \
    try {
#define API_END(c)                                                              \
    } catch (const OomError &) {                                                \
        return fail(c, ST_E_NOMEM, "device scratch allocation failed");        \
    } catch (const std::bad_alloc &) {                                          \
        return fail(c, ST_E_NOMEM, "host allocation failed");                  \
    }
// entry points on one grid: a batch context (st_create_batch) takes the
// st_case_* and st_batch_* calls instead
#define SINGLE_CASE(c)                                                          \
    do {                                                                        \
        if ((c) && (c)->nb > 1)                                                 \
            return fail(c, ST_E_UNSUPPORTED, "batch context: use the st_case_ and st_batch_ calls"); \
    } while (0)

extern "C" {

const char *st_status_string(int s) {
    switch (s) {
        case ST_OK: return "ok";
        case ST_E_ARG: return "bad argument";
        case ST_E_NOMEM: return "out of memory";
        case ST_E_CUDA: return "CUDA error";
        case ST_E_UNSUPPORTED: return "unsupported size or mode";
        case ST_E_NONFINITE: return "non-finite value in the state";
        case ST_E_NODEVICE: return "no usable CUDA device";
        default: return "unknown status";
    }
}

const char *st_last_error(const st_ctx *c) { return c ? c->err.c_str() : "null context"; }

void st_default_params(st_params *p, int nx, int ny, int nz) {
    std::memset(p, 0, sizeof(*p));
    p->nx = nx; p->ny = ny; p->nz = nz;
    p->x_leng = p->y_leng = p->z_leng = 2.0 * M_PI;
    p->re = 0.0;
    p->re1 = 100.0; p->re2 = 100.0; p->pr = 0.7; p->sc = 1.0;
    p->gamma1 = 1.4; p->gamma2 = 1.09; p->epsilon = 0.198265856; p->vis_exp = 0.76;
    p->bulk_ratio = 0.0; p->t_ratio = 1.0;
    p->hyper_param = 1; p->rk_mode = 0; p->cfl_cal = 0.5; p->c_beta_scale = 1.0; p->device = 0;
    p->family = ST_FAMILY_MF;
    p->precision = ST_PRECISION_FP64;
}

int st_create(const st_params *p, st_ctx **out) { return st_create_batch(p, 1, out); }

int st_create_batch(const st_params *p, int ncase, st_ctx **out) {
    if (!p || !out || ncase < 1 || ncase > 1024) return ST_E_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return ST_E_NODEVICE; }
    if (p->device < 0 || p->device >= ndev) return ST_E_ARG;
    if (p->family != ST_FAMILY_MF && p->family != ST_FAMILY_PERIODIC) return ST_E_ARG;
    if (p->rk_mode != 0 && p->rk_mode != 1) return ST_E_ARG;
    if (p->precision != ST_PRECISION_FP64 && p->precision != ST_PRECISION_FP32) return ST_E_ARG;
    const int n[3] = {p->nx, p->ny, p->nz};
    for (int d = 0; d < 3; d++)
        if (n[d] % kLanes != 0 || n[d] < kLanes || choose_seg(n[d]) == 0) return ST_E_UNSUPPORTED;
    // FP32 mode: a CTA of the line kernels owns 32 lines (two per thread)
    if (p->precision == ST_PRECISION_FP32 && (p->ny % (2 * kLanes) != 0 || (p->nx * p->nz) % (2 * kLanes) != 0))
        return ST_E_UNSUPPORTED;
    st_ctx *c = new (std::nothrow) st_ctx();
    if (!c) return ST_E_NOMEM;
    c->p = *p;
    c->dev = p->device;
    c->dm.n[0] = p->nx; c->dm.n[1] = p->ny; c->dm.n[2] = p->nz;
    c->dm.n3 = (size_t)p->nx * p->ny * p->nz;
    c->nb = c->na = ncase;
    c->fs = (size_t)ncase * c->dm.n3;
    for (int d = 0; d < 3; d++) c->seg[d] = choose_seg(n[d]);
    auto bail = [&](int code, const char *m) { c->err = m; st_destroy(c); return code; };
    if (cudaSetDevice(c->dev) != cudaSuccess) return bail(ST_E_CUDA, "cudaSetDevice");
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(ST_E_CUDA, "cudaStreamCreate");
    c->stream = c->own_stream;
    // Setup_Grid src/grid.f:15-112 (uniform grids, Uniform_X :116-128)
    const double leng[3] = {p->x_leng, p->y_leng, p->z_leng}, start[3] = {p->x_start, p->y_start, p->z_start};
    double D[3];
    for (int d = 0; d < 3; d++) {
        c->s1[d] = 1.0 / leng[d];
        c->s2[d] = c->s1[d] * c->s1[d];
        double g1 = start[d] + leng[d] * (double)(0) / (double)(n[d] - 1);
        double g2 = start[d] + leng[d] * (double)(1) / (double)(n[d] - 1);
        D[d] = g2 - g1;
    }
    c->DX = D[0]; c->DY = D[1]; c->DZ = D[2];
    // Define_Param src/define_nonperiodic_mf.f:182-204
    c->Re1_inv = p->re1 > 0.0 ? 1.0 / p->re1 : 0.0;
    c->Re2_inv = p->re2 > 0.0 ? 1.0 / p->re2 : 0.0;
    c->Pr_inv = p->pr > 0.0 ? 1.0 / p->pr : 0.0;
    c->Sc_inv = p->sc > 0.0 ? 1.0 / p->sc : 0.0;
    if (p->family == ST_FAMILY_PERIODIC) {
        // Define_Param src/define_periodic_sf.f:178-189: one fluid, Re_inv = 1/Re.
        // The shared RHS code sees Y = 1 and gamma_eff = gamma, for which the
        // mixture expressions reduce exactly to the single-fluid ones.
        c->Re1_inv = p->re > 0.0 ? 1.0 / p->re : 0.0;
        c->Re2_inv = 0.0;
    }
    fill_consts(c->k);
    if (build_tables(c) != ST_OK) return bail(ST_E_NOMEM, "tables");
    const size_t b = c->fs * sizeof(double);      // one field of every case
    auto al = [&](double **q, int nf) { return cudaMalloc((void **)q, nf * b) == cudaSuccess &&
                                              cudaMemset(*q, 0, nf * b) == cudaSuccess; };
    auto alf = [&](float **q, int nf) { return cudaMalloc((void **)q, nf * b / 2) == cudaSuccess &&
                                               cudaMemset(*q, 0, nf * b / 2) == cudaSuccess; };
    bool ok = al(&c->Q, 5) && al(&c->QW, 5) && al(&c->Y, 1) && al(&c->rYW, 1) && al(&c->gamma_eff, 1);
    if (p->precision == ST_PRECISION_FP32) {
        ok = ok && alf(&c->dQf, 5) && alf(&c->drYif, 1);
        for (int g = 0; g < 12 && ok; g++) ok = alf(&c->gradf[g], 1);
        for (int h = 0; h < 4 && ok; h++) ok = alf(&c->hypf[h], 1);
        for (int h = 0; h < 3 && ok; h++) ok = alf(&c->dYdf[h], 1);
    } else {
        ok = ok && al(&c->dQ, 5) && al(&c->drYi, 1);
        for (int g = 0; g < 12 && ok; g++) ok = al(&c->grad[g], 1);
        for (int h = 0; h < 4 && ok; h++) ok = al(&c->hyp[h], 1);
        for (int h = 0; h < 3 && ok; h++) ok = al(&c->dYd[h], 1);
    }
    const size_t sb = (size_t)ncase * kScal * sizeof(double);
    ok = ok && cudaMalloc((void **)&c->dscal, sb) == cudaSuccess && cudaMemset(c->dscal, 0, sb) == cudaSuccess &&
         cudaMallocHost((void **)&c->hpinned, sb) == cudaSuccess;
    if (!ok) { cudaGetLastError(); return bail(ST_E_NOMEM, "device allocation of the COMMON blocks failed"); }
    if (p->family == ST_FAMILY_PERIODIC) {
        if (dev_fill(c, c->gamma_eff, c->fs, p->gamma1) != ST_OK || dev_fill(c, c->Y, c->fs, 1.0) != ST_OK ||
            cudaStreamSynchronize(c->stream) != cudaSuccess)
            return bail(ST_E_CUDA, "initialising the single-fluid fields");
    }
    *out = c;
    return ST_OK;
}

int st_destroy(st_ctx *c) {
    if (!c) return ST_E_ARG;
    cudaSetDevice(c->dev);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto &r : c->prec) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    for (auto e : c->evpool) cudaEventDestroy(e);
    if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
    for (auto g : c->batch_graphs) if (g) cudaGraphExecDestroy(g);
    free_tables(c);
    double *arrs[] = {c->Q, c->dQ, c->QW, c->Y, c->drYi, c->rYW, c->gamma_eff, c->dscal};
    for (double *a : arrs) if (a) cudaFree(a);
    for (double *a : c->grad) if (a) cudaFree(a);
    for (double *a : c->hyp) if (a) cudaFree(a);
    for (double *a : c->dYd) if (a) cudaFree(a);
    float *farrs[] = {c->dQf, c->drYif};
    for (float *a : farrs) if (a) cudaFree(a);
    for (float *a : c->gradf) if (a) cudaFree(a);
    for (float *a : c->hypf) if (a) cudaFree(a);
    for (float *a : c->dYdf) if (a) cudaFree(a);
    for (auto &e : c->pool) cudaFree(e.p);
    if (c->hpinned) cudaFreeHost(c->hpinned);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
    return ST_OK;
}

int st_sync(st_ctx *c) {
    API_BEGIN(c)
    ST_CUDA(c, cudaStreamSynchronize(c->stream));
    return ST_OK;
    API_END(c)
}

// ---- state -------------------------------------------------------------------
int st_set_state(st_ctx *c, const double *Q, const double *Y) {
    SINGLE_CASE(c);
    if (!Q) return ST_E_ARG;
    if (!Y && (!c || c->p.family != ST_FAMILY_PERIODIC)) return ST_E_ARG;
    API_BEGIN(c)
    const size_t b = c->dm.n3 * 8;
    ST_CUDA(c, cudaMemcpyAsync(c->Q, Q, 5 * b, cudaMemcpyDefault, c->stream));
    // the periodic family has no species: its Y stays 1
    if (c->p.family != ST_FAMILY_PERIODIC) ST_CUDA(c, cudaMemcpyAsync(c->Y, Y, b, cudaMemcpyDefault, c->stream));
    ST_CUDA(c, cudaMemsetAsync(c->QW, 0, 5 * b, c->stream));
    if (fp32_mode(c)) {
        ST_CUDA(c, cudaMemsetAsync(c->dQf, 0, 5 * b / 2, c->stream));
        ST_CUDA(c, cudaMemsetAsync(c->drYif, 0, b / 2, c->stream));
    } else {
        ST_CUDA(c, cudaMemsetAsync(c->dQ, 0, 5 * b, c->stream));
        ST_CUDA(c, cudaMemsetAsync(c->drYi, 0, b, c->stream));
    }
    ST_CUDA(c, cudaMemsetAsync(c->rYW, 0, b, c->stream));
    ST_CUDA(c, cudaMemsetAsync(c->dscal + 7, 0, sizeof(double), c->stream));
    ST_CUDA(c, cudaStreamSynchronize(c->stream));
    return ST_OK;
    API_END(c)
}

int st_get_state(st_ctx *c, double *Q, double *Y) {
    SINGLE_CASE(c);
    API_BEGIN(c)
    const size_t b = c->dm.n3 * 8;
    if (Q) ST_CUDA(c, cudaMemcpyAsync(Q, c->Q, 5 * b, cudaMemcpyDefault, c->stream));
    if (Y) ST_CUDA(c, cudaMemcpyAsync(Y, c->Y, b, cudaMemcpyDefault, c->stream));
    ST_CUDA(c, cudaStreamSynchronize(c->stream));
    return ST_OK;
    API_END(c)
}

int st_set_tstep(st_ctx *c, double t) {
    SINGLE_CASE(c);
    API_BEGIN(c)
    c->Tstep = t;
    c->hpinned[6] = t;
    ST_CUDA(c, cudaMemcpyAsync(c->dscal + 6, c->hpinned + 6, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    ST_CUDA(c, cudaStreamSynchronize(c->stream));
    return ST_OK;
    API_END(c)
}

int st_get_tstep(st_ctx *c, double *t) {
    SINGLE_CASE(c);
    if (!t) return ST_E_ARG;
    API_BEGIN(c)
    ST_CUDA(c, cudaMemcpyAsync(c->hpinned + 6, c->dscal + 6, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    ST_CUDA(c, cudaStreamSynchronize(c->stream));
    c->Tstep = c->hpinned[6];
    *t = c->Tstep;
    return ST_OK;
    API_END(c)
}

// COMMON array by name: a double array, or (FP32 mode) a float one in *pf
static double *common_ptr(st_ctx *c, const char *name, int *nf, float **pf) {
    static const char *gn[12] = {"dux_dx", "duy_dx", "duz_dx", "dux_dy", "duy_dy", "duz_dy",
                                 "dux_dz", "duy_dz", "duz_dz", "dTdx", "dTdy", "dTdz"};
    static const char *hn[4] = {"beta_hyper", "visc_hyper", "k_hyper", "D_hyper"};
    *nf = 1;
    *pf = nullptr;
    for (int q = 0; q < 12; q++) if (!std::strcmp(name, gn[q])) { *pf = c->gradf[q]; return c->grad[q]; }
    for (int q = 0; q < 4; q++) if (!std::strcmp(name, hn[q])) { *pf = c->hypf[q]; return c->hyp[q]; }
    if (!std::strcmp(name, "gamma_eff")) return c->gamma_eff;
    if (!std::strcmp(name, "drYi")) { *pf = c->drYif; return c->drYi; }
    if (!std::strcmp(name, "rYW")) return c->rYW;
    *nf = 5;
    if (!std::strcmp(name, "dQ")) { *pf = c->dQf; return c->dQ; }
    if (!std::strcmp(name, "QW")) return c->QW;
    return nullptr;
}

int st_get_common(st_ctx *c, const char *name, double *out) {
    SINGLE_CASE(c);
    if (!name || !out) return ST_E_ARG;
    API_BEGIN(c)
    int nf;
    float *pf;
    double *p = common_ptr(c, name, &nf, &pf);
    if (!p && !pf) return fail(c, ST_E_ARG, std::string("unknown COMMON array ") + name);
    if (pf) {   // FP32 mode: widened on the device
        Scratch t(c, nf);
        ST_TRY(dev_to_double(c, pf, t, nf * c->dm.n3));
        ST_CUDA(c, cudaMemcpyAsync(out, t, nf * c->dm.n3 * 8, cudaMemcpyDefault, c->stream));
        ST_CUDA(c, cudaStreamSynchronize(c->stream));
        return ST_OK;
    }
    ST_CUDA(c, cudaMemcpyAsync(out, p, nf * c->dm.n3 * 8, cudaMemcpyDefault, c->stream));
    ST_CUDA(c, cudaStreamSynchronize(c->stream));
    return ST_OK;
    API_END(c)
}

int st_set_common(st_ctx *c, const char *name, const double *in) {
    SINGLE_CASE(c);
    if (!name || !in) return ST_E_ARG;
    API_BEGIN(c)
    int nf;
    float *pf;
    double *p = common_ptr(c, name, &nf, &pf);
    if (!p && !pf) return fail(c, ST_E_ARG, std::string("unknown COMMON array ") + name);
    if (pf) {   // FP32 mode: rounded to float on the device
        Scratch t(c, nf);
        ST_CUDA(c, cudaMemcpyAsync(t, in, nf * c->dm.n3 * 8, cudaMemcpyDefault, c->stream));
        ST_TRY(dev_to_float(c, t, pf, nf * c->dm.n3));
        ST_CUDA(c, cudaStreamSynchronize(c->stream));
        return ST_OK;
    }
    ST_CUDA(c, cudaMemcpyAsync(p, in, nf * c->dm.n3 * 8, cudaMemcpyDefault, c->stream));
    ST_CUDA(c, cudaStreamSynchronize(c->stream));
    return ST_OK;
    API_END(c)
}

// ---- line solvers --------------------------------------------------------------
int st_tridiagonal(st_ctx *c, const double *A, const double *B, const double *C, double *R, int n, int lot,
                   int nper) {
    if (!A || !B || !C || !R || n < 1 || lot < 1) return ST_E_ARG;
    API_BEGIN(c)
    const size_t N = (size_t)n * lot, bytes = N * 8;
    double *buf = nullptr;
    ST_CUDA(c, cudaMalloc((void **)&buf, 4 * bytes));
    double *dA = buf, *dB = buf + N, *dC = buf + 2 * N, *dR = buf + 3 * N;
    const double *src[4] = {A, B, C, R};
    double *dst[4] = {dA, dB, dC, dR};
    for (int q = 0; q < 4; q++) cudaMemcpyAsync(dst[q], src[q], bytes, cudaMemcpyDefault, c->stream);
    int rc = dev_tridiagonal(c, dA, dB, dC, dR, n, lot, nper);
    if (rc == ST_OK) cudaMemcpyAsync(R, dR, bytes, cudaMemcpyDefault, c->stream);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    cudaFree(buf);
    if (rc != ST_OK) return rc;
    if (e != cudaSuccess) return fail(c, ST_E_CUDA, cudaGetErrorString(e));
    return ST_OK;
    API_END(c)
}

int st_pentadiagonal(st_ctx *c, const double *A, const double *B, const double *C, const double *D,
                     const double *E, double *R, int n, int lot, int nper) {
    if (!A || !B || !C || !D || !E || !R || n < 1 || lot < 1) return ST_E_ARG;
    API_BEGIN(c)
    const size_t N = (size_t)n * lot, bytes = N * 8;
    double *buf = nullptr;
    ST_CUDA(c, cudaMalloc((void **)&buf, 6 * bytes));
    const double *src[6] = {A, B, C, D, E, R};
    for (int q = 0; q < 6; q++) cudaMemcpyAsync(buf + q * N, src[q], bytes, cudaMemcpyDefault, c->stream);
    int rc = dev_pentadiagonal(c, buf, buf + N, buf + 2 * N, buf + 3 * N, buf + 4 * N, buf + 5 * N, n, lot, nper);
    if (rc == ST_OK) cudaMemcpyAsync(R, buf + 5 * N, bytes, cudaMemcpyDefault, c->stream);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    cudaFree(buf);
    if (rc != ST_OK) return rc;
    if (e != cudaSuccess) return fail(c, ST_E_CUDA, cudaGetErrorString(e));
    return ST_OK;
    API_END(c)
}

// ---- derivatives and filters ------------------------------------------------
// asym: 0 / 1 for the _sym / _asym routines of the _mf family, PER for the
// periodic family's routines (no suffix).  Each family only has its own.
static const int PER = 2;
static int family_ok(st_ctx *c, int asym) {
    const bool per = c->p.family == ST_FAMILY_PERIODIC;
    if (per != (asym == PER))
        return fail(c, ST_E_UNSUPPORTED, per ? "the periodic family has no _sym/_asym routines"
                                             : "periodic routines need a ST_FAMILY_PERIODIC context");
    return ST_OK;
}
#define FAMILY_CHECK(c, asym) \
    do { int rc_ = family_ok(c, asym); if (rc_ != ST_OK) return rc_; } while (0)

static int do_dfd(st_ctx *c, int dir, int asym, const double *F, double *dF, int iadd, double cadd) {
    SINGLE_CASE(c);
    if (!F || !dF || (iadd != 0 && iadd != 1)) return ST_E_ARG;
    if (!c) return ST_E_ARG;
    FAMILY_CHECK(c, asym);
    if (asym == PER) asym = 0;
    API_BEGIN(c)
    Args a(c);
    double *dFd = a.map(dF, 1, iadd == 1, true);
    const double *Fd = a.map(F, 1, true, false);
    ST_TRY(dev_dfd(c, dir, asym, Fd, dFd, iadd, cadd));
    return a.finish();
    API_END(c)
}
static int do_d2(st_ctx *c, int dir, int asym, const double *F, double *dF, double *d2F, int iadd) {
    SINGLE_CASE(c);
    if (!F || !d2F || (iadd && !dF)) return ST_E_ARG;
    if (!c) return ST_E_ARG;
    FAMILY_CHECK(c, asym);
    if (asym == PER) asym = 0;
    API_BEGIN(c)
    Args a(c);
    const double *Fd = a.map(F, 1, true, false);
    double *d2 = a.map(d2F, 1, false, true);
    double *d1 = iadd ? a.map(dF, 1, false, true) : nullptr;
    ST_TRY(dev_d2fd2(c, dir, asym, Fd, d1, d2, iadd));
    return a.finish();
    API_END(c)
}
static int do_filter(st_ctx *c, int dir, int asym, const double *F, double *F0) {
    SINGLE_CASE(c);
    if (!F || !F0) return ST_E_ARG;
    if (!c) return ST_E_ARG;
    FAMILY_CHECK(c, asym);
    if (asym == PER) asym = 0;
    API_BEGIN(c)
    Args a(c);
    const double *Fd = a.map(F, 1, true, false);
    double *Od = a.map(F0, 1, false, true);
    ST_TRY(dev_filter(c, dir, asym, Fd, Od));
    return a.finish();
    API_END(c)
}
static int do_gauss(st_ctx *c, int dir, const double *F, double *Fg) {
    SINGLE_CASE(c);
    if (!F || !Fg) return ST_E_ARG;
    API_BEGIN(c)
    Args a(c);
    const double *Fd = a.map(F, 1, true, false);
    double *Od = a.map(Fg, 1, false, true);
    if (Fd == Od) {
        Scratch t(c);
        ST_TRY(dev_gauss(c, dir, Fd, t));
        ST_CUDA(c, cudaMemcpyAsync(Od, t, c->dm.n3 * 8, cudaMemcpyDeviceToDevice, c->stream));
    } else {
        ST_TRY(dev_gauss(c, dir, Fd, Od));
    }
    return a.finish();
    API_END(c)
}

int st_dfdx_sym(st_ctx *c, const double *F, double *dF, int iadd, double cadd) { return do_dfd(c, 0, 0, F, dF, iadd, cadd); }
int st_dfdy_sym(st_ctx *c, const double *F, double *dF, int iadd, double cadd) { return do_dfd(c, 1, 0, F, dF, iadd, cadd); }
int st_dfdz_sym(st_ctx *c, const double *F, double *dF, int iadd, double cadd) { return do_dfd(c, 2, 0, F, dF, iadd, cadd); }
int st_dfdx_asym(st_ctx *c, const double *F, double *dF, int iadd, double cadd) { return do_dfd(c, 0, 1, F, dF, iadd, cadd); }
int st_dfdy_asym(st_ctx *c, const double *F, double *dF, int iadd, double cadd) { return do_dfd(c, 1, 1, F, dF, iadd, cadd); }
int st_dfdz_asym(st_ctx *c, const double *F, double *dF, int iadd, double cadd) { return do_dfd(c, 2, 1, F, dF, iadd, cadd); }
int st_d2fdx2_sym(st_ctx *c, const double *F, double *dF, double *d2F, int iadd) { return do_d2(c, 0, 0, F, dF, d2F, iadd); }
int st_d2fdy2_sym(st_ctx *c, const double *F, double *dF, double *d2F, int iadd) { return do_d2(c, 1, 0, F, dF, d2F, iadd); }
int st_d2fdz2_sym(st_ctx *c, const double *F, double *dF, double *d2F, int iadd) { return do_d2(c, 2, 0, F, dF, d2F, iadd); }
int st_d2fdx2_asym(st_ctx *c, const double *F, double *dF, double *d2F, int iadd) { return do_d2(c, 0, 1, F, dF, d2F, iadd); }
int st_d2fdy2_asym(st_ctx *c, const double *F, double *dF, double *d2F, int iadd) { return do_d2(c, 1, 1, F, dF, d2F, iadd); }
int st_d2fdz2_asym(st_ctx *c, const double *F, double *dF, double *d2F, int iadd) { return do_d2(c, 2, 1, F, dF, d2F, iadd); }
int st_compact_filter_x_sym(st_ctx *c, const double *F, double *F0) { return do_filter(c, 0, 0, F, F0); }
int st_compact_filter_y_sym(st_ctx *c, const double *F, double *F0) { return do_filter(c, 1, 0, F, F0); }
int st_compact_filter_z_sym(st_ctx *c, const double *F, double *F0) { return do_filter(c, 2, 0, F, F0); }
int st_compact_filter_x_asym(st_ctx *c, const double *F, double *F0) { return do_filter(c, 0, 1, F, F0); }
int st_compact_filter_y_asym(st_ctx *c, const double *F, double *F0) { return do_filter(c, 1, 1, F, F0); }
int st_compact_filter_z_asym(st_ctx *c, const double *F, double *F0) { return do_filter(c, 2, 1, F, F0); }
int st_dfdx(st_ctx *c, const double *F, double *dF, int iadd, double cadd) { return do_dfd(c, 0, PER, F, dF, iadd, cadd); }
int st_dfdy(st_ctx *c, const double *F, double *dF, int iadd, double cadd) { return do_dfd(c, 1, PER, F, dF, iadd, cadd); }
int st_dfdz(st_ctx *c, const double *F, double *dF, int iadd, double cadd) { return do_dfd(c, 2, PER, F, dF, iadd, cadd); }
int st_d2fdx2(st_ctx *c, const double *F, double *dF, double *d2F, int iadd) { return do_d2(c, 0, PER, F, dF, d2F, iadd); }
int st_d2fdy2(st_ctx *c, const double *F, double *dF, double *d2F, int iadd) { return do_d2(c, 1, PER, F, dF, d2F, iadd); }
int st_d2fdz2(st_ctx *c, const double *F, double *dF, double *d2F, int iadd) { return do_d2(c, 2, PER, F, dF, d2F, iadd); }
int st_compact_filter_x(st_ctx *c, const double *F, double *F0) { return do_filter(c, 0, PER, F, F0); }
int st_compact_filter_y(st_ctx *c, const double *F, double *F0) { return do_filter(c, 1, PER, F, F0); }
int st_compact_filter_z(st_ctx *c, const double *F, double *F0) { return do_filter(c, 2, PER, F, F0); }
int st_gaussian_filter_x(st_ctx *c, const double *F, double *Fg) { return do_gauss(c, 0, F, Fg); }
int st_gaussian_filter_y(st_ctx *c, const double *F, double *Fg) { return do_gauss(c, 1, F, Fg); }
int st_gaussian_filter_z(st_ctx *c, const double *F, double *Fg) { return do_gauss(c, 2, F, Fg); }

int st_compact_filter(st_ctx *c, const double *F, double *F0, int nvar) {
    SINGLE_CASE(c);
    if (!F || !F0 || nvar < 1) return ST_E_ARG;
    API_BEGIN(c)
    Args a(c);
    const double *Fd = a.map(F, nvar, true, false);
    double *Od = a.map(F0, nvar, false, true);
    ST_TRY(dev_compact_filter(c, Fd, Od, nvar));
    return a.finish();
    API_END(c)
}

int st_gaussian_filter(st_ctx *c, const double *F, double *Fg, int nvar) {
    SINGLE_CASE(c);
    if (!F || !Fg || nvar < 1) return ST_E_ARG;
    API_BEGIN(c)
    Args a(c);
    const double *Fd = a.map(F, nvar, true, false);
    double *Od = a.map(Fg, nvar, false, true);
    if (Fd == Od) return fail(c, ST_E_ARG, "Gaussian_Filter output may not alias its input");
    ST_TRY(dev_gaussian_filter(c, Fd, Od, nvar));
    return a.finish();
    API_END(c)
}

// ---- physics operators ---------------------------------------------------------
// Y argument of the physics routines: required in the _mf family; the
// periodic family's routines take none (pass NULL), and its Y field is 1.
static bool y_missing(st_ctx *c, const void *Y) {
    return !Y && (!c || c->p.family != ST_FAMILY_PERIODIC);
}
static int mf_only(st_ctx *c, const char *what) {
    if (c && c->p.family == ST_FAMILY_PERIODIC)
        return fail(c, ST_E_UNSUPPORTED, std::string(what) + " has no counterpart in the periodic family");
    return ST_OK;
}
#define MF_ONLY(c, what) \
    do { int rc_ = mf_only(c, what); if (rc_ != ST_OK) return rc_; } while (0)

int st_compute_gamma(st_ctx *c, const double *Y) {
    SINGLE_CASE(c);
    if (!Y) return ST_E_ARG;
    MF_ONLY(c, "Compute_gamma");
    API_BEGIN(c)
    Args a(c);
    ST_TRY(dev_compute_gamma(c, a.map(Y, 1, true, false)));
    return a.finish();
    API_END(c)
}

int st_rhs(st_ctx *c, double *Q, double *Qrhs, const double *Y) {
    SINGLE_CASE(c);
    if (!Q || !Qrhs || y_missing(c, Y)) return ST_E_ARG;
    API_BEGIN(c)
    Args a(c);
    double *Qd = a.map(Q, 5, true, true);
    double *Rd = a.map(Qrhs, 5, false, true);
    const double *Yd = Y ? a.map(Y, 1, true, false) : c->Y;
    ST_TRY(dev_rhs(c, Qd, Rd, Yd));
    return a.finish();
    API_END(c)
}

int st_compute_hyper(st_ctx *c, const double *Q, const double *Y) {
    SINGLE_CASE(c);
    if (!Q || y_missing(c, Y)) return ST_E_ARG;
    API_BEGIN(c)
    Args a(c);
    const double *Qd = a.map(Q, 5, true, false);
    const double *Yd = Y ? a.map(Y, 1, true, false) : c->Y;
    ST_TRY(dev_compute_hyper(c, Qd, Yd));
    return a.finish();
    API_END(c)
}

int st_hyper_rhs(st_ctx *c, const double *Q, double *Qrhs, const double *Y) {
    SINGLE_CASE(c);
    if (!Q || !Qrhs || y_missing(c, Y)) return ST_E_ARG;
    API_BEGIN(c)
    Args a(c);
    const double *Qd = a.map(Q, 5, true, false);
    double *Rd = a.map(Qrhs, 5, true, true);
    const double *Yd = Y ? a.map(Y, 1, true, false) : c->Y;
    ST_TRY(dev_hyper_rhs(c, Qd, Rd, Yd));
    return a.finish();
    API_END(c)
}

int st_species_rhs(st_ctx *c, const double *Q, double *Qrhs, const double *Y, double *Yrhs) {
    SINGLE_CASE(c);
    if (!Q || !Qrhs || !Y || !Yrhs) return ST_E_ARG;
    MF_ONLY(c, "Species_RHS");
    API_BEGIN(c)
    Args a(c);
    const double *Qd = a.map(Q, 5, true, false);
    double *Rd = a.map(Qrhs, 5, true, true);
    const double *Yd = a.map(Y, 1, true, false);
    double *YRd = a.map(Yrhs, 1, true, true);
    ST_TRY(dev_species_rhs(c, Qd, Rd, Yd, YRd));
    return a.finish();
    API_END(c)
}

int st_bc_rhs(st_ctx *c, double *Q, double *Qrhs, const double *Y, double *Yrhs, double time) {
    SINGLE_CASE(c);
    (void)time;
    if (!Q || !Qrhs || !Y || !Yrhs) return ST_E_ARG;
    MF_ONLY(c, "bc_RHS");
    API_BEGIN(c)
    Args a(c);
    double *Qd = a.map(Q, 5, true, true);
    double *Rd = a.map(Qrhs, 5, true, true);
    const double *Yd = a.map(Y, 1, true, false);
    double *YRd = a.map(Yrhs, 1, true, true);
    ST_TRY(dev_bc_rhs(c, Qd, Rd, Yd, YRd));
    return a.finish();
    API_END(c)
}

int st_sponge_forcing(st_ctx *c, const double *Q, double *Qrhs, const double *Y, double *Yrhs) {
    SINGLE_CASE(c);
    if (!Q || !Qrhs || !Y || !Yrhs) return ST_E_ARG;
    MF_ONLY(c, "Sponge_Forcing");
    API_BEGIN(c)
    Args a(c);
    const double *Qd = a.map(Q, 5, true, false);
    double *Rd = a.map(Qrhs, 5, true, true);
    const double *Yd = a.map(Y, 1, true, false);
    double *YRd = a.map(Yrhs, 1, true, true);
    ST_TRY(dev_sponge(c, Qd, Rd, Yd, YRd));
    return a.finish();
    API_END(c)
}

int st_fix_pressure(st_ctx *c, double *Q, const double *Y) {
    SINGLE_CASE(c);
    (void)Y;
    if (!Q) return ST_E_ARG;
    API_BEGIN(c)
    Args a(c);
    ST_TRY(dev_fix_pressure(c, a.map(Q, 5, true, true)));
    return a.finish();
    API_END(c)
}

int st_compute_cfl(st_ctx *c, const double *Q, double *cfl_stab, double *cfl_resv) {
    SINGLE_CASE(c);
    if (!Q) return ST_E_ARG;
    API_BEGIN(c)
    Args a(c);
    const double *Qd = a.map(Q, 5, true, false);
    ST_TRY(dev_compute_cfl(c, Qd, true, cfl_stab, cfl_resv));
    return a.finish();
    API_END(c)
}

int st_compute_tstep(st_ctx *c, const double *Q, const double *Y, double cfl_resv, int step, double *tstep) {
    SINGLE_CASE(c);
    if (!Q || y_missing(c, Y)) return ST_E_ARG;
    API_BEGIN(c)
    Args a(c);
    const double *Qd = a.map(Q, 5, true, false);
    const double *Yd = Y ? a.map(Y, 1, true, false) : c->Y;
    ST_TRY(dev_compute_tstep(c, Qd, Yd, step, false, cfl_resv));
    ST_CUDA(c, cudaMemcpyAsync(c->hpinned + 6, c->dscal + 6, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    ST_TRY(a.finish());
    c->Tstep = c->hpinned[6];
    if (tstep) *tstep = c->Tstep;
    return ST_OK;
    API_END(c)
}

// ---- time integration ------------------------------------------------------------
static int read_time(st_ctx *c, double *time) {
    ST_CUDA(c, cudaMemcpyAsync(c->hpinned + 7, c->dscal + 7, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    ST_CUDA(c, cudaStreamSynchronize(c->stream));
    if (time) *time = c->hpinned[7];
    return ST_OK;
}

int st_lddrk4(st_ctx *c, double *time, int *step) {
    SINGLE_CASE(c);
    if (!time || !step) return ST_E_ARG;
    API_BEGIN(c)
    c->hpinned[7] = *time;
    ST_CUDA(c, cudaMemcpyAsync(c->dscal + 7, c->hpinned + 7, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    ST_TRY(dev_lddrk4(c, true));
    ST_TRY(dev_monitors(c));
    ST_TRY(read_time(c, time));
    *step = *step + 1;
    return ST_OK;
    API_END(c)
}

int st_step(st_ctx *c, double *time, int *step) {
    SINGLE_CASE(c);
    if (!time || !step) return ST_E_ARG;
    API_BEGIN(c)
    c->hpinned[7] = *time;
    ST_CUDA(c, cudaMemcpyAsync(c->dscal + 7, c->hpinned + 7, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    ST_TRY(dev_compute_cfl(c, c->Q, false, nullptr, nullptr));
    ST_TRY(dev_compute_tstep(c, c->Q, c->Y, *step, true, 0.0));
    ST_TRY(dev_lddrk4(c, true));
    ST_TRY(read_time(c, time));
    *step = *step + 1;
    return ST_OK;
    API_END(c)
}

// the main-loop body without host synchronisation (dt and time stay on the device)
static int enqueue_step(st_ctx *c, int step) {
    ST_TRY(dev_compute_cfl(c, c->Q, false, nullptr, nullptr));
    ST_TRY(dev_compute_tstep(c, c->Q, c->Y, step, true, 0.0));
    ST_TRY(dev_lddrk4(c, true));
    return ST_OK;
}

}  // extern "C"

// captures fn's launches on the context stream into *out (kernels counted in *nk)
template <class Fn>
static int capture_graph(st_ctx *c, cudaGraphExec_t *out, long long *nk, Fn fn) {
    cudaGraph_t g = nullptr;
    const long long l0 = c->launches;
    ST_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int rc = fn();
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    c->launches = l0;
    if (rc != ST_OK) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return fail(c, ST_E_CUDA, std::string("step capture: ") + cudaGetErrorString(e));
    size_t nn = 0;
    cudaGraphGetNodes(g, nullptr, &nn);
    std::vector<cudaGraphNode_t> nodes(nn);
    if (nn) cudaGraphGetNodes(g, nodes.data(), &nn);
    long long k = 0;
    for (auto nd : nodes) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) k++;
    }
    *nk = k;
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { *out = nullptr; return fail(c, ST_E_CUDA, cudaGetErrorString(e)); }
    return ST_OK;
}

extern "C" {

int st_step_async(st_ctx *c, int step) {
    if (step < 0) return ST_E_ARG;
    if (c && c->nb > 1) return st_batch_step_async(c);
    API_BEGIN(c)
    // Compute_Tstep's branch depends on the step number only up to step 2;
    // from then on every step is the same sequence of launches on the same
    // buffers, captured once as a CUDA graph and replayed.
    if (step < 2 || c->prof) return enqueue_step(c, step);
    if (!c->step_graph) ST_TRY(capture_graph(c, &c->step_graph, &c->graph_kernels, [&] { return enqueue_step(c, step); }));
    ST_CUDA(c, cudaGraphLaunch(c->step_graph, c->stream));
    c->launches += c->graph_kernels;
    return ST_OK;
    API_END(c)
}

// ---- batches of same-size cases ----------------------------------------------
static int case_ok(st_ctx *c, int k) {
    if (k < 0 || k >= c->nb) return fail(c, ST_E_ARG, "case index out of range");
    return ST_OK;
}

int st_batch_info(st_ctx *c, int *ncase, int *nactive) {
    if (!c) return ST_E_ARG;
    if (ncase) *ncase = c->nb;
    if (nactive) *nactive = c->na;
    return ST_OK;
}

int st_set_active(st_ctx *c, int nactive) {
    if (!c || nactive < 1 || nactive > c->nb) return ST_E_ARG;
    c->na = nactive;
    return ST_OK;
}

int st_case_start(st_ctx *c, int k, const double *Q, const double *Y, double time) {
    if (!c || !Q) return ST_E_ARG;
    if (!Y && c->p.family != ST_FAMILY_PERIODIC) return ST_E_ARG;
    API_BEGIN(c)
    ST_TRY(case_ok(c, k));
    CaseWindow w(c, k);
    const size_t b = c->dm.n3 * 8;
    for (int l = 0; l < 5; l++)
        ST_CUDA(c, cudaMemcpyAsync(c->Q + l * c->fs, Q + l * c->dm.n3, b, cudaMemcpyDefault, c->stream));
    if (c->p.family != ST_FAMILY_PERIODIC) ST_CUDA(c, cudaMemcpyAsync(c->Y, Y, b, cudaMemcpyDefault, c->stream));
    // scalars: time, step count 0 (time step and reductions are recomputed)
    c->hpinned[0] = time;
    ST_CUDA(c, cudaMemsetAsync(c->dscal, 0, kScal * sizeof(double), c->stream));
    ST_CUDA(c, cudaMemcpyAsync(c->dscal + SC_TIME, c->hpinned, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    // the set-up before the main loop, src/main_mf.f:100-101 (src/main.f:100)
    if (c->p.family != ST_FAMILY_PERIODIC) ST_TRY(dev_compute_gamma(c, c->Y));
    ST_TRY(dev_compute_hyper(c, c->Q, c->Y));
    ST_CUDA(c, cudaStreamSynchronize(c->stream));
    return ST_OK;
    API_END(c)
}

int st_case_get(st_ctx *c, int k, double *Q, double *Y, double *time, int *step) {
    if (!c) return ST_E_ARG;
    API_BEGIN(c)
    ST_TRY(case_ok(c, k));
    const size_t b = c->dm.n3 * 8, off = (size_t)k * c->dm.n3;
    if (Q)
        for (int l = 0; l < 5; l++)
            ST_CUDA(c, cudaMemcpyAsync(Q + l * c->dm.n3, c->Q + l * c->fs + off, b, cudaMemcpyDefault, c->stream));
    if (Y) ST_CUDA(c, cudaMemcpyAsync(Y, c->Y + off, b, cudaMemcpyDefault, c->stream));
    ST_CUDA(c, cudaMemcpyAsync(c->hpinned, c->dscal + (size_t)k * kScal, kScal * sizeof(double),
                               cudaMemcpyDeviceToHost, c->stream));
    ST_CUDA(c, cudaStreamSynchronize(c->stream));
    if (time) *time = c->hpinned[SC_TIME];
    if (step) *step = (int)c->hpinned[SC_STEP];
    return ST_OK;
    API_END(c)
}

int st_case_move(st_ctx *c, int src, int dst) {
    if (!c) return ST_E_ARG;
    API_BEGIN(c)
    ST_TRY(case_ok(c, src));
    ST_TRY(case_ok(c, dst));
    if (src == dst) return ST_OK;
    const size_t n3 = c->dm.n3, so = (size_t)src * n3, d = (size_t)dst * n3;
    auto mv = [&](auto *a, int nf) -> int {
        if (!a) return ST_OK;
        const size_t es = sizeof(*a);
        for (int l = 0; l < nf; l++)
            ST_CUDA(c, cudaMemcpyAsync(a + l * c->fs + d, a + l * c->fs + so, n3 * es, cudaMemcpyDeviceToDevice,
                                       c->stream));
        return ST_OK;
    };
    // the state and what the next step reads before recomputing it: gamma_eff
    // (Compute_CFL) and /HYPER/ (Compute_Tstep)
    ST_TRY(mv(c->Q, 5));
    ST_TRY(mv(c->Y, 1));
    ST_TRY(mv(c->gamma_eff, 1));
    for (int h = 0; h < 4; h++) { ST_TRY(mv(c->hyp[h], 1)); ST_TRY(mv(c->hypf[h], 1)); }
    ST_CUDA(c, cudaMemcpyAsync(c->dscal + (size_t)dst * kScal, c->dscal + (size_t)src * kScal,
                               kScal * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    ST_CUDA(c, cudaStreamSynchronize(c->stream));
    return ST_OK;
    API_END(c)
}

// one main-loop step of every active case; each case's Compute_Tstep takes
// its own step count from its scalars
static int enqueue_batch_step(st_ctx *c) {
    ST_TRY(dev_compute_cfl(c, c->Q, false, nullptr, nullptr));
    ST_TRY(dev_compute_tstep(c, c->Q, c->Y, -1, true, 0.0));
    ST_TRY(dev_lddrk4(c, true));
    return ST_OK;
}

int st_batch_step_async(st_ctx *c) {
    API_BEGIN(c)
    // the first step runs eagerly: it sizes the scratch pool, which a
    // captured graph then reuses (no allocation happens inside a capture)
    if (c->prof || !c->batch_warm) {
        ST_TRY(enqueue_batch_step(c));
        c->batch_warm = true;
        return ST_OK;
    }
    if ((int)c->batch_graphs.size() < c->nb) {
        c->batch_graphs.assign(c->nb, nullptr);
        c->batch_graph_kernels.assign(c->nb, 0);
    }
    cudaGraphExec_t &g = c->batch_graphs[c->na - 1];
    if (!g) ST_TRY(capture_graph(c, &g, &c->batch_graph_kernels[c->na - 1], [&] { return enqueue_batch_step(c); }));
    ST_CUDA(c, cudaGraphLaunch(g, c->stream));
    c->launches += c->batch_graph_kernels[c->na - 1];
    return ST_OK;
    API_END(c)
}

int st_get_time(st_ctx *c, double *time) {
    SINGLE_CASE(c);
    if (!time) return ST_E_ARG;
    API_BEGIN(c)
    return read_time(c, time);
    API_END(c)
}

int st_set_time(st_ctx *c, double time) {
    SINGLE_CASE(c);
    API_BEGIN(c)
    c->hpinned[7] = time;
    ST_CUDA(c, cudaMemcpyAsync(c->dscal + 7, c->hpinned + 7, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    ST_CUDA(c, cudaStreamSynchronize(c->stream));
    return ST_OK;
    API_END(c)
}

int st_memory(st_ctx *c, long long *bytes) {
    if (!c || !bytes) return ST_E_ARG;
    const size_t fb = c->fs * sizeof(double);
    // COMMON mirrors (13 double state fields; 25 intermediate fields, float in
    // the FP32 mode), tables, scalars and the scratch pool
    const size_t ib = fp32_mode(c) ? fb / 2 : fb;
    size_t b = 13 * fb + 25 * ib + c->table_bytes + (size_t)c->nb * kScal * sizeof(double);
    for (auto &e : c->pool) b += e.bytes;
    *bytes = (long long)b;
    return ST_OK;
}

int st_query(st_ctx *c) {
    if (!c) return ST_E_ARG;
    if (cudaSetDevice(c->dev) != cudaSuccess) return fail(c, ST_E_CUDA, "cudaSetDevice");
    cudaError_t e = cudaStreamQuery(c->stream);
    if (e == cudaSuccess) return 1;
    if (e == cudaErrorNotReady) { cudaGetLastError(); return 0; }
    return fail(c, ST_E_CUDA, cudaGetErrorString(e));
}

int st_set_stream(st_ctx *c, void *stream) {
    API_BEGIN(c)
    ST_CUDA(c, cudaStreamSynchronize(c->stream));
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    return ST_OK;
    API_END(c)
}

int st_get_stream(st_ctx *c, void **stream) {
    if (!c || !stream) return ST_E_ARG;
    *stream = (void *)c->stream;
    return ST_OK;
}

int st_profile(st_ctx *c, int enable) {
    if (!c) return ST_E_ARG;
    c->prof = enable != 0;
    return ST_OK;
}

int st_launch_count(st_ctx *c, long long *count) {
    if (!c || !count) return ST_E_ARG;
    *count = c->launches;
    return ST_OK;
}

int st_profile_report(st_ctx *c, char *buf, int buflen) {
    if (!buf || buflen < 3) return ST_E_ARG;
    API_BEGIN(c)
    ST_CUDA(c, cudaStreamSynchronize(c->stream));
    struct Agg { long long n = 0; double ms = 0, bytes = 0; };
    std::vector<std::pair<std::string, Agg>> agg;
    for (auto &r : c->prec) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, r.a, r.b);
        size_t k = 0;
        while (k < agg.size() && agg[k].first != r.name) k++;
        if (k == agg.size()) agg.push_back({r.name, Agg()});
        agg[k].second.n++; agg[k].second.ms += ms; agg[k].second.bytes += r.bytes;
        c->evpool.push_back(r.a); c->evpool.push_back(r.b);
    }
    c->prec.clear();
    cudaGetLastError();
    std::string s = "{";
    char tmp[256];
    for (size_t k = 0; k < agg.size(); k++) {
        std::snprintf(tmp, sizeof(tmp), "%s\"%s\": {\"launches\": %lld, \"ms\": %.6f, \"bytes\": %.1f}",
                      k ? ", " : "", agg[k].first.c_str(), agg[k].second.n, agg[k].second.ms, agg[k].second.bytes);
        s += tmp;
    }
    s += "}";
    if ((int)s.size() + 1 > buflen) return fail(c, ST_E_ARG, "report buffer too small");
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return ST_OK;
    API_END(c)
}

// ---- Output-side diagnostics -------------------------------------------------
int st_compute_grad(st_ctx *c, double *Grad, double *maxdil, double *enstrophy) {
    SINGLE_CASE(c);
    if (!maxdil || !enstrophy) return ST_E_ARG;
    MF_ONLY(c, "Compute_Grad");
    API_BEGIN(c)
    Args a(c);
    double *Gd = Grad ? a.map(Grad, 4, false, true) : nullptr;
    ST_TRY(dev_compute_grad(c, Gd, maxdil, enstrophy));
    return a.finish();
    API_END(c)
}

int st_shell_count(st_ctx *c, int *n_avg) {
    if (!c || !n_avg) return ST_E_ARG;
    *n_avg = shell_count(c);
    return ST_OK;
}

int st_compute_srm_stats(st_ctx *c, double *hmix, double *tke_total, double *ur_avg, double *y_avg) {
    SINGLE_CASE(c);
    if (!hmix || !tke_total) return ST_E_ARG;
    MF_ONLY(c, "Compute_SRM_Stats");
    API_BEGIN(c)
    ST_TRY(dev_compute_srm_stats(c, hmix, tke_total, ur_avg, y_avg));
    return ST_OK;
    API_END(c)
}

int st_generate_shock_surface(st_ctx *c, double *rad_avg, double *rad_skew_rms) {
    SINGLE_CASE(c);
    if (!rad_avg || !rad_skew_rms) return ST_E_ARG;
    MF_ONLY(c, "Generate_Shock_Surface");
    API_BEGIN(c)
    ST_TRY(dev_shock_surface(c, rad_avg, rad_skew_rms));
    return ST_OK;
    API_END(c)
}

int st_make_padded_arrays(st_ctx *c, const double *Grad, double *W, double *xx, double *yy, double *zz) {
    SINGLE_CASE(c);
    if (!W) return ST_E_ARG;
    MF_ONLY(c, "MakePaddedArrays");
    API_BEGIN(c)
    Args a(c);
    const double *Gd = Grad ? a.map(Grad, 4, true, false) : nullptr;
    const size_t np = padded_nodes(c), wbytes = 11 * np * sizeof(double);
    const bool wdev = on_device(c, W);
    // staged: whole scratch fields covering the 11 padded fields
    Scratch ws(c, wdev ? 1 : (int)((11 * np + c->fs - 1) / c->fs));
    double *Wd = wdev ? W : (double *)ws;
    ST_TRY(dev_make_padded_arrays(c, Gd, Wd));
    if (!wdev) ST_CUDA(c, cudaMemcpyAsync(W, Wd, wbytes, cudaMemcpyDeviceToHost, c->stream));
    ST_TRY(a.finish());
    double *out[3] = {xx, yy, zz};
    std::vector<double> cor[3];
    double *cp[3];
    for (int d = 0; d < 3; d++) { cor[d].resize(c->dm.n[d] + 1); cp[d] = cor[d].data(); }
    padded_coords(c, cp);
    for (int d = 0; d < 3; d++)
        if (out[d]) ST_CUDA(c, cudaMemcpy(out[d], cp[d], cor[d].size() * sizeof(double), cudaMemcpyDefault));
    return ST_OK;
    API_END(c)
}

int st_write_visual(st_ctx *c, const double *Grad, const char *vis_path, const char *prefix, int cue_vis,
                    double time, int step) {
    SINGLE_CASE(c);
    if (!vis_path || !prefix || cue_vis < 0 || cue_vis > 999) return ST_E_ARG;
    MF_ONLY(c, "Write_Visual_Silo");
    API_BEGIN(c)
    Args a(c);
    const double *Gd = Grad ? a.map(Grad, 4, true, false) : nullptr;
    const size_t np = padded_nodes(c);
    Scratch ws(c, (int)((11 * np + c->fs - 1) / c->fs));
    ST_TRY(dev_make_padded_arrays(c, Gd, ws));
    ST_TRY(a.finish());
    std::vector<double> cor[3];
    double *cp[3];
    for (int d = 0; d < 3; d++) { cor[d].resize(c->dm.n[d] + 1); cp[d] = cor[d].data(); }
    padded_coords(c, cp);
    std::string dir;
    const std::string path = visual_path(vis_path, prefix, cue_vis, &dir);
    if (mkdir(dir.c_str(), S_IRWXU | S_IRWXG) != 0 && errno != EEXIST)
        return fail(c, ST_E_ARG, "cannot create directory " + dir + ": " + std::strerror(errno));
    const double *ccp[3] = {cp[0], cp[1], cp[2]};
    return write_vtk(c, path, ws, ccp, time, step);
    API_END(c)
}

int st_get_monitors(st_ctx *c, double out[10]) {
    SINGLE_CASE(c);
    if (!out) return ST_E_ARG;
    API_BEGIN(c)
    ST_TRY(dev_monitors(c));
    ST_CUDA(c, cudaMemcpyAsync(c->hpinned, c->dscal, 8 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    ST_CUDA(c, cudaStreamSynchronize(c->stream));
    std::memcpy(out, c->mon, 8 * sizeof(double));
    out[8] = c->hpinned[1];
    out[9] = c->hpinned[6];
    return ST_OK;
    API_END(c)
}

}  // extern "C"
