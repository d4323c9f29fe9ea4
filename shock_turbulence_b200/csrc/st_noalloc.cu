// st_noalloc.cu - st_tridiagonal_noalloc: the general tridiagonal solve of
// st_tridiagonal, for callers that must not allocate device memory.
//
// st_tridiagonal needs two working copies of A and B (the reference's
// tridiagonal_serial overwrites its coefficients, src/tridiagonal.f90:274-284).
// It gets them from cudaMalloc/cudaMallocAsync, and it stages host arrays
// through more device buffers.  Some callers cannot allow that: a host program
// that owns all device memory through its own pool and must not see a second
// allocator touch the device, and code on a latency budget where an allocation
// can block on the driver and stall the device's other work.  This entry point takes the working copies
// from a fixed array in the library's static device memory instead.
//
// Limits and rules:
//  - n * lot must not exceed kNoAllocMaxElems (262144, i.e. 2 x 2 MiB of
//    scratch per device); larger systems are rejected with ST_E_ARG.
//  - A, B, C and R must be device memory of the context's device; host arrays
//    are rejected (staging them would allocate).
//  - The first call on each device looks up the scratch array's address with
//    cudaGetSymbolAddress; the driver may load the library's device code at
//    that moment.  Make that first call before any stream capture begins.
//  - Nothing in the scratch has to start at zero: each call copies A and B
//    into it in full before the solve reads it.
//  - The scratch is one array per device, shared by every context on that
//    device.  Calls whose GPU work overlaps (different streams, threads or
//    contexts on one device) race on it.  Calls on one stream are ordered and
//    safe; the call returns once R is written (it synchronises its stream).
#include <mutex>
#include <new>
#include "st_internal.h"

namespace st {

// defined in st_kernels.cu: tridiagonal_serial / tridiagonal_periodic_serial,
// thread per line, arrays (lot,n) with lot fastest; a and b are overwritten.
__global__ void k_tri_general(double *a, double *b, const double *cc, double *R, int n, int lot,
                              int nper);

namespace {

constexpr size_t kNoAllocMaxElems = size_t(1) << 18;
constexpr int kMaxDevices = 64;

// working copies of A and B: a call with N = n*lot elements puts A's copy in
// the first N entries and B's copy right after it, in entries N .. 2N-1
__device__ __align__(256) double g_tri_scratch[2 * kNoAllocMaxElems];

std::mutex g_setup_mu;
double *g_scratch_ptr[kMaxDevices] = {};

// With `dev` current: returns the scratch address on that device, looking it
// up on the first call for the device.
int scratch_on(st_ctx *c, int dev, double **out) {
    if (dev < 0 || dev >= kMaxDevices)
        return fail(c, ST_E_UNSUPPORTED, "st_tridiagonal_noalloc: device ordinal above 63");
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
        double *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void **)&p, g_tri_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return fail(c, ST_E_CUDA, std::string("st_tridiagonal_noalloc: cudaGetSymbolAddress: ") +
                                          cudaGetErrorString(e));
        }
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return ST_OK;
}

bool on_device(const void *p, int dev) {
    cudaPointerAttributes at{};
    bool ok = cudaPointerGetAttributes(&at, p) == cudaSuccess &&
              (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) && at.device == dev;
    cudaGetLastError();
    return ok;
}

}  // namespace
}  // namespace st

using namespace st;

// The body runs inside a try block: a std::bad_alloc from building an error
// message must not cross the C boundary into a Fortran or C caller.
static int tridiagonal_noalloc(st_ctx *c, const double *A, const double *B, const double *C, double *R,
                               int n, int lot, int nper) {
    if (!A || !B || !C || !R || n < 1 || lot < 1) return fail(c, ST_E_ARG, "st_tridiagonal_noalloc: bad argument");
    const size_t N = (size_t)n * lot;
    if (N > kNoAllocMaxElems)
        return fail(c, ST_E_ARG, "st_tridiagonal_noalloc: n*lot = " + std::to_string(N) +
                                     " exceeds the limit of " + std::to_string(kNoAllocMaxElems));
    if (cudaSetDevice(c->dev) != cudaSuccess) {
        cudaGetLastError();
        return fail(c, ST_E_CUDA, "cudaSetDevice");
    }
    if (!on_device(A, c->dev) || !on_device(B, c->dev) || !on_device(C, c->dev) || !on_device(R, c->dev))
        return fail(c, ST_E_ARG, "st_tridiagonal_noalloc: A, B, C and R must be device arrays of the context's device");
    double *a = nullptr;
    int rc = scratch_on(c, c->dev, &a);
    if (rc != ST_OK) return rc;
    double *b = a + N;
    ST_CUDA(c, cudaMemcpyAsync(a, A, N * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    ST_CUDA(c, cudaMemcpyAsync(b, B, N * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    c->launches++;
    k_tri_general<<<(lot + 127) / 128, 128, 0, c->stream>>>(a, b, C, R, n, lot, nper);
    ST_CUDA(c, cudaGetLastError());
    ST_CUDA(c, cudaStreamSynchronize(c->stream));
    return ST_OK;
}

extern "C" int st_tridiagonal_noalloc(st_ctx *c, const double *A, const double *B, const double *C,
                                      double *R, int n, int lot, int nper) {
    if (!c) return ST_E_ARG;
    try {
        return tridiagonal_noalloc(c, A, B, C, R, n, lot, nper);
    } catch (const std::bad_alloc &) {
        return fail(c, ST_E_NOMEM, "host allocation failed");
    }
}
