// fsg_noalloc.cu -- LocPrfPP (solver.f90:123-179) for callers that cannot allocate device memory.
//
// Who needs it: hosts whose device memory is owned by their own pool allocator (a framework's
// caching allocator, or a Fortran driver that reserves its arrays once at start-up) and that do
// not let a library call cudaMalloc/cudaFree per call: those calls synchronise the device and
// can fail when the pool already holds the memory.  fsg_locprf_pp allocates its work arrays on
// every call; this entry point takes every input and output as device memory the caller owns
// and keeps the kernel's per-profile work arrays (optical-depth steps, source-function
// derivative, Bezier control term: 3 * ntau doubles per profile) in the fixed array below.
//
// The array lives in every GPU that loads the library, for the life of the process.  All calls
// share it and it keeps the last call's contents; the kernel writes every element it reads
// before reading it, so nothing needs clearing.  Two calls whose kernels overlap on the GPU
// (different streams, or different host threads) race on it.
#include "fsg_internal.cuh"

#include <mutex>

#define FSG_NOALLOC_WORK_DOUBLES (1 << 20)   // 8 MiB: nprof * ntau * 3 <= 1,048,576

static __device__ __align__(256) double g_locprf_work[FSG_NOALLOC_WORK_DOUBLES];

void fsg_launch_locprf(cudaStream_t, int, int, const double *, int, const double *, const double *, const double *,
                       double *, double *);

namespace {
// device address of g_locprf_work per device, looked up once with that device current
std::mutex g_mu;
double *g_work_ptr[64];
bool g_work_ready[64];

int work_ptr(int dev, double **out) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (dev < 0 || dev >= 64) return FSG_E_ARG;
    if (!g_work_ready[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_locprf_work);
        if (e != cudaSuccess || p == nullptr) { cudaGetLastError(); return FSG_E_CUDA; }
        g_work_ptr[dev] = (double *)p;
        g_work_ready[dev] = true;
    }
    *out = g_work_ptr[dev];
    return FSG_OK;
}
}  // namespace

extern "C" int fsg_locprf_pp_noalloc(int nprof, int nmu, const double *d_xmu, int ntau, const double *d_xki,
                                     const double *d_src, const double *d_rhox, double *d_ploc, void *stream) {
    if (nprof < 0 || nmu < 1 || ntau < 3 || !d_xmu || !d_xki || !d_src || !d_rhox || !d_ploc) return FSG_E_ARG;
    if ((int64_t)nprof * ntau * 3 > FSG_NOALLOC_WORK_DOUBLES) return FSG_E_ARG;   // beyond the fixed work array
    if (nprof == 0) return FSG_OK;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return FSG_E_CUDA; }
    double *work = nullptr;
    int rc = work_ptr(dev, &work);
    if (rc != FSG_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    cudaGetLastError();                 // an earlier call's leftover error is not this launch's
    fsg_launch_locprf(s, nprof, nmu, d_xmu, ntau, d_xki, d_src, d_rhox, d_ploc, work);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return FSG_E_CUDA;
    return cudaStreamSynchronize(s) == cudaSuccess ? FSG_OK : FSG_E_CUDA;
}
