// mg_noalloc.cu — mgfvm_masserror_f64_noalloc: the mass residual without any
// device allocation by the caller or by the library.
//
// mgfvm_masserror_f64 needs a small device scratch buffer for its fixed-order
// reduction (one row of partial sums per block plus a completion counter), which the
// caller allocates.  Some callers cannot: a host program whose device memory is owned
// and pooled by another runtime (for example the reference's OpenACC data regions),
// or code on a latency-critical path that must not enter the CUDA allocator.  This
// variant keeps that scratch in the file-scope array below instead.
//
//   * The array is NOALLOC_SCRATCH_DOUBLES doubles (about 512 KiB) of static device
//     memory; every GPU that loads this library holds it until the process exits.
//   * It bounds the level size: at most NOALLOC_MAX_CELLS = 1,048,576 interior cells
//     ((npx-2)*(npy-2), e.g. a 1024 x 1024 grid); larger levels are rejected.
//   * All calls on a device share the array and it keeps the last call's contents;
//     each call clears its completion counter before launching.  Calls that overlap
//     on the GPU (different streams, or different host threads) race on the array.
//   * The first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (the host-side name of a __device__ array is not a device
//     address); make that first call on each device before any stream capture.  The
//     address is cached per device ordinal for the life of the process: after a
//     cudaDeviceReset the cached address is stale, so do not call this entry point
//     on a device after resetting it.
//   * The work runs on the caller's stream, with the scratch address of the current
//     device: a non-null stream must belong to the current device (checked, EINVAL).
//   * Nothing here calls cudaMalloc, cudaFree or an allocating library routine.
#include <mutex>

#include "mg_kernels.cuh"
#include "mgfvm_host.h"

namespace {

constexpr long long NOALLOC_MAX_CELLS = 1LL << 20;
constexpr int NOALLOC_MAX_BLOCKS = (int)((NOALLOC_MAX_CELLS + mg::BLOCK - 1) / mg::BLOCK);
constexpr size_t NOALLOC_SCRATCH_DOUBLES = (size_t)NOALLOC_MAX_BLOCKS * mg::RED_STRIDE + 32;

__device__ __align__(256) double g_noalloc_scratch[NOALLOC_SCRATCH_DOUBLES];

constexpr int MAX_DEVICES = 64;
std::mutex g_lock;
double *g_scratch_addr[MAX_DEVICES] = {nullptr};

// Device address of g_noalloc_scratch on the current device, looked up once per device.
int scratch_address(double **out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return mgfvm_fail(MGFVM_ECUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= MAX_DEVICES) return mgfvm_fail(MGFVM_EUNSUPPORTED, "device ordinal %d", dev);
    std::lock_guard<std::mutex> g(g_lock);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return mgfvm_fail(MGFVM_ECUDA, "cudaGetSymbolAddress of the reduction scratch on device %d: %s", dev,
                              cudaGetErrorString(e));
        g_scratch_addr[dev] = static_cast<double *>(p);
    }
    *out = g_scratch_addr[dev];
    return MGFVM_OK;
}

}  // namespace

extern "C" int mgfvm_masserror_f64_noalloc(const double *u, const double *v, const double *areax,
                                           const double *areay, double *su, double *pp, int npx, int npy,
                                           double *err_out, void *stream)
{
    if (!u || !v || !areax || !areay || !su || !pp || !err_out)
        return mgfvm_fail(MGFVM_EINVAL, "null device pointer");
    if (npx < 3 || npy < 3) return mgfvm_fail(MGFVM_EINVAL, "level %d x %d has no interior", npx, npy);
    const long long cells = (long long)(npx - 2) * (npy - 2);
    if (cells > NOALLOC_MAX_CELLS)
        return mgfvm_fail(MGFVM_EINVAL,
                          "mgfvm_masserror_f64_noalloc: %lld interior cells exceed its fixed scratch "
                          "limit of %lld; use mgfvm_masserror_f64 with a caller buffer",
                          cells, NOALLOC_MAX_CELLS);
    cudaStream_t s = (cudaStream_t)stream;
    if (s) {
        // the scratch address is that of the current device; a stream of another device
        // would hand its kernel a foreign address
        int cur = -1, sdev = -1;
        cudaError_t e = cudaGetDevice(&cur);
        if (e == cudaSuccess) e = cudaStreamGetDevice(s, &sdev);
        if (e != cudaSuccess) return mgfvm_fail(MGFVM_ECUDA, "stream device: %s", cudaGetErrorString(e));
        if (sdev != cur)
            return mgfvm_fail(MGFVM_EINVAL,
                              "mgfvm_masserror_f64_noalloc: the stream belongs to device %d, the current device is %d",
                              sdev, cur);
    }
    double *scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc != MGFVM_OK) return rc;
    const size_t nb = mg::raw_masserror_blocks(npx, npy);
    // the completion counter sits right after this call's partial sums; an earlier
    // call with more blocks may have left a partial sum there
    cudaError_t e = cudaMemsetAsync(scratch + nb * mg::RED_STRIDE, 0, sizeof(double), s);
    if (e == cudaSuccess) e = mg::raw_masserror(u, v, areax, areay, su, pp, npx, npy, err_out, scratch, s);
    if (e != cudaSuccess) return mgfvm_fail(MGFVM_ECUDA, "mass residual: %s", cudaGetErrorString(e));
    return MGFVM_OK;
}
