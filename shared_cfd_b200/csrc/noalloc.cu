// noalloc.cu -- scfd_rms_noalloc: the RMS of check_convergence computed without
// any device allocation, for callers that cannot call cudaMalloc.
//
// Who needs it: code that owns all device memory itself and forbids the
// libraries it links from allocating, e.g. a Fortran solver whose device
// arrays come from OpenACC / CUDA Fortran data regions, a host framework with a
// fixed memory pool, or code that enqueues work between its own allocations.
// scfd_rms needs a context, and creating one allocates the context's arena.
//
// The per-block partial sums of the reduction live in g_rms_partials below, a
// file-scope device array that every GPU which loads this library holds until
// the process exits (SCFD_NOALLOC_MAX_BLOCKS doubles = 32 KB).  In host code
// the symbol is only a host-side stand-in, so its device address is looked up
// with cudaGetSymbolAddress once per device, on the first call made while that
// device is current; that first call should therefore come before any stream
// capture.  The cached address belongs to the device's primary context: after
// cudaDeviceReset (or anything else that destroys that context) the module is
// loaded again at a new address, so do not reset a device between calls.  All
// calls share the array: calls that overlap on the GPU (from different streams
// or threads) race.  Every partial used by a call is written
// by that call before it is read, so nothing has to be cleared.
#include <cuda_runtime.h>

#include <mutex>

#include "scfd_internal.h"

namespace scfd {

static __device__ __align__(256) double g_rms_partials[SCFD_NOALLOC_MAX_BLOCKS];

namespace {

constexpr int kBlocksPerPlane = SCFD_NOALLOC_MAX_BLOCKS / SCFD_MAX_PLANES;  // 64
static_assert(SCFD_MAX_PLANES * kBlocksPerPlane <= SCFD_NOALLOC_MAX_BLOCKS,
              "the scratch must hold the partial sums of every plane");

struct RefLayout {
    int np, dimq, ix, jx;  // ix = nimax+4, jx = njmax+4
    int ni[SCFD_MAX_PLANES], nj[SCFD_MAX_PLANES];
};

// partial sums of (q(E) - qp(E))^2 over the interior cells of plane blockIdx.y,
// read from arrays in the reference layout q(1:dimq,-1:nimax+2,-1:njmax+2,Nplane)
__global__ void k_rms_ref_partial(RefLayout L, const double* __restrict__ q, const double* __restrict__ qp,
                                  double* partials) {
    __shared__ double sh[256];
    const int p = blockIdx.y;
    const int ni = L.ni[p], nj = L.nj[p];
    const int kE = L.dimq - 1;
    double acc = 0.0;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < (long long)ni * nj;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % ni) + 1, j = (int)(idx / ni) + 1;
        const long long o = (long long)L.dimq * ((i + 1) + (long long)L.ix * ((j + 1) + (long long)L.jx * p)) + kE;
        const double d = q[o] - qp[o];
        acc += d * d;
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.y * gridDim.x + blockIdx.x] = sh[0];
}

__global__ void k_rms_ref_final(const double* partials, int n, double cells, double* out) {
    double s = 0.0;
    for (int k = 0; k < n; ++k) s += partials[k];
    *out = sqrt(s) / cells;
}

std::mutex g_mu;
double* g_dev_ptr[256] = {nullptr};

// Device address of g_rms_partials on the current device (looked up once).
cudaError_t partials_ptr(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 256) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_dev_ptr[dev]) {
        double* ptr = nullptr;
        e = cudaGetSymbolAddress((void**)&ptr, g_rms_partials);
        if (e != cudaSuccess) return e;
        g_dev_ptr[dev] = ptr;
    }
    *out = g_dev_ptr[dev];
    return cudaSuccess;
}

}  // namespace
}  // namespace scfd

extern "C" int scfd_rms_noalloc(const scfd_desc* d, const double* d_q, const double* d_qp, double* d_rms,
                                void* stream) {
    using namespace scfd;
    if (!d || !d_q || !d_qp || !d_rms) return SCFD_E_ARG;
    if (d->abi_version != SCFD_ABI_VERSION || d->ny < 1 || d->ny > SCFD_MAX_SPECIES) return SCFD_E_ARG;
    // the scratch holds kBlocksPerPlane partial sums for at most SCFD_MAX_PLANES planes
    if (d->nplane < 1 || d->nplane > SCFD_MAX_PLANES) return SCFD_E_ARG;
    RefLayout L{};
    L.np = d->nplane;
    L.dimq = d->ny + 3;
    int nimax = 0, njmax = 0;
    double cells = 0.0;
    for (int p = 0; p < L.np; ++p) {
        if (d->ni[p] < 1 || d->nj[p] < 1) return SCFD_E_ARG;
        L.ni[p] = d->ni[p];
        L.nj[p] = d->nj[p];
        nimax = d->ni[p] > nimax ? d->ni[p] : nimax;
        njmax = d->nj[p] > njmax ? d->nj[p] : njmax;
        cells = cells + (double)d->ni[p] * d->nj[p];
    }
    L.ix = nimax + 4;
    L.jx = njmax + 4;
    double* partials = nullptr;
    if (partials_ptr(&partials) != cudaSuccess) return SCFD_E_CUDA;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    dim3 grid(kBlocksPerPlane, L.np);
    k_rms_ref_partial<<<grid, 256, 0, s>>>(L, d_q, d_qp, partials);
    k_rms_ref_final<<<1, 1, 0, s>>>(partials, kBlocksPerPlane * L.np, cells, d_rms);
    return cudaGetLastError() == cudaSuccess ? SCFD_OK : SCFD_E_CUDA;
}
