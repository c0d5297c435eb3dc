// k_shard.cu -- device side of the block-sharded step (scfd_dstep): packing
// the cells this rank's planes lend to other ranks' ghost copies, scattering
// the cells received, and the local halves of the cross-rank reductions that
// replace the MPI_Allreduce of dt_grbl (store/time_step/global/set_dt.f90:40)
// and the MPI_Reduce of omega and the inner residual
// (store/time_scheme/NR/q2d/time_NR_viscous.f90:87-90).
//
// Reduction slots hold doubles; a status travels as -status so that the MIN
// of the slot over the ranks is the largest (worst) status.
#include "scfd_internal.h"

namespace scfd {

// out[k*n + t] = (w | vhi)(component k, cells[t]): component-major, so the
// reads of one component are gathers and the writes are coalesced.
__global__ void k_halo_pack(View v, const long long* __restrict__ cells, int n, double* __restrict__ out) {
    const long long N = v.ncell;
    const int K = v.W + v.nY;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < (long long)n * K;
         idx += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(idx / n);
        const long long t = idx - (long long)k * n;
        const long long c = cells[t];
        out[idx] = k < v.W ? v.w[k * N + c] : v.vhi[(k - v.W) * N + c];
    }
}

__global__ void k_halo_unpack(View v, const HaloImport* __restrict__ imp, int n, const double* __restrict__ buf) {
    const long long N = v.ncell;
    const int K = v.W + v.nY;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < (long long)n * K;
         idx += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(idx / n);
        const HaloImport e = imp[idx - (long long)k * n];
        const double x = buf[e.off + k * e.n];
        if (k < v.W)
            v.w[k * N + e.slot] = x;
        else
            v.vhi[(k - v.W) * N + e.slot] = x;
    }
}

__device__ __forceinline__ void take_status(DevScalars* sc, double neg) {
    const int st = (int)(-neg);
    if (st > 0) atomicMax(&sc->status, st);
}

__global__ void k_dt_export(View v, double* red) {
    red[0] = v.dt_mode == SCFD_DT_GLOBAL ? __longlong_as_double((long long)v.sc->dtmin_bits) : 0.0;
    red[1] = -(double)v.sc->status;
}

// dt_grbl and the time from the global minimum (set_dt.f90:40-42)
__global__ void k_dt_import(View v, const double* red) {
    DevScalars* sc = v.sc;
    if (v.dt_mode == SCFD_DT_GLOBAL) {
        sc->dt_grbl = red[0];
        sc->tt = sc->tt + sc->dt_grbl;
    } else if (v.dt_mode == SCFD_DT_FIXED) {
        sc->dt_grbl = v.dt_fixed;
        sc->tt = sc->tt + sc->dt_grbl;
    }
    take_status(sc, red[1]);
}

// the per-strip partials of the backward sweep, reduced in strip order
__global__ void k_res_export(View v, const double* partials, int nstrips, double* red) {
    double res, om;
    reduce_partials(partials, nstrips, res, om);
    if (threadIdx.x == 0) {
        red[0] = res;
        red[1] = om;
        red[2] = -(double)v.sc->status;
    }
}

// The global omega candidate decides the omega test on every rank alike
// (time_NR_viscous.f90:75-78) and gives the step's residual and omega, also on
// a rank without planes; the update kernels then read red[0..1] as the
// partials of a single strip.
__global__ void k_res_import(View v, const double* red, int inner) {
    DevScalars* sc = v.sc;
    take_status(sc, red[2]);
    if (red[1] < v.omega_min) atomicMax(&sc->status, SCFD_E_OMEGA);
    if (inner == 1) sc->res1 = red[0];
    sc->res = red[0];
    sc->omega = fmin(v.omega_max, red[1]);
    log_inner(sc, inner, red[1], red[0]);
}

__global__ void k_status_export(View v, double* red) { red[0] = -(double)v.sc->status; }

__global__ void k_status_import(View v, const double* red) { take_status(v.sc, red[0]); }

static int grid_for(long long work) {
    long long b = (work + 255) / 256;
    if (b > 148 * 8) b = 148 * 8;
    return b < 1 ? 1 : (int)b;
}

int launch_halo_pack(const View& v, cudaStream_t s, const long long* cells, int n, double* out) {
    if (n <= 0) return 0;
    k_halo_pack<<<grid_for((long long)n * (v.W + v.nY)), 256, 0, s>>>(v, cells, n, out);
    return 1;
}

int launch_halo_unpack(const View& v, cudaStream_t s, const HaloImport* imp, int n, const double* buf) {
    if (n <= 0) return 0;
    k_halo_unpack<<<grid_for((long long)n * (v.W + v.nY)), 256, 0, s>>>(v, imp, n, buf);
    return 1;
}

int launch_dt_export(const View& v, cudaStream_t s, double* red) {
    k_dt_export<<<1, 1, 0, s>>>(v, red);
    return 1;
}

int launch_dt_import(const View& v, cudaStream_t s, const double* red) {
    k_dt_import<<<1, 1, 0, s>>>(v, red);
    return 1;
}

int launch_res_export(const View& v, cudaStream_t s, const double* partials, int nstrips, double* red) {
    k_res_export<<<1, 1024, 0, s>>>(v, partials, nstrips, red);
    return 1;
}

int launch_res_import(const View& v, cudaStream_t s, const double* red, int inner) {
    k_res_import<<<1, 1, 0, s>>>(v, red, inner);
    return 1;
}

int launch_status_export(const View& v, cudaStream_t s, double* red) {
    k_status_export<<<1, 1, 0, s>>>(v, red);
    return 1;
}

int launch_status_import(const View& v, cudaStream_t s, const double* red) {
    k_status_import<<<1, 1, 0, s>>>(v, red);
    return 1;
}

}  // namespace scfd
