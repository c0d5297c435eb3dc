// k_misc.cu -- time step (store/time_step/{global,local}/set_dt.f90), the
// check_convergence RMS (store/core/check_convergence.f90:17-28), step
// bookkeeping of the device scalars, and the FP32 copy of the primitive
// field used by the mixed-precision residual.
#include <algorithm>

#include "scfd_internal.h"

namespace scfd {

__global__ void k_dt_reset(View v) {
    v.sc->dtmin_bits = 0x7FF0000000000000ull;  // +inf
}

__global__ void k_set_dt(View v) {
    const int p = v.P.act[blockIdx.y];
    const int ni = v.P.ni[p], nj = v.P.nj[p];
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    double dtc = 1e300;
    if (idx < ni * nj) {
        const int i = idx % ni + 1, j = idx / ni + 1;
        const long long N = v.ncell;
        const long long c = cidx(v.P, p, i, j);
        const long long cim = cidx(v.P, p, i - 1, j), cjm = cidx(v.P, p, i, j - 1);
        const double rho = v.w[c], u = v.w[N + c], vv = v.w[2 * N + c], pr = v.w[3 * N + c];
        const double a = sqrt(v.w[(v.D + 1) * N + c] * pr / rho);
        double uds = 0.0, un;
        un = v.vni[c] * u + v.vni[N + c] * vv;
        uds = uds + (fabs(un) + a) * v.dsi[c];
        un = v.vni[cim] * u + v.vni[N + cim] * vv;
        uds = uds + (fabs(un) + a) * v.dsi[cim];
        un = v.vnj[c] * u + v.vnj[N + c] * vv;
        uds = uds + (fabs(un) + a) * v.dsj[c];
        un = v.vnj[cjm] * u + v.vnj[N + cjm] * vv;
        uds = uds + (fabs(un) + a) * v.dsj[cjm];
        dtc = v.cfl * v.Vol[c] / fmax(uds, v.w[(v.D + 4) * N + c] / rho);
        v.dt_mat[c] = dtc;
    }
    if (v.dt_mode == SCFD_DT_GLOBAL) {
        for (int o = 16; o > 0; o >>= 1) dtc = fmin(dtc, __shfl_xor_sync(0xffffffffu, dtc, o));
        if ((threadIdx.x & 31) == 0 && dtc < 1e300)
            atomicMin(&v.sc->dtmin_bits, (unsigned long long)__double_as_longlong(dtc));
    }
}

// dt_grbl and tt (global: tt = tt + dt_grbl, set_dt.f90:40-42; fixed dt likewise)
__global__ void k_dt_final(View v) {
    if (v.dt_mode == SCFD_DT_GLOBAL) {
        v.sc->dt_grbl = __longlong_as_double((long long)v.sc->dtmin_bits);
        v.sc->tt = v.sc->tt + v.sc->dt_grbl;
    } else if (v.dt_mode == SCFD_DT_FIXED) {
        v.sc->dt_grbl = v.dt_fixed;
        v.sc->tt = v.sc->tt + v.sc->dt_grbl;
    }
}

// dt_mat of the updated planes and, for a global dt, their minimum in
// dtmin_bits (+inf when there is no cell)
int launch_set_dt_cells(const View& v, cudaStream_t s) {
    if (v.dt_mode == SCFD_DT_FIXED) return 0;
    int n = 0;
    if (v.dt_mode == SCFD_DT_GLOBAL) {
        k_dt_reset<<<1, 1, 0, s>>>(v);
        ++n;
    }
    int mx = 0;
    for (int a = 0; a < v.P.nact; ++a) {
        const int p = v.P.act[a];
        mx = v.P.ni[p] * v.P.nj[p] > mx ? v.P.ni[p] * v.P.nj[p] : mx;
    }
    if (v.P.nact == 0) return n;
    dim3 grid((mx + 255) / 256, v.P.nact);
    k_set_dt<<<grid, 256, 0, s>>>(v);
    return n + 1;
}

int launch_set_dt(const View& v, cudaStream_t s) {
    const int n = launch_set_dt_cells(v, s);
    if (v.dt_mode == SCFD_DT_LOCAL) return n;
    k_dt_final<<<1, 1, 0, s>>>(v);
    return n + 1;
}

// Deterministic two-pass RMS of q(E) - qp(E).
__global__ void k_rms_partial(View v, double* partial) {
    __shared__ double sh[256];
    const int p = v.P.act[blockIdx.y];
    const int ni = v.P.ni[p], nj = v.P.nj[p];
    double acc = 0.0;
    const long long N = v.ncell;
    const int kE = v.nY + 2;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < ni * nj; idx += gridDim.x * blockDim.x) {
        const int i = idx % ni + 1, j = idx / ni + 1;
        const long long c = cidx(v.P, p, i, j);
        const double d = v.q[kE * N + c] - v.qp[kE * N + c];
        acc += d * d;
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = sh[0];
}

__global__ void k_rms_final(const double* partial, int n, double cells, double* out) {
    double s = 0.0;
    for (int k = 0; k < n; ++k) s += partial[k];
    *out = sqrt(s) / cells;
}

int launch_rms(const View& v, cudaStream_t s, double* partial, double* out) {
    // a sharded context sums its own planes over the cell count of all planes
    const int gx = 64;
    int n = 0;
    if (v.P.nact > 0) {
        dim3 grid(gx, v.P.nact);
        k_rms_partial<<<grid, 256, 0, s>>>(v, partial);
        ++n;
    }
    double cells = 0.0;
    for (int p = 0; p < v.P.np; ++p) cells = cells + (double)v.P.ni[p] * v.P.nj[p];
    k_rms_final<<<1, 1, 0, s>>>(partial, gx * v.P.nact, cells, out);
    return n + 1;
}

// FP32 copies of w and vhi (all slots, ghosts included) for the mixed path.
__global__ void k_to_f32(const double* __restrict__ a, float* __restrict__ b, long long n) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        b[k] = (float)a[k];
}

// The slots of the updated planes only, when they are not all planes (a plane's
// slots are contiguous: base[p] .. base[p] + (nj+4)*pitch[p]).
__global__ void k_to_f32_planes(View v) {
    const int p = v.P.act[blockIdx.y];
    const long long b = v.P.base[p], n = (long long)(v.P.nj[p] + 4) * v.P.pitch[p], N = v.ncell;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        for (int m = 0; m < v.W; ++m) v.w32[m * N + b + k] = (float)v.w[m * N + b + k];
        for (int m = 0; m < v.nY; ++m) v.vhi32[m * N + b + k] = (float)v.vhi[m * N + b + k];
    }
}

int launch_to_f32(const View& v, cudaStream_t s) {
    if (v.P.nact < v.P.np) {
        if (v.P.nact == 0) return 0;
        k_to_f32_planes<<<dim3(148 * 4, v.P.nact), 256, 0, s>>>(v);
        return 1;
    }
    const long long nw = v.W * v.ncell, nv = v.nY * v.ncell;
    k_to_f32<<<1184, 256, 0, s>>>(v.w, v.w32, nw);
    k_to_f32<<<1184, 256, 0, s>>>(v.vhi, v.vhi32, nv);
    return 2;
}

}  // namespace scfd

namespace scfd {

// check_internal_loop_convergence (NR/q2d/sch_NR.raw.f90:222-237) on the device:
// status E_RESRATE when res/res1 > ResRateErr after the first step of the run;
// first_dual becomes false.
__global__ void k_step_end(View v, double warn, double err) {
    DevScalars* sc = v.sc;
    const double rr = sc->res / sc->res1;
    if (rr > warn && rr > err && !sc->first_dual) atomicMax(&sc->status, SCFD_E_RESRATE);
    sc->first_dual = 0;
}

// Field transposes between the reference layout f(1:nk,-1:nimax+2,-1:njmax+2,Nplane)
// (component fastest) and the structure-of-arrays cell slots: one thread per
// reference cell; dir 0 scatters ref -> SoA, dir 1 gathers SoA -> ref (cells
// beyond a smaller plane's ghost layers are written as zero).
__global__ void k_ref_soa(Planes P, long long N, int nk, int IX, int JX, long long nref, const double* ref,
                          double* soa, double* ref_out, int dir) {
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < nref;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % IX) - 1;
        const long long r = idx / IX;
        const int j = (int)(r % JX) - 1, p = (int)(r / JX);
        const bool in = i <= P.ni[p] + 2 && j <= P.nj[p] + 2;
        const long long c = in ? cidx(P, p, i, j) : 0;
        if (dir == 0) {
            if (in)
                for (int k = 0; k < nk; ++k) soa[k * N + c] = ref[idx * nk + k];
        } else {
            for (int k = 0; k < nk; ++k) ref_out[idx * nk + k] = in ? soa[k * N + c] : 0.0;
        }
    }
}

int launch_ref_soa(const View& v, cudaStream_t s, int nk, int IX, int JX, const double* ref, double* soa,
                   double* ref_out, int dir) {
    const long long nref = (long long)IX * JX * v.P.np;
    const int blocks = (int)std::min<long long>((nref + 255) / 256, 148LL * 16);
    k_ref_soa<<<blocks, 256, 0, s>>>(v.P, v.ncell, nk, IX, JX, nref, ref, soa, ref_out, dir);
    return 1;
}

int launch_step_end(const View& v, cudaStream_t s, double warn, double err) {
    k_step_end<<<1, 1, 0, s>>>(v, warn, err);
    return 1;
}

}  // namespace scfd
