// k_chem.cu -- point-implicit chemistry per cell: proceed_reaction ->
// reaction_chemeq2 -> chemeq2 (store/therm_lib/chemkin/flow/reactive/thermal_model.f90:45-73,
// store/therm_lib/chemkin/core/sub_chem.f90:1684-1819) with the UV source terms
// Fex_var (store/therm_lib/chemkin/uvhp/uv/FJ.f90:301-453).
//
// Work distribution.  Cells need very different numbers of CHEMEQ2 attempts, so
// the kernel is persistent: each thread pulls cells from a device counter and,
// in one loop, advances whichever cell it holds by one attempt, fetching a new
// cell when the current one reaches the end of the interval.  All lanes of a
// warp therefore stay on the same two Fex_var evaluations per iteration instead
// of idling behind the slowest cell of a fixed assignment.
//
// DVODE.  Where the reference hands the rest of an interval to DVODE after 10
// attempts (sub_chem.f90:1755-1775), k_chem queues the cell with the time and
// state reached, and k_chem_dvode, launched behind it, finishes the queued
// cells with the one-warp DVODE of chem_warp.cuh (a warp per cell, taken from
// the queue by a counter).  Such cells are rare and need hundreds of source
// evaluations each, so they leave the per-thread loop, whose registers and
// local memory stay sized for CHEMEQ2 alone.
#include "chem_warp.cuh"
#include "scfd_internal.h"

namespace scfd {

__device__ __forceinline__ long long cell_of(const View& v, long long k, int& pl) {
    // k enumerates the interior cells of the updated planes, plane by plane
    for (int a = 0; a < v.P.nact; ++a) {
        const int p = v.P.act[a];
        const long long n = (long long)v.P.ni[p] * v.P.nj[p];
        if (k < n) {
            pl = p;
            const int i = (int)(k % v.P.ni[p]) + 1, j = (int)(k / v.P.ni[p]) + 1;
            return cidx(v.P, p, i, j);
        }
        k -= n;
    }
    pl = -1;
    return -1;
}

__device__ bool ceq_load(const View& v, long long c, Ceq& s) {
    const long long N = v.ncell;
    const int ns = v.chem.ns, D = v.D;
    const double T = v.w[3 * N + c] / v.w[c] / v.w[(D + 3) * N + c];
    for (int k = 0; k < ns; ++k) {
        double n = v.q[k * N + c] * v.chem.inv_mw[k] * 1e-3;
        s.y[k] = fmax(n, 1e-40);
    }
    s.y[ns] = T;
    for (int k = 0; k <= ns; ++k) s.y0[k] = s.y[k];
    s.tt = 0.0;
    s.tout = v.sc->dt_grbl;
    s.dt = s.tout - s.tt;
    s.countersum = 0;
    s.substeps = 0;
    s.counter = 0.0;
    s.fell_back = false;
    s.evals = 0;
    return true;
}

__device__ void ceq_store(const View& v, long long c, const Ceq& s) {
    const long long N = v.ncell;
    const int ns = v.chem.ns;
    for (int k = 0; k < ns; ++k) {
        const double n = fmax(s.y[k], 1e-40);
        v.q[k * N + c] = n * v.chem.mws[k] * 1e3;
    }
}

__global__ void __launch_bounds__(128) k_chem(View v, long long ncells, unsigned long long* counter, int max_substeps,
                                              ChemQueue dq) {
    Ceq s;
    long long c = -1;
    long long attempts = 0, fallback = 0;
    int pl;
    // first cell
    long long k = (long long)atomicAdd(counter, 1ull);
    if (k < ncells) {
        c = cell_of(v, k, pl);
        ceq_load(v, c, s);
    }
    while (c >= 0) {
        const int r = ceq_attempt(v.chem, s, v.chem.rtol, max_substeps, attempts);
        if (r != 0) {
            if (r == 2) {
                // to DVODE from (tt, y0); k_chem_dvode stores the cell
                const unsigned long long e = atomicAdd(&dq.count[0], 1ull);
                if (e < (unsigned long long)dq.capacity) {
                    const int N = v.chem.ns + 1;
                    dq.cell[e] = c;
                    dq.tt[e] = s.tt;
                    for (int i = 0; i < N; ++i) dq.y[e * N + i] = s.y0[i];
                } else {
                    atomicMax(&v.sc->status, SCFD_E_CHEM);
                    ceq_store(v, c, s);
                }
                ++fallback;
            } else {
                if (r < 0) atomicMax(&v.sc->status, -r);
                ceq_store(v, c, s);
            }
            k = (long long)atomicAdd(counter, 1ull);
            if (k < ncells) {
                c = cell_of(v, k, pl);
                ceq_load(v, c, s);
            } else {
                c = -1;
            }
        }
    }
    // warp-aggregate the counters
    for (int o = 16; o > 0; o >>= 1) {
        attempts += __shfl_xor_sync(0xffffffffu, attempts, o);
        fallback += __shfl_xor_sync(0xffffffffu, fallback, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd((unsigned long long*)&v.sc->chem_attempts, (unsigned long long)attempts);
        atomicAdd((unsigned long long*)&v.sc->chem_fallback, (unsigned long long)fallback);
        atomicAdd((unsigned long long*)&v.sc->chem_attempts_last, (unsigned long long)attempts);
        atomicAdd((unsigned long long*)&v.sc->chem_fallback_last, (unsigned long long)fallback);
    }
}

// The queued cells, one warp each: DVODE from (tt, y) to dt_grbl, then the
// species back into q as ceq_store does.
__global__ void k_chem_dvode(View v, ChemQueue dq) {
    extern __shared__ __align__(16) double wsm[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const DevChem& ch = v.chem;
    const int ns = ch.ns, N = ns + 1;
    WarpMem w(wsm + (long long)wid * dq.warp_doubles, N, ns, ch.nr);
    unsigned long long queued = *reinterpret_cast<volatile unsigned long long*>(&dq.count[0]);
    if (queued > (unsigned long long)dq.capacity) queued = (unsigned long long)dq.capacity;
    const double tout = v.sc->dt_grbl;
    auto none = [](double) {};
    for (;;) {
        unsigned long long e = 0;
        if (lane == 0) e = atomicAdd(&dq.count[1], 1ull);
        e = __shfl_sync(0xffffffffu, e, 0);
        if (e >= queued) break;
        for (int i = lane; i < N; i += 32) w.y[i] = dq.y[e * N + i];
        __syncwarp();
        long long evals = 0;
        const int rc = warp_dvode_rest(ch, w, w.y, dq.tt[e], tout, evals, lane, none);
        if (rc != 0 && lane == 0) atomicMax(&v.sc->status, rc);
        const long long c = dq.cell[e];
        const long long NC = v.ncell;
        for (int k = lane; k < ns; k += 32) v.q[k * NC + c] = fmax(w.y[k], 1e-40) * ch.mws[k] * 1e3;
        __syncwarp();
    }
}

size_t chem_dvode_warp_doubles(int ns, int nr) { return (size_t)((warp_mem_doubles(ns, nr) + 1) & ~1); }

int chem_dvode_setup(int ns, int nr, int* warps_per_block) {
    int dev = 0, smem_max = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const int wbytes = (int)(chem_dvode_warp_doubles(ns, nr) * sizeof(double));
    const int wpb = smem_max / wbytes < 4 ? smem_max / wbytes : 4;
    if (wpb < 1) return (int)cudaErrorInvalidValue;
    *warps_per_block = wpb;
    if (wpb * wbytes > 48 * 1024)
        return (int)cudaFuncSetAttribute(k_chem_dvode, cudaFuncAttributeMaxDynamicSharedMemorySize, wpb * wbytes);
    return 0;
}

int launch_chem_impl(const View& v, cudaStream_t s, int max_substeps, unsigned long long* counter, int nsm,
                     const ChemQueue& dq) {
    long long n = 0;
    for (int a = 0; a < v.P.nact; ++a) n += (long long)v.P.ni[v.P.act[a]] * v.P.nj[v.P.act[a]];
    if (n == 0) return 0;
    cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s);
    cudaMemsetAsync(dq.count, 0, 2 * sizeof(unsigned long long), s);
    cudaMemsetAsync(&v.sc->chem_attempts_last, 0, 2 * sizeof(long long), s);
    // persistent grid: a few CTAs per SM, capped by the work
    long long blocks = (long long)nsm * 8;
    const long long need = (n + 127) / 128;
    if (blocks > need) blocks = need;
    if (blocks < 1) blocks = 1;
    k_chem<<<(unsigned)blocks, 128, 0, s>>>(v, n, counter, max_substeps > 0 ? max_substeps : 1000000, dq);
    // the DVODE pass: a persistent grid of warps; none has work unless k_chem queued cells
    const int wpb = dq.warps_per_block;
    k_chem_dvode<<<(unsigned)(nsm * 2), 32 * wpb, (size_t)wpb * dq.warp_doubles * sizeof(double), s>>>(v, dq);
    return 2;
}

}  // namespace scfd
