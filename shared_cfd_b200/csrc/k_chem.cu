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
// Where the reference hands the rest of an interval to DVODE after 10 attempts
// (sub_chem.f90:1755-1775) both this kernel and the CPU restatement take the
// implicit Rosenbrock substeps of chem_dev.cuh and count the cell (stated
// deviation).
#include "chem_dev.cuh"
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
    s.rejects = 0;
    s.evals = 0;
    s.h_carry = 0.0;
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

__global__ void __launch_bounds__(128) k_chem(View v, long long ncells, unsigned long long* counter, int max_substeps) {
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
            if (r < 0) atomicMax(&v.sc->status, -r);
            ceq_store(v, c, s);
            if (s.fell_back) ++fallback;
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
    }
}

int launch_chem_impl(const View& v, cudaStream_t s, int max_substeps, unsigned long long* counter, int nsm) {
    long long n = 0;
    for (int a = 0; a < v.P.nact; ++a) n += (long long)v.P.ni[v.P.act[a]] * v.P.nj[v.P.act[a]];
    if (n == 0) return 0;
    cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s);
    // persistent grid: a few CTAs per SM, capped by the work
    long long blocks = (long long)nsm * 8;
    const long long need = (n + 127) / 128;
    if (blocks > need) blocks = need;
    if (blocks < 1) blocks = 1;
    k_chem<<<(unsigned)blocks, 128, 0, s>>>(v, n, counter, max_substeps > 0 ? max_substeps : 1000000);
    return 1;
}

}  // namespace scfd
