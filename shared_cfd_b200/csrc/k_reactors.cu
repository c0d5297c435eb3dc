// k_reactors.cu -- batched constant-volume 0-D reactors (scfd_reactors_*).
//
// Each reactor is advanced by successive reaction_chemeq2 calls
// (store/therm_lib/chemkin/core/sub_chem.f90:1684-1713) over dt_call up to
// t_end, with the ignition delay of reaction_one_steps (sub_chem.f90:1467-1472)
// taken after every accepted substep (of CHEMEQ2, or of DVODE where an
// interval goes to it after 10 CHEMEQ2 attempts, sub_chem.f90:1755-1775):
//     if not ignited and T >= T0 + dT:  t_ign = t - (T - (T0 + dT)) / (T - T_old) * (t - t_old)
// where (t_old, T_old) is the previous accepted substep (initially t = 0, T0).
//
// One warp integrates one reactor with the one-warp source terms and DVODE of
// chem_warp.cuh.
//
// Work distribution (SCFD_REACTOR_QUEUE): reactors need very different numbers
// of substeps, so one persistent launch has every warp pull reactors from a
// device counter until none is left.  The batch lasts as long as its stiffest
// reactors, so the queue hands them out first (longest job first): a key
// kernel evaluates Fex at every reactor's initial state, a bitonic sort orders
// the reactors by decreasing |dT/dt| there (the initial heat release, which
// ranks the reactors' source-evaluation counts closely), and warps take
// reactors in that order.  The order changes no result.  The launch (resets,
// keys, sort, kernel) is captured in a CUDA graph at the first run and
// replayed afterwards.
// SCFD_REACTOR_PER_LAUNCH runs the same kernel once per reactor, as a loop
// over single-reactor calls would.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "chem_tables.h"
#include "chem_warp.cuh"
#include "scfd_internal.h"

namespace scfd {

struct ReactorArgs {
    int n, first, queue, max_substeps;
    double t_end, dT, dt_call;
    const double* T0;
    const double* vrho0;  // [n][ns]
    double* T_end;
    double* vrho_end;     // [n][ns]
    double* t_ign;
    long long* evals;
    int* flags;
    unsigned long long* counter;
    int* status;
    const int* order;     // queue position -> reactor
    int wstride;          // doubles of shared memory per warp
};

// Scalars of one CHEMEQ2 call (uniform over the warp).
struct CallState {
    double tt, tout, dt, counter;
    int countersum, substeps;
    bool fell_back;
    long long evals;
};

// One attempt (ceq_attempt of chem_dev.cuh) by one warp; 2: the rest of the
// interval goes to DVODE, from (tt, w.y).
__device__ int warp_ceq_attempt(const DevChem& ch, WarpMem& w, CallState& s, double rtol, int max_substeps, int lane) {
    const int ns = ch.ns, N = ns + 1;
    for (int i = lane; i < N; i += 32) w.y[i] = w.y0[i];
    __syncwarp();
    s.countersum += 1;
    if (s.countersum > 10) {
        s.fell_back = true;
        return 2;
    }
    s.evals += 2;
    const double dt = s.dt;
    warp_fex(ch, w.y, w.q0, w.p0, w, lane);
    for (int i = lane; i < ns; i += 32) {
        const double p0 = -w.p0[i] / (w.y[i] + 1e-300);
        w.p0[i] = p0;
        const double var = p0 * dt, var2 = var * var, var3 = var * var2;
        const double alp = (180.0 + 60.0 * var + 11.0 * var2 + var3) / (360.0 + 60.0 * var + 12.0 * var2 + var3);
        w.yp[i] = w.y0[i] + dt * (w.q0[i] - p0 * w.y0[i]) / (1.0 + alp * p0 * dt);
    }
    if (lane == 0) w.yp[ns] = w.y0[ns] + dt * (w.q0[ns] + w.p0[ns]);
    __syncwarp();
    warp_fex(ch, w.yp, w.q, w.p, w, lane);
    double ratio = 1e300;
    for (int i = lane; i < ns; i += 32) {
        double p = -w.p[i] / (w.yp[i] + 1e-300);
        p = 0.5 * (w.p0[i] + p);
        const double var = p * dt, var2 = var * var, var3 = var * var2;
        const double alp = (180.0 + 60.0 * var + 11.0 * var2 + var3) / (360.0 + 60.0 * var + 12.0 * var2 + var3);
        const double q = alp * w.q[i] + (1.0 - alp) * w.q0[i];
        const double y = w.y0[i] + dt * (q - p * w.y0[i]) / (1.0 + alp * p * dt);
        w.y[i] = y;
        const double v2 = (y * rtol + rtol * 1e-5) / fabs(y - w.yp[i] + 1e-300);
        ratio = (v2 < ratio || v2 != v2) ? v2 : ratio;
    }
    if (lane == 0) w.y[ns] = w.y0[ns] + 0.5 * dt * (w.q[ns] + w.p[ns] + w.q0[ns] + w.p0[ns]);
    ratio = warp_min_nan(ratio);
    __syncwarp();
    if (1.0 < ratio) {
        s.tt = s.tt + dt;
        if (s.tout <= s.tt) return 1;
        s.dt = dt * sqrt(ratio);
        if (++s.substeps > max_substeps) return -SCFD_E_CHEM;
        for (int i = lane; i < N; i += 32) w.y0[i] = w.y[i];
        __syncwarp();
        s.counter = 0.0;
        if (s.tout - s.tt < s.dt) s.dt = s.tout - s.tt;
        return 0;
    }
    s.counter = s.counter + 1.0;
    s.dt = dt * sqrt(ratio) / s.counter;
    if (s.counter > 10.0) return -SCFD_E_CHEM;
    return 0;
}

// Reactor scalars (uniform over the warp).
struct ReactorState {
    CallState s;
    double T0, t_old, T_old, t_ign, tg;
    bool ignited, fell_back;
};

// Starts a reaction_chemeq2 call at time r.tg from the moles in w.y.
__device__ void warp_call(const ReactorArgs& a, ReactorState& r, WarpMem& w, int N, int lane) {
    for (int j = lane; j < N; j += 32) w.y0[j] = w.y[j];
    __syncwarp();
    const double rest = a.t_end - r.tg;
    r.s.tt = 0.0;
    r.s.tout = (a.dt_call > 0.0 && a.dt_call < rest) ? a.dt_call : rest;
    r.s.dt = r.s.tout;
    r.s.countersum = 0;
    r.s.substeps = 0;
    r.s.counter = 0.0;
    r.s.fell_back = false;
}

// Whole reactor k by one warp: successive reaction_chemeq2 calls over dt_call
// with the ignition test after every accepted substep (see the file comment).
__device__ void warp_reactor(const DevChem& ch, const ReactorArgs& a, WarpMem& w, int k, int lane) {
    const int ns = ch.ns, N = ns + 1;
    ReactorState r;
    r.T0 = a.T0[k];
    for (int j = lane; j < ns; j += 32) w.y[j] = fmax(a.vrho0[(long long)k * ns + j] * ch.inv_mw[j] * 1e-3, 1e-40);
    if (lane == 0) w.y[ns] = r.T0;
    __syncwarp();
    r.s.evals = 0;
    r.tg = 0.0;
    r.t_old = 0.0;
    r.T_old = r.T0;
    r.t_ign = -1.0;
    r.ignited = false;
    r.fell_back = false;
    warp_call(a, r, w, N, lane);
    int rc = 0;
    // the ignition test of an accepted substep ending at tt (of this call) with temperature T
    auto track = [&](double tt, double T) {
        const double t = r.tg + tt, Tig = r.T0 + a.dT;
        if (!r.ignited && T >= Tig) {
            r.t_ign = t - (T - Tig) / (T - r.T_old) * (t - r.t_old);
            r.ignited = true;
        }
        r.T_old = T;
        r.t_old = t;
    };
    auto on_dvode_step = [&](double tn) { track(tn, w.yh[ns]); };
    for (;;) {
        const double t_before = r.s.tt;
        rc = warp_ceq_attempt(ch, w, r.s, ch.rtol, a.max_substeps, lane);
        r.fell_back = r.fell_back || r.s.fell_back;
        if (rc == 2) {
            // DVODE from (tt, w.y) to tout: the result in w.y
            rc = warp_dvode_rest(ch, w, w.y, r.s.tt, r.s.tout, r.s.evals, lane, on_dvode_step) == 0 ? 1 : -SCFD_E_CHEM;
        } else if (r.s.tt > t_before) {  // accepted substep
            track(r.s.tt, w.y[ns]);
        }
        if (rc == 1) {
            r.tg = r.tg + r.s.tout;
            for (int j = lane; j < ns; j += 32)
                w.y[j] = fmax(fmax(w.y[j], 1e-40) * ch.mws[j] * 1e3 * ch.inv_mw[j] * 1e-3, 1e-40);
            __syncwarp();
            if (a.t_end - r.tg > 1e-12 * a.t_end) {
                warp_call(a, r, w, N, lane);
                continue;
            }
            rc = 0;
            break;
        }
        if (rc < 0) break;
    }
    if (lane == 0) {
        a.T_end[k] = w.y[ns];
        a.t_ign[k] = r.ignited ? r.t_ign : -1.0;
        a.evals[k] = r.s.evals;
        a.flags[k] = (r.ignited ? SCFD_REACTOR_IGNITED : 0) | (r.fell_back ? SCFD_REACTOR_FELL_BACK : 0) |
                     (rc < 0 ? SCFD_REACTOR_FAILED : 0);
        if (rc < 0) atomicMax(a.status, -rc);
    }
    for (int j = lane; j < ns; j += 32) a.vrho_end[(long long)k * ns + j] = fmax(w.y[j], 1e-40) * ch.mws[j] * 1e3;
    __syncwarp();
}

// Fex / Jex of independent states, one thread each (scfd_chem_rates).
__global__ void k_chem_rates(DevChem ch, int n, const double* states, double* dndt, double* jac) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int N = ch.ns + 1;
    double y[kMaxSpecies + 1], f[kMaxSpecies + 1];
    for (int i = 0; i < N; ++i) y[i] = states[(size_t)c * N + i];
    if (jac)
        dev_jex(ch, y, f, jac + (size_t)c * N * N);
    else
        dev_fex(ch, y, f);
    for (int i = 0; i < N; ++i) dndt[(size_t)c * N + i] = f[i];
}

// One warp per reactor; in queue mode each warp takes reactors from the
// device counter until none is left.
__global__ void __launch_bounds__(128) k_reactors(DevChem ch, ReactorArgs a) {
    extern __shared__ __align__(16) double wsm[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpMem w(wsm + (long long)wid * a.wstride, ch.ns + 1, ch.ns, ch.nr);
    if (!a.queue) {
        if (blockIdx.x == 0 && wid == 0) warp_reactor(ch, a, w, a.first, lane);
        return;
    }
    for (;;) {
        unsigned long long k = 0;
        if (lane == 0) k = atomicAdd(a.counter, 1ull);
        k = __shfl_sync(0xffffffffu, k, 0);
        if (k >= (unsigned long long)a.n) break;
        warp_reactor(ch, a, w, a.order[k], lane);
    }
}

// Queue keys: -|dT/dt| of Fex at the initial state (ascending key = stiffest
// first); positions n .. npow2-1 pad the sort with +inf.
__global__ void k_reactor_keys(DevChem ch, ReactorArgs a, int npow2, double* key, int* idx) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= npow2) return;
    double kv = __longlong_as_double(0x7FF0000000000000ll);
    if (k < a.n) {
        const int ns = ch.ns;
        double y[kMaxSpecies + 1], f[kMaxSpecies + 1];
        for (int j = 0; j < ns; ++j) y[j] = fmax(a.vrho0[(long long)k * ns + j] * ch.inv_mw[j] * 1e-3, 1e-40);
        y[ns] = a.T0[k];
        dev_fex(ch, y, f);
        kv = -fabs(f[ns]);
        if (kv != kv) kv = 0.0;
    }
    key[k] = kv;
    idx[k] = k;
}

// One compare-exchange stage (size kk, distance j) of a bitonic sort of
// (key, idx) ascending, ties by index.
__global__ void k_bitonic_stage(double* key, int* idx, int npow2, int kk, int j) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npow2) return;
    const int l = i ^ j;
    if (l <= i) return;
    const double ki = key[i], kl = key[l];
    const int ii = idx[i], il = idx[l];
    const bool gt = ki > kl || (ki == kl && ii > il);
    const bool up = (i & kk) == 0;
    if (gt == up) {
        key[i] = kl;
        key[l] = ki;
        idx[i] = il;
        idx[l] = ii;
    }
}

}  // namespace scfd

using namespace scfd;

struct scfd_reactors {
    int n_max = 0, ns = 0, n = 0, nsm = 1;
    cudaStream_t stream = nullptr;
    char* arena = nullptr;
    DevChem ch{};
    double *T0 = nullptr, *vrho0 = nullptr, *T_end = nullptr, *vrho_end = nullptr, *t_ign = nullptr;
    long long* evals = nullptr;
    int* flags = nullptr;
    int* status = nullptr;
    unsigned long long* counter = nullptr;
    double* qkey = nullptr;  // queue order: sort keys and reactor indices, npow2 each
    int* qidx = nullptr;
    int npow2 = 1;
    int wstride = 0;  // doubles of shared memory per warp
    int wpb = 4;      // warps per block of the queued launch
    // graph of the queued launch, valid for the descriptor values it was captured with
    cudaGraphExec_t graph = nullptr;
    int graph_n = -1, graph_max = -1;
    double graph_t_end = -1.0, graph_dT = -1.0, graph_dt_call = -1.0;
    long long launches = 0;
    std::string err;
};

namespace {

#define RCK(x)                                                      \
    do {                                                            \
        cudaError_t e_ = (x);                                       \
        if (e_ != cudaSuccess) {                                    \
            r->err = std::string(#x ": ") + cudaGetErrorString(e_); \
            return SCFD_E_CUDA;                                     \
        }                                                           \
    } while (0)

template <typename T>
T* carve_r(char*& p, size_t n) {
    T* out = reinterpret_cast<T*>(p);
    p += (n * sizeof(T) + 255) & ~(size_t)255;
    return out;
}

int enqueue(scfd_reactors* r, const scfd_reactor_desc* d) {
    ReactorArgs a{};
    a.n = d->n;
    a.max_substeps = d->max_substeps > 0 ? d->max_substeps : 1000000;
    a.t_end = d->t_end;
    a.dT = d->dT_ign;
    a.dt_call = d->dt_call;
    a.T0 = r->T0;
    a.vrho0 = r->vrho0;
    a.T_end = r->T_end;
    a.vrho_end = r->vrho_end;
    a.t_ign = r->t_ign;
    a.evals = r->evals;
    a.flags = r->flags;
    a.counter = r->counter;
    a.status = r->status;
    a.wstride = r->wstride;
    a.order = r->qidx;
    const size_t wbytes = (size_t)r->wstride * sizeof(double);
    if (d->mode == SCFD_REACTOR_PER_LAUNCH) {
        RCK(cudaMemsetAsync(r->status, 0, sizeof(int), r->stream));
        a.queue = 0;
        for (int k = 0; k < d->n; ++k) {
            a.first = k;
            k_reactors<<<1, 32, wbytes, r->stream>>>(r->ch, a);
        }
        RCK(cudaGetLastError());
        r->launches = d->n;
        return 0;
    }
    a.queue = 1;
    // one warp per reactor, up to 16 warps per SM; beyond that the queue hands
    // each warp several reactors
    const long long warps = std::min<long long>(d->n, (long long)r->nsm * 16);
    const unsigned blocks = (unsigned)((warps + r->wpb - 1) / r->wpb);
    const bool reuse = r->graph && r->graph_n == d->n && r->graph_t_end == d->t_end && r->graph_dT == d->dT_ign &&
                       r->graph_max == a.max_substeps && r->graph_dt_call == d->dt_call;
    if (!reuse) {
        if (r->graph) {
            cudaGraphExecDestroy(r->graph);
            r->graph = nullptr;
        }
        cudaGraph_t g = nullptr;
        RCK(cudaStreamBeginCapture(r->stream, cudaStreamCaptureModeThreadLocal));
        cudaMemsetAsync(r->status, 0, sizeof(int), r->stream);
        cudaMemsetAsync(r->counter, 0, sizeof(unsigned long long), r->stream);
        // the queue order: stiffest reactors first
        int np2 = 1;
        while (np2 < d->n) np2 <<= 1;
        const unsigned sb = (unsigned)((np2 + 255) / 256);
        k_reactor_keys<<<sb, 256, 0, r->stream>>>(r->ch, a, np2, r->qkey, r->qidx);
        for (int kk = 2; kk <= np2; kk <<= 1)
            for (int j = kk >> 1; j > 0; j >>= 1) k_bitonic_stage<<<sb, 256, 0, r->stream>>>(r->qkey, r->qidx, np2, kk, j);
        k_reactors<<<blocks, 32 * r->wpb, r->wpb * wbytes, r->stream>>>(r->ch, a);
        RCK(cudaStreamEndCapture(r->stream, &g));
        const cudaError_t e = cudaGraphInstantiate(&r->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            r->graph = nullptr;
            r->err = std::string("graph instantiate: ") + cudaGetErrorString(e);
            return SCFD_E_CUDA;
        }
        r->graph_n = d->n;
        r->graph_t_end = d->t_end;
        r->graph_dT = d->dT_ign;
        r->graph_max = a.max_substeps;
        r->graph_dt_call = d->dt_call;
    }
    RCK(cudaGraphLaunch(r->graph, r->stream));
    // kernels in the graph: the keys, the sort stages, the reactors
    int np2 = 1, stages = 0;
    while (np2 < d->n) np2 <<= 1;
    for (int kk = 2; kk <= np2; kk <<= 1)
        for (int j = kk >> 1; j > 0; j >>= 1) ++stages;
    r->launches = 2 + stages;
    return 0;
}

}  // namespace

extern "C" {

int scfd_reactors_create(const scfd_chem* chem, int n_max, scfd_reactors** out) {
    if (!chem || !out || n_max < 1 || chem->ns < 1 || chem->ns > SCFD_MAX_SPECIES || chem->nr < 0 ||
        chem->nr > SCFD_MAX_REACTIONS)
        return SCFD_E_ARG;
    *out = nullptr;
    scfd_reactors* r = new scfd_reactors();
    r->n_max = n_max;
    r->ns = chem->ns;
    const ChemTables tabs(*chem);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&r->nsm, cudaDevAttrMultiProcessorCount, dev);
    auto fail = [&](cudaError_t e) {
        r->err = cudaGetErrorString(e);
        scfd_reactors_destroy(r);
        return SCFD_E_CUDA;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(e);
    const size_t nn = (size_t)n_max, nv = nn * r->ns;
    const int ns = chem->ns, nr = chem->nr;
    r->wstride = (warp_mem_doubles(ns, nr) + 1) & ~1;
    // up to 4 warps per block, as many as the shared memory per block allows
    int smem_max = 0;
    cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const int wbytes = r->wstride * (int)sizeof(double);
    r->wpb = std::min(4, smem_max / wbytes);
    if (r->wpb < 1) {
        r->err = "mechanism too large for one warp's shared memory";
        scfd_reactors_destroy(r);
        return SCFD_E_ARG;
    }
    if (r->wpb * wbytes > 48 * 1024) {
        e = cudaFuncSetAttribute(k_reactors, cudaFuncAttributeMaxDynamicSharedMemorySize, r->wpb * wbytes);
        if (e != cudaSuccess) return fail(e);
    }
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    while (r->npow2 < n_max) r->npow2 <<= 1;
    const size_t bytes = tabs.bytes() + 3 * al(nn * 8) + 2 * al(nv * 8) + al(nn * 8) + al(nn * 4) + 2 * 256 +
                         al((size_t)r->npow2 * 8) + al((size_t)r->npow2 * 4);
    e = cudaMalloc(&r->arena, bytes);
    if (e != cudaSuccess) return fail(e);
    char* p = r->arena;
    e = tabs.upload(r->ch, p, r->stream);
    if (e != cudaSuccess) return fail(e);
    r->T0 = carve_r<double>(p, nn);
    r->vrho0 = carve_r<double>(p, nv);
    r->T_end = carve_r<double>(p, nn);
    r->vrho_end = carve_r<double>(p, nv);
    r->t_ign = carve_r<double>(p, nn);
    r->evals = carve_r<long long>(p, nn);
    r->flags = carve_r<int>(p, nn);
    r->status = carve_r<int>(p, 1);
    r->counter = carve_r<unsigned long long>(p, 1);
    r->qkey = carve_r<double>(p, r->npow2);
    r->qidx = carve_r<int>(p, r->npow2);
    if (p > r->arena + bytes) {
        r->err = "arena overflow";
        scfd_reactors_destroy(r);
        return SCFD_E_CUDA;
    }
    e = cudaStreamSynchronize(r->stream);  // the host tables must outlive their copies
    if (e != cudaSuccess) return fail(e);
    *out = r;
    return 0;
}

int scfd_reactors_destroy(scfd_reactors* r) {
    if (!r) return SCFD_E_ARG;
    if (r->graph) cudaGraphExecDestroy(r->graph);
    if (r->arena) cudaFree(r->arena);
    if (r->stream) cudaStreamDestroy(r->stream);
    delete r;
    return 0;
}

int scfd_reactors_upload(scfd_reactors* r, int n, const double* T0, const double* vrho0) {
    if (!r || !T0 || !vrho0 || n < 1 || n > r->n_max) return SCFD_E_ARG;
    RCK(cudaMemcpyAsync(r->T0, T0, sizeof(double) * n, cudaMemcpyHostToDevice, r->stream));
    RCK(cudaMemcpyAsync(r->vrho0, vrho0, sizeof(double) * n * r->ns, cudaMemcpyHostToDevice, r->stream));
    RCK(cudaStreamSynchronize(r->stream));
    r->n = n;
    return 0;
}

int scfd_reactors_launch(scfd_reactors* r, const scfd_reactor_desc* d) {
    if (!r || !d || d->abi_version != SCFD_ABI_VERSION || d->n < 1 || d->n != r->n || !(d->t_end > 0.0) ||
        (d->mode != SCFD_REACTOR_QUEUE && d->mode != SCFD_REACTOR_PER_LAUNCH))
        return SCFD_E_ARG;
    return enqueue(r, d);
}

int scfd_reactors_download(scfd_reactors* r, double* T_end, double* vrho_end, double* t_ign, int64_t* evals,
                           int32_t* flags) {
    if (!r || r->n < 1) return SCFD_E_ARG;
    const size_t n = (size_t)r->n;
    if (T_end) RCK(cudaMemcpyAsync(T_end, r->T_end, sizeof(double) * n, cudaMemcpyDeviceToHost, r->stream));
    if (vrho_end)
        RCK(cudaMemcpyAsync(vrho_end, r->vrho_end, sizeof(double) * n * r->ns, cudaMemcpyDeviceToHost, r->stream));
    if (t_ign) RCK(cudaMemcpyAsync(t_ign, r->t_ign, sizeof(double) * n, cudaMemcpyDeviceToHost, r->stream));
    if (evals) RCK(cudaMemcpyAsync(evals, r->evals, sizeof(long long) * n, cudaMemcpyDeviceToHost, r->stream));
    if (flags) RCK(cudaMemcpyAsync(flags, r->flags, sizeof(int) * n, cudaMemcpyDeviceToHost, r->stream));
    int status = 0;
    RCK(cudaMemcpyAsync(&status, r->status, sizeof(int), cudaMemcpyDeviceToHost, r->stream));
    RCK(cudaStreamSynchronize(r->stream));
    return status;
}

int scfd_reactors_run(scfd_reactors* r, const scfd_reactor_desc* d, const double* T0, const double* vrho0,
                      double* T_end, double* vrho_end, double* t_ign, int64_t* evals, int32_t* flags) {
    if (!d) return SCFD_E_ARG;
    int st = scfd_reactors_upload(r, d->n, T0, vrho0);
    if (st) return st;
    if ((st = scfd_reactors_launch(r, d))) return st;
    return scfd_reactors_download(r, T_end, vrho_end, t_ign, evals, flags);
}

void* scfd_reactors_stream(scfd_reactors* r) { return r ? (void*)r->stream : nullptr; }

int scfd_reactors_launch_count(const scfd_reactors* r, int64_t* launches) {
    if (!r || !launches) return SCFD_E_ARG;
    *launches = r->launches;
    return 0;
}

int scfd_chem_rates(const scfd_chem* chem, int n, const double* states, double* dndt, double* jac) {
    if (!chem || n < 0 || (n > 0 && (!states || !dndt)) || chem->ns < 1 || chem->ns > SCFD_MAX_SPECIES ||
        chem->nr < 0 || chem->nr > SCFD_MAX_REACTIONS)
        return SCFD_E_ARG;
    if (n == 0) return 0;
    const ChemTables tabs(*chem);
    const size_t N = (size_t)chem->ns + 1;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t bs = al(n * N * 8), bj = jac ? al(n * N * N * 8) : 0;
    char* arena = nullptr;
    cudaStream_t st = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&arena, tabs.bytes() + 2 * bs + bj);
    DevChem ch{};
    char* p = arena;
    if (e == cudaSuccess) e = tabs.upload(ch, p, st);
    double* ds = reinterpret_cast<double*>(p);
    double* dd = reinterpret_cast<double*>(p + bs);
    double* dj = jac ? reinterpret_cast<double*>(p + 2 * bs) : nullptr;
    if (e == cudaSuccess) e = cudaMemcpyAsync(ds, states, n * N * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        k_chem_rates<<<(n + 127) / 128, 128, 0, st>>>(ch, n, ds, dd, dj);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(dndt, dd, n * N * 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && jac) e = cudaMemcpyAsync(jac, dj, n * N * N * 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (arena) cudaFree(arena);
    if (st) cudaStreamDestroy(st);
    return e == cudaSuccess ? 0 : SCFD_E_CUDA;
}

}  // extern "C"

