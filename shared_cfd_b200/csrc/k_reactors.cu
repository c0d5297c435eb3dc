// k_reactors.cu -- batched constant-volume 0-D reactors (scfd_reactors_*).
//
// Each reactor is advanced by successive reaction_chemeq2 calls
// (store/therm_lib/chemkin/core/sub_chem.f90:1684-1713) over dt_call up to
// t_end, with the ignition delay of reaction_one_steps (sub_chem.f90:1467-1472)
// taken after every accepted substep (CHEMEQ2, or the Rosenbrock substeps of
// chem_dev.cuh after the fallback):
//     if not ignited and T >= T0 + dT:  t_ign = t - (T - (T0 + dT)) / (T - T_old) * (t - t_old)
// where (t_old, T_old) is the previous accepted substep (initially t = 0, T0).
//
// Work distribution (SCFD_REACTOR_QUEUE): reactors need very different numbers
// of substeps, so one persistent launch has every thread pull reactors from a
// device counter and, in one loop, advance the reactor it holds by one attempt,
// fetching the next reactor when the current one reaches t_end.  The launch
// (status and counter reset + kernel) is captured in a CUDA graph at the first
// run and replayed afterwards.  SCFD_REACTOR_PER_LAUNCH runs the same kernel
// once per reactor, as a loop over single-reactor calls would.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "chem_dev.cuh"
#include "chem_tables.h"
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
};

struct Reactor {
    Ceq s;        // the current reaction_chemeq2 call, local time 0..tout
    double T0, t_old, T_old, t_ign;
    double tg;    // time at the start of the current call
    long long attempts;
    int k;
    bool ignited, fell_back;
};

// Starts a reaction_chemeq2 call at time r.tg from the moles in r.s.y.
__device__ void reactor_call(const ReactorArgs& a, Reactor& r, int ns) {
    for (int j = 0; j <= ns; ++j) r.s.y0[j] = r.s.y[j];
    const double rest = a.t_end - r.tg;
    r.s.tt = 0.0;
    r.s.tout = (a.dt_call > 0.0 && a.dt_call < rest) ? a.dt_call : rest;
    r.s.dt = r.s.tout;
    r.s.countersum = 0;
    r.s.substeps = 0;
    r.s.counter = 0.0;
    r.s.ratio = 0.0;
    r.s.fell_back = false;
    r.s.rejects = 0;
}

__device__ void reactor_load(const DevChem& ch, const ReactorArgs& a, int k, Reactor& r) {
    const int ns = ch.ns;
    r.k = k;
    r.T0 = a.T0[k];
    for (int j = 0; j < ns; ++j) r.s.y[j] = fmax(a.vrho0[(long long)k * ns + j] * ch.inv_mw[j] * 1e-3, 1e-40);
    r.s.y[ns] = r.T0;
    r.s.evals = 0;
    r.tg = 0.0;
    r.t_old = 0.0;
    r.T_old = r.T0;
    r.t_ign = -1.0;
    r.attempts = 0;
    r.ignited = false;
    r.fell_back = false;
    reactor_call(a, r, ns);
}

__device__ void reactor_store(const DevChem& ch, const ReactorArgs& a, const Reactor& r, int rc) {
    const int ns = ch.ns, k = r.k;
    a.T_end[k] = r.s.y[ns];
    for (int j = 0; j < ns; ++j) a.vrho_end[(long long)k * ns + j] = fmax(r.s.y[j], 1e-40) * ch.mws[j] * 1e3;
    a.t_ign[k] = r.ignited ? r.t_ign : -1.0;
    a.evals[k] = r.s.evals;
    a.flags[k] = (r.ignited ? SCFD_REACTOR_IGNITED : 0) | (r.fell_back ? SCFD_REACTOR_FELL_BACK : 0) |
                 (rc < 0 ? SCFD_REACTOR_FAILED : 0);
    if (rc < 0) atomicMax(a.status, -rc);
}

// One attempt (CHEMEQ2, or a Rosenbrock substep after the fallback) of reactor
// r; starts the next reaction_chemeq2 call when one ends (moles floored at
// 1e-40 and passed through the partial densities, as between the reference's
// calls).  Returns 1 at t_end, 0 to continue, <0 error.
__device__ int reactor_attempt(const DevChem& ch, const ReactorArgs& a, Reactor& r) {
    const int ns = ch.ns;
    const double t_before = r.s.tt;
    int rc = ceq_attempt(ch, r.s, ch.rtol, a.max_substeps, r.attempts);
    r.fell_back = r.fell_back || r.s.fell_back;
    if (r.s.tt > t_before) {  // accepted substep
        const double T = r.s.y[ns], t = r.tg + r.s.tt, Tig = r.T0 + a.dT;
        if (!r.ignited && T >= Tig) {
            r.t_ign = t - (T - Tig) / (T - r.T_old) * (t - r.t_old);
            r.ignited = true;
        }
        r.T_old = T;
        r.t_old = t;
    }
    if (rc == 1) {
        r.tg = r.tg + r.s.tout;
        for (int j = 0; j < ns; ++j)
            r.s.y[j] = fmax(fmax(r.s.y[j], 1e-40) * ch.mws[j] * 1e3 * ch.inv_mw[j] * 1e-3, 1e-40);
        if (a.t_end - r.tg > 1e-12 * a.t_end) {
            reactor_call(a, r, ns);
            rc = 0;
        }
    }
    return rc;
}

__global__ void __launch_bounds__(64) k_reactors(DevChem ch, ReactorArgs a) {
    Reactor r;
    bool have = false;
    if (a.queue) {
        const unsigned long long k = atomicAdd(a.counter, 1ull);
        if (k < (unsigned long long)a.n) {
            reactor_load(ch, a, (int)k, r);
            have = true;
        }
    } else if (blockIdx.x == 0 && threadIdx.x == 0) {
        reactor_load(ch, a, a.first, r);
        have = true;
    }
    while (have) {
        const int rc = reactor_attempt(ch, a, r);
        if (rc != 0) {
            reactor_store(ch, a, r, rc);
            have = false;
            if (a.queue) {
                const unsigned long long k = atomicAdd(a.counter, 1ull);
                if (k < (unsigned long long)a.n) {
                    reactor_load(ch, a, (int)k, r);
                    have = true;
                }
            }
        }
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
    if (d->mode == SCFD_REACTOR_PER_LAUNCH) {
        RCK(cudaMemsetAsync(r->status, 0, sizeof(int), r->stream));
        a.queue = 0;
        for (int k = 0; k < d->n; ++k) {
            a.first = k;
            k_reactors<<<1, 32, 0, r->stream>>>(r->ch, a);
        }
        RCK(cudaGetLastError());
        r->launches = d->n;
        return 0;
    }
    a.queue = 1;
    // one thread per reactor up to one warp per SM scheduler pair; beyond that
    // the queue hands each thread several reactors
    const long long threads = std::min<long long>(d->n, (long long)r->nsm * 64);
    const unsigned blocks = (unsigned)((threads + 63) / 64);
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
        k_reactors<<<blocks, 64, 0, r->stream>>>(r->ch, a);
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
    r->launches = 1;
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
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t bytes = tabs.bytes() + 3 * al(nn * 8) + 2 * al(nv * 8) + al(nn * 8) + al(nn * 4) + 2 * 256;
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

}  // extern "C"
