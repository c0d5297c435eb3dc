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
// One warp integrates one reactor: every source-term evaluation spreads the
// species thermo and the reaction rates over the lanes (the rates are summed
// per species in Fex_var's order), the Rosenbrock substep's Jex spreads the
// reactions' derivative rows over the lanes and sums them per species in
// Jex's order, its LU works on rows across lanes, and the serial-order sums
// and the triangular solves run on lane 0, so each step does the arithmetic of
// the one-thread code (chem_dev.cuh) in the same order.
//
// Work distribution (SCFD_REACTOR_QUEUE): reactors need very different numbers
// of substeps, so one persistent launch has every warp pull reactors from a
// device counter until none is left.  The launch (status and counter reset +
// kernel) is captured in a CUDA graph at the first run and replayed afterwards.
// SCFD_REACTOR_PER_LAUNCH runs the same kernel once per reactor, as a loop
// over single-reactor calls would.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "chem_dev.cuh"
#include "chem_tables.h"
#include "scfd_internal.h"

namespace scfd {

// Per-species contribution lists of the reaction rates, in the order in which
// Fex_var (FJ.f90:301-453) accumulates them: entry 2*i + kind adds the forward
// (kind 0) or reverse (kind 1) rate of reaction i; p lists the production
// terms, m the destruction terms; mref[i] is the reaction whose third-body
// term reaction i uses (-1: none yet).
//
// For Fex / Jex (FJ.f90:152-709), the net list of species j, n_ptr[j] ..
// n_ptr[j+1], holds 2*i + 1 for every reactant slot of j in reaction i and
// 2*i for every product slot, reactions in order and reactants first, as the
// reference subtracts and adds Dr; dref[i] is the last reaction up to i that
// sets dlnkdlnM (third-body or fall-off rate; -1: none yet).
struct RateLists {
    const int* p_ptr;  // [ns+1]
    const int* p_ent;
    const int* m_ptr;  // [ns+1]
    const int* m_ent;
    const int* mref;   // [nr]
    const int* n_ptr;  // [ns+1]
    const int* n_ent;
    const int* dref;   // [nr]
};

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
    RateLists rl;
    int wstride;          // doubles of shared memory per warp
};

// Shared-memory arrays of one warp (one reactor); N = ns + 1.
struct WarpMem {
    double *y0, *y, *yp, *q0, *p0, *q, *p, *f0, *k1, *k2, *M;
    double *mu, *e, *cv, *lm, *rf, *rr;
    double *dmu, *dcv, *vm, *dl, *dr, *drdn;  // Jex: per-species T-derivatives, per-reaction terms
    int* piv;
    __device__ WarpMem(double* b, int N, int ns, int nr) {
        y0 = b; y = y0 + N; yp = y + N; q0 = yp + N; p0 = q0 + N; q = p0 + N; p = q + N;
        f0 = p + N; k1 = f0 + N; k2 = k1 + N; M = k2 + N;
        mu = M + N * N; e = mu + ns; cv = e + ns; lm = cv + ns; rf = lm + nr; rr = rf + nr;
        dmu = rr + nr; dcv = dmu + ns; vm = dcv + ns; dl = vm + nr; dr = dl + nr; drdn = dr + nr;
        piv = reinterpret_cast<int*>(drdn + nr * N);
    }
};

__host__ __device__ inline int warp_mem_doubles(int ns, int nr) {
    const int N = ns + 1;
    return 10 * N + N * N + 5 * ns + 6 * nr + nr * N + (N + 1) / 2 + 1;
}

// Fex_var of the state n (shared memory) by one warp: species thermo and
// reaction rates across lanes, per-species sums in the serial order.
__device__ __noinline__ void warp_fex(const DevChem& ch, const RateLists& rl, const double* n, double* dndtp, double* dndtm,
                         WarpMem& w, int lane) {
    const int ns = ch.ns, nr = ch.nr;
    double sn = 0.0;
    if (lane == 0)
        for (int j = 0; j < ns; ++j) sn += n[j];
    sn = __shfl_sync(0xffffffffu, sn, 0);
    FexPre f;
    fex_pre(f, n[ns], sn);
    for (int j = lane; j < ns; j += 32) species_thermo(ch, j, f, w.mu[j], w.e[j], w.cv[j]);
    for (int i = lane; i < nr; i += 32)
        if (ch.exist_m[i]) w.lm[i] = third_body_logM(ch, i, n, f);
    __syncwarp();
    for (int i = lane; i < nr; i += 32) {
        const int r = rl.mref[i];
        reaction_rates(ch, i, n, f, r >= 0 ? w.lm[r] : 0.0, w.mu, w.rf[i], w.rr[i]);
    }
    __syncwarp();
    for (int j = lane; j < ns; j += 32) {
        double a = 0.0;
        for (int k = rl.p_ptr[j]; k < rl.p_ptr[j + 1]; ++k) {
            const int en = rl.p_ent[k];
            a = a + ((en & 1) ? w.rr[en >> 1] : w.rf[en >> 1]);
        }
        dndtp[j] = a;
        a = 0.0;
        for (int k = rl.m_ptr[j]; k < rl.m_ptr[j + 1]; ++k) {
            const int en = rl.m_ent[k];
            a = a - ((en & 1) ? w.rr[en >> 1] : w.rf[en >> 1]);
        }
        dndtm[j] = a;
    }
    __syncwarp();
    if (lane == 0) {
        double de = 0.0, cv = 0.0;
        for (int j = 0; j < ns; ++j) {
            de = de + w.e[j] * (dndtp[j] + dndtm[j]);
            cv = cv + w.cv[j] * n[j];
        }
        dndtp[ns] = fmax(-de * f.T / cv, 0.0);
        dndtm[ns] = fmin(-de * f.T / cv, 0.0);
    }
    __syncwarp();
}

// Fex (J == nullptr) or Jex (FJ.f90:152-709) of the state n (shared memory)
// by one warp: species thermo and reactions across lanes, the per-species
// sums in the reference's serial order (net lists), the T row on lane j.
// dndt[0..ns] and, for Jex, J (row-major N x N) are written to shared memory.
__device__ __noinline__ void warp_jex(const DevChem& ch, const RateLists& rl, const double* n, double* dndt, double* J,
                         WarpMem& w, int lane) {
    const int ns = ch.ns, nr = ch.nr, N = ns + 1;
    const bool jac = J != nullptr;
    double sn = 0.0;
    if (lane == 0)
        for (int j = 0; j < ns; ++j) sn += n[j];
    sn = __shfl_sync(0xffffffffu, sn, 0);
    if (jac) sn = fmax(sn, 1e-300);
    FexPre f;
    fex_pre(f, n[ns], sn);
    double cdmurt[7], cdcpr[7];
    jex_pre(f.T, cdmurt, cdcpr);
    for (int j = lane; j < ns; j += 32) species_thermo_d(ch, j, f, cdmurt, cdcpr, w.mu[j], w.dmu[j], w.e[j], w.cv[j], w.dcv[j]);
    for (int i = lane; i < nr; i += 32)
        if (ch.exist_m[i]) {
            double tmp = f.sn;
            const int nm = ch.numm[i];
            for (int j = 0; j < nm; ++j) tmp = tmp + ch.men[i * ns + j] * n[ch.indm[i * ns + j]];
            w.vm[i] = tmp;
            w.lm[i] = (tmp == f.sn) ? f.logsn : log(tmp);
        }
    __syncwarp();
    for (int i = lane; i < nr; i += 32) {
        const int r = rl.mref[i];
        double dl = 0.0;  // read only where this reaction sets it (dref)
        reaction_jac(ch, i, n, f, r >= 0 ? w.lm[r] : 0.0, w.mu, w.dmu, dl, w.dr[i], w.drdn + i * N);
        w.dl[i] = dl;
    }
    __syncwarp();
    if (jac)
        for (int i = lane; i < nr; i += 32)
            if (ch.exist_m[i]) {
                const int d = rl.dref[i];
                reaction_jac_m(ch, i, w.dr[i], d >= 0 ? w.dl[d] : 0.0, w.vm[i], w.drdn + i * N);
            }
    __syncwarp();
    for (int j = lane; j < ns; j += 32) {
        double a = 0.0;
        for (int k = rl.n_ptr[j]; k < rl.n_ptr[j + 1]; ++k) {
            const int en = rl.n_ent[k];
            a = (en & 1) ? a - w.dr[en >> 1] : a + w.dr[en >> 1];
        }
        dndt[j] = a;
    }
    if (jac)
        for (int t = lane; t < ns * N; t += 32) {
            const int j = t / N, c = t - j * N;
            double a = 0.0;
            for (int k = rl.n_ptr[j]; k < rl.n_ptr[j + 1]; ++k) {
                const int en = rl.n_ent[k];
                const double v = w.drdn[(en >> 1) * N + c];
                a = (en & 1) ? a - v : a + v;
            }
            J[j * N + c] = a;
        }
    __syncwarp();
    if (lane == 0) {
        double de = 0.0, cv = 0.0, dcv = 0.0, t1 = 0.0, t2 = 0.0;
        for (int j = 0; j < ns; ++j) {
            if (jac) t1 = t1 + w.e[j] * J[j * N + ns];
            de = de + w.e[j] * dndt[j];
            dcv = dcv + w.cv[j] * dndt[j];
            cv = cv + w.cv[j] * n[j];
            t2 = t2 + w.dcv[j] * n[j];
        }
        dndt[ns] = -de * f.T / cv;
        if (jac) J[ns * N + ns] = -(f.T * t1 + dcv + dndt[ns] * t2) / cv;
    }
    __syncwarp();
    if (jac) {
        double cv = 0.0;  // the same sum on every lane
        for (int j = 0; j < ns; ++j) cv = cv + w.cv[j] * n[j];
        for (int j = lane; j < ns; j += 32) {
            double t = 0.0;
            for (int k = 0; k < ns; ++k) t = t + w.e[k] * J[k * N + j];
            J[ns * N + j] = -(f.T * t + dndt[ns] * w.cv[j]) / cv;
        }
    }
    __syncwarp();
}

// NaN-propagating min / max over the warp (order-free: exact comparisons)
__device__ inline double warp_min_nan(double v) {
    for (int o = 16; o > 0; o >>= 1) {
        const double u = __shfl_xor_sync(0xffffffffu, v, o);
        v = (u < v || u != u) ? u : v;
    }
    return v;
}
__device__ inline double warp_max_nan(double v) {
    for (int o = 16; o > 0; o >>= 1) {
        const double u = __shfl_xor_sync(0xffffffffu, v, o);
        v = (u > v || u != u) ? u : v;
    }
    return v;
}

// Scalars of one CHEMEQ2 call (uniform over the warp).
struct CallState {
    double tt, tout, dt, counter, h_carry;
    int countersum, substeps, rejects;
    bool fell_back;
    long long evals;
};

// Rosenbrock substep (be_attempt of chem_dev.cuh) by one warp: Jex for the
// matrix, Fex for the second stage.
__device__ int warp_ros_attempt(const DevChem& ch, const RateLists& rl, WarpMem& w, CallState& s, double rtol,
                                int max_substeps, int lane) {
    const int ns = ch.ns, N = ns + 1;
    const double gam = 1.7071067811865475;
    double h = s.dt;
    if (s.tout - s.tt < h) h = s.tout - s.tt;
    // M = I - gamma h J with Jex's exact Jacobian at y0; f0 = Fex(y0) (Jex's dndt)
    warp_jex(ch, rl, w.y0, w.f0, w.M, w, lane);
    for (int t = lane; t < N * N; t += 32) {
        const int i = t / N, j = t - i * N;
        w.M[t] = (i == j ? 1.0 : 0.0) - gam * h * w.M[t];
    }
    __syncwarp();
    // LU with partial pivoting: first largest pivot, rows eliminated across lanes
    bool ok = true;
    for (int k = 0; k < N && ok; ++k) {
        int pk = k;
        if (lane == 0) {
            double best = fabs(w.M[k * N + k]);
            for (int i = k + 1; i < N; ++i)
                if (fabs(w.M[i * N + k]) > best) {
                    best = fabs(w.M[i * N + k]);
                    pk = i;
                }
            w.piv[k] = pk;
            if (!(best > 0.0)) pk = -1;
        }
        pk = __shfl_sync(0xffffffffu, pk, 0);
        if (pk < 0) {
            ok = false;
            break;
        }
        if (pk != k)
            for (int j = lane; j < N; j += 32) {
                const double t = w.M[k * N + j];
                w.M[k * N + j] = w.M[pk * N + j];
                w.M[pk * N + j] = t;
            }
        __syncwarp();
        const double inv = 1.0 / w.M[k * N + k];
        for (int i = k + 1 + lane; i < N; i += 32) {
            const double l = w.M[i * N + k] * inv;
            w.M[i * N + k] = l;
            for (int j = k + 1; j < N; ++j) w.M[i * N + j] = w.M[i * N + j] - l * w.M[k * N + j];
        }
        __syncwarp();
    }
    double err = 1e300;
    if (ok) {
        if (lane == 0) {
            for (int i = 0; i < N; ++i) w.k1[i] = w.f0[i];
            lu_solve(w.M, w.piv, N, w.k1);
        }
        __syncwarp();
        for (int i = lane; i < N; i += 32) w.y[i] = w.y0[i] + h * w.k1[i];
        __syncwarp();
        warp_jex(ch, rl, w.y, w.q, nullptr, w, lane);
        if (lane == 0) {
            for (int i = 0; i < N; ++i) w.k2[i] = w.q[i] - 2.0 * w.k1[i];
            lu_solve(w.M, w.piv, N, w.k2);
        }
        __syncwarp();
        double e = 0.0;
        for (int i = lane; i < N; i += 32) {
            w.y[i] = w.y0[i] + 1.5 * h * w.k1[i] + 0.5 * h * w.k2[i];
            const double ei = fabs(0.5 * h * (w.k1[i] + w.k2[i])) / be_weight(i, ns, w.y[i], rtol);
            e = (ei > e || ei != ei) ? ei : e;
        }
        err = warp_max_nan(e);
    }
    s.evals += 2;
    __syncwarp();
    if (!(err <= 1.0)) {
        s.dt = h * (err == err && err < 1e300 ? fmax(0.2, 0.8 / sqrt(err)) : 0.25);
        if (++s.rejects > 30) return -SCFD_E_CHEM;
        return 0;
    }
    s.rejects = 0;
    s.tt = s.tt + h;
    for (int i = lane; i < N; i += 32) w.y0[i] = w.y[i];
    __syncwarp();
    s.dt = h * fmin(2.0, fmax(0.2, 0.8 / sqrt(fmax(err, 1e-10))));
    s.h_carry = s.dt;
    if (s.tout <= s.tt) return 1;
    if (++s.substeps > max_substeps) return -SCFD_E_CHEM;
    return 0;
}

// One attempt (ceq_attempt of chem_dev.cuh) by one warp.
__device__ int warp_ceq_attempt(const DevChem& ch, const RateLists& rl, WarpMem& w, CallState& s, double rtol,
                                int max_substeps, int lane) {
    if (s.fell_back) return warp_ros_attempt(ch, rl, w, s, rtol, max_substeps, lane);
    const int ns = ch.ns, N = ns + 1;
    for (int i = lane; i < N; i += 32) w.y[i] = w.y0[i];
    __syncwarp();
    s.countersum += 1;
    if (s.countersum > 10) {
        s.fell_back = true;
        s.rejects = 0;
        if (s.h_carry > 0.0) s.dt = s.h_carry;
        return warp_ros_attempt(ch, rl, w, s, rtol, max_substeps, lane);
    }
    s.evals += 2;
    const double dt = s.dt;
    warp_fex(ch, rl, w.y, w.q0, w.p0, w, lane);
    for (int i = lane; i < ns; i += 32) {
        const double p0 = -w.p0[i] / (w.y[i] + 1e-300);
        w.p0[i] = p0;
        const double var = p0 * dt, var2 = var * var, var3 = var * var2;
        const double alp = (180.0 + 60.0 * var + 11.0 * var2 + var3) / (360.0 + 60.0 * var + 12.0 * var2 + var3);
        w.yp[i] = w.y0[i] + dt * (w.q0[i] - p0 * w.y0[i]) / (1.0 + alp * p0 * dt);
    }
    if (lane == 0) w.yp[ns] = w.y0[ns] + dt * (w.q0[ns] + w.p0[ns]);
    __syncwarp();
    warp_fex(ch, rl, w.yp, w.q, w.p, w, lane);
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
    r.s.rejects = 0;
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
    r.s.h_carry = 0.0;
    r.tg = 0.0;
    r.t_old = 0.0;
    r.T_old = r.T0;
    r.t_ign = -1.0;
    r.ignited = false;
    r.fell_back = false;
    warp_call(a, r, w, N, lane);
    int rc = 0;
    for (;;) {
        const double t_before = r.s.tt;
        rc = warp_ceq_attempt(ch, a.rl, w, r.s, ch.rtol, a.max_substeps, lane);
        r.fell_back = r.fell_back || r.s.fell_back;
        if (r.s.tt > t_before) {  // accepted substep
            const double T = w.y[ns], t = r.tg + r.s.tt, Tig = r.T0 + a.dT;
            if (!r.ignited && T >= Tig) {
                r.t_ign = t - (T - Tig) / (T - r.T_old) * (t - r.t_old);
                r.ignited = true;
            }
            r.T_old = T;
            r.t_old = t;
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
        warp_reactor(ch, a, w, (int)k, lane);
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
    RateLists rl{};
    int wstride = 0;  // doubles of shared memory per warp
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
    a.rl = r->rl;
    a.wstride = r->wstride;
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
    const unsigned blocks = (unsigned)((warps + 3) / 4);
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
        k_reactors<<<blocks, 128, 4 * wbytes, r->stream>>>(r->ch, a);
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
    // per-species rate lists in the accumulation order of Fex_var (FJ.f90:301-453)
    const int ns = chem->ns, nr = chem->nr;
    std::vector<int> pp(ns + 1, 0), mp(ns + 1, 0), np_(ns + 1, 0), pe, me, ne_, mref(nr > 0 ? nr : 1, -1),
        dref(nr > 0 ? nr : 1, -1);
    {
        std::vector<std::vector<int>> pl(ns), ml(ns), nl(ns);
        int last = -1, lastd = -1;
        for (int i = 0; i < nr; ++i) {
            if (chem->exist_m[i]) last = i;
            mref[i] = last;
            const int rs0 = chem->rstate[i][0], rs1 = chem->rstate[i][1];
            if (rs1 >= 4 || (rs0 == 0 && (rs1 == 2 || rs1 == 3))) lastd = i;
            dref[i] = lastd;
            for (int k = 0; k < chem->numnu[i][0]; ++k) nl[chem->indnu[i][0][k]].push_back(2 * i + 1);
            for (int k = 0; k < chem->numnu[i][1]; ++k) nl[chem->indnu[i][1][k]].push_back(2 * i);
            const int nreac = chem->numnu[i][0], nprod = chem->numnu[i][1];
            for (int k = 0; k < nreac; ++k) ml[chem->indnu[i][0][k]].push_back(2 * i);
            for (int k = 0; k < nprod; ++k) pl[chem->indnu[i][1][k]].push_back(2 * i);
            if (chem->rstate[i][0] == 0) {
                for (int k = 0; k < nreac; ++k) pl[chem->indnu[i][0][k]].push_back(2 * i + 1);
                for (int k = 0; k < nprod; ++k) ml[chem->indnu[i][1][k]].push_back(2 * i + 1);
            }
        }
        for (int j = 0; j < ns; ++j) {
            pe.insert(pe.end(), pl[j].begin(), pl[j].end());
            me.insert(me.end(), ml[j].begin(), ml[j].end());
            ne_.insert(ne_.end(), nl[j].begin(), nl[j].end());
            pp[j + 1] = (int)pe.size();
            mp[j + 1] = (int)me.size();
            np_[j + 1] = (int)ne_.size();
        }
        if (pe.empty()) pe.push_back(0);
        if (me.empty()) me.push_back(0);
        if (ne_.empty()) ne_.push_back(0);
    }
    r->wstride = (warp_mem_doubles(ns, nr) + 1) & ~1;
    const int blk_smem = 4 * r->wstride * (int)sizeof(double);
    if (blk_smem > 48 * 1024) {
        e = cudaFuncSetAttribute(k_reactors, cudaFuncAttributeMaxDynamicSharedMemorySize, blk_smem);
        if (e != cudaSuccess) return fail(e);
    }
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t bytes = tabs.bytes() + 3 * al(nn * 8) + 2 * al(nv * 8) + al(nn * 8) + al(nn * 4) + 2 * 256 +
                         2 * al(pp.size() * 4) + al(pe.size() * 4) + al(me.size() * 4) + al(mref.size() * 4) +
                         al(np_.size() * 4) + al(ne_.size() * 4) + al(dref.size() * 4);
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
    int* dpp = carve_r<int>(p, pp.size());
    int* dpe = carve_r<int>(p, pe.size());
    int* dmp = carve_r<int>(p, mp.size());
    int* dme = carve_r<int>(p, me.size());
    int* dmr = carve_r<int>(p, mref.size());
    int* dnp = carve_r<int>(p, np_.size());
    int* dne = carve_r<int>(p, ne_.size());
    int* ddr = carve_r<int>(p, dref.size());
    for (auto cp : {std::make_pair(dpp, &pp), std::make_pair(dpe, &pe), std::make_pair(dmp, &mp),
                    std::make_pair(dme, &me), std::make_pair(dmr, &mref), std::make_pair(dnp, &np_),
                    std::make_pair(dne, &ne_), std::make_pair(ddr, &dref)}) {
        e = cudaMemcpyAsync(cp.first, cp.second->data(), cp.second->size() * sizeof(int), cudaMemcpyHostToDevice,
                            r->stream);
        if (e != cudaSuccess) return fail(e);
    }
    r->rl = RateLists{dpp, dpe, dmp, dme, dmr, dnp, dne, ddr};
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

