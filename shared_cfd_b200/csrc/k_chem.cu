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
// (sub_chem.f90:1755-1775) both this kernel and the CPU restatement keep taking
// alpha-QSS substeps and count the cell (stated deviation).
#include "scfd_internal.h"

namespace scfd {

__device__ void dev_fex_var(const DevChem& ch, const double* n, double* dndtp, double* dndtm) {
    const int ns = ch.ns;
    const double pst = 1.01325e6, Ru = 8.3144621e7;
    const double loge210 = (double)0.43429448190325f;
    const double T = n[ns];
    const double logT = log(T), Tinv = 1.0 / T;
    const double logPRT = log(pst / Ru) - logT;
    double sn = 0.0;
    for (int j = 0; j < ns; ++j) sn += n[j];
    const double logsn = log(sn);
    const double T2 = T * T, T3 = T2 * T, T4 = T3 * T;
    const double cmurt[7] = {1.0 - logT, -T / 2.0, -T2 / 6.0, -T3 / 12.0, -T4 / 20.0, Tinv, -1.0};
    const double chrt[7] = {1.0, T / 2.0, T2 / 3.0, T3 / 4.0, T4 / 5.0, Tinv, 0.0};
    const double ccpr[7] = {1.0, T, T2, T3, T4, 0.0, 0.0};
    double vmu0rt[kMaxSpecies], vert[kMaxSpecies], vcvr[kMaxSpecies];
    for (int j = 0; j < ns; ++j) {
        const double* cf = ch.coeff + (j * 2 + (T <= ch.tcommon[j] ? 0 : 1)) * 7;
        double t1 = 0.0, t2 = -1.0, t3 = -1.0;
#pragma unroll
        for (int i = 0; i < 7; ++i) {
            const double c = cf[i];
            t1 = t1 + c * cmurt[i];
            t2 = t2 + c * chrt[i];
            t3 = t3 + c * ccpr[i];
        }
        vmu0rt[j] = t1;
        vert[j] = t2;
        vcvr[j] = t3;
        dndtp[j] = 0.0;
        dndtm[j] = 0.0;
    }
    const double dd = 0.14;
    double vlogM = 0.0;
    for (int i = 0; i < ch.nr; ++i) {
        const int rs0 = ch.rstate[2 * i], rs1 = ch.rstate[2 * i + 1];
        if (ch.exist_m[i]) {
            double tmp = sn;
            const int nm = ch.numm[i];
            for (int j = 0; j < nm; ++j) tmp = tmp + ch.men[i * ns + j] * n[ch.indm[i * ns + j]];
            vlogM = (tmp == sn) ? logsn : log(tmp);
        }
        const double* abe = ch.abe + 3 * i;
        double vlogk1 = abe[0] + abe[1] * logT - abe[2] * Tinv;
        double vlogk2 = 0.0;
        if (rs1 >= 4) vlogk1 = vlogk1 + vlogM;
        const int* ind = ch.indnu + 6 * i;
        const int nreac = ch.numnu[2 * i], nprod = ch.numnu[2 * i + 1];
        if (rs0 == 0) {
            const double* cabe = ch.cabe + 3 * i;
            if (rs1 == 1 || rs1 == 5) {
                vlogk2 = cabe[0] + cabe[1] * logT - cabe[2] * Tinv;
                if (rs1 == 5) vlogk2 = vlogk2 + vlogM;
            } else {
                if (rs1 == 2 || rs1 == 3) {
                    const double logk0 = cabe[0] + cabe[1] * logT - cabe[2] * Tinv;
                    const double logkinf = vlogk1;
                    const double log_Pr = logk0 - logkinf + vlogM;
                    const double Pr = exp(log_Pr);
                    vlogk1 = logkinf + log(Pr / (1.0 + Pr));
                    if (rs1 == 3) {
                        const double* tr = ch.troe + 4 * i;
                        const double aa = tr[0];
                        const double logFcent =
                            log10((1.0 - aa) * exp(-T * tr[1]) + aa * exp(-T * tr[2]) + exp(-Tinv * tr[3]));
                        const double cc = -0.4 - 0.67 * logFcent;
                        const double nn = 0.75 - 1.27 * logFcent;
                        const double logPrc = log_Pr * loge210 + cc;
                        const double a = logPrc / (nn - dd * logPrc);
                        const double logF = 1.0 / (1.0 + a * a) * logFcent;
                        vlogk1 = vlogk1 + logF / loge210;
                    }
                }
                double t1 = 0.0;
                for (int k = 0; k < nreac; ++k) t1 = t1 - vmu0rt[ind[k]];
                for (int k = 0; k < nprod; ++k) t1 = t1 + vmu0rt[ind[3 + k]];
                vlogk2 = vlogk1 - ch.snu[i] * logPRT + t1;
            }
        }
        double r = exp(vlogk1);
        for (int k = 0; k < nreac; ++k) r = r * n[ind[k]];
        for (int k = 0; k < nreac; ++k) dndtm[ind[k]] = dndtm[ind[k]] - r;
        for (int k = 0; k < nprod; ++k) dndtp[ind[3 + k]] = dndtp[ind[3 + k]] + r;
        if (rs0 == 0) {
            r = exp(vlogk2);
            for (int k = 0; k < nprod; ++k) r = r * n[ind[3 + k]];
            for (int k = 0; k < nreac; ++k) dndtp[ind[k]] = dndtp[ind[k]] + r;
            for (int k = 0; k < nprod; ++k) dndtm[ind[3 + k]] = dndtm[ind[3 + k]] - r;
        }
    }
    double de = 0.0, cv = 0.0;
    for (int j = 0; j < ns; ++j) {
        de = de + vert[j] * (dndtp[j] + dndtm[j]);
        cv = cv + vcvr[j] * n[j];
    }
    dndtp[ns] = fmax(-de * T / cv, 0.0);
    dndtm[ns] = fmin(-de * T / cv, 0.0);
}

// Per-thread CHEMEQ2 state machine (sub_chem.f90:1714-1819).
struct Ceq {
    double y[kMaxSpecies + 1], y0[kMaxSpecies + 1];
    double tt, tout, dt, ratio, counter;
    int countersum, substeps;
    bool fell_back;
};

// One attempt; returns 1 when the interval is done, 0 to continue, <0 error.
__device__ int ceq_attempt(const DevChem& ch, Ceq& s, double rtol, int max_substeps, long long& attempts) {
    const int ns = ch.ns;
    double yp[kMaxSpecies + 1], p[kMaxSpecies + 1], q[kMaxSpecies + 1], p0[kMaxSpecies + 1], q0[kMaxSpecies + 1];
    for (int i = 0; i <= ns; ++i) s.y[i] = s.y0[i];
    s.countersum += 1;
    if (s.countersum > 10) s.fell_back = true;
    ++attempts;
    const double dt = s.dt;
    dev_fex_var(ch, s.y, q0, p0);
    for (int i = 0; i < ns; ++i) {
        p0[i] = -p0[i] / (s.y[i] + 1e-300);
        const double var = p0[i] * dt, var2 = var * var, var3 = var * var2;
        const double alp = (180.0 + 60.0 * var + 11.0 * var2 + var3) / (360.0 + 60.0 * var + 12.0 * var2 + var3);
        yp[i] = s.y0[i] + dt * (q0[i] - p0[i] * s.y0[i]) / (1.0 + alp * p0[i] * dt);
    }
    yp[ns] = s.y0[ns] + dt * (q0[ns] + p0[ns]);
    double ratio = 1e300;
    dev_fex_var(ch, yp, q, p);
    for (int i = 0; i < ns; ++i) {
        p[i] = -p[i] / (yp[i] + 1e-300);
        p[i] = 0.5 * (p0[i] + p[i]);
        const double var = p[i] * dt, var2 = var * var, var3 = var * var2;
        const double alp = (180.0 + 60.0 * var + 11.0 * var2 + var3) / (360.0 + 60.0 * var + 12.0 * var2 + var3);
        q[i] = alp * q[i] + (1.0 - alp) * q0[i];
        s.y[i] = s.y0[i] + dt * (q[i] - p[i] * s.y0[i]) / (1.0 + alp * p[i] * dt);
        const double v2 = (s.y[i] * rtol + rtol * 1e-5) / fabs(s.y[i] - yp[i] + 1e-300);
        ratio = fmin(ratio, v2);
    }
    s.y[ns] = s.y0[ns] + 0.5 * dt * (q[ns] + p[ns] + q0[ns] + p0[ns]);
    s.ratio = ratio;
    if (1.0 < ratio) {
        // accepted
        s.tt = s.tt + dt;
        if (s.tout <= s.tt) return 1;
        s.dt = dt * sqrt(ratio);
        if (++s.substeps > max_substeps) return -SCFD_E_CHEM;
        for (int i = 0; i <= ns; ++i) s.y0[i] = s.y[i];
        s.counter = 0.0;
        if (s.tout - s.tt < s.dt) s.dt = s.tout - s.tt;
        return 0;
    }
    s.counter = s.counter + 1.0;
    s.dt = dt * sqrt(ratio) / s.counter;
    if (s.counter > 10.0) return -SCFD_E_CHEM;
    return 0;
}

__device__ __forceinline__ long long cell_of(const View& v, long long k, int& pl) {
    // k enumerates interior cells plane by plane
    for (int p = 0; p < v.P.np; ++p) {
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
    for (int p = 0; p < v.P.np; ++p) n += (long long)v.P.ni[p] * v.P.nj[p];
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
