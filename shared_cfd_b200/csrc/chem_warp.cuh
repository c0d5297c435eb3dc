// chem_warp.cuh -- one warp per chemistry state: the UV source terms Fex_var,
// Fex and Jex (store/therm_lib/chemkin/uvhp/uv/FJ.f90:152-709) spread over the
// lanes, and the DVODE integrator (store/therm_lib/chemkin/core/dvode.f) that
// finishes a CHEMEQ2 interval after 10 attempts (sub_chem.f90:1755-1775).
// Shared by the batched 0-D reactors (k_reactors.cu) and the flow chemistry's
// DVODE pass (k_chem.cu).
//
// Every source-term evaluation spreads the species thermo and the reaction
// rates over the lanes and sums the rates per species in the reference's
// order (DevChem::rl), the serial-order sums run on lane 0, so each
// evaluation does the arithmetic of the one-thread code (chem_dev.cuh) in the
// same order.
//
// DVODE.  The path the reference takes: MF = 21 (BDF with the exact Jacobian
// Jex, saved and reused, JSV = 1), ITASK = 1, ITOL = 1, IOPT = 0 (MAXORD 5,
// MXSTEP 500), ISTATE = 1 on every call, and ISTATE = -1 (MXSTEP steps before
// TOUT) answered by calling again from where it stopped, at most
// max_recalc = 50 times (mod_chem.raw.f90:27).  The Nordsieck array YH, the
// iteration matrix and its LU, and the saved Jacobian live in the warp's
// shared memory; the integrator's scalars are held, identical, by every lane.
// Element-wise updates run one row per lane with the reference's operation
// order per element; the weighted RMS norms, the pivot search and the
// initial-step bound (order-dependent loops) run on lane 0 and are broadcast.
// The routines follow dvode.f's: DVODE 2-1672, DVHIN 1673-1810, DVINDY
// 1811-1933, DVSTEP 1934-2368, DVSET 2369-2567, DVJUST 2568-2727, DVNLSD
// 2728-2956, DVJAC 2957-3234, DVSOL 3261-3356, DGEFA / DGESL 3816-4061.
#pragma once

#include "chem_dev.cuh"

namespace scfd {

// Shared-memory arrays of one warp; N = ns + 1.
struct WarpMem {
    double *y0, *y, *yp, *q0, *p0, *q, *p;                                  // CHEMEQ2
    double *mu, *e, *cv, *lm, *rf, *rr, *dmu, *dcv, *vm, *dl, *dr, *drdn;  // Fex / Jex
    double *yh, *ewt, *savf, *acor, *tmp, *dy, *wm, *js;                   // DVODE
    int* ipvt;
    __device__ WarpMem(double* b, int N, int ns, int nr) {
        y0 = b; y = y0 + N; yp = y + N; q0 = yp + N; p0 = q0 + N; q = p0 + N; p = q + N;
        mu = p + N; e = mu + ns; cv = e + ns; lm = cv + ns; rf = lm + nr; rr = rf + nr;
        dmu = rr + nr; dcv = dmu + ns; vm = dcv + ns; dl = vm + nr; dr = dl + nr; drdn = dr + nr;
        yh = drdn + nr * N; ewt = yh + 7 * N; savf = ewt + N; acor = savf + N; tmp = acor + N; dy = tmp + N;
        wm = dy + N; js = wm + N * N;
        ipvt = reinterpret_cast<int*>(js + N * N);
    }
};

__host__ __device__ inline int warp_mem_doubles(int ns, int nr) {
    const int N = ns + 1;
    return 7 * N + 5 * ns + 6 * nr + nr * N + 12 * N + 2 * N * N + (N + 1) / 2 + 1;
}

// Fex_var of the state n (shared memory) by one warp: species thermo and
// reaction rates across lanes, per-species sums in the serial order.
inline __device__ __noinline__ void warp_fex(const DevChem& ch, const double* n, double* dndtp, double* dndtm, WarpMem& w,
                                      int lane) {
    const RateLists& rl = ch.rl;
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
// dndt[0..ns] and, for Jex, d dndt_r / d n_c at J[r * jr + c * jc] are
// written to shared memory.
inline __device__ __noinline__ void warp_jex(const DevChem& ch, const double* n, double* dndt, double* J, int jr, int jc,
                                      WarpMem& w, int lane) {
    const RateLists& rl = ch.rl;
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
    for (int j = lane; j < ns; j += 32)
        species_thermo_d(ch, j, f, cdmurt, cdcpr, w.mu[j], w.dmu[j], w.e[j], w.cv[j], w.dcv[j]);
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
            J[j * jr + c * jc] = a;
        }
    __syncwarp();
    if (lane == 0) {
        double de = 0.0, cv = 0.0, dcv = 0.0, t1 = 0.0, t2 = 0.0;
        for (int j = 0; j < ns; ++j) {
            if (jac) t1 = t1 + w.e[j] * J[j * jr + ns * jc];
            de = de + w.e[j] * dndt[j];
            dcv = dcv + w.cv[j] * dndt[j];
            cv = cv + w.cv[j] * n[j];
            t2 = t2 + w.dcv[j] * n[j];
        }
        dndt[ns] = -de * f.T / cv;
        if (jac) J[ns * jr + ns * jc] = -(f.T * t1 + dcv + dndt[ns] * t2) / cv;
    }
    __syncwarp();
    if (jac) {
        double cv = 0.0;  // the same sum on every lane
        for (int j = 0; j < ns; ++j) cv = cv + w.cv[j] * n[j];
        for (int j = lane; j < ns; j += 32) {
            double t = 0.0;
            for (int k = 0; k < ns; ++k) t = t + w.e[k] * J[k * jr + j * jc];
            J[ns * jr + j * jc] = -(f.T * t + dndt[ns] * w.cv[j]) / cv;
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

namespace dvw {

constexpr int MAXORD = 5;          // MORD(2), BDF
constexpr int MXSTEP = 500;        // MXSTP0
constexpr int MAX_RECALC = 50;     // mod_chem.raw.f90:27
constexpr double UROUND = 2.220446049250313080847e-16;  // DUMACH: 2**-52

// Fortran MAX / MIN of two reals as the reference's compiler evaluates them
__device__ inline double fmax2(double a, double b) { return a < b ? b : a; }
__device__ inline double fmin2(double a, double b) { return b < a ? b : a; }

// real ** integer by binary powering
__device__ inline double ipow(double x, int m) {
    unsigned k = m < 0 ? -m : m;
    double y = (k % 2) ? x : 1.0;
    while (k >>= 1) {
        x = x * x;
        if (k % 2) y = y * x;
    }
    return m < 0 ? 1.0 / y : y;
}

// COMMON /DVOD01/, /DVOD02/ (the members the METH 2 / MITER 1 path uses),
// plus DVSTEP's SAVEd ETAQ, ETAQM1; identical on every lane.
struct Scalars {
    double acnrm, ccmxj, conp, crate, drc, el[14], eta, etamax, h, hmin, hmxi, hnew, hscal, prl1, rc, rl1, tau[14],
        tq[6], tn, hu, etaq, etaqm1;
    int icf, init, ipup, jcur, jstart, kflag, kuth, l, lmax, msbj, newh, newq, nq, nqnyh, nqwait, nslj, nslp, ncfn, netf,
        nfe, nje, nlu, nni, nqu, nst;
};

// One warp's integrator.  Vectors are 0-based in shared memory; YH(i, j) and
// A(i, j) take the reference's 1-based indices.
struct Warp {
    const DevChem& ch;
    WarpMem& w;
    const int n, lane;
    long long& evals;  // Fex / Jex evaluations
    Scalars s;

    __device__ Warp(const DevChem& c, WarpMem& wm_, int lane_, long long& ev)
        : ch(c), w(wm_), n(c.ns + 1), lane(lane_), evals(ev), s() {}

    __device__ double& YH(int i, int j) { return w.yh[(i - 1) + (j - 1) * n]; }
    __device__ double& A(int i, int j) { return w.wm[(i - 1) + (j - 1) * n]; }

    // F and JAC: Fex, and Jex into the iteration-matrix storage (column-major)
    __device__ void f(const double* y, double* ydot) {
        warp_jex(ch, y, ydot, nullptr, 0, 0, w, lane);
        ++evals;
    }
    __device__ void jac(const double* y) {
        warp_jex(ch, y, w.tmp, w.wm, 1, n, w, lane);
        ++evals;
    }

    // DVNORM (dvode.f:3467-3500), lane 0 in the reference's order
    __device__ double vnorm(const double* v) {
        double r = 0.0;
        if (lane == 0) {
            double sum = 0.0;
            for (int i = 0; i < n; ++i) sum = sum + (v[i] * w.ewt[i]) * (v[i] * w.ewt[i]);
            r = sqrt(sum / n);
        }
        r = __shfl_sync(0xffffffffu, r, 0);
        __syncwarp();
        return r;
    }

    // DEWSET with ITOL = 1 and the inversion of DVODE; false on a weight <= 0
    __device__ bool ewset(double rtol, double atol) {
        bool bad = false;
        for (int i = lane; i < n; i += 32) {
            const double e = rtol * fabs(w.yh[i]) + atol;
            if (e <= 0.0) bad = true;
            w.ewt[i] = e;
        }
        __syncwarp();
        if (__any_sync(0xffffffffu, bad)) return false;
        for (int i = lane; i < n; i += 32) w.ewt[i] = 1.0 / w.ewt[i];
        __syncwarp();
        return true;
    }

    // DGEFA (dvode.f:3816-3931); returns INFO.  Column j > k of each
    // elimination step is one lane's.
    __device__ int gefa() {
        int info = 0;
        for (int k = 1; k <= n - 1; ++k) {
            int l = k;
            if (lane == 0) {  // IDAMAX of column k from row k
                double dmax = fabs(A(k, k));
                for (int i = k + 1; i <= n; ++i) {
                    const double xmag = fabs(A(i, k));
                    if (xmag > dmax) {
                        l = i;
                        dmax = xmag;
                    }
                }
                w.ipvt[k - 1] = l;
            }
            l = __shfl_sync(0xffffffffu, l, 0);
            const double alk = A(l, k);
            __syncwarp();
            if (alk == 0.0) {
                info = k;
                continue;
            }
            if (lane == 0 && l != k) {
                A(l, k) = A(k, k);
                A(k, k) = alk;
            }
            __syncwarp();
            const double t = -1.0 / A(k, k);
            for (int i = k + 1 + lane; i <= n; i += 32) A(i, k) = t * A(i, k);  // DSCAL
            __syncwarp();
            for (int j = k + 1 + lane; j <= n; j += 32) {
                const double tj = A(l, j);
                if (l != k) {
                    A(l, j) = A(k, j);
                    A(k, j) = tj;
                }
                for (int i = k + 1; i <= n; ++i) A(i, j) = A(i, j) + tj * A(i, k);  // DAXPY
            }
            __syncwarp();
        }
        if (lane == 0) w.ipvt[n - 1] = n;
        __syncwarp();
        if (A(n, n) == 0.0) info = n;
        return info;
    }

    // DGESL with JOB = 0 (dvode.f:3932-4061): A x = b in place (b 0-based)
    __device__ void gesl(double* b) {
        for (int k = 1; k <= n - 1; ++k) {
            const int l = w.ipvt[k - 1];
            const double t = b[l - 1];
            __syncwarp();
            if (lane == 0 && l != k) {
                b[l - 1] = b[k - 1];
                b[k - 1] = t;
            }
            __syncwarp();
            for (int i = k + 1 + lane; i <= n; i += 32) b[i - 1] = b[i - 1] + t * A(i, k);
            __syncwarp();
        }
        for (int kb = 1; kb <= n; ++kb) {
            const int k = n + 1 - kb;
            if (lane == 0) b[k - 1] = b[k - 1] / A(k, k);
            __syncwarp();
            const double t = -b[k - 1];
            for (int i = 1 + lane; i <= k - 1; i += 32) b[i - 1] = b[i - 1] + t * A(i, k);
            __syncwarp();
        }
    }

    // DVSET, METH 2 (dvode.f:2369-2567): scalars only
    __device__ void vset() {
        const double flotl = (double)s.l;
        const int nq = s.nq, nqm1 = nq - 1, nqm2 = nq - 2;
        double* el = s.el;
        for (int i = 3; i <= s.l; ++i) el[i] = 0.0;
        el[1] = 1.0;
        el[2] = 1.0;
        double alph0 = -1.0, ahatn0 = -1.0, hsum = s.h, rxi = 1.0, rxis = 1.0;
        if (nq != 1) {
            for (int j = 1; j <= nqm2; ++j) {
                hsum = hsum + s.tau[j];
                rxi = s.h / hsum;
                const int jp1 = j + 1;
                alph0 = alph0 - 1.0 / (double)jp1;
                for (int iback = 1; iback <= jp1; ++iback) {
                    const int i = (j + 3) - iback;
                    el[i] = el[i] + el[i - 1] * rxi;
                }
            }
            alph0 = alph0 - 1.0 / (double)nq;
            rxis = -el[2] - alph0;
            hsum = hsum + s.tau[nqm1];
            rxi = s.h / hsum;
            ahatn0 = -el[2] - rxi;
            for (int iback = 1; iback <= nq; ++iback) {
                const int i = (nq + 2) - iback;
                el[i] = el[i] + el[i - 1] * rxis;
            }
        }
        const double t1 = 1.0 - ahatn0 + alph0;
        const double t2 = 1.0 + (double)nq * t1;
        s.tq[2] = fabs(alph0 * t2 / t1);
        s.tq[5] = fabs(t2 / (el[s.l] * rxi / rxis));
        if (s.nqwait == 1) {
            const double cnqm1 = rxis / el[s.l];
            const double t3 = alph0 + 1.0 / (double)nq;
            const double t4 = ahatn0 + rxi;
            double elp = t3 / (1.0 - t4 + t3);
            s.tq[1] = fabs(elp / cnqm1);
            hsum = hsum + s.tau[nq];
            rxi = s.h / hsum;
            const double t5 = alph0 - 1.0 / (double)(nq + 1);
            const double t6 = ahatn0 - rxi;
            elp = t2 / (1.0 - t6 + t5);
            s.tq[3] = fabs(elp * rxi * (flotl + 1.0) * t5);
        }
        s.tq[4] = 0.1 * s.tq[2];  // CORTES
    }

    // DVJUST, METH 2 (dvode.f:2568-2727)
    __device__ void vjust(int iord) {
        if (s.nq == 2 && iord != 1) return;
        const int nqm1 = s.nq - 1, nqm2 = s.nq - 2;
        double* el = s.el;
        if (iord != 1) {
            for (int j = 1; j <= s.lmax; ++j) el[j] = 0.0;
            el[3] = 1.0;
            double hsum = 0.0;
            for (int j = 1; j <= nqm2; ++j) {
                hsum = hsum + s.tau[j];
                const double xi = hsum / s.hscal;
                const int jp1 = j + 1;
                for (int iback = 1; iback <= jp1; ++iback) {
                    const int i = (j + 4) - iback;
                    el[i] = el[i] * xi + el[i - 1];
                }
            }
            for (int r = 1 + lane; r <= n; r += 32)
                for (int j = 3; j <= s.nq; ++j) YH(r, j) = YH(r, j) - YH(r, s.l) * el[j];
            __syncwarp();
            return;
        }
        for (int j = 1; j <= s.lmax; ++j) el[j] = 0.0;
        el[3] = 1.0;
        double alph0 = -1.0, alph1 = 1.0, prod = 1.0, xiold = 1.0, hsum = s.hscal;
        if (s.nq != 1) {
            for (int j = 1; j <= nqm1; ++j) {
                const int jp1 = j + 1;
                hsum = hsum + s.tau[jp1];
                const double xi = hsum / s.hscal;
                prod = prod * xi;
                alph0 = alph0 - 1.0 / (double)jp1;
                alph1 = alph1 + 1.0 / xi;
                for (int iback = 1; iback <= jp1; ++iback) {
                    const int i = (j + 4) - iback;
                    el[i] = el[i] * xiold + el[i - 1];
                }
                xiold = xi;
            }
        }
        const double t1 = (-alph0 - alph1) / prod;
        const int lp1 = s.l + 1, nqp1 = s.nq + 1;
        for (int r = 1 + lane; r <= n; r += 32) {
            YH(r, lp1) = t1 * YH(r, s.lmax);
            for (int j = 3; j <= nqp1; ++j) YH(r, j) = YH(r, j) + el[j] * YH(r, lp1);  // DAXPY
        }
        __syncwarp();
    }

    // DVJAC, MITER 1 with JSV 1 (dvode.f:2957-3234); returns IERPJ
    __device__ int vjac(const double* y) {
        const double hrl1 = s.h * s.rl1;
        int jok = 1;
        if (s.nst == 0 || s.nst > s.nslj + s.msbj) jok = -1;
        if (s.icf == 1 && s.drc < s.ccmxj) jok = -1;
        if (s.icf == 2) jok = -1;
        const int lenp = n * n;
        if (jok == -1) {
            ++s.nje;
            s.nslj = s.nst;
            s.jcur = 1;
            jac(y);  // every element of the matrix is written
            for (int i = lane; i < lenp; i += 32) w.js[i] = w.wm[i];
        } else {
            s.jcur = 0;
            for (int i = lane; i < lenp; i += 32) w.wm[i] = w.js[i];
        }
        const double con = -hrl1;
        for (int i = lane; i < lenp; i += 32) w.wm[i] = con * w.wm[i];
        __syncwarp();
        for (int i = 1 + lane; i <= n; i += 32) A(i, i) = A(i, i) + 1.0;
        __syncwarp();
        ++s.nlu;
        return gefa() != 0 ? 1 : 0;
    }

    // DVNLSD, METH 2 / MITER 1 (dvode.f:2728-2956); corrector iterate in w.dy
    __device__ void vnlsd(int& nflag) {
        const double CCMAX = 0.3, CRDOWN = 0.3, RDIV = 2.0;
        const int MAXCOR = 3, MSBP = 20;
        double* y = w.dy;
        if (s.jstart == 0) s.nslp = 0;
        if (nflag == 0) s.icf = 0;
        if (nflag == -2) s.ipup = 1;
        if (s.jstart == 0 || s.jstart == -1) s.ipup = 1;
        s.drc = fabs(s.rc - 1.0);
        if (s.drc > CCMAX || s.nst >= s.nslp + MSBP) s.ipup = 1;
        for (;;) {  // 220
            int m = 0;
            double delp = 0.0, del = 0.0;
            for (int i = 1 + lane; i <= n; i += 32) y[i - 1] = YH(i, 1);
            __syncwarp();
            f(y, w.savf);
            ++s.nfe;
            if (s.ipup > 0) {
                const int ierpj = vjac(y);
                s.ipup = 0;
                s.rc = 1.0;
                s.drc = 0.0;
                s.crate = 1.0;
                s.nslp = s.nst;
                if (ierpj != 0) {  // 430
                    nflag = -1;
                    s.icf = 2;
                    s.ipup = 1;
                    return;
                }
            }
            for (int i = lane; i < n; i += 32) w.acor[i] = 0.0;
            __syncwarp();
            bool retry = false;
            for (;;) {  // 270 / 350
                for (int i = 1 + lane; i <= n; i += 32)
                    y[i - 1] = (s.rl1 * s.h) * w.savf[i - 1] - (s.rl1 * YH(i, 2) + w.acor[i - 1]);
                __syncwarp();
                gesl(y);
                ++s.nni;
                if (s.rc != 1.0) {
                    const double cscale = 2.0 / (1.0 + s.rc);
                    for (int i = lane; i < n; i += 32) y[i] = cscale * y[i];
                    __syncwarp();
                }
                del = vnorm(y);
                for (int i = 1 + lane; i <= n; i += 32) {
                    w.acor[i - 1] = w.acor[i - 1] + y[i - 1];
                    y[i - 1] = YH(i, 1) + w.acor[i - 1];
                }
                __syncwarp();
                if (m != 0) s.crate = fmax2(CRDOWN * s.crate, del / delp);  // 400
                const double dcon = del * fmin2(1.0, s.crate) / s.tq[4];
                if (dcon <= 1.0) {  // 450
                    nflag = 0;
                    s.jcur = 0;
                    s.icf = 0;
                    if (m == 0) s.acnrm = del;
                    if (m > 0) s.acnrm = vnorm(w.acor);
                    return;
                }
                ++m;
                if (m == MAXCOR || (m >= 2 && del > RDIV * delp)) {  // 410
                    if (s.jcur == 1) {  // 430
                        nflag = -1;
                        s.icf = 2;
                        s.ipup = 1;
                        return;
                    }
                    s.icf = 1;
                    s.ipup = 1;
                    retry = true;
                    break;
                }
                delp = del;
                f(y, w.savf);
                ++s.nfe;
            }
            if (!retry) return;
        }
    }

    // YH1(i) +/-= YH1(i + LDYH) over the Pascal triangle of DVSTEP (prediction
    // at 200, its undoing at 430 / 500): per row, columns in the reference's order
    __device__ void pascal(double sgn) {
        for (int r = 1 + lane; r <= n; r += 32)
            for (int jb = 1; jb <= s.nq; ++jb)
                for (int c = s.nq + 1 - jb; c <= s.nq; ++c) YH(r, c) = YH(r, c) + sgn * YH(r, c + 1);
        __syncwarp();
    }

    // DVSTEP (dvode.f:1934-2368)
    __device__ void vstep() {
        const int KFC = -3, KFH = -7, MXNCF = 10;
        const double ADDON = 1.0e-6, BIAS1 = 6.0, BIAS2 = 6.0, BIAS3 = 10.0, ETACF = 0.25, ETAMIN = 0.1, ETAMXF = 0.2,
                     ETAMX1 = 1.0e4, ETAMX2 = 10.0, ETAMX3 = 10.0, ONEPSM = 1.00001, THRESH = 1.5;
        s.kflag = 0;
        const double told = s.tn;
        int ncf = 0;
        s.jcur = 0;
        int nflag = 0;
        int go;  // 0: 200, 1: 20 (JSTART > 0), 2: 150
        if (s.jstart > 0) {
            go = 1;
        } else {  // JSTART = 0
            s.lmax = MAXORD + 1;
            s.nq = 1;
            s.l = 2;
            s.nqnyh = s.nq * n;
            s.tau[1] = s.h;
            s.prl1 = 1.0;
            s.rc = 0.0;
            s.etamax = ETAMX1;
            s.nqwait = 2;
            s.hscal = s.h;
            go = 0;
        }
        for (;;) {
            if (go == 1) {  // 20 / 50
                if (s.kuth == 1) {
                    s.eta = fmin2(s.eta, s.h / s.hscal);
                    s.newh = 1;
                }
                if (s.newh == 0) {
                    go = 0;
                    continue;
                }
                if (s.newq < s.nq) {
                    vjust(-1);
                    s.nq = s.newq;
                    s.l = s.nq + 1;
                    s.nqwait = s.l;
                } else if (s.newq > s.nq) {
                    vjust(1);
                    s.nq = s.newq;
                    s.l = s.nq + 1;
                    s.nqwait = s.l;
                }
                go = 2;
                continue;
            }
            if (go == 2) {  // 150: rescale YH by eta
                for (int r = 1 + lane; r <= n; r += 32) {
                    double rr = 1.0;
                    for (int j = 2; j <= s.l; ++j) {
                        rr = rr * s.eta;
                        YH(r, j) = rr * YH(r, j);
                    }
                }
                __syncwarp();
                s.h = s.hscal * s.eta;
                s.hscal = s.h;
                s.rc = s.rc * s.eta;
                s.nqnyh = s.nq * n;
                go = 0;
                continue;
            }
            // 200: predict
            s.tn = s.tn + s.h;
            pascal(1.0);
            vset();
            s.rl1 = 1.0 / s.el[2];
            s.rc = s.rc * (s.rl1 / s.prl1);
            s.prl1 = s.rl1;
            vnlsd(nflag);
            if (nflag != 0) {
                ++ncf;
                ++s.ncfn;
                s.etamax = 1.0;
                s.tn = told;
                pascal(-1.0);
                if (nflag < -1) {  // 680
                    if (nflag == -2) s.kflag = -3;
                    if (nflag == -3) s.kflag = -4;
                    s.jstart = 1;
                    return;
                }
                if (fabs(s.h) <= s.hmin * ONEPSM || ncf == MXNCF) {  // 670
                    s.kflag = -2;
                    s.jstart = 1;
                    return;
                }
                s.eta = ETACF;
                s.eta = fmax2(s.eta, s.hmin / fabs(s.h));
                nflag = -1;
                go = 2;
                continue;
            }
            // 450: local error test
            const double dsm = s.acnrm / s.tq[2];
            if (dsm > 1.0) {  // 500
                s.kflag = s.kflag - 1;
                ++s.netf;
                nflag = -2;
                s.tn = told;
                pascal(-1.0);
                if (fabs(s.h) <= s.hmin * ONEPSM) {  // 660
                    s.kflag = -1;
                    s.jstart = 1;
                    return;
                }
                s.etamax = 1.0;
                if (s.kflag > KFC) {
                    const double flotl = (double)s.l;
                    s.eta = 1.0 / (pow(BIAS2 * dsm, 1.0 / flotl) + ADDON);
                    s.eta = fmax2(fmax2(s.eta, s.hmin / fabs(s.h)), ETAMIN);
                    if (s.kflag <= -2 && s.eta > ETAMXF) s.eta = ETAMXF;
                    go = 2;
                    continue;
                }
                if (s.kflag == KFH) {  // 530 -> 660
                    s.kflag = -1;
                    s.jstart = 1;
                    return;
                }
                if (s.nq != 1) {
                    s.eta = fmax2(ETAMIN, s.hmin / fabs(s.h));
                    vjust(-1);
                    s.l = s.nq;
                    s.nq = s.nq - 1;
                    s.nqwait = s.l;
                    go = 2;
                    continue;
                }
                // 540: order 1 again from the last accepted state; Y is the
                // corrector's last iterate, as in the reference
                s.eta = fmax2(ETAMIN, s.hmin / fabs(s.h));
                s.h = s.h * s.eta;
                s.hscal = s.h;
                s.tau[1] = s.h;
                f(w.dy, w.savf);
                ++s.nfe;
                for (int i = 1 + lane; i <= n; i += 32) YH(i, 2) = s.h * w.savf[i - 1];
                __syncwarp();
                s.nqwait = 10;
                go = 0;
                continue;
            }
            // the step is accepted
            s.kflag = 0;
            ++s.nst;
            s.hu = s.h;
            s.nqu = s.nq;
            for (int iback = 1; iback <= s.nq; ++iback) {
                const int i = s.l - iback;
                s.tau[i + 1] = s.tau[i];
            }
            s.tau[1] = s.h;
            for (int r = 1 + lane; r <= n; r += 32)
                for (int j = 1; j <= s.l; ++j) YH(r, j) = YH(r, j) + s.el[j] * w.acor[r - 1];  // DAXPY
            __syncwarp();
            --s.nqwait;
            if (s.l != s.lmax && s.nqwait == 1) {
                for (int i = 1 + lane; i <= n; i += 32) YH(i, s.lmax) = w.acor[i - 1];
                __syncwarp();
                s.conp = s.tq[5];
            }
            if (s.etamax == 1.0) {  // 490
                if (s.nqwait < 2) s.nqwait = 2;
                s.newq = s.nq;
                s.newh = 0;
                s.eta = 1.0;
                s.hnew = s.h;
            } else {  // 560: step and order for the next step
                const double flotl = (double)s.l;
                s.etaq = 1.0 / (pow(BIAS2 * dsm, 1.0 / flotl) + ADDON);
                if (s.nqwait != 0) {  // 600
                    s.eta = s.etaq;
                    s.newq = s.nq;
                } else {
                    s.nqwait = 2;
                    s.etaqm1 = 0.0;
                    if (s.nq != 1) {
                        const double ddn = vnorm(&YH(1, s.l)) / s.tq[1];
                        s.etaqm1 = 1.0 / (pow(BIAS1 * ddn, 1.0 / (flotl - 1.0)) + ADDON);
                    }
                    double etaqp1 = 0.0;  // 570
                    if (s.l != s.lmax) {
                        const double cnquot = (s.tq[5] / s.conp) * ipow(s.h / s.tau[2], s.l);
                        for (int i = 1 + lane; i <= n; i += 32) w.savf[i - 1] = w.acor[i - 1] - cnquot * YH(i, s.lmax);
                        __syncwarp();
                        const double dup = vnorm(w.savf) / s.tq[3];
                        etaqp1 = 1.0 / (pow(BIAS3 * dup, 1.0 / (flotl + 1.0)) + ADDON);
                    }
                    // 580 / 590
                    int pick;  // 0: q (600), -1: q-1 (610), +1: q+1 (620)
                    if (s.etaq >= etaqp1)
                        pick = s.etaq < s.etaqm1 ? -1 : 0;
                    else
                        pick = etaqp1 > s.etaqm1 ? 1 : -1;
                    if (pick == 0) {
                        s.eta = s.etaq;
                        s.newq = s.nq;
                    } else if (pick == -1) {
                        s.eta = s.etaqm1;
                        s.newq = s.nq - 1;
                    } else {
                        s.eta = etaqp1;
                        s.newq = s.nq + 1;
                        for (int i = 1 + lane; i <= n; i += 32) YH(i, s.lmax) = w.acor[i - 1];
                        __syncwarp();
                    }
                }
                // 630
                if (s.eta < THRESH || s.etamax == 1.0) {  // 640
                    s.newq = s.nq;
                    s.newh = 0;
                    s.eta = 1.0;
                    s.hnew = s.h;
                } else {
                    s.eta = fmin2(s.eta, s.etamax);
                    s.eta = s.eta / fmax2(1.0, fabs(s.h) * s.hmxi * s.eta);
                    s.newh = 1;
                    s.hnew = s.h * s.eta;
                }
            }
            // 690 / 700
            s.etamax = ETAMX3;
            if (s.nst <= 10) s.etamax = ETAMX2;
            const double r = 1.0 / s.tq[2];
            for (int i = lane; i < n; i += 32) w.acor[i] = r * w.acor[i];
            __syncwarp();
            s.jstart = 1;
            return;
        }
    }

    // DVHIN (dvode.f:1673-1810) with Y0 = YH(., 1), YDOT = YH(., 2), Y = w.dy
    // and TEMP = w.acor; returns IER
    __device__ int vhin(double t0, double tout, double atol, double& h0, int& niter) {
        const double* y0 = w.yh;
        const double* ydot = w.yh + n;
        double* y = w.dy;
        double* temp = w.acor;
        niter = 0;
        const double tdist = fabs(tout - t0);
        const double tround = UROUND * fmax2(fabs(t0), fabs(tout));
        if (tdist < 2.0 * tround) return -1;
        const double hlb = 100.0 * tround;
        double hub = 0.1 * tdist;
        if (lane == 0)
            for (int i = 0; i < n; ++i) {
                const double delyi = 0.1 * fabs(y0[i]) + atol;
                const double afi = fabs(ydot[i]);
                if (afi * hub > delyi) hub = delyi / afi;
            }
        hub = __shfl_sync(0xffffffffu, hub, 0);
        int iter = 0;
        double hg = sqrt(hlb * hub);
        if (hub < hlb) {
            h0 = hg;
        } else {
            double hnew;
            for (;;) {  // 50
                const double h = copysign(hg, tout - t0);
                for (int i = lane; i < n; i += 32) y[i] = y0[i] + h * ydot[i];
                __syncwarp();
                f(y, temp);
                for (int i = lane; i < n; i += 32) temp[i] = (temp[i] - ydot[i]) / h;
                __syncwarp();
                const double yddnrm = vnorm(temp);
                if (yddnrm * hub * hub > 2.0)
                    hnew = sqrt(2.0 / yddnrm);
                else
                    hnew = sqrt(hg * hub);
                ++iter;
                if (iter >= 4) break;
                const double hrat = hnew / hg;
                if (hrat > 0.5 && hrat < 2.0) break;
                if (iter >= 2 && hnew > 2.0 * hg) {
                    hnew = hg;
                    break;
                }
                hg = hnew;
            }
            h0 = hnew * 0.5;  // 80
            if (h0 < hlb) h0 = hlb;
            if (h0 > hub) h0 = hub;
        }
        h0 = copysign(h0, tout - t0);  // 90
        niter = iter;
        return 0;
    }

    // DVINDY with K = 0 (dvode.f:1811-1933): YH interpolated at t into dky
    __device__ int vindy(double t, double* dky) {
        const double tfuzz = 100.0 * UROUND * copysign(fabs(s.tn) + fabs(s.hu), s.hu);
        const double tp = s.tn - s.hu - tfuzz;
        const double tn1 = s.tn + tfuzz;
        if ((t - tp) * (t - tn1) > 0.0) return -2;
        const double sv = (t - s.tn) / s.h;
        for (int i = 1 + lane; i <= n; i += 32) {
            double d = 1.0 * YH(i, s.l);
            for (int jb = 1; jb <= s.nq; ++jb) {
                const int jp1 = s.nq - jb + 1;
                d = 1.0 * YH(i, jp1) + sv * d;
            }
            dky[i - 1] = d;
        }
        __syncwarp();
        return 0;
    }

    // DVODE with ISTATE = 1, ITASK = 1 (dvode.f:2-1672).  y (shared, n values)
    // holds the state at t on entry; on return ISTATE: 2 with y at tout and
    // t = tout, or < 0 with y and t of the last accepted step (-1: MXSTEP steps;
    // -2 too much accuracy; -3 illegal input; -4 error test failures; -5
    // convergence failures; -6 a zero error weight).  accepted(tn) runs after
    // every accepted step, with YH(., 1) the new state.
    template <typename ACC>
    __device__ int solve(double* y, double& t, double tout, double rtol, double atol, ACC& accepted) {
        if (tout == t) return 1;
        s.init = 0;
        s.hmxi = 0.0;
        s.hmin = 0.0;
        double h0 = 0.0;
        s.tn = t;
        s.jstart = 0;
        s.ccmxj = 0.2;
        s.msbj = 50;
        s.nst = s.nje = s.nni = s.ncfn = s.netf = s.nlu = s.nslj = 0;
        const int nslast = 0;
        s.hu = 0.0;
        s.nqu = 0;
        f(y, &YH(1, 2));
        s.nfe = 1;
        for (int i = lane; i < n; i += 32) w.yh[i] = y[i];
        __syncwarp();
        s.nq = 1;
        s.h = 1.0;
        if (!ewset(rtol, atol)) return -3;
        int niter = 0;
        if (vhin(t, tout, atol, h0, niter) != 0) return -3;
        s.nfe += niter;
        s.h = h0;
        for (int i = lane; i < n; i += 32) w.yh[n + i] = h0 * w.yh[n + i];
        __syncwarp();
        bool first = true;
        int istate = 0;
        for (;;) {
            if (!first) {  // 250
                if (s.nst - nslast >= MXSTEP) {
                    istate = -1;
                    break;
                }
                if (!ewset(rtol, atol)) {
                    istate = -6;
                    break;
                }
            }
            // 270
            const double tolsf = UROUND * vnorm(w.yh);
            if (tolsf > 1.0) {
                istate = s.nst == 0 ? -3 : -2;
                break;
            }
            first = false;
            vstep();
            if (s.kflag == -1) {
                istate = -4;
                break;
            }
            if (s.kflag < 0) {  // -2; -3 and -4 are not reached with MITER 1
                istate = -5;
                break;
            }
            s.init = 1;
            s.kuth = 0;
            accepted(s.tn);
            if ((s.tn - tout) * s.h < 0.0) continue;  // 310 -> 250
            if (vindy(tout, y) != 0) return -3;
            t = tout;
            return 2;
        }
        // 580: the last accepted state
        for (int i = lane; i < n; i += 32) y[i] = w.yh[i];
        __syncwarp();
        t = s.tn;
        return istate;
    }
};

}  // namespace dvw

// The rest of a CHEMEQ2 interval, sub_chem.f90:1755-1775: DVODE from (tt, y)
// to tout with control_chem.inp's rtol and atol; ISTATE = -1 calls it again
// from where it stopped, at most max_recalc times; any other failure is
// SCFD_E_CHEM.  y (shared memory, ns + 1 values) is the state in and out.
// accepted(t) runs after every accepted step with w.yh[0..ns] the state.
template <typename ACC>
__device__ int warp_dvode_rest(const DevChem& ch, WarpMem& w, double* y, double tt, double tout, long long& evals,
                               int lane, ACC& accepted) {
    dvw::Warp dv(ch, w, lane, evals);
    double t = tt;
    int nrecalc = 0;
    for (;;) {
        const int istate = dv.solve(y, t, tout, ch.rtol, ch.atol, accepted);
        if (istate > 0) return 0;
        if (istate == -1 && ++nrecalc <= dvw::MAX_RECALC) continue;
        return SCFD_E_CHEM;
    }
}

}  // namespace scfd
