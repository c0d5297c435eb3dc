// chem_dev.cuh -- device restatement of the UV source terms Fex_var, Fex and
// their exact Jacobian Jex (store/therm_lib/chemkin/uvhp/uv/FJ.f90:152-709) and
// of one CHEMEQ2 attempt (store/therm_lib/chemkin/core/sub_chem.f90:1714-1819),
// one thread each; shared by the flow chemistry kernel and the batched 0-D
// reactors (whose one-warp versions and DVODE are in chem_warp.cuh).
#pragma once

#include "div_pos.cuh"
#include "scfd_internal.h"

namespace scfd {

// Per-evaluation constants of Fex_var (FJ.f90:301-453) at temperature T.
struct FexPre {
    double T, logT, Tinv, logPRT, sn, logsn;
    double cmurt[7], chrt[7], ccpr[7];
};

__device__ inline void fex_pre(FexPre& f, double T, double sn) {
    const double pst = 1.01325e6, Ru = 8.3144621e7;
    f.T = T;
    f.logT = log(T);
    f.Tinv = 1.0 / T;
    f.logPRT = log(pst / Ru) - f.logT;
    f.sn = sn;
    f.logsn = log(sn);
    const double T2 = T * T, T3 = T2 * T, T4 = T3 * T;
    const double cm[7] = {1.0 - f.logT, -T / 2.0, -T2 / 6.0, -T3 / 12.0, -T4 / 20.0, f.Tinv, -1.0};
    const double ch[7] = {1.0, T / 2.0, T2 / 3.0, T3 / 4.0, T4 / 5.0, f.Tinv, 0.0};
    const double cp[7] = {1.0, T, T2, T3, T4, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        f.cmurt[i] = cm[i];
        f.chrt[i] = ch[i];
        f.ccpr[i] = cp[i];
    }
}

// mu0/RT, e/RT and cv/R of species j (NASA-7).
__device__ inline void species_thermo(const DevChem& ch, int j, const FexPre& f, double& mu, double& e, double& cv) {
    const double* cf = ch.coeff + (j * 2 + (f.T <= ch.tcommon[j] ? 0 : 1)) * 7;
    double t1 = 0.0, t2 = -1.0, t3 = -1.0;
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        const double c = cf[i];
        t1 = t1 + c * f.cmurt[i];
        t2 = t2 + c * f.chrt[i];
        t3 = t3 + c * f.ccpr[i];
    }
    mu = t1;
    e = t2;
    cv = t3;
}

// log of the third-body concentration of reaction i (reactions with exist_m).
__device__ inline double third_body_logM(const DevChem& ch, int i, const double* n, const FexPre& f) {
    const int ns = ch.ns;
    double tmp = f.sn;
    const int nm = ch.numm[i];
    for (int j = 0; j < nm; ++j) tmp = tmp + ch.men[i * ns + j] * n[ch.indm[i * ns + j]];
    return (tmp == f.sn) ? f.logsn : log(tmp);
}

// Forward and reverse rates of reaction i (rr = 0 for irreversible reactions);
// vlogM is the third-body term in effect for it.
__device__ inline void reaction_rates(const DevChem& ch, int i, const double* n, const FexPre& f, double vlogM,
                                      const double* vmu0rt, double& rf, double& rr) {
    const double loge210 = (double)0.43429448190325f;
    const double dd = 0.14;
    const int rs0 = ch.rstate[2 * i], rs1 = ch.rstate[2 * i + 1];
    const double* abe = ch.abe + 3 * i;
    double vlogk1 = abe[0] + abe[1] * f.logT - abe[2] * f.Tinv;
    double vlogk2 = 0.0;
    if (rs1 >= 4) vlogk1 = vlogk1 + vlogM;
    const int* ind = ch.indnu + 6 * i;
    const int nreac = ch.numnu[2 * i], nprod = ch.numnu[2 * i + 1];
    if (rs0 == 0) {
        const double* cabe = ch.cabe + 3 * i;
        if (rs1 == 1 || rs1 == 5) {
            vlogk2 = cabe[0] + cabe[1] * f.logT - cabe[2] * f.Tinv;
            if (rs1 == 5) vlogk2 = vlogk2 + vlogM;
        } else {
            if (rs1 == 2 || rs1 == 3) {
                const double logk0 = cabe[0] + cabe[1] * f.logT - cabe[2] * f.Tinv;
                const double logkinf = vlogk1;
                const double log_Pr = logk0 - logkinf + vlogM;
                const double Pr = exp(log_Pr);
                vlogk1 = logkinf + log(Pr / (1.0 + Pr));
                if (rs1 == 3) {
                    const double* tr = ch.troe + 4 * i;
                    const double aa = tr[0];
                    const double logFcent =
                        log10((1.0 - aa) * exp(-f.T * tr[1]) + aa * exp(-f.T * tr[2]) + exp(-f.Tinv * tr[3]));
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
            vlogk2 = vlogk1 - ch.snu[i] * f.logPRT + t1;
        }
    }
    double r = exp(vlogk1);
    for (int k = 0; k < nreac; ++k) r = r * n[ind[k]];
    rf = r;
    rr = 0.0;
    if (rs0 == 0) {
        r = exp(vlogk2);
        for (int k = 0; k < nprod; ++k) r = r * n[ind[3 + k]];
        rr = r;
    }
}

// Fex_var (FJ.f90:301-453): production (dndtp >= 0) and destruction (dndtm <= 0)
// rates of the species, and the positive / negative part of dT/dt at
// constant volume.  As in the reference, a reaction with a third-body flag but
// no third-body table uses the third-body term of the last reaction that had one.
__device__ inline void dev_fex_var(const DevChem& ch, const double* n, double* dndtp, double* dndtm) {
    const int ns = ch.ns;
    double sn = 0.0;
    for (int j = 0; j < ns; ++j) sn += n[j];
    FexPre f;
    fex_pre(f, n[ns], sn);
    double vmu0rt[kMaxSpecies], vert[kMaxSpecies], vcvr[kMaxSpecies];
    for (int j = 0; j < ns; ++j) {
        species_thermo(ch, j, f, vmu0rt[j], vert[j], vcvr[j]);
        dndtp[j] = 0.0;
        dndtm[j] = 0.0;
    }
    double vlogM = 0.0;
    for (int i = 0; i < ch.nr; ++i) {
        if (ch.exist_m[i]) vlogM = third_body_logM(ch, i, n, f);
        double rf, rr;
        reaction_rates(ch, i, n, f, vlogM, vmu0rt, rf, rr);
        const int* ind = ch.indnu + 6 * i;
        const int nreac = ch.numnu[2 * i], nprod = ch.numnu[2 * i + 1];
        for (int k = 0; k < nreac; ++k) dndtm[ind[k]] = dndtm[ind[k]] - rf;
        for (int k = 0; k < nprod; ++k) dndtp[ind[3 + k]] = dndtp[ind[3 + k]] + rf;
        if (ch.rstate[2 * i] == 0) {
            for (int k = 0; k < nreac; ++k) dndtp[ind[k]] = dndtp[ind[k]] + rr;
            for (int k = 0; k < nprod; ++k) dndtm[ind[3 + k]] = dndtm[ind[3 + k]] - rr;
        }
    }
    double de = 0.0, cv = 0.0;
    for (int j = 0; j < ns; ++j) {
        de = de + vert[j] * (dndtp[j] + dndtm[j]);
        cv = cv + vcvr[j] * n[j];
    }
    dndtp[ns] = fmax(-de * f.T / cv, 0.0);
    dndtm[ns] = fmin(-de * f.T / cv, 0.0);
}

// T-derivatives of mu0/RT and cv/R per NASA-7 coefficient (the cdmurt and
// cdcpr of set_coeff_more, store/therm_lib/chemkin/core/sub_chem.f90:91-150).
__device__ inline void jex_pre(double T, double* cdmurt, double* cdcpr) {
    const double Ti1 = 1.0 / T, Ti2 = Ti1 * Ti1, T2 = T * T, T3 = T2 * T;
    cdmurt[0] = -Ti1;
    cdmurt[1] = -1.0 / 2.0;
    cdmurt[2] = -T / 3.0;
    cdmurt[3] = -T2 / 4.0;
    cdmurt[4] = -T3 / 5.0;
    cdmurt[5] = -Ti2;
    cdmurt[6] = 0.0;
    cdcpr[0] = 0.0;
    cdcpr[1] = 1.0;
    cdcpr[2] = 2.0 * T;
    cdcpr[3] = 3.0 * T2;
    cdcpr[4] = 4.0 * T3;
    cdcpr[5] = 0.0;
    cdcpr[6] = 0.0;
}

// mu0/RT, its T-derivative, e/RT, cv/R and its T-derivative of species j (Jex).
__device__ inline void species_thermo_d(const DevChem& ch, int j, const FexPre& f, const double* cdmurt,
                                        const double* cdcpr, double& mu, double& dmu, double& e, double& cv,
                                        double& dcv) {
    const double* cf = ch.coeff + (j * 2 + (f.T <= ch.tcommon[j] ? 0 : 1)) * 7;
    double t1 = 0.0, t2 = 0.0, t3 = -1.0, t4 = -1.0, t5 = 0.0;
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        const double c = cf[i];
        t1 = t1 + c * f.cmurt[i];
        t2 = t2 + c * cdmurt[i];
        t3 = t3 + c * f.chrt[i];
        t4 = t4 + c * f.ccpr[i];
        t5 = t5 + c * cdcpr[i];
    }
    mu = t1;
    dmu = t2;
    e = t3;
    cv = t4;
    dcv = t5;
}

// One reaction of Jex (store/therm_lib/chemkin/uvhp/uv/FJ.f90:519-660): its
// net rate Dr and the derivatives drdn[0..ns] of Dr with respect to n_1..n_ns
// and T, before the third-body term (reaction_jac_m).  vlogM is the
// third-body term in effect; dlnkdlnM is set when this reaction has a
// third-body or fall-off rate, and otherwise keeps the value of an earlier
// reaction (the reference's variable lives across the reaction loop).
__device__ inline void reaction_jac(const DevChem& ch, int i, const double* n, const FexPre& f, double vlogM,
                                    const double* vmu0rt, const double* vdmu0rt, double& dlnkdlnM, double& Dr,
                                    double* drdn) {
    const double loge210 = (double)0.43429448190325f;
    const double dd = 0.14;
    const int ns = ch.ns;
    const int rs0 = ch.rstate[2 * i], rs1 = ch.rstate[2 * i + 1];
    const double* abe = ch.abe + 3 * i;
    double vlogk1 = abe[0] + abe[1] * f.logT - abe[2] * f.Tinv;
    double dlnkdT1 = (abe[1] + abe[2] * f.Tinv) * f.Tinv;
    double vlogk2 = 0.0, dlnkdT2 = 0.0;
    if (rs1 >= 4) {
        vlogk1 = vlogk1 + vlogM;
        dlnkdlnM = 1.0;
    }
    const int* ind = ch.indnu + 6 * i;
    const int nreac = ch.numnu[2 * i], nprod = ch.numnu[2 * i + 1];
    if (rs0 == 0) {
        const double* cabe = ch.cabe + 3 * i;
        if (rs1 == 1 || rs1 == 5) {
            vlogk2 = cabe[0] + cabe[1] * f.logT - cabe[2] * f.Tinv;
            dlnkdT2 = (cabe[1] + cabe[2] * f.Tinv) * f.Tinv;
            if (rs1 == 5) vlogk2 = vlogk2 + vlogM;
        } else {
            if (rs1 == 2 || rs1 == 3) {
                const double logk0 = cabe[0] + cabe[1] * f.logT - cabe[2] * f.Tinv;
                const double dlnk0dT = (cabe[1] + cabe[2] * f.Tinv) * f.Tinv;
                const double logkinf = vlogk1, dlnkinfdT = dlnkdT1;
                const double log_Pr = logk0 - logkinf + vlogM;
                const double Pr = exp(log_Pr);
                vlogk1 = logkinf + log(Pr / (1.0 + Pr));
                dlnkdT1 = (dlnk0dT + Pr * dlnkinfdT) / (1.0 + Pr);
                dlnkdlnM = 1.0 / (1.0 + Pr);
                if (rs1 == 3) {
                    const double* tr = ch.troe + 4 * i;
                    const double dlnPrdT = dlnk0dT - dlnkinfdT;
                    const double aa = tr[0];
                    const double e2 = exp(-f.T * tr[1]), e3 = exp(-f.T * tr[2]), e4 = exp(-tr[3] * f.Tinv);
                    const double Fcent = (1.0 - aa) * e2 + aa * e3 + e4;
                    const double dFcentdT = -(1.0 - aa) * tr[1] * e2 - aa * tr[2] * e3 + tr[3] * (f.Tinv * f.Tinv) * e4;
                    const double dlnFcentdT = dFcentdT / Fcent;
                    const double logFcent = log10(Fcent);
                    const double cc = -0.4 - 0.67 * logFcent;
                    const double nn = 0.75 - 1.27 * logFcent;
                    const double logPrc = log_Pr * loge210 + cc;
                    const double q = nn - dd * logPrc;
                    const double t1 = logPrc / q;
                    const double t2 = 1.0 / (1.0 + t1 * t1);
                    const double logF = t2 * logFcent;
                    vlogk1 = vlogk1 + logF / loge210;
                    dlnkdT1 = dlnkdT1 + t2 * (-2.0 * logF * t1 / (q * q) *
                                                  (nn * dlnPrdT + (1.27 * logPrc - 0.67 * nn) * dlnFcentdT) +
                                              dlnFcentdT);
                    dlnkdlnM = dlnkdlnM - 2.0 * t2 * logF * t1 / (q * q) * nn;
                }
            }
            double numu0rt = 0.0, nudmu0rt = 0.0;
            for (int k = 0; k < nreac; ++k) {
                numu0rt = numu0rt - vmu0rt[ind[k]];
                nudmu0rt = nudmu0rt - vdmu0rt[ind[k]];
            }
            for (int k = 0; k < nprod; ++k) {
                numu0rt = numu0rt + vmu0rt[ind[3 + k]];
                nudmu0rt = nudmu0rt + vdmu0rt[ind[3 + k]];
            }
            vlogk2 = vlogk1 - ch.snu[i] * f.logPRT + numu0rt;
            dlnkdT2 = dlnkdT1 + ch.snu[i] * f.Tinv + nudmu0rt;
        }
    }
    for (int k = 0; k < ns; ++k) drdn[k] = 0.0;
    double r = exp(vlogk1);
    for (int k = 0; k < nreac; ++k) r = r * n[ind[k]];
    Dr = r;
    drdn[ns] = dlnkdT1 * r;
    for (int k = 0; k < nreac; ++k) drdn[ind[k]] = drdn[ind[k]] + r / n[ind[k]];
    if (rs0 == 0) {
        r = exp(vlogk2);
        for (int k = 0; k < nprod; ++k) r = r * n[ind[3 + k]];
        Dr = Dr - r;
        drdn[ns] = drdn[ns] - r * dlnkdT2;
        for (int k = 0; k < nprod; ++k) drdn[ind[3 + k]] = drdn[ind[3 + k]] - r / n[ind[3 + k]];
    }
}

// Third-body part of Jex's derivatives of reaction i (FJ.f90:646-655), for
// reactions with exist_m: vM is the third-body concentration.
__device__ inline void reaction_jac_m(const DevChem& ch, int i, double Dr, double dlnkdlnM, double vM, double* drdn) {
    const int ns = ch.ns;
    const double t = Dr * dlnkdlnM / vM;
    for (int k = 0; k < ns; ++k) drdn[k] = drdn[k] + t;
    const int nm = ch.numm[i];
    for (int k = 0; k < nm; ++k) drdn[ch.indm[i * ns + k]] = drdn[ch.indm[i * ns + k]] + t * ch.men[i * ns + k];
}

// Fex (FJ.f90:152-300): net rates dn/dt of the species and dT/dt at constant
// volume (the right-hand side the reference hands DVODE).
__device__ inline void dev_fex(const DevChem& ch, const double* n, double* dndt) {
    const int ns = ch.ns;
    double sn = 0.0;
    for (int j = 0; j < ns; ++j) sn += n[j];
    FexPre f;
    fex_pre(f, n[ns], sn);
    double vmu0rt[kMaxSpecies], vert[kMaxSpecies], vcvr[kMaxSpecies];
    for (int j = 0; j < ns; ++j) {
        species_thermo(ch, j, f, vmu0rt[j], vert[j], vcvr[j]);
        dndt[j] = 0.0;
    }
    double vlogM = 0.0;
    for (int i = 0; i < ch.nr; ++i) {
        if (ch.exist_m[i]) vlogM = third_body_logM(ch, i, n, f);
        double rf, rr;
        reaction_rates(ch, i, n, f, vlogM, vmu0rt, rf, rr);
        const double Dr = ch.rstate[2 * i] == 0 ? rf - rr : rf;
        const int* ind = ch.indnu + 6 * i;
        const int nreac = ch.numnu[2 * i], nprod = ch.numnu[2 * i + 1];
        for (int k = 0; k < nreac; ++k) dndt[ind[k]] = dndt[ind[k]] - Dr;
        for (int k = 0; k < nprod; ++k) dndt[ind[3 + k]] = dndt[ind[3 + k]] + Dr;
    }
    double de = 0.0, cv = 0.0;
    for (int j = 0; j < ns; ++j) {
        de = de + vert[j] * dndt[j];
        cv = cv + vcvr[j] * n[j];
    }
    dndt[ns] = -de * f.T / cv;
}

// Jex (FJ.f90:454-709): the net rates dndt (as Fex) and their exact Jacobian
// J (row-major (ns+1) x (ns+1), J[i*(ns+1)+j] = d dndt_i / d n_j, T last).
__device__ inline void dev_jex(const DevChem& ch, const double* n, double* dndt, double* J) {
    const int ns = ch.ns, N = ns + 1;
    double sn = 0.0;
    for (int j = 0; j < ns; ++j) sn += n[j];
    sn = fmax(sn, 1e-300);
    FexPre f;
    fex_pre(f, n[ns], sn);
    double cdmurt[7], cdcpr[7];
    jex_pre(f.T, cdmurt, cdcpr);
    double vmu0rt[kMaxSpecies], vdmu0rt[kMaxSpecies], vert[kMaxSpecies], vcvr[kMaxSpecies], vdcvr[kMaxSpecies];
    for (int j = 0; j < ns; ++j) {
        species_thermo_d(ch, j, f, cdmurt, cdcpr, vmu0rt[j], vdmu0rt[j], vert[j], vcvr[j], vdcvr[j]);
        dndt[j] = 0.0;
        for (int i = 0; i < N; ++i) J[j * N + i] = 0.0;
    }
    double vM = 0.0, vlogM = 0.0, dlnkdlnM = 0.0;
    double drdn[kMaxSpecies + 1];
    for (int i = 0; i < ch.nr; ++i) {
        if (ch.exist_m[i]) {
            double tmp = sn;
            const int nm = ch.numm[i];
            for (int j = 0; j < nm; ++j) tmp = tmp + ch.men[i * ns + j] * n[ch.indm[i * ns + j]];
            vM = tmp;
            vlogM = (tmp == sn) ? f.logsn : log(tmp);
        }
        double Dr;
        reaction_jac(ch, i, n, f, vlogM, vmu0rt, vdmu0rt, dlnkdlnM, Dr, drdn);
        if (ch.exist_m[i]) reaction_jac_m(ch, i, Dr, dlnkdlnM, vM, drdn);
        const int* ind = ch.indnu + 6 * i;
        const int nreac = ch.numnu[2 * i], nprod = ch.numnu[2 * i + 1];
        for (int k = 0; k < nreac; ++k) {
            const int s = ind[k];
            dndt[s] = dndt[s] - Dr;
            for (int j = 0; j < N; ++j) J[s * N + j] = J[s * N + j] - drdn[j];
        }
        for (int k = 0; k < nprod; ++k) {
            const int s = ind[3 + k];
            dndt[s] = dndt[s] + Dr;
            for (int j = 0; j < N; ++j) J[s * N + j] = J[s * N + j] + drdn[j];
        }
    }
    double de = 0.0, cv = 0.0, dcv = 0.0, t1 = 0.0, t2 = 0.0;
    for (int j = 0; j < ns; ++j) {
        t1 = t1 + vert[j] * J[j * N + ns];
        de = de + vert[j] * dndt[j];
        dcv = dcv + vcvr[j] * dndt[j];
        cv = cv + vcvr[j] * n[j];
        t2 = t2 + vdcvr[j] * n[j];
    }
    dndt[ns] = -de * f.T / cv;
    J[ns * N + ns] = -(f.T * t1 + dcv + dndt[ns] * t2) / cv;
    for (int j = 0; j < ns; ++j) {
        double t = 0.0;
        for (int k = 0; k < ns; ++k) t = t + vert[k] * J[k * N + j];
        J[ns * N + j] = -(f.T * t + dndt[ns] * vcvr[j]) / cv;
    }
}

// Per-thread CHEMEQ2 state machine (sub_chem.f90:1714-1819).
struct Ceq {
    double y[kMaxSpecies + 1], y0[kMaxSpecies + 1];
    double tt, tout, dt, ratio, counter;
    int countersum, substeps;
    bool fell_back;   // the interval went to DVODE (sub_chem.f90:1755-1775)
    long long evals;  // source-term evaluations
};

// One attempt; returns 1 when the interval is done, 0 to continue, <0 error,
// 2 when 10 attempts are used up and the rest of the interval, from (tt, y0),
// goes to DVODE (sub_chem.f90:1755-1775).  The predictor's and corrector's
// quotients go through div_pos (branch-free, within one unit in the last place;
// k_chem 1.25 -> 1.18 ms per launch at 786 k cells): their denominators are
// y + 1e-300 with y >= 0 (a species' moles stay non-negative: p, q >= 0 and
// (1 - alp) p dt < 1 for every p dt >= 0), 360 + 60 v + 12 v^2 + v^3 with v >= 0,
// and 1 + alp p dt >= 1.
__device__ inline int ceq_attempt(const DevChem& ch, Ceq& s, double rtol, int max_substeps, long long& attempts) {
    const int ns = ch.ns;
    double yp[kMaxSpecies + 1], p[kMaxSpecies + 1], q[kMaxSpecies + 1], p0[kMaxSpecies + 1], q0[kMaxSpecies + 1];
    for (int i = 0; i <= ns; ++i) s.y[i] = s.y0[i];
    s.countersum += 1;
    if (s.countersum > 10) {
        s.fell_back = true;
        return 2;
    }
    ++attempts;
    s.evals += 2;
    const double dt = s.dt;
    dev_fex_var(ch, s.y, q0, p0);
    for (int i = 0; i < ns; ++i) {
        p0[i] = div_pos(-p0[i], s.y[i] + 1e-300);
        const double var = p0[i] * dt, var2 = var * var, var3 = var * var2;
        const double alp = div_pos(180.0 + 60.0 * var + 11.0 * var2 + var3, 360.0 + 60.0 * var + 12.0 * var2 + var3);
        yp[i] = s.y0[i] + div_pos(dt * (q0[i] - p0[i] * s.y0[i]), 1.0 + alp * p0[i] * dt);
    }
    yp[ns] = s.y0[ns] + dt * (q0[ns] + p0[ns]);
    double ratio = 1e300;
    dev_fex_var(ch, yp, q, p);
    for (int i = 0; i < ns; ++i) {
        p[i] = div_pos(-p[i], yp[i] + 1e-300);
        p[i] = 0.5 * (p0[i] + p[i]);
        const double var = p[i] * dt, var2 = var * var, var3 = var * var2;
        const double alp = div_pos(180.0 + 60.0 * var + 11.0 * var2 + var3, 360.0 + 60.0 * var + 12.0 * var2 + var3);
        q[i] = alp * q[i] + (1.0 - alp) * q0[i];
        s.y[i] = s.y0[i] + div_pos(dt * (q[i] - p[i] * s.y0[i]), 1.0 + alp * p[i] * dt);
        const double v2 = (s.y[i] * rtol + rtol * 1e-5) / fabs(s.y[i] - yp[i] + 1e-300);
        ratio = (v2 < ratio || v2 != v2) ? v2 : ratio;  // a NaN ratio rejects the attempt
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

}  // namespace scfd
