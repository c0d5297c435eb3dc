// CPU restatement of the CEA equilibrium path (test infrastructure: the
// checker of the CUDA kernel, never the product).
//
// Follows store/therm_lib/NASA/core:
//   cea              sub_chem.f90:1320-1651 (Newton on element potentials)
//   cea_hp, cea_tp   sub_chem.f90:1652-2248 (fixed p and h; fixed p and T)
//   initialize_cea   sub_chem.f90:1136-1287 (stream states, element lists, masks)
//   set_therm_data   sub_chem.f90:159-170   (YAc, element mass fractions)
//   LU               LU.f90:1-83            (pivoted LU, singular below 1e-30)
//   calc_vThrt / calc_vTcpr / calc_vTmurt / calc_vTmu / check_section_number
//                    func_chem.f90:42-155
// Indices are kept 1-based (arrays sized +1) so that each statement reads like
// the Fortran it restates; the reduced system of a one-stream cell is
// compressed to its element list exactly as sub_chem.f90:1456-1469 does.
// Entry points carry the orc_ prefix and the scfd_cea_* signatures; device
// pointers there are host pointers here and the stream argument is ignored.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../include/scfd_b200.h"

namespace {

const double Ru = 8.3144621, pst = 1e5, eps = 1e-9, initial_eps = 1e-5, Y_eps = 1e-6, TSIZE = 1e-11,
             TTSIZE = 1e-14;
constexpr int NSX = SCFD_CEA_MAX_SPECIES + 1, NEX = SCFD_CEA_MAX_ELEMENTS + 3;

struct Model {
    scfd_cea_data d;
    int ns, ne, nt;
    double co[NSX][SCFD_CEA_MAX_SECTIONS + 1][10];  // co(k,l,j) as co[j][l][k]
    double Ac[NEX][NSX], YAc[NEX][NSX], MW[NSX];
    double b0f[NEX], b0o[NEX], maskf[NSX], masko[NSX], maskbf[NEX], maskbo[NEX], Yfe[NEX], Yoe[NEX];
    int nef, neo, elistf[NEX], elisto[NEX], nelistf[NEX], nelisto[NEX];
    scfd_cea_info info;
    int64_t fails[2];
};

int check_section_number(const Model& m, int j, double T) {
    const scfd_cea_data& d = m.d;
    int num = -1;
    if (d.trange[j - 1][0][0] > T) {
        num = 1;
    } else {
        for (int l = 1; l <= d.nsec[j - 1]; ++l)
            if (d.trange[j - 1][l - 1][1] > T) {
                num = l;
                break;
            }
    }
    if (num == -1) num = d.nsec[j - 1];
    return num;
}

int check_section_number_trans(const Model& m, int i, double T) {
    const scfd_cea_data& d = m.d;
    int num = -1;
    if (d.trange_t[i - 1][0][0] > T) num = 1;
    for (int l = 1; l <= d.ntsec[i - 1]; ++l)
        if (d.trange_t[i - 1][l - 1][1] > T) {
            num = l;
            break;
        }
    if (num == -1) num = d.ntsec[i - 1];
    return num;
}

void calc_vThrt(double T, double logT, double* vT) {  // vT[1..9]
    double TT = 1.0 / (T * T);
    vT[1] = -TT;
    TT = TT * T;
    vT[2] = TT * logT;
    vT[8] = TT;
    TT = TT * T;
    vT[3] = TT;
    TT = TT * T;
    vT[4] = TT / 2.0;
    TT = TT * T;
    vT[5] = TT / 3.0;
    TT = TT * T;
    vT[6] = TT / 4.0;
    TT = TT * T;
    vT[7] = TT / 5.0;
    vT[9] = 0.0;
}
void calc_vTcpr(double T, double* vT) {
    double TT = 1.0 / (T * T);
    vT[1] = TT;
    TT = TT * T;
    vT[2] = TT;
    TT = TT * T;
    vT[3] = TT;
    TT = TT * T;
    vT[4] = TT;
    TT = TT * T;
    vT[5] = TT;
    TT = TT * T;
    vT[6] = TT;
    TT = TT * T;
    vT[7] = TT;
    vT[8] = 0.0;
    vT[9] = 0.0;
}
void calc_vTmurt(double T, double logT, double* vT) {
    double TT = 1.0 / (T * T);
    vT[1] = -TT / 2.0;
    TT = TT * T;
    vT[2] = TT * (1.0 + logT);
    vT[8] = TT;
    TT = TT * T;
    vT[3] = TT * (1.0 - logT);
    vT[9] = -TT;
    TT = TT * T;
    vT[4] = -TT / 2.0;
    TT = TT * T;
    vT[5] = -TT / 6.0;
    TT = TT * T;
    vT[6] = -TT / 12.0;
    TT = TT * T;
    vT[7] = -TT / 20.0;
}
void calc_vTmu(double T, double logT, double* vT) {
    const double TT = 1.0 / (T * T);
    vT[1] = logT;
    vT[2] = TT * T;
    vT[3] = TT;
    vT[4] = 1.0;
}
double dot9(const double* c, const double* v) {  // c[1..9], v[1..9]
    double s = 0.0;
    for (int k = 1; k <= 9; ++k) s = s + c[k] * v[k];
    return s;
}

// LU.f90: A(1:n,1:n) in A[i][j]; returns true when singular
bool LU(double A[NEX][NEX], double* b, double* x, int n) {
    for (int k = 1; k <= n; ++k) {
        double p = std::fabs(A[k][k]);
        int ip = k;
        for (int i = k + 1; i <= n; ++i) {
            const double dtemp = std::fabs(A[i][k]);
            if (p < dtemp) {
                p = dtemp;
                ip = i;
            }
        }
        if (p < 1e-30) return true;
        if (ip != k) {
            for (int i = 1; i <= n; ++i) {
                const double dtemp = A[k][i];
                A[k][i] = A[ip][i];
                A[ip][i] = dtemp;
            }
            const double dtemp = b[k];
            b[k] = b[ip];
            b[ip] = dtemp;
        }
        double dtemp = 1.0 / A[k][k];
        for (int i = k + 1; i <= n; ++i) A[i][k] = A[i][k] * dtemp;
        for (int j = k + 1; j <= n; ++j) {
            dtemp = A[k][j];
            for (int i = k + 1; i <= n; ++i) A[i][j] = A[i][j] - dtemp * A[i][k];
        }
    }
    double c[NEX] = {0};
    for (int k = 1; k <= n; ++k) {
        c[k] = b[k];
        for (int j = 1; j <= k - 1; ++j) c[k] = c[k] - A[k][j] * c[j];
    }
    x[n] = c[n] / A[n][n];
    for (int k = n - 1; k >= 1; --k) {
        x[k] = c[k];
        for (int j = k + 1; j <= n; ++j) x[k] = x[k] - A[k][j] * x[j];
        x[k] = x[k] / A[k][k];
    }
    return false;
}

struct CeaOut {
    double MWave, kappa, mu, DHi[3], H;
    double Yv[NSX], vhi[NSX];
    int counter;
    int status;  // 0, 1 = stopped at the iteration limit, 2 = singular twice
};

// cea (sub_chem.f90:1320-1651); n[1..ns]
void cea(const Model& M, double rho, const double* Y /*[1..2]*/, double E, double& T, double* n, CeaOut& o) {
    const int ns = M.ns, ne = M.ne, nt = M.nt;
    double b0[NEX] = {0}, b[NEX] = {0}, bd[NEX] = {0}, vpi[NEX] = {0};
    double vmurt[NSX], vert[NSX], Dlogn[NSX], logn[NSX];
    int sec_num[NSX];
    double Ad[NEX][NEX];
    int elist[NEX], nelist[NEX], nen = 0;
    bool REDUCEflag, debugflag = false;
    double vTmurt[10], vTcpr[10], vThrt[10], vTmu[5];
    o.status = 0;

    const double logrhoRu = std::log(rho * Ru / pst);
    for (int i = 1; i <= ne + 2; ++i) b0[i] = Y[1] * M.b0f[i] + Y[2] * M.b0o[i];
    double b0max = b0[1];
    for (int i = 2; i <= ne; ++i)
        if (b0[i] > b0max) b0max = b0[i];

    if (Y[1] < Y_eps) {
        REDUCEflag = true;
        nen = M.neo;
        std::memcpy(elist, M.elisto, sizeof(elist));
        std::memcpy(nelist, M.nelisto, sizeof(nelist));
        for (int j = 1; j <= ns; ++j) n[j] = n[j] * M.masko[j];
        for (int i = 1; i <= ne + 2; ++i) b0[i] = b0[i] * M.maskbo[i];
    } else if (Y[2] < Y_eps) {
        REDUCEflag = true;
        nen = M.nef;
        std::memcpy(elist, M.elistf, sizeof(elist));
        std::memcpy(nelist, M.nelistf, sizeof(nelist));
        for (int j = 1; j <= ns; ++j) n[j] = n[j] * M.maskf[j];
        for (int i = 1; i <= ne + 2; ++i) b0[i] = b0[i] * M.maskbf[i];
    } else {
        REDUCEflag = false;
    }

    double sn = 0.0;
    for (int j = 1; j <= ns; ++j) sn = sn + n[j];
    const double tinyn = TSIZE * sn;
    const double logtinyn = std::log(tinyn);
    const double tinytinyn = TTSIZE * sn;
    const double logtinytinyn = std::log(tinytinyn);

    double logT = std::log(T);
    calc_vThrt(T, logT, vThrt);
    for (int i = 1; i <= ne + 2; ++i) b[i] = 0.0;
    for (int j = 1; j <= ns; ++j) {
        vert[j] = 0.0;
        logn[j] = logtinyn;
    }
    for (int j = 1; j <= ns; ++j) {
        sec_num[j] = check_section_number(M, j, T);
        if (n[j] > tinyn) {
            vert[j] = dot9(M.co[j][sec_num[j]], vThrt) - 1.0;
            logn[j] = std::log(n[j]);
            for (int i = 1; i <= ne; ++i) b[i] = b[i] + M.Ac[i][j] * n[j];
            b[ne + 1] = b[ne + 1] + vert[j] * n[j];
        }
    }

    bool flag = true;
    for (int i = 1; i <= ne; ++i)
        if (b0[i] > eps && std::fabs(b0[i] - b[i]) > b0max * eps) flag = false;
    if (std::fabs(E - b[ne + 1] * Ru * T) > eps * std::fabs(E)) flag = false;

    int counter = 0;
    if (!flag) {
        counter = 1;
        for (;;) {
            b0[ne + 1] = E / (Ru * T);
            for (int i = 1; i <= ne; ++i) b[i] = 0.0;
            for (int i = 1; i <= ne + 2; ++i) bd[i] = b0[i];
            bd[ne + 1] = bd[ne + 1] - b[ne + 1];
            for (int i = 1; i <= ne + 2; ++i)
                for (int j = 1; j <= ne + 2; ++j) Ad[i][j] = 0.0;
            calc_vTmurt(T, logT, vTmurt);
            calc_vTcpr(T, vTcpr);
            for (int k = 1; k <= ns; ++k) {
                vmurt[k] = dot9(M.co[k][sec_num[k]], vTmurt) + logrhoRu + logT + logn[k];
                if (n[k] > tinyn) {
                    const double vmurtn = vmurt[k] * n[k];
                    for (int i = 1; i <= ne; ++i) {
                        for (int j = i; j <= ne; ++j) Ad[i][j] = Ad[i][j] + M.Ac[i][k] * M.Ac[j][k] * n[k];
                        Ad[i][ne + 1] = Ad[i][ne + 1] + M.Ac[i][k] * vert[k] * n[k];
                        b[i] = b[i] + M.Ac[i][k] * n[k];
                        bd[i] = bd[i] + M.Ac[i][k] * (vmurtn - n[k]);
                    }
                    Ad[ne + 1][ne + 1] =
                        Ad[ne + 1][ne + 1] + n[k] * (vert[k] * vert[k] + dot9(M.co[k][sec_num[k]], vTcpr) - 1.0);
                    bd[ne + 1] = bd[ne + 1] + vmurtn * vert[k];
                }
            }
            for (int i = 1; i <= ne + 1; ++i)
                for (int j = i; j <= ne + 1; ++j) Ad[j][i] = Ad[i][j];

            bool LUflag;
            if (REDUCEflag) {
                for (int i = 1; i <= nen; ++i) {
                    for (int j = 1; j <= nen; ++j) Ad[i][j] = Ad[elist[i]][elist[j]];
                    bd[i] = bd[elist[i]];
                }
                LUflag = LU(Ad, bd, vpi, nen);
                if (!LUflag) {
                    for (int i = nen; i >= 1; --i) vpi[elist[i]] = vpi[i];
                    for (int i = 1; i <= ne + 1 - nen; ++i) vpi[nelist[i]] = -1e300;
                }
            } else {
                LUflag = LU(Ad, bd, vpi, ne + 1);
            }

            if (LUflag) {
                if (debugflag) {  // the reference prints its state and stops
                    o.status = 2;
                    break;
                }
                debugflag = true;
                for (int j = 1; j <= ns; ++j) n[j] = n[j] + initial_eps;
                b[ne + 1] = 0.0;
                for (int j = 1; j <= ns; ++j) logn[j] = logtinytinyn;
                for (int j = 1; j <= ns; ++j) {
                    if (n[j] < tinytinyn)
                        n[j] = tinytinyn;
                    else
                        logn[j] = std::log(n[j]);
                    if (n[j] > tinyn) {
                        vert[j] = dot9(M.co[j][sec_num[j]], vThrt) - 1.0;
                        b[ne + 1] = b[ne + 1] + vert[j] * n[j];
                    }
                }
                sn = 0.0;
                for (int j = 1; j <= ns; ++j) sn = sn + n[j];
                continue;
            }

            const double DlogT = vpi[ne + 1];
            for (int j = 1; j <= ns; ++j) {
                double tmp = 0.0;
                for (int i = 1; i <= ne; ++i) tmp = tmp + M.Ac[i][j] * vpi[i];
                Dlogn[j] = -vmurt[j] + tmp + vert[j] * DlogT;
            }

            double lambda1 = 0.0, lambda2 = 1e300;
            const double logsn = std::log(sn);
            for (int j = 1; j <= ns; ++j) {
                if (logn[j] - logsn > -18.420681)
                    lambda1 = std::fmax(lambda1, std::fabs(Dlogn[j]));
                else if (Dlogn[j] > 0.0)
                    lambda2 = std::fmin(lambda2, std::fabs((-logn[j] + logsn - 9.2103404) / Dlogn[j]));
            }
            lambda1 = 2.0 / std::fmax(std::fmax(5.0 * std::fabs(DlogT), std::fabs(lambda1)), 2.0);
            const double omega_var = std::fmin(1.0, std::fmin(lambda1, lambda2));

            T = T * std::exp(omega_var * DlogT);
            logT = std::log(T);
            for (int j = 1; j <= ns; ++j) sec_num[j] = check_section_number(M, j, T);

            b[ne + 1] = 0.0;
            double Dnmax = 0.0;
            for (int j = 1; j <= ns; ++j) logn[j] = logtinytinyn;
            calc_vThrt(T, logT, vThrt);
            for (int j = 1; j <= ns; ++j) {
                n[j] = n[j] * std::exp(omega_var * Dlogn[j]);
                if (n[j] < tinytinyn)
                    n[j] = tinytinyn;
                else
                    logn[j] = std::log(n[j]);
                if (n[j] > tinyn) {
                    vert[j] = dot9(M.co[j][sec_num[j]], vThrt) - 1.0;
                    b[ne + 1] = b[ne + 1] + vert[j] * n[j];
                    const double tmp = std::fabs(Dlogn[j]) * n[j];
                    if (Dnmax < tmp) Dnmax = tmp;
                }
            }
            sn = 0.0;
            for (int j = 1; j <= ns; ++j) sn = sn + n[j];

            flag = true;
            if (std::fabs(Dnmax) > eps * sn) flag = false;
            for (int i = 1; i <= ne; ++i)
                if (b0[i] > eps && std::fabs(b0[i] - b[i]) > b0max * eps) flag = false;
            if (std::fabs(DlogT) > eps && std::fabs(E - b[ne + 1] * Ru * T) > eps * std::fabs(E)) flag = false;
            if (counter > 500) flag = true;
            if (flag) break;
            counter = counter + 1;
        }
        if (o.status == 0 && counter > 500) o.status = 1;
    }
    o.counter = counter;

    o.MWave = 1e3 / sn;
    calc_vTcpr(T, vTcpr);
    double kappa = 0.0;
    for (int i = 1; i <= ns; ++i)
        if (n[i] > tinyn) kappa = kappa + n[i] * dot9(M.co[i][sec_num[i]], vTcpr);
    kappa = kappa / (kappa - sn);
    o.kappa = kappa;

    double tmp = Ru * T;
    double vhe[NEX], MWd[NEX];
    for (int j = 1; j <= ne; ++j) vhe[j] = MWd[j] = 0.0;
    for (int i = 1; i <= ns; ++i) {
        double dh = 0.0;
        for (int j = 1; j <= 9; ++j) dh = dh + M.co[i][sec_num[i]][j] * vThrt[j];
        o.vhi[i] = tmp / M.MW[i] * dh * 1e3;
        const double tmp2 = tmp * n[i] * dh;
        for (int j = 1; j <= ne; ++j) {
            vhe[j] = vhe[j] + M.YAc[j][i] * tmp2;
            MWd[j] = MWd[j] + M.YAc[j][i] * n[i];
        }
    }
    o.DHi[1] = o.DHi[2] = 0.0;
    for (int i = 1; i <= ne; ++i) {
        tmp = 1.0 / (Y[1] * M.Yfe[i] + Y[2] * M.Yoe[i] + 1e-300) * (kappa * Ru * MWd[i] * T - (kappa - 1.0) * vhe[i]);
        o.DHi[1] = o.DHi[1] + M.Yfe[i] * tmp;
        o.DHi[2] = o.DHi[2] + M.Yoe[i] * tmp;
    }
    for (int i = 1; i <= ns; ++i) o.Yv[i] = n[i] * M.MW[i] * 1e-3;

    calc_vTmu(T, logT, vTmu);
    double muN[NSX];
    for (int i = 1; i <= nt; ++i) {
        const int sect = check_section_number_trans(M, i, T);
        const double* a = M.d.trans[i - 1][sect - 1];
        double s = 0.0;
        for (int k = 1; k <= 4; ++k) s = s + a[k - 1] * vTmu[k];
        muN[i] = std::exp(s);
    }
    double mu = 0.0;
    for (int i = 1; i <= nt; ++i) {
        double denom = 0.0;
        const double MWi = M.MW[M.d.tr2th[i - 1] + 1];
        for (int j = 1; j <= nt; ++j) {
            const double MWj = M.MW[M.d.tr2th[j - 1] + 1];
            const double f = 1.0 + std::sqrt(muN[i] / muN[j]) * std::pow(MWj / MWi, 0.25);
            const double phi = 0.25 * (f * f) * std::sqrt(2.0 * MWj / (MWi + MWj));
            denom = denom + n[M.d.tr2th[j - 1] + 1] * phi;
        }
        mu = mu + n[M.d.tr2th[i - 1] + 1] * muN[i] / denom;
    }
    o.mu = mu * 1e-7;
}

// The mixture properties that close cea_hp and cea_tp (sub_chem.f90:1902-1961,
// 2192-2247): MWave from sn, kappa, vhi = Ru 1e3 T / MW h/RT (and H for tp),
// Yv, Wilke mu.
void hp_tp_tail(const Model& M, double T, double logT, double sn, double tinyn, const int* sec_num, const double* n,
                bool with_H, CeaOut& o) {
    const int ns = M.ns, nt = M.nt;
    double vTcpr[10], vThrt[10], vTmu[5];
    o.MWave = 1e3 / sn;
    calc_vTcpr(T, vTcpr);
    double kappa = 0.0;
    for (int i = 1; i <= ns; ++i)
        if (n[i] > tinyn) kappa = kappa + n[i] * dot9(M.co[i][sec_num[i]], vTcpr);
    o.kappa = kappa / (kappa - sn);
    calc_vThrt(T, logT, vThrt);
    double H = 0.0;
    const double tmp = Ru * 1e3 * T;
    for (int i = 1; i <= ns; ++i) {
        double dh = 0.0;
        for (int j = 1; j <= 9; ++j) dh = dh + M.co[i][sec_num[i]][j] * vThrt[j];
        o.vhi[i] = tmp / M.MW[i] * dh;
        H = H + n[i] * dh;
    }
    o.H = with_H ? H * Ru * T : 0.0;
    for (int i = 1; i <= ns; ++i) o.Yv[i] = n[i] * M.MW[i] * 1e-3;
    calc_vTmu(T, logT, vTmu);
    double muN[NSX];
    for (int i = 1; i <= nt; ++i) {
        const int sect = check_section_number_trans(M, i, T);
        const double* a = M.d.trans[i - 1][sect - 1];
        double s = 0.0;
        for (int k = 1; k <= 4; ++k) s = s + a[k - 1] * vTmu[k];
        muN[i] = std::exp(s);
    }
    double mu = 0.0;
    for (int i = 1; i <= nt; ++i) {
        double denom = 0.0;
        const double MWi = M.MW[M.d.tr2th[i - 1] + 1];
        for (int j = 1; j <= nt; ++j) {
            const double MWj = M.MW[M.d.tr2th[j - 1] + 1];
            const double f = 1.0 + std::sqrt(muN[i] / muN[j]) * std::pow(MWj / MWi, 0.25);
            const double phi = 0.25 * (f * f) * std::sqrt(2.0 * MWj / (MWi + MWj));
            denom = denom + n[M.d.tr2th[j - 1] + 1] * phi;
        }
        mu = mu + n[M.d.tr2th[i - 1] + 1] * muN[i] / denom;
    }
    o.mu = mu * 1e-7;
    o.DHi[1] = o.DHi[2] = 0.0;
}

// cea_hp (sub_chem.f90:1652-1962): equilibrium at fixed p and h; the unknowns
// are pi_1..pi_ne, ln sn and ln T.  The reference's singular-matrix retry has
// no bound (it cycles past the iteration test); here it counts towards the
// same 500-iteration limit.
void cea_hp(const Model& M, double p, const double* Y, double H, double& T, double* n, CeaOut& o) {
    const int ns = M.ns, ne = M.ne;
    double b0[NEX] = {0}, b[NEX] = {0}, bd[NEX] = {0}, vpi[NEX] = {0};
    double vmurt[NSX], vhrt[NSX], Dlogn[NSX], logn[NSX];
    int sec_num[NSX];
    double Ad[NEX][NEX];
    int elist[NEX], nelist[NEX], nen = 0;
    bool REDUCEflag;
    double vTmurt[10], vTcpr[10], vThrt[10];
    o.status = 0;

    const double logP = std::log(p / pst);
    for (int i = 1; i <= ne + 2; ++i) b0[i] = Y[1] * M.b0f[i] + Y[2] * M.b0o[i];
    double b0max = b0[1];
    for (int i = 2; i <= ne; ++i)
        if (b0[i] > b0max) b0max = b0[i];
    double sn = 0.0;
    for (int j = 1; j <= ns; ++j) sn = sn + n[j];
    b0[ne + 1] = sn;

    if (Y[1] < Y_eps) {
        REDUCEflag = true;
        nen = M.neo + 1;
        std::memcpy(elist, M.elisto, sizeof(elist));
        std::memcpy(nelist, M.nelisto, sizeof(nelist));
        for (int j = 1; j <= ns; ++j) n[j] = n[j] * M.masko[j];
    } else if (Y[2] < Y_eps) {
        REDUCEflag = true;
        nen = M.nef + 1;
        std::memcpy(elist, M.elistf, sizeof(elist));
        std::memcpy(nelist, M.nelistf, sizeof(nelist));
        for (int j = 1; j <= ns; ++j) n[j] = n[j] * M.maskf[j];
    } else {
        REDUCEflag = false;
    }

    const double tinyn = TSIZE * sn;
    const double logtinyn = std::log(tinyn);
    const double tinytinyn = TTSIZE * sn;
    const double logtinytinyn = std::log(tinytinyn);

    double logT = std::log(T);
    calc_vThrt(T, logT, vThrt);
    for (int i = 1; i <= ne + 2; ++i) b[i] = 0.0;
    b[ne + 1] = sn;
    for (int j = 1; j <= ns; ++j) {
        vhrt[j] = 0.0;
        logn[j] = logtinyn;
    }
    for (int j = 1; j <= ns; ++j) {
        sec_num[j] = check_section_number(M, j, T);
        if (n[j] > tinyn) {
            vhrt[j] = dot9(M.co[j][sec_num[j]], vThrt);
            logn[j] = std::log(n[j]);
            for (int i = 1; i <= ne; ++i) b[i] = b[i] + M.Ac[i][j] * n[j];
            b[ne + 2] = b[ne + 2] + vhrt[j] * n[j];
        }
    }
    bool flag = true;
    for (int i = 1; i <= ne; ++i)
        if (b0[i] > eps && std::fabs(b0[i] - b[i]) > b0max * eps) flag = false;
    if (std::fabs(H - b[ne + 2] * Ru * T) > eps * std::fabs(H)) flag = false;

    int counter = 0;
    if (!flag) {
        counter = 1;
        for (;;) {
            b0[ne + 2] = H / (Ru * T);
            for (int i = 1; i <= ne; ++i) b[i] = 0.0;
            for (int i = 1; i <= ne + 2; ++i) bd[i] = b0[i];
            bd[ne + 1] = b0[ne + 1] - b[ne + 1];
            bd[ne + 2] = b0[ne + 2] - b[ne + 2];
            for (int i = 1; i <= ne + 2; ++i)
                for (int j = 1; j <= ne + 2; ++j) Ad[i][j] = 0.0;
            calc_vTmurt(T, logT, vTmurt);
            calc_vTcpr(T, vTcpr);
            for (int k = 1; k <= ns; ++k) {
                vmurt[k] = dot9(M.co[k][sec_num[k]], vTmurt) + logn[k] - std::log(b0[ne + 1]) + logP;
                if (n[k] > tinyn) {
                    const double vmurtn = vmurt[k] * n[k];
                    for (int i = 1; i <= ne; ++i) {
                        for (int j = i; j <= ne; ++j) Ad[i][j] = Ad[i][j] + M.Ac[i][k] * M.Ac[j][k] * n[k];
                        Ad[i][ne + 1] = Ad[i][ne + 1] + M.Ac[i][k] * n[k];
                        Ad[i][ne + 2] = Ad[i][ne + 2] + M.Ac[i][k] * vhrt[k] * n[k];
                        b[i] = b[i] + M.Ac[i][k] * n[k];
                        bd[i] = bd[i] + M.Ac[i][k] * (vmurtn - n[k]);
                    }
                    Ad[ne + 1][ne + 2] = Ad[ne + 1][ne + 2] + n[k] * vhrt[k];
                    Ad[ne + 2][ne + 2] =
                        Ad[ne + 2][ne + 2] + n[k] * (vhrt[k] * vhrt[k] + dot9(M.co[k][sec_num[k]], vTcpr));
                    bd[ne + 1] = bd[ne + 1] + vmurtn;
                    bd[ne + 2] = bd[ne + 2] + vmurtn * vhrt[k];
                }
            }
            Ad[ne + 1][ne + 1] = b[ne + 1] - b0[ne + 1];
            for (int i = 1; i <= ne + 2; ++i)
                for (int j = i + 1; j <= ne + 2; ++j) Ad[j][i] = Ad[i][j];

            bool LUflag;
            if (REDUCEflag) {
                for (int i = 1; i <= nen; ++i) {
                    for (int j = 1; j <= nen; ++j) Ad[i][j] = Ad[elist[i]][elist[j]];
                    bd[i] = bd[elist[i]];
                }
                LUflag = LU(Ad, bd, vpi, nen);
                if (!LUflag) {
                    for (int i = nen; i >= 1; --i) vpi[elist[i]] = vpi[i];
                    for (int i = 1; i <= ne + 2 - nen; ++i) vpi[nelist[i]] = -1e300;
                }
            } else {
                LUflag = LU(Ad, bd, vpi, ne + 2);
            }
            if (LUflag) {
                for (int j = 1; j <= ns; ++j) n[j] = n[j] + initial_eps;
                sn = 0.0;
                b[ne + 2] = 0.0;
                for (int j = 1; j <= ns; ++j) logn[j] = logtinytinyn;
                for (int j = 1; j <= ns; ++j) {
                    if (n[j] < tinytinyn)
                        n[j] = tinytinyn;
                    else
                        logn[j] = std::log(n[j]);
                    if (n[j] > tinyn) {
                        vhrt[j] = dot9(M.co[j][sec_num[j]], vThrt);
                        b[ne + 2] = b[ne + 2] + vhrt[j] * n[j];
                        sn = sn + n[j];
                    }
                }
                b[ne + 1] = sn;
                counter = counter + 1;
                if (counter > 500) break;
                continue;
            }

            const double Dlogsn = vpi[ne + 1];
            const double DlogT = vpi[ne + 2];
            for (int j = 1; j <= ns; ++j) {
                double tmp = 0.0;
                for (int i = 1; i <= ne; ++i) tmp = tmp + M.Ac[i][j] * vpi[i];
                Dlogn[j] = -vmurt[j] + tmp + Dlogsn + vhrt[j] * DlogT;
            }
            double lambda1 = 0.0, lambda2 = 1e300;
            const double logsn = std::log(b0[ne + 1]);
            for (int j = 1; j <= ns; ++j) {
                if (logn[j] - logsn > -18.420681)
                    lambda1 = std::fmax(lambda1, std::fabs(Dlogn[j]));
                else if (Dlogn[j] > 0.0)
                    lambda2 = std::fmin(lambda2, std::fabs((-logn[j] + logsn - 9.2103404) / (Dlogn[j] - Dlogsn)));
            }
            lambda1 = 2.0 / std::fmax(std::fmax(std::fmax(5.0 * std::fabs(DlogT), 5.0 * std::fabs(Dlogsn)),
                                                std::fabs(lambda1)),
                                      2.0);
            const double omega_var = std::fmin(1.0, std::fmin(lambda1, lambda2));

            b0[ne + 1] = b0[ne + 1] * std::exp(omega_var * Dlogsn);
            T = T * std::exp(omega_var * DlogT);
            logT = std::log(T);
            for (int j = 1; j <= ns; ++j) sec_num[j] = check_section_number(M, j, T);

            sn = 0.0;
            b[ne + 2] = 0.0;
            double Dnmax = 0.0;
            for (int j = 1; j <= ns; ++j) logn[j] = logtinytinyn;
            calc_vThrt(T, logT, vThrt);
            for (int j = 1; j <= ns; ++j) {
                n[j] = n[j] * std::exp(omega_var * Dlogn[j]);
                if (n[j] < tinytinyn)
                    n[j] = tinytinyn;
                else
                    logn[j] = std::log(n[j]);
                if (n[j] > tinyn) {
                    vhrt[j] = dot9(M.co[j][sec_num[j]], vThrt);
                    b[ne + 2] = b[ne + 2] + vhrt[j] * n[j];
                    sn = sn + n[j];
                    const double tmp = std::fabs(Dlogn[j]) * n[j];
                    if (Dnmax < tmp) Dnmax = tmp;
                }
            }
            b[ne + 1] = sn;

            flag = true;
            if (std::fabs(Dnmax) > eps * sn) flag = false;
            for (int i = 1; i <= ne; ++i)
                if (b0[i] > eps && std::fabs(b0[i] - b[i]) > b0max * eps) flag = false;
            if (std::fabs(Dlogsn) > eps || std::fabs(b0[ne + 1] - b[ne + 1]) > eps * std::fabs(sn)) flag = false;
            if (std::fabs(DlogT) > eps || std::fabs(H - b[ne + 2] * Ru * T) > eps * std::fabs(H)) flag = false;
            if (counter > 500) flag = true;
            if (flag) break;
            counter = counter + 1;
        }
        if (counter > 500) o.status = 1;
    }
    o.counter = counter;
    hp_tp_tail(M, T, logT, sn, tinyn, sec_num, n, false, o);
}

// cea_tp (sub_chem.f90:1963-2248): equilibrium at fixed T and p; the
// unknowns are pi_1..pi_ne and ln sn.  H is returned.  The singular-matrix
// retry is bounded as in cea_hp.
void cea_tp(const Model& M, double p, const double* Y, double T, double* n, CeaOut& o) {
    const int ns = M.ns, ne = M.ne;
    double b0[NEX] = {0}, b[NEX] = {0}, bd[NEX] = {0}, vpi[NEX] = {0};
    double vmurt[NSX], Dlogn[NSX], logn[NSX];
    int sec_num[NSX];
    double Ad[NEX][NEX];
    int elist[NEX], nelist[NEX], nen = 0;
    bool REDUCEflag;
    double vTmurt[10];
    o.status = 0;

    const double logP = std::log(p / pst);
    for (int i = 1; i <= ne + 2; ++i) b0[i] = Y[1] * M.b0f[i] + Y[2] * M.b0o[i];
    double b0max = b0[1];
    for (int i = 2; i <= ne; ++i)
        if (b0[i] > b0max) b0max = b0[i];
    double sn = 0.0;
    for (int j = 1; j <= ns; ++j) sn = sn + n[j];
    b0[ne + 1] = sn;

    if (Y[1] < Y_eps) {
        REDUCEflag = true;
        nen = M.neo;
        std::memcpy(elist, M.elisto, sizeof(elist));
        std::memcpy(nelist, M.nelisto, sizeof(nelist));
        for (int j = 1; j <= ns; ++j) n[j] = n[j] * M.masko[j];
    } else if (Y[2] < Y_eps) {
        REDUCEflag = true;
        nen = M.nef;
        std::memcpy(elist, M.elistf, sizeof(elist));
        std::memcpy(nelist, M.nelistf, sizeof(nelist));
        for (int j = 1; j <= ns; ++j) n[j] = n[j] * M.maskf[j];
    } else {
        REDUCEflag = false;
    }

    const double tinyn = TSIZE * sn;
    const double logtinyn = std::log(tinyn);
    const double tinytinyn = TTSIZE * sn;
    const double logtinytinyn = std::log(tinytinyn);

    const double logT = std::log(T);
    for (int i = 1; i <= ne + 2; ++i) b[i] = 0.0;
    b[ne + 1] = sn;
    for (int j = 1; j <= ns; ++j) logn[j] = logtinyn;
    for (int j = 1; j <= ns; ++j) {
        sec_num[j] = check_section_number(M, j, T);
        if (n[j] > tinyn) {
            logn[j] = std::log(n[j]);
            for (int i = 1; i <= ne; ++i) b[i] = b[i] + M.Ac[i][j] * n[j];
        }
    }
    bool flag = true;
    for (int i = 1; i <= ne; ++i)
        if (b0[i] > eps && std::fabs(b0[i] - b[i]) > b0max * eps) flag = false;

    int counter = 0;
    if (!flag) {
        counter = 1;
        for (;;) {
            for (int i = 1; i <= ne; ++i) b[i] = 0.0;
            for (int i = 1; i <= ne + 2; ++i) bd[i] = b0[i];
            bd[ne + 1] = b0[ne + 1] - b[ne + 1];
            for (int i = 1; i <= ne + 2; ++i)
                for (int j = 1; j <= ne + 2; ++j) Ad[i][j] = 0.0;
            calc_vTmurt(T, logT, vTmurt);
            for (int k = 1; k <= ns; ++k) {
                vmurt[k] = dot9(M.co[k][sec_num[k]], vTmurt) + logn[k] - std::log(b0[ne + 1]) + logP;
                if (n[k] > tinyn) {
                    const double vmurtn = vmurt[k] * n[k];
                    for (int i = 1; i <= ne; ++i) {
                        for (int j = i; j <= ne; ++j) Ad[i][j] = Ad[i][j] + M.Ac[i][k] * M.Ac[j][k] * n[k];
                        Ad[i][ne + 1] = Ad[i][ne + 1] + M.Ac[i][k] * n[k];
                        b[i] = b[i] + M.Ac[i][k] * n[k];
                        bd[i] = bd[i] + M.Ac[i][k] * (vmurtn - n[k]);
                    }
                    bd[ne + 1] = bd[ne + 1] + vmurtn;
                }
            }
            Ad[ne + 1][ne + 1] = b[ne + 1] - b0[ne + 1];
            for (int i = 1; i <= ne + 1; ++i)
                for (int j = i + 1; j <= ne + 1; ++j) Ad[j][i] = Ad[i][j];

            bool LUflag;
            if (REDUCEflag) {
                for (int i = 1; i <= nen; ++i) {
                    for (int j = 1; j <= nen; ++j) Ad[i][j] = Ad[elist[i]][elist[j]];
                    bd[i] = bd[elist[i]];
                }
                LUflag = LU(Ad, bd, vpi, nen);
                if (!LUflag) {
                    for (int i = nen; i >= 1; --i) vpi[elist[i]] = vpi[i];
                    for (int i = 1; i <= ne + 1 - nen; ++i) vpi[nelist[i]] = -1e300;
                }
            } else {
                LUflag = LU(Ad, bd, vpi, ne + 1);
            }
            if (LUflag) {
                for (int j = 1; j <= ns; ++j) n[j] = n[j] + initial_eps;
                sn = 0.0;
                for (int j = 1; j <= ns; ++j) logn[j] = logtinytinyn;
                for (int j = 1; j <= ns; ++j) {
                    if (n[j] < tinytinyn)
                        n[j] = tinytinyn;
                    else
                        logn[j] = std::log(n[j]);
                    if (n[j] > tinyn) sn = sn + n[j];
                }
                b[ne + 1] = sn;
                counter = counter + 1;
                if (counter > 500) break;
                continue;
            }

            const double Dlogsn = vpi[ne + 1];
            for (int j = 1; j <= ns; ++j) {
                double tmp = 0.0;
                for (int i = 1; i <= ne; ++i) tmp = tmp + M.Ac[i][j] * vpi[i];
                Dlogn[j] = -vmurt[j] + tmp + Dlogsn;
            }
            double lambda1 = 0.0, lambda2 = 1e300;
            const double logsn = std::log(b0[ne + 1]);
            for (int j = 1; j <= ns; ++j) {
                if (logn[j] - logsn > -18.420681)
                    lambda1 = std::fmax(lambda1, std::fabs(Dlogn[j]));
                else if (Dlogn[j] > 0.0)
                    lambda2 = std::fmin(lambda2, std::fabs((-logn[j] + logsn - 9.2103404) / (Dlogn[j] - Dlogsn)));
            }
            lambda1 = 2.0 / std::fmax(std::fmax(5.0 * std::fabs(Dlogsn), std::fabs(lambda1)), 2.0);
            const double omega_var = std::fmin(1.0, std::fmin(lambda1, lambda2));

            b0[ne + 1] = b0[ne + 1] * std::exp(omega_var * Dlogsn);
            sn = 0.0;
            double Dnmax = 0.0;
            for (int j = 1; j <= ns; ++j) logn[j] = logtinytinyn;
            for (int j = 1; j <= ns; ++j) {
                n[j] = n[j] * std::exp(omega_var * Dlogn[j]);
                if (n[j] < tinytinyn)
                    n[j] = tinytinyn;
                else
                    logn[j] = std::log(n[j]);
                if (n[j] > tinyn) {
                    sn = sn + n[j];
                    const double tmp = std::fabs(Dlogn[j]) * n[j];
                    if (Dnmax < tmp) Dnmax = tmp;
                }
            }
            b[ne + 1] = sn;

            flag = true;
            if (std::fabs(Dnmax) > eps * sn) flag = false;
            for (int i = 1; i <= ne; ++i)
                if (b0[i] > eps && std::fabs(b0[i] - b[i]) > b0max * eps) flag = false;
            if (std::fabs(Dlogsn) > eps || std::fabs(b0[ne + 1] - b[ne + 1]) > eps * std::fabs(sn)) flag = false;
            if (counter > 500) flag = true;
            if (flag) break;
            counter = counter + 1;
        }
        if (counter > 500) o.status = 1;
    }
    o.counter = counter;
    hp_tp_tail(M, T, logT, sn, tinyn, sec_num, n, true, o);
}

// calc_ini of initialize_cea (sub_chem.f90:1237-1287)
void calc_ini(const Model& M, double T, double* n, double& E, double& MWave, double* Yfoe) {
    const int ns = M.ns, ne = M.ne;
    double sn = 0.0, sm = 0.0;
    for (int j = 1; j <= ns; ++j) {
        sn = sn + n[j];
        sm = sm + n[j] * M.MW[j];
    }
    MWave = sm / sn;
    for (int j = 1; j <= ns; ++j) n[j] = n[j] / sm * 1e3;
    double vThrt[10];
    calc_vThrt(T, std::log(T), vThrt);
    E = 0.0;
    for (int j = 1; j <= ns; ++j) {
        const int nsc = check_section_number(M, j, T);
        double tmp = -1.0;
        for (int k = 1; k <= 9; ++k) tmp = tmp + vThrt[k] * M.co[j][nsc][k];
        E = E + tmp * n[j];
    }
    E = E * Ru * T;
    for (int i = 1; i <= ne; ++i) Yfoe[i] = 0.0;
    for (int j = 1; j <= ns; ++j) {
        const double tmp = n[j] * M.MW[j] * 1e-3;
        for (int i = 1; i <= ne; ++i) Yfoe[i] = Yfoe[i] + M.YAc[i][j] * tmp;
    }
}

bool valid(const scfd_cea_data& d) {
    if (d.abi_version != SCFD_ABI_VERSION) return false;
    if (d.ns < 1 || d.ns > SCFD_CEA_MAX_SPECIES || d.ne < 1 || d.ne > SCFD_CEA_MAX_ELEMENTS || d.nt < 0 ||
        d.nt > d.ns)
        return false;
    for (int j = 0; j < d.ns; ++j)
        if (d.nsec[j] < 1 || d.nsec[j] > SCFD_CEA_MAX_SECTIONS || !(d.mw[j] > 0.0)) return false;
    for (int i = 0; i < d.nt; ++i)
        if (d.ntsec[i] < 1 || d.ntsec[i] > SCFD_CEA_MAX_TSECTIONS || d.tr2th[i] < 0 || d.tr2th[i] >= d.ns)
            return false;
    if (!(d.pf > 0.0 && d.po > 0.0 && d.Tf > 0.0 && d.To > 0.0)) return false;
    double sf = 0.0, so = 0.0;
    for (int j = 0; j < d.ns; ++j) {
        if (d.nf[j] < 0.0 || d.no[j] < 0.0) return false;
        sf += d.nf[j];
        so += d.no[j];
    }
    return sf > 0.0 && so > 0.0;
}

}  // namespace

struct scfd_cea : Model {};

extern "C" {

int orc_cea_create(const scfd_cea_data* data, scfd_cea** out) {
    if (!data || !out) return SCFD_E_ARG;
    *out = nullptr;
    if (!valid(*data)) return SCFD_E_ARG;
    scfd_cea* h = new scfd_cea();
    Model& M = *h;
    std::memset(&M, 0, sizeof(Model));
    M.d = *data;
    const scfd_cea_data& d = M.d;
    M.ns = d.ns;
    M.ne = d.ne;
    M.nt = d.nt;
    const int ns = M.ns, ne = M.ne;
    for (int j = 1; j <= ns; ++j) {
        M.MW[j] = d.mw[j - 1];
        for (int l = 1; l <= d.nsec[j - 1]; ++l)
            for (int k = 1; k <= 9; ++k) M.co[j][l][k] = d.co[j - 1][l - 1][k - 1];
        for (int i = 1; i <= ne; ++i) M.Ac[i][j] = d.ac[j - 1][i - 1];
    }
    // set_therm_data: YAc (sub_chem.f90:159-170)
    for (int j = 1; j <= ns; ++j) {
        double tmp = 0.0;
        for (int i = 1; i <= ne; ++i) {
            M.YAc[i][j] = d.mwe[i - 1] * M.Ac[i][j];
            tmp = tmp + M.YAc[i][j];
        }
        tmp = 1.0 / tmp;
        for (int i = 1; i <= ne; ++i) M.YAc[i][j] = M.YAc[i][j] * tmp;
    }
    // initialize_cea (sub_chem.f90:1136-1230), flag 'uv'
    scfd_cea_info& inf = M.info;
    double nf[NSX], no[NSX];
    double sumo = 0.0, sumf = 0.0;
    for (int j = 1; j <= ns; ++j) {
        nf[j] = d.nf[j - 1];
        no[j] = d.no[j - 1];
        sumo = sumo + M.MW[j] * no[j];
        sumf = sumf + M.MW[j] * nf[j];
    }
    inf.of = sumo / sumf;
    double Ef, Eo, MWf, MWo;
    calc_ini(M, d.Tf, nf, Ef, MWf, M.Yfe);
    calc_ini(M, d.To, no, Eo, MWo, M.Yoe);
    for (int j = 1; j <= ns; ++j)
        for (int i = 1; i <= ne; ++i) {
            M.b0f[i] = M.b0f[i] + M.Ac[i][j] * nf[j];
            M.b0o[i] = M.b0o[i] + M.Ac[i][j] * no[j];
        }
    int nshiftf = 0, nshifto = 0;
    for (int i = 1; i <= ne + 2; ++i) M.maskbf[i] = M.maskbo[i] = 1.0;
    for (int i = 1; i <= ne; ++i) {
        if (M.b0f[i] == 0.0) {
            M.maskbf[i] = 0.0;
            nshiftf = nshiftf + 1;
            M.nelistf[nshiftf] = i;
        } else {
            M.elistf[i - nshiftf] = i;
        }
        if (M.b0o[i] == 0.0) {
            M.maskbo[i] = 0.0;
            nshifto = nshifto + 1;
            M.nelisto[nshifto] = i;
        } else {
            M.elisto[i - nshifto] = i;
        }
    }
    M.elisto[ne + 1 - nshifto] = ne + 1;
    M.elisto[ne + 2 - nshifto] = ne + 2;
    M.neo = ne + 1 - nshifto;
    M.elistf[ne + 1 - nshiftf] = ne + 1;
    M.elistf[ne + 2 - nshiftf] = ne + 2;
    M.nef = ne + 1 - nshiftf;
    for (int j = 1; j <= ns; ++j) {
        M.masko[j] = 1.0;
        M.maskf[j] = 1.0;
        for (int i = 1; i <= nshifto; ++i)
            if (M.Ac[M.nelisto[i]][j] != 0.0) M.masko[j] = 0.0;
        for (int i = 1; i <= nshiftf; ++i)
            if (M.Ac[M.nelistf[i]][j] != 0.0) M.maskf[j] = 0.0;
        if (M.masko[j] != 1.0) M.masko[j] = 1e-100;
        if (M.maskf[j] != 1.0) M.maskf[j] = 1e-100;
    }
    for (int i = 1; i <= ne; ++i) {
        inf.fuel.b0[i - 1] = M.b0f[i];
        inf.oxidizer.b0[i - 1] = M.b0o[i];
        inf.fuel.ye[i - 1] = M.Yfe[i];
        inf.oxidizer.ye[i - 1] = M.Yoe[i];
    }
    double Y[3];
    CeaOut o;
    scfd_cea_stream* st[2] = {&inf.fuel, &inf.oxidizer};
    double* ns_[2] = {nf, no};
    const double Es[2] = {Ef, Eo}, MWs[2] = {MWf, MWo}, ps[2] = {d.pf, d.po}, Ts[2] = {d.Tf, d.To};
    for (int s = 0; s < 2; ++s) {
        Y[1] = s == 0 ? 1.0 : 0.0;
        Y[2] = s == 0 ? 0.0 : 1.0;
        double rho = ps[s] / (Ru * 1e3 / MWs[s] * Ts[s]);
        double* n = ns_[s];
        for (int j = 1; j <= ns; ++j) n[j] = n[j] + initial_eps;
        double T = Ts[s];
        scfd_cea_stream& S = *st[s];
        if (d.init_hp) {
            // sub_chem.f90:1206-1211: H = E + p/rho, cea_hp, then rho and E again
            const double H = Es[s] + ps[s] / rho;
            cea_hp(M, ps[s], Y, H, T, n, o);
            rho = ps[s] / (Ru * 1e3 / o.MWave * T);
            S.e = H - ps[s] / rho;
            S.p = ps[s];
            S.h = H;
        } else {
            cea(M, rho, Y, Es[s], T, n, o);
            if (o.status == 2) {
                delete h;
                return SCFD_E_SINGULAR;
            }
            S.e = Es[s];
            S.p = rho * Ru * 1e3 / o.MWave * T;
            S.h = S.e + S.p / rho;
        }
        S.rho = rho;
        S.T = T;
        S.mw = o.MWave;
        S.kappa = o.kappa;
        S.mu = o.mu;
        for (int j = 1; j <= ns; ++j) S.n[j - 1] = n[j];
        (s == 0 ? inf.iters_fuel : inf.iters_oxidizer) = o.counter;
    }
    double sm = 0.0;
    for (int j = 1; j <= ns; ++j) sm = sm + (no[j] + nf[j]);
    inf.n_init = sm / ns;
    *out = h;
    return 0;
}

int orc_cea_destroy(scfd_cea* h) {
    if (!h) return SCFD_E_ARG;
    delete h;
    return 0;
}

int orc_cea_info_get(const scfd_cea* h, scfd_cea_info* info) {
    if (!h || !info) return SCFD_E_ARG;
    *info = h->info;
    return 0;
}

int orc_cea_solve(scfd_cea* h, int64_t ncell, const double* rho, const double* Y, const double* e, double* T,
                  double* n, double* mwave, double* kappa, double* mu, double* Yv, double* vhi, double* DHi,
                  int32_t* iters, void* /*stream*/) {
    if (!h || ncell < 0) return SCFD_E_ARG;
    if (ncell > 0 && (!rho || !Y || !e || !T || !n)) return SCFD_E_ARG;
    const Model& M = *h;
    const int ns = M.ns;
    int64_t f0 = 0, f1 = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : f0, f1)
    for (int64_t c = 0; c < ncell; ++c) {
        double nn[NSX], y[3];
        CeaOut o;
        for (int j = 1; j <= ns; ++j) nn[j] = n[(j - 1) * ncell + c];
        y[1] = Y[c];
        y[2] = Y[ncell + c];
        double t = T[c];
        cea(M, rho[c], y, e[c], t, nn, o);
        if (o.status == 1) f0 += 1;
        if (o.status == 2) f1 += 1;
        T[c] = t;
        for (int j = 1; j <= ns; ++j) n[(j - 1) * ncell + c] = nn[j];
        if (mwave) mwave[c] = o.MWave;
        if (kappa) kappa[c] = o.kappa;
        if (mu) mu[c] = o.mu;
        if (iters) iters[c] = o.status == 2 ? -1 : o.counter;
        if (DHi) {
            DHi[c] = o.DHi[1];
            DHi[ncell + c] = o.DHi[2];
        }
        for (int j = 1; j <= ns; ++j) {
            if (Yv) Yv[(j - 1) * ncell + c] = o.Yv[j];
            if (vhi) vhi[(j - 1) * ncell + c] = o.vhi[j];
        }
    }
    h->fails[0] += f0;
    h->fails[1] += f1;
    return 0;
}

// fixed p and h (hp) or fixed p and T (tp) over ncell cells
static int solve_hp_tp(scfd_cea* h, bool hp, int64_t ncell, const double* p, const double* Y, const double* hh,
                       double* T, double* n, double* hout, double* mwave, double* kappa, double* mu, double* Yv,
                       double* vhi, int32_t* iters) {
    if (!h || ncell < 0) return SCFD_E_ARG;
    if (ncell > 0 && (!p || !Y || !T || !n || (hp && !hh))) return SCFD_E_ARG;
    const Model& M = *h;
    const int ns = M.ns;
    int64_t f0 = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : f0)
    for (int64_t c = 0; c < ncell; ++c) {
        double nn[NSX], y[3];
        CeaOut o;
        for (int j = 1; j <= ns; ++j) nn[j] = n[(j - 1) * ncell + c];
        y[1] = Y[c];
        y[2] = Y[ncell + c];
        double t = T[c];
        if (hp)
            cea_hp(M, p[c], y, hh[c], t, nn, o);
        else
            cea_tp(M, p[c], y, t, nn, o);
        if (o.status == 1) f0 += 1;
        if (hp) T[c] = t;
        for (int j = 1; j <= ns; ++j) n[(j - 1) * ncell + c] = nn[j];
        if (hout) hout[c] = o.H;
        if (mwave) mwave[c] = o.MWave;
        if (kappa) kappa[c] = o.kappa;
        if (mu) mu[c] = o.mu;
        if (iters) iters[c] = o.counter;
        for (int j = 1; j <= ns; ++j) {
            if (Yv) Yv[(j - 1) * ncell + c] = o.Yv[j];
            if (vhi) vhi[(j - 1) * ncell + c] = o.vhi[j];
        }
    }
    h->fails[0] += f0;
    return 0;
}

int orc_cea_solve_hp(scfd_cea* h, int64_t ncell, const double* p, const double* Y, const double* hh, double* T,
                     double* n, double* mwave, double* kappa, double* mu, double* Yv, double* vhi, int32_t* iters,
                     void* /*stream*/) {
    return solve_hp_tp(h, true, ncell, p, Y, hh, T, n, nullptr, mwave, kappa, mu, Yv, vhi, iters);
}

int orc_cea_solve_tp(scfd_cea* h, int64_t ncell, const double* p, const double* Y, const double* T, double* n,
                     double* hh, double* mwave, double* kappa, double* mu, double* Yv, double* vhi, int32_t* iters,
                     void* /*stream*/) {
    return solve_hp_tp(h, false, ncell, p, Y, nullptr, const_cast<double*>(T), n, hh, mwave, kappa, mu, Yv, vhi,
                       iters);
}

int orc_cea_status(scfd_cea* h, int64_t* counts) {
    if (!h || !counts) return SCFD_E_ARG;
    counts[0] = h->fails[0];
    counts[1] = h->fails[1];
    h->fails[0] = h->fails[1] = 0;
    return counts[1] ? SCFD_E_SINGULAR : 0;
}

}  // extern "C"
