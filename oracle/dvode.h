// dvode.h -- the DVODE integrator as the reference calls it, restated in C++
// (test infrastructure: part of the CPU restatement that checks the CUDA path).
//
// Follows store/therm_lib/chemkin/core/dvode.f (Brown, Byrne, Hindmarsh,
// "VODE: a variable-coefficient ODE solver", SIAM J. Sci. Stat. Comput. 10,
// 1989) on the one path the reference uses, sub_chem.f90:1755-1775:
// MF = 21 (BDF, METH = 2, with the user's exact Jacobian, MITER = 1, saved
// and reused, JSV = 1), ITASK = 1 (integrate past TOUT and interpolate),
// ITOL = 1 (scalar tolerances), IOPT = 0 (MAXORD 5, MXSTEP 500, HMIN = HMAX
// limits off), ISTATE = 1 on every call.  The state lives in the Nordsieck
// array YH (column-major, N x (MAXORD + 1)); dvode.f routine by routine:
//   DVODE   dvode.f:2-1672     driver (start, error weights, step loop, exits)
//   DVHIN   dvode.f:1673-1810  initial step size
//   DVINDY  dvode.f:1811-1933  interpolation of YH at TOUT
//   DVSTEP  dvode.f:1934-2368  one step with step / order control
//   DVSET   dvode.f:2369-2567  BDF coefficients EL and test constants TQ
//   DVJUST  dvode.f:2568-2727  YH adjustment on an order change
//   DVNLSD  dvode.f:2728-2956  Newton iteration on the corrector
//   DVJAC   dvode.f:2957-3234  Jacobian and the LU of I - h l1 J (DGEFA)
//   DVSOL   dvode.f:3261-3356  solve with the LU (DGESL)
//   DEWSET, DVNORM, DGEFA, DGESL, IDAMAX  dvode.f:3419-3500, 3816-4061, 4907-
// The loop order of every sum and update is the Fortran's.  F and JAC are
// Fex and Jex (FJ.f90:152-300, 454-709), i.e. fex_jex of this file's includer.

namespace dvode {

constexpr int NMAX = SCFD_MAX_SPECIES + 1;
constexpr int MAXORD = 5;          // MORD(2), BDF
constexpr int LMAXC = MAXORD + 1;  // Nordsieck columns
constexpr int MXSTEP = 500;        // MXSTP0
constexpr double UROUND = 2.220446049250313080847e-16;  // DUMACH: 2**-52

struct State {
    // COMMON /DVOD01/, /DVOD02/ (the members the METH 2 / MITER 1 path uses)
    double acnrm = 0, ccmxj = 0, conp = 0, crate = 0, drc = 0, el[14] = {}, eta = 0, etamax = 0, h = 0, hmin = 0,
           hmxi = 0, hnew = 0, hscal = 0, prl1 = 0, rc = 0, rl1 = 0, tau[14] = {}, tq[6] = {}, tn = 0;
    int icf = 0, init = 0, ipup = 0, jcur = 0, jstart = 0, kflag = 0, kuth = 0, l = 0, lmax = 0, msbj = 0, n = 0,
        newh = 0, newq = 0, nq = 0, nqnyh = 0, nqwait = 0, nslj = 0, nslp = 0;
    double hu = 0;
    int ncfn = 0, netf = 0, nfe = 0, nje = 0, nlu = 0, nni = 0, nqu = 0, nst = 0;
    // DVSTEP's SAVEd locals that outlive one call of it
    double etaq = 0, etaqm1 = 0;
    // RWORK / IWORK pieces
    double yh[NMAX * (LMAXC + 1)];  // YH(LDYH, LMAX), 1-based via YH(i, j); one spare column
    double ewt[NMAX + 1], savf[NMAX + 1], acor[NMAX + 1], ftem[NMAX + 1];
    double wm[NMAX * NMAX + 1];     // the iteration matrix, then its LU (column-major, 1-based)
    double js[NMAX * NMAX + 1];     // the saved Jacobian
    int ipvt[NMAX + 1];
    double& YH(int i, int j) { return yh[(i - 1) + (j - 1) * n]; }
    double& YH1(int k) { return yh[k - 1]; }  // YH viewed as one vector, 1-based
    double& A(int i, int j) { return wm[(i - 1) + (j - 1) * n + 1]; }
};

// F(N, T, Y, YDOT) and JAC(N, T, Y, ..., PD): y and ydot are 1-based arrays
template <typename FEX, typename JEX>
struct System {
    FEX f;
    JEX jac;
    long long* evals;
};

// real ** integer as Fortran compilers evaluate it (binary powering)
inline double ipow(double x, int m) {
    unsigned n = m < 0 ? -m : m;
    double y = (n % 2) ? x : 1.0;
    while (n >>= 1) {
        x = x * x;
        if (n % 2) y = y * x;
    }
    return m < 0 ? 1.0 / y : y;
}

inline double vnorm(int n, const double* v, const double* w) {  // DVNORM, dvode.f:3467-3500
    double sum = 0.0;
    for (int i = 1; i <= n; ++i) sum = sum + (v[i] * w[i]) * (v[i] * w[i]);
    return std::sqrt(sum / n);
}

inline void ewset(int n, double rtol, double atol, const double* ycur, double* ewt) {  // DEWSET ITOL 1
    for (int i = 1; i <= n; ++i) ewt[i] = rtol * std::fabs(ycur[i]) + atol;
}

inline int idamax(int n, const double* dx) {  // IDAMAX with INCX = 1, dx 1-based
    if (n <= 0) return 0;
    int imax = 1;
    if (n == 1) return imax;
    double dmax = std::fabs(dx[1]);
    for (int i = 2; i <= n; ++i) {
        const double xmag = std::fabs(dx[i]);
        if (xmag > dmax) {
            imax = i;
            dmax = xmag;
        }
    }
    return imax;
}

// DGEFA (dvode.f:3816-3931): LU with partial pivoting, column-oriented
inline int gefa(State& s) {
    const int n = s.n;
    int info = 0;
    for (int k = 1; k <= n - 1; ++k) {
        const int kp1 = k + 1;
        const int l = idamax(n - k + 1, &s.A(k, k) - 1) + k - 1;
        s.ipvt[k] = l;
        if (s.A(l, k) == 0.0) {
            info = k;
            continue;
        }
        if (l != k) {
            const double t = s.A(l, k);
            s.A(l, k) = s.A(k, k);
            s.A(k, k) = t;
        }
        double t = -1.0 / s.A(k, k);
        for (int i = k + 1; i <= n; ++i) s.A(i, k) = t * s.A(i, k);  // DSCAL
        for (int j = kp1; j <= n; ++j) {
            t = s.A(l, j);
            if (l != k) {
                s.A(l, j) = s.A(k, j);
                s.A(k, j) = t;
            }
            for (int i = k + 1; i <= n; ++i) s.A(i, j) = s.A(i, j) + t * s.A(i, k);  // DAXPY
        }
    }
    s.ipvt[n] = n;
    if (s.A(n, n) == 0.0) info = n;
    return info;
}

// DGESL with JOB = 0 (dvode.f:3932-4061): solves A x = b in place, b 1-based
inline void gesl(State& s, double* b) {
    const int n = s.n;
    for (int k = 1; k <= n - 1; ++k) {
        const int l = s.ipvt[k];
        const double t = b[l];
        if (l != k) {
            b[l] = b[k];
            b[k] = t;
        }
        for (int i = k + 1; i <= n; ++i) b[i] = b[i] + t * s.A(i, k);
    }
    for (int kb = 1; kb <= n; ++kb) {
        const int k = n + 1 - kb;
        b[k] = b[k] / s.A(k, k);
        const double t = -b[k];
        for (int i = 1; i <= k - 1; ++i) b[i] = b[i] + t * s.A(i, k);
    }
}

// DVSET, METH 2 (dvode.f:2369-2567)
inline void vset(State& s) {
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
    s.tq[2] = std::fabs(alph0 * t2 / t1);
    s.tq[5] = std::fabs(t2 / (el[s.l] * rxi / rxis));
    if (s.nqwait == 1) {
        const double cnqm1 = rxis / el[s.l];
        const double t3 = alph0 + 1.0 / (double)nq;
        const double t4 = ahatn0 + rxi;
        double elp = t3 / (1.0 - t4 + t3);
        s.tq[1] = std::fabs(elp / cnqm1);
        hsum = hsum + s.tau[nq];
        rxi = s.h / hsum;
        const double t5 = alph0 - 1.0 / (double)(nq + 1);
        const double t6 = ahatn0 - rxi;
        elp = t2 / (1.0 - t6 + t5);
        s.tq[3] = std::fabs(elp * rxi * (flotl + 1.0) * t5);
    }
    s.tq[4] = 0.1 * s.tq[2];  // CORTES
}

// DVJUST, METH 2 (dvode.f:2568-2727)
inline void vjust(State& s, int iord) {
    if (s.nq == 2 && iord != 1) return;
    const int nqm1 = s.nq - 1, nqm2 = s.nq - 2, n = s.n;
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
        for (int j = 3; j <= s.nq; ++j)
            for (int i = 1; i <= n; ++i) s.YH(i, j) = s.YH(i, j) - s.YH(i, s.l) * el[j];
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
    const int lp1 = s.l + 1;
    for (int i = 1; i <= n; ++i) s.YH(i, lp1) = t1 * s.YH(i, s.lmax);
    const int nqp1 = s.nq + 1;
    for (int j = 3; j <= nqp1; ++j)
        for (int i = 1; i <= n; ++i) s.YH(i, j) = s.YH(i, j) + el[j] * s.YH(i, lp1);  // DAXPY
}

// DVJAC, MITER 1 with JSV 1 (dvode.f:2957-3234); returns IERPJ
template <typename SYS>
int vjac(State& s, SYS& sys, const double* y) {
    const int n = s.n;
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
        for (int i = 1; i <= lenp; ++i) s.wm[i] = 0.0;
        sys.jac(s.tn, y, s);  // fills A(i, j) = d f_i / d y_j
        for (int i = 1; i <= lenp; ++i) s.js[i] = s.wm[i];
    } else {
        s.jcur = 0;
        for (int i = 1; i <= lenp; ++i) s.wm[i] = s.js[i];
    }
    const double con = -hrl1;
    for (int i = 1; i <= lenp; ++i) s.wm[i] = con * s.wm[i];
    for (int i = 1; i <= n; ++i) s.A(i, i) = s.A(i, i) + 1.0;
    ++s.nlu;
    return gefa(s) != 0 ? 1 : 0;
}

// DVNLSD, METH 2 / MITER 1 (dvode.f:2728-2956); nflag in / out
template <typename SYS>
void vnlsd(State& s, SYS& sys, double* y, int& nflag) {
    const int n = s.n;
    const double CCMAX = 0.3, CRDOWN = 0.3, RDIV = 2.0;
    const int MAXCOR = 3, MSBP = 20;
    if (s.jstart == 0) s.nslp = 0;
    if (nflag == 0) s.icf = 0;
    if (nflag == -2) s.ipup = 1;
    if (s.jstart == 0 || s.jstart == -1) s.ipup = 1;
    s.drc = std::fabs(s.rc - 1.0);
    if (s.drc > CCMAX || s.nst >= s.nslp + MSBP) s.ipup = 1;
    for (;;) {  // 220
        int m = 0;
        double delp = 0.0, del = 0.0;
        for (int i = 1; i <= n; ++i) y[i] = s.YH(i, 1);
        sys.f(s.tn, y, s.savf);
        ++s.nfe;
        if (s.ipup > 0) {
            const int ierpj = vjac(s, sys, y);
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
        for (int i = 1; i <= n; ++i) s.acor[i] = 0.0;
        bool retry = false;
        for (;;) {  // 270 / 350
            for (int i = 1; i <= n; ++i) y[i] = (s.rl1 * s.h) * s.savf[i] - (s.rl1 * s.YH(i, 2) + s.acor[i]);
            gesl(s, y);
            ++s.nni;
            if (s.rc != 1.0) {
                const double cscale = 2.0 / (1.0 + s.rc);
                for (int i = 1; i <= n; ++i) y[i] = cscale * y[i];
            }
            del = vnorm(n, y, s.ewt);
            for (int i = 1; i <= n; ++i) s.acor[i] = s.acor[i] + y[i];
            for (int i = 1; i <= n; ++i) y[i] = s.YH(i, 1) + s.acor[i];
            if (m != 0) s.crate = std::max(CRDOWN * s.crate, del / delp);  // 400
            const double dcon = del * std::min(1.0, s.crate) / s.tq[4];
            if (dcon <= 1.0) {  // 450
                nflag = 0;
                s.jcur = 0;
                s.icf = 0;
                if (m == 0) s.acnrm = del;
                if (m > 0) s.acnrm = vnorm(n, s.acor, s.ewt);
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
            sys.f(s.tn, y, s.savf);
            ++s.nfe;
        }
        if (!retry) return;
    }
}

// DVSTEP (dvode.f:1934-2368); y is scratch for the corrector
template <typename SYS>
void vstep(State& s, SYS& sys, double* y) {
    const int n = s.n, ldyh = n;
    const int KFC = -3, KFH = -7, MXNCF = 10;
    const double ADDON = 1.0e-6, BIAS1 = 6.0, BIAS2 = 6.0, BIAS3 = 10.0, ETACF = 0.25, ETAMIN = 0.1, ETAMXF = 0.2,
                 ETAMX1 = 1.0e4, ETAMX2 = 10.0, ETAMX3 = 10.0, ONEPSM = 1.00001, THRESH = 1.5;
    s.kflag = 0;
    const double told = s.tn;
    int ncf = 0;
    s.jcur = 0;
    int nflag = 0;
    auto predict_undo = [&]() {
        int i1 = s.nqnyh + 1;
        for (int jb = 1; jb <= s.nq; ++jb) {
            i1 = i1 - ldyh;
            for (int i = i1; i <= s.nqnyh; ++i) s.YH1(i) = s.YH1(i) - s.YH1(i + ldyh);
        }
    };
    int go = 0;  // 0: 200, 1: 20 (JSTART > 0), 2: 150
    if (s.jstart > 0) {
        go = 1;
    } else {  // JSTART = 0 (the path of ISTATE = 1)
        s.lmax = MAXORD + 1;
        s.nq = 1;
        s.l = 2;
        s.nqnyh = s.nq * ldyh;
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
                s.eta = std::min(s.eta, s.h / s.hscal);
                s.newh = 1;
            }
            if (s.newh == 0) {
                go = 0;
                continue;
            }
            if (s.newq < s.nq) {
                vjust(s, -1);
                s.nq = s.newq;
                s.l = s.nq + 1;
                s.nqwait = s.l;
            } else if (s.newq > s.nq) {
                vjust(s, 1);
                s.nq = s.newq;
                s.l = s.nq + 1;
                s.nqwait = s.l;
            }
            go = 2;
            continue;
        }
        if (go == 2) {  // 150: rescale YH by eta
            double r = 1.0;
            for (int j = 2; j <= s.l; ++j) {
                r = r * s.eta;
                for (int i = 1; i <= n; ++i) s.YH(i, j) = r * s.YH(i, j);
            }
            s.h = s.hscal * s.eta;
            s.hscal = s.h;
            s.rc = s.rc * s.eta;
            s.nqnyh = s.nq * ldyh;
            go = 0;
            continue;
        }
        // 200: predict
        s.tn = s.tn + s.h;
        {
            int i1 = s.nqnyh + 1;
            for (int jb = 1; jb <= s.nq; ++jb) {
                i1 = i1 - ldyh;
                for (int i = i1; i <= s.nqnyh; ++i) s.YH1(i) = s.YH1(i) + s.YH1(i + ldyh);
            }
        }
        vset(s);
        s.rl1 = 1.0 / s.el[2];
        s.rc = s.rc * (s.rl1 / s.prl1);
        s.prl1 = s.rl1;
        vnlsd(s, sys, y, nflag);
        if (nflag != 0) {
            ++ncf;
            ++s.ncfn;
            s.etamax = 1.0;
            s.tn = told;
            predict_undo();
            if (nflag < -1) {  // 680
                if (nflag == -2) s.kflag = -3;
                if (nflag == -3) s.kflag = -4;
                s.jstart = 1;
                return;
            }
            if (std::fabs(s.h) <= s.hmin * ONEPSM || ncf == MXNCF) {  // 670
                s.kflag = -2;
                s.jstart = 1;
                return;
            }
            s.eta = ETACF;
            s.eta = std::max(s.eta, s.hmin / std::fabs(s.h));
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
            predict_undo();
            if (std::fabs(s.h) <= s.hmin * ONEPSM) {  // 660
                s.kflag = -1;
                s.jstart = 1;
                return;
            }
            s.etamax = 1.0;
            if (s.kflag > KFC) {
                const double flotl = (double)s.l;
                s.eta = 1.0 / (std::pow(BIAS2 * dsm, 1.0 / flotl) + ADDON);
                s.eta = std::max(std::max(s.eta, s.hmin / std::fabs(s.h)), ETAMIN);
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
                s.eta = std::max(ETAMIN, s.hmin / std::fabs(s.h));
                vjust(s, -1);
                s.l = s.nq;
                s.nq = s.nq - 1;
                s.nqwait = s.l;
                go = 2;
                continue;
            }
            // 540: restart at order 1 from the last accepted state
            s.eta = std::max(ETAMIN, s.hmin / std::fabs(s.h));
            s.h = s.h * s.eta;
            s.hscal = s.h;
            s.tau[1] = s.h;
            sys.f(s.tn, y, s.savf);
            ++s.nfe;
            for (int i = 1; i <= n; ++i) s.YH(i, 2) = s.h * s.savf[i];
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
        for (int j = 1; j <= s.l; ++j)
            for (int i = 1; i <= n; ++i) s.YH(i, j) = s.YH(i, j) + s.el[j] * s.acor[i];  // DAXPY
        --s.nqwait;
        if (s.l != s.lmax && s.nqwait == 1) {
            for (int i = 1; i <= n; ++i) s.YH(i, s.lmax) = s.acor[i];
            s.conp = s.tq[5];
        }
        bool to690 = false;
        if (s.etamax == 1.0) {  // 490
            if (s.nqwait < 2) s.nqwait = 2;
            s.newq = s.nq;
            s.newh = 0;
            s.eta = 1.0;
            s.hnew = s.h;
            to690 = true;
        } else {  // 560: step and order for the next step
            const double flotl = (double)s.l;
            s.etaq = 1.0 / (std::pow(BIAS2 * dsm, 1.0 / flotl) + ADDON);
            if (s.nqwait != 0) {  // 600
                s.eta = s.etaq;
                s.newq = s.nq;
            } else {
                s.nqwait = 2;
                s.etaqm1 = 0.0;
                if (s.nq != 1) {
                    const double ddn = vnorm(n, &s.YH(1, s.l) - 1, s.ewt) / s.tq[1];
                    s.etaqm1 = 1.0 / (std::pow(BIAS1 * ddn, 1.0 / (flotl - 1.0)) + ADDON);
                }
                double etaqp1 = 0.0;  // 570
                if (s.l != s.lmax) {
                    const double cnquot = (s.tq[5] / s.conp) * ipow(s.h / s.tau[2], s.l);
                    for (int i = 1; i <= n; ++i) s.savf[i] = s.acor[i] - cnquot * s.YH(i, s.lmax);
                    const double dup = vnorm(n, s.savf, s.ewt) / s.tq[3];
                    etaqp1 = 1.0 / (std::pow(BIAS3 * dup, 1.0 / (flotl + 1.0)) + ADDON);
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
                    for (int i = 1; i <= n; ++i) s.YH(i, s.lmax) = s.acor[i];
                }
            }
            // 630
            if (s.eta < THRESH || s.etamax == 1.0) {  // 640
                s.newq = s.nq;
                s.newh = 0;
                s.eta = 1.0;
                s.hnew = s.h;
            } else {
                s.eta = std::min(s.eta, s.etamax);
                s.eta = s.eta / std::max(1.0, std::fabs(s.h) * s.hmxi * s.eta);
                s.newh = 1;
                s.hnew = s.h * s.eta;
            }
            to690 = true;
        }
        if (to690) {  // 690 / 700
            s.etamax = ETAMX3;
            if (s.nst <= 10) s.etamax = ETAMX2;
            const double r = 1.0 / s.tq[2];
            for (int i = 1; i <= n; ++i) s.acor[i] = r * s.acor[i];
        }
        s.jstart = 1;
        return;
    }
}

// DVHIN (dvode.f:1673-1810); y0, ydot, temp, y 1-based; returns IER
template <typename SYS>
int vhin(State& s, SYS& sys, double t0, const double* y0, const double* ydot, double tout, double atol, double* y,
         double* temp, double& h0, int& niter) {
    const int n = s.n;
    niter = 0;
    const double tdist = std::fabs(tout - t0);
    const double tround = UROUND * std::max(std::fabs(t0), std::fabs(tout));
    if (tdist < 2.0 * tround) return -1;
    const double hlb = 100.0 * tround;
    double hub = 0.1 * tdist;
    for (int i = 1; i <= n; ++i) {
        const double delyi = 0.1 * std::fabs(y0[i]) + atol;
        const double afi = std::fabs(ydot[i]);
        if (afi * hub > delyi) hub = delyi / afi;
    }
    int iter = 0;
    double hg = std::sqrt(hlb * hub);
    if (hub < hlb) {
        h0 = hg;
    } else {
        double hnew;
        for (;;) {  // 50
            const double h = std::copysign(hg, tout - t0);
            const double t1 = t0 + h;
            for (int i = 1; i <= n; ++i) y[i] = y0[i] + h * ydot[i];
            sys.f(t1, y, temp);
            for (int i = 1; i <= n; ++i) temp[i] = (temp[i] - ydot[i]) / h;
            const double yddnrm = vnorm(n, temp, s.ewt);
            if (yddnrm * hub * hub > 2.0)
                hnew = std::sqrt(2.0 / yddnrm);
            else
                hnew = std::sqrt(hg * hub);
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
    h0 = std::copysign(h0, tout - t0);  // 90
    niter = iter;
    return 0;
}

// DVINDY with K = 0 (dvode.f:1811-1933): YH interpolated at t into dky; IFLAG
inline int vindy(State& s, double t, double* dky) {
    const int n = s.n;
    const double tfuzz = 100.0 * UROUND * std::copysign(std::fabs(s.tn) + std::fabs(s.hu), s.hu);
    const double tp = s.tn - s.hu - tfuzz;
    const double tn1 = s.tn + tfuzz;
    if ((t - tp) * (t - tn1) > 0.0) return -2;
    const double sv = (t - s.tn) / s.h;
    for (int i = 1; i <= n; ++i) dky[i] = 1.0 * s.YH(i, s.l);
    for (int jb = 1; jb <= s.nq; ++jb) {
        const int j = s.nq - jb, jp1 = j + 1;
        for (int i = 1; i <= n; ++i) dky[i] = 1.0 * s.YH(i, jp1) + sv * dky[i];
    }
    return 0;
}

// DVODE with ISTATE = 1, ITASK = 1 (dvode.f:2-1672).  y (1-based, n values)
// holds the state at t on entry; on return ISTATE: 2 with y at tout and
// t = tout, or < 0 with y and t of the last accepted step (-1: MXSTEP steps
// taken; -2 too much accuracy; -3 illegal input; -4 error test failures; -5
// convergence failures; -6 a zero error weight).  `accepted(tn, yh1)` is
// called after every accepted step.
template <typename SYS, typename ACC>
int solve(State& s, SYS& sys, int n, double* y, double& t, double tout, double rtol, double atol, ACC accepted) {
    if (tout == t) return 1;
    s.init = 0;
    s.n = n;
    s.hmxi = 0.0;
    s.hmin = 0.0;
    double h0 = 0.0;
    s.tn = t;
    s.jstart = 0;
    s.ccmxj = 0.2;
    s.msbj = 50;
    s.nst = s.nje = s.nni = s.ncfn = s.netf = s.nlu = s.nslj = 0;
    int nslast = 0;
    s.hu = 0.0;
    s.nqu = 0;
    sys.f(t, y, &s.YH(1, 2) - 1);
    s.nfe = 1;
    for (int i = 1; i <= n; ++i) s.YH(i, 1) = y[i];
    s.nq = 1;
    s.h = 1.0;
    ewset(n, rtol, atol, &s.YH(1, 1) - 1, s.ewt);
    for (int i = 1; i <= n; ++i) {
        if (s.ewt[i] <= 0.0) return -3;
        s.ewt[i] = 1.0 / s.ewt[i];
    }
    int niter = 0;
    if (vhin(s, sys, t, &s.YH(1, 1) - 1, &s.YH(1, 2) - 1, tout, atol, y, s.acor, h0, niter) != 0) return -3;
    s.nfe += niter;
    s.h = h0;
    for (int i = 1; i <= n; ++i) s.YH(i, 2) = h0 * s.YH(i, 2);
    bool first = true;
    int istate = 0;
    for (;;) {
        if (!first) {  // 250
            if (s.nst - nslast >= MXSTEP) {
                istate = -1;
                break;
            }
            ewset(n, rtol, atol, &s.YH(1, 1) - 1, s.ewt);
            bool bad = false;
            for (int i = 1; i <= n; ++i) {
                if (s.ewt[i] <= 0.0) {
                    bad = true;
                    break;
                }
                s.ewt[i] = 1.0 / s.ewt[i];
            }
            if (bad) {
                istate = -6;
                break;
            }
        }
        // 270
        double tolsf = UROUND * vnorm(n, &s.YH(1, 1) - 1, s.ewt);
        if (tolsf > 1.0) {
            istate = s.nst == 0 ? -3 : -2;
            break;
        }
        first = false;
        vstep(s, sys, y);
        if (s.kflag == -1) {
            istate = -4;
            break;
        }
        if (s.kflag == -2) {
            istate = -5;
            break;
        }
        if (s.kflag < 0) {  // -3, -4: not reached with MITER 1 (no preconditioner)
            istate = -5;
            break;
        }
        s.init = 1;
        s.kuth = 0;
        accepted(s.tn, &s.YH(1, 1) - 1);
        if ((s.tn - tout) * s.h < 0.0) continue;  // 310 -> 250
        if (vindy(s, tout, y) != 0) return -3;
        t = tout;
        return 2;
    }
    // 580: the last accepted state
    for (int i = 1; i <= n; ++i) y[i] = s.YH(i, 1);
    t = s.tn;
    return istate;
}

}  // namespace dvode
