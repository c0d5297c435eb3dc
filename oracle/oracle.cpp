// oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement, in FP64 and in the reference's Fortran loop order, of the
// shared_cfd routines on the per-step residual-and-implicit-update path.  It is
// the checker for the CUDA library: only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline / reference arm load it.  The product never calls it.
//
// It exposes the C ABI of include/scfd_b200.h under the prefix orc_ instead of
// scfd_, so one Python driver can run the same case through either library.
//
// Parity status: the reference (Fortran 90, Python 2 generator) cannot be built
// in this image (no Fortran compiler, no python2).  This restatement is pinned
// (a) against the reference's own data fixtures: the byte layout and the
// thermodynamic state of sample/no27.chemkin_reaction/restart.bin (q together
// with the R, gamma, p that the reference stored per cell), and the block
// connectivity of the forward-step samples no06-no09, and (b) by hand
// derivation; it is "restatement-pinned", not binary-pinned.
//
// Every routine cites the reference file:lines it restates.  Array objects keep
// the reference's index ranges (FArr below is a column-major array with Fortran
// lower bounds) so the restatement can be read next to the Fortran.

#include "../include/scfd_b200.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

// ---------------------------------------------------------------------------
// Column-major array with arbitrary lower bounds, like a Fortran array.
// ---------------------------------------------------------------------------
struct FArr {
    std::vector<double> v;
    int rank = 0;
    int lo[5] = {0, 0, 0, 0, 0};
    int ext[5] = {1, 1, 1, 1, 1};
    long str[5] = {0, 0, 0, 0, 0};
    void init(std::initializer_list<std::pair<int, int>> r) {
        rank = (int)r.size();
        long s = 1;
        int k = 0;
        for (auto& p : r) {
            lo[k] = p.first;
            ext[k] = p.second - p.first + 1;
            str[k] = s;
            s *= ext[k];
            ++k;
        }
        v.assign((size_t)s, 0.0);
    }
    inline double& operator()(int a) { return v[a - lo[0]]; }
    inline double& operator()(int a, int b) { return v[(a - lo[0]) + str[1] * (b - lo[1])]; }
    inline double& operator()(int a, int b, int c) {
        return v[(a - lo[0]) + str[1] * (b - lo[1]) + str[2] * (c - lo[2])];
    }
    inline double& operator()(int a, int b, int c, int d) {
        return v[(a - lo[0]) + str[1] * (b - lo[1]) + str[2] * (c - lo[2]) + str[3] * (d - lo[3])];
    }
    inline double& operator()(int a, int b, int c, int d, int e) {
        return v[(a - lo[0]) + str[1] * (b - lo[1]) + str[2] * (c - lo[2]) + str[3] * (d - lo[3]) +
                 str[4] * (e - lo[4])];
    }
    void fill(double x) { std::fill(v.begin(), v.end(), x); }
};

inline double sq(double a) { return a * a; }
inline double fsign(double a, double b) { return b >= 0.0 ? std::fabs(a) : -std::fabs(a); }

const double R_uni = 8.3144621e3;           // store/core/prmtr.f90:4
const double Ru_cgs = 8.3144621e7;          // mod_chem.raw.f90:8
const double invRc = 1.0 / (double)1.987f;  // mod_chem.raw.f90:9 (single-precision literal, quirk Q3)
const double pst = 1.01325e6;               // mod_chem.raw.f90:11
const double n_eps = 1e-40;                 // mod_chem.raw.f90:14
const double loge210 = (double)0.43429448190325f;  // FJ.f90:166 (single-precision literal, quirk Q3)

}  // namespace

struct orc_ctx {
    scfd_desc d{};
    std::string err;
    int np = 0, nY = 0, D = 0, W = 0, nimax = 0, njmax = 0;
    int indxg = 0, indxht = 0, indxR = 0, indxMu = 0;
    int ni[SCFD_MAX_PLANES]{}, nj[SCFD_MAX_PLANES]{};
    bool committed = false, have_chem = false;
    std::vector<int> geo_set;
    std::vector<int32_t> cut;  // 11 ints per record
    std::vector<scfd_bc> bcs;
    scfd_chem ch{};

    // store/core/variable.f90:24-63
    FArr q, qp, qpp, w, DHi, vhi;
    FArr wHli, wHri, wHlj, wHrj, TGi, TGj, Sq, TGvi, TGvj, Svq;
    FArr Vol, Area, dsi, dsj, geojacc, geojaci, geojacj, vni, vnj, xh, rh, x, r;
    FArr dt_mat;
    double dt_grbl = 0.0, tt = 0.0;
    // store/time_scheme/NR/q2d/var_NR.f90 (superset of var_lusgs)
    FArr Ap, Am, Bp, Bm, alpha, dsci, dscj, vnci, vncj, dpdq, dqdt, Dq;
    FArr pre1, pre2, pre_sca, phi;  // store/time_scheme/dual/2d/var_dual.f90
    bool first_dual = true;
    double res1 = 0.0, res = 0.0, omega_last = 0.0;
    // omega before the omega_max cap and res of every inner iteration of the
    // last step (internal_res.dat, time_NR_viscous.f90:87-95)
    double il_omega[SCFD_INNER_LOG] = {}, il_res[SCFD_INNER_LOG] = {};
    long long chem_attempts = 0, chem_fallback = 0;
    int status = SCFD_OK;
    // block sharding (scfd_set_partition): planes owned by this rank, the
    // cells each rank exports to the others' ghost copies, the exchange buffers
    // and the position of a staged step (scfd_dstep)
    int nranks = 1, rank = 0;
    std::vector<int> owner;
    std::vector<std::vector<std::array<int, 3>>> exports;  // per rank: (i, j, plane)
    long long seg = 0;
    std::vector<double> halo, red;
    int ds_stage = 0, ds_j = 0, ds_status = 0;
    long long ds_att0 = 0, ds_fb0 = 0;
    bool own(int p) const { return nranks <= 1 || owner[p - 1] == rank; }  // p 1-based

    int fail(int code, const std::string& m) {
        err = m;
        return code;
    }
    double DTLG(int i, int j, int p) {  // DT_LOCAL_GLOBAL substitution (checkout_flow.py:120-132)
        return d.dt_mode == SCFD_DT_LOCAL ? dt_mat(i, j, p) : dt_grbl;
    }
};

namespace {

// ===========================================================================
// Geometry: store/dim/{2d,q2d}/geometry.f90, LU-SGS set_vnc_dsc, set_geojac
// ===========================================================================
double area_triangle(double a1, double a2, double b1, double b2, double c1, double c2) {
    return 1.0 / 2.0 * (a1 * (b2 - c2) + b1 * (c2 - a2) + c1 * (a2 - b2));  // geometry.f90:170-175
}
double dis_point(double x1, double y1, double x2, double y2) {
    return std::sqrt(sq(x1 - x2) + sq(y1 - y2));  // geometry.f90:176-181
}

void set_xr(orc_ctx& c) {  // geometry.f90:79-106, with quirk Q1 (lines 95-96, 102-103)
    auto& x = c.x;
    auto& r = c.r;
    auto& xh = c.xh;
    auto& rh = c.rh;
    for (int p = 1; p <= c.np; ++p) {
        for (int j = 1; j <= c.nj[p - 1]; ++j)
            for (int i = 1; i <= c.ni[p - 1]; ++i) {
                x(i, j, p) = 1.0 / 4.0 * (xh(i - 1, j - 1, p) + xh(i, j - 1, p) + xh(i - 1, j, p) + xh(i, j, p));
                r(i, j, p) = 1.0 / 4.0 * (rh(i - 1, j - 1, p) + rh(i, j - 1, p) + rh(i - 1, j, p) + rh(i, j, p));
            }
        for (int j = 1; j <= c.nj[p - 1]; ++j) {
            x(0, j, p) = 2.0 * x(1, j, p) - x(2, j, p);
            r(0, j, p) = 2.0 * r(1, j, p) - r(2, j, p);
            // x(ni+1,j,plane) with ni the per-plane ARRAY: a vector subscript that
            // writes column ni(k)+1 for every plane k (right side evaluated first).
            int nk = c.d.quirk_q1 ? c.np : 1;
            std::vector<double> vx(nk), vr(nk);
            std::vector<int> col(nk);
            for (int k = 0; k < nk; ++k) {
                int nn = c.d.quirk_q1 ? c.ni[k] : c.ni[p - 1];
                col[k] = nn + 1;
                vx[k] = 2.0 * x(nn, j, p) - x(nn - 1, j, p);
                vr[k] = 2.0 * r(nn, j, p) - r(nn - 1, j, p);
            }
            for (int k = 0; k < nk; ++k) x(col[k], j, p) = vx[k];
            for (int k = 0; k < nk; ++k) r(col[k], j, p) = vr[k];
        }
        for (int i = 0; i <= c.ni[p - 1] + 1; ++i) {
            x(i, 0, p) = 2.0 * x(i, 1, p) - x(i, 2, p);
            r(i, 0, p) = 2.0 * r(i, 1, p) - r(i, 2, p);
            int nk = c.d.quirk_q1 ? c.np : 1;
            std::vector<double> vx(nk), vr(nk);
            std::vector<int> row(nk);
            for (int k = 0; k < nk; ++k) {
                int nn = c.d.quirk_q1 ? c.nj[k] : c.nj[p - 1];
                row[k] = nn + 1;
                vx[k] = 2.0 * x(i, nn, p) - x(i, nn - 1, p);
                vr[k] = 2.0 * r(i, nn, p) - r(i, nn - 1, p);
            }
            for (int k = 0; k < nk; ++k) x(i, row[k], p) = vx[k];
            for (int k = 0; k < nk; ++k) r(i, row[k], p) = vr[k];
        }
    }
}

void init_geometry(orc_ctx& c) {
    set_xr(c);
    const bool q2d = c.d.dim == SCFD_DIM_Q2D;
    auto& xh = c.xh;
    auto& rh = c.rh;
    for (int p = 1; p <= c.np; ++p) {
        int ni = c.ni[p - 1], nj = c.nj[p - 1];
        // set_Area_Vol: 2d geometry.f90:107-122, q2d 117-119
        for (int j = 1; j <= nj; ++j)
            for (int i = 1; i <= ni; ++i) {
                double Aabd = area_triangle(xh(i - 1, j - 1, p), rh(i - 1, j - 1, p), xh(i, j - 1, p),
                                            rh(i, j - 1, p), xh(i - 1, j, p), rh(i - 1, j, p));
                double Abcd = area_triangle(xh(i, j - 1, p), rh(i, j - 1, p), xh(i, j, p), rh(i, j, p),
                                            xh(i - 1, j, p), rh(i - 1, j, p));
                if (q2d) {
                    c.Area(i, j, p) = Aabd + Abcd;
                    c.Vol(i, j, p) = (rh(i - 1, j - 1, p) + rh(i, j - 1, p) + rh(i - 1, j, p)) * Aabd / 3.0 +
                                     (rh(i, j - 1, p) + rh(i, j, p) + rh(i - 1, j, p)) * Abcd / 3.0;
                } else {
                    c.Area(i, j, p) = 0.0;
                    c.Vol(i, j, p) = Aabd + Abcd;
                }
            }
        // set_dsij: geometry.f90:123-140 (q2d multiplies by mean r, 131/137)
        for (int j = 0; j <= nj; ++j)
            for (int i = 1; i <= ni; ++i) {
                double ds = dis_point(xh(i - 1, j, p), rh(i - 1, j, p), xh(i, j, p), rh(i, j, p));
                if (q2d) ds = ds * (rh(i - 1, j, p) + rh(i, j, p)) / 2.0;
                c.dsj(i, j, p) = ds;
            }
        for (int j = 1; j <= nj; ++j)
            for (int i = 0; i <= ni; ++i) {
                double ds = dis_point(xh(i, j - 1, p), rh(i, j - 1, p), xh(i, j, p), rh(i, j, p));
                if (q2d) ds = ds * (rh(i, j - 1, p) + rh(i, j, p)) / 2.0;
                c.dsi(i, j, p) = ds;
            }
        // set_vn: geometry.f90:141-169
        for (int j = 1; j <= nj; ++j)
            for (int i = 0; i <= ni; ++i) {
                double nx = rh(i, j, p) - rh(i, j - 1, p);
                double nr = -(xh(i, j, p) - xh(i, j - 1, p));
                double sd = std::sqrt(sq(nx) + sq(nr));
                c.vni(1, i, j, p) = nx / sd;
                c.vni(2, i, j, p) = nr / sd;
            }
        for (int j = 0; j <= nj; ++j)
            for (int i = 1; i <= ni; ++i) {
                double nx = -(rh(i, j, p) - rh(i - 1, j, p));
                double nr = xh(i, j, p) - xh(i - 1, j, p);
                double sd = std::sqrt(sq(nx) + sq(nr));
                c.vnj(1, i, j, p) = nx / sd;
                c.vnj(2, i, j, p) = nr / sd;
            }
        // set_vnc_dsc: LU-SGS/q2d/sch_lusgs.raw.f90:151-187 (2d omits the r scaling)
        for (int j = 1; j <= nj; ++j)
            for (int i = 1; i <= ni; ++i) {
                double a1 = (xh(i - 1, j - 1, p) + xh(i, j - 1, p)) * 0.5, a2 = (rh(i - 1, j - 1, p) + rh(i, j - 1, p)) * 0.5;
                double b1 = (xh(i, j - 1, p) + xh(i, j, p)) * 0.5, b2 = (rh(i, j - 1, p) + rh(i, j, p)) * 0.5;
                double c1 = (xh(i - 1, j, p) + xh(i, j, p)) * 0.5, c2 = (rh(i - 1, j, p) + rh(i, j, p)) * 0.5;
                double d1 = (xh(i - 1, j - 1, p) + xh(i - 1, j, p)) * 0.5, d2 = (rh(i - 1, j - 1, p) + rh(i - 1, j, p)) * 0.5;
                double dci = std::sqrt(sq(c1 - a1) + sq(c2 - a2));
                double dcj = std::sqrt(sq(b1 - d1) + sq(b2 - d2));
                c.vnci(1, i, j, p) = (b1 - d1) / dcj;
                c.vnci(2, i, j, p) = (b2 - d2) / dcj;
                c.vncj(1, i, j, p) = (c1 - a1) / dci;
                c.vncj(2, i, j, p) = (c2 - a2) / dci;
                if (q2d) {
                    dci = dci * (c2 + a2) * 0.5;
                    dcj = dcj * (b2 + d2) * 0.5;
                }
                c.dsci(i, j, p) = dci;
                c.dscj(i, j, p) = dcj;
            }
        // set_geojac: viscous/no-nV/q2d/sch_viscous.f90:1-73
        auto& x = c.x;
        auto& r = c.r;
        for (int j = 1; j <= nj; ++j)
            for (int i = 1; i <= ni; ++i) {
                double dxdxi = (x(i + 1, j, p) - x(i - 1, j, p)) * 0.5;
                double dydxi = (r(i + 1, j, p) - r(i - 1, j, p)) * 0.5;
                double dxdeta = (x(i, j + 1, p) - x(i, j - 1, p)) * 0.5;
                double dydeta = (r(i, j + 1, p) - r(i, j - 1, p)) * 0.5;
                double det = dxdxi * dydeta - dydxi * dxdeta;
                c.geojacc(1, 1, i, j, p) = dydeta / det;
                c.geojacc(1, 2, i, j, p) = -dxdeta / det;
                c.geojacc(2, 1, i, j, p) = -dydxi / det;
                c.geojacc(2, 2, i, j, p) = dxdxi / det;
            }
        for (int j = 1; j <= nj; ++j)
            for (int i = 0; i <= ni; ++i) {
                double dxdxi = x(i + 1, j, p) - x(i, j, p);
                double dydxi = r(i + 1, j, p) - r(i, j, p);
                double dxdeta = (x(i + 1, j + 1, p) + x(i, j + 1, p) - x(i + 1, j - 1, p) - x(i, j - 1, p)) * 0.25;
                double dydeta = (r(i + 1, j + 1, p) + r(i, j + 1, p) - r(i + 1, j - 1, p) - r(i, j - 1, p)) * 0.25;
                double det = dxdxi * dydeta - dydxi * dxdeta;
                c.geojaci(1, 1, i, j, p) = dydeta / det;
                c.geojaci(1, 2, i, j, p) = -dxdeta / det;
                c.geojaci(2, 1, i, j, p) = -dydxi / det;
                c.geojaci(2, 2, i, j, p) = dxdxi / det;
            }
        for (int j = 0; j <= nj; ++j)
            for (int i = 1; i <= ni; ++i) {
                double dxdxi = (x(i + 1, j + 1, p) + x(i + 1, j, p) - x(i - 1, j + 1, p) - x(i - 1, j, p)) * 0.25;
                double dydxi = (r(i + 1, j + 1, p) + r(i + 1, j, p) - r(i - 1, j + 1, p) - r(i - 1, j, p)) * 0.25;
                double dxdeta = x(i, j + 1, p) - x(i, j, p);
                double dydeta = r(i, j + 1, p) - r(i, j, p);
                double det = dxdxi * dydeta - dydxi * dxdeta;
                c.geojacj(1, 1, i, j, p) = dydeta / det;
                c.geojacj(1, 2, i, j, p) = -dxdeta / det;
                c.geojacj(2, 1, i, j, p) = -dydxi / det;
                c.geojacj(2, 2, i, j, p) = dxdxi / det;
            }
    }
}

// ===========================================================================
// Chemkin thermodynamics: store/therm_lib/chemkin/core/sub_chem.f90
// ===========================================================================
inline int sec_of(const scfd_chem& ch, int k, double T) {  // check_section_number, sub_chem.f90:3-19
    return T <= ch.tthre[k][2] ? 0 : 1;
}

// calc_T, sub_chem.f90:1507-1645.  n over ns (= ns_tocalc for reactive flow).
// Returns 0 or SCFD_E_TNEWTON.
int calc_T(const scfd_chem& ch, const double* vrho, double rho, double E, double& T, double& kappa,
           double& MWave, double* DHi, double* vhi, double& mu) {
    const int ns = ch.ns;
    double n[SCFD_MAX_SPECIES];
    double tmp = rho * 1e-11;
    for (int j = 0; j < ns; ++j) n[j] = vrho[j] > tmp ? vrho[j] * (1.0 / ch.mws[j]) * 1e-3 : 0.0;
    double Eobj = E * 1e1 * rho / Ru_cgs;
    int k = 1;
    const int max_T_loop = 1000;
    double cvnow = 0.0;
    int sec[SCFD_MAX_SPECIES];
    double chrt[6], ccpr[6];
    for (;;) {
        for (int j = 0; j < ns; ++j) sec[j] = sec_of(ch, j, T);
        // set_coeff_less, sub_chem.f90:20-49
        double Ti1 = 1.0 / T, T2 = T * T, T3 = T2 * T, T4 = T3 * T;
        chrt[0] = 1.0; chrt[1] = T / 2.0; chrt[2] = T2 / 3.0; chrt[3] = T3 / 4.0; chrt[4] = T4 / 5.0; chrt[5] = Ti1;
        ccpr[0] = 1.0; ccpr[1] = T; ccpr[2] = T2; ccpr[3] = T3; ccpr[4] = T4; ccpr[5] = 0.0;
        double Enow = 0.0;
        cvnow = 0.0;
        for (int j = 0; j < ns; ++j) {
            if (n[j] > 0.0) {
                double de = -1.0, dcv = -1.0;
                for (int i = 0; i < 6; ++i) {
                    de = de + ch.coeff[j][sec[j]][i] * chrt[i];
                    dcv = dcv + ch.coeff[j][sec[j]][i] * ccpr[i];
                }
                Enow = Enow + de * n[j];
                cvnow = cvnow + dcv * n[j];
            }
        }
        double dT = (Eobj - Enow * T) / cvnow;
        if (std::fabs(dT) < 1e-8 || (std::fabs(dT) < 1e-4 && std::fabs(T - 1e3) < 1e-4) || k > max_T_loop) break;
        T = std::max(100.0, T + dT);
        k = k + 1;
    }
    if (k > max_T_loop) return SCFD_E_TNEWTON;
    double sn = 0.0;
    for (int j = 0; j < ns; ++j) sn = sn + n[j];
    kappa = 1.0 + sn / cvnow;
    MWave = rho / sn * 1e-3;
    tmp = Ru_cgs * 1e-4 * T;
    for (int j = 0; j < ns; ++j) {
        double dh = 0.0;
        for (int i = 0; i < 6; ++i) dh = dh + ch.coeff[j][sec[j]][i] * chrt[i];
        DHi[j] = tmp * (1.0 / ch.mws[j]) * (kappa - (kappa - 1.0) * dh);
        vhi[j] = tmp * (1.0 / ch.mws[j]) * dh;
    }
    // Wilke mixture viscosity, sub_chem.f90:1602-1633
    int tsec[SCFD_MAX_SPECIES];
    for (int i = 0; i < ch.nt; ++i) {  // check_section_number_trans, sub_chem.f90:150-171
        tsec[i] = -1;
        if (ch.trange_trans[i][0][0] > T) tsec[i] = 0;
        for (int l = 0; l < ch.num_sctn_trans[i]; ++l)
            if (ch.trange_trans[i][l][1] > T) {
                tsec[i] = l;
                break;
            }
        if (tsec[i] == -1) tsec[i] = ch.num_sctn_trans[i] - 1;
    }
    double logT = std::log(T), invT = 1.0 / T;
    double cmu[4] = {logT, invT, invT * invT, 1.0};
    double muN[SCFD_MAX_SPECIES];
    for (int i = 0; i < ch.nt; ++i) {
        if (n[ch.tr2th[i]] > 0.0) {
            double t = 0.0;
            for (int j = 0; j < 4; ++j) t = t + cmu[j] * ch.trans[i][tsec[i]][j];
            muN[i] = std::exp(t);
        } else {
            muN[i] = 0.0;
        }
    }
    mu = 0.0;
    for (int i = 0; i < ch.nt; ++i) {
        if (muN[i] > 0.0) {
            int it = ch.tr2th[i];
            double denom = 0.0;
            for (int j = 0; j < ch.nt; ++j) {
                if (muN[j] > 0.0) {
                    int jt = ch.tr2th[j];
                    double phi = 0.25 * sq(1.0 + std::sqrt(muN[i] / muN[j]) * std::pow(ch.mws[jt] / ch.mws[it], 0.25)) *
                                 std::sqrt(2.0 * ch.mws[jt] / (ch.mws[it] + ch.mws[jt]));
                    denom = denom + n[jt] * phi;
                }
            }
            mu = mu + n[it] * muN[i] / denom;
        }
    }
    mu = mu * 1e-7;
    return 0;
}

// Fex_var, store/therm_lib/chemkin/uvhp/uv/FJ.f90:301-453 (UV, constant volume).
void fex_var(const scfd_chem& ch, const double* n, double* dndtp, double* dndtm) {
    const int ns = ch.ns;
    double T = n[ns];
    double logT = std::log(T), Tinv = 1.0 / T;
    double logPRT = std::log(pst / Ru_cgs) - logT;
    double sn = 0.0;
    for (int j = 0; j < ns; ++j) sn += n[j];
    double logsn = std::log(sn);
    double cmurt[7], chrt[7], ccpr[7];
    double T2 = T * T, T3 = T2 * T, T4 = T3 * T;
    cmurt[0] = (1.0 - logT); cmurt[1] = -T / 2.0; cmurt[2] = -T2 / 6.0; cmurt[3] = -T3 / 12.0;
    cmurt[4] = -T4 / 20.0; cmurt[5] = Tinv; cmurt[6] = -1.0;
    chrt[0] = 1.0; chrt[1] = T / 2.0; chrt[2] = T2 / 3.0; chrt[3] = T3 / 4.0; chrt[4] = T4 / 5.0; chrt[5] = Tinv; chrt[6] = 0.0;
    ccpr[0] = 1.0; ccpr[1] = T; ccpr[2] = T2; ccpr[3] = T3; ccpr[4] = T4; ccpr[5] = 0.0; ccpr[6] = 0.0;
    double vmu0rt[SCFD_MAX_SPECIES], vert[SCFD_MAX_SPECIES], vcvr[SCFD_MAX_SPECIES];
    for (int j = 0; j < ns; ++j) {
        int s = sec_of(ch, j, T);
        double t1 = 0.0, t2 = -1.0, t3 = -1.0;
        for (int i = 0; i < 7; ++i) {
            double cf = ch.coeff[j][s][i];
            t1 = t1 + cf * cmurt[i];
            t2 = t2 + cf * chrt[i];
            t3 = t3 + cf * ccpr[i];
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
        if (ch.exist_m[i]) {
            double tmp = sn;
            for (int j = 0; j < ch.numm[i]; ++j) tmp = tmp + ch.men[i][j] * n[ch.indm[i][j]];
            vlogM = (tmp == sn) ? logsn : std::log(tmp);
        }
        double vlogk1 = ch.abe[i][0] + ch.abe[i][1] * logT - ch.abe[i][2] * Tinv;
        double vlogk2 = 0.0;
        if (ch.rstate[i][1] >= 4) vlogk1 = vlogk1 + vlogM;
        if (ch.rstate[i][0] == 0) {
            if (ch.rstate[i][1] == 1 || ch.rstate[i][1] == 5) {
                vlogk2 = ch.cabe[i][0] + ch.cabe[i][1] * logT - ch.cabe[i][2] * Tinv;
                if (ch.rstate[i][1] == 5) vlogk2 = vlogk2 + vlogM;
            } else {
                if (ch.rstate[i][1] == 2 || ch.rstate[i][1] == 3) {
                    double logk0 = ch.cabe[i][0] + ch.cabe[i][1] * logT - ch.cabe[i][2] * Tinv;
                    double logkinf = vlogk1;
                    double log_Pr = logk0 - logkinf + vlogM;
                    double Pr = std::exp(log_Pr);
                    vlogk1 = logkinf + std::log(Pr / (1.0 + Pr));
                    if (ch.rstate[i][1] == 3) {
                        double aa = ch.troe[i][0];
                        double logFcent = std::log10((1.0 - aa) * std::exp(-T * ch.troe[i][1]) +
                                                     aa * std::exp(-T * ch.troe[i][2]) + std::exp(-Tinv * ch.troe[i][3]));
                        double cc = -0.4 - 0.67 * logFcent;
                        double nn = 0.75 - 1.27 * logFcent;
                        double logPrc = log_Pr * loge210 + cc;
                        double logF = 1.0 / (1.0 + sq(logPrc / (nn - dd * logPrc))) * logFcent;
                        vlogk1 = vlogk1 + logF / loge210;
                    }
                }
                double t1 = 0.0;
                for (int k = 0; k < ch.numnu[i][0]; ++k) t1 = t1 - vmu0rt[ch.indnu[i][0][k]];
                for (int k = 0; k < ch.numnu[i][1]; ++k) t1 = t1 + vmu0rt[ch.indnu[i][1][k]];
                vlogk2 = vlogk1 - ch.snu[i] * logPRT + t1;
            }
        }
        double r = std::exp(vlogk1);
        for (int k = 0; k < ch.numnu[i][0]; ++k) r = r * n[ch.indnu[i][0][k]];
        for (int k = 0; k < ch.numnu[i][0]; ++k) {
            int it = ch.indnu[i][0][k];
            dndtm[it] = dndtm[it] - r;
        }
        for (int k = 0; k < ch.numnu[i][1]; ++k) {
            int it = ch.indnu[i][1][k];
            dndtp[it] = dndtp[it] + r;
        }
        if (ch.rstate[i][0] == 0) {
            r = std::exp(vlogk2);
            for (int k = 0; k < ch.numnu[i][1]; ++k) r = r * n[ch.indnu[i][1][k]];
            for (int k = 0; k < ch.numnu[i][0]; ++k) {
                int it = ch.indnu[i][0][k];
                dndtp[it] = dndtp[it] + r;
            }
            for (int k = 0; k < ch.numnu[i][1]; ++k) {
                int it = ch.indnu[i][1][k];
                dndtm[it] = dndtm[it] - r;
            }
        }
    }
    double de = 0.0, cv = 0.0;
    for (int j = 0; j < ns; ++j) {
        de = de + vert[j] * (dndtp[j] + dndtm[j]);
        cv = cv + vcvr[j] * n[j];
    }
    dndtp[ns] = std::max(-de * T / cv, 0.0);
    dndtm[ns] = std::min(-de * T / cv, 0.0);
}

// Fex (J == nullptr; FJ.f90:152-300) or Jex (FJ.f90:454-709): net rates dndt of
// the species and dT/dt at constant volume, and with J the exact Jacobian,
// row-major (ns+1) x (ns+1), J[i*(ns+1)+j] = d dndt_i / d n_j (T last).  The
// T-derivative coefficients are those of set_coeff_more (sub_chem.f90:91-150).
void fex_jex(const scfd_chem& ch, const double* n, double* dndt, double* J) {
    const int ns = ch.ns, N = ns + 1;
    const bool jac = J != nullptr;
    const double T = n[ns];
    const double logT = std::log(T), Tinv = 1.0 / T;
    const double logPRT = std::log(pst / Ru_cgs) - logT;
    double sn = 0.0;
    for (int j = 0; j < ns; ++j) sn += n[j];
    if (jac) sn = std::max(sn, 1e-300);
    const double logsn = std::log(sn);
    const double Ti2 = Tinv * Tinv, T2 = T * T, T3 = T2 * T, T4 = T3 * T;
    const double cmurt[7] = {1.0 - logT, -T / 2.0, -T2 / 6.0, -T3 / 12.0, -T4 / 20.0, Tinv, -1.0};
    const double chrt[7] = {1.0, T / 2.0, T2 / 3.0, T3 / 4.0, T4 / 5.0, Tinv, 0.0};
    const double ccpr[7] = {1.0, T, T2, T3, T4, 0.0, 0.0};
    const double cdmurt[7] = {-Tinv, -1.0 / 2.0, -T / 3.0, -T2 / 4.0, -T3 / 5.0, -Ti2, 0.0};
    const double cdcpr[7] = {0.0, 1.0, 2.0 * T, 3.0 * T2, 4.0 * T3, 0.0, 0.0};
    double vmu0rt[SCFD_MAX_SPECIES], vdmu0rt[SCFD_MAX_SPECIES], vert[SCFD_MAX_SPECIES], vcvr[SCFD_MAX_SPECIES],
        vdcvrdT[SCFD_MAX_SPECIES];
    for (int j = 0; j < ns; ++j) {
        const int s = sec_of(ch, j, T);
        double t1 = 0.0, t2 = 0.0, t3 = -1.0, t4 = -1.0, t5 = 0.0;
        for (int i = 0; i < 7; ++i) {
            const double tmp = ch.coeff[j][s][i];
            t1 = t1 + tmp * cmurt[i];
            t2 = t2 + tmp * cdmurt[i];
            t3 = t3 + tmp * chrt[i];
            t4 = t4 + tmp * ccpr[i];
            t5 = t5 + tmp * cdcpr[i];
        }
        vmu0rt[j] = t1;
        vdmu0rt[j] = t2;
        vert[j] = t3;
        vcvr[j] = t4;
        vdcvrdT[j] = t5;
        dndt[j] = 0.0;
        if (jac)
            for (int i = 0; i < N; ++i) J[j * N + i] = 0.0;
    }
    const double dd = 0.14;
    double vM = 0.0, vlogM = 0.0, dlnkdlnM = 0.0;
    double drdn[SCFD_MAX_SPECIES + 1];
    for (int i = 0; i < ch.nr; ++i) {
        if (ch.exist_m[i]) {
            double tmp = sn;
            for (int j = 0; j < ch.numm[i]; ++j) tmp = tmp + ch.men[i][j] * n[ch.indm[i][j]];
            vM = tmp;
            vlogM = (tmp == sn) ? logsn : std::log(tmp);
        }
        double vlogk1 = ch.abe[i][0] + ch.abe[i][1] * logT - ch.abe[i][2] * Tinv;
        double dlnkdT1 = (ch.abe[i][1] + ch.abe[i][2] * Tinv) * Tinv;
        double vlogk2 = 0.0, dlnkdT2 = 0.0;
        if (ch.rstate[i][1] >= 4) {
            vlogk1 = vlogk1 + vlogM;
            dlnkdlnM = 1.0;
        }
        if (ch.rstate[i][0] == 0) {
            if (ch.rstate[i][1] == 1 || ch.rstate[i][1] == 5) {
                vlogk2 = ch.cabe[i][0] + ch.cabe[i][1] * logT - ch.cabe[i][2] * Tinv;
                dlnkdT2 = (ch.cabe[i][1] + ch.cabe[i][2] * Tinv) * Tinv;
                if (ch.rstate[i][1] == 5) vlogk2 = vlogk2 + vlogM;
            } else {
                if (ch.rstate[i][1] == 2 || ch.rstate[i][1] == 3) {
                    const double logk0 = ch.cabe[i][0] + ch.cabe[i][1] * logT - ch.cabe[i][2] * Tinv;
                    const double dlnk0dT = (ch.cabe[i][1] + ch.cabe[i][2] * Tinv) * Tinv;
                    const double logkinf = vlogk1, dlnkinfdT = dlnkdT1;
                    const double log_Pr = logk0 - logkinf + vlogM;
                    const double Pr = std::exp(log_Pr);
                    vlogk1 = logkinf + std::log(Pr / (1.0 + Pr));
                    dlnkdT1 = (dlnk0dT + Pr * dlnkinfdT) / (1.0 + Pr);
                    dlnkdlnM = 1.0 / (1.0 + Pr);
                    if (ch.rstate[i][1] == 3) {
                        const double dlnPrdT = dlnk0dT - dlnkinfdT;
                        const double aa = ch.troe[i][0];
                        const double Fcent = (1.0 - aa) * std::exp(-T * ch.troe[i][1]) +
                                             aa * std::exp(-T * ch.troe[i][2]) + std::exp(-ch.troe[i][3] * Tinv);
                        const double dFcentdT = -(1.0 - aa) * ch.troe[i][1] * std::exp(-T * ch.troe[i][1]) -
                                                aa * ch.troe[i][2] * std::exp(-T * ch.troe[i][2]) +
                                                ch.troe[i][3] * sq(Tinv) * std::exp(-ch.troe[i][3] * Tinv);
                        const double dlnFcentdT = dFcentdT / Fcent;
                        const double logFcent = std::log10(Fcent);
                        const double cc = -0.4 - 0.67 * logFcent;
                        const double nn = 0.75 - 1.27 * logFcent;
                        const double logPrc = log_Pr * loge210 + cc;
                        const double temp1 = logPrc / (nn - dd * logPrc);
                        const double temp2 = 1.0 / (1.0 + sq(temp1));
                        const double logF = temp2 * logFcent;
                        vlogk1 = vlogk1 + logF / loge210;
                        dlnkdT1 = dlnkdT1 + temp2 * (-2.0 * logF * temp1 / sq(nn - dd * logPrc) *
                                                         (nn * dlnPrdT + (1.27 * logPrc - 0.67 * nn) * dlnFcentdT) +
                                                     dlnFcentdT);
                        dlnkdlnM = dlnkdlnM - 2.0 * temp2 * logF * temp1 / sq(nn - dd * logPrc) * nn;
                    }
                }
                double numu0rt = 0.0, nudmu0rt = 0.0;
                for (int k = 0; k < ch.numnu[i][0]; ++k) {
                    numu0rt = numu0rt - vmu0rt[ch.indnu[i][0][k]];
                    nudmu0rt = nudmu0rt - vdmu0rt[ch.indnu[i][0][k]];
                }
                for (int k = 0; k < ch.numnu[i][1]; ++k) {
                    numu0rt = numu0rt + vmu0rt[ch.indnu[i][1][k]];
                    nudmu0rt = nudmu0rt + vdmu0rt[ch.indnu[i][1][k]];
                }
                vlogk2 = vlogk1 - ch.snu[i] * logPRT + numu0rt;
                dlnkdT2 = dlnkdT1 + ch.snu[i] * Tinv + nudmu0rt;
            }
        }
        for (int k = 0; k < ns; ++k) drdn[k] = 0.0;
        double r = std::exp(vlogk1);
        for (int k = 0; k < ch.numnu[i][0]; ++k) r = r * n[ch.indnu[i][0][k]];
        double Dr = r;
        drdn[ns] = dlnkdT1 * r;
        for (int k = 0; k < ch.numnu[i][0]; ++k) {
            const int it = ch.indnu[i][0][k];
            drdn[it] = drdn[it] + r / n[it];
        }
        if (ch.rstate[i][0] == 0) {
            r = std::exp(vlogk2);
            for (int k = 0; k < ch.numnu[i][1]; ++k) r = r * n[ch.indnu[i][1][k]];
            Dr = Dr - r;
            drdn[ns] = drdn[ns] - r * dlnkdT2;
            for (int k = 0; k < ch.numnu[i][1]; ++k) {
                const int it = ch.indnu[i][1][k];
                drdn[it] = drdn[it] - r / n[it];
            }
        }
        if (ch.exist_m[i]) {
            const double temp1 = Dr * dlnkdlnM / vM;
            for (int k = 0; k < ns; ++k) drdn[k] = drdn[k] + temp1;
            for (int k = 0; k < ch.numm[i]; ++k) drdn[ch.indm[i][k]] = drdn[ch.indm[i][k]] + temp1 * ch.men[i][k];
        }
        for (int k = 0; k < ch.numnu[i][0]; ++k) {
            const int it = ch.indnu[i][0][k];
            dndt[it] = dndt[it] - Dr;
            if (jac)
                for (int j = 0; j < N; ++j) J[it * N + j] = J[it * N + j] - drdn[j];
        }
        for (int k = 0; k < ch.numnu[i][1]; ++k) {
            const int it = ch.indnu[i][1][k];
            dndt[it] = dndt[it] + Dr;
            if (jac)
                for (int j = 0; j < N; ++j) J[it * N + j] = J[it * N + j] + drdn[j];
        }
    }
    double de = 0.0, cv = 0.0, dcv = 0.0, temp1 = 0.0, temp2 = 0.0;
    for (int j = 0; j < ns; ++j) {
        if (jac) temp1 = temp1 + vert[j] * J[j * N + ns];
        de = de + vert[j] * dndt[j];
        dcv = dcv + vcvr[j] * dndt[j];
        cv = cv + vcvr[j] * n[j];
        temp2 = temp2 + vdcvrdT[j] * n[j];
    }
    dndt[ns] = -de * T / cv;
    if (!jac) return;
    J[ns * N + ns] = -(T * temp1 + dcv + dndt[ns] * temp2) / cv;
    for (int j = 0; j < ns; ++j) {
        double t = 0.0;
        for (int k = 0; k < ns; ++k) t = t + vert[k] * J[k * N + j];
        J[ns * N + j] = -(T * t + dndt[ns] * vcvr[j]) / cv;
    }
}

}  // namespace

namespace {

// Ignition delay of reaction_one_steps (sub_chem.f90:1467-1472), taken after
// every accepted substep: the first time T >= T0 + dT, interpolated linearly
// from the previous accepted substep (initially t = 0, T0).
struct Ignition {
    double T0, dT, t_old, T_old, t_ign;
    bool ignited;
    double t_off;  // time at the start of the current reaction_chemeq2 call
};

void track_ignition(Ignition& g, double tt, double T) {
    const double t = g.t_off + tt;
    const double Tig = g.T0 + g.dT;
    if (!g.ignited && T >= Tig) {
        g.t_ign = t - (T - Tig) / (T - g.T_old) * (t - g.t_old);
        g.ignited = true;
    }
    g.T_old = T;
    g.t_old = t;
}

#include "dvode.h"

// Rest of an interval after 10 CHEMEQ2 attempts, sub_chem.f90:1755-1775: DVODE
// with MF = 21 on Fex and Jex (dvode.h) from (tt, y) to tout, rtol and atol
// of control_chem.inp; ISTATE = -1 (MXSTEP steps taken before tout) restarts
// it from where it stopped, at most max_recalc = 50 times
// (mod_chem.raw.f90:27); any other failure is SCFD_E_CHEM (the reference
// stops).  With `ign`, the ignition test runs after every accepted DVODE step.
int dvode_rest(const scfd_chem& ch, double* y, double tt, double tout, long long& evals, Ignition* ign) {
    const int N = ch.ns + 1;
    struct Sys {
        const scfd_chem& ch;
        long long& evals;
        int N;
        void f(double, const double* yy, double* dy) {
            fex_jex(ch, yy + 1, dy + 1, nullptr);
            ++evals;
        }
        void jac(double, const double* yy, dvode::State& s) {
            double d[SCFD_MAX_SPECIES + 1], J[(SCFD_MAX_SPECIES + 1) * (SCFD_MAX_SPECIES + 1)];
            fex_jex(ch, yy + 1, d, J);
            ++evals;
            for (int i = 0; i < N; ++i)
                for (int j = 0; j < N; ++j) s.A(i + 1, j + 1) = J[i * N + j];
        }
    } sys{ch, evals, N};
    dvode::State st;
    double y1[SCFD_MAX_SPECIES + 2];
    for (int i = 0; i < N; ++i) y1[i + 1] = y[i];
    auto acc = [&](double tn, const double* yh1) {
        if (ign) track_ignition(*ign, tn, yh1[N]);
    };
    double t = tt;
    int nrecalc = 0;
    for (;;) {
        const int istate = dvode::solve(st, sys, N, y1, t, tout, ch.rtol, ch.atol, acc);
        if (istate > 0) break;
        if (istate == -1 && ++nrecalc <= 50) continue;
        for (int i = 0; i < N; ++i) y[i] = y1[i + 1];
        return SCFD_E_CHEM;
    }
    for (int i = 0; i < N; ++i) y[i] = y1[i + 1];
    return 0;
}

// chemeq2, sub_chem.f90:1714-1819; returns 0, or SCFD_E_CHEM.  With `ign`,
// the ignition test runs after every accepted substep; `evals` counts the
// source-term evaluations.
int chemeq2(const scfd_chem& ch, double* y, double tt, double tout, double rtol, long long& attempts,
            bool& fell_back, int max_substeps, Ignition* ign = nullptr, long long* evals = nullptr) {
    long long ev_local = 0;
    long long& ev = evals ? *evals : ev_local;
    const int ns = ch.ns;
    double y0[SCFD_MAX_SPECIES + 1], yp[SCFD_MAX_SPECIES + 1], p[SCFD_MAX_SPECIES + 1], q[SCFD_MAX_SPECIES + 1],
        p0[SCFD_MAX_SPECIES + 1], q0[SCFD_MAX_SPECIES + 1];
    double dt = tout - tt, ratio = 1e300;
    int countersum = 0;
    int substeps = 0;
    fell_back = false;
    for (;;) {
        for (int i = 0; i <= ns; ++i) y0[i] = y[i];
        double counter = 0.0;
        if (tout - tt < dt) dt = tout - tt;
        for (;;) {
            for (int i = 0; i <= ns; ++i) y[i] = y0[i];
            countersum = countersum + 1;
            // after 10 attempts the rest of the interval goes to DVODE
            // (sub_chem.f90:1755-1775); the cell is counted
            if (countersum > 10) {
                fell_back = true;
                return dvode_rest(ch, y, tt, tout, ev, ign);
            }
            ++attempts;
            ev += 2;
            // predictor
            fex_var(ch, y, q0, p0);
            for (int i = 0; i < ns; ++i) {
                p0[i] = -p0[i] / (y[i] + 1e-300);
                double var = p0[i] * dt, var2 = var * var, var3 = var * var2;
                double alp = (180.0 + 60.0 * var + 11.0 * var2 + var3) / (360.0 + 60.0 * var + 12.0 * var2 + var3);
                yp[i] = y0[i] + dt * (q0[i] - p0[i] * y0[i]) / (1.0 + alp * p0[i] * dt);
            }
            yp[ns] = y0[ns] + dt * (q0[ns] + p0[ns]);
            // corrector
            ratio = 1e300;
            fex_var(ch, yp, q, p);
            for (int i = 0; i < ns; ++i) {
                p[i] = -p[i] / (yp[i] + 1e-300);
                p[i] = 0.5 * (p0[i] + p[i]);
                double var = p[i] * dt, var2 = var * var, var3 = var * var2;
                double alp = (180.0 + 60.0 * var + 11.0 * var2 + var3) / (360.0 + 60.0 * var + 12.0 * var2 + var3);
                q[i] = alp * q[i] + (1.0 - alp) * q0[i];
                y[i] = y0[i] + dt * (q[i] - p[i] * y0[i]) / (1.0 + alp * p[i] * dt);
                var = (y[i] * rtol + rtol * 1e-5) / std::fabs(y[i] - yp[i] + 1e-300);
                ratio = (var < ratio || var != var) ? var : ratio;  // a NaN ratio rejects the attempt
            }
            y[ns] = y0[ns] + 0.5 * dt * (q[ns] + p[ns] + q0[ns] + p0[ns]);
            if (1.0 < ratio) break;
            counter = counter + 1.0;
            dt = dt * std::sqrt(ratio) / counter;
            if (counter > 10.0) return SCFD_E_CHEM;
        }
        tt = tt + dt;
        if (ign) track_ignition(*ign, tt, y[ns]);
        if (tout <= tt) break;
        dt = dt * std::sqrt(ratio);
        if (++substeps > max_substeps) return SCFD_E_CHEM;
    }
    return 0;
}

// ===========================================================================
// Flow routines
// ===========================================================================
void set_w(orc_ctx& c) {  // store/core/scheme.f90:1-29
    const int nY = c.nY;
    for (int p = 1; p <= c.np; ++p) {
        if (!c.own(p)) continue;
#pragma omp parallel for
        for (int j = 1; j <= c.nj[p - 1]; ++j)
            for (int i = 1; i <= c.ni[p - 1]; ++i) {
                double tmp = 0.0;
                for (int k = 1; k <= nY; ++k) tmp = tmp + c.q(k, i, j, p);
                c.w(1, i, j, p) = tmp;
                tmp = 1.0 / tmp;
                c.w(2, i, j, p) = c.q(nY + 1, i, j, p) * tmp;
                c.w(3, i, j, p) = c.q(nY + 2, i, j, p) * tmp;
                for (int k = 1; k <= nY; ++k) c.w(k + 4, i, j, p) = c.q(k, i, j, p) * tmp;
            }
    }
}

int set_thermo_prop(orc_ctx& c) {
    const int nY = c.nY;
    if (c.d.thermo == SCFD_THERMO_IDEAL) {  // store/therm_lib/ideal/thermal_model.raw.f90:7-33
        const double kg = c.d.kappa, Rg = c.d.rgas, nu = c.d.nu_gas;
        for (int p = 1; p <= c.np; ++p) {
            if (!c.own(p)) continue;
#pragma omp parallel for
            for (int j = 1; j <= c.nj[p - 1]; ++j)
                for (int i = 1; i <= c.ni[p - 1]; ++i) {
                    double ei = c.q(nY + 3, i, j, p) / c.w(1, i, j, p) - 0.5 * (sq(c.w(2, i, j, p)) + sq(c.w(3, i, j, p)));
                    double T = ei * (kg - 1.0) / Rg;
                    c.w(4, i, j, p) = c.w(1, i, j, p) * Rg * T;
                    c.w(c.indxg, i, j, p) = kg;
                    c.w(c.indxht, i, j, p) = (c.q(nY + 3, i, j, p) + c.w(4, i, j, p)) / c.w(1, i, j, p);
                    if (c.d.mu_model == SCFD_MU_SUTHERLAND) {
                        // Sutherland law (replaces mu = rho*nu for the flat-plate configuration)
                        c.w(c.indxMu, i, j, p) = c.d.suth_mu0 * std::pow(T / c.d.suth_t0, 1.5) *
                                                 (c.d.suth_t0 + c.d.suth_s) / (T + c.d.suth_s);
                    } else {
                        c.w(c.indxMu, i, j, p) = c.w(1, i, j, p) * nu;
                    }
                    c.w(c.indxR, i, j, p) = Rg;
                    for (int k = 1; k <= nY; ++k) c.DHi(k, i, j, p) = 0.0;
                    c.vhi(1, i, j, p) = kg / (kg - 1.0) * Rg * T;
                }
        }
        return 0;
    }
    // chemkin: flow/reactive/thermal_model.f90:13-42 (cold flow is identical with ns_tocalc = ns)
    int st = 0;
    for (int p = 1; p <= c.np; ++p) {
        if (!c.own(p)) continue;
#pragma omp parallel for reduction(max : st)
        for (int j = 1; j <= c.nj[p - 1]; ++j)
            for (int i = 1; i <= c.ni[p - 1]; ++i) {
                double ei = c.q(nY + 3, i, j, p) / c.w(1, i, j, p) - 0.5 * (sq(c.w(2, i, j, p)) + sq(c.w(3, i, j, p)));
                double T = c.w(4, i, j, p) / (c.w(1, i, j, p) * c.w(c.indxR, i, j, p));
                double vrho[SCFD_MAX_SPECIES], DH[SCFD_MAX_SPECIES], vh[SCFD_MAX_SPECIES];
                for (int k = 0; k < nY; ++k) vrho[k] = c.q(k + 1, i, j, p);
                double kappa, MW, mu;
                int s = calc_T(c.ch, vrho, c.w(1, i, j, p), ei, T, kappa, MW, DH, vh, mu);
                if (s) st = std::max(st, s);
                for (int k = 0; k < nY; ++k) {
                    c.DHi(k + 1, i, j, p) = DH[k];
                    c.vhi(k + 1, i, j, p) = vh[k];
                }
                c.w(c.indxMu, i, j, p) = mu;
                c.w(c.indxR, i, j, p) = R_uni / MW;
                c.w(4, i, j, p) = c.w(1, i, j, p) * c.w(c.indxR, i, j, p) * T;
                c.w(c.indxg, i, j, p) = kappa;
                c.w(c.indxht, i, j, p) = (c.q(nY + 3, i, j, p) + c.w(4, i, j, p)) / c.w(1, i, j, p);
            }
    }
    return st;
}

// store/time_step/{global,local}/set_dt.f90, in two parts: set_dt_cells fills
// dt_mat of the owned planes and returns their smallest value, set_dt_apply
// sets dt_grbl and the time from the (global) minimum.
double set_dt_cells(orc_ctx& c) {
    double tmp = 1e300;
    if (c.d.dt_mode == SCFD_DT_FIXED) return tmp;
    for (int p = 1; p <= c.np; ++p) {
        if (!c.own(p)) continue;
#pragma omp parallel for reduction(min : tmp)
        for (int j = 1; j <= c.nj[p - 1]; ++j)
            for (int i = 1; i <= c.ni[p - 1]; ++i) {
                double rho = c.w(1, i, j, p), u = c.w(2, i, j, p), v = c.w(3, i, j, p), pr = c.w(4, i, j, p);
                double a = std::sqrt(c.w(c.indxg, i, j, p) * pr / rho);
                double uds = 0.0, un;
                un = c.vni(1, i, j, p) * u + c.vni(2, i, j, p) * v;
                uds = uds + (std::fabs(un) + a) * c.dsi(i, j, p);
                un = c.vni(1, i - 1, j, p) * u + c.vni(2, i - 1, j, p) * v;
                uds = uds + (std::fabs(un) + a) * c.dsi(i - 1, j, p);
                un = c.vnj(1, i, j, p) * u + c.vnj(2, i, j, p) * v;
                uds = uds + (std::fabs(un) + a) * c.dsj(i, j, p);
                un = c.vnj(1, i, j - 1, p) * u + c.vnj(2, i, j - 1, p) * v;
                uds = uds + (std::fabs(un) + a) * c.dsj(i, j - 1, p);
                c.dt_mat(i, j, p) = c.d.cfl * c.Vol(i, j, p) / std::max(uds, c.w(c.indxMu, i, j, p) / rho);
                if (tmp > c.dt_mat(i, j, p)) tmp = c.dt_mat(i, j, p);
            }
    }
    return tmp;
}

void set_dt_apply(orc_ctx& c, double tmp) {
    if (c.d.dt_mode == SCFD_DT_FIXED) {
        c.dt_grbl = c.d.dt_fixed;
        c.tt = c.tt + c.dt_grbl;
    } else if (c.d.dt_mode == SCFD_DT_GLOBAL) {
        c.dt_grbl = tmp;
        c.tt = c.tt + c.dt_grbl;
    }
}

void set_dt(orc_ctx& c) { set_dt_apply(c, set_dt_cells(c)); }

int proceed_reaction(orc_ctx& c) {  // flow/reactive/thermal_model.f90:45-73 + reaction_chemeq2 1684-1713
    const int ns = c.ch.ns;
    int st = 0;
    long long att = 0, fb = 0;
    const int maxsub = c.d.chem_max_substeps > 0 ? c.d.chem_max_substeps : 1000000;
    for (int p = 1; p <= c.np; ++p) {
        if (!c.own(p)) continue;
#pragma omp parallel for reduction(max : st) reduction(+ : att, fb) schedule(dynamic, 16)
        for (int j = 1; j <= c.nj[p - 1]; ++j)
            for (int i = 1; i <= c.ni[p - 1]; ++i) {
                double T = c.w(4, i, j, p) / c.w(1, i, j, p) / c.w(c.indxR, i, j, p);
                double n[SCFD_MAX_SPECIES + 1];
                for (int k = 0; k < ns; ++k) {
                    n[k] = c.q(k + 1, i, j, p) * (1.0 / c.ch.mws[k]) * 1e-3;
                    n[k] = std::max(n[k], n_eps);
                }
                n[ns] = T;
                long long a = 0;
                bool fbk = false;
                int s = chemeq2(c.ch, n, 0.0, c.dt_grbl, c.ch.rtol, a, fbk, maxsub);
                att += a;
                if (fbk) ++fb;
                if (s) st = std::max(st, s);
                for (int k = 0; k < ns; ++k) {
                    n[k] = std::max(n[k], n_eps);
                    c.q(k + 1, i, j, p) = n[k] * c.ch.mws[k] * 1e3;
                }
            }
    }
    c.chem_attempts += att;
    c.chem_fallback += fb;
    return st;
}

// set_BC: section_exchange (store/cond/no-nV/condition.tail.f90:2-70), the
// boundary descriptors in place of the user loops, set_corners (331-356).
void copy_cell(orc_ctx& c, int id, int jd, int pd, int is, int js, int ps) {
    if (!c.own(pd)) return;
    for (int k = 1; k <= c.W; ++k) c.w(k, id, jd, pd) = c.w(k, is, js, ps);
    for (int k = 1; k <= c.nY; ++k) c.vhi(k, id, jd, pd) = c.vhi(k, is, js, ps);
}

// The copies of section_exchange in the reference's order, as
// f(dst i, j, plane, src i, j, plane).
template <typename F>
void for_each_halo_copy(const orc_ctx& c, F copy_cell) {
    for (size_t n = 0; n < c.cut.size() / 11; ++n) {
        const int32_t* r = &c.cut[n * 11];
        int geo = r[0], width = r[1], order = r[2], p1 = r[3], c1 = r[4], s1 = r[5], pm1 = r[6], p2 = r[7],
            c2 = r[8], s2 = r[9], pm2 = r[10];
        for (int inc = 0; inc <= width - 1; ++inc) {
            int a = s1 + inc, b = s2 + inc * order;
            switch (geo) {
                case 1:  // i-i
                    copy_cell(c1 + pm1, a, p1, c2, b, p2);
                    copy_cell(c1 + pm1 * 2, a, p1, c2 - pm2, b, p2);
                    copy_cell(c2 + pm2, b, p2, c1, a, p1);
                    copy_cell(c2 + pm2 * 2, b, p2, c1 - pm1, a, p1);
                    break;
                case 2:  // i-j
                    copy_cell(c1 + pm1, a, p1, b, c2, p2);
                    copy_cell(c1 + pm1 * 2, a, p1, b, c2 - pm2, p2);
                    copy_cell(b, c2 + pm2, p2, c1, a, p1);
                    copy_cell(b, c2 + pm2 * 2, p2, c1 - pm1, a, p1);
                    break;
                case 3:  // j-i
                    copy_cell(a, c1 + pm1, p1, c2, b, p2);
                    copy_cell(a, c1 + pm1 * 2, p1, c2 - pm2, b, p2);
                    copy_cell(c2 + pm2, b, p2, a, c1, p1);
                    copy_cell(c2 + pm2 * 2, b, p2, a, c1 - pm1, p1);
                    break;
                case 4:  // j-j
                    copy_cell(a, c1 + pm1, p1, b, c2, p2);
                    copy_cell(a, c1 + pm1 * 2, p1, b, c2 - pm2, p2);
                    copy_cell(b, c2 + pm2, p2, a, c1, p1);
                    copy_cell(b, c2 + pm2 * 2, p2, a, c1 - pm1, p1);
                    break;
            }
        }
    }
}

void section_exchange(orc_ctx& c) {
    for_each_halo_copy(c, [&](int id, int jd, int pd, int is, int js, int ps) { copy_cell(c, id, jd, pd, is, js, ps); });
}

void apply_bc(orc_ctx& c, const scfd_bc& b) {
    const int p = b.plane, ni = c.ni[p - 1], nj = c.nj[p - 1];
    if (!c.own(p)) return;
    const int W = c.W, nY = c.nY;
    for (int s = b.first; s <= b.last; ++s) {
        int ib, jb, i1, j1, i2, j2;
        double n1, n2;
        switch (b.side) {
            case SCFD_SIDE_ILO: ib = 1; jb = s; i1 = 0; j1 = s; i2 = -1; j2 = s;
                n1 = c.vni(1, 0, s, p); n2 = c.vni(2, 0, s, p); break;
            case SCFD_SIDE_IHI: ib = ni; jb = s; i1 = ni + 1; j1 = s; i2 = ni + 2; j2 = s;
                n1 = c.vni(1, ni, s, p); n2 = c.vni(2, ni, s, p); break;
            case SCFD_SIDE_JLO: ib = s; jb = 1; i1 = s; j1 = 0; i2 = s; j2 = -1;
                n1 = c.vnj(1, s, 0, p); n2 = c.vnj(2, s, 0, p); break;
            default: ib = s; jb = nj; i1 = s; j1 = nj + 1; i2 = s; j2 = nj + 2;
                n1 = c.vnj(1, s, nj, p); n2 = c.vnj(2, s, nj, p); break;
        }
        switch (b.kind) {
            case SCFD_BC_EXTRAP:
                copy_cell(c, i1, j1, p, ib, jb, p);
                break;
            case SCFD_BC_FIXED:
                for (int k = 1; k <= W; ++k) c.w(k, i1, j1, p) = b.value[k - 1];
                for (int k = 1; k <= nY; ++k) c.vhi(k, i1, j1, p) = b.value[W + k - 1];
                break;
            case SCFD_BC_OUTFLOW_P:
                copy_cell(c, i1, j1, p, ib, jb, p);
                c.w(4, i1, j1, p) = b.value[0];
                break;
            case SCFD_BC_SLIP: {
                copy_cell(c, i1, j1, p, ib, jb, p);
                double u = c.w(2, ib, jb, p), v = c.w(3, ib, jb, p);
                double un = u * n1 + v * n2;
                c.w(2, i1, j1, p) = u - 2.0 * un * n1;
                c.w(3, i1, j1, p) = v - 2.0 * un * n2;
                break;
            }
            case SCFD_BC_NOSLIP:
                copy_cell(c, i1, j1, p, ib, jb, p);
                c.w(2, i1, j1, p) = b.value[0] * 2.0 - c.w(2, ib, jb, p);
                c.w(3, i1, j1, p) = b.value[1] * 2.0 - c.w(3, ib, jb, p);
                break;
            case SCFD_BC_FIXED_PIN: {
                double pin = c.w(4, ib, jb, p);
                for (int k = 1; k <= W; ++k) c.w(k, i1, j1, p) = b.value[k - 1];
                for (int k = 1; k <= nY; ++k) c.vhi(k, i1, j1, p) = b.value[W + k - 1];
                c.w(1, i1, j1, p) = pin * b.value[W + nY] / b.value[W + nY + 1];
                c.w(4, i1, j1, p) = pin;
                break;
            }
        }
        copy_cell(c, i2, j2, p, i1, j1, p);
    }
}

void set_corners(orc_ctx& c) {  // condition.tail.f90:331-356
    for (int p = 1; p <= c.np; ++p)
        for (int pi = -1; pi <= 1 && c.own(p); pi += 2) {
            int i = pi < 0 ? 1 : c.ni[p - 1];
            for (int pj = -1; pj <= 1; pj += 2) {
                int j = pj < 0 ? 1 : c.nj[p - 1];
                for (int k = 1; k <= c.W; ++k)
                    c.w(k, i + pi, j + pj, p) =
                        1.0 / 3.0 * (c.w(k, i, j, p) + c.w(k, i, j + pj, p) + c.w(k, i + pi, j, p));
                for (int k = 1; k <= c.nY; ++k)
                    c.vhi(k, i + pi, j + pj, p) =
                        1.0 / 3.0 * (c.vhi(k, i, j, p) + c.vhi(k, i, j + pj, p) + c.vhi(k, i + pi, j, p));
            }
        }
}

void set_BC(orc_ctx& c) {
    section_exchange(c);
    for (auto& b : c.bcs)
        if (b.side == SCFD_SIDE_ILO || b.side == SCFD_SIDE_IHI) apply_bc(c, b);
    for (auto& b : c.bcs)
        if (b.side == SCFD_SIDE_JLO || b.side == SCFD_SIDE_JHI) apply_bc(c, b);
    set_corners(c);
}

// set_HV MUSCL: store/high_order/muscl/muscl.f90:7-73 (upwind = phi_mus 0,
// store/high_order/upwind/upwind.f90:1-37 gives the same face states).
void set_HV(orc_ctx& c) {
    const int W = c.W;
    const double eps = 1e-300;
    const double phi = c.d.recon == SCFD_RECON_MUSCL ? c.d.phi_mus : 0.0, km = c.d.k_mus;
    for (int p = 1; p <= c.np; ++p) {
        if (!c.own(p)) continue;
        int ni = c.ni[p - 1], nj = c.nj[p - 1];
        FArr dui, dli, duj, dlj;
        dui.init({{1, W}, {0, ni + 1}, {1, nj}});
        dli.init({{1, W}, {0, ni + 1}, {1, nj}});
        duj.init({{1, W}, {1, ni}, {0, nj + 1}});
        dlj.init({{1, W}, {1, ni}, {0, nj + 1}});
#pragma omp parallel for
        for (int j = 1; j <= nj; ++j)
            for (int i = 0; i <= ni + 1; ++i)
                for (int k = 1; k <= W; ++k) {
                    double Du = c.w(k, i + 1, j, p) - c.w(k, i, j, p);
                    double Dl = c.w(k, i, j, p) - c.w(k, i - 1, j, p);
                    double s = (2.0 * Du * Dl) / (sq(Du) + sq(Dl) + eps);
                    dui(k, i, j) = 0.5 * s * ((1.0 + km * s) * Du + (1.0 - km * s) * Dl);
                    dli(k, i, j) = 0.5 * s * ((1.0 + km * s) * Dl + (1.0 - km * s) * Du);
                }
#pragma omp parallel for
        for (int j = 1; j <= nj; ++j)
            for (int i = 0; i <= ni; ++i)
                for (int k = 1; k <= W; ++k) {
                    c.wHli(k, i, j, p) = c.w(k, i, j, p) + phi * 0.5 * dui(k, i, j);
                    c.wHri(k, i, j, p) = c.w(k, i + 1, j, p) - phi * 0.5 * dli(k, i + 1, j);
                }
#pragma omp parallel for
        for (int j = 0; j <= nj + 1; ++j)
            for (int i = 1; i <= ni; ++i)
                for (int k = 1; k <= W; ++k) {
                    double Du = c.w(k, i, j + 1, p) - c.w(k, i, j, p);
                    double Dl = c.w(k, i, j, p) - c.w(k, i, j - 1, p);
                    double s = (2.0 * Du * Dl) / (sq(Du) + sq(Dl) + eps);
                    duj(k, i, j) = 0.5 * s * ((1.0 + km * s) * Du + (1.0 - km * s) * Dl);
                    dlj(k, i, j) = 0.5 * s * ((1.0 + km * s) * Dl + (1.0 - km * s) * Du);
                }
#pragma omp parallel for
        for (int j = 0; j <= nj; ++j)
            for (int i = 1; i <= ni; ++i)
                for (int k = 1; k <= W; ++k) {
                    c.wHlj(k, i, j, p) = c.w(k, i, j, p) + phi * 0.5 * duj(k, i, j);
                    c.wHrj(k, i, j, p) = c.w(k, i, j + 1, p) - phi * 0.5 * dlj(k, i, j + 1);
                }
    }
}

// SLAU face flux: store/core/scheme.f90:71-153 (one face).
void slau_face(const orc_ctx& c, const double* wHl, const double* wHr, const double* vn, double* tg) {
    const int nY = c.nY, D = c.D;
    double phil[SCFD_MAX_SPECIES + 3], phir[SCFD_MAX_SPECIES + 3];
    double rhol = wHl[0], ul = wHl[1], vl = wHl[2], pl = wHl[3], gmmal = wHl[c.indxg - 1];
    for (int k = 0; k < nY; ++k) phil[k] = wHl[4 + k];
    phil[nY] = ul; phil[nY + 1] = vl; phil[nY + 2] = wHl[c.indxht - 1];
    double al = std::sqrt(gmmal * pl / rhol);
    double unl = vn[0] * ul + vn[1] * vl;
    double rhor = wHr[0], ur = wHr[1], vr = wHr[2], pr = wHr[3], gmmar = wHr[c.indxg - 1];
    for (int k = 0; k < nY; ++k) phir[k] = wHr[4 + k];
    phir[nY] = ur; phir[nY + 1] = vr; phir[nY + 2] = wHr[c.indxht - 1];
    double ar = std::sqrt(gmmar * pr / rhor);
    double unr = vn[0] * ur + vn[1] * vr;
    double dp = pr - pl;
    double a_bar = 0.5 * (ar + al);
    double p_bar = 0.5 * (pr + pl);
    double ml = unl / a_bar, mr = unr / a_bar;
    double m_tilde = std::min(1.0, 1.0 / a_bar * std::sqrt(0.5 * (sq(ul) + sq(vl) + sq(ur) + sq(vr))));
    double chi = sq(1.0 - m_tilde);
    double gp = -std::max(std::min(ml, 0.0), -1.0);
    double gm = std::min(std::max(mr, 0.0), 1.0);
    double g = gp * gm;
    double un_bar_abs = (std::fabs(unr) * rhor + std::fabs(unl) * rhol) / (rhor + rhol);
    double un_bar_abs_p = (1.0 - g) * un_bar_abs + g * std::fabs(unl);
    double un_bar_abs_m = (1.0 - g) * un_bar_abs + g * std::fabs(unr);
    double dm = 0.5 * (rhol * (unl + un_bar_abs_p) + rhor * (unr - un_bar_abs_m) - chi / a_bar * dp);
    double betar, betal;
    if (std::fabs(mr) < 1.0) betar = 0.25 * (2.0 + mr) * sq(mr - 1.0);
    else betar = 0.5 * (1.0 - fsign(1.0, mr));
    if (std::fabs(ml) < 1.0) betal = 0.25 * (2.0 - ml) * sq(ml + 1.0);
    else betal = 0.5 * (1.0 + fsign(1.0, ml));
    double p_tilde = p_bar + 0.5 * (betal - betar) * (pl - pr) + (1.0 - chi) * (betar + betal - 1.0) * p_bar;
    for (int k = 0; k < D; ++k) {
        double nk = (k == nY) ? vn[0] : (k == nY + 1 ? vn[1] : 0.0);
        tg[k] = 0.5 * (dm + std::fabs(dm)) * phil[k] + 0.5 * (dm - std::fabs(dm)) * phir[k] + p_tilde * nk;
    }
}

void set_TG(orc_ctx& c) {  // store/core/scheme.f90:31-259
    const int W = c.W, D = c.D;
    for (int p = 1; p <= c.np; ++p) {
        if (!c.own(p)) continue;
        int ni = c.ni[p - 1], nj = c.nj[p - 1];
#pragma omp parallel for
        for (int j = 1; j <= nj; ++j)
            for (int i = 0; i <= ni; ++i) {
                double wl[SCFD_BC_MAXVAL], wr[SCFD_BC_MAXVAL], vn[2], tg[SCFD_MAX_SPECIES + 3];
                for (int k = 0; k < W; ++k) { wl[k] = c.wHli(k + 1, i, j, p); wr[k] = c.wHri(k + 1, i, j, p); }
                vn[0] = c.vni(1, i, j, p); vn[1] = c.vni(2, i, j, p);
                slau_face(c, wl, wr, vn, tg);
                for (int k = 0; k < D; ++k) c.TGi(k + 1, i, j, p) = tg[k];
            }
#pragma omp parallel for
        for (int j = 0; j <= nj; ++j)
            for (int i = 1; i <= ni; ++i) {
                double wl[SCFD_BC_MAXVAL], wr[SCFD_BC_MAXVAL], vn[2], tg[SCFD_MAX_SPECIES + 3];
                for (int k = 0; k < W; ++k) { wl[k] = c.wHlj(k + 1, i, j, p); wr[k] = c.wHrj(k + 1, i, j, p); }
                vn[0] = c.vnj(1, i, j, p); vn[1] = c.vnj(2, i, j, p);
                slau_face(c, wl, wr, vn, tg);
                for (int k = 0; k < D; ++k) c.TGj(k + 1, i, j, p) = tg[k];
            }
    }
}

// set_TGv: store/viscosity/viscous/no-nV/{2d,q2d}/sch_viscous.f90:75-321
void set_TGv(orc_ctx& c) {
    const int nY = c.nY, D = c.D;
    const bool q2d = c.d.dim == SCFD_DIM_Q2D;
    if (!c.d.viscous) {  // store/viscosity/non-viscous/sch_viscous.f90 (init_TGv zeros)
        c.TGvi.fill(0.0); c.TGvj.fill(0.0); c.Svq.fill(0.0);
        return;
    }
    const double Sc = c.d.schmidt, Pr = c.d.prandtl;
    for (int p = 1; p <= c.np; ++p) {
        if (!c.own(p)) continue;
        int ni = c.ni[p - 1], nj = c.nj[p - 1];
        FArr Tdeg;
        Tdeg.init({{0, ni + 1}, {0, nj + 1}});
        for (int j = 0; j <= nj + 1; ++j)
            for (int i = 0; i <= ni + 1; ++i)
                Tdeg(i, j) = c.w(4, i, j, p) / c.w(1, i, j, p) / c.w(c.indxR, i, j, p);
        auto flux = [&](int i, int j, int dir, double* out) {
            // dir 0: i-face between (i,j) and (i+1,j); dir 1: j-face between (i,j),(i,j+1)
            int i2 = dir == 0 ? i + 1 : i, j2 = dir == 0 ? j : j + 1;
            double rho = (c.w(1, i, j, p) + c.w(1, i2, j2, p)) * 0.5;
            double u = (c.w(2, i, j, p) + c.w(2, i2, j2, p)) * 0.5;
            double v = (c.w(3, i, j, p) + c.w(3, i2, j2, p)) * 0.5;
            double gamm = (c.w(c.indxg, i, j, p) + c.w(c.indxg, i2, j2, p)) * 0.5;
            double Rgas = (c.w(c.indxR, i, j, p) + c.w(c.indxR, i2, j2, p)) * 0.5;
            double mu = (c.w(c.indxMu, i, j, p) + c.w(c.indxMu, i2, j2, p)) * 0.5;
            double lhi[SCFD_MAX_SPECIES];
            for (int k = 1; k <= nY; ++k) lhi[k - 1] = (c.vhi(k, i, j, p) + c.vhi(k, i2, j2, p)) * 0.5;
            double Dd = mu / rho / Sc;
            double k_heat = mu * gamm / (gamm - 1.0) * Rgas / Pr;
            double dudxi, dvdxi, dTdxi, dudeta, dvdeta, dTdeta;
            double dwdxi[SCFD_MAX_SPECIES], dwdeta[SCFD_MAX_SPECIES];
            double g11, g12, g21, g22;
            if (dir == 0) {
                dudxi = c.w(2, i + 1, j, p) - c.w(2, i, j, p);
                dvdxi = c.w(3, i + 1, j, p) - c.w(3, i, j, p);
                dTdxi = Tdeg(i + 1, j) - Tdeg(i, j);
                for (int k = 1; k <= nY; ++k) dwdxi[k - 1] = c.w(4 + k, i + 1, j, p) - c.w(4 + k, i, j, p);
                dudeta = (c.w(2, i + 1, j + 1, p) + c.w(2, i, j + 1, p) - c.w(2, i + 1, j - 1, p) - c.w(2, i, j - 1, p)) * 0.25;
                dvdeta = (c.w(3, i + 1, j + 1, p) + c.w(3, i, j + 1, p) - c.w(3, i + 1, j - 1, p) - c.w(3, i, j - 1, p)) * 0.25;
                dTdeta = (Tdeg(i + 1, j + 1) + Tdeg(i, j + 1) - Tdeg(i + 1, j - 1) - Tdeg(i, j - 1)) * 0.25;
                for (int k = 1; k <= nY; ++k)
                    dwdeta[k - 1] = (c.w(4 + k, i + 1, j + 1, p) + c.w(4 + k, i, j + 1, p) - c.w(4 + k, i + 1, j - 1, p) -
                                     c.w(4 + k, i, j - 1, p)) * 0.25;
                g11 = c.geojaci(1, 1, i, j, p); g12 = c.geojaci(1, 2, i, j, p);
                g21 = c.geojaci(2, 1, i, j, p); g22 = c.geojaci(2, 2, i, j, p);
            } else {
                dudxi = (c.w(2, i + 1, j + 1, p) + c.w(2, i + 1, j, p) - c.w(2, i - 1, j + 1, p) - c.w(2, i - 1, j, p)) * 0.25;
                dvdxi = (c.w(3, i + 1, j + 1, p) + c.w(3, i + 1, j, p) - c.w(3, i - 1, j + 1, p) - c.w(3, i - 1, j, p)) * 0.25;
                dTdxi = (Tdeg(i + 1, j + 1) + Tdeg(i + 1, j) - Tdeg(i - 1, j + 1) - Tdeg(i - 1, j)) * 0.25;
                for (int k = 1; k <= nY; ++k)
                    dwdxi[k - 1] = (c.w(4 + k, i + 1, j + 1, p) + c.w(4 + k, i + 1, j, p) - c.w(4 + k, i - 1, j + 1, p) -
                                    c.w(4 + k, i - 1, j, p)) * 0.25;
                dudeta = c.w(2, i, j + 1, p) - c.w(2, i, j, p);
                dvdeta = c.w(3, i, j + 1, p) - c.w(3, i, j, p);
                dTdeta = Tdeg(i, j + 1) - Tdeg(i, j);
                for (int k = 1; k <= nY; ++k) dwdeta[k - 1] = c.w(4 + k, i, j + 1, p) - c.w(4 + k, i, j, p);
                g11 = c.geojacj(1, 1, i, j, p); g12 = c.geojacj(1, 2, i, j, p);
                g21 = c.geojacj(2, 1, i, j, p); g22 = c.geojacj(2, 2, i, j, p);
            }
            double dudx = dudxi * g11 + dudeta * g21;
            double dvdx = dvdxi * g11 + dvdeta * g21;
            double dTdx = dTdxi * g11 + dTdeta * g21;
            double dudr = dudxi * g12 + dudeta * g22;
            double dvdr = dvdxi * g12 + dvdeta * g22;
            double dTdr = dTdxi * g12 + dTdeta * g22;
            double hidwdx = 0.0, hidwdr = 0.0;
            double dwdx[SCFD_MAX_SPECIES], dwdr[SCFD_MAX_SPECIES];
            for (int k = 0; k < nY; ++k) {
                dwdx[k] = dwdxi[k] * g11 + dwdeta[k] * g21;
                hidwdx = hidwdx + dwdx[k] * lhi[k];
                dwdr[k] = dwdxi[k] * g12 + dwdeta[k] * g22;
                hidwdr = hidwdr + dwdr[k] * lhi[k];
            }
            double divu = q2d ? dudx + dvdr + v / c.r(i, j, p) : dudx + dvdr;
            double t_xx = -2.0 / 3.0 * mu * divu + 2.0 * mu * dudx;
            double t_rr = -2.0 / 3.0 * mu * divu + 2.0 * mu * dvdr;
            double t_xr = mu * (dvdx + dudr);
            double qx = -k_heat * dTdx - rho * Dd * hidwdx;
            double qr = -k_heat * dTdr - rho * Dd * hidwdr;
            double Ev[SCFD_MAX_SPECIES + 3], Fv[SCFD_MAX_SPECIES + 3];
            for (int k = 0; k < nY; ++k) { Ev[k] = rho * Dd * dwdx[k]; Fv[k] = rho * Dd * dwdr[k]; }
            Ev[nY] = t_xx; Ev[nY + 1] = t_xr; Ev[nY + 2] = u * t_xx + v * t_xr - qx;
            Fv[nY] = t_xr; Fv[nY + 1] = t_rr; Fv[nY + 2] = u * t_xr + v * t_rr - qr;
            double n1 = dir == 0 ? c.vni(1, i, j, p) : c.vnj(1, i, j, p);
            double n2 = dir == 0 ? c.vni(2, i, j, p) : c.vnj(2, i, j, p);
            for (int k = 0; k < D; ++k) out[k] = Ev[k] * n1 + Fv[k] * n2;
        };
#pragma omp parallel for
        for (int j = 1; j <= nj; ++j)
            for (int i = 0; i <= ni; ++i) {
                double out[SCFD_MAX_SPECIES + 3];
                flux(i, j, 0, out);
                for (int k = 0; k < D; ++k) c.TGvi(k + 1, i, j, p) = out[k];
            }
#pragma omp parallel for
        for (int j = 0; j <= nj; ++j)
            for (int i = 1; i <= ni; ++i) {
                double out[SCFD_MAX_SPECIES + 3];
                flux(i, j, 1, out);
                for (int k = 0; k < D; ++k) c.TGvj(k + 1, i, j, p) = out[k];
            }
        if (q2d) {  // Svq, q2d sch_viscous.f90:291-319
#pragma omp parallel for
            for (int j = 1; j <= nj; ++j)
                for (int i = 1; i <= ni; ++i) {
                    double v = c.w(3, i, j, p), mu = c.w(c.indxMu, i, j, p);
                    double dudxi = (c.w(2, i + 1, j, p) - c.w(2, i - 1, j, p)) * 0.5;
                    double dvdxi = (c.w(3, i + 1, j, p) - c.w(3, i - 1, j, p)) * 0.5;
                    double dudeta = (c.w(2, i, j + 1, p) - c.w(2, i, j - 1, p)) * 0.5;
                    double dvdeta = (c.w(3, i, j + 1, p) - c.w(3, i, j - 1, p)) * 0.5;
                    double dudx = dudxi * c.geojacc(1, 1, i, j, p) + dudeta * c.geojacc(2, 1, i, j, p);
                    double dvdr = dvdxi * c.geojacc(1, 2, i, j, p) + dvdeta * c.geojacc(2, 2, i, j, p);
                    double divu = dudx + dvdr + v / c.r(i, j, p);
                    double t_tt = -2.0 / 3.0 * mu * divu + 2.0 * mu * v / c.r(i, j, p);
                    for (int k = 1; k <= D; ++k) c.Svq(k, i, j, p) = 0.0;
                    c.Svq(nY + 2, i, j, p) = -t_tt;
                }
        }
    }
}

void set_Sq(orc_ctx& c) {  // store/dim/q2d/Sq.f90:1-18 (2d: init_Sq zeros)
    if (c.d.dim != SCFD_DIM_Q2D) return;
    for (int p = 1; p <= c.np; ++p)
        for (int j = 1; j <= c.nj[p - 1] && c.own(p); ++j)
            for (int i = 1; i <= c.ni[p - 1]; ++i) {
                for (int k = 1; k <= c.D; ++k) c.Sq(k, i, j, p) = 0.0;
                c.Sq(c.nY + 2, i, j, p) = c.w(4, i, j, p);
            }
}

inline double rhs_k(orc_ctx& c, int k, int i, int j, int p) {  // e.g. time_lusgs_viscous.f90:16-20
    return c.dsi(i - 1, j, p) * (c.TGi(k, i - 1, j, p) - c.TGvi(k, i - 1, j, p)) -
           c.dsi(i, j, p) * (c.TGi(k, i, j, p) - c.TGvi(k, i, j, p)) +
           c.dsj(i, j - 1, p) * (c.TGj(k, i, j - 1, p) - c.TGvj(k, i, j - 1, p)) -
           c.dsj(i, j, p) * (c.TGj(k, i, j, p) - c.TGvj(k, i, j, p)) +
           c.Area(i, j, p) * (c.Sq(k, i, j, p) + c.Svq(k, i, j, p));
}

void calc_next_step_euler(orc_ctx& c) {  // store/time_scheme/euler/time_euler_viscous.raw.f90:1-23
    for (int p = 1; p <= c.np; ++p) {
        if (!c.own(p)) continue;
#pragma omp parallel for
        for (int j = 1; j <= c.nj[p - 1]; ++j)
            for (int i = 1; i <= c.ni[p - 1]; ++i) {
                double dt = c.DTLG(i, j, p);
                for (int k = 1; k <= c.D; ++k)
                    c.q(k, i, j, p) = c.qp(k, i, j, p) + dt / c.Vol(i, j, p) * rhs_k(c, k, i, j, p);
            }
    }
}

// set_ABpm: LU-SGS/q2d/sch_lusgs.raw.f90:1-149 (alpha with Vol/dt) and
// NR/q2d/sch_NR.raw.f90:1-149 (alpha with 3Vol/(2dt)); dpdq on q2d only.
// set_ABpm of LU-SGS and NR, and of the precon schemes
// (time_scheme/precon/2d/sch_precon.raw.f90:1-202, preconLU-SGS/2d the same
// with alpha from Vol/dt): low-Mach reference velocity Ur, preconditioned
// spectral radii, the local time step written to dt_mat, pre1 = phh (Y, u, v,
// H) with phh = -1/(c^2 + 1/phi), pre2 = (g1 Vs/2 + DHi, -g1 u, -g1 v, g1), and
// the Jacobians premultiplied by I + pre1 pre2^T.
void set_ABpm(orc_ctx& c) {
    const int nY = c.nY, D = c.D;
    const bool nr = c.d.scheme == SCFD_SCHEME_NR || c.d.scheme == SCFD_SCHEME_PRECON;
    const bool q2d = c.d.dim == SCFD_DIM_Q2D;
    const bool pc = c.d.scheme == SCFD_SCHEME_PRECON || c.d.scheme == SCFD_SCHEME_PRECON_LUSGS;
    for (int p = 1; p <= c.np; ++p) {
        if (!c.own(p)) continue;
#pragma omp parallel for
        for (int j = 1; j <= c.nj[p - 1]; ++j)
            for (int i = 1; i <= c.ni[p - 1]; ++i) {
                std::vector<double> A(D * D), B(D * D), tA(D), tB(D);
                auto a = [&](int r, int cc) -> double& { return A[(r - 1) + D * (cc - 1)]; };
                auto b = [&](int r, int cc) -> double& { return B[(r - 1) + D * (cc - 1)]; };
                double rho = c.w(1, i, j, p), u = c.w(2, i, j, p), v = c.w(3, i, j, p), pr = c.w(4, i, j, p);
                double gamm = c.w(c.indxg, i, j, p), H = c.w(c.indxht, i, j, p);
                double cs = std::sqrt(gamm * pr / rho), gmmad = gamm - 1.0, Vs = sq(u) + sq(v);
                double unA = c.vnci(1, i, j, p) * u + c.vnci(2, i, j, p) * v;
                double unB = c.vncj(1, i, j, p) * u + c.vncj(2, i, j, p) * v;
                double nuA = std::fabs(unA) + cs, nuB = std::fabs(unB) + cs;
                if (pc) {
                    const double Vv = c.w(c.indxMu, i, j, p) / rho / std::min(c.dsci(i, j, p), c.dscj(i, j, p));
                    const double Ur = std::min(std::max(Vv, std::sqrt(Vs)), cs);
                    c.phi(i, j, p) = 1.0 / sq(Ur) - 1.0 / sq(cs);
                    const double alp = 0.5 * (1.0 - sq(Ur / cs));
                    double ud = unA * (1.0 - alp), cd = std::sqrt(sq(alp) * sq(unA) + sq(Ur));
                    nuA = std::fabs(ud) + cd;
                    ud = unB * (1.0 - alp);
                    cd = std::sqrt(sq(alp) * sq(unB) + sq(Ur));
                    nuB = std::fabs(ud) + cd;
                    const double uds = nuA * (c.dsi(i, j, p) + c.dsi(i - 1, j, p)) + nuB * (c.dsj(i, j, p) + c.dsj(i, j - 1, p));
                    c.dt_mat(i, j, p) = c.d.cfl * c.Vol(i, j, p) / std::max(uds, c.w(c.indxMu, i, j, p) / rho);
                    const double phh = -1.0 / (sq(cs) + 1.0 / c.phi(i, j, p));
                    for (int k = 1; k <= nY; ++k) c.pre1(k, i, j, p) = phh * c.w(4 + k, i, j, p);
                    c.pre1(nY + 1, i, j, p) = phh * u;
                    c.pre1(nY + 2, i, j, p) = phh * v;
                    c.pre1(nY + 3, i, j, p) = phh * H;
                    for (int k = 1; k <= nY; ++k) c.pre2(k, i, j, p) = 0.5 * gmmad * Vs + c.DHi(k, i, j, p);
                    c.pre2(nY + 1, i, j, p) = -gmmad * u;
                    c.pre2(nY + 2, i, j, p) = -gmmad * v;
                    c.pre2(nY + 3, i, j, p) = gmmad;
                }
                if (q2d) {
                    for (int k = 1; k <= nY; ++k) c.dpdq(k, i, j, p) = 0.5 * gmmad * Vs + c.DHi(k, i, j, p);
                    c.dpdq(nY + 1, i, j, p) = -gmmad * u;
                    c.dpdq(nY + 2, i, j, p) = -gmmad * v;
                    c.dpdq(nY + 3, i, j, p) = gmmad;
                }
                a(nY + 1, nY + 1) = u * (3.0 - gamm); a(nY + 2, nY + 1) = v; a(nY + 3, nY + 1) = H - sq(u) * gmmad;
                a(nY + 1, nY + 2) = -v * gmmad; a(nY + 2, nY + 2) = u; a(nY + 3, nY + 2) = -u * v * gmmad;
                a(nY + 1, nY + 3) = gmmad; a(nY + 2, nY + 3) = 0.0; a(nY + 3, nY + 3) = u * gamm;
                for (int k = 1; k <= nY; ++k) {
                    tA[k - 1] = -c.w(4 + k, i, j, p) * u;
                    a(k, nY + 1) = c.w(4 + k, i, j, p); a(k, nY + 2) = 0.0; a(k, nY + 3) = 0.0;
                }
                tA[nY] = -sq(u) + 0.5 * gmmad * Vs;
                tA[nY + 1] = -u * v;
                tA[nY + 2] = u * (-H + 0.5 * gmmad * Vs);
                b(nY + 1, nY + 1) = v; b(nY + 2, nY + 1) = -u * gmmad; b(nY + 3, nY + 1) = -u * v * gmmad;
                b(nY + 1, nY + 2) = u; b(nY + 2, nY + 2) = v * (3.0 - gamm); b(nY + 3, nY + 2) = H - sq(v) * gmmad;
                b(nY + 1, nY + 3) = 0.0; b(nY + 2, nY + 3) = gmmad; b(nY + 3, nY + 3) = v * gamm;
                for (int k = 1; k <= nY; ++k) {
                    tB[k - 1] = -c.w(4 + k, i, j, p) * v;
                    b(k, nY + 1) = 0.0; b(k, nY + 2) = c.w(4 + k, i, j, p); b(k, nY + 3) = 0.0;
                }
                tB[nY] = -v * u;
                tB[nY + 1] = -sq(v) + 0.5 * gmmad * Vs;
                tB[nY + 2] = v * (-H + 0.5 * gmmad * Vs);
                for (int k = 1; k <= nY; ++k) {
                    for (int l = 1; l <= nY; ++l) { a(l, k) = tA[l - 1]; b(l, k) = tB[l - 1]; }
                    a(k, k) = tA[k - 1] + u;
                    a(nY + 1, k) = tA[nY] + c.DHi(k, i, j, p);
                    a(nY + 2, k) = tA[nY + 1];
                    a(nY + 3, k) = tA[nY + 2] + c.DHi(k, i, j, p) * u;
                    b(k, k) = tB[k - 1] + v;
                    b(nY + 1, k) = tB[nY];
                    b(nY + 2, k) = tB[nY + 1] + c.DHi(k, i, j, p);
                    b(nY + 3, k) = tB[nY + 2] + c.DHi(k, i, j, p) * v;
                }
                if (pc) {  // multiply preM (sch_precon.raw.f90:148-166)
                    for (int k = 1; k <= D; ++k) {
                        double tmp = 0.0;
                        for (int l = 1; l <= D; ++l) tmp = tmp + c.pre2(l, i, j, p) * a(l, k);
                        for (int l = 1; l <= D; ++l) a(l, k) = a(l, k) + c.pre1(l, i, j, p) * tmp;
                    }
                    for (int k = 1; k <= D; ++k) {
                        double tmp = 0.0;
                        for (int l = 1; l <= D; ++l) tmp = tmp + c.pre2(l, i, j, p) * b(l, k);
                        for (int l = 1; l <= D; ++l) b(l, k) = b(l, k) + c.pre1(l, i, j, p) * tmp;
                    }
                }
                for (int cc = 1; cc <= D; ++cc)
                    for (int rr = 1; rr <= D; ++rr) {
                        double at = c.vnci(1, i, j, p) * a(rr, cc) + c.vnci(2, i, j, p) * b(rr, cc);
                        c.Ap(rr, cc, i, j, p) = at * 0.5;
                        c.Am(rr, cc, i, j, p) = at * 0.5;
                        double bt = c.vncj(1, i, j, p) * a(rr, cc) + c.vncj(2, i, j, p) * b(rr, cc);
                        c.Bp(rr, cc, i, j, p) = bt * 0.5;
                        c.Bm(rr, cc, i, j, p) = bt * 0.5;
                    }
                for (int k = 1; k <= D; ++k) {
                    c.Ap(k, k, i, j, p) = c.Ap(k, k, i, j, p) + nuA * 0.5;
                    c.Am(k, k, i, j, p) = c.Am(k, k, i, j, p) - nuA * 0.5;
                    c.Bp(k, k, i, j, p) = c.Bp(k, k, i, j, p) + nuB * 0.5;
                    c.Bm(k, k, i, j, p) = c.Bm(k, k, i, j, p) - nuB * 0.5;
                }
                double dtl = c.DTLG(i, j, p);
                double tmp = nr ? 3.0 * c.Vol(i, j, p) / (2.0 * dtl) + c.dsci(i, j, p) * nuA + c.dscj(i, j, p) * nuB
                                : c.Vol(i, j, p) / dtl + c.dsci(i, j, p) * nuA + c.dscj(i, j, p) * nuB;
                c.alpha(i, j, p) = 1.0 / tmp;
            }
    }
}

void set_dqdt(orc_ctx& c) {  // NR/q2d/sch_NR.raw.f90:151-180
    for (int p = 1; p <= c.np; ++p) {
        if (!c.own(p)) continue;
#pragma omp parallel for
        for (int j = 1; j <= c.nj[p - 1]; ++j)
            for (int i = 1; i <= c.ni[p - 1]; ++i) {
                double dtl = c.DTLG(i, j, p);
                for (int k = 1; k <= c.D; ++k) {
                    if (c.first_dual)
                        c.dqdt(k, i, j, p) = (c.q(k, i, j, p) - c.qp(k, i, j, p)) / dtl;
                    else
                        c.dqdt(k, i, j, p) = (3.0 * c.q(k, i, j, p) - 4.0 * c.qp(k, i, j, p) + c.qpp(k, i, j, p)) / (2.0 * dtl);
                }
            }
    }
}

// set_ABpm of the preconditioned dual time, store/time_scheme/dual/2d/
// sch_dual.raw.f90:1-209: low-Mach reference velocity, preconditioned spectral
// radii, pseudo time step from cfl_tau, the scalars and vectors of Gamma^-1,
// S and S^-1 (pre_sca, pre1, pre2) and the split Jacobians multiplied by
// Gamma^-1 (a rank-one update, 156-181).
void set_ABpm_dual(orc_ctx& c) {
    const int nY = c.nY, D = c.D;
    for (int p = 1; p <= c.np; ++p) {
        if (!c.own(p)) continue;
#pragma omp parallel for
        for (int j = 1; j <= c.nj[p - 1]; ++j)
            for (int i = 1; i <= c.ni[p - 1]; ++i) {
                std::vector<double> A(D * D), B(D * D), tA(D), tB(D), At(D * D), Bt(D * D);
                auto a = [&](int r, int cc) -> double& { return A[(r - 1) + D * (cc - 1)]; };
                auto b = [&](int r, int cc) -> double& { return B[(r - 1) + D * (cc - 1)]; };
                const double rho = c.w(1, i, j, p), u = c.w(2, i, j, p), v = c.w(3, i, j, p), pr = c.w(4, i, j, p);
                const double gamm = c.w(c.indxg, i, j, p), H = c.w(c.indxht, i, j, p);
                const double cs = std::sqrt(gamm * pr / rho), gmmad = gamm - 1.0, Vs = sq(u) + sq(v);
                const double unA = c.vnci(1, i, j, p) * u + c.vnci(2, i, j, p) * v;
                const double unB = c.vncj(1, i, j, p) * u + c.vncj(2, i, j, p) * v;
                const double Vv = c.w(c.indxMu, i, j, p) / rho / std::min(c.dsci(i, j, p), c.dscj(i, j, p));
                const double Ur = std::min(std::max(Vv, std::sqrt(Vs)), cs);
                c.phi(i, j, p) = 1.0 / sq(Ur) - 1.0 / sq(cs);
                const double alp = 0.5 * (1.0 - sq(Ur / cs));
                double ud = unA * (1.0 - alp), cd = std::sqrt(sq(alp) * sq(unA) + sq(Ur));
                const double nuA = std::fabs(ud) + cd;
                ud = unB * (1.0 - alp);
                cd = std::sqrt(sq(alp) * sq(unB) + sq(Ur));
                const double nuB = std::fabs(ud) + cd;
                const double uds = nuA * (c.dsi(i, j, p) + c.dsi(i - 1, j, p)) + nuB * (c.dsj(i, j, p) + c.dsj(i, j - 1, p));
                const double dtau = c.d.cfl_tau * c.Vol(i, j, p) / std::max(uds, c.w(c.indxMu, i, j, p) / rho);
                c.alpha(i, j, p) = 1.0 / (c.Vol(i, j, p) / dtau + c.dsci(i, j, p) * nuA + c.dscj(i, j, p) * nuB);
                const double beta = 3.0 * c.Vol(i, j, p) / (2.0 * c.DTLG(i, j, p)) * c.alpha(i, j, p);
                const double ph = c.phi(i, j, p);
                c.pre_sca(1, i, j, p) = 1.0 + beta;
                c.pre_sca(2, i, j, p) = -1.0 / (1.0 / ph + sq(cs));
                c.pre_sca(3, i, j, p) = -1.0 / (1.0 / ph + sq(cs)) / (1.0 / beta + 1.0);
                c.pre_sca(4, i, j, p) = beta / ((1.0 + beta) / ph + sq(cs));
                for (int k = 1; k <= nY; ++k) c.pre1(k, i, j, p) = c.w(4 + k, i, j, p);
                c.pre1(nY + 1, i, j, p) = u;
                c.pre1(nY + 2, i, j, p) = v;
                c.pre1(nY + 3, i, j, p) = H;
                for (int k = 1; k <= nY; ++k) c.pre2(k, i, j, p) = 0.5 * gmmad * Vs + c.DHi(k, i, j, p);
                c.pre2(nY + 1, i, j, p) = -gmmad * u;
                c.pre2(nY + 2, i, j, p) = -gmmad * v;
                c.pre2(nY + 3, i, j, p) = gmmad;
                // pure A and B, as set_ABpm of LU-SGS (sch_dual.raw.f90:85-154)
                a(nY + 1, nY + 1) = u * (3.0 - gamm); a(nY + 2, nY + 1) = v; a(nY + 3, nY + 1) = H - sq(u) * gmmad;
                a(nY + 1, nY + 2) = -v * gmmad; a(nY + 2, nY + 2) = u; a(nY + 3, nY + 2) = -u * v * gmmad;
                a(nY + 1, nY + 3) = gmmad; a(nY + 2, nY + 3) = 0.0; a(nY + 3, nY + 3) = u * gamm;
                for (int k = 1; k <= nY; ++k) {
                    tA[k - 1] = -c.w(4 + k, i, j, p) * u;
                    a(k, nY + 1) = c.w(4 + k, i, j, p); a(k, nY + 2) = 0.0; a(k, nY + 3) = 0.0;
                }
                tA[nY] = -sq(u) + 0.5 * gmmad * Vs;
                tA[nY + 1] = -u * v;
                tA[nY + 2] = u * (-H + 0.5 * gmmad * Vs);
                b(nY + 1, nY + 1) = v; b(nY + 2, nY + 1) = -u * gmmad; b(nY + 3, nY + 1) = -u * v * gmmad;
                b(nY + 1, nY + 2) = u; b(nY + 2, nY + 2) = v * (3.0 - gamm); b(nY + 3, nY + 2) = H - sq(v) * gmmad;
                b(nY + 1, nY + 3) = 0.0; b(nY + 2, nY + 3) = gmmad; b(nY + 3, nY + 3) = v * gamm;
                for (int k = 1; k <= nY; ++k) {
                    tB[k - 1] = -c.w(4 + k, i, j, p) * v;
                    b(k, nY + 1) = 0.0; b(k, nY + 2) = c.w(4 + k, i, j, p); b(k, nY + 3) = 0.0;
                }
                tB[nY] = -v * u;
                tB[nY + 1] = -sq(v) + 0.5 * gmmad * Vs;
                tB[nY + 2] = v * (-H + 0.5 * gmmad * Vs);
                for (int k = 1; k <= nY; ++k) {
                    for (int l = 1; l <= nY; ++l) { a(l, k) = tA[l - 1]; b(l, k) = tB[l - 1]; }
                    a(k, k) = tA[k - 1] + u;
                    a(nY + 1, k) = tA[nY] + c.DHi(k, i, j, p);
                    a(nY + 2, k) = tA[nY + 1];
                    a(nY + 3, k) = tA[nY + 2] + c.DHi(k, i, j, p) * u;
                    b(k, k) = tB[k - 1] + v;
                    b(nY + 1, k) = tB[nY];
                    b(nY + 2, k) = tB[nY + 1] + c.DHi(k, i, j, p);
                    b(nY + 3, k) = tB[nY + 2] + c.DHi(k, i, j, p) * v;
                }
                // multiply Gamma^-1 (156-181)
                for (int k = 1; k <= D; ++k) {
                    double ta = 0.0, tb = 0.0;
                    for (int l = 1; l <= D; ++l) {
                        ta = ta + c.pre2(l, i, j, p) * a(l, k);
                        tb = tb + c.pre2(l, i, j, p) * b(l, k);
                    }
                    ta = c.pre_sca(2, i, j, p) * ta;
                    tb = c.pre_sca(2, i, j, p) * tb;
                    for (int l = 1; l <= D; ++l) {
                        a(l, k) = a(l, k) + c.pre1(l, i, j, p) * ta;
                        b(l, k) = b(l, k) + c.pre1(l, i, j, p) * tb;
                    }
                }
                for (int cc = 1; cc <= D; ++cc)
                    for (int rr = 1; rr <= D; ++rr) {
                        const double at = c.vnci(1, i, j, p) * a(rr, cc) + c.vnci(2, i, j, p) * b(rr, cc);
                        c.Ap(rr, cc, i, j, p) = at * 0.5;
                        c.Am(rr, cc, i, j, p) = at * 0.5;
                        const double bt = c.vncj(1, i, j, p) * a(rr, cc) + c.vncj(2, i, j, p) * b(rr, cc);
                        c.Bp(rr, cc, i, j, p) = bt * 0.5;
                        c.Bm(rr, cc, i, j, p) = bt * 0.5;
                    }
                for (int k = 1; k <= D; ++k) {
                    c.Ap(k, k, i, j, p) = c.Ap(k, k, i, j, p) + nuA * 0.5;
                    c.Am(k, k, i, j, p) = c.Am(k, k, i, j, p) - nuA * 0.5;
                    c.Bp(k, k, i, j, p) = c.Bp(k, k, i, j, p) + nuB * 0.5;
                    c.Bm(k, k, i, j, p) = c.Bm(k, k, i, j, p) - nuB * 0.5;
                }
            }
    }
}

// The sweeps of time_dual_viscous.f90:1-95 on the owned planes: the RHS
// multiplied by Gamma^-1, forward sweep with S^-1, the S step, backward sweep
// with S^-1; returns the plane-local residual and omega candidate (the omega
// test, relaxation and q update are nr_apply, 96-125).
void dual_sweeps(orc_ctx& c, double& res_out, double& omega_out) {
    const int nY = c.nY, D = c.D;
    auto& Dq = c.Dq;
    double omega = 1e300, res = 0.0;
    // Dq += s * (pre2 . Dq) * pre1 at cell (i, j, p)
    auto rank1 = [&](int s, int i, int j, int p) {
        double t = 0.0;
        for (int l = 1; l <= D; ++l) t = t + c.pre2(l, i, j, p) * Dq(l, i, j, p);
        for (int l = 1; l <= D; ++l) Dq(l, i, j, p) = Dq(l, i, j, p) + c.pre_sca(s, i, j, p) * t * c.pre1(l, i, j, p);
    };
    for (int p = 1; p <= c.np; ++p) {
        if (!c.own(p)) continue;
        const int ni = c.ni[p - 1], nj = c.nj[p - 1];
#pragma omp parallel for
        for (int j = 1; j <= nj; ++j)
            for (int i = 1; i <= ni; ++i) {
                for (int k = 1; k <= D; ++k) Dq(k, i, j, p) = rhs_k(c, k, i, j, p) - c.Vol(i, j, p) * c.dqdt(k, i, j, p);
                rank1(2, i, j, p);
            }
        for (int j = 0; j <= nj; ++j)
            for (int k = 1; k <= D; ++k) Dq(k, 0, j, p) = 0.0;
        for (int i = 0; i <= ni; ++i)
            for (int k = 1; k <= D; ++k) Dq(k, i, 0, p) = 0.0;
        for (int sm = 2; sm <= ni + nj; ++sm) {
            const int ilo = std::max(1, sm - nj), ihi = std::min(sm - 1, ni);
#pragma omp parallel for
            for (int i = ilo; i <= ihi; ++i) {
                const int j = sm - i;
                double dqs[SCFD_MAX_SPECIES + 3];
                for (int k = 1; k <= D; ++k) {
                    double s1 = 0.0, s2 = 0.0;
                    for (int l = 1; l <= D; ++l) {
                        s1 += c.Ap(k, l, i - 1, j, p) * Dq(l, i - 1, j, p);
                        s2 += c.Bp(k, l, i, j - 1, p) * Dq(l, i, j - 1, p);
                    }
                    dqs[k - 1] = c.dsci(i - 1, j, p) * s1 + c.dscj(i, j - 1, p) * s2;
                }
                for (int k = 1; k <= D; ++k) Dq(k, i, j, p) = c.alpha(i, j, p) * (Dq(k, i, j, p) + dqs[k - 1]);
                rank1(4, i, j, p);
                for (int k = 1; k <= D; ++k) Dq(k, i, j, p) = 1.0 / c.pre_sca(1, i, j, p) * Dq(k, i, j, p);
            }
        }
#pragma omp parallel for
        for (int j = 1; j <= nj; ++j)
            for (int i = 1; i <= ni; ++i) {
                rank1(3, i, j, p);
                for (int k = 1; k <= D; ++k) Dq(k, i, j, p) = c.pre_sca(1, i, j, p) * Dq(k, i, j, p);
            }
        for (int j = 1; j <= nj + 1; ++j)
            for (int k = 1; k <= D; ++k) Dq(k, ni + 1, j, p) = 0.0;
        for (int i = 1; i <= ni + 1; ++i)
            for (int k = 1; k <= D; ++k) Dq(k, i, nj + 1, p) = 0.0;
        for (int sm = ni + nj; sm >= 2; --sm) {
            const int ilo = std::max(1, sm - nj), ihi = std::min(sm - 1, ni);
#pragma omp parallel for reduction(min : omega) reduction(+ : res)
            for (int i = ilo; i <= ihi; ++i) {
                const int j = sm - i;
                double dqs[SCFD_MAX_SPECIES + 3];
                for (int k = 1; k <= D; ++k) {
                    double s1 = 0.0, s2 = 0.0;
                    for (int l = 1; l <= D; ++l) {
                        s1 += c.Am(k, l, i + 1, j, p) * Dq(l, i + 1, j, p);
                        s2 += c.Bm(k, l, i, j + 1, p) * Dq(l, i, j + 1, p);
                    }
                    dqs[k - 1] = c.dsci(i + 1, j, p) * s1 + c.dscj(i, j + 1, p) * s2;
                }
                for (int k = 1; k <= D; ++k) Dq(k, i, j, p) = Dq(k, i, j, p) - c.alpha(i, j, p) * dqs[k - 1];
                rank1(4, i, j, p);
                for (int k = 1; k <= D; ++k) Dq(k, i, j, p) = 1.0 / c.pre_sca(1, i, j, p) * Dq(k, i, j, p);
                res = res + sq(Dq(nY + 3, i, j, p));
                for (int k = 1; k <= nY; ++k)
                    if (Dq(k, i, j, p) < 0.0) omega = std::min(omega, -c.q(k, i, j, p) / Dq(k, i, j, p) * c.d.dq_max);
            }
        }
    }
    res_out = res;
    omega_out = omega;
}

// calc_next_step_implicit: LU-SGS/{2d,q2d}/time_lusgs_viscous.f90 and
// NR/{2d,q2d}/time_NR_viscous.f90:1-109, in two parts: lusgs_sweeps (the
// sweeps over the owned planes; LU-SGS also updates q there) returns the
// plane-local residual and omega candidate, nr_apply relaxes q with the
// (global) omega.  Returns 0 or SCFD_E_OMEGA.
void lusgs_sweeps(orc_ctx& c, double& res_out, double& omega_out) {
    const int nY = c.nY, D = c.D;
    const bool nr = c.d.scheme == SCFD_SCHEME_NR || c.d.scheme == SCFD_SCHEME_PRECON;
    const bool pc = c.d.scheme == SCFD_SCHEME_PRECON || c.d.scheme == SCFD_SCHEME_PRECON_LUSGS;
    const bool q2d = c.d.dim == SCFD_DIM_Q2D;
    auto& Dq = c.Dq;
    double omega = 1e300;
    double res = 0.0;
    for (int p = 1; p <= c.np; ++p) {
        if (!c.own(p)) continue;
        int ni = c.ni[p - 1], nj = c.nj[p - 1];
#pragma omp parallel for
        for (int j = 1; j <= nj; ++j)
            for (int i = 1; i <= ni; ++i) {
                double sm[SCFD_MAX_SPECIES + 3];
                for (int k = 1; k <= D; ++k) sm[k - 1] = rhs_k(c, k, i, j, p);
                if (pc) {  // Dq = Dq_small + pre1 (pre2 . Dq_small) (time_precon_viscous.f90:24)
                    double t = 0.0;
                    for (int k = 1; k <= D; ++k) t = t + c.pre2(k, i, j, p) * sm[k - 1];
                    for (int k = 1; k <= D; ++k) sm[k - 1] = sm[k - 1] + c.pre1(k, i, j, p) * t;
                }
                for (int k = 1; k <= D; ++k)
                    Dq(k, i, j, p) = nr ? sm[k - 1] - c.Vol(i, j, p) * c.dqdt(k, i, j, p) : sm[k - 1];
            }
        for (int j = 0; j <= nj; ++j)
            for (int k = 1; k <= D; ++k) Dq(k, 0, j, p) = 0.0;
        for (int i = 0; i <= ni; ++i)
            for (int k = 1; k <= D; ++k) Dq(k, i, 0, p) = 0.0;
        // forward hyperplanes sm = i + j
        for (int sm = 2; sm <= ni + nj; ++sm) {
            int ilo = std::max(1, sm - nj), ihi = std::min(sm - 1, ni);
#pragma omp parallel for
            for (int i = ilo; i <= ihi; ++i) {
                int j = sm - i;
                double dqs[SCFD_MAX_SPECIES + 3];
                for (int k = 1; k <= D; ++k) {
                    double s1 = 0.0, s2 = 0.0;
                    for (int l = 1; l <= D; ++l) {
                        s1 += c.Ap(k, l, i - 1, j, p) * Dq(l, i - 1, j, p);
                        s2 += c.Bp(k, l, i, j - 1, p) * Dq(l, i, j - 1, p);
                    }
                    dqs[k - 1] = c.dsci(i - 1, j, p) * s1 + c.dscj(i, j - 1, p) * s2;
                }
                for (int k = 1; k <= D; ++k) Dq(k, i, j, p) = c.alpha(i, j, p) * (Dq(k, i, j, p) + dqs[k - 1]);
                if (q2d) {
                    double tmp = 0.0;
                    for (int l = 1; l <= nY + 1; ++l) tmp = tmp + Dq(l, i, j, p) * c.dpdq(l, i, j, p);
                    tmp = tmp + Dq(nY + 3, i, j, p) * c.dpdq(nY + 3, i, j, p);
                    tmp = Dq(nY + 2, i, j, p) + c.alpha(i, j, p) * c.Area(i, j, p) * tmp;
                    Dq(nY + 2, i, j, p) = tmp / (1.0 - c.alpha(i, j, p) * c.Area(i, j, p) * c.dpdq(nY + 2, i, j, p));
                }
            }
        }
        for (int j = 1; j <= nj + 1; ++j)
            for (int k = 1; k <= D; ++k) Dq(k, ni + 1, j, p) = 0.0;
        for (int i = 1; i <= ni + 1; ++i)
            for (int k = 1; k <= D; ++k) Dq(k, i, nj + 1, p) = 0.0;
        for (int sm = ni + nj; sm >= 2; --sm) {
            int ilo = std::max(1, sm - nj), ihi = std::min(sm - 1, ni);
#pragma omp parallel for reduction(min : omega) reduction(+ : res)
            for (int i = ilo; i <= ihi; ++i) {
                int j = sm - i;
                double dqs[SCFD_MAX_SPECIES + 3];
                for (int k = 1; k <= D; ++k) {
                    double s1 = 0.0, s2 = 0.0;
                    for (int l = 1; l <= D; ++l) {
                        s1 += c.Am(k, l, i + 1, j, p) * Dq(l, i + 1, j, p);
                        s2 += c.Bm(k, l, i, j + 1, p) * Dq(l, i, j + 1, p);
                    }
                    dqs[k - 1] = c.dsci(i + 1, j, p) * s1 + c.dscj(i, j + 1, p) * s2;
                }
                for (int k = 1; k <= D; ++k) Dq(k, i, j, p) = Dq(k, i, j, p) - c.alpha(i, j, p) * dqs[k - 1];
                if (nr) {
                    res = res + sq(Dq(nY + 3, i, j, p));
                    for (int k = 1; k <= nY; ++k)
                        if (Dq(k, i, j, p) < 0.0) omega = std::min(omega, -c.q(k, i, j, p) / Dq(k, i, j, p) * c.d.dq_max);
                }
            }
        }
        if (!nr) {
#pragma omp parallel for
            for (int j = 1; j <= nj; ++j)
                for (int i = 1; i <= ni; ++i)
                    for (int k = 1; k <= D; ++k) c.q(k, i, j, p) = c.q(k, i, j, p) + Dq(k, i, j, p);
        }
    }
    res_out = res;
    omega_out = omega;
}

// The omega test, residual bookkeeping and q += omega*Dq of
// time_NR_viscous.f90:75-108.  omega is the smallest candidate (the running
// minimum of the reference falls below omega_min exactly when it does).
int nr_apply(orc_ctx& c, int step_internal, double res, double omega) {
    if (step_internal >= 1 && step_internal <= SCFD_INNER_LOG) {
        c.il_omega[step_internal - 1] = omega;
        c.il_res[step_internal - 1] = res;
    }
    if (omega < c.d.omega_min) return SCFD_E_OMEGA;
    if (step_internal == 1) c.res1 = res;
    c.res = res;
    omega = std::min(c.d.omega_max, omega);
    c.omega_last = omega;
    for (int p = 1; p <= c.np; ++p) {
        if (!c.own(p)) continue;
#pragma omp parallel for
        for (int j = 1; j <= c.nj[p - 1]; ++j)
            for (int i = 1; i <= c.ni[p - 1]; ++i)
                for (int k = 1; k <= c.D; ++k) c.q(k, i, j, p) = c.q(k, i, j, p) + omega * c.Dq(k, i, j, p);
    }
    return 0;
}

int calc_next_step_implicit(orc_ctx& c, int step_internal) {
    double res, omega;
    if (c.d.scheme == SCFD_SCHEME_DUAL) {
        dual_sweeps(c, res, omega);
        return nr_apply(c, step_internal, res, omega);
    }
    lusgs_sweeps(c, res, omega);
    if (c.d.scheme != SCFD_SCHEME_NR && c.d.scheme != SCFD_SCHEME_PRECON) return 0;
    return nr_apply(c, step_internal, res, omega);
}

// the set_ABpm of the configured implicit scheme
void set_ABpm_scheme(orc_ctx& c) {
    if (c.d.scheme == SCFD_SCHEME_DUAL)
        set_ABpm_dual(c);
    else
        set_ABpm(c);
}

// dual time (NR, the preconditioned dual and precon) share the main loop of
// NR/q2d/main.main.raw.f90, dual/2d/main.main.raw.f90 and precon/2d/main.main.raw.f90
bool dual_time(const orc_ctx& c) {
    return c.d.scheme == SCFD_SCHEME_NR || c.d.scheme == SCFD_SCHEME_DUAL || c.d.scheme == SCFD_SCHEME_PRECON;
}

void copy_arr(FArr& dst, const FArr& src) { dst.v = src.v; }

int part_primitive(orc_ctx& c) {
    set_w(c);
    return set_thermo_prop(c);
}

int part_main(orc_ctx& c) {  // store/core/main.part_main.f90 + dim/q2d/main.part_main.f90
    set_BC(c);
    set_HV(c);
    set_TG(c);
    set_TGv(c);
    set_Sq(c);
    return 0;
}

int step_body(orc_ctx& c, scfd_stats* st);

// One physical step; the statistics are filled in also when the step stops
// with an error code.
int step(orc_ctx& c, int stepno, scfd_stats* st) {
    long long att0 = c.chem_attempts, fb0 = c.chem_fallback;
    if (st) std::memset(st, 0, sizeof(*st));
    int s = step_body(c, st);
    if (st) {
        st->dt_grbl = c.dt_grbl;
        st->tt = c.tt;
        st->res = c.res;
        st->res1 = c.res1;
        st->omega = c.omega_last;
        st->chem_attempts = c.chem_attempts - att0;
        st->chem_fallback_cells = c.chem_fallback - fb0;
        st->status = s;
    }
    (void)stepno;
    return s;
}

int step_body(orc_ctx& c, scfd_stats* st) {
    int s = 0;
    const bool reactive = c.d.thermo == SCFD_THERMO_CHEMKIN_REACTIVE;
    if (dual_time(c)) {
        // NR/q2d/main.main.raw.f90:1-20 (dual/2d/main.main.raw.f90:1-20 alike), with proceed_reaction after set_dt as in
        // LU-SGS/q2d/main.main.point_implicit.f90:1-3 when the model is reactive.
        if ((s = part_primitive(c))) return s;
        set_dt(c);
        if (reactive && (s = proceed_reaction(c))) return s;
        copy_arr(c.qpp, c.qp);
        copy_arr(c.qp, c.q);
        int j = 1;
        while (j < c.d.num_internal_loop) {
            if (st) st->inner_iters = j;
            if ((s = part_primitive(c))) return s;
            part_main(c);
            set_ABpm_scheme(c);
            set_dqdt(c);
            if ((s = calc_next_step_implicit(c, j))) return s;
            ++j;
        }
        if (st) { st->inner_iters = j - 1; }
        // check_internal_loop_convergence, sch_NR.raw.f90:222-237
        int warn = 0;
        if (c.res / c.res1 > c.d.res_rate_warn) {
            warn = 1;
            if (c.res / c.res1 > c.d.res_rate_err && !c.first_dual) s = SCFD_E_RESRATE;
        }
        if (st) st->res_warn = warn;
        c.first_dual = false;
    } else {
        if (reactive) {  // point-implicit variants: main.main.point_implicit.f90
            if ((s = part_primitive(c))) return s;
            set_dt(c);
            if ((s = proceed_reaction(c))) return s;
            copy_arr(c.qp, c.q);
            if ((s = part_primitive(c))) return s;
        } else {
            copy_arr(c.qp, c.q);
            if ((s = part_primitive(c))) return s;
            set_dt(c);
        }
        part_main(c);
        if (c.d.scheme == SCFD_SCHEME_EULER) {
            calc_next_step_euler(c);
        } else {
            set_ABpm(c);
            calc_next_step_implicit(c, 1);
        }
    }
    return s;
}

// ---------------------------------------------------------------------------
// Block sharding: each rank updates the planes it owns; the ghost copies of
// section_exchange whose source lies on another rank's plane read the values
// that rank exported (in place of MPI_COMMUNICATIONS_*, condition.tail.f90:
// 71-330), and dt, omega and the residual are reduced over the ranks.
// ---------------------------------------------------------------------------
void build_exports(orc_ctx& c) {
    c.exports.assign(c.nranks, {});
    for_each_halo_copy(c, [&](int, int, int pd, int is, int js, int ps) {
        const int q = c.owner[ps - 1];
        if (c.owner[pd - 1] != q) c.exports[q].push_back({ps, js, is});
    });
    size_t mx = 0;
    for (auto& e : c.exports) {
        std::sort(e.begin(), e.end());
        e.erase(std::unique(e.begin(), e.end()), e.end());
        mx = std::max(mx, e.size());
    }
    c.seg = (long long)mx * (c.W + c.nY);
    c.halo.assign((size_t)std::max(1LL, c.seg * c.nranks), 0.0);
}

// this rank's segment: component-major, halo[rank*seg + k*n + t]
void halo_pack(orc_ctx& c) {
    const auto& e = c.exports[c.rank];
    const size_t n = e.size();
    double* out = c.halo.data() + (size_t)c.rank * c.seg;
    for (size_t t = 0; t < n; ++t) {
        const int p = e[t][0], j = e[t][1], i = e[t][2];
        for (int k = 1; k <= c.W; ++k) out[(k - 1) * n + t] = c.w(k, i, j, p);
        for (int k = 1; k <= c.nY; ++k) out[(c.W + k - 1) * n + t] = c.vhi(k, i, j, p);
    }
}

void halo_unpack(orc_ctx& c) {
    for (int q = 0; q < c.nranks; ++q) {
        if (q == c.rank) continue;
        const auto& e = c.exports[q];
        const size_t n = e.size();
        const double* in = c.halo.data() + (size_t)q * c.seg;
        for (size_t t = 0; t < n; ++t) {
            const int p = e[t][0], j = e[t][1], i = e[t][2];
            for (int k = 1; k <= c.W; ++k) c.w(k, i, j, p) = in[(k - 1) * n + t];
            for (int k = 1; k <= c.nY; ++k) c.vhi(k, i, j, p) = in[(c.W + k - 1) * n + t];
        }
    }
}

enum { DS_BEGIN = 0, DS_AFTER_DT, DS_INNER, DS_AFTER_HALO_NR, DS_AFTER_RES, DS_AFTER_HALO, DS_AFTER_STATUS };

// The staged physical step of scfd_dstep: step_body with its reductions and
// the halo copies turned into requests.  A status seen on any rank becomes the
// step's status at the next reduction, where every rank stops together.
int dstep(orc_ctx& c, scfd_dreq* req, scfd_stats* st) {
    const bool nr = dual_time(c);
    const bool reactive = c.d.thermo == SCFD_THERMO_CHEMKIN_REACTIVE;
    auto keep = [&](int s) { c.ds_status = std::max(c.ds_status, s); };
    auto reduce = [&](int nsum, int nmin, int next) {
        req->kind = SCFD_DREQ_REDUCE;
        req->nsum = nsum;
        req->nmin = nmin;
        req->buf = c.red.data();
        c.ds_stage = next;
        return 0;
    };
    auto exchange = [&](int next) {
        halo_pack(c);
        req->kind = SCFD_DREQ_HALO;
        req->nranks = c.nranks;
        req->seg = c.seg;
        req->buf = c.halo.data();
        c.ds_stage = next;
        return 0;
    };
    auto finish = [&]() {
        if (st) {
            std::memset(st, 0, sizeof(*st));
            st->dt_grbl = c.dt_grbl;
            st->tt = c.tt;
            st->res = c.res;
            st->res1 = c.res1;
            st->omega = c.omega_last;
            st->chem_attempts = c.chem_attempts - c.ds_att0;
            st->chem_fallback_cells = c.chem_fallback - c.ds_fb0;
            st->status = c.ds_status;
            st->inner_iters = nr ? c.ds_j - (c.ds_stage == DS_INNER ? 1 : 0) : 0;
            st->res_warn = c.ds_stage == DS_INNER && nr && c.res / c.res1 > c.d.res_rate_warn ? 1 : 0;
        }
        req->kind = SCFD_DREQ_DONE;
        req->buf = nullptr;
        c.ds_stage = DS_BEGIN;
        return c.ds_status;
    };
    for (;;) {
        switch (c.ds_stage) {
            case DS_BEGIN:
                c.ds_status = 0;
                c.ds_j = 0;
                c.ds_att0 = c.chem_attempts;
                c.ds_fb0 = c.chem_fallback;
                if (!nr && !reactive) copy_arr(c.qp, c.q);
                keep(part_primitive(c));
                c.red[0] = set_dt_cells(c);
                c.red[1] = -(double)c.ds_status;
                return reduce(0, 2, DS_AFTER_DT);
            case DS_AFTER_DT:
                set_dt_apply(c, c.red[0]);
                keep((int)-c.red[1]);
                if (c.ds_status) return finish();
                if (reactive) keep(proceed_reaction(c));
                if (nr) {
                    copy_arr(c.qpp, c.qp);
                    copy_arr(c.qp, c.q);
                    c.ds_j = 1;
                    c.ds_stage = DS_INNER;
                    continue;
                }
                if (reactive) {
                    copy_arr(c.qp, c.q);
                    keep(part_primitive(c));
                }
                return exchange(DS_AFTER_HALO);
            case DS_INNER:
                if (c.ds_j >= c.d.num_internal_loop) {
                    // check_internal_loop_convergence, sch_NR.raw.f90:222-237
                    if (c.res / c.res1 > c.d.res_rate_warn && c.res / c.res1 > c.d.res_rate_err && !c.first_dual)
                        keep(SCFD_E_RESRATE);
                    const int s = finish();
                    c.first_dual = false;
                    return s;
                }
                keep(part_primitive(c));
                return exchange(DS_AFTER_HALO_NR);
            case DS_AFTER_HALO_NR: {
                halo_unpack(c);
                part_main(c);
                set_ABpm_scheme(c);
                set_dqdt(c);
                double res, om;
                if (c.d.scheme == SCFD_SCHEME_DUAL)
                    dual_sweeps(c, res, om);
                else
                    lusgs_sweeps(c, res, om);
                c.red[0] = res;
                c.red[1] = om;
                c.red[2] = -(double)c.ds_status;
                return reduce(1, 2, DS_AFTER_RES);
            }
            case DS_AFTER_RES:
                keep((int)-c.red[2]);
                if (!c.ds_status) keep(nr_apply(c, c.ds_j, c.red[0], c.red[1]));
                if (c.ds_status) return finish();
                ++c.ds_j;
                c.ds_stage = DS_INNER;
                continue;
            case DS_AFTER_HALO:
                halo_unpack(c);
                part_main(c);
                if (c.d.scheme == SCFD_SCHEME_EULER) {
                    calc_next_step_euler(c);
                } else {
                    set_ABpm(c);
                    calc_next_step_implicit(c, 1);
                }
                c.red[0] = -(double)c.ds_status;
                return reduce(0, 1, DS_AFTER_STATUS);
            default:  // DS_AFTER_STATUS
                keep((int)-c.red[0]);
                return finish();
        }
    }
}

// reference layout copy helpers: (k, -1:nimax+2, -1:njmax+2, plane)
void load_ref(FArr& dst, const double* src, int nk) {
    std::memcpy(dst.v.data(), src, sizeof(double) * dst.v.size());
    (void)nk;
}

}  // namespace

// ===========================================================================
// C ABI (orc_ prefix)
// ===========================================================================
extern "C" {

int orc_abi_version(void) { return SCFD_ABI_VERSION; }

int orc_create(const scfd_desc* d, orc_ctx** out) {
    if (!d || !out) return SCFD_E_ARG;
    if (d->abi_version != SCFD_ABI_VERSION) return SCFD_E_ARG;
    if (d->nplane < 1 || d->nplane > SCFD_MAX_PLANES || d->ny < 1 || d->ny > SCFD_MAX_SPECIES) return SCFD_E_ARG;
    if (d->scheme != SCFD_SCHEME_EULER && d->scheme != SCFD_SCHEME_LUSGS && d->scheme != SCFD_SCHEME_NR &&
        d->scheme != SCFD_SCHEME_DUAL && d->scheme != SCFD_SCHEME_PRECON && d->scheme != SCFD_SCHEME_PRECON_LUSGS)
        return SCFD_E_UNSUPPORTED;
    if (d->scheme == SCFD_SCHEME_DUAL) {  // checkout_flow.py:159-168; no reacting variant of dual
        if (d->dim != SCFD_DIM_2D || d->dt_mode == SCFD_DT_LOCAL || d->thermo == SCFD_THERMO_CHEMKIN_REACTIVE)
            return SCFD_E_UNSUPPORTED;
        if (!(d->cfl_tau > 0.0)) return SCFD_E_ARG;
    }
    // precon / preconLU-SGS: 2d only, local time step (checkout_flow.py:154-160,171-177)
    if ((d->scheme == SCFD_SCHEME_PRECON || d->scheme == SCFD_SCHEME_PRECON_LUSGS) &&
        (d->dim != SCFD_DIM_2D || d->dt_mode != SCFD_DT_LOCAL || d->thermo == SCFD_THERMO_CHEMKIN_REACTIVE))
        return SCFD_E_UNSUPPORTED;
    auto* c = new orc_ctx();
    c->d = *d;
    c->np = d->nplane;
    c->nY = d->ny;
    c->D = c->nY + 3;
    c->W = c->D + 5;
    c->indxg = c->D + 2;
    c->indxht = c->D + 3;
    c->indxR = c->D + 4;
    c->indxMu = c->D + 5;
    for (int p = 0; p < c->np; ++p) {
        c->ni[p] = d->ni[p];
        c->nj[p] = d->nj[p];
        if (c->ni[p] < 2 || c->nj[p] < 2) { delete c; return SCFD_E_ARG; }
        c->nimax = std::max(c->nimax, c->ni[p]);
        c->njmax = std::max(c->njmax, c->nj[p]);
    }
    c->geo_set.assign(c->np, 0);
    int np = c->np, NI = c->nimax, NJ = c->njmax, D = c->D, W = c->W, nY = c->nY;
    c->q.init({{1, D}, {-1, NI + 2}, {-1, NJ + 2}, {1, np}});
    c->qp.init({{1, D}, {-1, NI + 2}, {-1, NJ + 2}, {1, np}});
    c->qpp.init({{1, D}, {-1, NI + 2}, {-1, NJ + 2}, {1, np}});
    c->w.init({{1, W}, {-1, NI + 2}, {-1, NJ + 2}, {1, np}});
    c->DHi.init({{1, nY}, {1, NI}, {1, NJ}, {1, np}});
    c->vhi.init({{1, nY}, {-1, NI + 2}, {-1, NJ + 2}, {1, np}});
    c->wHli.init({{1, W}, {0, NI}, {1, NJ}, {1, np}});
    c->wHri.init({{1, W}, {0, NI}, {1, NJ}, {1, np}});
    c->wHlj.init({{1, W}, {1, NI}, {0, NJ}, {1, np}});
    c->wHrj.init({{1, W}, {1, NI}, {0, NJ}, {1, np}});
    c->TGi.init({{1, D}, {0, NI}, {1, NJ}, {1, np}});
    c->TGj.init({{1, D}, {1, NI}, {0, NJ}, {1, np}});
    c->Sq.init({{1, D}, {1, NI}, {1, NJ}, {1, np}});
    c->TGvi.init({{1, D}, {0, NI}, {1, NJ}, {1, np}});
    c->TGvj.init({{1, D}, {1, NI}, {0, NJ}, {1, np}});
    c->Svq.init({{1, D}, {1, NI}, {1, NJ}, {1, np}});
    c->Vol.init({{1, NI}, {1, NJ}, {1, np}});
    c->Area.init({{1, NI}, {1, NJ}, {1, np}});
    c->dsi.init({{0, NI}, {1, NJ}, {1, np}});
    c->dsj.init({{1, NI}, {0, NJ}, {1, np}});
    c->geojacc.init({{1, 2}, {1, 2}, {1, NI}, {1, NJ}, {1, np}});
    c->geojaci.init({{1, 2}, {1, 2}, {0, NI}, {1, NJ}, {1, np}});
    c->geojacj.init({{1, 2}, {1, 2}, {1, NI}, {0, NJ}, {1, np}});
    c->vni.init({{1, 2}, {0, NI}, {1, NJ}, {1, np}});
    c->vnj.init({{1, 2}, {1, NI}, {0, NJ}, {1, np}});
    c->xh.init({{0, NI}, {0, NJ}, {1, np}});
    c->rh.init({{0, NI}, {0, NJ}, {1, np}});
    c->x.init({{0, NI + 1}, {0, NJ + 1}, {1, np}});
    c->r.init({{0, NI + 1}, {0, NJ + 1}, {1, np}});
    c->dt_mat.init({{1, NI}, {1, NJ}, {1, np}});
    bool impl = d->scheme == SCFD_SCHEME_LUSGS || d->scheme == SCFD_SCHEME_NR || d->scheme == SCFD_SCHEME_DUAL ||
                d->scheme == SCFD_SCHEME_PRECON || d->scheme == SCFD_SCHEME_PRECON_LUSGS;
    if (d->scheme == SCFD_SCHEME_DUAL || d->scheme == SCFD_SCHEME_PRECON || d->scheme == SCFD_SCHEME_PRECON_LUSGS) {
        c->pre1.init({{1, D}, {1, NI}, {1, NJ}, {1, np}});
        c->pre2.init({{1, D}, {1, NI}, {1, NJ}, {1, np}});
        c->pre_sca.init({{1, 4}, {1, NI}, {1, NJ}, {1, np}});
        c->phi.init({{1, NI}, {1, NJ}, {1, np}});
    }
    if (impl) {
        c->Ap.init({{1, D}, {1, D}, {0, NI + 1}, {0, NJ + 1}, {1, np}});
        c->Am.init({{1, D}, {1, D}, {0, NI + 1}, {0, NJ + 1}, {1, np}});
        c->Bp.init({{1, D}, {1, D}, {0, NI + 1}, {0, NJ + 1}, {1, np}});
        c->Bm.init({{1, D}, {1, D}, {0, NI + 1}, {0, NJ + 1}, {1, np}});
        c->Dq.init({{1, D}, {0, NI + 1}, {0, NJ + 1}, {1, np}});
    }
    c->alpha.init({{1, NI}, {1, NJ}, {1, np}});
    c->dsci.init({{0, NI + 1}, {0, NJ + 1}, {1, np}});
    c->dscj.init({{0, NI + 1}, {0, NJ + 1}, {1, np}});
    c->vnci.init({{1, 2}, {1, NI}, {1, NJ}, {1, np}});
    c->vncj.init({{1, 2}, {1, NI}, {1, NJ}, {1, np}});
    c->dpdq.init({{1, D}, {1, NI}, {1, NJ}, {1, np}});
    c->dqdt.init({{1, D}, {1, NI}, {1, NJ}, {1, np}});
    *out = c;
    return 0;
}

int orc_destroy(orc_ctx* c) {
    delete c;
    return 0;
}

int orc_last_error(const orc_ctx* c, char* buf, int len) {
    if (!c || !buf || len <= 0) return SCFD_E_ARG;
    std::snprintf(buf, (size_t)len, "%s", c->err.c_str());
    return 0;
}

int orc_set_geometry(orc_ctx* c, int plane, const double* xh, const double* rh) {
    if (!c || plane < 1 || plane > c->np || !xh || !rh) return SCFD_E_ARG;
    int ni = c->ni[plane - 1], nj = c->nj[plane - 1];
    for (int j = 0; j <= nj; ++j)
        for (int i = 0; i <= ni; ++i) {
            c->xh(i, j, plane) = xh[i + (ni + 1) * j];
            c->rh(i, j, plane) = rh[i + (ni + 1) * j];
        }
    c->geo_set[plane - 1] = 1;
    return 0;
}

int orc_set_connectivity(orc_ctx* c, const int32_t* recs, int n) {
    if (!c || n < 0 || (n > 0 && !recs)) return SCFD_E_ARG;
    c->cut.assign(recs, recs + 11 * n);
    return 0;
}

int orc_set_bc(orc_ctx* c, const scfd_bc* b, int n) {
    if (!c || n < 0 || (n > 0 && !b)) return SCFD_E_ARG;
    c->bcs.assign(b, b + n);
    return 0;
}

int orc_set_chem(orc_ctx* c, const scfd_chem* ch) {
    if (!c || !ch) return SCFD_E_ARG;
    c->ch = *ch;
    c->have_chem = true;
    return 0;
}

int orc_commit(orc_ctx* c) {
    if (!c) return SCFD_E_ARG;
    for (int p = 0; p < c->np; ++p)
        if (!c->geo_set[p]) return c->fail(SCFD_E_STATE, "geometry of a plane not set");
    if (c->d.thermo != SCFD_THERMO_IDEAL && !c->have_chem) return c->fail(SCFD_E_STATE, "chem tables not set");
    init_geometry(*c);
    if (c->nranks > 1) build_exports(*c);
    c->red.assign(4, 0.0);
    c->committed = true;
    return 0;
}

int orc_set_partition(orc_ctx* c, const int32_t* owner, int nranks, int rank) {
    if (!c || !owner || nranks < 1 || nranks > SCFD_MAX_RANKS || rank < 0 || rank >= nranks) return SCFD_E_ARG;
    if (c->committed) return c->fail(SCFD_E_STATE, "partition after commit");
    for (int p = 0; p < c->np; ++p)
        if (owner[p] < 0 || owner[p] >= nranks) return c->fail(SCFD_E_ARG, "plane owner out of range");
    c->owner.assign(owner, owner + c->np);
    c->nranks = nranks;
    c->rank = rank;
    return 0;
}

int orc_dstep(orc_ctx* c, int stepno, scfd_dreq* req, scfd_stats* st) {
    if (!c || !req) return SCFD_E_ARG;
    req->kind = SCFD_DREQ_DONE;
    req->buf = nullptr;
    if (!c->committed) return c->fail(SCFD_E_STATE, "dstep before commit");
    (void)stepno;
    return dstep(*c, req, st);
}

int orc_upload(orc_ctx* c, const double* q, const double* w, const double* vhi, double tt) {
    if (!c || !q || !w) return SCFD_E_ARG;
    if (!c->committed) return SCFD_E_STATE;
    load_ref(c->q, q, c->D);
    load_ref(c->w, w, c->W);
    if (vhi) load_ref(c->vhi, vhi, c->nY);
    c->qp.v = c->q.v;
    c->qpp.v = c->q.v;
    c->tt = tt;
    c->first_dual = true;
    return 0;
}

int orc_prepare(orc_ctx* c, int stepno) {
    if (!c || !c->committed) return SCFD_E_STATE;
    int s = part_primitive(*c);
    if (s) return s;
    set_BC(*c);
    (void)stepno;
    return 0;
}

int orc_step(orc_ctx* c, int stepno, scfd_stats* st) {
    if (!c || !c->committed) return SCFD_E_STATE;
    if (c->nranks > 1) return c->fail(SCFD_E_STATE, "partitioned context: step through dstep");
    return step(*c, stepno, st);
}

int orc_run(orc_ctx* c, int stepno, int nsteps, scfd_stats* st) {
    if (!c || !c->committed) return SCFD_E_STATE;
    if (c->nranks > 1) return c->fail(SCFD_E_STATE, "partitioned context: step through dstep");
    for (int n = 0; n < nsteps; ++n) {
        int s = step(*c, stepno + n, st);
        if (s) return s;
    }
    return 0;
}

int orc_inner_log(orc_ctx* c, double* omega, double* res, int n) {  // time_NR_viscous.f90:87-95
    if (!c || !c->committed || n < 0) return -SCFD_E_ARG;
    const bool dual_time = c->d.scheme == SCFD_SCHEME_NR || c->d.scheme == SCFD_SCHEME_DUAL ||
                           c->d.scheme == SCFD_SCHEME_PRECON;
    if (!dual_time) return 0;
    const int m = std::min(std::min(n, std::max(0, c->d.num_internal_loop - 1)), SCFD_INNER_LOG);
    for (int k = 0; k < m; ++k) {
        if (omega) omega[k] = c->il_omega[k];
        if (res) res[k] = c->il_res[k];
    }
    return m;
}

int orc_rms(orc_ctx* c, double* rms) {  // store/core/check_convergence.f90:17-32
    if (!c || !rms) return SCFD_E_ARG;
    double tmp = 0.0, smc = 0.0;
    for (int p = 1; p <= c->np; ++p) {
        for (int j = 1; j <= c->nj[p - 1] && c->own(p); ++j)
            for (int i = 1; i <= c->ni[p - 1]; ++i) tmp = tmp + sq(c->q(c->nY + 3, i, j, p) - c->qp(c->nY + 3, i, j, p));
        smc = smc + (double)(c->ni[p - 1] * c->nj[p - 1]);
    }
    *rms = std::sqrt(tmp) / smc;
    return (*rms != *rms) ? SCFD_E_NAN : 0;
}

int orc_download(orc_ctx* c, double* q, double* w, double* vhi, double* tt) {
    if (!c) return SCFD_E_ARG;
    if (q) std::memcpy(q, c->q.v.data(), sizeof(double) * c->q.v.size());
    if (w) std::memcpy(w, c->w.v.data(), sizeof(double) * c->w.v.size());
    if (vhi) std::memcpy(vhi, c->vhi.v.data(), sizeof(double) * c->vhi.v.size());
    if (tt) *tt = c->tt;
    return 0;
}

// out_bin / restart_bin / set_bc_q (store/core/inout.f90:1-200) on the
// single-process (PC) path: Fortran unformatted sequential records, big-endian.
static void be_put(std::string& o, const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t k = n; k-- > 0;) o.push_back((char)b[k]);
}
static void be_get(const char* in, void* p, size_t n) {
    unsigned char* b = static_cast<unsigned char*>(p);
    for (size_t k = 0; k < n; ++k) b[n - 1 - k] = (unsigned char)in[k];
}

int orc_write_restart(orc_ctx* c, const char* path, int step) {
    if (!c || !path) return SCFD_E_ARG;
    if (!c->committed) return SCFD_E_STATE;
    const int nY = c->nY;
    FArr q = c->q;  // set_bc_q writes the copy that is written
    auto bcq = [&](int i, int j, int plane) {  // inout.f90:155-161
        double tmp = c->w(1, i, j, plane);
        for (int k = 1; k <= nY; ++k) q(k, i, j, plane) = tmp * c->w(k + 4, i, j, plane);
        q(nY + 1, i, j, plane) = tmp * c->w(2, i, j, plane);
        q(nY + 2, i, j, plane) = tmp * c->w(3, i, j, plane);
        q(nY + 3, i, j, plane) = tmp * c->w(c->indxht, i, j, plane) - c->w(4, i, j, plane);
    };
    for (int plane = 1; plane <= c->np; ++plane) {
        const int ni = c->ni[plane - 1], nj = c->nj[plane - 1];
        for (int j = 1; j <= nj; ++j) {
            bcq(0, j, plane);
            bcq(ni + 1, j, plane);
        }
        for (int i = 0; i <= ni + 1; ++i) {
            bcq(i, 0, plane);
            bcq(i, nj + 1, plane);
        }
    }
    std::string out, rec;
    auto record = [&]() {
        const int32_t n = (int32_t)rec.size();
        be_put(out, &n, 4);
        out += rec;
        be_put(out, &n, 4);
        rec.clear();
    };
    const int32_t s32 = step;
    be_put(rec, &s32, 4);
    record();
    be_put(rec, &c->tt, 8);
    record();
    for (int plane = 1; plane <= c->np; ++plane)  // inout.f90:49-51
        for (int k = 0; k <= c->nj[plane - 1] + 1; ++k)
            for (int j = 0; j <= c->ni[plane - 1] + 1; ++j) {
                for (int i = 1; i <= c->D; ++i) be_put(rec, &q(i, j, k, plane), 8);
                be_put(rec, &c->w(c->indxR, j, k, plane), 8);
                be_put(rec, &c->w(c->indxg, j, k, plane), 8);
                be_put(rec, &c->w(4, j, k, plane), 8);
            }
    record();
    FILE* f = std::fopen(path, "wb");
    if (!f) return SCFD_E_IO;
    const bool ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
    return (std::fclose(f) == 0 && ok) ? 0 : SCFD_E_IO;
}

int orc_write_geometry(orc_ctx* c, const char* path) {  // out_geo_bin, geometry.f90:182-193
    if (!c || !path) return SCFD_E_ARG;
    for (int p = 0; p < c->np; ++p)
        if (!c->geo_set[p]) return SCFD_E_STATE;
    std::string out, rec;
    auto record = [&]() {
        const int32_t n = (int32_t)rec.size();
        be_put(out, &n, 4);
        out += rec;
        be_put(out, &n, 4);
        rec.clear();
    };
    for (int plane = 1; plane <= c->np; ++plane) {
        const int32_t ni = c->ni[plane - 1], nj = c->nj[plane - 1];
        be_put(rec, &ni, 4);
        record();
        be_put(rec, &nj, 4);
        record();
        for (int j = 0; j <= nj; ++j)
            for (int i = 0; i <= ni; ++i) {
                be_put(rec, &c->xh(i, j, plane), 8);
                be_put(rec, &c->rh(i, j, plane), 8);
            }
        record();
    }
    FILE* f = std::fopen(path, "wb");
    if (!f) return SCFD_E_IO;
    const bool ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
    return (std::fclose(f) == 0 && ok) ? 0 : SCFD_E_IO;
}

int orc_read_restart(orc_ctx* c, const char* path, int* step, double* tt) {
    if (!c || !path || !step) return SCFD_E_ARG;
    if (!c->committed) return SCFD_E_STATE;
    FILE* f = std::fopen(path, "rb");
    if (!f) return SCFD_E_IO;
    std::string buf;
    char tmp[1 << 16];
    size_t n;
    while ((n = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.append(tmp, n);
    std::fclose(f);
    std::vector<std::string> recs;
    for (size_t pos = 0; pos < buf.size();) {
        int32_t a = 0, b = 0;
        if (pos + 4 > buf.size()) return SCFD_E_IO;
        be_get(&buf[pos], &a, 4);
        if (a < 0 || pos + 8 + (size_t)a > buf.size()) return SCFD_E_IO;
        be_get(&buf[pos + 4 + a], &b, 4);
        if (a != b) return SCFD_E_IO;
        recs.push_back(buf.substr(pos + 4, (size_t)a));
        pos += 8 + (size_t)a;
    }
    size_t need = 0;
    for (int p = 0; p < c->np; ++p) need += (size_t)(c->ni[p] + 2) * (c->nj[p] + 2) * (c->D + 3) * 8;
    if (recs.size() != 3 || recs[0].size() != 4 || recs[1].size() != 8 || recs[2].size() != need) return SCFD_E_IO;
    int32_t s32;
    be_get(recs[0].data(), &s32, 4);
    be_get(recs[1].data(), &c->tt, 8);
    const char* fp = recs[2].data();
    for (int plane = 1; plane <= c->np; ++plane)  // inout.f90:96-98
        for (int k = 0; k <= c->nj[plane - 1] + 1; ++k)
            for (int j = 0; j <= c->ni[plane - 1] + 1; ++j) {
                for (int i = 1; i <= c->D; ++i, fp += 8) be_get(fp, &c->q(i, j, k, plane), 8);
                be_get(fp, &c->w(c->indxR, j, k, plane), 8);
                be_get(fp + 8, &c->w(c->indxg, j, k, plane), 8);
                be_get(fp + 16, &c->w(4, j, k, plane), 8);
                fp += 24;
            }
    c->qp.v = c->q.v;
    c->qpp.v = c->q.v;
    c->first_dual = true;
    c->ds_stage = 0;
    *step = s32;
    if (tt) *tt = c->tt;
    return 0;
}

int orc_download_qp(orc_ctx* c, double* qp) {
    if (!c || !qp) return SCFD_E_ARG;
    std::memcpy(qp, c->qp.v.data(), sizeof(double) * c->qp.v.size());
    return 0;
}

int orc_get_stream(orc_ctx* c, void** s) {
    if (!c || !s) return SCFD_E_ARG;
    *s = nullptr;
    return 0;
}

int orc_launch_count(const orc_ctx* c, int64_t* n) {
    if (!c || !n) return SCFD_E_ARG;
    *n = 0;
    return 0;
}

int orc_set_bc_values(orc_ctx* c, int bc, const double* value) {
    if (!c || !value || bc < 0 || bc >= (int)c->bcs.size()) return SCFD_E_ARG;
    std::memcpy(c->bcs[bc].value, value, sizeof(c->bcs[bc].value));
    return 0;
}

// The objective of scfd_adjoint_run on the restatement (forward only: the
// reference has no adjoint): J = sum over the window's states of
// sum_cells ds * p, p = (kappa-1)(E - |rho u|^2 / (2 rho)) of the first interior
// cells along the descriptor, ds the boundary face length.
int orc_adjoint_run(orc_ctx* c, const scfd_adj_desc* d, double* J, double* grad, int64_t* counts) {
    if (!c || !d || !J) return SCFD_E_ARG;
    if (!c->committed) return SCFD_E_STATE;
    if (!d->forward_only) return SCFD_E_UNSUPPORTED;
    if (d->nsteps < 1 || d->win_first < 0 || d->win_first > d->win_last || d->win_last >= d->nsteps ||
        d->obj_bc < 0 || d->obj_bc >= (int)c->bcs.size())
        return SCFD_E_ARG;
    const scfd_bc& b = c->bcs[d->obj_bc];
    const int p = b.plane, ni = c->ni[p - 1], nj = c->nj[p - 1], nY = c->nY;
    auto term = [&]() {
        double t = 0.0;
        for (int s = b.first; s <= b.last; ++s) {
            int i, j;
            double ds;
            switch (b.side) {
                case SCFD_SIDE_ILO: i = 1; j = s; ds = c->dsi(0, s, p); break;
                case SCFD_SIDE_IHI: i = ni; j = s; ds = c->dsi(ni, s, p); break;
                case SCFD_SIDE_JLO: i = s; j = 1; ds = c->dsj(s, 0, p); break;
                default: i = s; j = nj; ds = c->dsj(s, nj, p); break;
            }
            double rho = 0.0;
            for (int k = 1; k <= nY; ++k) rho = rho + c->q(k, i, j, p);
            const double mx = c->q(nY + 1, i, j, p), my = c->q(nY + 2, i, j, p);
            t = t + ds * (c->d.kappa - 1.0) * (c->q(nY + 3, i, j, p) - 0.5 * (mx * mx + my * my) / rho);
        }
        return t;
    };
    const std::vector<double> q0 = c->q.v;
    const double tt0 = c->tt;
    double sum = 0.0;
    for (int n = 0; n <= d->win_last; ++n) {
        if (n >= d->win_first) sum = sum + term();
        if (n < d->win_last) {
            const int s = step(*c, n + 1, nullptr);
            if (s) return s;
        }
    }
    c->q.v = q0;
    c->qp.v = q0;
    c->qpp.v = q0;
    c->tt = tt0;
    *J = sum;
    (void)grad;
    if (counts) {
        counts[0] = d->win_last;
        counts[1] = 0;
    }
    return 0;
}

int orc_tuning(orc_ctx* c, char* json, int len) {  // no launch shapes on the CPU
    if (!c || !json || len <= 0) return SCFD_E_ARG;
    std::snprintf(json, (size_t)len, "{\"enabled\": false}");
    return 0;
}

int orc_profile(orc_ctx* c, int enable) {
    (void)enable;
    return c ? 0 : SCFD_E_ARG;
}

int orc_kernel_stats(orc_ctx* c, int kind, double* ms, int64_t* n, char* name, int namelen) {
    (void)kind;
    if (!c) return SCFD_E_ARG;
    if (ms) *ms = 0.0;
    if (n) *n = 0;
    if (name && namelen > 0) name[0] = 0;
    return 0;
}

// Single-cell entry points for unit tests of the thermochemistry.
int orc_calc_T(const scfd_chem* ch, const double* vrho, double rho, double E, double* T, double* kappa,
               double* MW, double* DHi, double* vhi, double* mu) {
    return calc_T(*ch, vrho, rho, E, *T, *kappa, *MW, DHi, vhi, *mu);
}

int orc_chem_rates(const scfd_chem* ch, int n, const double* states, double* dndt, double* jac) {
    if (!ch || n < 0 || (n > 0 && (!states || !dndt)) || ch->ns < 1 || ch->ns > SCFD_MAX_SPECIES ||
        ch->nr < 0 || ch->nr > SCFD_MAX_REACTIONS)
        return SCFD_E_ARG;
    const int N = ch->ns + 1;
    for (int c = 0; c < n; ++c)
        fex_jex(*ch, states + (size_t)c * N, dndt + (size_t)c * N, jac ? jac + (size_t)c * N * N : nullptr);
    return 0;
}

int orc_fex_var(const scfd_chem* ch, const double* n, double* p, double* m) {
    fex_var(*ch, n, p, m);
    return 0;
}

// DVODE (dvode.h) on test problems with known solutions, through the
// reference's driver loop (restart on ISTATE = -1): problem 0 is the linear
// system y' = A y (A row-major n x n), problem 1 Robertson's kinetics
// (n = 3).  y: the state at t0 on entry, at tout on return.  Returns the
// final ISTATE; *nst the accepted steps over all restarts.
int orc_dvode_test(int problem, int n, const double* A, double* y, double t0, double tout, double rtol,
                   double atol, int64_t* nst) {
    if (n < 1 || n > SCFD_MAX_SPECIES + 1 || (problem == 1 && n != 3) || (problem == 0 && !A)) return -99;
    struct Sys {
        int problem, n;
        const double* A;
        void f(double, const double* yy, double* dy) {
            if (problem == 0) {
                for (int i = 0; i < n; ++i) {
                    double a = 0.0;
                    for (int j = 0; j < n; ++j) a += A[i * n + j] * yy[j + 1];
                    dy[i + 1] = a;
                }
            } else {
                dy[1] = -0.04 * yy[1] + 1.0e4 * yy[2] * yy[3];
                dy[3] = 3.0e7 * yy[2] * yy[2];
                dy[2] = -dy[1] - dy[3];
            }
        }
        void jac(double, const double* yy, dvode::State& s) {
            if (problem == 0) {
                for (int i = 0; i < n; ++i)
                    for (int j = 0; j < n; ++j) s.A(i + 1, j + 1) = A[i * n + j];
            } else {
                s.A(1, 1) = -0.04;
                s.A(1, 2) = 1.0e4 * yy[3];
                s.A(1, 3) = 1.0e4 * yy[2];
                s.A(3, 1) = 0.0;
                s.A(3, 2) = 6.0e7 * yy[2];
                s.A(3, 3) = 0.0;
                s.A(2, 1) = -s.A(1, 1) - s.A(3, 1);
                s.A(2, 2) = -s.A(1, 2) - s.A(3, 2);
                s.A(2, 3) = -s.A(1, 3) - s.A(3, 3);
            }
        }
    } sys{problem, n, A};
    dvode::State st;
    double y1[SCFD_MAX_SPECIES + 2];
    for (int i = 0; i < n; ++i) y1[i + 1] = y[i];
    double t = t0;
    int64_t steps = 0;
    int istate = 0;
    for (int recalc = 0; recalc <= 1000; ++recalc) {
        istate = dvode::solve(st, sys, n, y1, t, tout, rtol, atol, [](double, const double*) {});
        steps += st.nst;
        if (istate != -1) break;
    }
    for (int i = 0; i < n; ++i) y[i] = y1[i + 1];
    if (nst) *nst = steps;
    return istate;
}

int orc_chemeq2(const scfd_chem* ch, double* y, double tout, int64_t* attempts, int* fell_back) {
    long long a = 0;
    bool fb = false;
    int s = chemeq2(*ch, y, 0.0, tout, ch->rtol, a, fb, 1000000);
    if (attempts) *attempts = a;
    if (fell_back) *fell_back = fb ? 1 : 0;
    return s;
}

// ---- batched constant-volume 0-D reactors: successive reaction_chemeq2 calls
// (sub_chem.f90:1684-1713) over dt_call up to t_end per reactor, with the
// ignition test of reaction_one_steps; reactors in parallel over OpenMP threads.
struct orc_reactors {
    scfd_chem ch;
    int n_max = 0, n = 0, status = 0;
    long long launches = 0;
    std::vector<double> T0, vrho0, T_end, vrho_end, t_ign;
    std::vector<int64_t> evals;
    std::vector<int32_t> flags;
};

int orc_reactors_create(const scfd_chem* ch, int n_max, orc_reactors** out) {
    if (!ch || !out || n_max < 1 || ch->ns < 1 || ch->ns > SCFD_MAX_SPECIES || ch->nr < 0 ||
        ch->nr > SCFD_MAX_REACTIONS)
        return SCFD_E_ARG;
    orc_reactors* r = new orc_reactors();
    r->ch = *ch;
    r->n_max = n_max;
    const size_t nn = (size_t)n_max, nv = nn * ch->ns;
    r->T0.assign(nn, 0.0);
    r->vrho0.assign(nv, 0.0);
    r->T_end.assign(nn, 0.0);
    r->vrho_end.assign(nv, 0.0);
    r->t_ign.assign(nn, -1.0);
    r->evals.assign(nn, 0);
    r->flags.assign(nn, 0);
    *out = r;
    return 0;
}

int orc_reactors_destroy(orc_reactors* r) {
    if (!r) return SCFD_E_ARG;
    delete r;
    return 0;
}

int orc_reactors_upload(orc_reactors* r, int n, const double* T0, const double* vrho0) {
    if (!r || !T0 || !vrho0 || n < 1 || n > r->n_max) return SCFD_E_ARG;
    std::copy(T0, T0 + n, r->T0.begin());
    std::copy(vrho0, vrho0 + (size_t)n * r->ch.ns, r->vrho0.begin());
    r->n = n;
    return 0;
}

int orc_reactors_launch(orc_reactors* r, const scfd_reactor_desc* d) {
    if (!r || !d || d->abi_version != SCFD_ABI_VERSION || d->n < 1 || d->n != r->n || !(d->t_end > 0.0) ||
        (d->mode != SCFD_REACTOR_QUEUE && d->mode != SCFD_REACTOR_PER_LAUNCH))
        return SCFD_E_ARG;
    const scfd_chem& ch = r->ch;
    const int ns = ch.ns, maxsub = d->max_substeps > 0 ? d->max_substeps : 1000000;
    double inv[SCFD_MAX_SPECIES];
    for (int j = 0; j < ns; ++j) inv[j] = 1.0 / ch.mws[j];  // invMW
    int worst = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(max : worst)
    for (int k = 0; k < d->n; ++k) {
        double y[SCFD_MAX_SPECIES + 1];
        for (int j = 0; j < ns; ++j) y[j] = std::max(r->vrho0[(size_t)k * ns + j] * inv[j] * 1e-3, 1e-40);
        y[ns] = r->T0[k];
        Ignition g{r->T0[k], d->dT_ign, 0.0, r->T0[k], -1.0, false, 0.0};
        long long att = 0, ev = 0;
        bool fb = false, any_fb = false;
        int rc = 0;
        // successive reaction_chemeq2 calls over dt_call: moles floored at n_eps
        // and passed through the partial densities between calls
        double tg = 0.0;
        for (;;) {
            const double rest = d->t_end - tg;
            const double tout = (d->dt_call > 0.0 && d->dt_call < rest) ? d->dt_call : rest;
            g.t_off = tg;
            rc = chemeq2(ch, y, 0.0, tout, ch.rtol, att, fb, maxsub, &g, &ev);
            any_fb = any_fb || fb;
            if (rc) break;
            tg = tg + tout;
            for (int j = 0; j < ns; ++j) y[j] = std::max(std::max(y[j], 1e-40) * ch.mws[j] * 1e3 * inv[j] * 1e-3, 1e-40);
            if (!(d->t_end - tg > 1e-12 * d->t_end)) break;
        }
        r->T_end[k] = y[ns];
        for (int j = 0; j < ns; ++j) r->vrho_end[(size_t)k * ns + j] = std::max(y[j], 1e-40) * ch.mws[j] * 1e3;
        r->t_ign[k] = g.ignited ? g.t_ign : -1.0;
        r->evals[k] = ev;
        r->flags[k] = (g.ignited ? SCFD_REACTOR_IGNITED : 0) | (any_fb ? SCFD_REACTOR_FELL_BACK : 0) |
                      (rc ? SCFD_REACTOR_FAILED : 0);
        worst = std::max(worst, rc);
    }
    r->status = worst;
    r->launches = 0;
    return 0;
}

int orc_reactors_download(orc_reactors* r, double* T_end, double* vrho_end, double* t_ign, int64_t* evals,
                          int32_t* flags) {
    if (!r || r->n < 1) return SCFD_E_ARG;
    const size_t n = (size_t)r->n, nv = n * r->ch.ns;
    if (T_end) std::copy(r->T_end.begin(), r->T_end.begin() + n, T_end);
    if (vrho_end) std::copy(r->vrho_end.begin(), r->vrho_end.begin() + nv, vrho_end);
    if (t_ign) std::copy(r->t_ign.begin(), r->t_ign.begin() + n, t_ign);
    if (evals) std::copy(r->evals.begin(), r->evals.begin() + n, evals);
    if (flags) std::copy(r->flags.begin(), r->flags.begin() + n, flags);
    return r->status;
}

int orc_reactors_run(orc_reactors* r, const scfd_reactor_desc* d, const double* T0, const double* vrho0,
                     double* T_end, double* vrho_end, double* t_ign, int64_t* evals, int32_t* flags) {
    if (!d) return SCFD_E_ARG;
    int st = orc_reactors_upload(r, d->n, T0, vrho0);
    if (st) return st;
    if ((st = orc_reactors_launch(r, d))) return st;
    return orc_reactors_download(r, T_end, vrho_end, t_ign, evals, flags);
}

void* orc_reactors_stream(orc_reactors*) { return nullptr; }

int orc_reactors_launch_count(const orc_reactors* r, int64_t* launches) {
    if (!r || !launches) return SCFD_E_ARG;
    *launches = r->launches;
    return 0;
}

}  // extern "C"
