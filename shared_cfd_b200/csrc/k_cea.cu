// k_cea.cu -- CEA chemical equilibrium per cell (scfd_cea_*).
//
// `cea` of store/therm_lib/NASA/core/sub_chem.f90:1320-1651: at fixed density
// rho, internal energy E (J/kg) and fuel / oxidizer mass fractions Y(1:2), a
// Newton iteration on the element potentials pi_1..pi_ne and ln T finds the
// equilibrium moles n_j (mol/kg).  Each iteration assembles the symmetric
// (ne+1) x (ne+1) system of the Gordon-McBride element-potential method over
// the species above the trace level tinyn = 1e-11 sum(n), solves it with a
// partially pivoted LU (NASA/core/LU.f90), and takes the damped update
//     dln n_j = -mu_j/RT + sum_i a_ij pi_i + (h_j/RT - 1) dln T,
//     omega   = min(1, 2 / max(5|dln T|, max_j |dln n_j|, 2), lambda2)
// until the element balance, the energy and the largest |dln n_j| n_j agree to
// 1e-9 (500 iterations at most).  The equilibrium state then gives the mixture
// weight, gamma = cp/(cp - R), the species enthalpies vhi, the DHi terms and
// the Wilke-mixed viscosity.  k_cea_hptp restates cea_hp and cea_tp
// (sub_chem.f90:1652-2248) the same way, with ln sum(n) (and for hp ln T) among
// the unknowns.
//
// Layout: one thread per cell; the species vectors are register arrays of a
// compile-time length (exactly 9 species / 3 elements for the hydrogen-air
// set, up to 12 / 4 with 3 temperature sections, 32 / 6 / 6 otherwise) and the
// tables are staged in shared memory once per block.  Cells where one stream is absent
// (Y < 1e-6) drop the elements only that stream carries; the reference
// compresses the system to the kept rows (sub_chem.f90:1456-1469), this kernel
// keeps the full system and makes the dropped rows and columns identity rows,
// which leaves every pivot choice and every update of a kept entry unchanged.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "scfd_internal.h"

namespace {

constexpr double RU = 8.3144621;      // mod_chem.raw.f90:6
constexpr double PST = 1e5;
constexpr double EPS = 1e-9;
constexpr double INITIAL_EPS = 1e-5;
constexpr double Y_EPS = 1e-6;
constexpr double TSIZE = 1e-11;
constexpr double TTSIZE = 1e-14;
constexpr int MAX_ITER = 500;

template <int NS, int NE, int NSEC>
struct CeaTab {
    int ns, ne, nt, pad;
    int nsec[NS];
    int ntsec[NS];
    int tr2th[NS];
    double tlo[NS];              // Trange(1,1,j)
    double thi[NS][NSEC];        // Trange(2,l,j)
    double co[NS][NSEC][9];
    double mw[NS];
    double ac[NE][NS];
    double yac[NE][NS];
    double ttlo[NS];
    double tthi[NS][3];
    double trans[NS][3][4];
    double wmw[NS][NS];          // (MW_j / MW_i)^0.25 of fits i, j
    double wsq[NS][NS];          // sqrt(2 MW_j / (MW_i + MW_j))
    double b0f[NE], b0o[NE], yfe[NE], yoe[NE];
    double maskf[NS], masko[NS];
    double keepf[NE], keepo[NE]; // maskbf / maskbo of the elements
};

using TabH2Air = CeaTab<9, 3, 3>;   // the 9-species H/O/N set, exactly
using TabSmall = CeaTab<12, 4, 3>;
using TabBig = CeaTab<SCFD_CEA_MAX_SPECIES, SCFD_CEA_MAX_ELEMENTS, SCFD_CEA_MAX_SECTIONS>;

// check_section_number (NASA/core/func_chem.f90:42-61)
template <class Tab, int NSEC>
__device__ __forceinline__ int section(const Tab& t, int j, double T) {
    if (t.tlo[j] > T) return 0;
#pragma unroll
    for (int l = 0; l < NSEC; ++l)
        if (l < t.nsec[j] && t.thi[j][l] > T) return l;
    return t.nsec[j] - 1;
}

__device__ __forceinline__ int tsection(const double* thi, double tlo, int nsec, double T) {
    if (tlo > T) return 0;
    for (int l = 0; l < nsec; ++l)
        if (thi[l] > T) return l;
    return nsec - 1;
}

// calc_vThrt, calc_vTcpr, calc_vTmurt (func_chem.f90:63-148), in their
// multiplication order
__device__ __forceinline__ void v_hrt(double T, double logT, double* v) {
    double tt = 1.0 / (T * T);
    v[0] = -tt;
    tt = tt * T;
    v[1] = tt * logT;
    v[7] = tt;
    tt = tt * T;
    v[2] = tt;
    tt = tt * T;
    v[3] = tt / 2.0;
    tt = tt * T;
    v[4] = tt / 3.0;
    tt = tt * T;
    v[5] = tt / 4.0;
    tt = tt * T;
    v[6] = tt / 5.0;
    v[8] = 0.0;
}
__device__ __forceinline__ void v_cpr(double T, double* v) {
    double tt = 1.0 / (T * T);
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        v[k] = tt;
        tt = tt * T;
    }
    v[7] = 0.0;
    v[8] = 0.0;
}
__device__ __forceinline__ void v_murt(double T, double logT, double* v) {
    double tt = 1.0 / (T * T);
    v[0] = -tt / 2.0;
    tt = tt * T;
    v[1] = tt * (1.0 + logT);
    v[7] = tt;
    tt = tt * T;
    v[2] = tt * (1.0 - logT);
    v[8] = -tt;
    tt = tt * T;
    v[3] = -tt / 2.0;
    tt = tt * T;
    v[4] = -tt / 6.0;
    tt = tt * T;
    v[5] = -tt / 12.0;
    tt = tt * T;
    v[6] = -tt / 20.0;
}
__device__ __forceinline__ double dot9(const double* c, const double* v) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 9; ++k) s += c[k] * v[k];
    return s;
}

struct CellOut {
    double* mwave;
    double* kappa;
    double* mu;
    double* Yv;
    double* vhi;
    double* DHi;
    int32_t* iters;
};

// EXACT: the species set has exactly NS species and NE elements, so that the
// counts are compile-time constants and no register holds an unused slot.
template <int NS, int NE, int NSEC, bool EXACT, int MINB>
__global__ void __launch_bounds__(128, MINB) k_cea(const CeaTab<NS, NE, NSEC>* __restrict__ gtab, int64_t ncell,
                                             const double* __restrict__ rho_in, const double* __restrict__ Y_in,
                                             const double* __restrict__ E_in, double* __restrict__ T_io,
                                             double* __restrict__ n_io, CellOut out,
                                             unsigned long long* __restrict__ fails) {
    using Tab = CeaTab<NS, NE, NSEC>;
    extern __shared__ double smem_tab[];
    {
        const double* src = reinterpret_cast<const double*>(gtab);
        for (int k = threadIdx.x; k < (int)(sizeof(Tab) / sizeof(double)); k += blockDim.x) smem_tab[k] = src[k];
    }
    __syncthreads();
    const Tab& t = *reinterpret_cast<const Tab*>(smem_tab);
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    const int ns = EXACT ? NS : t.ns, ne = EXACT ? NE : t.ne, nt = t.nt;
    constexpr int M = NE + 1;

    const double rho = rho_in[c], Y0 = Y_in[c], Y1 = Y_in[ncell + c], E = E_in[c];
    double T = T_io[c];
    double n[NS], logn[NS], vert[NS], dl[NS];
#pragma unroll
    for (int j = 0; j < NS; ++j) n[j] = j < ns ? n_io[(int64_t)j * ncell + c] : 0.0;

    const double logrhoRu = log(rho * RU / PST);
    double b0[NE], keep[NE];
    double b0max = 0.0;
#pragma unroll
    for (int i = 0; i < NE; ++i) {
        b0[i] = i < ne ? Y0 * t.b0f[i] + Y1 * t.b0o[i] : 0.0;
        keep[i] = 1.0;
    }
    // maxval(b0(1:ne)): the elements are amounts >= 0
    b0max = b0[0];
#pragma unroll
    for (int i = 1; i < NE; ++i)
        if (i < ne && b0[i] > b0max) b0max = b0[i];
    const int mode = Y0 < Y_EPS ? 1 : (Y1 < Y_EPS ? 2 : 0);
    if (mode) {
#pragma unroll
        for (int j = 0; j < NS; ++j)
            if (j < ns) n[j] = n[j] * (mode == 1 ? t.masko[j] : t.maskf[j]);
#pragma unroll
        for (int i = 0; i < NE; ++i) {
            keep[i] = i < ne ? (mode == 1 ? t.keepo[i] : t.keepf[i]) : 1.0;
            b0[i] = b0[i] * keep[i];
        }
    }
    double sn = 0.0;
#pragma unroll
    for (int j = 0; j < NS; ++j)
        if (j < ns) sn += n[j];
    const double tinyn = TSIZE * sn;
    const double logtinyn = log(tinyn);
    const double tinytinyn = TTSIZE * sn;
    const double logtinytinyn = log(tinytinyn);

    double logT = log(T);
    double vh[9];
    v_hrt(T, logT, vh);
    double b[NE], bE = 0.0;
#pragma unroll
    for (int i = 0; i < NE; ++i) b[i] = 0.0;
#pragma unroll
    for (int j = 0; j < NS; ++j) {
        vert[j] = 0.0;
        logn[j] = logtinyn;
        if (j < ns && n[j] > tinyn) {
            const int s = section<Tab, NSEC>(t, j, T);
            vert[j] = dot9(t.co[j][s], vh) - 1.0;
            logn[j] = log(n[j]);
#pragma unroll
            for (int i = 0; i < NE; ++i)
                if (i < ne) b[i] += t.ac[i][j] * n[j];
            bE += vert[j] * n[j];
        }
    }
    bool flag = true;
#pragma unroll
    for (int i = 0; i < NE; ++i)
        if (i < ne && b0[i] > EPS && fabs(b0[i] - b[i]) > b0max * EPS) flag = false;
    if (fabs(E - bE * RU * T) > EPS * fabs(E)) flag = false;

    int counter = 0;
    bool singular = false;
    if (!flag) {
        counter = 1;
        bool retried = false;
        for (;;) {
            const double b0E = E / (RU * T);
            double A[M][M], bd[M], vpi[M];
#pragma unroll
            for (int i = 0; i < NE; ++i) {
                b[i] = 0.0;
                bd[i] = b0[i];
            }
            bd[NE] = b0E - bE;
#pragma unroll
            for (int i = 0; i < M; ++i)
#pragma unroll
                for (int j = 0; j < M; ++j) A[i][j] = 0.0;
            double vm[9], vc[9];
            v_murt(T, logT, vm);
            v_cpr(T, vc);
            double aEE = 0.0;
#pragma unroll
            for (int k = 0; k < NS; ++k) {
                if (k >= ns) continue;
                const int s = section<Tab, NSEC>(t, k, T);
                dl[k] = dot9(t.co[k][s], vm) + logrhoRu + logT + logn[k];
                if (n[k] > tinyn) {
                    const double vmurtn = dl[k] * n[k];
#pragma unroll
                    for (int i = 0; i < NE; ++i) {
                        if (i >= ne) continue;
                        const double aik = t.ac[i][k];
#pragma unroll
                        for (int j = i; j < NE; ++j)
                            if (j < ne) A[i][j] += aik * t.ac[j][k] * n[k];
                        A[i][NE] += aik * vert[k] * n[k];
                        b[i] += aik * n[k];
                        bd[i] += aik * (vmurtn - n[k]);
                    }
                    aEE += n[k] * (vert[k] * vert[k] + dot9(t.co[k][s], vc) - 1.0);
                    bd[NE] += vmurtn * vert[k];
                }
            }
            A[NE][NE] = aEE;
#pragma unroll
            for (int i = 0; i < M; ++i)
#pragma unroll
                for (int j = i + 1; j < M; ++j) A[j][i] = A[i][j];
            // unused element slots (ne < NE) and dropped elements: identity rows
#pragma unroll
            for (int r = 0; r < NE; ++r) {
                if (r < ne && keep[r] != 0.0) continue;
#pragma unroll
                for (int j = 0; j < M; ++j) {
                    A[r][j] = 0.0;
                    A[j][r] = 0.0;
                }
                A[r][r] = 1.0;
                bd[r] = 0.0;
            }
            // LU.f90: partial pivoting (first largest |A(i,k)|), singular when
            // the pivot is below 1e-30
            bool sing = false;
#pragma unroll
            for (int k = 0; k < M; ++k) {
                double p = fabs(A[k][k]);
                int ip = k;
#pragma unroll
                for (int i = k + 1; i < M; ++i) {
                    const double d = fabs(A[i][k]);
                    if (p < d) {
                        p = d;
                        ip = i;
                    }
                }
                if (p < 1e-30) sing = true;
                // unconditional selects: a predicated swap makes the
                // compiler index the rows by ip and move A to local memory
#pragma unroll
                for (int i = k + 1; i < M; ++i) {
                    const bool sw = i == ip;
#pragma unroll
                    for (int j = 0; j < M; ++j) {
                        const double x = A[k][j], y = A[i][j];
                        A[k][j] = sw ? y : x;
                        A[i][j] = sw ? x : y;
                    }
                    const double x = bd[k], y = bd[i];
                    bd[k] = sw ? y : x;
                    bd[i] = sw ? x : y;
                }
                const double inv = 1.0 / A[k][k];
#pragma unroll
                for (int i = k + 1; i < M; ++i) A[i][k] = A[i][k] * inv;
#pragma unroll
                for (int j = k + 1; j < M; ++j) {
                    const double a = A[k][j];
#pragma unroll
                    for (int i = k + 1; i < M; ++i) A[i][j] = A[i][j] - a * A[i][k];
                }
            }
            if (sing) {
                if (retried) {  // the reference writes its debug state and stops
                    singular = true;
                    break;
                }
                retried = true;
                bE = 0.0;
#pragma unroll
                for (int j = 0; j < NS; ++j) {
                    if (j >= ns) continue;
                    n[j] = n[j] + INITIAL_EPS;
                    logn[j] = logtinytinyn;
                    if (n[j] < tinytinyn)
                        n[j] = tinytinyn;
                    else
                        logn[j] = log(n[j]);
                    if (n[j] > tinyn) {
                        vert[j] = dot9(t.co[j][section<Tab, NSEC>(t, j, T)], vh) - 1.0;
                        bE += vert[j] * n[j];
                    }
                }
                sn = 0.0;
#pragma unroll
                for (int j = 0; j < NS; ++j)
                    if (j < ns) sn += n[j];
                continue;
            }
            double cc[M];
#pragma unroll
            for (int k = 0; k < M; ++k) {
                cc[k] = bd[k];
#pragma unroll
                for (int j = 0; j < k; ++j) cc[k] = cc[k] - A[k][j] * cc[j];
            }
            vpi[M - 1] = cc[M - 1] / A[M - 1][M - 1];
#pragma unroll
            for (int k = M - 2; k >= 0; --k) {
                double x = cc[k];
#pragma unroll
                for (int j = k + 1; j < M; ++j) x = x - A[k][j] * vpi[j];
                vpi[k] = x / A[k][k];
            }
#pragma unroll
            for (int r = 0; r < NE; ++r)
                if (r < ne && keep[r] == 0.0) vpi[r] = -1e300;

            const double dlogT = vpi[NE];
#pragma unroll
            for (int j = 0; j < NS; ++j) {
                if (j >= ns) continue;
                double s = 0.0;
#pragma unroll
                for (int i = 0; i < NE; ++i)
                    if (i < ne) s += t.ac[i][j] * vpi[i];
                dl[j] = -dl[j] + s + vert[j] * dlogT;
            }
            double lambda1 = 0.0, lambda2 = 1e300;
            const double logsn = log(sn);
#pragma unroll
            for (int j = 0; j < NS; ++j) {
                if (j >= ns) continue;
                if (logn[j] - logsn > -18.420681)
                    lambda1 = fmax(lambda1, fabs(dl[j]));
                else if (dl[j] > 0.0)
                    lambda2 = fmin(lambda2, fabs((-logn[j] + logsn - 9.2103404) / dl[j]));
            }
            lambda1 = 2.0 / fmax(fmax(5.0 * fabs(dlogT), fabs(lambda1)), 2.0);
            const double om = fmin(1.0, fmin(lambda1, lambda2));

            T = T * exp(om * dlogT);
            logT = log(T);
            bE = 0.0;
            double dnmax = 0.0;
            v_hrt(T, logT, vh);
#pragma unroll
            for (int j = 0; j < NS; ++j) {
                if (j >= ns) continue;
                n[j] = n[j] * exp(om * dl[j]);
                logn[j] = logtinytinyn;
                if (n[j] < tinytinyn)
                    n[j] = tinytinyn;
                else
                    logn[j] = log(n[j]);
                if (n[j] > tinyn) {
                    vert[j] = dot9(t.co[j][section<Tab, NSEC>(t, j, T)], vh) - 1.0;
                    bE += vert[j] * n[j];
                    const double x = fabs(dl[j]) * n[j];
                    if (dnmax < x) dnmax = x;
                }
            }
            sn = 0.0;
#pragma unroll
            for (int j = 0; j < NS; ++j)
                if (j < ns) sn += n[j];
            flag = true;
            if (fabs(dnmax) > EPS * sn) flag = false;
#pragma unroll
            for (int i = 0; i < NE; ++i)
                if (i < ne && b0[i] > EPS && fabs(b0[i] - b[i]) > b0max * EPS) flag = false;
            if (fabs(dlogT) > EPS && fabs(E - bE * RU * T) > EPS * fabs(E)) flag = false;
            if (counter > MAX_ITER) flag = true;
            if (flag) break;
            ++counter;
        }
    }
    if (singular) atomicAdd(&fails[1], 1ull);
    else if (counter > MAX_ITER) atomicAdd(&fails[0], 1ull);

    T_io[c] = T;
#pragma unroll
    for (int j = 0; j < NS; ++j)
        if (j < ns) n_io[(int64_t)j * ncell + c] = n[j];
    if (out.iters) out.iters[c] = singular ? -1 : counter;
    if (out.mwave) out.mwave[c] = 1e3 / sn;

    // kappa, vhi, DHi (sub_chem.f90:1596-1628)
    double vc[9];
    v_cpr(T, vc);
    double kap = 0.0;
#pragma unroll
    for (int i = 0; i < NS; ++i)
        if (i < ns && n[i] > tinyn) kap += n[i] * dot9(t.co[i][section<Tab, NSEC>(t, i, T)], vc);
    kap = kap / (kap - sn);
    if (out.kappa) out.kappa[c] = kap;
    const double rt = RU * T;
    double vhe[NE], mwd[NE];
#pragma unroll
    for (int i = 0; i < NE; ++i) vhe[i] = mwd[i] = 0.0;
#pragma unroll
    for (int i = 0; i < NS; ++i) {
        if (i >= ns) continue;
        const double dh = dot9(t.co[i][section<Tab, NSEC>(t, i, T)], vh);
        if (out.vhi) out.vhi[(int64_t)i * ncell + c] = rt / t.mw[i] * dh * 1e3;
        const double tmp2 = rt * n[i] * dh;
#pragma unroll
        for (int j = 0; j < NE; ++j) {
            if (j >= ne) continue;
            vhe[j] += t.yac[j][i] * tmp2;
            mwd[j] += t.yac[j][i] * n[i];
        }
    }
    if (out.DHi) {
        double d0 = 0.0, d1 = 0.0;
#pragma unroll
        for (int i = 0; i < NE; ++i) {
            if (i >= ne) continue;
            const double x = 1.0 / (Y0 * t.yfe[i] + Y1 * t.yoe[i] + 1e-300) *
                             (kap * RU * mwd[i] * T - (kap - 1.0) * vhe[i]);
            d0 += t.yfe[i] * x;
            d1 += t.yoe[i] * x;
        }
        out.DHi[c] = d0;
        out.DHi[ncell + c] = d1;
    }
    if (out.Yv) {
#pragma unroll
        for (int i = 0; i < NS; ++i)
            if (i < ns) out.Yv[(int64_t)i * ncell + c] = n[i] * t.mw[i] * 1e-3;
    }
    if (out.mu) {
        // calc_vTmu (func_chem.f90:143-155) and the Wilke mixing rule
        const double tt = 1.0 / (T * T);
        const double vmu1 = tt * T, vmu2 = tt;
        // sqrt(muN_i / muN_j) as sqrt(muN_i) * rsqrt(muN_j): nt square roots
        // instead of nt^2 (a few ulp apart from the quotient's root)
        double sq[NS], rs[NS];
#pragma unroll
        for (int i = 0; i < NS; ++i) {
            sq[i] = rs[i] = 0.0;
            if (i >= nt) continue;
            const int s = tsection(t.tthi[i], t.ttlo[i], t.ntsec[i], T);
            const double* a = t.trans[i][s];
            const double muN = exp(a[0] * logT + a[1] * vmu1 + a[2] * vmu2 + a[3] * 1.0);
            sq[i] = sqrt(muN);
            rs[i] = rsqrt(muN);
        }
        double nfit[NS];  // n(tr2th(i))
#pragma unroll
        for (int i = 0; i < NS; ++i) {
            nfit[i] = 0.0;
#pragma unroll
            for (int k = 0; k < NS; ++k)
                if (i < nt && k == t.tr2th[i]) nfit[i] = n[k];
        }
        double mu = 0.0;
#pragma unroll
        for (int i = 0; i < NS; ++i) {
            if (i >= nt) continue;
            double denom = 0.0;
#pragma unroll
            for (int j = 0; j < NS; ++j) {
                if (j >= nt) continue;
                const double f = 1.0 + sq[i] * rs[j] * t.wmw[i][j];
                const double phi = 0.25 * (f * f) * t.wsq[i][j];
                denom += nfit[j] * phi;
            }
            mu += nfit[i] * (sq[i] * sq[i]) / denom;
        }
        out.mu[c] = mu * 1e-7;
    }
}

// LU.f90 on a register matrix (partial pivoting, singular below 1e-30), row
// swaps as unconditional selects; x = A^-1 b.  Returns false when singular.
template <int M>
__device__ __forceinline__ bool lu_solve_reg(double (&A)[M][M], double (&bd)[M], double (&x)[M]) {
    bool sing = false;
#pragma unroll
    for (int k = 0; k < M; ++k) {
        double p = fabs(A[k][k]);
        int ip = k;
#pragma unroll
        for (int i = k + 1; i < M; ++i) {
            const double d = fabs(A[i][k]);
            if (p < d) {
                p = d;
                ip = i;
            }
        }
        if (p < 1e-30) sing = true;
#pragma unroll
        for (int i = k + 1; i < M; ++i) {
            const bool sw = i == ip;
#pragma unroll
            for (int j = 0; j < M; ++j) {
                const double a = A[k][j], b = A[i][j];
                A[k][j] = sw ? b : a;
                A[i][j] = sw ? a : b;
            }
            const double a = bd[k], b = bd[i];
            bd[k] = sw ? b : a;
            bd[i] = sw ? a : b;
        }
        const double inv = 1.0 / A[k][k];
#pragma unroll
        for (int i = k + 1; i < M; ++i) A[i][k] = A[i][k] * inv;
#pragma unroll
        for (int j = k + 1; j < M; ++j) {
            const double a = A[k][j];
#pragma unroll
            for (int i = k + 1; i < M; ++i) A[i][j] = A[i][j] - a * A[i][k];
        }
    }
    double cc[M];
#pragma unroll
    for (int k = 0; k < M; ++k) {
        cc[k] = bd[k];
#pragma unroll
        for (int j = 0; j < k; ++j) cc[k] = cc[k] - A[k][j] * cc[j];
    }
    x[M - 1] = cc[M - 1] / A[M - 1][M - 1];
#pragma unroll
    for (int k = M - 2; k >= 0; --k) {
        double v = cc[k];
#pragma unroll
        for (int j = k + 1; j < M; ++j) v = v - A[k][j] * x[j];
        x[k] = v / A[k][k];
    }
    return !sing;
}

struct HpTpOut {
    double* h;  // tp: mixture enthalpy
    double* mwave;
    double* kappa;
    double* mu;
    double* Yv;
    double* vhi;
    int32_t* iters;
};

// cea_hp (HP) and cea_tp (sub_chem.f90:1652-2248), one cell per thread.  The
// unknowns are pi_0..pi_{ne-1}, ln sn (slot NE) and for hp ln T (slot NE+1);
// as in k_cea, dropped and unused element slots are identity rows.  The
// singular-matrix retry, unbounded in the reference, counts towards the
// 500-iteration limit.
template <int NS, int NE, int NSEC, bool EXACT, bool HP>
__global__ void __launch_bounds__(128, 2) k_cea_hptp(const CeaTab<NS, NE, NSEC>* __restrict__ gtab, int64_t ncell,
                                                    const double* __restrict__ p_in, const double* __restrict__ Y_in,
                                                    const double* __restrict__ h_in, double* __restrict__ T_io,
                                                    double* __restrict__ n_io, HpTpOut out,
                                                    unsigned long long* __restrict__ fails) {
    using Tab = CeaTab<NS, NE, NSEC>;
    extern __shared__ double smem_tab[];
    {
        const double* src = reinterpret_cast<const double*>(gtab);
        for (int k = threadIdx.x; k < (int)(sizeof(Tab) / sizeof(double)); k += blockDim.x) smem_tab[k] = src[k];
    }
    __syncthreads();
    const Tab& t = *reinterpret_cast<const Tab*>(smem_tab);
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    const int ns = EXACT ? NS : t.ns, ne = EXACT ? NE : t.ne, nt = t.nt;
    constexpr int M = HP ? NE + 2 : NE + 1;
    constexpr int SN = NE, LT = NE + 1;

    const double Y0 = Y_in[c], Y1 = Y_in[ncell + c];
    const double H = HP ? h_in[c] : 0.0;
    double T = T_io[c];
    double n[NS], logn[NS], vhrt[NS], dl[NS];
#pragma unroll
    for (int j = 0; j < NS; ++j) n[j] = j < ns ? n_io[(int64_t)j * ncell + c] : 0.0;

    const double logP = log(p_in[c] / PST);
    double b0[NE], keep[NE];
#pragma unroll
    for (int i = 0; i < NE; ++i) {
        b0[i] = i < ne ? Y0 * t.b0f[i] + Y1 * t.b0o[i] : 0.0;  // not masked in hp / tp
        keep[i] = 1.0;
    }
    double b0max = b0[0];
#pragma unroll
    for (int i = 1; i < NE; ++i)
        if (i < ne && b0[i] > b0max) b0max = b0[i];
    double sn = 0.0;
#pragma unroll
    for (int j = 0; j < NS; ++j)
        if (j < ns) sn += n[j];
    double b0sn = sn;  // b0(ne+1)
    const int mode = Y0 < Y_EPS ? 1 : (Y1 < Y_EPS ? 2 : 0);
    if (mode) {
#pragma unroll
        for (int j = 0; j < NS; ++j)
            if (j < ns) n[j] = n[j] * (mode == 1 ? t.masko[j] : t.maskf[j]);
#pragma unroll
        for (int i = 0; i < NE; ++i) keep[i] = i < ne ? (mode == 1 ? t.keepo[i] : t.keepf[i]) : 1.0;
    }
    const double tinyn = TSIZE * sn;
    const double logtinyn = log(tinyn);
    const double tinytinyn = TTSIZE * sn;
    const double logtinytinyn = log(tinytinyn);

    double logT = log(T);
    double vh[9];
    v_hrt(T, logT, vh);
    double b[NE], bsn = sn, bh = 0.0;  // b(1:ne), b(ne+1), b(ne+2)
#pragma unroll
    for (int i = 0; i < NE; ++i) b[i] = 0.0;
#pragma unroll
    for (int j = 0; j < NS; ++j) {
        vhrt[j] = 0.0;
        logn[j] = logtinyn;
        if (j < ns && n[j] > tinyn) {
            if (HP) vhrt[j] = dot9(t.co[j][section<Tab, NSEC>(t, j, T)], vh);
            logn[j] = log(n[j]);
#pragma unroll
            for (int i = 0; i < NE; ++i)
                if (i < ne) b[i] += t.ac[i][j] * n[j];
            bh += vhrt[j] * n[j];
        }
    }
    bool flag = true;
#pragma unroll
    for (int i = 0; i < NE; ++i)
        if (i < ne && b0[i] > EPS && fabs(b0[i] - b[i]) > b0max * EPS) flag = false;
    if (HP && fabs(H - bh * RU * T) > EPS * fabs(H)) flag = false;

    int counter = 0;
    if (!flag) {
        counter = 1;
        for (;;) {
            double A[M][M], bd[M], vpi[M];
#pragma unroll
            for (int i = 0; i < M; ++i)
#pragma unroll
                for (int j = 0; j < M; ++j) A[i][j] = 0.0;
#pragma unroll
            for (int i = 0; i < NE; ++i) {
                b[i] = 0.0;
                bd[i] = b0[i];
            }
            bd[SN] = b0sn - bsn;
            if constexpr (HP) bd[LT] = H / (RU * T) - bh;
            double vm[9], vc[9];
            v_murt(T, logT, vm);
            if (HP) v_cpr(T, vc);
            const double lb0sn = log(b0sn);
            double aSL = 0.0, aLL = 0.0;
#pragma unroll
            for (int k = 0; k < NS; ++k) {
                if (k >= ns) continue;
                const int s = section<Tab, NSEC>(t, k, T);
                dl[k] = dot9(t.co[k][s], vm) + logn[k] - lb0sn + logP;
                if (n[k] > tinyn) {
                    const double vmurtn = dl[k] * n[k];
#pragma unroll
                    for (int i = 0; i < NE; ++i) {
                        if (i >= ne) continue;
                        const double aik = t.ac[i][k];
#pragma unroll
                        for (int j = i; j < NE; ++j)
                            if (j < ne) A[i][j] += aik * t.ac[j][k] * n[k];
                        A[i][SN] += aik * n[k];
                        if constexpr (HP) A[i][LT] += aik * vhrt[k] * n[k];
                        b[i] += aik * n[k];
                        bd[i] += aik * (vmurtn - n[k]);
                    }
                    if constexpr (HP) {
                        aSL += n[k] * vhrt[k];
                        aLL += n[k] * (vhrt[k] * vhrt[k] + dot9(t.co[k][s], vc));
                        bd[LT] += vmurtn * vhrt[k];
                    }
                    bd[SN] += vmurtn;
                }
            }
            A[SN][SN] = bsn - b0sn;
            if constexpr (HP) {
                A[SN][LT] = aSL;
                A[LT][LT] = aLL;
            }
#pragma unroll
            for (int i = 0; i < M; ++i)
#pragma unroll
                for (int j = i + 1; j < M; ++j) A[j][i] = A[i][j];
#pragma unroll
            for (int r = 0; r < NE; ++r) {
                if (r < ne && keep[r] != 0.0) continue;
#pragma unroll
                for (int j = 0; j < M; ++j) {
                    A[r][j] = 0.0;
                    A[j][r] = 0.0;
                }
                A[r][r] = 1.0;
                bd[r] = 0.0;
            }
            if (!lu_solve_reg<M>(A, bd, vpi)) {
                sn = 0.0;
                bh = 0.0;
#pragma unroll
                for (int j = 0; j < NS; ++j) {
                    if (j >= ns) continue;
                    n[j] = n[j] + INITIAL_EPS;
                    logn[j] = logtinytinyn;
                    if (n[j] < tinytinyn)
                        n[j] = tinytinyn;
                    else
                        logn[j] = log(n[j]);
                    if (n[j] > tinyn) {
                        if (HP) {
                            vhrt[j] = dot9(t.co[j][section<Tab, NSEC>(t, j, T)], vh);
                            bh += vhrt[j] * n[j];
                        }
                        sn += n[j];
                    }
                }
                bsn = sn;
                counter = counter + 1;
                if (counter > MAX_ITER) break;
                continue;
            }
#pragma unroll
            for (int r = 0; r < NE; ++r)
                if (r < ne && keep[r] == 0.0) vpi[r] = -1e300;
            const double dlsn = vpi[SN];
            const double dlogT = HP ? vpi[LT] : 0.0;
#pragma unroll
            for (int j = 0; j < NS; ++j) {
                if (j >= ns) continue;
                double x = 0.0;
#pragma unroll
                for (int i = 0; i < NE; ++i)
                    if (i < ne) x += t.ac[i][j] * vpi[i];
                dl[j] = HP ? -dl[j] + x + dlsn + vhrt[j] * dlogT : -dl[j] + x + dlsn;
            }
            double lambda1 = 0.0, lambda2 = 1e300;
            const double logsn = lb0sn;
#pragma unroll
            for (int j = 0; j < NS; ++j) {
                if (j >= ns) continue;
                if (logn[j] - logsn > -18.420681)
                    lambda1 = fmax(lambda1, fabs(dl[j]));
                else if (dl[j] > 0.0)
                    lambda2 = fmin(lambda2, fabs((-logn[j] + logsn - 9.2103404) / (dl[j] - dlsn)));
            }
            if (HP)
                lambda1 = 2.0 / fmax(fmax(fmax(5.0 * fabs(dlogT), 5.0 * fabs(dlsn)), fabs(lambda1)), 2.0);
            else
                lambda1 = 2.0 / fmax(fmax(5.0 * fabs(dlsn), fabs(lambda1)), 2.0);
            const double om = fmin(1.0, fmin(lambda1, lambda2));
            b0sn = b0sn * exp(om * dlsn);
            if (HP) {
                T = T * exp(om * dlogT);
                logT = log(T);
                v_hrt(T, logT, vh);
            }
            sn = 0.0;
            bh = 0.0;
            double dnmax = 0.0;
#pragma unroll
            for (int j = 0; j < NS; ++j) {
                if (j >= ns) continue;
                n[j] = n[j] * exp(om * dl[j]);
                logn[j] = logtinytinyn;
                if (n[j] < tinytinyn)
                    n[j] = tinytinyn;
                else
                    logn[j] = log(n[j]);
                if (n[j] > tinyn) {
                    if (HP) {
                        vhrt[j] = dot9(t.co[j][section<Tab, NSEC>(t, j, T)], vh);
                        bh += vhrt[j] * n[j];
                    }
                    sn += n[j];
                    const double x = fabs(dl[j]) * n[j];
                    if (dnmax < x) dnmax = x;
                }
            }
            bsn = sn;
            flag = true;
            if (fabs(dnmax) > EPS * sn) flag = false;
#pragma unroll
            for (int i = 0; i < NE; ++i)
                if (i < ne && b0[i] > EPS && fabs(b0[i] - b[i]) > b0max * EPS) flag = false;
            if (fabs(dlsn) > EPS || fabs(b0sn - bsn) > EPS * fabs(sn)) flag = false;
            if (HP && (fabs(dlogT) > EPS || fabs(H - bh * RU * T) > EPS * fabs(H))) flag = false;
            if (counter > MAX_ITER) flag = true;
            if (flag) break;
            ++counter;
        }
    }
    if (counter > MAX_ITER) atomicAdd(&fails[0], 1ull);
    if (HP) T_io[c] = T;
#pragma unroll
    for (int j = 0; j < NS; ++j)
        if (j < ns) n_io[(int64_t)j * ncell + c] = n[j];
    if (out.iters) out.iters[c] = counter;
    if (out.mwave) out.mwave[c] = 1e3 / sn;
    double vc[9];
    v_cpr(T, vc);
    double kap = 0.0;
#pragma unroll
    for (int i = 0; i < NS; ++i)
        if (i < ns && n[i] > tinyn) kap += n[i] * dot9(t.co[i][section<Tab, NSEC>(t, i, T)], vc);
    if (out.kappa) out.kappa[c] = kap / (kap - sn);
    v_hrt(T, logT, vh);
    const double rt3 = RU * 1e3 * T;
    double hsum = 0.0;
#pragma unroll
    for (int i = 0; i < NS; ++i) {
        if (i >= ns) continue;
        const double dh = dot9(t.co[i][section<Tab, NSEC>(t, i, T)], vh);
        if (out.vhi) out.vhi[(int64_t)i * ncell + c] = rt3 / t.mw[i] * dh;
        hsum += n[i] * dh;
        if (out.Yv) out.Yv[(int64_t)i * ncell + c] = n[i] * t.mw[i] * 1e-3;
    }
    if (!HP && out.h) out.h[c] = hsum * RU * T;
    if (out.mu) {
        const double tt = 1.0 / (T * T);
        double sq[NS], rs[NS], nfit[NS];
#pragma unroll
        for (int i = 0; i < NS; ++i) {
            sq[i] = rs[i] = nfit[i] = 0.0;
            if (i >= nt) continue;
            const int s = tsection(t.tthi[i], t.ttlo[i], t.ntsec[i], T);
            const double* a = t.trans[i][s];
            const double muN = exp(a[0] * logT + a[1] * (tt * T) + a[2] * tt + a[3] * 1.0);
            sq[i] = sqrt(muN);
            rs[i] = rsqrt(muN);
#pragma unroll
            for (int k = 0; k < NS; ++k)
                if (k == t.tr2th[i]) nfit[i] = n[k];
        }
        double mu = 0.0;
#pragma unroll
        for (int i = 0; i < NS; ++i) {
            if (i >= nt) continue;
            double denom = 0.0;
#pragma unroll
            for (int j = 0; j < NS; ++j) {
                if (j >= nt) continue;
                const double f = 1.0 + sq[i] * rs[j] * t.wmw[i][j];
                denom += nfit[j] * (0.25 * (f * f) * t.wsq[i][j]);
            }
            mu += nfit[i] * (sq[i] * sq[i]) / denom;
        }
        out.mu[c] = mu * 1e-7;
    }
}

template <class Tab>
void fill_tab(Tab& t, const scfd_cea_data& d, const double* b0f, const double* b0o, const double* yfe,
              const double* yoe, const double* maskf, const double* masko, const double* keepf,
              const double* keepo, const std::vector<double>& yac) {
    std::memset(&t, 0, sizeof(Tab));
    t.ns = d.ns;
    t.ne = d.ne;
    t.nt = d.nt;
    const int nsecmax = (int)(sizeof(t.thi[0]) / sizeof(double));
    for (int j = 0; j < d.ns; ++j) {
        t.nsec[j] = d.nsec[j];
        t.tlo[j] = d.trange[j][0][0];
        for (int l = 0; l < d.nsec[j] && l < nsecmax; ++l) {
            t.thi[j][l] = d.trange[j][l][1];
            for (int k = 0; k < 9; ++k) t.co[j][l][k] = d.co[j][l][k];
        }
        t.mw[j] = d.mw[j];
        for (int i = 0; i < d.ne; ++i) {
            t.ac[i][j] = d.ac[j][i];
            t.yac[i][j] = yac[(size_t)i * d.ns + j];
        }
        t.maskf[j] = maskf[j];
        t.masko[j] = masko[j];
    }
    for (int i = 0; i < d.nt; ++i) {
        t.ntsec[i] = d.ntsec[i];
        t.tr2th[i] = d.tr2th[i];
        t.ttlo[i] = d.trange_t[i][0][0];
        for (int l = 0; l < d.ntsec[i]; ++l) {
            t.tthi[i][l] = d.trange_t[i][l][1];
            for (int k = 0; k < 4; ++k) t.trans[i][l][k] = d.trans[i][l][k];
        }
    }
    for (int i = 0; i < d.nt; ++i)
        for (int j = 0; j < d.nt; ++j) {
            const double mi = d.mw[d.tr2th[i]], mj = d.mw[d.tr2th[j]];
            t.wmw[i][j] = std::pow(mj / mi, 0.25);
            t.wsq[i][j] = std::sqrt(2.0 * mj / (mi + mj));
        }
    for (int i = 0; i < d.ne; ++i) {
        t.b0f[i] = b0f[i];
        t.b0o[i] = b0o[i];
        t.yfe[i] = yfe[i];
        t.yoe[i] = yoe[i];
        t.keepf[i] = keepf[i];
        t.keepo[i] = keepo[i];
    }
}

}  // namespace

enum { KIND_9_3 = 0, KIND_SMALL = 1, KIND_BIG = 2 };

struct scfd_cea {
    scfd_cea_data data;
    scfd_cea_info info;
    int kind = KIND_SMALL;
    void* d_tab = nullptr;
    size_t tab_bytes = 0;
    unsigned long long* d_fail = nullptr;
    cudaStream_t last = nullptr;
};

namespace {

int cea_launch(scfd_cea* h, int64_t ncell, const double* rho, const double* Y, const double* e, double* T,
               double* n, const CellOut& out, cudaStream_t st) {
    if (ncell == 0) return 0;
    const int threads = 128;
    const int64_t blocks = (ncell + threads - 1) / threads;
    if (blocks > 0x7fffffff) return SCFD_E_ARG;
    // three resident blocks of 128 threads (168 registers) measured faster
    // than two (no spills) and than four (more spills) on B200
    if (h->kind == KIND_9_3)
        k_cea<9, 3, 3, true, 3><<<(unsigned)blocks, threads, sizeof(TabH2Air), st>>>(
            (const TabH2Air*)h->d_tab, ncell, rho, Y, e, T, n, out, h->d_fail);
    else if (h->kind == KIND_SMALL)
        k_cea<12, 4, 3, false, 3><<<(unsigned)blocks, threads, sizeof(TabSmall), st>>>(
            (const TabSmall*)h->d_tab, ncell, rho, Y, e, T, n, out, h->d_fail);
    else
        k_cea<SCFD_CEA_MAX_SPECIES, SCFD_CEA_MAX_ELEMENTS, SCFD_CEA_MAX_SECTIONS, false, 1>
            <<<(unsigned)blocks, threads, sizeof(TabBig), st>>>((const TabBig*)h->d_tab, ncell, rho, Y, e, T, n,
                                                                 out, h->d_fail);
    return cudaGetLastError() == cudaSuccess ? 0 : SCFD_E_CUDA;
}

template <bool HP>
int cea_hptp_launch(scfd_cea* h, int64_t ncell, const double* p, const double* Y, const double* hh, double* T,
                    double* n, const HpTpOut& out, cudaStream_t st) {
    if (ncell == 0) return 0;
    const int threads = 128;
    const int64_t blocks = (ncell + threads - 1) / threads;
    if (blocks > 0x7fffffff) return SCFD_E_ARG;
    if (h->kind == KIND_9_3)
        k_cea_hptp<9, 3, 3, true, HP><<<(unsigned)blocks, threads, sizeof(TabH2Air), st>>>(
            (const TabH2Air*)h->d_tab, ncell, p, Y, hh, T, n, out, h->d_fail);
    else if (h->kind == KIND_SMALL)
        k_cea_hptp<12, 4, 3, false, HP><<<(unsigned)blocks, threads, sizeof(TabSmall), st>>>(
            (const TabSmall*)h->d_tab, ncell, p, Y, hh, T, n, out, h->d_fail);
    else
        k_cea_hptp<SCFD_CEA_MAX_SPECIES, SCFD_CEA_MAX_ELEMENTS, SCFD_CEA_MAX_SECTIONS, false, HP>
            <<<(unsigned)blocks, threads, sizeof(TabBig), st>>>((const TabBig*)h->d_tab, ncell, p, Y, hh, T, n, out,
                                                                 h->d_fail);
    return cudaGetLastError() == cudaSuccess ? 0 : SCFD_E_CUDA;
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

// calc_ini of initialize_cea (sub_chem.f90:1237-1287): moles per kg, the
// energy at T, the mixture weight and the element mass fractions
void calc_ini(const scfd_cea_data& d, const std::vector<double>& yac, double T, double* n, double* E, double* mw,
              double* ye) {
    double sn = 0.0, sm = 0.0;
    for (int j = 0; j < d.ns; ++j) {
        sn += n[j];
        sm += n[j] * d.mw[j];
    }
    *mw = sm / sn;
    for (int j = 0; j < d.ns; ++j) n[j] = n[j] / sm * 1e3;
    double vh[9];
    {
        const double logT = std::log(T);
        double tt = 1.0 / (T * T);
        vh[0] = -tt;
        tt = tt * T;
        vh[1] = tt * logT;
        vh[7] = tt;
        tt = tt * T;
        vh[2] = tt;
        tt = tt * T;
        vh[3] = tt / 2.0;
        tt = tt * T;
        vh[4] = tt / 3.0;
        tt = tt * T;
        vh[5] = tt / 4.0;
        tt = tt * T;
        vh[6] = tt / 5.0;
        vh[8] = 0.0;
    }
    double e = 0.0;
    for (int j = 0; j < d.ns; ++j) {
        int s = -1;
        if (d.trange[j][0][0] > T)
            s = 0;
        else
            for (int l = 0; l < d.nsec[j]; ++l)
                if (d.trange[j][l][1] > T) {
                    s = l;
                    break;
                }
        if (s < 0) s = d.nsec[j] - 1;
        double x = -1.0;
        for (int k = 0; k < 9; ++k) x = x + vh[k] * d.co[j][s][k];
        e = e + x * n[j];
    }
    *E = e * RU * T;
    for (int i = 0; i < d.ne; ++i) ye[i] = 0.0;
    for (int j = 0; j < d.ns; ++j) {
        const double x = n[j] * d.mw[j] * 1e-3;
        for (int i = 0; i < d.ne; ++i) ye[i] = ye[i] + yac[(size_t)i * d.ns + j] * x;
    }
}

}  // namespace

extern "C" {

int scfd_cea_create(const scfd_cea_data* data, scfd_cea** out) {
    if (!data || !out) return SCFD_E_ARG;
    *out = nullptr;
    const scfd_cea_data& d = *data;
    if (!valid(d)) return SCFD_E_ARG;
    scfd_cea* h = new scfd_cea();
    h->data = d;
    const int ns = d.ns, ne = d.ne;
    // YAc (set_therm_data, sub_chem.f90:159-170)
    std::vector<double> yac((size_t)ne * ns);
    for (int j = 0; j < ns; ++j) {
        double s = 0.0;
        for (int i = 0; i < ne; ++i) {
            yac[(size_t)i * ns + j] = d.mwe[i] * d.ac[j][i];
            s = s + yac[(size_t)i * ns + j];
        }
        s = 1.0 / s;
        for (int i = 0; i < ne; ++i) yac[(size_t)i * ns + j] *= s;
    }
    // initialize_cea (sub_chem.f90:1136-1230)
    scfd_cea_info& inf = h->info;
    std::memset(&inf, 0, sizeof(inf));
    double sumo = 0.0, sumf = 0.0;
    for (int j = 0; j < ns; ++j) {
        sumo += d.mw[j] * d.no[j];
        sumf += d.mw[j] * d.nf[j];
    }
    inf.of = sumo / sumf;
    std::vector<double> nf(d.nf, d.nf + ns), no(d.no, d.no + ns);
    double Ef, Eo, MWf, MWo;
    calc_ini(d, yac, d.Tf, nf.data(), &Ef, &MWf, inf.fuel.ye);
    calc_ini(d, yac, d.To, no.data(), &Eo, &MWo, inf.oxidizer.ye);
    double b0f[SCFD_CEA_MAX_ELEMENTS] = {0}, b0o[SCFD_CEA_MAX_ELEMENTS] = {0};
    for (int j = 0; j < ns; ++j)
        for (int i = 0; i < ne; ++i) {
            b0f[i] = b0f[i] + d.ac[j][i] * nf[j];
            b0o[i] = b0o[i] + d.ac[j][i] * no[j];
        }
    double keepf[SCFD_CEA_MAX_ELEMENTS], keepo[SCFD_CEA_MAX_ELEMENTS];
    std::vector<double> maskf(ns, 1.0), masko(ns, 1.0);
    for (int i = 0; i < ne; ++i) {
        keepf[i] = b0f[i] == 0.0 ? 0.0 : 1.0;
        keepo[i] = b0o[i] == 0.0 ? 0.0 : 1.0;
        inf.fuel.b0[i] = b0f[i];
        inf.oxidizer.b0[i] = b0o[i];
    }
    for (int j = 0; j < ns; ++j)
        for (int i = 0; i < ne; ++i) {
            if (keepo[i] == 0.0 && d.ac[j][i] != 0.0) masko[j] = 1e-100;
            if (keepf[i] == 0.0 && d.ac[j][i] != 0.0) maskf[j] = 1e-100;
        }
    int nsecmax = 1, ntsecmax = 1;
    for (int j = 0; j < ns; ++j) nsecmax = std::max(nsecmax, d.nsec[j]);
    for (int i = 0; i < d.nt; ++i) ntsecmax = std::max(ntsecmax, d.ntsec[i]);
    const bool small = nsecmax <= 3 && ntsecmax <= 3;
    h->kind = small && ns == 9 && ne == 3 ? KIND_9_3 : (small && ns <= 12 && ne <= 4 ? KIND_SMALL : KIND_BIG);
    std::vector<char> tab;
    if (h->kind == KIND_9_3) {
        tab.resize(sizeof(TabH2Air));
        fill_tab(*(TabH2Air*)tab.data(), d, b0f, b0o, inf.fuel.ye, inf.oxidizer.ye, maskf.data(), masko.data(),
                 keepf, keepo, yac);
    } else if (h->kind == KIND_SMALL) {
        tab.resize(sizeof(TabSmall));
        fill_tab(*(TabSmall*)tab.data(), d, b0f, b0o, inf.fuel.ye, inf.oxidizer.ye, maskf.data(), masko.data(),
                 keepf, keepo, yac);
    } else {
        tab.resize(sizeof(TabBig));
        fill_tab(*(TabBig*)tab.data(), d, b0f, b0o, inf.fuel.ye, inf.oxidizer.ye, maskf.data(), masko.data(),
                 keepf, keepo, yac);
    }
    h->tab_bytes = tab.size();
    auto fail = [&](cudaError_t) {
        scfd_cea_destroy(h);
        return SCFD_E_CUDA;
    };
    cudaError_t e = cudaMalloc(&h->d_tab, h->tab_bytes);
    if (e != cudaSuccess) return fail(e);
    e = cudaMalloc(&h->d_fail, 2 * sizeof(unsigned long long));
    if (e != cudaSuccess) return fail(e);
    if ((e = cudaMemcpy(h->d_tab, tab.data(), h->tab_bytes, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemset(h->d_fail, 0, 2 * sizeof(unsigned long long))) != cudaSuccess)
        return fail(e);

    // the two stream states: cea at the stream's own density and energy
    const double rhof = d.pf / (RU * 1e3 / MWf * d.Tf), rhoo = d.po / (RU * 1e3 / MWo * d.To);
    for (int j = 0; j < ns; ++j) {
        nf[j] = nf[j] + INITIAL_EPS;
        no[j] = no[j] + INITIAL_EPS;
    }
    // cell 0: fuel (Y = 1, 0); cell 1: oxidizer (Y = 0, 1).  'uv': cea at the
    // stream's rho and e; 'hp': cea_hp at its p and h = e + p/rho
    // (sub_chem.f90:1196-1228)
    std::vector<double> hbuf(2 * (6 + 3 * ns + 3 + 2), 0.0);
    double* rho = hbuf.data();
    double* Y = rho + 2;
    double* E = Y + 4;
    double* T = E + 2;
    double* n = T + 2;
    double* mwv = n + 2 * ns;
    double* kap = mwv + 2;
    double* mu = kap + 2;
    const double Es[2] = {Ef, Eo}, ps[2] = {d.pf, d.po};
    rho[0] = rhof;
    rho[1] = rhoo;
    Y[0] = 1.0;
    Y[1] = 0.0;
    Y[2] = 0.0;
    Y[3] = 1.0;
    for (int s2 = 0; s2 < 2; ++s2) E[s2] = d.init_hp ? Es[s2] + ps[s2] / rho[s2] : Es[s2];
    T[0] = d.Tf;
    T[1] = d.To;
    for (int j = 0; j < ns; ++j) {
        n[2 * j] = nf[j];
        n[2 * j + 1] = no[j];
    }
    const size_t nb = hbuf.size() * sizeof(double);
    double* dbuf = nullptr;
    int32_t* dit = nullptr;
    if ((e = cudaMalloc(&dbuf, nb + 2 * sizeof(double) + 2 * sizeof(int32_t))) != cudaSuccess) return fail(e);
    double* dp = (double*)((char*)dbuf + nb);
    dit = (int32_t*)(dp + 2);
    int32_t it[2] = {0, 0};
    e = cudaMemcpy(dbuf, hbuf.data(), nb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dp, ps, sizeof(ps), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const size_t off_mw = (size_t)(mwv - hbuf.data());
        const size_t off_T = (size_t)(T - hbuf.data()), off_n = (size_t)(n - hbuf.data());
        int rc;
        if (d.init_hp) {
            HpTpOut o{nullptr, dbuf + off_mw, dbuf + off_mw + 2, dbuf + off_mw + 4, nullptr, nullptr, dit};
            rc = cea_hptp_launch<true>(h, 2, dp, dbuf + 2, dbuf + 6, dbuf + off_T, dbuf + off_n, o, 0);
        } else {
            CellOut o{dbuf + off_mw, dbuf + off_mw + 2, dbuf + off_mw + 4, nullptr, nullptr, nullptr, dit};
            rc = cea_launch(h, 2, dbuf, dbuf + 2, dbuf + 6, dbuf + off_T, dbuf + off_n, o, 0);
        }
        if (rc != 0) e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpy(hbuf.data(), dbuf, nb, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(it, dit, sizeof(it), cudaMemcpyDeviceToHost);
    }
    cudaFree(dbuf);
    if (e != cudaSuccess) return fail(e);
    unsigned long long hf[2];
    if ((e = cudaMemcpy(hf, h->d_fail, sizeof(hf), cudaMemcpyDeviceToHost)) != cudaSuccess) return fail(e);
    cudaMemset(h->d_fail, 0, sizeof(hf));
    if (hf[1]) {
        scfd_cea_destroy(h);
        return SCFD_E_SINGULAR;
    }
    scfd_cea_stream* st[2] = {&inf.fuel, &inf.oxidizer};
    for (int s2 = 0; s2 < 2; ++s2) {
        scfd_cea_stream& o = *st[s2];
        o.T = T[s2];
        o.mw = mwv[s2];
        o.kappa = kap[s2];
        o.mu = mu[s2];
        if (d.init_hp) {
            o.p = ps[s2];
            o.h = E[s2];
            o.rho = o.p / (RU * 1e3 / o.mw * o.T);
            o.e = o.h - o.p / o.rho;
        } else {
            o.rho = rho[s2];
            o.e = Es[s2];
            o.p = o.rho * RU * 1e3 / o.mw * o.T;
            o.h = o.e + o.p / o.rho;
        }
        for (int j = 0; j < ns; ++j) o.n[j] = n[2 * j + s2];
    }
    inf.iters_fuel = it[0];
    inf.iters_oxidizer = it[1];
    double sm = 0.0;
    for (int j = 0; j < ns; ++j) sm += inf.oxidizer.n[j] + inf.fuel.n[j];
    inf.n_init = sm / ns;
    *out = h;
    return 0;
}

int scfd_cea_destroy(scfd_cea* h) {
    if (!h) return SCFD_E_ARG;
    if (h->d_tab) cudaFree(h->d_tab);
    if (h->d_fail) cudaFree(h->d_fail);
    delete h;
    return 0;
}

int scfd_cea_info_get(const scfd_cea* h, scfd_cea_info* info) {
    if (!h || !info) return SCFD_E_ARG;
    *info = h->info;
    return 0;
}

int scfd_cea_solve(scfd_cea* h, int64_t ncell, const double* rho, const double* Y, const double* e, double* T,
                   double* n, double* mwave, double* kappa, double* mu, double* Yv, double* vhi, double* DHi,
                   int32_t* iters, void* stream) {
    if (!h || ncell < 0) return SCFD_E_ARG;
    if (ncell > 0 && (!rho || !Y || !e || !T || !n)) return SCFD_E_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    h->last = st;
    const CellOut o{mwave, kappa, mu, Yv, vhi, DHi, iters};
    return cea_launch(h, ncell, rho, Y, e, T, n, o, st);
}

int scfd_cea_solve_hp(scfd_cea* h, int64_t ncell, const double* p, const double* Y, const double* hh, double* T,
                      double* n, double* mwave, double* kappa, double* mu, double* Yv, double* vhi, int32_t* iters,
                      void* stream) {
    if (!h || ncell < 0) return SCFD_E_ARG;
    if (ncell > 0 && (!p || !Y || !hh || !T || !n)) return SCFD_E_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    h->last = st;
    const HpTpOut o{nullptr, mwave, kappa, mu, Yv, vhi, iters};
    return cea_hptp_launch<true>(h, ncell, p, Y, hh, T, n, o, st);
}

int scfd_cea_solve_tp(scfd_cea* h, int64_t ncell, const double* p, const double* Y, const double* T, double* n,
                      double* hh, double* mwave, double* kappa, double* mu, double* Yv, double* vhi, int32_t* iters,
                      void* stream) {
    if (!h || ncell < 0) return SCFD_E_ARG;
    if (ncell > 0 && (!p || !Y || !T || !n)) return SCFD_E_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    h->last = st;
    const HpTpOut o{hh, mwave, kappa, mu, Yv, vhi, iters};
    return cea_hptp_launch<false>(h, ncell, p, Y, nullptr, const_cast<double*>(T), n, o, st);
}

int scfd_cea_status(scfd_cea* h, int64_t* counts) {
    if (!h || !counts) return SCFD_E_ARG;
    if (cudaStreamSynchronize(h->last) != cudaSuccess) return SCFD_E_CUDA;
    unsigned long long hf[2];
    if (cudaMemcpy(hf, h->d_fail, sizeof(hf), cudaMemcpyDeviceToHost) != cudaSuccess) return SCFD_E_CUDA;
    if (cudaMemset(h->d_fail, 0, sizeof(hf)) != cudaSuccess) return SCFD_E_CUDA;
    counts[0] = (int64_t)hf[0];
    counts[1] = (int64_t)hf[1];
    return hf[1] ? SCFD_E_SINGULAR : 0;
}

}  // extern "C"
