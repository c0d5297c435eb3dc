// k_thermo.cu -- set_w + set_thermo_prop per interior cell.
//
// store/core/scheme.f90:1-29 (set_w), store/therm_lib/ideal/thermal_model.raw.f90:7-33
// (ideal gas) and store/therm_lib/chemkin/flow/{reactive,cold}/thermal_model.f90:13-42
// with calc_T (store/therm_lib/chemkin/core/sub_chem.f90:1507-1645).
//
// One thread per cell; HBM traffic per cell: read q (D) + w(4), w(R) guesses,
// write w (W), vhi (nY), DHi (nY).  The chemkin branch is FP64 compute-bound:
// NASA-7 polynomials in the T Newton loop and the Wilke mixture sum.
#include "div_pos.cuh"
#include "scfd_internal.h"

namespace scfd {

__device__ __forceinline__ double sqd(double a) { return a * a; }

__device__ __forceinline__ void set_status(DevScalars* sc, int code) { atomicMax(&sc->status, code); }

// calc_T restated for the device.  The Wilke sum uses sqrt(muN_i)/sqrt(muN_j)
// in place of sqrt(muN_i/muN_j) and per-pair constants prepared on the host;
// the result equals the reference's up to rounding.
__device__ int dev_calc_T(const DevChem& ch, const double* vrho, double rho, double E, double& T, double& kappa,
                          double& MWave, double* DHi, double* vhi, double& mu) {
    const int ns = ch.ns;
    double n[kMaxSpecies];
    const double tmp0 = rho * 1e-11;
    for (int j = 0; j < ns; ++j) n[j] = vrho[j] > tmp0 ? vrho[j] * ch.inv_mw[j] * 1e-3 : 0.0;
    const double Ru = 8.3144621e7;
    const double Eobj = E * 1e1 * rho / Ru;
    int k = 1;
    double cvnow = 0.0;
    double chrt[6];
    for (;;) {
        const double Ti1 = 1.0 / T, T2 = T * T, T3 = T2 * T, T4 = T3 * T;
        chrt[0] = 1.0; chrt[1] = T / 2.0; chrt[2] = T2 / 3.0; chrt[3] = T3 / 4.0; chrt[4] = T4 / 5.0; chrt[5] = Ti1;
        const double ccpr[5] = {1.0, T, T2, T3, T4};
        double Enow = 0.0;
        cvnow = 0.0;
        for (int j = 0; j < ns; ++j) {
            if (n[j] > 0.0) {
                const double* cf = ch.coeff + (j * 2 + (T <= ch.tcommon[j] ? 0 : 1)) * 7;
                double de = -1.0, dcv = -1.0;
#pragma unroll
                for (int i = 0; i < 5; ++i) {
                    de = de + cf[i] * chrt[i];
                    dcv = dcv + cf[i] * ccpr[i];
                }
                de = de + cf[5] * chrt[5];
                Enow = Enow + de * n[j];
                cvnow = cvnow + dcv * n[j];
            }
        }
        const double dT = (Eobj - Enow * T) / cvnow;
        if (fabs(dT) < 1e-8 || (fabs(dT) < 1e-4 && fabs(T - 1e3) < 1e-4) || k > 1000) break;
        T = fmax(100.0, T + dT);
        k = k + 1;
    }
    if (k > 1000) return SCFD_E_TNEWTON;
    double sn = 0.0;
    for (int j = 0; j < ns; ++j) sn = sn + n[j];
    kappa = 1.0 + sn / cvnow;
    MWave = rho / sn * 1e-3;
    const double tmp = Ru * 1e-4 * T;
    for (int j = 0; j < ns; ++j) {
        const double* cf = ch.coeff + (j * 2 + (T <= ch.tcommon[j] ? 0 : 1)) * 7;
        double dh = 0.0;
#pragma unroll
        for (int i = 0; i < 6; ++i) dh = dh + cf[i] * chrt[i];
        DHi[j] = tmp * ch.inv_mw[j] * (kappa - (kappa - 1.0) * dh);
        vhi[j] = tmp * ch.inv_mw[j] * dh;
    }
    // Wilke (sub_chem.f90:1602-1633)
    const double logT = log(T), invT = 1.0 / T;
    const double cmu[4] = {logT, invT, invT * invT, 1.0};
    double muN[kMaxSpecies], smu[kMaxSpecies], rsmu[kMaxSpecies];
    for (int i = 0; i < ch.nt; ++i) {
        int sec = -1;
        const double* tr = ch.trange + i * 10;
        if (tr[0] > T) sec = 0;
        const int nsec = ch.nsec[i];
        for (int l = 0; l < nsec; ++l)
            if (tr[2 * l + 1] > T) {
                sec = l;
                break;
            }
        if (sec == -1) sec = nsec - 1;
        if (n[ch.tr2th[i]] > 0.0) {
            const double* c4 = ch.trans + (i * 5 + sec) * 4;
            double t = 0.0;
#pragma unroll
            for (int j = 0; j < 4; ++j) t = t + cmu[j] * c4[j];
            muN[i] = exp(t);
            smu[i] = sqrt(muN[i]);
            rsmu[i] = 1.0 / smu[i];
        } else {
            muN[i] = 0.0;
            smu[i] = 0.0;
            rsmu[i] = 0.0;
        }
    }
    mu = 0.0;
    for (int i = 0; i < ch.nt; ++i) {
        if (muN[i] > 0.0) {
            const int it = ch.tr2th[i];
            double denom = 0.0;
            for (int j = 0; j < ch.nt; ++j) {
                if (muN[j] > 0.0) {
                    const int jt = ch.tr2th[j];
                    const double a = 1.0 + smu[i] * rsmu[j] * ch.wc1[i * ch.nt + j];
                    const double phi = 0.25 * (a * a) * ch.wc2[i * ch.nt + j];
                    denom = denom + n[jt] * phi;
                }
            }
            mu = mu + n[it] * muN[i] / denom;
        }
    }
    mu = mu * 1e-7;
    return 0;
}

template <int NS>
__device__ __forceinline__ double pick(const double* a, int k) {
    double r = 0.0;
#pragma unroll
    for (int m = 0; m < NS; ++m)
        if (m == k) r = a[m];
    return r;
}

// calc_T for a mechanism of exactly NS species (and at most NS viscosity
// fits): the same arithmetic as dev_calc_T with the species loops unrolled, so
// that the species vectors stay in registers (n(tr2th(i)) gathered by selects
// instead of an indexed load).  Its quotients, and those of k_thermo_fixed, go
// through div_pos (branch-free, within one unit in the last place; 0.138 ->
// 0.124 ms per launch at 786 k cells): their denominators are T >= 100, the
// mixture's cv and mole sum, its molecular weight, the density, sqrt(mu_i)
// and the Wilke sums, all positive, and the constants 3 and 5.
template <int NS>
__device__ __forceinline__ int dev_calc_T_fixed(const DevChem& ch, const double* vrho, double rho, double E, double& T, double& kappa,
                          double& MWave, double* DHi, double* vhi, double& mu) {
    constexpr int SZ = NS;
    constexpr int UNR = NS;
    const int ns = NS;
    const int nt = ch.nt;
    double n[SZ];
    const double tmp0 = rho * 1e-11;
#pragma unroll UNR
    for (int j = 0; j < SZ; ++j)
        if (j < ns) n[j] = vrho[j] > tmp0 ? vrho[j] * ch.inv_mw[j] * 1e-3 : 0.0;
    const double Ru = 8.3144621e7;
    const double Eobj = E * 1e1 * rho * (1.0 / Ru);
    int k = 1;
    double cvnow = 0.0;
    double chrt[6];
    for (;;) {
        const double Ti1 = div_pos(1.0, T), T2 = T * T, T3 = T2 * T, T4 = T3 * T;
        chrt[0] = 1.0; chrt[1] = T * 0.5; chrt[2] = div_pos(T2, 3.0); chrt[3] = T3 * 0.25; chrt[4] = div_pos(T4, 5.0); chrt[5] = Ti1;
        const double ccpr[5] = {1.0, T, T2, T3, T4};
        double Enow = 0.0;
        cvnow = 0.0;
#pragma unroll UNR
        for (int j = 0; j < SZ; ++j) {
            if (j < ns && n[j] > 0.0) {
                const double* cf = ch.coeff + (j * 2 + (T <= ch.tcommon[j] ? 0 : 1)) * 7;
                double de = -1.0, dcv = -1.0;
#pragma unroll
                for (int i = 0; i < 5; ++i) {
                    de = de + cf[i] * chrt[i];
                    dcv = dcv + cf[i] * ccpr[i];
                }
                de = de + cf[5] * chrt[5];
                Enow = Enow + de * n[j];
                cvnow = cvnow + dcv * n[j];
            }
        }
        const double dT = div_pos(Eobj - Enow * T, cvnow);
        if (fabs(dT) < 1e-8 || (fabs(dT) < 1e-4 && fabs(T - 1e3) < 1e-4) || k > 1000) break;
        T = fmax(100.0, T + dT);
        k = k + 1;
    }
    if (k > 1000) return SCFD_E_TNEWTON;
    double sn = 0.0;
#pragma unroll UNR
    for (int j = 0; j < SZ; ++j)
        if (j < ns) sn = sn + n[j];
    kappa = 1.0 + div_pos(sn, cvnow);
    MWave = div_pos(rho, sn) * 1e-3;
    const double tmp = Ru * 1e-4 * T;
#pragma unroll UNR
    for (int j = 0; j < SZ; ++j) {
        if (j >= ns) continue;
        const double* cf = ch.coeff + (j * 2 + (T <= ch.tcommon[j] ? 0 : 1)) * 7;
        double dh = 0.0;
#pragma unroll
        for (int i = 0; i < 6; ++i) dh = dh + cf[i] * chrt[i];
        DHi[j] = tmp * ch.inv_mw[j] * (kappa - (kappa - 1.0) * dh);
        vhi[j] = tmp * ch.inv_mw[j] * dh;
    }
    // Wilke (sub_chem.f90:1602-1633)
    const double logT = log(T), invT = div_pos(1.0, T);
    const double cmu[4] = {logT, invT, invT * invT, 1.0};
    double muN[SZ], smu[SZ], rsmu[SZ], nf[SZ];  // nf[i] = n(tr2th(i))
#pragma unroll UNR
    for (int i = 0; i < SZ; ++i) {
        muN[i] = smu[i] = rsmu[i] = nf[i] = 0.0;
        if (i >= nt) continue;
        nf[i] = pick<SZ>(n, ch.tr2th[i]);
        int sec = -1;
        const double* tr = ch.trange + i * 10;
        if (tr[0] > T) sec = 0;
        const int nsec = ch.nsec[i];
        for (int l = 0; l < nsec; ++l)
            if (tr[2 * l + 1] > T) {
                sec = l;
                break;
            }
        if (sec == -1) sec = nsec - 1;
        if (nf[i] > 0.0) {
            const double* c4 = ch.trans + (i * 5 + sec) * 4;
            double t = 0.0;
#pragma unroll
            for (int j = 0; j < 4; ++j) t = t + cmu[j] * c4[j];
            muN[i] = exp(t);
            smu[i] = sqrt(muN[i]);
            rsmu[i] = div_pos(1.0, smu[i]);
        } else {
            muN[i] = 0.0;
            smu[i] = 0.0;
            rsmu[i] = 0.0;
        }
    }
    mu = 0.0;
#pragma unroll UNR
    for (int i = 0; i < SZ; ++i) {
        if (i < nt && muN[i] > 0.0) {
            double denom = 0.0;
#pragma unroll UNR
            for (int j = 0; j < SZ; ++j) {
                if (j < nt && muN[j] > 0.0) {
                    const double a = 1.0 + smu[i] * rsmu[j] * ch.wc1[i * nt + j];
                    const double phi = 0.25 * (a * a) * ch.wc2[i * nt + j];
                    denom = denom + nf[j] * phi;
                }
            }
            mu = mu + div_pos(nf[i] * muN[i], denom);
        }
    }
    mu = mu * 1e-7;
    return 0;
}

// set_w + set_thermo_prop for a chemkin mechanism of exactly NS species
// (k_thermo's chemkin branch with dev_calc_T_fixed), built for two resident
// blocks of 256 threads: 128 registers.  With 178 unconstrained registers it
// measured 1.4x slower than this, k_thermo's local-memory vectors 2x slower
// after the same rewrite.
template <int NS>
__global__ void __launch_bounds__(256, 2) k_thermo_fixed(View v) {
    const int p = v.P.act[blockIdx.y];
    const int ni = v.P.ni[p], nj = v.P.nj[p];
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= ni * nj) return;
    const int i = idx % ni + 1, j = idx / ni + 1;
    const long long c = cidx(v.P, p, i, j);
    const long long N = v.ncell;
    constexpr int nY = NS, D = NS + 3;
    constexpr int ig = D + 1, iht = D + 2, iR = D + 3, imu = D + 4;
    const double* q = v.q;
    double* w = v.w;
    double vrho[NS], DH[NS], vh[NS];
    double tmp = 0.0;
#pragma unroll
    for (int k = 0; k < nY; ++k) {
        vrho[k] = q[k * N + c];
        tmp = tmp + vrho[k];
    }
    const double rho = tmp;
    w[c] = rho;
    tmp = div_pos(1.0, tmp);
    const double u = q[nY * N + c] * tmp;
    const double vv = q[(nY + 1) * N + c] * tmp;
    w[N + c] = u;
    w[2 * N + c] = vv;
#pragma unroll
    for (int k = 0; k < nY; ++k) w[(k + 4) * N + c] = vrho[k] * tmp;
    const double qE = q[(nY + 2) * N + c];
    const double ei = div_pos(qE, rho) - 0.5 * (u * u + vv * vv);
    double T = div_pos(w[3 * N + c], rho * w[iR * N + c]);
    double kappa, MW, mu;
    const int st = dev_calc_T_fixed<NS>(v.chem, vrho, rho, ei, T, kappa, MW, DH, vh, mu);
    if (st) set_status(v.sc, st);
#pragma unroll
    for (int k = 0; k < nY; ++k) {
        v.DHi[k * N + c] = DH[k];
        v.vhi[k * N + c] = vh[k];
    }
    w[imu * N + c] = mu;
    const double Rm = div_pos(8.3144621e3, MW);
    w[iR * N + c] = Rm;
    const double pr = rho * Rm * T;
    w[3 * N + c] = pr;
    w[ig * N + c] = kappa;
    w[iht * N + c] = div_pos(qE + pr, rho);
}

__global__ void __launch_bounds__(256) k_thermo(View v) {
    const int p = v.P.act[blockIdx.y];
    const int ni = v.P.ni[p], nj = v.P.nj[p];
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= ni * nj) return;
    const int i = idx % ni + 1, j = idx / ni + 1;
    const long long c = cidx(v.P, p, i, j);
    const long long N = v.ncell;
    const int nY = v.nY, D = v.D;
    const int ig = D + 1, iht = D + 2, iR = D + 3, imu = D + 4;  // 0-based indxg.. indxMu
    const double* q = v.q;
    double* w = v.w;
    // set_w
    double tmp = 0.0;
    for (int k = 0; k < nY; ++k) tmp = tmp + q[k * N + c];
    const double rho = tmp;
    w[c] = rho;
    tmp = 1.0 / tmp;
    const double u = q[nY * N + c] * tmp;
    const double vv = q[(nY + 1) * N + c] * tmp;
    w[N + c] = u;
    w[2 * N + c] = vv;
    for (int k = 0; k < nY; ++k) w[(k + 4) * N + c] = q[k * N + c] * tmp;
    const double qE = q[(nY + 2) * N + c];
    const double ei = qE / rho - 0.5 * (u * u + vv * vv);
    if (v.thermo == SCFD_THERMO_IDEAL) {
        const double kg = v.kappa, Rg = v.rgas;
        const double T = ei * (kg - 1.0) / Rg;
        const double pr = rho * Rg * T;
        w[3 * N + c] = pr;
        w[ig * N + c] = kg;
        w[iht * N + c] = (qE + pr) / rho;
        if (v.mu_model == SCFD_MU_SUTHERLAND)
            w[imu * N + c] = v.suth_mu0 * pow(T / v.suth_t0, 1.5) * (v.suth_t0 + v.suth_s) / (T + v.suth_s);
        else
            w[imu * N + c] = rho * v.nu_gas;
        w[iR * N + c] = Rg;
        for (int k = 0; k < nY; ++k) v.DHi[k * N + c] = 0.0;
        v.vhi[c] = kg / (kg - 1.0) * Rg * T;
        return;
    }
    double vrho[kMaxSpecies], DH[kMaxSpecies], vh[kMaxSpecies];
    for (int k = 0; k < nY; ++k) vrho[k] = q[k * N + c];
    double T = w[3 * N + c] / (rho * w[iR * N + c]);
    double kappa, MW, mu;
    const int st = dev_calc_T(v.chem, vrho, rho, ei, T, kappa, MW, DH, vh, mu);
    if (st) set_status(v.sc, st);
    for (int k = 0; k < nY; ++k) {
        v.DHi[k * N + c] = DH[k];
        v.vhi[k * N + c] = vh[k];
    }
    w[imu * N + c] = mu;
    const double Rm = 8.3144621e3 / MW;
    w[iR * N + c] = Rm;
    const double pr = rho * Rm * T;
    w[3 * N + c] = pr;
    w[ig * N + c] = kappa;
    w[iht * N + c] = (qE + pr) / rho;
}

int launch_thermo(const View& v, cudaStream_t s, int cells_per_plane_max) {
    if (v.P.nact == 0) return 0;
    const int bs = v.thermo_block == 64 || v.thermo_block == 256 ? v.thermo_block : 128;
    dim3 grid((cells_per_plane_max + bs - 1) / bs, v.P.nact);
    // the 9-species mechanisms (the reacting benchmark's) take the unrolled kernel
    if (v.thermo != SCFD_THERMO_IDEAL && v.chem.ns == 9 && v.nY == 9 && v.chem.nt <= 9)
        k_thermo_fixed<9><<<grid, bs, 0, s>>>(v);
    else
        k_thermo<<<grid, bs, 0, s>>>(v);
    return 1;
}

}  // namespace scfd
