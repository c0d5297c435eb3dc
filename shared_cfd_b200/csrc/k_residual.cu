// k_residual.cu -- fused residual kernel: set_HV (MUSCL) + set_TG (SLAU) +
// set_TGv (viscous, 2d / q2d) + set_Sq + Svq + right-hand-side assembly, and per
// scheme the explicit Euler update, or the LU-SGS / NR right-hand side and the
// diagonal coefficients of set_ABpm.
//
// Restated from store/high_order/muscl/muscl.f90:7-73, store/core/scheme.f90:31-259,
// store/viscosity/viscous/no-nV/{2d,q2d}/sch_viscous.f90:75-321, store/dim/q2d/Sq.f90,
// store/time_scheme/euler/time_euler_viscous.raw.f90, LU-SGS/q2d/time_lusgs_viscous.f90:12-23,
// NR/q2d/time_NR_viscous.f90:17-26, NR/q2d/sch_NR.raw.f90:27-45,142-144,151-180.
//
// One CTA owns a TX x TY tile of cells.  The face fluxes ds*(TG - TGv) of the
// tile's (TX+1)*TY i-faces and TX*(TY+1) j-faces are computed once into shared
// memory and summed per cell, so no face array goes to HBM: per cell the kernel
// reads w (W), vhi (nY) and the metrics and writes D values.
//
// RT is the arithmetic type of reconstruction and fluxes (double for the plain
// path, float for the mixed path); the right-hand-side sum, the dual-time
// defect Vol*dqdt and the update stay in double.
#include "scfd_internal.h"

namespace scfd {

constexpr int TX = 32, TY = 8, NT = TX * TY;

template <typename RT>
struct Eps;
template <>
struct Eps<double> {
    static __device__ __forceinline__ double v() { return 1e-300; }
};
template <>
struct Eps<float> {
    static __device__ __forceinline__ float v() { return 1e-37f; }
};

template <typename RT>
__device__ __forceinline__ RT ldw(const View& v, int k, long long c) {
    if constexpr (sizeof(RT) == 4)
        return __ldg(v.w32 + k * v.ncell + c);
    else
        return __ldg(v.w + k * v.ncell + c);
}
template <typename RT>
__device__ __forceinline__ RT ldvhi(const View& v, int k, long long c) {
    if constexpr (sizeof(RT) == 4)
        return __ldg(v.vhi32 + k * v.ncell + c);
    else
        return __ldg(v.vhi + k * v.ncell + c);
}
__device__ __forceinline__ double ldg(const double* a, long long c) { return __ldg(a + c); }

// MUSCL face states of one component from the 4-cell stencil (muscl.f90:28-44,
// 52-68).  wl = w0 + phi/2 * delta_u(cell 0); wr = w1 - phi/2 * delta_l(cell 1).
template <typename RT>
__device__ __forceinline__ void muscl(RT wm1, RT w0, RT w1, RT w2, RT phi, RT km, RT& wl, RT& wr) {
    const RT half = RT(0.5), one = RT(1);
    RT Du = w1 - w0, Dl = w0 - wm1;
    RT s = (RT(2) * Du * Dl) / (Du * Du + Dl * Dl + Eps<RT>::v());
    RT du = half * s * ((one + km * s) * Du + (one - km * s) * Dl);
    wl = w0 + phi * half * du;
    Du = w2 - w1;
    Dl = w1 - w0;
    s = (RT(2) * Du * Dl) / (Du * Du + Dl * Dl + Eps<RT>::v());
    RT dl = half * s * ((one + km * s) * Dl + (one - km * s) * Du);
    wr = w1 - phi * half * dl;
}

// SLAU flux (scheme.f90:71-153).  wl/wr hold rho,u,v,p,Y(1:nY),gamma,ht as
// [0..3], [4..3+nY], [4+nY], [5+nY].
template <typename RT>
__device__ __forceinline__ void slau(int nY, const RT* wl, const RT* wr, RT n1, RT n2, RT* tg) {
    const RT half = RT(0.5), one = RT(1);
    const RT rhol = wl[0], ul = wl[1], vl = wl[2], pl = wl[3], gl = wl[4 + nY];
    const RT rhor = wr[0], ur = wr[1], vr = wr[2], pr = wr[3], gr = wr[4 + nY];
    const RT al = sqrt(gl * pl / rhol), ar = sqrt(gr * pr / rhor);
    const RT unl = n1 * ul + n2 * vl, unr = n1 * ur + n2 * vr;
    const RT dp = pr - pl;
    const RT a_bar = half * (ar + al);
    const RT p_bar = half * (pr + pl);
    const RT ml = unl / a_bar, mr = unr / a_bar;
    const RT m_tilde = fmin(one, one / a_bar * sqrt(half * (ul * ul + vl * vl + ur * ur + vr * vr)));
    const RT chi = (one - m_tilde) * (one - m_tilde);
    const RT gp = -fmax(fmin(ml, RT(0)), -one);
    const RT gm = fmin(fmax(mr, RT(0)), one);
    const RT g = gp * gm;
    const RT ub = (fabs(unr) * rhor + fabs(unl) * rhol) / (rhor + rhol);
    const RT ubp = (one - g) * ub + g * fabs(unl);
    const RT ubm = (one - g) * ub + g * fabs(unr);
    const RT dm = half * (rhol * (unl + ubp) + rhor * (unr - ubm) - chi / a_bar * dp);
    RT betar, betal;
    if (fabs(mr) < one)
        betar = RT(0.25) * (RT(2) + mr) * ((mr - one) * (mr - one));
    else
        betar = half * (one - copysign(one, mr));
    if (fabs(ml) < one)
        betal = RT(0.25) * (RT(2) - ml) * ((ml + one) * (ml + one));
    else
        betal = half * (one + copysign(one, ml));
    const RT pt = p_bar + half * (betal - betar) * (pl - pr) + (one - chi) * (betar + betal - one) * p_bar;
    const RT dp_ = half * (dm + fabs(dm)), dn_ = half * (dm - fabs(dm));
    for (int k = 0; k < nY; ++k) tg[k] = dp_ * wl[4 + k] + dn_ * wr[4 + k];
    tg[nY] = dp_ * ul + dn_ * ur + pt * n1;
    tg[nY + 1] = dp_ * vl + dn_ * vr + pt * n2;
    tg[nY + 2] = dp_ * wl[5 + nY] + dn_ * wr[5 + nY];
}

// Viscous face flux (sch_viscous.f90:125-197 for i-faces, 214-286 j-faces).
// Cells a (i,j) and b (the neighbour across the face).  Gradient stencils as in
// the reference; T = p/rho/R is formed from w on the fly (Tdeg, lines 104-110).
template <typename RT, bool IFACE>
__device__ void visc_face(const View& v, int p, int i, int j, RT n1, RT n2, bool q2d, RT* out) {
    const int nY = v.nY;
    const int iR = v.D + 3, ig = v.D + 1, imu = v.D + 4;
    const int i2 = IFACE ? i + 1 : i, j2 = IFACE ? j : j + 1;
    const long long ca = cidx(v.P, p, i, j), cb = cidx(v.P, p, i2, j2);
    auto T = [&](long long c) -> RT { return ldw<RT>(v, 3, c) / ldw<RT>(v, 0, c) / ldw<RT>(v, iR, c); };
    const RT half = RT(0.5), q4 = RT(0.25);
    const RT rho = (ldw<RT>(v, 0, ca) + ldw<RT>(v, 0, cb)) * half;
    const RT u = (ldw<RT>(v, 1, ca) + ldw<RT>(v, 1, cb)) * half;
    const RT vv = (ldw<RT>(v, 2, ca) + ldw<RT>(v, 2, cb)) * half;
    const RT gamm = (ldw<RT>(v, ig, ca) + ldw<RT>(v, ig, cb)) * half;
    const RT Rgas = (ldw<RT>(v, iR, ca) + ldw<RT>(v, iR, cb)) * half;
    const RT mu = (ldw<RT>(v, imu, ca) + ldw<RT>(v, imu, cb)) * half;
    const RT Dd = mu / rho / RT(v.schmidt);
    const RT k_heat = mu * gamm / (gamm - RT(1)) * Rgas / RT(v.prandtl);
    // stencil cells for the cross derivative
    long long c_p1, c_p2, c_m1, c_m2;  // (+): cells summed, (-): cells subtracted
    if (IFACE) {
        c_p1 = cidx(v.P, p, i + 1, j + 1); c_p2 = cidx(v.P, p, i, j + 1);
        c_m1 = cidx(v.P, p, i + 1, j - 1); c_m2 = cidx(v.P, p, i, j - 1);
    } else {
        c_p1 = cidx(v.P, p, i + 1, j + 1); c_p2 = cidx(v.P, p, i + 1, j);
        c_m1 = cidx(v.P, p, i - 1, j + 1); c_m2 = cidx(v.P, p, i - 1, j);
    }
    const RT dN_u = ldw<RT>(v, 1, cb) - ldw<RT>(v, 1, ca);
    const RT dN_v = ldw<RT>(v, 2, cb) - ldw<RT>(v, 2, ca);
    const RT dN_T = T(cb) - T(ca);
    const RT dC_u = (ldw<RT>(v, 1, c_p1) + ldw<RT>(v, 1, c_p2) - ldw<RT>(v, 1, c_m1) - ldw<RT>(v, 1, c_m2)) * q4;
    const RT dC_v = (ldw<RT>(v, 2, c_p1) + ldw<RT>(v, 2, c_p2) - ldw<RT>(v, 2, c_m1) - ldw<RT>(v, 2, c_m2)) * q4;
    const RT dC_T = (T(c_p1) + T(c_p2) - T(c_m1) - T(c_m2)) * q4;
    // geojac of the face
    const double* gj = IFACE ? v.gji : v.gjj;
    const long long N = v.ncell;
    const RT g11 = RT(ldg(gj, ca)), g12 = RT(ldg(gj, N + ca)), g21 = RT(ldg(gj, 2 * N + ca)), g22 = RT(ldg(gj, 3 * N + ca));
    // xi derivative is the normal one on i-faces, the cross one on j-faces
    const RT dudxi = IFACE ? dN_u : dC_u, dudeta = IFACE ? dC_u : dN_u;
    const RT dvdxi = IFACE ? dN_v : dC_v, dvdeta = IFACE ? dC_v : dN_v;
    const RT dTdxi = IFACE ? dN_T : dC_T, dTdeta = IFACE ? dC_T : dN_T;
    const RT dudx = dudxi * g11 + dudeta * g21;
    const RT dvdx = dvdxi * g11 + dvdeta * g21;
    const RT dTdx = dTdxi * g11 + dTdeta * g21;
    const RT dudr = dudxi * g12 + dudeta * g22;
    const RT dvdr = dvdxi * g12 + dvdeta * g22;
    const RT dTdr = dTdxi * g12 + dTdeta * g22;
    RT hidwdx = RT(0), hidwdr = RT(0);
    const RT rhoD = rho * Dd;
    for (int k = 0; k < nY; ++k) {
        const int kw = 4 + k;
        const RT dN = ldw<RT>(v, kw, cb) - ldw<RT>(v, kw, ca);
        const RT dC = (ldw<RT>(v, kw, c_p1) + ldw<RT>(v, kw, c_p2) - ldw<RT>(v, kw, c_m1) - ldw<RT>(v, kw, c_m2)) * q4;
        const RT dxi = IFACE ? dN : dC, deta = IFACE ? dC : dN;
        const RT dwdx = dxi * g11 + deta * g21;
        const RT dwdr = dxi * g12 + deta * g22;
        const RT lhi = (ldvhi<RT>(v, k, ca) + ldvhi<RT>(v, k, cb)) * half;
        hidwdx = hidwdx + dwdx * lhi;
        hidwdr = hidwdr + dwdr * lhi;
        out[k] = rhoD * dwdx * n1 + rhoD * dwdr * n2;
    }
    RT divu = dudx + dvdr;
    if (q2d) divu = dudx + dvdr + vv / RT(ldg(v.r, ca));
    const RT t_xx = -RT(2) / RT(3) * mu * divu + RT(2) * mu * dudx;
    const RT t_rr = -RT(2) / RT(3) * mu * divu + RT(2) * mu * dvdr;
    const RT t_xr = mu * (dvdx + dudr);
    const RT qx = -k_heat * dTdx - rho * Dd * hidwdx;
    const RT qr = -k_heat * dTdr - rho * Dd * hidwdr;
    out[nY] = t_xx * n1 + t_xr * n2;
    out[nY + 1] = t_xr * n1 + t_rr * n2;
    out[nY + 2] = (u * t_xx + vv * t_xr - qx) * n1 + (u * t_xr + vv * t_rr - qr) * n2;
}

template <typename RT, bool IFACE>
__device__ void face_flux(const View& v, int p, int i, int j, RT* fout) {
    const int nY = v.nY, D = v.D;
    const int iht = D + 2, ig = D + 1;
    const RT phi = RT(v.recon == SCFD_RECON_MUSCL ? v.phi_mus : 0.0), km = RT(v.k_mus);
    // components needed by SLAU: rho,u,v,p,Y(1:nY),gamma,ht -> 6+nY of W
    RT wl[kMaxSpecies + 6], wr[kMaxSpecies + 6];
    long long cm1, c0, c1, c2;
    if (IFACE) {
        cm1 = cidx(v.P, p, i - 1, j); c0 = cidx(v.P, p, i, j); c1 = cidx(v.P, p, i + 1, j); c2 = cidx(v.P, p, i + 2, j);
    } else {
        cm1 = cidx(v.P, p, i, j - 1); c0 = cidx(v.P, p, i, j); c1 = cidx(v.P, p, i, j + 1); c2 = cidx(v.P, p, i, j + 2);
    }
    const int nc = 6 + nY;
    for (int m = 0; m < nc; ++m) {
        const int k = m < 4 + nY ? m : (m == 4 + nY ? ig : iht);
        muscl<RT>(ldw<RT>(v, k, cm1), ldw<RT>(v, k, c0), ldw<RT>(v, k, c1), ldw<RT>(v, k, c2), phi, km, wl[m], wr[m]);
    }
    const long long N = v.ncell;
    const double* vn = IFACE ? v.vni : v.vnj;
    const RT n1 = RT(ldg(vn, c0)), n2 = RT(ldg(vn, N + c0));
    RT tg[kMaxSpecies + 3];
    slau<RT>(nY, wl, wr, n1, n2, tg);
    const RT ds = RT(ldg(IFACE ? v.dsi : v.dsj, c0));
    if (v.viscous) {
        RT tv[kMaxSpecies + 3];
        visc_face<RT, IFACE>(v, p, i, j, n1, n2, v.dim == SCFD_DIM_Q2D, tv);
        for (int k = 0; k < D; ++k) fout[k] = ds * (tg[k] - tv[k]);
    } else {
        for (int k = 0; k < D; ++k) fout[k] = ds * tg[k];
    }
}

template <typename RT, int MODE>
__global__ void __launch_bounds__(NT) k_residual(View v) {
    extern __shared__ unsigned char smraw[];
    RT* FI = reinterpret_cast<RT*>(smraw);
    const int D = v.D, nY = v.nY;
    RT* FJ = FI + TY * (TX + 1) * D;
    const int p = v.P.act[blockIdx.z];
    const int ni = v.P.ni[p], nj = v.P.nj[p];
    const int i0 = blockIdx.x * TX + 1, j0 = blockIdx.y * TY + 1;
    if (i0 > ni || j0 > nj) return;
    const int tid = threadIdx.x;
    for (int f = tid; f < TY * (TX + 1); f += NT) {
        const int fy = f / (TX + 1), fx = f - fy * (TX + 1);
        const int i = i0 - 1 + fx, j = j0 + fy;
        if (i <= ni && j <= nj) face_flux<RT, true>(v, p, i, j, FI + f * D);
    }
    for (int f = tid; f < (TY + 1) * TX; f += NT) {
        const int fy = f / TX, fx = f - fy * TX;
        const int i = i0 + fx, j = j0 - 1 + fy;
        if (i <= ni && j <= nj) face_flux<RT, false>(v, p, i, j, FJ + f * D);
    }
    __syncthreads();
    const int tx = tid % TX, ty = tid / TX;
    const int i = i0 + tx, j = j0 + ty;
    if (i > ni || j > nj) return;
    const long long N = v.ncell;
    const long long c = cidx(v.P, p, i, j);
    const bool q2d = v.dim == SCFD_DIM_Q2D;
    const double area = v.Area[c];
    // Svq (q2d viscous source, sch_viscous.f90:297-316) and Sq (Sq.f90:13)
    double svq_my = 0.0, sq_my = 0.0;
    if (q2d) {
        sq_my = v.w[3 * N + c];
        if (v.viscous) {
            const double vv = v.w[2 * N + c], mu = v.w[(D + 4) * N + c];
            const long long cip = cidx(v.P, p, i + 1, j), cim = cidx(v.P, p, i - 1, j);
            const long long cjp = cidx(v.P, p, i, j + 1), cjm = cidx(v.P, p, i, j - 1);
            const double dudxi = (v.w[N + cip] - v.w[N + cim]) * 0.5;
            const double dvdxi = (v.w[2 * N + cip] - v.w[2 * N + cim]) * 0.5;
            const double dudeta = (v.w[N + cjp] - v.w[N + cjm]) * 0.5;
            const double dvdeta = (v.w[2 * N + cjp] - v.w[2 * N + cjm]) * 0.5;
            const double dudx = dudxi * v.gjc[c] + dudeta * v.gjc[2 * N + c];
            const double dvdr = dvdxi * v.gjc[N + c] + dvdeta * v.gjc[3 * N + c];
            const double r = v.r[c];
            const double divu = dudx + dvdr + vv / r;
            const double t_tt = -2.0 / 3.0 * mu * divu + 2.0 * mu * vv / r;
            svq_my = -t_tt;
        }
    }
    const RT* fim = FI + (ty * (TX + 1) + tx) * D;
    const RT* fip = fim + D;
    const RT* fjm = FJ + (ty * TX + tx) * D;
    const RT* fjp = FJ + ((ty + 1) * TX + tx) * D;
    double dtl = v.dt_mode == SCFD_DT_LOCAL ? v.dt_mat[c] : v.sc->dt_grbl;
    if (MODE == RES_EULER) {
        const double f = dtl / v.Vol[c];
        for (int k = 0; k < D; ++k) {
            const double src = k == nY + 1 ? area * (sq_my + svq_my) : area * 0.0;
            const double rhs = (double)fim[k] - (double)fip[k] + (double)fjm[k] - (double)fjp[k] + src;
            v.q[k * N + c] = v.qp[k * N + c] + f * rhs;
        }
        return;
    }
    const double vol = v.Vol[c];
    const bool first = v.sc->first_dual != 0;
    if (MODE == RES_PRECON || MODE == RES_PRECON_LUSGS) {
        // set_ABpm of time_scheme/precon/2d (sch_precon.raw.f90:28-77, 194-197):
        // low-Mach reference velocity, preconditioned spectral radii, the local
        // time step (written to dt_mat: set_dqdt and alpha use it), phh of
        // pre1 = phh (Y, u, v, H); then Dq = R + pre1 (pre2 . R) [- Vol dqdt]
        // (time_precon_viscous.f90:18-27)
        const double rho = v.w[c], u = v.w[N + c], vv = v.w[2 * N + c], pr = v.w[3 * N + c];
        const double gamm = v.w[(D + 1) * N + c], H = v.w[(D + 2) * N + c];
        const double mu = v.w[(D + 4) * N + c], dsa = v.dsci[c], dsb = v.dscj[c];
        const double cs = sqrt(gamm * pr / rho);
        const double unA = v.vnci[c] * u + v.vnci[N + c] * vv;
        const double unB = v.vncj[c] * u + v.vncj[N + c] * vv;
        const double Vs = u * u + vv * vv;
        const double Vv = mu / rho / fmin(dsa, dsb);
        const double Ur = fmin(fmax(Vv, sqrt(Vs)), cs);
        const double phi = 1.0 / (Ur * Ur) - 1.0 / (cs * cs);
        const double alp = 0.5 * (1.0 - (Ur / cs) * (Ur / cs));
        double ud = unA * (1.0 - alp), cd = sqrt(alp * alp * (unA * unA) + Ur * Ur);
        const double nuA = fabs(ud) + cd;
        ud = unB * (1.0 - alp);
        cd = sqrt(alp * alp * (unB * unB) + Ur * Ur);
        const double nuB = fabs(ud) + cd;
        const long long cim = cidx(v.P, p, i - 1, j), cjm = cidx(v.P, p, i, j - 1);
        const double uds = nuA * (v.dsi[c] + v.dsi[cim]) + nuB * (v.dsj[c] + v.dsj[cjm]);
        const double dt = v.cfl * vol / fmax(uds, mu / rho);
        v.dt_mat[c] = dt;
        const double phh = -1.0 / (cs * cs + 1.0 / phi);
        const double tmp = MODE == RES_PRECON ? 3.0 * vol / (2.0 * dt) + dsa * nuA + dsb * nuB
                                              : vol / dt + dsa * nuA + dsb * nuB;
        v.alpha[c] = 1.0 / tmp;
        v.nuA[c] = nuA;
        v.nuB[c] = nuB;
        v.pre[c] = phh;
        const double g1 = gamm - 1.0;
        double R[kMaxSpecies + 3];
        double t = 0.0;
        for (int k = 0; k < D; ++k) {
            const double src = k == nY + 1 ? area * (sq_my + svq_my) : area * 0.0;
            R[k] = (double)fim[k] - (double)fip[k] + (double)fjm[k] - (double)fjp[k] + src;
            const double p2 = k < nY ? 0.5 * g1 * Vs + v.DHi[k * N + c]
                                     : (k == nY ? -g1 * u : (k == nY + 1 ? -g1 * vv : g1));
            t = t + p2 * R[k];
        }
        for (int k = 0; k < D; ++k) {
            const double p1 = k < nY ? phh * v.w[(4 + k) * N + c] : phh * (k == nY ? u : (k == nY + 1 ? vv : H));
            double rhs = R[k] + p1 * t;
            if (MODE == RES_PRECON) {
                const double qk = v.q[k * N + c], qpk = v.qp[k * N + c];
                const double dqdt = first ? (qk - qpk) / dt : (3.0 * qk - 4.0 * qpk + v.qpp[k * N + c]) / (2.0 * dt);
                rhs = rhs - vol * dqdt;
            }
            v.Dq[k * N + c] = rhs;
        }
        return;
    }
    for (int k = 0; k < D; ++k) {
        const double src = k == nY + 1 ? area * (sq_my + svq_my) : area * 0.0;
        double rhs = (double)fim[k] - (double)fip[k] + (double)fjm[k] - (double)fjp[k] + src;
        if (MODE == RES_NR || MODE == RES_DUAL) {
            const double qk = v.q[k * N + c], qpk = v.qp[k * N + c];
            const double dqdt = first ? (qk - qpk) / dtl : (3.0 * qk - 4.0 * qpk + v.qpp[k * N + c]) / (2.0 * dtl);
            rhs = rhs - vol * dqdt;
        }
        v.Dq[k * N + c] = rhs;
    }
    // set_ABpm: spectral radii and alpha (sch_lusgs.raw.f90:27-42,134-136; sch_NR 143-144)
    const double rho = v.w[c], u = v.w[N + c], vv = v.w[2 * N + c], pr = v.w[3 * N + c];
    const double gamm = v.w[(D + 1) * N + c];
    const double cs = sqrt(gamm * pr / rho);
    const double unA = v.vnci[c] * u + v.vnci[N + c] * vv;
    const double unB = v.vncj[c] * u + v.vncj[N + c] * vv;
    if (MODE == RES_DUAL) {
        // set_ABpm of the preconditioned dual time (dual/2d/sch_dual.raw.f90:38-83):
        // low-Mach reference velocity, preconditioned spectral radii, pseudo time
        // step from cfl_tau, and the scalars of Gamma^-1, S, S^-1
        const double mu = v.w[(D + 4) * N + c], dsa = v.dsci[c], dsb = v.dscj[c];
        const double Vs = u * u + vv * vv;
        const double Vv = mu / rho / fmin(dsa, dsb);
        const double Ur = fmin(fmax(Vv, sqrt(Vs)), cs);
        const double phi = 1.0 / (Ur * Ur) - 1.0 / (cs * cs);
        const double alp = 0.5 * (1.0 - (Ur / cs) * (Ur / cs));
        double ud = unA * (1.0 - alp), cd = sqrt(alp * alp * (unA * unA) + Ur * Ur);
        const double nuA = fabs(ud) + cd;
        ud = unB * (1.0 - alp);
        cd = sqrt(alp * alp * (unB * unB) + Ur * Ur);
        const double nuB = fabs(ud) + cd;
        const long long cim = cidx(v.P, p, i - 1, j), cjm = cidx(v.P, p, i, j - 1);
        const double uds = nuA * (v.dsi[c] + v.dsi[cim]) + nuB * (v.dsj[c] + v.dsj[cjm]);
        const double dtau = v.cfl_tau * vol / fmax(uds, mu / rho);
        const double al = 1.0 / (vol / dtau + dsa * nuA + dsb * nuB);
        const double beta = 3.0 * vol / (2.0 * dtl) * al;
        const double c2 = cs * cs;
        const double s2 = -1.0 / (1.0 / phi + c2);
        v.alpha[c] = al;
        v.nuA[c] = nuA;
        v.nuB[c] = nuB;
        v.pre[c] = 1.0 + beta;
        v.pre[N + c] = s2;
        v.pre[2 * N + c] = -1.0 / (1.0 / phi + c2) / (1.0 / beta + 1.0);
        v.pre[3 * N + c] = beta / ((1.0 + beta) / phi + c2);
        // Dq += pre_sca(2) * (pre2 . Dq) * pre1 (time_dual_viscous.f90:29), pre1 =
        // (Y, u, v, H), pre2 = (g1 Vs/2 + DHi, -g1 u, -g1 v, g1)
        const double g1 = gamm - 1.0, H = v.w[(D + 2) * N + c];
        double t = 0.0;
        for (int k = 0; k < nY; ++k) t = t + (0.5 * g1 * Vs + v.DHi[k * N + c]) * v.Dq[k * N + c];
        t = t + (-g1 * u) * v.Dq[nY * N + c];
        t = t + (-g1 * vv) * v.Dq[(nY + 1) * N + c];
        t = t + g1 * v.Dq[(nY + 2) * N + c];
        for (int k = 0; k < nY; ++k) v.Dq[k * N + c] = v.Dq[k * N + c] + s2 * t * v.w[(4 + k) * N + c];
        v.Dq[nY * N + c] = v.Dq[nY * N + c] + s2 * t * u;
        v.Dq[(nY + 1) * N + c] = v.Dq[(nY + 1) * N + c] + s2 * t * vv;
        v.Dq[(nY + 2) * N + c] = v.Dq[(nY + 2) * N + c] + s2 * t * H;
        return;
    }
    const double nuA = fabs(unA) + cs, nuB = fabs(unB) + cs;
    const double tmp = MODE == RES_NR ? 3.0 * vol / (2.0 * dtl) + v.dsci[c] * nuA + v.dscj[c] * nuB
                                      : vol / dtl + v.dsci[c] * nuA + v.dscj[c] * nuB;
    v.alpha[c] = 1.0 / tmp;
    v.nuA[c] = nuA;
    v.nuB[c] = nuB;
}

template <typename RT, int MODE>
static void launch_t(const View& v, cudaStream_t s) {
    int nimax = 0, njmax = 0;
    for (int a = 0; a < v.P.nact; ++a) {
        const int p = v.P.act[a];
        nimax = v.P.ni[p] > nimax ? v.P.ni[p] : nimax;
        njmax = v.P.nj[p] > njmax ? v.P.nj[p] : njmax;
    }
    if (v.P.nact == 0) return;
    dim3 grid((nimax + TX - 1) / TX, (njmax + TY - 1) / TY, v.P.nact);
    const size_t smem = (size_t)(TY * (TX + 1) + (TY + 1) * TX) * v.D * sizeof(RT);
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_residual<RT, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        attr_set = true;
    }
    k_residual<RT, MODE><<<grid, NT, smem, s>>>(v);
}

// need_coeffs: the caller's sweep reads alpha/nuA/nuB from the cell arrays,
// which only this generic kernel writes.
int launch_residual(const View& v, cudaStream_t s, int mode, bool need_coeffs) {
    if (mode != RES_DUAL && mode != RES_PRECON && mode != RES_PRECON_LUSGS && !need_coeffs &&
        launch_residual2(v, s, mode))
        return 1;
    const bool mixed = v.precision == SCFD_PREC_MIXED;
    if (mode == RES_EULER) {
        if (mixed) launch_t<float, RES_EULER>(v, s); else launch_t<double, RES_EULER>(v, s);
    } else if (mode == RES_LUSGS) {
        if (mixed) launch_t<float, RES_LUSGS>(v, s); else launch_t<double, RES_LUSGS>(v, s);
    } else if (mode == RES_DUAL) {
        if (mixed) launch_t<float, RES_DUAL>(v, s); else launch_t<double, RES_DUAL>(v, s);
    } else if (mode == RES_PRECON) {
        if (mixed) launch_t<float, RES_PRECON>(v, s); else launch_t<double, RES_PRECON>(v, s);
    } else if (mode == RES_PRECON_LUSGS) {
        if (mixed) launch_t<float, RES_PRECON_LUSGS>(v, s); else launch_t<double, RES_PRECON_LUSGS>(v, s);
    } else {
        if (mixed) launch_t<float, RES_NR>(v, s); else launch_t<double, RES_NR>(v, s);
    }
    return 1;
}

}  // namespace scfd
