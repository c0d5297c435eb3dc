// adj_face.cuh -- the inviscid face flux of the explicit ideal-gas step and its
// hand-written reverse (adjoint) mode, callable from host and device code.
//
// Forward: MUSCL face states of one component (store/high_order/muscl/
// muscl.f90:28-44, 52-68: w_l = w0 + phi/2 du(0), w_r = w1 - phi/2 dl(1) with
// the limiter s = 2 Du Dl / (Du^2 + Dl^2 + eps)) and the SLAU flux
// (store/core/scheme.f90:71-153).  The reverse functions take the adjoint of
// the outputs and add the adjoint of the inputs; the piecewise parts of SLAU
// (min, max, abs, sign and the |M| < 1 branches of beta) take the branch the
// forward values select, and the limiter, which has no branch, is
// differentiated exactly.  State vectors hold rho, u, v, p, Y(1:nY), gamma, h_t
// at [0..3], [4..3+nY], [4+nY], [5+nY].
#pragma once

#include <math.h>

#ifdef __CUDACC__
#include "div_pos.cuh"
#define SCFD_HD __host__ __device__ __forceinline__
#else
#define SCFD_HD inline
#endif

namespace scfd {
namespace adj {

constexpr double kEps = 1e-300;  // muscl.f90 epsln

// a / b for a positive normal b: on the device the branch-free quotient of
// div_pos.cuh (within one unit in the last place; the adjoint run of 300 steps
// at 196 k cells takes 62 ms with it, 68 without), on the host IEEE division.
// Every b below is a sum of squares plus eps, a density, a sound speed or a
// sum of them, or a positive square root.
SCFD_HD double qdiv(double a, double b) {
#ifdef __CUDA_ARCH__
    return div_pos(a, b);
#else
    return a / b;
#endif
}

SCFD_HD void muscl_fwd(double wm1, double w0, double w1, double w2, double phi, double km, double& wl, double& wr) {
    double Du = w1 - w0, Dl = w0 - wm1;
    double s = qdiv(2.0 * Du * Dl, Du * Du + Dl * Dl + kEps);
    const double du = 0.5 * s * ((1.0 + km * s) * Du + (1.0 - km * s) * Dl);
    wl = w0 + phi * 0.5 * du;
    Du = w2 - w1;
    Dl = w1 - w0;
    s = qdiv(2.0 * Du * Dl, Du * Du + Dl * Dl + kEps);
    const double dl = 0.5 * s * ((1.0 + km * s) * Dl + (1.0 - km * s) * Du);
    wr = w1 - phi * 0.5 * dl;
}

// ds/da and ds/db of s = 2ab / (a^2 + b^2 + eps), written so that a = b = 0 gives 0
SCFD_HD void limiter_grad(double a, double b, double iQ, double& sa, double& sb) {
    const double ra = 2.0 * b * iQ, rb = 2.0 * a * iQ;
    sa = ra * (1.0 - 2.0 * a * a * iQ);
    sb = rb * (1.0 - 2.0 * b * b * iQ);
}

// One-sided slope d(a, b) = s/2 ((1 + km s) a + (1 - km s) b), s = s(a, b): adds
// its adjoint g times the partial derivatives to ab, bb.
SCFD_HD void slope_rev(double a, double b, double km, double g, double& ab, double& bb) {
    const double iQ = qdiv(1.0, a * a + b * b + kEps);
    const double s = 2.0 * a * b * iQ;
    const double A = (1.0 + km * s) * a + (1.0 - km * s) * b;
    const double dds = 0.5 * A + 0.5 * s * km * (a - b);
    double sa, sb;
    limiter_grad(a, b, iQ, sa, sb);
    ab += g * (0.5 * s * (1.0 + km * s) + dds * sa);
    bb += g * (0.5 * s * (1.0 - km * s) + dds * sb);
}

// adds to bm1 .. b2 the adjoint of the stencil given the adjoints wlb, wrb
SCFD_HD void muscl_rev(double wm1, double w0, double w1, double w2, double phi, double km, double wlb, double wrb,
                       double& bm1, double& b0, double& b1, double& b2) {
    // w_l = w0 + phi/2 d(Du = w1 - w0, Dl = w0 - wm1)
    b0 += wlb;
    double gDu = 0.0, gDl = 0.0;
    slope_rev(w1 - w0, w0 - wm1, km, wlb * phi * 0.5, gDu, gDl);
    b1 += gDu;
    b0 += gDl - gDu;
    bm1 -= gDl;
    // w_r = w1 - phi/2 d(Dl2 = w1 - w0, Du2 = w2 - w1), the slope led by Dl2
    b1 += wrb;
    double gDl2 = 0.0, gDu2 = 0.0;
    slope_rev(w1 - w0, w2 - w1, km, -wrb * phi * 0.5, gDl2, gDu2);
    b2 += gDu2;
    b1 += gDl2 - gDu2;
    b0 -= gDl2;
}

SCFD_HD double sgn(double x) { return x >= 0.0 ? 1.0 : -1.0; }

// SLAU (scheme.f90:71-153) of the face with unit normal (n1, n2)
SCFD_HD void slau_fwd(int nY, const double* wl, const double* wr, double n1, double n2, double* tg) {
    const double rhol = wl[0], ul = wl[1], vl = wl[2], pl = wl[3], gl = wl[4 + nY];
    const double rhor = wr[0], ur = wr[1], vr = wr[2], pr = wr[3], gr = wr[4 + nY];
    const double al = sqrt(qdiv(gl * pl, rhol)), ar = sqrt(qdiv(gr * pr, rhor));
    const double unl = n1 * ul + n2 * vl, unr = n1 * ur + n2 * vr;
    const double dp = pr - pl;
    const double a_bar = 0.5 * (ar + al);
    const double p_bar = 0.5 * (pr + pl);
    const double ia = qdiv(1.0, a_bar);
    const double ml = unl * ia, mr = unr * ia;
    const double m_tilde = fmin(1.0, ia * sqrt(0.5 * (ul * ul + vl * vl + ur * ur + vr * vr)));
    const double chi = (1.0 - m_tilde) * (1.0 - m_tilde);
    const double gp = -fmax(fmin(ml, 0.0), -1.0);
    const double gm = fmin(fmax(mr, 0.0), 1.0);
    const double g = gp * gm;
    const double ub = qdiv(fabs(unr) * rhor + fabs(unl) * rhol, rhor + rhol);
    const double ubp = (1.0 - g) * ub + g * fabs(unl);
    const double ubm = (1.0 - g) * ub + g * fabs(unr);
    const double dm = 0.5 * (rhol * (unl + ubp) + rhor * (unr - ubm) - chi * ia * dp);
    const double betar = fabs(mr) < 1.0 ? 0.25 * (2.0 + mr) * ((mr - 1.0) * (mr - 1.0)) : 0.5 * (1.0 - copysign(1.0, mr));
    const double betal = fabs(ml) < 1.0 ? 0.25 * (2.0 - ml) * ((ml + 1.0) * (ml + 1.0)) : 0.5 * (1.0 + copysign(1.0, ml));
    const double pt = p_bar + 0.5 * (betal - betar) * (pl - pr) + (1.0 - chi) * (betar + betal - 1.0) * p_bar;
    const double dpp = 0.5 * (dm + fabs(dm)), dnn = 0.5 * (dm - fabs(dm));
    for (int k = 0; k < nY; ++k) tg[k] = dpp * wl[4 + k] + dnn * wr[4 + k];
    tg[nY] = dpp * ul + dnn * ur + pt * n1;
    tg[nY + 1] = dpp * vl + dnn * vr + pt * n2;
    tg[nY + 2] = dpp * wl[5 + nY] + dnn * wr[5 + nY];
}

// adds to wlb, wrb the adjoint of the face states given the adjoint tgb of the flux
SCFD_HD void slau_rev(int nY, const double* wl, const double* wr, double n1, double n2, const double* tgb, double* wlb,
                      double* wrb) {
    // forward values
    const double rhol = wl[0], ul = wl[1], vl = wl[2], pl = wl[3], gl = wl[4 + nY];
    const double rhor = wr[0], ur = wr[1], vr = wr[2], pr = wr[3], gr = wr[4 + nY];
    const double Al = qdiv(gl * pl, rhol), Ar = qdiv(gr * pr, rhor);
    const double al = sqrt(Al), ar = sqrt(Ar);
    const double unl = n1 * ul + n2 * vl, unr = n1 * ur + n2 * vr;
    const double dp = pr - pl;
    const double a_bar = 0.5 * (ar + al);
    const double p_bar = 0.5 * (pr + pl);
    const double ia = qdiv(1.0, a_bar), ia2 = ia * ia;
    const double ml = unl * ia, mr = unr * ia;
    const double S = 0.5 * (ul * ul + vl * vl + ur * ur + vr * vr);
    const double sq = sqrt(S);
    const double mraw = ia * sq;
    const double m_tilde = fmin(1.0, mraw);
    const double chi = (1.0 - m_tilde) * (1.0 - m_tilde);
    const double gp = -fmax(fmin(ml, 0.0), -1.0);
    const double gm = fmin(fmax(mr, 0.0), 1.0);
    const double g = gp * gm;
    const double num = fabs(unr) * rhor + fabs(unl) * rhol, den = rhor + rhol;
    const double iden = qdiv(1.0, den);
    const double ub = num * iden;
    const double ubp = (1.0 - g) * ub + g * fabs(unl);
    const double ubm = (1.0 - g) * ub + g * fabs(unr);
    const double dm = 0.5 * (rhol * (unl + ubp) + rhor * (unr - ubm) - chi * ia * dp);
    const bool rin = fabs(mr) < 1.0, lin = fabs(ml) < 1.0;
    const double betar = rin ? 0.25 * (2.0 + mr) * ((mr - 1.0) * (mr - 1.0)) : 0.5 * (1.0 - copysign(1.0, mr));
    const double betal = lin ? 0.25 * (2.0 - ml) * ((ml + 1.0) * (ml + 1.0)) : 0.5 * (1.0 + copysign(1.0, ml));
    const double dpp = 0.5 * (dm + fabs(dm)), dnn = 0.5 * (dm - fabs(dm));
    // reverse of the flux components
    double dppb = 0.0, dnnb = 0.0;
    for (int k = 0; k < nY; ++k) {
        dppb += tgb[k] * wl[4 + k];
        dnnb += tgb[k] * wr[4 + k];
        wlb[4 + k] += tgb[k] * dpp;
        wrb[4 + k] += tgb[k] * dnn;
    }
    double ulb = tgb[nY] * dpp, urb = tgb[nY] * dnn;
    double vlb = tgb[nY + 1] * dpp, vrb = tgb[nY + 1] * dnn;
    dppb += tgb[nY] * ul + tgb[nY + 1] * vl + tgb[nY + 2] * wl[5 + nY];
    dnnb += tgb[nY] * ur + tgb[nY + 1] * vr + tgb[nY + 2] * wr[5 + nY];
    wlb[5 + nY] += tgb[nY + 2] * dpp;
    wrb[5 + nY] += tgb[nY + 2] * dnn;
    const double ptb = tgb[nY] * n1 + tgb[nY + 1] * n2;
    // dpp, dnn
    const double s = sgn(dm);
    const double dmb = dppb * 0.5 * (1.0 + s) + dnnb * 0.5 * (1.0 - s);
    // pt
    double p_barb = ptb * (1.0 + (1.0 - chi) * (betar + betal - 1.0));
    const double betalb = ptb * (0.5 * (pl - pr) + (1.0 - chi) * p_bar);
    const double betarb = ptb * (-0.5 * (pl - pr) + (1.0 - chi) * p_bar);
    double plb = ptb * 0.5 * (betal - betar), prb = -ptb * 0.5 * (betal - betar);
    double chib = -ptb * (betar + betal - 1.0) * p_bar;
    double mrb = 0.0, mlb = 0.0;
    if (rin) mrb += betarb * 0.25 * ((mr - 1.0) * (mr - 1.0) + (2.0 + mr) * 2.0 * (mr - 1.0));
    if (lin) mlb += betalb * 0.25 * (-(ml + 1.0) * (ml + 1.0) + (2.0 - ml) * 2.0 * (ml + 1.0));
    // dm
    double rholb = dmb * 0.5 * (unl + ubp), rhorb = dmb * 0.5 * (unr - ubm);
    double unlb = dmb * 0.5 * rhol, unrb = dmb * 0.5 * rhor;
    const double ubpb = dmb * 0.5 * rhol, ubmb = -dmb * 0.5 * rhor;
    chib += -dmb * 0.5 * dp * ia;
    double a_barb = dmb * 0.5 * chi * dp * ia2;
    const double dpb = -dmb * 0.5 * chi * ia;
    // ubp, ubm
    double ubb = ubpb * (1.0 - g) + ubmb * (1.0 - g);
    const double gb = ubpb * (fabs(unl) - ub) + ubmb * (fabs(unr) - ub);
    unlb += ubpb * g * sgn(unl);
    unrb += ubmb * g * sgn(unr);
    // ub = num / den
    const double numb = ubb * iden, denb = -ubb * num * iden * iden;
    unrb += numb * rhor * sgn(unr);
    rhorb += numb * fabs(unr) + denb;
    unlb += numb * rhol * sgn(unl);
    rholb += numb * fabs(unl) + denb;
    // g = gp gm
    const double gpb = gb * gm, gmb = gb * gp;
    if (ml < 0.0 && ml > -1.0) mlb += -gpb;
    if (mr > 0.0 && mr < 1.0) mrb += gmb;
    // chi, m_tilde
    const double mtb = chib * (-2.0 * (1.0 - m_tilde));
    const double mrawb = mraw < 1.0 ? mtb : 0.0;
    const double sqb = mrawb * ia;
    a_barb += -mrawb * sq * ia2;
    if (sq > 0.0) {
        const double Sb = qdiv(sqb, 2.0 * sq);
        ulb += Sb * ul;
        vlb += Sb * vl;
        urb += Sb * ur;
        vrb += Sb * vr;
    }
    // Mach numbers
    unlb += mlb * ia;
    unrb += mrb * ia;
    a_barb += -(mlb * unl + mrb * unr) * ia2;
    // p_bar, a_bar, dp
    prb += 0.5 * p_barb + dpb;
    plb += 0.5 * p_barb - dpb;
    const double alb = 0.5 * a_barb, arb = 0.5 * a_barb;
    // normal velocities
    ulb += n1 * unlb;
    vlb += n2 * unlb;
    urb += n1 * unrb;
    vrb += n2 * unrb;
    // sound speeds a = sqrt(gamma p / rho)
    const double irl = qdiv(1.0, rhol), irr = qdiv(1.0, rhor);
    const double Alb = qdiv(0.5 * alb, al), Arb = qdiv(0.5 * arb, ar);
    wlb[4 + nY] += Alb * pl * irl;
    plb += Alb * gl * irl;
    rholb += -Alb * Al * irl;
    wrb[4 + nY] += Arb * pr * irr;
    prb += Arb * gr * irr;
    rhorb += -Arb * Ar * irr;
    wlb[0] += rholb;
    wlb[1] += ulb;
    wlb[2] += vlb;
    wlb[3] += plb;
    wrb[0] += rhorb;
    wrb[1] += urb;
    wrb[2] += vrb;
    wrb[3] += prb;
}

// The ideal-gas primitive state from q (set_w, store/core/scheme.f90:1-29, and
// the ideal thermal model, therm_lib/ideal/thermal_model.raw.f90:7-33):
// rho = sum q_k, u, v, Y_k = q/rho, p = rho (kappa-1) ei, h_t = (E + p)/rho.
// Adds to qb the adjoint of q given the adjoints of rho, u, v, p, Y_k, h_t.
SCFD_HD void ideal_prim_rev(int nY, const double* q, double kappa, double rhob, double ub, double vb, double pb,
                            const double* Yb, double htb, double* qb) {
    double rho = 0.0;
    for (int k = 0; k < nY; ++k) rho = rho + q[k];
    const double ir = qdiv(1.0, rho), ir2 = ir * ir;
    const double u = q[nY] * ir, v = q[nY + 1] * ir, E = q[nY + 2];
    const double ei = E * ir - 0.5 * (u * u + v * v);
    const double p = rho * (kappa - 1.0) * ei;
    double Eb = htb * ir;
    pb += htb * ir;
    rhob += -htb * (E + p) * ir2;
    rhob += pb * (kappa - 1.0) * ei;
    const double eib = pb * rho * (kappa - 1.0);
    Eb += eib * ir;
    rhob += -eib * E * ir2;
    ub += -eib * u;
    vb += -eib * v;
    for (int k = 0; k < nY; ++k) {
        qb[k] += Yb[k] * ir;
        rhob += -Yb[k] * q[k] * ir2;
    }
    qb[nY] += ub * ir;
    qb[nY + 1] += vb * ir;
    rhob += -(ub * q[nY] + vb * q[nY + 1]) * ir2;
    qb[nY + 2] += Eb;
    for (int k = 0; k < nY; ++k) qb[k] += rhob;
}

// p of the objective, straight from q: (kappa-1)(E - |rho u|^2 / (2 rho)), and
// its gradient
SCFD_HD double ideal_p(int nY, const double* q, double kappa) {
    double rho = 0.0;
    for (int k = 0; k < nY; ++k) rho = rho + q[k];
    return (kappa - 1.0) * (q[nY + 2] - 0.5 * (q[nY] * q[nY] + q[nY + 1] * q[nY + 1]) / rho);
}
SCFD_HD void ideal_p_rev(int nY, const double* q, double kappa, double pb, double* qb) {
    double rho = 0.0;
    for (int k = 0; k < nY; ++k) rho = rho + q[k];
    const double m2 = q[nY] * q[nY] + q[nY + 1] * q[nY + 1];
    for (int k = 0; k < nY; ++k) qb[k] += pb * (kappa - 1.0) * 0.5 * m2 / (rho * rho);
    qb[nY] += -pb * (kappa - 1.0) * q[nY] / rho;
    qb[nY + 1] += -pb * (kappa - 1.0) * q[nY + 1] / rho;
    qb[nY + 2] += pb * (kappa - 1.0);
}

}  // namespace adj
}  // namespace scfd
