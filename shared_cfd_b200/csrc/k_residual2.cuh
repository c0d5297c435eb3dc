// k_residual2.cuh -- the fused residual kernel for compile-time species counts,
// with the tile's primitive field staged in shared memory.
//
// Same arithmetic as k_residual.cu: set_HV (store/high_order/muscl/muscl.f90:7-73),
// set_TG (store/core/scheme.f90:31-259), set_TGv (store/viscosity/viscous/no-nV/
// {2d,q2d}/sch_viscous.f90:75-321), set_Sq (store/dim/q2d/Sq.f90) and the
// right-hand side of the time schemes.  A CTA owns TX x TY cells (32 x 8 by
// default); it first copies w (W components), vhi (nY) and T = p/(rho R) of the
// tile plus a 2-cell halo into shared memory with coalesced loads, then
// computes the TY(TX+1) i-faces and (TY+1)TX j-faces of the tile from shared
// memory (about two faces per thread), then sums faces and sources per cell.
// The FP64 kernel stages w and T only and reads vhi through L1: its 16x8 tile
// then takes 61 KB of shared memory and three CTAs fit on an SM (with vhi
// staged, two), which its latency-bound faces need more than the loads.
// The LU-SGS coefficients are formed later by the record packer, so this
// kernel writes only the D values of the right-hand side (or the explicit
// update).  The tile shape is one of residual2_tiles(), picked per context by
// the autotuner; every shape computes each face and cell with the same
// arithmetic in the same order.  The FP32 and FP64 instantiations are compiled
// in k_residual2_f32.cu and k_residual2_f64.cu.
#pragma once

#include "div_pos.cuh"
#include "scfd_internal.h"

namespace scfd {

namespace {

template <int TX_, int TY_, int NTH_>
struct Tile {
    static constexpr int TX = TX_, TY = TY_, HX = TX + 4, HY = TY + 4, NTH = NTH_;
    static constexpr int NFI = TY * (TX + 1), NFJ = (TY + 1) * TX;
    static_assert(NTH >= TX * TY, "one thread per cell in the sum phase");
};
using Tile0 = Tile<32, 8, 288>;
using Tile1 = Tile<16, 16, 288>;
using Tile2 = Tile<64, 4, 288>;
using Tile3 = Tile<16, 8, 160>;

template <typename RT>
__device__ __forceinline__ RT eps_of();
template <>
__device__ __forceinline__ double eps_of<double>() { return 1e-300; }
template <>
__device__ __forceinline__ float eps_of<float>() { return 1e-37f; }

template <typename RT>
struct Smem {
    RT* w;   // [W][HY][HX]
    RT* vh;  // [NY][HY][HX]
    RT* T;   // [HY][HX]
    RT* FI;  // [NFI][D]
    RT* FJ;  // [NFJ][D]
};

// vhi staged in shared memory (FP32); the FP64 faces read it through L1 instead,
// which keeps the FP64 tile at three CTAs per SM
template <typename RT>
constexpr bool kStageVh = sizeof(RT) == 4;

}  // namespace

// The face's quotients go through div_pos (a branch-free quotient): the 2 (NY + 6)
// limiter quotients and the SLAU and viscous ones then overlap, and the FP64
// residual takes 0.42 ms instead of 0.59 at 786 k cells (FP32 0.36 instead of
// 0.44).  Their denominators are sums of squares plus eps, densities, a sound
// speed, gamma - 1 and positive constants.
template <typename RT, int NY, typename TL>
__device__ __forceinline__ void face2(const View& v, const Smem<RT>& S, int p, int i, int j, int ix, int jy, bool iface,
                                      RT* out) {
    constexpr int D = NY + 3;
    constexpr int HX = TL::HX, HS = TL::HY * TL::HX;
    const RT phi = RT(v.recon == SCFD_RECON_MUSCL ? v.phi_mus : 0.0), km = RT(v.k_mus);
    const RT half = RT(0.5), one = RT(1), two = RT(2);
    // smem cell offsets along the face normal: m1, 0 (left), 1 (right), 2
    const int st = iface ? 1 : HX;
    const int c0 = jy * HX + ix;
    RT wl[NY + 6], wr[NY + 6];
#pragma unroll
    for (int m = 0; m < NY + 6; ++m) {
        const RT* a = S.w + m * HS + c0;
        const RT wm1 = a[-st], w0 = a[0], w1 = a[st], w2 = a[2 * st];
        RT Du = w1 - w0, Dl = w0 - wm1;
        RT s = div_pos(two * Du * Dl, Du * Du + Dl * Dl + eps_of<RT>());
        const RT du = half * s * ((one + km * s) * Du + (one - km * s) * Dl);
        wl[m] = w0 + phi * half * du;
        Du = w2 - w1;
        Dl = w1 - w0;
        s = div_pos(two * Du * Dl, Du * Du + Dl * Dl + eps_of<RT>());
        const RT dl = half * s * ((one + km * s) * Dl + (one - km * s) * Du);
        wr[m] = w1 - phi * half * dl;
    }
    const long long N = v.ncell;
    const long long cg = cidx(v.P, p, i, j);
    const double* vn = iface ? v.vni : v.vnj;
    const RT n1 = RT(__ldg(vn + cg)), n2 = RT(__ldg(vn + N + cg));
    // SLAU (scheme.f90:71-153)
    RT tg[D];
    {
        const RT rhol = wl[0], ul = wl[1], vl = wl[2], pl = wl[3], gl = wl[4 + NY];
        const RT rhor = wr[0], ur = wr[1], vr = wr[2], pr = wr[3], gr = wr[4 + NY];
        const RT al = sqrt(div_pos(gl * pl, rhol)), ar = sqrt(div_pos(gr * pr, rhor));
        const RT unl = n1 * ul + n2 * vl, unr = n1 * ur + n2 * vr;
        const RT dp = pr - pl;
        const RT a_bar = half * (ar + al);
        const RT p_bar = half * (pr + pl);
        const RT ia = div_pos(one, a_bar);
        const RT ml = unl * ia, mr = unr * ia;
        const RT m_tilde = fmin(one, ia * sqrt(half * (ul * ul + vl * vl + ur * ur + vr * vr)));
        const RT chi = (one - m_tilde) * (one - m_tilde);
        const RT gp = -fmax(fmin(ml, RT(0)), -one);
        const RT gm = fmin(fmax(mr, RT(0)), one);
        const RT g = gp * gm;
        const RT ub = div_pos(fabs(unr) * rhor + fabs(unl) * rhol, rhor + rhol);
        const RT ubp = (one - g) * ub + g * fabs(unl);
        const RT ubm = (one - g) * ub + g * fabs(unr);
        const RT dm = half * (rhol * (unl + ubp) + rhor * (unr - ubm) - chi * ia * dp);
        const RT betar = fabs(mr) < one ? RT(0.25) * (two + mr) * ((mr - one) * (mr - one)) : half * (one - copysign(one, mr));
        const RT betal = fabs(ml) < one ? RT(0.25) * (two - ml) * ((ml + one) * (ml + one)) : half * (one + copysign(one, ml));
        const RT pt = p_bar + half * (betal - betar) * (pl - pr) + (one - chi) * (betar + betal - one) * p_bar;
        const RT dpp = half * (dm + fabs(dm)), dnn = half * (dm - fabs(dm));
#pragma unroll
        for (int k = 0; k < NY; ++k) tg[k] = dpp * wl[4 + k] + dnn * wr[4 + k];
        tg[NY] = dpp * ul + dnn * ur + pt * n1;
        tg[NY + 1] = dpp * vl + dnn * vr + pt * n2;
        tg[NY + 2] = dpp * wl[5 + NY] + dnn * wr[5 + NY];
    }
    const RT ds = RT(__ldg((iface ? v.dsi : v.dsj) + cg));
    if (!v.viscous) {
#pragma unroll
        for (int k = 0; k < D; ++k) out[k] = ds * tg[k];
        return;
    }
    // viscous face flux (sch_viscous.f90:125-197, 214-286)
    const int iR = D + 3, ig = D + 1, imu = D + 4;
    const int cb = c0 + st;  // the cell across the face
    // cross-derivative stencil: (+1,+1) (0,+1) - (+1,-1) - (0,-1) in (normal, tangential)
    const int tn = iface ? HX : 1;  // tangential stride
    const int p1 = c0 + st + tn, p2 = c0 + tn, m1 = c0 + st - tn, m2 = c0 - tn;
    auto W_ = [&](int k, int c) { return S.w[k * HS + c]; };
    const RT q4 = RT(0.25);
    const RT rho = (W_(0, c0) + W_(0, cb)) * half;
    const RT u = (W_(1, c0) + W_(1, cb)) * half;
    const RT vv = (W_(2, c0) + W_(2, cb)) * half;
    const RT gamm = (W_(ig, c0) + W_(ig, cb)) * half;
    const RT Rgas = (W_(iR, c0) + W_(iR, cb)) * half;
    const RT mu = (W_(imu, c0) + W_(imu, cb)) * half;
    const RT Dd = div_pos(div_pos(mu, rho), RT(v.schmidt));
    const RT k_heat = div_pos(div_pos(mu * gamm, gamm - one) * Rgas, RT(v.prandtl));
    const RT dN_u = W_(1, cb) - W_(1, c0), dN_v = W_(2, cb) - W_(2, c0), dN_T = S.T[cb] - S.T[c0];
    const RT dC_u = (W_(1, p1) + W_(1, p2) - W_(1, m1) - W_(1, m2)) * q4;
    const RT dC_v = (W_(2, p1) + W_(2, p2) - W_(2, m1) - W_(2, m2)) * q4;
    const RT dC_T = (S.T[p1] + S.T[p2] - S.T[m1] - S.T[m2]) * q4;
    const double* gj = iface ? v.gji : v.gjj;
    const RT g11 = RT(__ldg(gj + cg)), g12 = RT(__ldg(gj + N + cg)), g21 = RT(__ldg(gj + 2 * N + cg)),
             g22 = RT(__ldg(gj + 3 * N + cg));
    const RT dudxi = iface ? dN_u : dC_u, dudeta = iface ? dC_u : dN_u;
    const RT dvdxi = iface ? dN_v : dC_v, dvdeta = iface ? dC_v : dN_v;
    const RT dTdxi = iface ? dN_T : dC_T, dTdeta = iface ? dC_T : dN_T;
    const RT dudx = dudxi * g11 + dudeta * g21, dvdx = dvdxi * g11 + dvdeta * g21, dTdx = dTdxi * g11 + dTdeta * g21;
    const RT dudr = dudxi * g12 + dudeta * g22, dvdr = dvdxi * g12 + dvdeta * g22, dTdr = dTdxi * g12 + dTdeta * g22;
    RT hidwdx = RT(0), hidwdr = RT(0);
    const RT rhoD = rho * Dd;
    RT tv[D];
#pragma unroll
    for (int k = 0; k < NY; ++k) {
        const int kw = 4 + k;
        const RT dN = W_(kw, cb) - W_(kw, c0);
        const RT dC = (W_(kw, p1) + W_(kw, p2) - W_(kw, m1) - W_(kw, m2)) * q4;
        const RT dxi = iface ? dN : dC, deta = iface ? dC : dN;
        const RT dwdx = dxi * g11 + deta * g21, dwdr = dxi * g12 + deta * g22;
        RT lhi;
        if constexpr (kStageVh<RT>) {
            lhi = (S.vh[k * HS + c0] + S.vh[k * HS + cb]) * half;
        } else {
            const long long cgb = cg + (iface ? 1 : v.P.pitch[p]);
            lhi = (RT(__ldg(v.vhi + k * N + cg)) + RT(__ldg(v.vhi + k * N + cgb))) * half;
        }
        hidwdx = hidwdx + dwdx * lhi;
        hidwdr = hidwdr + dwdr * lhi;
        tv[k] = rhoD * dwdx * n1 + rhoD * dwdr * n2;
    }
    RT divu = dudx + dvdr;
    if (v.dim == SCFD_DIM_Q2D) divu = dudx + dvdr + vv / RT(__ldg(v.r + cidx(v.P, p, i, j)));
    const RT t_xx = -two / RT(3) * mu * divu + two * mu * dudx;
    const RT t_rr = -two / RT(3) * mu * divu + two * mu * dvdr;
    const RT t_xr = mu * (dvdx + dudr);
    const RT qx = -k_heat * dTdx - rho * Dd * hidwdx;
    const RT qr = -k_heat * dTdr - rho * Dd * hidwdr;
    tv[NY] = t_xx * n1 + t_xr * n2;
    tv[NY + 1] = t_xr * n1 + t_rr * n2;
    tv[NY + 2] = (u * t_xx + vv * t_xr - qx) * n1 + (u * t_xr + vv * t_rr - qr) * n2;
#pragma unroll
    for (int k = 0; k < D; ++k) out[k] = ds * (tg[k] - tv[k]);
}

template <typename RT, int NY, int MODE, typename TL>
__global__ void __launch_bounds__(TL::NTH) k_residual2(View v) {
    constexpr int TX = TL::TX, TY = TL::TY, HX = TL::HX, NTH = TL::NTH, NFI = TL::NFI, NFJ = TL::NFJ;
    constexpr int D = NY + 3, W = D + 5, HS = TL::HY * HX;
    extern __shared__ __align__(16) unsigned char smraw[];
    Smem<RT> S;
    S.w = reinterpret_cast<RT*>(smraw);
    constexpr int NVH = kStageVh<RT> ? NY : 0;  // staged vhi components
    S.vh = S.w + W * HS;
    S.T = S.vh + NVH * HS;
    S.FI = S.T + HS;
    S.FJ = S.FI + NFI * D;
    const int p = v.P.act[blockIdx.z];
    const int ni = v.P.ni[p], nj = v.P.nj[p];
    const int i0 = blockIdx.x * TX + 1, j0 = blockIdx.y * TY + 1;
    if (i0 > ni || j0 > nj) return;
    const int tid = threadIdx.x;
    const long long N = v.ncell;
    // stage w, vhi: rows j0-2 .. j0+TY+1, columns i0-2 .. i0+TX+1 (coalesced along i)
    const long long base0 = cidx(v.P, p, i0 - 2, j0 - 2);
    const int pitch = v.P.pitch[p];
    // FP64: the tile's face metrics and vhi (read through L1 in the faces) and the
    // cell phase's q, qp, qpp, Vol and Area are prefetched into L2 first, so that
    // their loads wait on L2 instead of DRAM (0.425 -> 0.401 ms at 786 k cells; the
    // FP32 kernel stages vhi and gains nothing).  Addresses are clamped to each
    // array's cells.
    if constexpr (sizeof(RT) == 8) {
        auto pf = [&](const double* a, long long c) {
            c = c < 0 ? 0 : (c >= N ? N - 1 : c);
            asm volatile("prefetch.global.L2 [%0];" ::"l"(a + c));
        };
        constexpr int LF = (TX + 2 + 15) / 16 + 1, LC = (TX + 15) / 16 + 1, NR = TY + 2;
        const int nfa = NY + 6 + (v.viscous ? 8 : 0);
        for (int e = tid; e < nfa * NR * LF; e += NTH) {
            const int a = e / (NR * LF), rem = e - a * (NR * LF), r = rem / LF, l = rem - r * LF;
            const double* arr;
            if (a < NY) arr = v.vhi + (long long)a * N;
            else {
                const int b = a - NY;
                arr = b < 2 ? v.vni + b * N : b < 4 ? v.vnj + (b - 2) * N : b == 4 ? v.dsi : b == 5 ? v.dsj
                    : b < 10 ? v.gji + (b - 6) * N : v.gjj + (b - 10) * N;
            }
            pf(arr, cidx(v.P, p, i0 - 1, j0 - 1 + r) + l * 16);
        }
        if (MODE == RES_NR) {
            for (int e = tid; e < (3 * D + 2) * TY * LC; e += NTH) {
                const int a = e / (TY * LC), rem = e - a * (TY * LC), r = rem / LC, l = rem - r * LC;
                const double* arr = a < D ? v.q + (long long)a * N : a < 2 * D ? v.qp + (long long)(a - D) * N
                    : a < 3 * D ? v.qpp + (long long)(a - 2 * D) * N : a == 3 * D ? v.Vol : v.Area;
                pf(arr, cidx(v.P, p, i0, j0 + r) + l * 16);
            }
        }
    }
    for (int e = tid; e < (W + NVH) * HS; e += NTH) {
        const int comp = e / HS, rem = e - comp * HS;
        const int jy = rem / HX, ix = rem - jy * HX;
        const int i = i0 - 2 + ix, j = j0 - 2 + jy;
        RT val = RT(0);
        if (i <= ni + 2 && j <= nj + 2) {
            const long long c = base0 + (long long)jy * pitch + ix;
            // the FP32 tile is rounded from the FP64 state here (the values the
            // generic kernel's FP32 copies hold)
            val = comp < W ? RT(__ldg(v.w + comp * N + c)) : RT(__ldg(v.vhi + (comp - W) * N + c));
        }
        S.w[e] = val;  // S.vh follows S.w contiguously
    }
    __syncthreads();
    for (int e = tid; e < HS; e += NTH) {
        const RT rr = S.w[e];
        S.T[e] = rr != RT(0) ? S.w[3 * HS + e] / rr / S.w[(D + 3) * HS + e] : RT(0);
    }
    __syncthreads();
    // faces: i-faces f < NFI, j-faces after
    for (int f = tid; f < NFI + NFJ; f += NTH) {
        if (f < NFI) {
            const int fy = f / (TX + 1), fx = f - fy * (TX + 1);
            const int i = i0 - 1 + fx, j = j0 + fy;
            if (i <= ni && j <= nj) face2<RT, NY, TL>(v, S, p, i, j, fx + 1, fy + 2, true, S.FI + f * D);
        } else {
            const int g = f - NFI;
            const int fy = g / TX, fx = g - fy * TX;
            const int i = i0 + fx, j = j0 - 1 + fy;
            if (i <= ni && j <= nj) face2<RT, NY, TL>(v, S, p, i, j, fx + 2, fy + 1, false, S.FJ + g * D);
        }
    }
    __syncthreads();
    if (tid >= TX * TY) return;
    const int tx = tid % TX, ty = tid / TX;
    const int i = i0 + tx, j = j0 + ty;
    if (i > ni || j > nj) return;
    const long long c = cidx(v.P, p, i, j);
    const bool q2d = v.dim == SCFD_DIM_Q2D;
    const double area = v.Area[c];
    double svq_my = 0.0, sq_my = 0.0;
    if (q2d) {
        sq_my = v.w[3 * N + c];
        if (v.viscous) {
            // Svq (q2d sch_viscous.f90:297-316)
            const double vv = v.w[2 * N + c], mu = v.w[(D + 4) * N + c];
            const long long cip = c + 1, cim = c - 1, cjp = c + pitch, cjm = c - pitch;
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
    const RT* fim = S.FI + (ty * (TX + 1) + tx) * D;
    const RT* fip = fim + D;
    const RT* fjm = S.FJ + (ty * TX + tx) * D;
    const RT* fjp = S.FJ + ((ty + 1) * TX + tx) * D;
    const double dtl = v.dt_mode == SCFD_DT_LOCAL ? v.dt_mat[c] : v.sc->dt_grbl;
    if (MODE == RES_EULER) {
        const double fct = dtl / v.Vol[c];
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const double src = k == NY + 1 ? area * (sq_my + svq_my) : area * 0.0;
            const double rhs = (double)fim[k] - (double)fip[k] + (double)fjm[k] - (double)fjp[k] + src;
            v.q[k * N + c] = v.qp[k * N + c] + fct * rhs;
        }
        return;
    }
    const double vol = v.Vol[c];
    const bool first = v.sc->first_dual != 0;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        const double src = k == NY + 1 ? area * (sq_my + svq_my) : area * 0.0;
        double rhs = (double)fim[k] - (double)fip[k] + (double)fjm[k] - (double)fjp[k] + src;
        if (MODE == RES_NR) {
            const double qk = v.q[k * N + c], qpk = v.qp[k * N + c];
            const double dqdt = first ? (qk - qpk) / dtl : (3.0 * qk - 4.0 * qpk + v.qpp[k * N + c]) / (2.0 * dtl);
            rhs = rhs - vol * dqdt;
        }
        v.Dq[k * N + c] = rhs;
    }
}

template <typename RT, int NY, int MODE, typename TL>
inline void launch2(const View& v, cudaStream_t s) {
    constexpr int D = NY + 3, W = D + 5, TX = TL::TX, TY = TL::TY;
    int nimax = 0, njmax = 0;
    for (int a = 0; a < v.P.nact; ++a) {
        const int p = v.P.act[a];
        nimax = v.P.ni[p] > nimax ? v.P.ni[p] : nimax;
        njmax = v.P.nj[p] > njmax ? v.P.nj[p] : njmax;
    }
    if (v.P.nact == 0) return;
    dim3 grid((nimax + TX - 1) / TX, (njmax + TY - 1) / TY, v.P.nact);
    const size_t smem =
        ((size_t)(W + (kStageVh<RT> ? NY : 0) + 1) * TL::HY * TL::HX + (size_t)(TL::NFI + TL::NFJ) * D) * sizeof(RT);
    // the attribute is per device: set it before every launch (host only, cheap)
    cudaFuncSetAttribute(k_residual2<RT, NY, MODE, TL>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    k_residual2<RT, NY, MODE, TL><<<grid, TL::NTH, smem, s>>>(v);
}

template <typename RT, int NY, int MODE>
inline void by_tile(const View& v, cudaStream_t s) {
    switch (v.res_tile) {
        case 1: launch2<RT, NY, MODE, Tile1>(v, s); break;
        case 2: launch2<RT, NY, MODE, Tile2>(v, s); break;
        case 3: launch2<RT, NY, MODE, Tile3>(v, s); break;
        default: launch2<RT, NY, MODE, Tile0>(v, s); break;
    }
}

template <typename RT, int NY>
inline void by_mode_rt(const View& v, cudaStream_t s, int mode) {
    if (mode == RES_EULER)
        by_tile<RT, NY, RES_EULER>(v, s);
    else if (mode == RES_LUSGS)
        by_tile<RT, NY, RES_LUSGS>(v, s);
    else
        by_tile<RT, NY, RES_NR>(v, s);
}

// the launchers of one record precision (k_residual2_f32.cu, k_residual2_f64.cu);
// false when no specialised kernel exists for this species count
bool launch_residual2_f32(const View& v, cudaStream_t s, int mode);
bool launch_residual2_f64(const View& v, cudaStream_t s, int mode);

template <typename RT>
inline bool launch_residual2_rt(const View& v, cudaStream_t s, int mode) {
    switch (v.nY) {
        case 1: by_mode_rt<RT, 1>(v, s, mode); return true;
        case 8: by_mode_rt<RT, 8>(v, s, mode); return true;
        case 9: by_mode_rt<RT, 9>(v, s, mode); return true;
        default: return false;
    }
}

}  // namespace scfd
