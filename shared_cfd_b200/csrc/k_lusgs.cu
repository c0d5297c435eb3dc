// k_lusgs.cu -- LU-SGS forward / backward sweeps and the NR relaxation update.
//
// Restates calc_next_step_implicit of store/time_scheme/LU-SGS/{2d,q2d}/time_lusgs_viscous.f90
// and NR/{2d,q2d}/time_NR_viscous.f90:30-108 with the split Jacobians of
// set_ABpm (sch_lusgs.raw.f90:43-132, NR/q2d/sch_NR.raw.f90:43-140).
//
// Schedule.  The reference walks hyperplanes i+j = const.  Here one warp owns a
// strip of 32 rows (one row per lane) and walks the columns; lane l lags lane
// l-1 by one step, so at step t lane l updates column t-l.  The i-1 neighbour
// is the lane's own previous cell (registers) and the j-1 neighbour is lane l-1
// one step earlier (__shfl_up).  Strip s+1 gets the top row of strip s through
// a global buffer and a progress counter (st.release / ld.acquire, bounded
// spin).  Every cell still sees exactly the neighbour values of the reference's
// dependency order; only cells of one hyperplane may run in another order,
// which the reference leaves to OpenMP anyway.
//
// Jacobians.  A+ x, B+ x, A- x, B- x are formed matrix-free in O(D) from the
// cell state instead of reading four dense D x D matrices (4.6 KB per cell at
// nY = 9):  with n the cell normal, un = n.u, S = sum of species components,
// nm = n1 x_mx + n2 x_my and P = dpdq . x,
//   (n1 A + n2 B) x = [Y_l; u; v; H] (nm - un S) + un x + [0; n1 P; n2 P; un P],
// and A(+/-) x = ((n1 A + n2 B) x +/- nu x) / 2.  This equals the reference's
// matmul up to rounding.
#include "scfd_internal.h"

namespace scfd {

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// bounded wait: 2^22 polls (of the order of a second) before giving up
constexpr long long kSpinLimit = 1ll << 22;

template <typename RT>
struct CellJ {
    RT u, v, H, g1, hvs;  // hvs = 0.5*g1*(u^2+v^2)
    RT nuA, nuB, a1, a2, b1, b2, dsa, dsb;
};

// Outputs dsa * (A(+/-) x) and dsb * (B(+/-) x).
template <typename RT, int D, bool PLUS>
__device__ __forceinline__ void jac_out(int nY, const CellJ<RT>& cj, const RT* Y, const RT* DH, const RT* x, RT* oa,
                                        RT* ob) {
    RT S = RT(0), P = RT(0);
    for (int k = 0; k < nY; ++k) {
        S += x[k];
        P += (cj.hvs + DH[k]) * x[k];
    }
    const RT xmx = x[nY], xmy = x[nY + 1], xE = x[nY + 2];
    P += -cj.g1 * cj.u * xmx - cj.g1 * cj.v * xmy + cj.g1 * xE;
    const RT half = RT(0.5);
    {
        const RT un = cj.a1 * cj.u + cj.a2 * cj.v;
        const RT nm = cj.a1 * xmx + cj.a2 * xmy;
        const RT base = nm - un * S;
        const RT lam = PLUS ? un + cj.nuA : un - cj.nuA;
        const RT f = half * cj.dsa;
        for (int k = 0; k < nY; ++k) oa[k] = f * (Y[k] * base + lam * x[k]);
        oa[nY] = f * (cj.u * base + lam * xmx + cj.a1 * P);
        oa[nY + 1] = f * (cj.v * base + lam * xmy + cj.a2 * P);
        oa[nY + 2] = f * (cj.H * base + lam * xE + un * P);
    }
    {
        const RT un = cj.b1 * cj.u + cj.b2 * cj.v;
        const RT nm = cj.b1 * xmx + cj.b2 * xmy;
        const RT base = nm - un * S;
        const RT lam = PLUS ? un + cj.nuB : un - cj.nuB;
        const RT f = half * cj.dsb;
        for (int k = 0; k < nY; ++k) ob[k] = f * (Y[k] * base + lam * x[k]);
        ob[nY] = f * (cj.u * base + lam * xmx + cj.b1 * P);
        ob[nY + 1] = f * (cj.v * base + lam * xmy + cj.b2 * P);
        ob[nY + 2] = f * (cj.H * base + lam * xE + un * P);
    }
}

// The preconditioned dual time (dual/2d/sch_dual.raw.f90:156-209): the split
// Jacobians are (I + s2 p1 p2^T)(n1 A + n2 B)/2 +/- nu/2 with p1 = (Y, u, v, H)
// and p2 . x = P(x) of the cell (pre1, pre2), so with z = (n1 A + n2 B) x
// formed as above, A(+/-) x = (z + s2 P(z) p1 +/- nu x) / 2.
template <typename RT>
__device__ __forceinline__ RT pfun(int nY, const CellJ<RT>& cj, const RT* DH, const RT* x) {
    RT P = RT(0);
    for (int k = 0; k < nY; ++k) P += (cj.hvs + DH[k]) * x[k];
    return P - cj.g1 * cj.u * x[nY] - cj.g1 * cj.v * x[nY + 1] + cj.g1 * x[nY + 2];
}

template <typename RT, int D, bool PLUS>
__device__ __forceinline__ void jac_out_dual(int nY, const CellJ<RT>& cj, RT s2, const RT* Y, const RT* DH,
                                             const RT* x, RT* oa, RT* ob) {
    RT S = RT(0);
    for (int k = 0; k < nY; ++k) S += x[k];
    const RT P = pfun(nY, cj, DH, x);
    const RT xmx = x[nY], xmy = x[nY + 1], xE = x[nY + 2];
    const RT half = RT(0.5);
    for (int dir = 0; dir < 2; ++dir) {
        const RT n1 = dir == 0 ? cj.a1 : cj.b1, n2 = dir == 0 ? cj.a2 : cj.b2;
        const RT nu = dir == 0 ? cj.nuA : cj.nuB, f = half * (dir == 0 ? cj.dsa : cj.dsb);
        RT* o = dir == 0 ? oa : ob;
        const RT un = n1 * cj.u + n2 * cj.v;
        const RT base = n1 * xmx + n2 * xmy - un * S;
        RT z[D];
        for (int k = 0; k < nY; ++k) z[k] = Y[k] * base + un * x[k];
        z[nY] = cj.u * base + un * xmx + n1 * P;
        z[nY + 1] = cj.v * base + un * xmy + n2 * P;
        z[nY + 2] = cj.H * base + un * xE + un * P;
        const RT g = s2 * pfun(nY, cj, DH, z);
        const RT lam = PLUS ? nu : -nu;
        for (int k = 0; k < nY; ++k) o[k] = f * (z[k] + g * Y[k] + lam * x[k]);
        o[nY] = f * (z[nY] + g * cj.u + lam * xmx);
        o[nY + 1] = f * (z[nY + 1] + g * cj.v + lam * xmy);
        o[nY + 2] = f * (z[nY + 2] + g * cj.H + lam * xE);
    }
}

// x += s * P(x) * p1
template <typename RT>
__device__ __forceinline__ void dual_rank1(int nY, const CellJ<RT>& cj, RT s, const RT* Y, const RT* DH, RT* x) {
    const RT g = s * pfun(nY, cj, DH, x);
    for (int k = 0; k < nY; ++k) x[k] += g * Y[k];
    x[nY] += g * cj.u;
    x[nY + 1] += g * cj.v;
    x[nY + 2] += g * cj.H;
}

struct StripList {
    const int2* strips;  // (plane, strip index in plane)
    int n;
};

// DIR 0: forward (L sweep), DIR 1: backward (U sweep).  D is the compile-time
// bound of dimq (registers); nY is the runtime species count.
template <typename RT, int DMAX, int DIR>
__global__ void __launch_bounds__(128) k_sweep(View v, StripList sl, double* xfer, int* progress, int* ticket,
                                               double* partials, int lusgs_update, long long xstride) {
    const int lane = threadIdx.x & 31;
    const int nY = v.nY, D = v.D;
    const long long N = v.ncell;
    const bool q2d = v.dim == SCFD_DIM_Q2D;
    const bool nr = dual_time_scheme(v.scheme);
    const bool dual = v.scheme == SCFD_SCHEME_DUAL;
    // precon / preconLU-SGS: the split Jacobians are (I + phh p1 p2^T)(n1 A + n2 B)/2
    // +/- nu/2 (sch_precon.raw.f90:148-186), the product of jac_out_dual with s2 = phh
    const bool pc = precon_scheme(v.scheme);
    for (;;) {
        int sid = 0;
        if (lane == 0) sid = atomicAdd(ticket, 1);
        sid = __shfl_sync(0xffffffffu, sid, 0);
        if (sid >= sl.n) break;
        const int2 st = sl.strips[sid];
        const int p = st.x, s = st.y;
        const int ni = v.P.ni[p], nj = v.P.nj[p];
        const int j = DIR == 0 ? 32 * s + 1 + lane : nj - 32 * s - lane;
        const bool rowok = j >= 1 && j <= nj;
        const bool has_prev = s > 0;
        // the top lane publishes when a next strip exists in this plane
        const bool publish = (lane == 31) && rowok && (32 * (s + 1) < nj);
        double* xout = xfer + (long long)sid * xstride;       // this strip's top row
        const double* xin = xfer + (long long)(sid - 1) * xstride;
        int* prog_out = progress + sid;
        const int* prog_in = progress + sid - 1;
        int seen = 0;
        RT outA[DMAX], outB[DMAX], x[DMAX];
#pragma unroll
        for (int k = 0; k < DMAX; ++k) { outA[k] = RT(0); outB[k] = RT(0); }
        double res = 0.0, omega = 1e300;
        bool omega_fail = false;
        for (int t = 0; t < ni + 31; ++t) {
            const int cc = t - lane;
            const bool act = rowok && cc >= 0 && cc < ni;
            // neighbour across the strip row direction: lane-1 one step earlier
            RT inB[DMAX];
#pragma unroll
            for (int k = 0; k < DMAX; ++k) inB[k] = __shfl_up_sync(0xffffffffu, outB[k], 1);
            if (lane == 0) {
                if (has_prev && act) {
                    if (seen <= cc) {
                        long long spins = 0;
                        for (;;) {
                            seen = ld_acquire(prog_in);
                            if (seen > cc) break;
                            if (++spins > kSpinLimit || v.sc->spin_abort) {
                                atomicExch(&v.sc->spin_abort, 1ull);
                                atomicMax(&v.sc->status, SCFD_E_SPIN);
                                seen = ni;  // give up: read whatever is there
                                break;
                            }
                        }
                    }
#pragma unroll
                    for (int k = 0; k < DMAX; ++k) inB[k] = k < D ? RT(__ldcg(xin + (long long)cc * D + k)) : RT(0);
                } else {
#pragma unroll
                    for (int k = 0; k < DMAX; ++k) inB[k] = RT(0);
                }
            }
            if (act) {
                const int i = DIR == 0 ? cc + 1 : ni - cc;
                const long long c = cidx(v.P, p, i, j);
                const RT al = RT(v.alpha[c]);
                if (cc == 0) {
#pragma unroll
                    for (int k = 0; k < DMAX; ++k) outA[k] = RT(0);
                }
                CellJ<RT> cj;
                cj.u = RT(v.w[N + c]);
                cj.v = RT(v.w[2 * N + c]);
                cj.H = RT(v.w[(D + 2) * N + c]);
                cj.g1 = RT(v.w[(D + 1) * N + c]) - RT(1);
                cj.hvs = RT(0.5) * cj.g1 * (cj.u * cj.u + cj.v * cj.v);
                RT Y[DMAX], DH[DMAX];
#pragma unroll
                for (int k = 0; k < DMAX; ++k)
                    if (k < nY) {
                        Y[k] = RT(v.w[(4 + k) * N + c]);
                        DH[k] = RT(v.DHi[k * N + c]);
                    }
                RT s1 = RT(1), s2 = RT(0), s4 = RT(0);
                if (dual) {
                    s1 = RT(v.pre[c]);
                    s2 = RT(v.pre[N + c]);
                    s4 = RT(v.pre[3 * N + c]);
                }
                RT rv[DMAX];
#pragma unroll
                for (int k = 0; k < DMAX; ++k) rv[k] = k < D ? RT(v.Dq[k * N + c]) : RT(0);
                if (DIR == 1 && dual) {
                    // second step of time_dual_viscous.f90:62-68 (S): Dq += s3 P(Dq) p1, Dq *= s1
                    dual_rank1(nY, cj, RT(v.pre[2 * N + c]), Y, DH, rv);
#pragma unroll
                    for (int k = 0; k < DMAX; ++k) rv[k] = s1 * rv[k];
                }
#pragma unroll
                for (int k = 0; k < DMAX; ++k)
                    if (k < D) x[k] = DIR == 0 ? al * (rv[k] + (outA[k] + inB[k])) : rv[k] - al * (outA[k] + inB[k]);
                if (dual) {
                    // S^-1 after each sweep (time_dual_viscous.f90:50-51, 84-85)
                    dual_rank1(nY, cj, s4, Y, DH, x);
#pragma unroll
                    for (int k = 0; k < DMAX; ++k) x[k] = RT(1) / s1 * x[k];
                }
                if (DIR == 0 && q2d) {
                    // semi-implicit axisymmetric pressure source (q2d time_lusgs_viscous.f90:38-44)
                    RT tmp = RT(0);
                    for (int l = 0; l <= nY; ++l) {
                        const RT dp = l < nY ? cj.hvs + DH[l] : -cj.g1 * cj.u;
                        tmp = tmp + x[l] * dp;
                    }
                    tmp = tmp + x[nY + 2] * cj.g1;
                    const RT aA = al * RT(v.Area[c]);
                    tmp = x[nY + 1] + aA * tmp;
                    x[nY + 1] = tmp / (RT(1) - aA * (-cj.g1 * cj.v));
                }
                cj.nuA = RT(v.nuA[c]);
                cj.nuB = RT(v.nuB[c]);
                cj.a1 = RT(v.vnci[c]); cj.a2 = RT(v.vnci[N + c]);
                cj.b1 = RT(v.vncj[c]); cj.b2 = RT(v.vncj[N + c]);
                cj.dsa = RT(v.dsci[c]); cj.dsb = RT(v.dscj[c]);
                if (dual)
                    jac_out_dual<RT, DMAX, DIR == 0>(nY, cj, s2, Y, DH, x, outA, outB);
                else if (pc)
                    jac_out_dual<RT, DMAX, DIR == 0>(nY, cj, RT(v.pre[c]), Y, DH, x, outA, outB);
                else
                    jac_out<RT, DMAX, DIR == 0>(nY, cj, Y, DH, x, outA, outB);
                if (DIR == 0 || nr || !lusgs_update) {
                    for (int k = 0; k < D; ++k) v.Dq[k * N + c] = double(x[k]);
                }
                if (DIR == 1) {
                    if (nr) {
                        const double dE = double(x[nY + 2]);
                        res = res + dE * dE;
                        for (int k = 0; k < nY; ++k) {
                            const double dk = double(x[k]);
                            if (dk < 0.0) {
                                omega = fmin(omega, -v.q[k * N + c] / dk * v.dq_max);
                                if (omega < v.omega_min) omega_fail = true;
                            }
                        }
                    } else if (lusgs_update) {
                        for (int k = 0; k < D; ++k) v.q[k * N + c] = v.q[k * N + c] + double(x[k]);
                    }
                }
                if (publish) {
                    for (int k = 0; k < D; ++k) xout[(long long)cc * D + k] = double(outB[k]);
                    if ((cc & 7) == 7 || cc == ni - 1) st_release(prog_out, cc + 1);
                }
            }
        }
        if (DIR == 1 && nr) {
            // deterministic warp reduction (fixed butterfly order)
            for (int o = 16; o > 0; o >>= 1) {
                res += __shfl_xor_sync(0xffffffffu, res, o);
                omega = fmin(omega, __shfl_xor_sync(0xffffffffu, omega, o));
            }
            const unsigned fail = __ballot_sync(0xffffffffu, omega_fail);
            if (lane == 0) {
                partials[2 * sid] = res;
                partials[2 * sid + 1] = omega;
                if (fail) atomicMax(&v.sc->status, SCFD_E_OMEGA);
            }
        }
    }
}

template <typename RT, int DMAX>
static void launch_dir(const View& v, cudaStream_t s, int dir, StripList sl, double* xfer, int* prog, int* ticket,
                       double* partials, int upd) {
    const int warps = sl.n < 4 ? sl.n : 4;
    const int blocks = (sl.n + warps - 1) / warps;
    int nimax = 0;
    for (int p = 0; p < v.P.np; ++p) nimax = v.P.ni[p] > nimax ? v.P.ni[p] : nimax;
    const long long xs = (long long)nimax * v.D;
    if (dir == 0)
        k_sweep<RT, DMAX, 0><<<blocks, 32 * warps, 0, s>>>(v, sl, xfer, prog, ticket, partials, upd, xs);
    else
        k_sweep<RT, DMAX, 1><<<blocks, 32 * warps, 0, s>>>(v, sl, xfer, prog, ticket, partials, upd, xs);
}

template <typename RT>
static void launch_rt(const View& v, cudaStream_t s, int dir, StripList sl, double* xfer, int* prog, int* ticket,
                      double* partials, int upd) {
    if (v.D <= 4)
        launch_dir<RT, 4>(v, s, dir, sl, xfer, prog, ticket, partials, upd);
    else if (v.D <= 8)
        launch_dir<RT, 8>(v, s, dir, sl, xfer, prog, ticket, partials, upd);
    else if (v.D <= 12)
        launch_dir<RT, 12>(v, s, dir, sl, xfer, prog, ticket, partials, upd);
    else if (v.D <= 16)
        launch_dir<RT, 16>(v, s, dir, sl, xfer, prog, ticket, partials, upd);
    else
        launch_dir<RT, 35>(v, s, dir, sl, xfer, prog, ticket, partials, upd);
}

int launch_sweep_reset(cudaStream_t s, int* progress, int* tickets, int nstrips_fwd, int nstrips_bwd) {
    // progress[0..nf) forward, progress[nf..nf+nb) backward; tickets[0], tickets[1]
    cudaMemsetAsync(progress, 0, sizeof(int) * (nstrips_fwd + nstrips_bwd), s);
    cudaMemsetAsync(tickets, 0, sizeof(int) * 2, s);
    return 0;
}

int launch_sweep(const View& v, cudaStream_t s, int dir, double* xfer, int* progress, double* partials, int* tickets,
                 int nstrips_fwd, int nstrips_bwd, const int* strip_tab_f, const int* strip_tab_b) {
    StripList f{(const int2*)strip_tab_f, nstrips_fwd}, b{(const int2*)strip_tab_b, nstrips_bwd};
    const bool mixed = v.precision == SCFD_PREC_MIXED;
    const int upd = dual_time_scheme(v.scheme) ? 0 : 1;
    const bool dual = v.scheme == SCFD_SCHEME_DUAL || precon_scheme(v.scheme);  // generic sweeps only
    if (!dual && dir == 0 && launch_sweep2(v, s, 0, f.strips, f.n, xfer, progress, tickets, partials, upd)) return 1;
    if (!dual && dir == 1 &&
        launch_sweep2(v, s, 1, b.strips, b.n, xfer, progress + nstrips_fwd, tickets + 1, partials, upd))
        return 1;
    if (dir == 0) {
        if (mixed) launch_rt<float>(v, s, 0, f, xfer, progress, tickets, partials, upd);
        else launch_rt<double>(v, s, 0, f, xfer, progress, tickets, partials, upd);
    } else {
        if (mixed) launch_rt<float>(v, s, 1, b, xfer, progress + nstrips_fwd, tickets + 1, partials, upd);
        else launch_rt<double>(v, s, 1, b, xfer, progress + nstrips_fwd, tickets + 1, partials, upd);
    }
    return 1;
}

// NR: global omega / res from the per-strip partials (fixed order), then
// q += omega*Dq (time_NR_viscous.f90:86-108).  Every CTA reduces the partials
// itself; CTA 0 also records the scalars.
__global__ void k_nr_update(View v, const double* partials, int nstrips, int inner) {
    __shared__ double s_omega;
    if (threadIdx.x == 0) {
        double res = 0.0, om = 1e300;
        for (int k = 0; k < nstrips; ++k) {
            res += partials[2 * k];
            om = fmin(om, partials[2 * k + 1]);
        }
        const double omf = fmin(v.omega_max, om);
        s_omega = omf;
        if (blockIdx.x == 0 && blockIdx.y == 0) {
            if (inner == 1) v.sc->res1 = res;
            v.sc->res = res;
            v.sc->omega = omf;
            log_inner(v.sc, inner, om, res);
        }
    }
    __syncthreads();
    if (v.sc->status == SCFD_E_OMEGA) return;
    const double om = s_omega;
    const int p = v.P.act[blockIdx.y];
    const int ni = v.P.ni[p], nj = v.P.nj[p];
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= ni * nj) return;
    const int i = idx % ni + 1, j = idx / ni + 1;
    const long long c = cidx(v.P, p, i, j);
    const long long N = v.ncell;
    for (int k = 0; k < v.D; ++k) v.q[k * N + c] = v.q[k * N + c] + om * v.Dq[k * N + c];
}

int launch_nr_update(const View& v, cudaStream_t s, const double* partials, int nstrips, int inner) {
    int mx = 0;
    for (int a = 0; a < v.P.nact; ++a) {
        const int p = v.P.act[a];
        mx = v.P.ni[p] * v.P.nj[p] > mx ? v.P.ni[p] * v.P.nj[p] : mx;
    }
    if (v.P.nact == 0) return 0;
    dim3 grid((mx + 255) / 256, v.P.nact);
    k_nr_update<<<grid, 256, 0, s>>>(v, partials, nstrips, inner);
    return 1;
}

}  // namespace scfd
