// k_sweep2.cu -- latency-hidden LU-SGS sweeps for compile-time species counts.
//
// Same schedule and arithmetic as k_lusgs.cu (warp per 32-row strip, lane per
// row, lane l at step t on column t-l, matrix-free split Jacobians), restating
// LU-SGS/{2d,q2d}/time_lusgs_viscous.f90 and NR/{2d,q2d}/time_NR_viscous.f90:30-108.
// The wavefront is latency-bound, so the per-cell inputs of the step that is
// PF-1 steps ahead are fetched with cp.async into a per-warp shared-memory
// ring while the current cell is computed; the strip-to-strip hand-off is read
// 8 columns at a time into shared memory.  One warp per CTA, so strips spread
// over the SMs.
#include "scfd_internal.h"

namespace scfd {

__device__ __forceinline__ int ld_acquire2(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release2(int* p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

constexpr long long kSpinLimit2 = 1ll << 22;

// Gathered inputs of one cell, in ring order.
template <int NY, int DIR>
struct SweepVars {
    static constexpr int D = NY + 3;
    static constexpr int DQ = 0;                // Dq(1:D): right-hand side / forward result
    static constexpr int AL = D;                // alpha
    static constexpr int NUA = D + 1, NUB = D + 2;
    static constexpr int U = D + 3, V = D + 4, G = D + 5, H = D + 6;
    static constexpr int Y = D + 7;             // Y(1:nY)
    static constexpr int DH = Y + NY;           // DHi(1:nY)
    static constexpr int A1 = DH + NY, A2 = A1 + 1, B1 = A1 + 2, B2 = A1 + 3, DSA = A1 + 4, DSB = A1 + 5, AREA = A1 + 6;
    static constexpr int Q = AREA + 1;          // backward only: q(1:D)
    static constexpr int NV = Q + (DIR == 1 ? D : 0);
};

struct SweepSrc {
    long long off[80];  // element offsets of each gathered field from the arena base
};

template <typename RT, int NY, int DIR, int PF>
__global__ void __launch_bounds__(32) k_sweep2(View v, const int2* strips, int nstrips, double* xfer, int* progress,
                                               int* ticket, double* partials, int lusgs_update, long long xstride,
                                               const double* base, SweepSrc src) {
    using SV = SweepVars<NY, DIR>;
    constexpr int D = SV::D;
    constexpr int NV = SV::NV;
    __shared__ double ring[PF][NV][32];
    __shared__ double xin[8][D];
    const int lane = threadIdx.x;
    const long long N = v.ncell;
    const bool q2d = v.dim == SCFD_DIM_Q2D;
    const bool nr = v.scheme == SCFD_SCHEME_NR;
    for (;;) {
        int sid = 0;
        if (lane == 0) sid = atomicAdd(ticket, 1);
        sid = __shfl_sync(0xffffffffu, sid, 0);
        if (sid >= nstrips) break;
        const int2 st = strips[sid];
        const int p = st.x, s = st.y;
        const int ni = v.P.ni[p], nj = v.P.nj[p];
        const int j = DIR == 0 ? 32 * s + 1 + lane : nj - 32 * s - lane;
        const bool rowok = j >= 1 && j <= nj;
        const bool has_prev = s > 0;
        const bool publish = (lane == 31) && rowok && (32 * (s + 1) < nj);
        double* xout = xfer + (long long)sid * xstride;
        const double* xsrc = xfer + (long long)(sid - 1) * xstride;
        int* prog_out = progress + sid;
        const int* prog_in = progress + sid - 1;
        const int nsteps = ni + 31;
        auto issue = [&](int tt) {
            const int cc = tt - lane;
            if (tt < nsteps && rowok && cc >= 0 && cc < ni) {
                const int i = DIR == 0 ? cc + 1 : ni - cc;
                const long long c = cidx(v.P, p, i, j);
                double* dst = &ring[tt % PF][0][lane];
#pragma unroll
                for (int k = 0; k < NV; ++k) cp_async8(dst + k * 32, base + src.off[k] + c);
            }
            cp_async_commit();
        };
#pragma unroll
        for (int tt = 0; tt < PF - 1; ++tt) issue(tt);
        RT outA[D], outB[D];
#pragma unroll
        for (int k = 0; k < D; ++k) { outA[k] = RT(0); outB[k] = RT(0); }
        double res = 0.0, omega = 1e300;
        bool omega_fail = false;
        for (int t = 0; t < nsteps; ++t) {
            issue(t + PF - 1);
            // hand-off from the previous strip, 8 columns at a time
            if (has_prev && (t & 7) == 0 && t < ni) {
                const int need = t + 8 < ni ? t + 8 : ni;
                if (lane == 0) {
                    long long spins = 0;
                    while (ld_acquire2(prog_in) < need) {
                        if (++spins > kSpinLimit2 || v.sc->spin_abort) {
                            atomicExch(&v.sc->spin_abort, 1ull);
                            atomicMax(&v.sc->status, SCFD_E_SPIN);
                            break;
                        }
                    }
                }
                __syncwarp();
                for (int e = lane; e < 8 * D; e += 32) {
                    const int col = t + e / D;
                    if (col < ni) (&xin[0][0])[e] = __ldcg(xsrc + (long long)t * D + e);
                }
                __syncwarp();
            }
            RT inB[D];
#pragma unroll
            for (int k = 0; k < D; ++k) inB[k] = __shfl_up_sync(0xffffffffu, outB[k], 1);
            if (lane == 0) {
#pragma unroll
                for (int k = 0; k < D; ++k) inB[k] = (has_prev && t < ni) ? RT(xin[t & 7][k]) : RT(0);
            }
            cp_async_wait<PF - 1>();
            const int cc = t - lane;
            if (rowok && cc >= 0 && cc < ni) {
                const double* r = &ring[t % PF][0][lane];
                auto g = [&](int k) { return r[k * 32]; };
                if (cc == 0) {
#pragma unroll
                    for (int k = 0; k < D; ++k) outA[k] = RT(0);
                }
                const RT al = RT(g(SV::AL));
                RT x[D];
#pragma unroll
                for (int k = 0; k < D; ++k) {
                    const RT rk = RT(g(SV::DQ + k));
                    x[k] = DIR == 0 ? al * (rk + (outA[k] + inB[k])) : rk - al * (outA[k] + inB[k]);
                }
                const RT u = RT(g(SV::U)), vv = RT(g(SV::V)), H = RT(g(SV::H));
                const RT g1 = RT(g(SV::G)) - RT(1);
                const RT hvs = RT(0.5) * g1 * (u * u + vv * vv);
                RT Y[NY], DH[NY];
#pragma unroll
                for (int k = 0; k < NY; ++k) {
                    Y[k] = RT(g(SV::Y + k));
                    DH[k] = RT(g(SV::DH + k));
                }
                if (DIR == 0 && q2d) {
                    RT tmp = RT(0);
#pragma unroll
                    for (int l = 0; l < NY; ++l) tmp = tmp + x[l] * (hvs + DH[l]);
                    tmp = tmp + x[NY] * (-g1 * u);
                    tmp = tmp + x[NY + 2] * g1;
                    const RT aA = al * RT(g(SV::AREA));
                    tmp = x[NY + 1] + aA * tmp;
                    x[NY + 1] = tmp / (RT(1) - aA * (-g1 * vv));
                }
                // matrix-free dsa*A(+/-)x and dsb*B(+/-)x
                RT S = RT(0), P = RT(0);
#pragma unroll
                for (int k = 0; k < NY; ++k) {
                    S += x[k];
                    P += (hvs + DH[k]) * x[k];
                }
                const RT xmx = x[NY], xmy = x[NY + 1], xE = x[NY + 2];
                P += -g1 * u * xmx - g1 * vv * xmy + g1 * xE;
#pragma unroll
                for (int dirn = 0; dirn < 2; ++dirn) {
                    const RT n1 = RT(g(dirn == 0 ? SV::A1 : SV::B1)), n2 = RT(g(dirn == 0 ? SV::A2 : SV::B2));
                    const RT nu = RT(g(dirn == 0 ? SV::NUA : SV::NUB));
                    const RT f = RT(0.5) * RT(g(dirn == 0 ? SV::DSA : SV::DSB));
                    const RT un = n1 * u + n2 * vv;
                    const RT base_ = n1 * xmx + n2 * xmy - un * S;
                    const RT lam = DIR == 0 ? un + nu : un - nu;
                    RT* o = dirn == 0 ? outA : outB;
#pragma unroll
                    for (int k = 0; k < NY; ++k) o[k] = f * (Y[k] * base_ + lam * x[k]);
                    o[NY] = f * (u * base_ + lam * xmx + n1 * P);
                    o[NY + 1] = f * (vv * base_ + lam * xmy + n2 * P);
                    o[NY + 2] = f * (H * base_ + lam * xE + un * P);
                }
                const int i = DIR == 0 ? cc + 1 : ni - cc;
                const long long c = cidx(v.P, p, i, j);
                if (DIR == 0 || nr || !lusgs_update) {
#pragma unroll
                    for (int k = 0; k < D; ++k) v.Dq[k * N + c] = double(x[k]);
                }
                if (DIR == 1) {
                    if (nr) {
                        const double dE = double(x[NY + 2]);
                        res = res + dE * dE;
#pragma unroll
                        for (int k = 0; k < NY; ++k) {
                            const double dk = double(x[k]);
                            if (dk < 0.0) {
                                omega = fmin(omega, -g(SV::Q + k) / dk * v.dq_max);
                                if (omega < v.omega_min) omega_fail = true;
                            }
                        }
                    } else if (lusgs_update) {
#pragma unroll
                        for (int k = 0; k < D; ++k) v.q[k * N + c] = g(SV::Q + k) + double(x[k]);
                    }
                }
                if (publish) {
#pragma unroll
                    for (int k = 0; k < D; ++k) xout[(long long)cc * D + k] = double(outB[k]);
                    if ((cc & 7) == 7 || cc == ni - 1) st_release2(prog_out, cc + 1);
                }
            }
        }
        cp_async_wait<0>();
        __syncwarp();
        if (DIR == 1 && nr) {
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

template <int NY, int DIR>
static SweepSrc make_src(const View& v, const double* base) {
    using SV = SweepVars<NY, DIR>;
    constexpr int D = SV::D;
    SweepSrc s{};
    const long long N = v.ncell;
    auto o = [&](const double* p) { return (long long)(p - base); };
    for (int k = 0; k < D; ++k) s.off[SV::DQ + k] = o(v.Dq) + k * N;
    s.off[SV::AL] = o(v.alpha);
    s.off[SV::NUA] = o(v.nuA);
    s.off[SV::NUB] = o(v.nuB);
    s.off[SV::U] = o(v.w) + 1 * N;
    s.off[SV::V] = o(v.w) + 2 * N;
    s.off[SV::G] = o(v.w) + (D + 1) * N;
    s.off[SV::H] = o(v.w) + (D + 2) * N;
    for (int k = 0; k < NY; ++k) {
        s.off[SV::Y + k] = o(v.w) + (4 + k) * N;
        s.off[SV::DH + k] = o(v.DHi) + k * N;
    }
    s.off[SV::A1] = o(v.vnci);
    s.off[SV::A2] = o(v.vnci) + N;
    s.off[SV::B1] = o(v.vncj);
    s.off[SV::B2] = o(v.vncj) + N;
    s.off[SV::DSA] = o(v.dsci);
    s.off[SV::DSB] = o(v.dscj);
    s.off[SV::AREA] = o(v.Area);
    if (DIR == 1)
        for (int k = 0; k < D; ++k) s.off[SV::Q + k] = o(v.q) + k * N;
    return s;
}

template <typename RT, int NY, int DIR>
static void launch2(const View& v, cudaStream_t s, const int2* strips, int n, double* xfer, int* prog, int* ticket,
                    double* partials, int upd) {
    // deepest ring that fits the 48 KB of static shared memory
    constexpr int NV = SweepVars<NY, DIR>::NV;
    constexpr int PF = (4 * NV * 32 * 8 + 8 * (NY + 3) * 8 <= 48 * 1024) ? 4 : 3;
    int nimax = 0;
    for (int p = 0; p < v.P.np; ++p) nimax = v.P.ni[p] > nimax ? v.P.ni[p] : nimax;
    const double* base = v.base;
    const SweepSrc src = make_src<NY, DIR>(v, base);
    k_sweep2<RT, NY, DIR, PF><<<n, 32, 0, s>>>(v, strips, n, xfer, prog, ticket, partials, upd,
                                               (long long)nimax * (NY + 3), base, src);
}

// true when a specialised kernel exists for this species count
bool launch_sweep2(const View& v, cudaStream_t s, int dir, const int2* strips, int n, double* xfer, int* prog,
                   int* ticket, double* partials, int upd) {
    const bool mixed = v.precision == SCFD_PREC_MIXED;
#define SCFD_SW(NYV)                                                                           \
    if (v.nY == NYV) {                                                                         \
        if (dir == 0) {                                                                        \
            if (mixed) launch2<float, NYV, 0>(v, s, strips, n, xfer, prog, ticket, partials, upd); \
            else launch2<double, NYV, 0>(v, s, strips, n, xfer, prog, ticket, partials, upd);      \
        } else {                                                                               \
            if (mixed) launch2<float, NYV, 1>(v, s, strips, n, xfer, prog, ticket, partials, upd); \
            else launch2<double, NYV, 1>(v, s, strips, n, xfer, prog, ticket, partials, upd);      \
        }                                                                                      \
        return true;                                                                           \
    }
    SCFD_SW(1)
    SCFD_SW(8)
    SCFD_SW(9)
#undef SCFD_SW
    return false;
}

}  // namespace scfd
