// k_sweep3.cu -- LU-SGS sweeps over TMA-streamed strip records.
//
// Restates calc_next_step_implicit of store/time_scheme/LU-SGS/{2d,q2d}/time_lusgs_viscous.f90
// and NR/{2d,q2d}/time_NR_viscous.f90:30-108 with the split Jacobians of set_ABpm
// (sch_lusgs.raw.f90:1-141, NR/q2d/sch_NR.raw.f90:1-149), applied matrix-free.
//
// Schedule (as k_lusgs.cu): one warp per 32-row strip, lane l on row 32s+1+l,
// at step t lane l updates column t-l; the i-1 neighbour is in registers, the
// j-1 neighbour comes from lane l-1 by __shfl_up, strip s+1 reads the top row of
// strip s through a global buffer with release/acquire progress counters.
//
// Data path.  The wavefront is latency-bound and its per-lane accesses hit 32
// different rows, so the inputs are first repacked (k_pack, coalesced through a
// shared-memory transpose) into a "strip record" layout
//     rec[strip][step t][field f][lane l]   (cell (i = t - l + 1, j = 32 s + 1 + l)),
// which makes every step of every strip one contiguous block of NF*32 values.
// The sweep streams those blocks, SPB steps per cp.async.bulk (TMA) copy, into a
// shared-memory ring of PFB copies (mbarrier completion), and writes its
// results back into the same block, contiguously.  The backward sweep reads the
// same records with steps and lanes reversed (step ni+30-t, lane 31-l).
// k_unpack applies q += omega*Dq back in the cell layout.
#include "async_ptx.h"
#include "scfd_internal.h"

namespace scfd {

using namespace ptx;

namespace {

constexpr long long kSpin3 = 1ll << 22;

// sum of a[B..E) as a balanced pairwise tree (short dependency chain)
template <int B, int E, typename T>
__device__ __forceinline__ T tree_sum(const T* a) {
    if constexpr (E - B == 1) {
        return a[B];
    } else {
        constexpr int M = (B + E) / 2;
        return tree_sum<B, M>(a) + tree_sum<M, E>(a);
    }
}
// record steps per bulk copy (FP64 records are twice as large: half as many
// steps, so that the ring of PFB copies fits in shared memory)
template <typename RT>
struct Spb {
    static constexpr int value = sizeof(RT) == 4 ? 8 : 4;
};
constexpr int SPB_MAX = 8;
constexpr int PFB = 3;  // bulk copies in the ring, PFB - 1 of them ahead of the sweep

}  // namespace

// Record fields (one cell):
//   x(1:D)        right-hand side; forward result; final Dq
//   al            alpha = 1/(Vol/dt + dsci nuA + dscj nuB)   (NR: 3 Vol/(2 dt))
//   aA, rq        alpha*Area and 1/(1 - alpha*Area*dpdq_my)  (q2d pressure source)
//   dp(1:D)       dpdq: species 0.5 g1 |u|^2 + DHi, then -g1 u, -g1 v, g1
//   cv(1:D)       Y(1:nY), u, v, H
//   per direction (A: vnci/dsci/nuA, B: vncj/dscj/nuB): f = ds/2, n1, n2, un, nu
//   qs(1:nY)      q species (NR positivity limiter)
template <int NY>
struct Rec {
    static constexpr int D = NY + 3;
    static constexpr int X = 0, AL = D, AA = D + 1, RQ = D + 2, DP = D + 3, CV = 2 * D + 3;
    static constexpr int FA = 3 * D + 3, N1A = FA + 1, N2A = FA + 2, UNA = FA + 3, NUA = FA + 4;
    static constexpr int FB = FA + 5, N1B = FB + 1, N2B = FB + 2, UNB = FB + 3, NUB = FB + 4;
    static constexpr int QS = FB + 5;
    static constexpr int NF = QS + NY;
};
// Block of one step: groups of G consecutive fields per lane, so a lane reads
// its cell with 16-byte loads: rec[step][group][lane][G].
template <typename T, int NY>
struct RecLayout {
    static constexpr int G = 16 / (int)sizeof(T);
    static constexpr int NF = Rec<NY>::NF;
    static constexpr int NG = (NF + G - 1) / G;
    static constexpr int STEP = NG * 32 * G;  // elements per step block
};

template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
    using type = float4;
};
template <>
struct Vec16<double> {
    using type = double2;
};

// strip table entry: plane, strip index in plane, index of the strip in the
// forward list (its record), unused
struct StripRec {
    const int4* tab;
    const long long* rec_off;  // per forward strip: first element of its records
    int n;
};

// ---------------------------------------------------------------------------
// k_pack: cell layout -> strip records (32 steps x 32 lanes of one strip per
// block; reads coalesced along i, writes coalesced 16-byte groups through a
// shared-memory transpose).  Forms alpha, the spectral radii and dpdq of
// set_ABpm (sch_lusgs.raw.f90:27-50,134-136; NR/q2d/sch_NR.raw.f90:43-50,143-144).
// ---------------------------------------------------------------------------
template <typename T, int NY>
__global__ void __launch_bounds__(1024) k_pack(View v, const int2* blk, const int4* strips, const long long* rec_off,
                                               T* rec, int nr_mode) {
    using R = Rec<NY>;
    using L = RecLayout<T, NY>;
    constexpr int D = R::D, G = L::G, NG = L::NG;
    __shared__ T tile[G][32][33];
    const int2 b = blk[blockIdx.x];
    const int4 st = strips[b.x];
    const int p = st.x, s = st.y;
    const int ni = v.P.ni[p], nj = v.P.nj[p];
    const int tt = threadIdx.x, l = threadIdx.y;
    const int t = b.y + tt;
    const int cc = t - l;
    const int i = cc + 1, j = 32 * s + 1 + l;
    const bool ok = cc >= 0 && cc < ni && j <= nj && t < ni + 31;
    const long long N = v.ncell;
    const long long c = ok ? cidx(v.P, p, i, j) : 0;
    double al = 0.0, nuA = 0.0, nuB = 0.0, u = 0.0, vv = 0.0, g1 = 0.0, hvs = 0.0, aA = 0.0, rq = 1.0;
    if (ok) {
        const double* w = v.w;
        const double rho = w[c], pr = w[3 * N + c];
        u = w[N + c];
        vv = w[2 * N + c];
        const double gamm = w[(D + 1) * N + c];
        g1 = gamm - 1.0;
        hvs = 0.5 * g1 * (u * u + vv * vv);
        const double cs = sqrt(gamm * pr / rho);
        nuA = fabs(v.vnci[c] * u + v.vnci[N + c] * vv) + cs;
        nuB = fabs(v.vncj[c] * u + v.vncj[N + c] * vv) + cs;
        const double dsa = v.dsci[c], dsb = v.dscj[c], vol = v.Vol[c];
        const double dtl = v.dt_mode == SCFD_DT_LOCAL ? v.dt_mat[c] : v.sc->dt_grbl;
        const double tmp = nr_mode ? 3.0 * vol / (2.0 * dtl) + dsa * nuA + dsb * nuB : vol / dtl + dsa * nuA + dsb * nuB;
        al = 1.0 / tmp;
        if (v.dim == SCFD_DIM_Q2D) {
            aA = al * v.Area[c];
            rq = 1.0 / (1.0 - aA * (-g1 * vv));
        }
    }
    auto field = [&](int k) -> double {
        if (!ok) return 0.0;
        if (k < R::AL) return v.Dq[(k - R::X) * N + c];
        if (k == R::AL) return al;
        if (k == R::AA) return aA;
        if (k == R::RQ) return rq;
        if (k < R::CV) {
            const int m = k - R::DP;
            if (m < NY) return hvs + v.DHi[m * N + c];
            if (m == NY) return -g1 * u;
            if (m == NY + 1) return -g1 * vv;
            return g1;
        }
        if (k < R::FA) {
            const int m = k - R::CV;
            if (m < NY) return v.w[(4 + m) * N + c];
            if (m == NY) return u;
            if (m == NY + 1) return vv;
            return v.w[(D + 2) * N + c];
        }
        if (k == R::FA) return 0.5 * v.dsci[c];
        if (k == R::N1A) return v.vnci[c];
        if (k == R::N2A) return v.vnci[N + c];
        if (k == R::UNA) return v.vnci[c] * u + v.vnci[N + c] * vv;
        if (k == R::NUA) return nuA;
        if (k == R::FB) return 0.5 * v.dscj[c];
        if (k == R::N1B) return v.vncj[c];
        if (k == R::N2B) return v.vncj[N + c];
        if (k == R::UNB) return v.vncj[c] * u + v.vncj[N + c] * vv;
        if (k == R::NUB) return nuB;
        if (k < R::NF) return v.q[(k - R::QS) * N + c];
        return 0.0;
    };
    T* out = rec + rec_off[b.x] + (long long)b.y * L::STEP;
    const int nt = min(32, ni + 31 - b.y);
    using V = typename Vec16<T>::type;
    // the fields of the next two groups are loaded before this group's barrier
    // and transpose, so that their global loads overlap it
    T cur[G], nxt[G], nx2[G];
#pragma unroll
    for (int e = 0; e < G; ++e) {
        cur[e] = T(field(e));
        nxt[e] = NG > 1 ? T(field(G + e)) : T(0);
    }
#pragma unroll
    for (int g = 0; g < NG; ++g) {
        if (g + 2 < NG) {
#pragma unroll
            for (int e = 0; e < G; ++e) nx2[e] = T(field((g + 2) * G + e));
        }
#pragma unroll
        for (int e = 0; e < G; ++e) tile[e][l][tt] = cur[e];
        __syncthreads();
        const int wl = threadIdx.x, wt = threadIdx.y;
        if (wt < nt) {
            T vals[G];
#pragma unroll
            for (int e = 0; e < G; ++e) vals[e] = tile[e][wl][wt];
            *reinterpret_cast<V*>(out + ((long long)wt * NG + g) * 32 * G + wl * G) = *reinterpret_cast<V*>(vals);
        }
        __syncthreads();
#pragma unroll
        for (int e = 0; e < G; ++e) {
            cur[e] = nxt[e];
            nxt[e] = nx2[e];
        }
    }
}

// ---------------------------------------------------------------------------
// the sweeps
// ---------------------------------------------------------------------------
// Records of one strip hold ni+31 step blocks plus kPad zero blocks before and
// after them, so the step loop runs in unguarded blocks of 8 steps with the
// prefetch reaching past either end.
constexpr int kPad = 8 + SPB_MAX * PFB;

template <typename RT, int NY, int DIR>
__global__ void __launch_bounds__(32) k_sweep3(View v, StripRec sl, RT* rec, double* xfer, long long xstride,
                                               int* progress, int* ticket, double* partials) {
    using R = Rec<NY>;
    using L = RecLayout<RT, NY>;
    using V = typename Vec16<RT>::type;
    constexpr int D = R::D, G = L::G, NG = L::NG, STEP = L::STEP;
    constexpr unsigned BLK = STEP * sizeof(RT);
    constexpr int SPB = Spb<RT>::value;
    static_assert(8 % SPB == 0, "bulk copies must tile the 8-step unroll");
    extern __shared__ __align__(128) unsigned char smraw[];
    RT* ring = reinterpret_cast<RT*>(smraw);                                        // [PFB][SPB][STEP]
    RT* xin = reinterpret_cast<RT*>(smraw + PFB * SPB * BLK);                       // [8][D]
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smraw + PFB * SPB * BLK + 8 * D * sizeof(double));
    const int lane = threadIdx.x;
    const bool nr = v.scheme == SCFD_SCHEME_NR;
    const bool q2d = v.dim == SCFD_DIM_Q2D;
    if (lane == 0) {
        for (int k = 0; k < PFB; ++k) mbar_init(&bar[k], 1);
        mbar_init_fence();
    }
    __syncwarp();
    unsigned phase = 0;  // bit k: parity of the next completion of ring slot k
    unsigned pend = 0;   // ring slots with a copy in flight
    bool bail = false;
    const int lf = DIR == 0 ? lane : 31 - lane;  // this lane's slot in a record block
    const long long gstep = DIR == 0 ? STEP : -STEP;
    for (;;) {
        int sid = 0;
        if (lane == 0) sid = atomicAdd(ticket, 1);
        sid = __shfl_sync(0xffffffffu, sid, 0);
        if (sid >= sl.n || bail) break;
        const int4 st = sl.tab[sid];
        const int p = st.x, s = st.y, fs = st.z;
        const int ni = v.P.ni[p], nj = v.P.nj[p];
        const int nstr = (nj + 31) / 32;
        const bool has_prev = DIR == 0 ? s > 0 : s < nstr - 1;
        const bool publish = lane == 31 && (DIR == 0 ? s < nstr - 1 : s > 0);
        // hand-off columns in the record precision (the values are the sweep's own)
        RT* xout = reinterpret_cast<RT*>(xfer) + (long long)sid * xstride;
        const RT* xsrc = reinterpret_cast<const RT*>(xfer) + (long long)(sid - 1) * xstride;
        int* prog_out = progress + sid;
        const int* prog_in = progress + sid - 1;
        const int nblk8 = (ni + 31 + 7) / 8;
        RT* srec = rec + sl.rec_off[fs];
        // record block of sweep step tt (forward order; the backward sweep walks it back)
        const RT* rd = srec + (DIR == 0 ? 0 : (long long)(ni + 30) * STEP);
        // bulk copy nb holds sweep steps SPB*nb .. SPB*nb+SPB-1; in memory order it
        // starts at the first of them (forward) or the last (backward)
        auto copy_src = [&](int nb) {
            return DIR == 0 ? rd + (long long)nb * SPB * STEP : rd - (long long)(nb * SPB + SPB - 1) * STEP;
        };
        if (lane == 0) {
#pragma unroll
            for (int b = 0; b < PFB - 1; ++b) {
                mbar_expect_tx(&bar[b], SPB * BLK);
                tma_bulk_g2s(ring + b * SPB * STEP, copy_src(b), SPB * BLK, &bar[b]);
            }
        }
        pend |= (1u << (PFB - 1)) - 1u;
        RT outA[D], outB[D];
#pragma unroll
        for (int k = 0; k < D; ++k) { outA[k] = RT(0); outB[k] = RT(0); }
        double res = 0.0;
        // smallest omega candidate q / (-Dq) of the lane.  FP64 keeps it as the pair
        // (q, -Dq), compared by cross-multiplication; FP32 keeps the ratio (fast
        // divide), since species held at the density floor (~1e-37) would
        // underflow an FP32 cross product.
        constexpr bool f32 = sizeof(RT) == 4;
        RT on = RT(__longlong_as_double(0x7FF0000000000000ll)), od = RT(1);
        RT* gblk = const_cast<RT*>(rd) + lf * G;
        for (int tb = 0; tb < nblk8 && !bail; ++tb) {
            const int t0 = tb * 8;
            const bool chunk = has_prev && t0 < ni;
            if (chunk) {
                const int need = t0 + 8 < ni ? t0 + 8 : ni;
                if (lane == 0) {
                    long long spins = 0;
                    while (ld_acquire_gpu(prog_in) < need) {
                        if (++spins > kSpin3 || v.sc->spin_abort) {
                            atomicExch(&v.sc->spin_abort, 1ull);
                            atomicMax(&v.sc->status, SCFD_E_SPIN);
                            break;
                        }
                    }
                }
                __syncwarp();
                for (int e = lane; e < 8 * D; e += 32) xin[e] = __ldcg(xsrc + (long long)t0 * D + e);
                __syncwarp();
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int t = t0 + u;
                const int tq = t / SPB;  // bulk copy holding step t
                const int slot = tq % PFB;
                if (u % SPB == 0) {
                    const int nb = tq + PFB - 1, sl2 = nb % PFB;
                    if (lane == 0) {
                        mbar_expect_tx(&bar[sl2], SPB * BLK);
                        tma_bulk_g2s(ring + sl2 * SPB * STEP, copy_src(nb), SPB * BLK, &bar[sl2]);
                    }
                    pend |= 1u << sl2;
                }
                RT inB[D];
#pragma unroll
                for (int k = 0; k < D; ++k) {
                    const RT sh = __shfl_up_sync(0xffffffffu, outB[k], 1);
                    inB[k] = lane == 0 ? (chunk ? xin[u * D + k] : RT(0)) : sh;
                }
                if (u % SPB == 0) {
                    long long spins = 0;
                    bool ok = true;
                    while (!mbar_try_wait(&bar[slot], (phase >> slot) & 1u)) {
                        if (++spins > kSpin3) {
                            ok = false;
                            break;
                        }
                    }
                    if (!__all_sync(0xffffffffu, ok)) {
                        if (lane == 0) atomicMax(&v.sc->status, SCFD_E_SPIN);
                        bail = true;
                        break;
                    }
                    phase ^= 1u << slot;
                    pend &= ~(1u << slot);
                }
                // this lane's cell: NG 16-byte loads (zero-filled outside the plane)
                RT f[NG * G];
                const int pos = DIR == 0 ? u % SPB : SPB - 1 - u % SPB;
                const V* src = reinterpret_cast<const V*>(ring + (slot * SPB + pos) * STEP) + lf;
#pragma unroll
                for (int g = 0; g < NG; ++g) *reinterpret_cast<V*>(&f[g * G]) = src[g * 32];
                const RT al = f[R::AL];
                RT x[D];
#pragma unroll
                for (int k = 0; k < D; ++k)
                    x[k] = DIR == 0 ? al * (f[R::X + k] + (outA[k] + inB[k])) : f[R::X + k] - al * (outA[k] + inB[k]);
                // P = dpdq.x; forward q2d: semi-implicit pressure source
                // (q2d time_lusgs_viscous.f90:38-44).  Both sums are pairwise trees.
                RT pr[D - 1];
#pragma unroll
                for (int k = 0; k < D - 1; ++k) {
                    const int kk = k < NY + 1 ? k : k + 1;  // every component but rho v
                    pr[k] = f[R::DP + kk] * x[kk];
                }
                RT P = tree_sum<0, D - 1>(pr);
                const RT S = tree_sum<0, NY>(x);
                if (DIR == 0 && q2d) x[NY + 1] = (x[NY + 1] + f[R::AA] * P) * f[R::RQ];
                P += f[R::DP + NY + 1] * x[NY + 1];
#pragma unroll
                for (int dn = 0; dn < 2; ++dn) {
                    const int b0 = dn == 0 ? R::FA : R::FB;
                    const RT fa = f[b0], n1 = f[b0 + 1], n2 = f[b0 + 2], un = f[b0 + 3], nu = f[b0 + 4];
                    // ds/2 folded into the coefficients: o = cv (fa base) + (fa lam) x [+ (fa P) n]
                    const RT fb = fa * (n1 * x[NY] + n2 * x[NY + 1] - un * S);
                    const RT fl = fa * (DIR == 0 ? un + nu : un - nu);
                    const RT fp = fa * P;
                    RT* o = dn == 0 ? outA : outB;
#pragma unroll
                    for (int k = 0; k < NY; ++k) o[k] = f[R::CV + k] * fb + fl * x[k];
                    o[NY] = f[R::CV + NY] * fb + fl * x[NY] + n1 * fp;
                    o[NY + 1] = f[R::CV + NY + 1] * fb + fl * x[NY + 1] + n2 * fp;
                    o[NY + 2] = f[R::CV + NY + 2] * fb + fl * x[NY + 2] + un * fp;
                }
                // results back into the record block (16-byte stores)
#pragma unroll
                for (int k = 0; k < D; ++k) f[R::X + k] = x[k];
#pragma unroll
                for (int g = 0; g < (D + G - 1) / G; ++g)
                    *reinterpret_cast<V*>(gblk + g * 32 * G) = *reinterpret_cast<V*>(&f[g * G]);
                gblk += gstep;
                if (DIR == 1 && nr) {
                    const double dE = double(x[NY + 2]);
                    res = res + dE * dE;
#pragma unroll
                    for (int k = 0; k < NY; ++k) {
                        // smallest q_k/(-Dq_k) over Dq_k < 0
                        const RT dk = x[k];
                        const RT qn = f[R::QS + k], qd = -dk;
                        if constexpr (f32) {
                            if (dk < RT(0)) on = fminf(on, __fdividef(qn, qd));
                        } else {
                            if (dk < RT(0) && qn * od < on * qd) {
                                on = qn;
                                od = qd;
                            }
                        }
                    }
                }
                const int cc = t - 31;
                if (publish && cc >= 0) {
#pragma unroll
                    for (int k = 0; k < D; ++k) xout[(long long)cc * D + k] = outB[k];
                }
                __syncwarp();
            }
            // columns published so far by the top lane
            const int done = t0 + 8 - 31;
            if (publish && done > 0) st_release_gpu(prog_out, done < ni ? done : ni);
        }
        // the copies still in flight (prefetches past the end, or all of them after
        // a wait gave up) land before the ring takes the next strip or the CTA exits
#pragma unroll
        for (int k = 0; k < PFB; ++k) {
            if (!((pend >> k) & 1u)) continue;
            long long spins = 0;
            while (!mbar_try_wait(&bar[k], (phase >> k) & 1u) && ++spins < kSpin3) {
            }
            phase ^= 1u << k;
            pend &= ~(1u << k);
        }
        if (bail) break;
        if (DIR == 1 && nr) {
            for (int o = 16; o > 0; o >>= 1) {
                res += __shfl_xor_sync(0xffffffffu, res, o);
                const RT on2 = __shfl_xor_sync(0xffffffffu, on, o), od2 = __shfl_xor_sync(0xffffffffu, od, o);
                if (on2 * od < on * od2) {  // FP32: od = 1, a plain minimum of the ratios
                    on = on2;
                    od = od2;
                }
            }
            if (lane == 0) {
                const double om = double(on) / double(od) * v.dq_max;  // -q/Dq*Dqmax of the limiting cell
                partials[2 * fs] = res;
                partials[2 * fs + 1] = om;
                if (om < v.omega_min) atomicMax(&v.sc->status, SCFD_E_OMEGA);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// k_unpack: q += omega * Dq from the records (LU-SGS: omega = 1; NR: the
// positivity-limited omega reduced from the per-strip partials in fixed order,
// time_NR_viscous.f90:86-108).
// ---------------------------------------------------------------------------
template <typename T, int NY>
__global__ void __launch_bounds__(1024) k_unpack(View v, const int2* blk, const int4* strips, const long long* rec_off,
                                                 const T* rec, const double* partials, int nstrips, int nr_mode,
                                                 int inner) {
    using R = Rec<NY>;
    using L = RecLayout<T, NY>;
    constexpr int D = R::D, G = L::G, NG = L::NG;
    __shared__ double tile[32][33];
    __shared__ double s_om;
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        double om = 1.0;
        if (nr_mode) {
            double res = 0.0, o = 1e300;
            for (int k = 0; k < nstrips; ++k) {
                res += partials[2 * k];
                o = fmin(o, partials[2 * k + 1]);
            }
            om = fmin(v.omega_max, o);
            if (blockIdx.x == 0) {
                if (inner == 1) v.sc->res1 = res;
                v.sc->res = res;
                v.sc->omega = om;
                log_inner(v.sc, inner, o, res);
            }
        }
        s_om = om;
    }
    __syncthreads();
    if (nr_mode && v.sc->status == SCFD_E_OMEGA) return;
    const double om = s_om;
    const int2 b = blk[blockIdx.x];
    const int4 st = strips[b.x];
    const int p = st.x, s = st.y;
    const int ni = v.P.ni[p], nj = v.P.nj[p];
    const T* in = rec + rec_off[b.x] + (long long)b.y * L::STEP;
    const int nt = min(32, ni + 31 - b.y);
    const long long N = v.ncell;
    // read (step y, lane x) coalesced, write cells (step x, lane y); component
    // k+1's record value and the cell's q are loaded before component k's
    // barriers, so that the loads overlap them
    const bool rd = (int)threadIdx.y < nt;
    const long long rbase = (long long)threadIdx.y * NG * 32 * G + threadIdx.x * G;
    const int tt = threadIdx.x, l = threadIdx.y;
    const int t = b.y + tt, cc = t - l, j = 32 * s + 1 + l;
    const bool wr = tt < nt && cc >= 0 && cc < ni && j <= nj;
    const long long c = wr ? cidx(v.P, p, cc + 1, j) : 0;
    double nxt = rd ? double(in[rbase]) : 0.0;
    double qn = wr ? v.q[c] : 0.0;
    for (int k = 0; k < D; ++k) {
        const double cur = nxt, qk = qn;
        if (k + 1 < D) {
            nxt = rd ? double(in[rbase + (long long)((k + 1) / G) * 32 * G + (k + 1) % G]) : 0.0;
            qn = wr ? v.q[(k + 1) * N + c] : 0.0;
        }
        if (rd) tile[threadIdx.y][threadIdx.x] = cur;
        __syncthreads();
        if (wr) v.q[k * N + c] = nr_mode ? qk + om * tile[tt][l] : qk + tile[tt][l];
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
int sweep3_pad_steps() { return kPad; }

size_t sweep3_record_elems(int ny, bool mixed) {
    switch (ny) {
        case 1: return mixed ? RecLayout<float, 1>::STEP : RecLayout<double, 1>::STEP;
        case 8: return mixed ? RecLayout<float, 8>::STEP : RecLayout<double, 8>::STEP;
        case 9: return mixed ? RecLayout<float, 9>::STEP : RecLayout<double, 9>::STEP;
        default: return 0;
    }
}

template <typename RT, int NY, int DIR>
static void sweep_launch(const View& v, cudaStream_t s, const Sweep3& w) {
    using L = RecLayout<RT, NY>;
    const size_t smem = (size_t)PFB * Spb<RT>::value * L::STEP * sizeof(RT) + 8 * (NY + 3) * sizeof(double) + PFB * 8;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_sweep3<RT, NY, DIR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    StripRec sl{DIR == 0 ? w.tab_f : w.tab_b, w.rec_off, w.nstrips};
    int* prog = w.progress + (DIR == 0 ? 0 : w.nstrips);
    int* tick = w.tickets + (DIR == 0 ? 0 : 1);
    k_sweep3<RT, NY, DIR><<<w.nstrips, 32, smem, s>>>(v, sl, reinterpret_cast<RT*>(w.rec), w.xfer, w.xstride, prog,
                                                      tick, w.partials);
}

template <typename RT, int NY>
static void run_t(const View& v, cudaStream_t s, const Sweep3& w, int what, int inner) {
    const bool nr = v.scheme == SCFD_SCHEME_NR;
    if (what == 0) {
        k_pack<RT, NY><<<w.nblk, dim3(32, 32), 0, s>>>(v, w.blk, w.tab_f, w.rec_off, reinterpret_cast<RT*>(w.rec), nr ? 1 : 0);
    } else if (what == 3) {
        k_unpack<RT, NY><<<w.nblk, dim3(32, 32), 0, s>>>(v, w.blk, w.tab_f, w.rec_off, reinterpret_cast<const RT*>(w.rec),
                                                         w.partials, w.nstrips, nr ? 1 : 0, inner);
    } else if (what == 1) {
        sweep_launch<RT, NY, 0>(v, s, w);
    } else {
        sweep_launch<RT, NY, 1>(v, s, w);
    }
}

// what: 0 pack, 1 forward sweep, 2 backward sweep, 3 unpack/update
int launch_sweep3(const View& v, cudaStream_t s, const Sweep3& w, int what, int inner) {
    const bool mixed = v.precision == SCFD_PREC_MIXED;
    switch (v.nY) {
        case 1: if (mixed) run_t<float, 1>(v, s, w, what, inner); else run_t<double, 1>(v, s, w, what, inner); return 1;
        case 8: if (mixed) run_t<float, 8>(v, s, w, what, inner); else run_t<double, 8>(v, s, w, what, inner); return 1;
        case 9: if (mixed) run_t<float, 9>(v, s, w, what, inner); else run_t<double, 9>(v, s, w, what, inner); return 1;
        default: return 0;
    }
}

}  // namespace scfd
